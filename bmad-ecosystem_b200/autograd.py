"""torch.autograd.Function over the library's adjoint kernel (bmadgpu_loss_grad): the tracking
loss as a differentiable function of element strengths, for optimisers.

    strengths = torch.tensor([...], dtype=torch.float64, requires_grad=True)
    loss = TrackingLoss.apply(strengths, problem)
    loss.backward()              # strengths.grad = d(loss)/d(strengths)

``problem`` is a StrengthProblem: the ring's element records, which elements the strengths
belong to (quadrupole k1, sextupole k2, octupole k3), the bunch, turns and checkpoint interval.
The forward pass rebuilds the lattice with the given strengths and runs the adjoint kernel once;
the gradient is kept for the backward pass. The reference has no counterpart (Tao differentiates
by one-sided finite differences, tao/code/tao_dmerit_mod.f90:162-180)."""
import ctypes as C

import numpy as np
import torch

from . import abi, lib

_ATTR = {abi.QUADRUPOLE: "k1", abi.SEXTUPOLE: "k2", abi.OCTUPOLE: "k3"}


class StrengthProblem:
    def __init__(self, ctx, elements, param, param_ele, bunch, n_turns, checkpoint_every=16):
        self.ctx = ctx
        self.elements = abi.element_array(elements) if not isinstance(elements, C.Array) else elements
        self.param = param
        self.param_ele = [int(i) for i in param_ele]
        self.attrs = [_ATTR[self.elements[i].key] for i in self.param_ele]
        self.bunch = bunch
        self.n_turns = n_turns
        self.checkpoint_every = checkpoint_every

    def strengths(self):
        return np.array([getattr(self.elements[i], a) for i, a in zip(self.param_ele, self.attrs)])

    def evaluate(self, values):
        """(loss, gradient) at the given strengths."""
        for i, a, v in zip(self.param_ele, self.attrs, values):
            setattr(self.elements[i], a, float(v))
        lat = lib.Lattice(self.ctx, self.elements, self.param)
        try:
            return lib.loss_grad(self.ctx, lat, self.bunch, self.n_turns, self.param_ele, self.checkpoint_every)
        finally:
            lat.close()


class TrackingLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, strengths, problem):
        values = strengths.detach().cpu().numpy().astype(np.float64)
        loss, grad = problem.evaluate(values)
        ctx.save_for_backward(torch.from_numpy(grad).to(strengths.device))
        return torch.tensor(loss, dtype=torch.float64, device=strengths.device)

    @staticmethod
    def backward(ctx, grad_out):
        (grad,) = ctx.saved_tensors
        return grad_out * grad, None
