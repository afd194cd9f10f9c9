"""Generates adjoint_config4_fd.json: central finite differences of the oracle's loss on the
differentiation workload (50-cell ring, 4,096 matched Gaussian particles from seed 2, 256
turns, loss = mean over particles of x^2 + y^2), for 12 quadrupole k1 and 12 sextupole k2 values.
The GPU test compares the adjoint kernel's gradient with these at full size (all 200 components
are compared there with finite differences of the GPU's own forward tracking).

Stencil: fourth-order central differences, [8 (L(+h) - L(-h)) - (L(+2h) - L(-2h))] / (12 h k),
at h = 1e-5 relative for quadrupoles and 2e-3 for sextupoles: over 256 turns a 1e-5 change of a
quadrupole moves the phase by ~4e-3 rad, so a second-order difference would carry ~3e-6
truncation error, while steps much below 1e-5 drown in the tracking's rounding (the coordinates
after 256 turns move by ~1e-11 relative between neighbouring strengths). Quadrupoles are also
differenced at the second-order h = 1e-7 for the record. Run from the repository root:
    python tests/golden/make_adjoint_fd.py
"""
import importlib
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from helpers import oracle_track  # noqa: E402

abi = importlib.import_module("bmad-ecosystem_b200.abi")
rings = importlib.import_module("bmad-ecosystem_b200.rings")

N_CELLS, N_PART, SEED, N_TURNS = 50, 4096, 2, 256
# 12 quadrupoles and 12 sextupoles spread over the ring (slots alternate quadrupole, sextupole,
# quadrupole, sextupole in each cell), the ring's first and last of each among them
QUAD_SLOTS = [0, 18, 34, 52, 68, 86, 102, 118, 136, 152, 170, 198]
SEXT_SLOTS = [1, 19, 35, 53, 69, 87, 103, 119, 137, 153, 171, 199]


def loss_of(elements, p, vec):
    o = oracle_track(elements, p, vec, N_TURNS)
    alive = o["state"] == abi.ALIVE
    return float(np.sum(o["vec"][0, alive] ** 2 + o["vec"][2, alive] ** 2) / vec.shape[1]), int(alive.sum())


def main():
    eles, p = rings.ring(N_CELLS)
    vec = rings.matched_gaussian(eles, N_PART, seed=SEED)
    strength = {abi.QUADRUPOLE: "k1", abi.SEXTUPOLE: "k2"}
    param_ele = [i for i, e in enumerate(eles) if e.key in strength]
    t0 = time.time()
    loss0, alive = loss_of(eles, p, vec)
    out = dict(n_cells=N_CELLS, n_particles=N_PART, seed=SEED, n_turns=N_TURNS, loss=loss0, alive=alive,
               param_ele=param_ele, entries=[])
    plan = [(s, 1e-5, 4) for s in QUAD_SLOTS] + [(s, 2e-3, 4) for s in SEXT_SLOTS] + \
           [(s, 1e-7, 2) for s in QUAD_SLOTS[:2]]
    for slot, h, order in plan:
        i = param_ele[slot]
        key = strength[eles[i].key]
        k0 = getattr(eles[i], key)

        def L(d):
            e2 = abi.element_array(eles)
            setattr(e2[i], key, k0 * (1 + d))
            return loss_of(e2, p, vec)[0]
        if order == 4:
            fd = (8 * (L(h) - L(-h)) - (L(2 * h) - L(-2 * h))) / (12 * h * k0)
        else:
            fd = (L(h) - L(-h)) / (2 * h * k0)
        out["entries"].append(dict(slot=slot, element=i, attr=key, h=h, order=order, fd=fd))
        print("slot %d element %d %s h=%g order %d fd=%.12e (%.0fs)" % (slot, i, key, h, order, fd, time.time() - t0),
              flush=True)
    with open(os.path.join(HERE, "adjoint_config4_fd.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
