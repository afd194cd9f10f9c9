"""Extracts the NAFF known-answer test of the reference's sim_utils regression test into
naff_kat.json: the three-tone input of regression_tests/sim_utils_test/sim_utils_test.f90 (its
amp1..3 and sig1..3 assignments, 32 samples) and the expected freq / amplitude lines of
regression_tests/sim_utils_test/output.correct ("naff-freq1..3", with their REL tolerances).
The 32 samples are built as the Fortran statements build them: sig1..3 are default-real (single
precision) literals stored in real(rp); cmplx() without a KIND gives a default (single precision)
complex, so the exponentials, the products with the single-precision amplitudes and their sum
are single precision, promoted to double on assignment to cdata. The samples go into the fixture.
Run from the repository root with the reference checked out at REF (default /root/reference)."""
import json
import os
import re
import sys

import numpy as np

REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
d = os.path.join(REF, "regression_tests", "sim_utils_test")
src = open(os.path.join(d, "sim_utils_test.f90")).read()
seg = src[src.index("! naff test"):src.index("call naff")]
amps = {int(k): [float(a), float(b)] for k, a, b in re.findall(r"amp(\d)\s*=\s*cmplx\(\s*([-\d.eE+]+)\s*,\s*([-\d.eE+]+)\s*\)", seg)}
sigs = {int(k): float(v) for k, v in re.findall(r"sig(\d)\s*=\s*([-\d.eE+]+)", seg)}
n = int(re.search(r"complex\(rp\) cdata\((\d+)\)", src).group(1))
want = []
for line in open(os.path.join(d, "output.correct")):
    m = re.match(r'"naff-freq(\d)"\s+REL\s+([-\d.eE+]+)\s+(.*)', line)
    if m:
        f, re_, im = (float(x) for x in m.group(3).split())
        want.append(dict(k=int(m.group(1)), rel=float(m.group(2)), freq=f, amp=[re_, im]))
cdata = []
for i in range(1, n + 1):
    tot = np.complex64(0)
    for k in sorted(amps):
        sig = float(np.float32(sigs[k]))
        phi = 2 * np.pi * (sig * (i - 1))
        e = np.exp(np.complex64(complex(0.0, -phi)))
        a = np.complex64(complex(np.float32(amps[k][0]), np.float32(amps[k][1])))
        tot = np.complex64(tot + np.complex64(a * e))
    cdata.append([float(tot.real), float(tot.imag)])
out = dict(source="regression_tests/sim_utils_test/sim_utils_test.f90:280-299 and output.correct",
           n_samples=n, cdata=cdata, tones=[dict(amp=amps[k], sig=sigs[k]) for k in sorted(amps)], expected=want)
json.dump(out, open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "naff_kat.json"), "w"), indent=1)
print(out)
