"""Generate tests/golden/sphere_spectra.json: analytic eigenvalues of the
single- and double-layer operators on the unit sphere for the spherical
harmonic Y_n^m (the reference's known-answer tests,
matlab/test/lap3d_dirichlet_routsTest.m:9-34 and
matlab/test/helm3d_dirichlet_routsTest.m:10-35), from scipy's spherical
Bessel functions:

  S_0 Y_n = Y_n / (2n+1)                 D_0 Y_n (principal value) = -Y_n / (2(2n+1))
  S_k Y_n = i k j_n(k) h_n(k) Y_n        D_k Y_n (principal value) = (i k^2 j_n'(k) h_n(k) - 1/2) Y_n

with h_n = j_n + i y_n (outgoing), kernels e^{ikr}/(4 pi r) and
n_y.(x-y)(1-ikr)e^{ikr}/(4 pi r^3).

    python tests/golden/make_golden.py
"""
import json
import os

from scipy.special import spherical_jn, spherical_yn

out = {"laplace": {}, "helmholtz": {}}
for n in range(0, 6):
    out["laplace"][str(n)] = {"S": 1.0 / (2 * n + 1), "D": -1.0 / (2 * (2 * n + 1))}
for k in (1.1, 2.0, 5.0):
    for n in range(0, 6):
        j = spherical_jn(n, k)
        jp = spherical_jn(n, k, derivative=True)
        h = j + 1j * spherical_yn(n, k)
        s = 1j * k * j * h
        d = 1j * k * k * jp * h - 0.5
        out["helmholtz"][f"{k}:{n}"] = {"S": [s.real, s.imag], "D": [d.real, d.imag]}
path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sphere_spectra.json")
with open(path, "w") as f:
    json.dump(out, f, indent=1, sort_keys=True)
print(path)
