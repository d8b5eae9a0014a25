"""Extra test surfaces: a torus on tensor Chebyshev nodes (iptype 12) and a
surface whose patches mix types and orders."""
import numpy as np

from fmm3dbie_b200 import surface as S


def torus_cheb(nu=12, nv=6, norder=5, R=2.0, r0=0.6, r1=0.15, m=3):
    """x = (R + r(p) cos t) cos p, (R + r(p) cos t) sin p, r(p) sin t with
    r(p) = r0 + r1 cos(m p), nu x nv quad patches on tensor Chebyshev nodes."""
    uvs, _, _, _ = S.disc_exps(12, norder)
    uvs = np.asarray(uvs).reshape(-1, 2)
    rows = []
    dp, dt = 2 * np.pi / nu, 2 * np.pi / nv
    for i in range(nu):
        for j in range(nv):
            p = i * dp + (uvs[:, 0] + 1) * 0.5 * dp
            t = j * dt + (uvs[:, 1] + 1) * 0.5 * dt
            r = r0 + r1 * np.cos(m * p)
            rp = -r1 * m * np.sin(m * p)
            rho = R + r * np.cos(t)
            x = np.stack([rho * np.cos(p), rho * np.sin(p), r * np.sin(t)], 1)
            xp = np.stack([rp * np.cos(t) * np.cos(p) - rho * np.sin(p),
                           rp * np.cos(t) * np.sin(p) + rho * np.cos(p), rp * np.sin(t)], 1)
            xt = np.stack([-r * np.sin(t) * np.cos(p), -r * np.sin(t) * np.sin(p), r * np.cos(t)], 1)
            du, dv = xp * 0.5 * dp, xt * 0.5 * dt
            n = np.cross(du, dv)
            n /= np.linalg.norm(n, axis=1)[:, None]
            rows.append(np.concatenate([x, du, dv, n], 1))
    npat = nu * nv
    return S.from_srcvals(np.full(npat, norder), np.full(npat, 12), np.concatenate(rows, 0))


def concat(*surfs, shifts=None):
    """One surface made of the patches of several (each shifted by a vector)."""
    shifts = shifts or [(0.0, 0.0, 0.0)] * len(surfs)
    sv, no, ip = [], [], []
    for s, d in zip(surfs, shifts):
        v = s.srcvals.copy()
        v[:, :3] += np.asarray(d)
        sv.append(v)
        no.append(s.norders)
        ip.append(s.iptype)
    return S.from_srcvals(np.concatenate(no), np.concatenate(ip), np.concatenate(sv, 0))
