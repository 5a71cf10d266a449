"""Direct (non-mesh) Ewald reciprocal sum in FP64 with torch on the GPU: the truth for
the PME error at sizes where the oracle's CPU sum would take minutes.  TEST
INFRASTRUCTURE ONLY (a checker used by tests/ and bench.py's error report; the
product never imports it).

E = CC / (2 pi V) sum_{m != 0} g(m) |S(m)|^2,  g(m) = exp(-pi^2 |m|^2 / beta^2) / |m|^2,
S(m) = sum_j q_j exp(2 pi i m . r_j), m = (mx / Lx, my / Ly, mz / Lz), and the force on
atom i  F_i = -(2 CC q_i / V) sum_{m != 0} g(m) m Im(S(m) exp(-2 pi i m . r_i)).
S(m) is a complex matrix product: per-atom tables e^{2 pi i k x / L} for |k| <= kmax,
W[(mx, my), j] = q_j ex[j, mx] ey[j, my], S[(mx, my), mz] = W @ ez.  Only half of the
sphere (mx >= 0, the rest by S(-m) = conj S(m)) is summed, weighted 2 where mx > 0.
"""
import math

import numpy as np

CC = 332.0716


def recip_forces(pos, q, box, beta, atoms, kmax, device="cuda", chunk_mx=4):
    """Reciprocal-space forces on `atoms` (indices) and the reciprocal energy."""
    import torch
    dt = torch.float64
    L = [float(b) for b in box]
    V = L[0] * L[1] * L[2]
    r = torch.as_tensor(np.asarray(pos, np.float64), dtype=dt, device=device)
    qq = torch.as_tensor(np.asarray(q, np.float64), dtype=dt, device=device)
    k = torch.arange(-kmax, kmax + 1, dtype=dt, device=device)
    tab = [torch.polar(torch.ones(len(q), 2 * kmax + 1, dtype=dt, device=device),
                       2 * math.pi * r[:, d:d + 1] * k[None, :] / L[d]) for d in range(3)]
    ex, ey, ez = tab
    mmax2 = (kmax / min(L)) ** 2
    fy = k / L[1]
    fz = k / L[2]
    sel = torch.as_tensor(np.asarray(atoms), device=device)
    F = torch.zeros(len(atoms), 3, dtype=dt, device=device)
    E = torch.zeros((), dtype=dt, device=device)
    qi = qq[sel]
    for mx0 in range(0, kmax + 1, chunk_mx):
        mxs = torch.arange(mx0, min(kmax + 1, mx0 + chunk_mx), device=device)
        # W[(mx, my), j] = q_j ex[j, mx] ey[j, my]
        W = (qq[None, None, :] * ex[:, kmax + mxs].T[:, None, :] * ey.T[None, :, :]).reshape(-1, len(q))
        S = (W @ ez).reshape(len(mxs), 2 * kmax + 1, 2 * kmax + 1)  # [mx, my, mz]
        fx = mxs.to(dt) / L[0]
        m2 = fx[:, None, None] ** 2 + fy[None, :, None] ** 2 + fz[None, None, :] ** 2
        wt = torch.where(mxs == 0, 1.0, 2.0).to(dt)[:, None, None].expand_as(m2).clone()
        # half space at mx = 0: my > 0, or my = 0 and mz > 0 (weight 2 for the pair +-m)
        if mx0 == 0:
            myi = torch.arange(-kmax, kmax + 1, device=device)
            half = (myi[:, None] > 0) | ((myi[:, None] == 0) & (myi[None, :] > 0))
            wt[0] = torch.where(half, 2.0, 0.0).to(dt)
        ok = (m2 <= mmax2) & (m2 > 0)
        g = torch.where(ok, torch.exp(-math.pi ** 2 * m2 / beta ** 2) / torch.where(ok, m2, 1.0), 0.0) * wt
        E = E + (g * S.abs() ** 2).sum()
        # forces on the selected atoms: Im(S(m) conj(e_i(m)))
        ei = (ex[sel][:, kmax + mxs][:, :, None, None] * ey[sel][:, None, :, None] * ez[sel][:, None, None, :])
        im = (S[None] * ei.conj()).imag * g[None]
        F[:, 0] += (im * fx[None, :, None, None]).sum((1, 2, 3))
        F[:, 1] += (im * fy[None, None, :, None]).sum((1, 2, 3))
        F[:, 2] += (im * fz[None, None, None, :]).sum((1, 2, 3))
    F = -(2.0 * CC / V) * qi[:, None] * F
    E = CC / (2.0 * math.pi * V) * E
    return F.cpu().numpy(), float(E)


def kmax_for(box, beta, tol=1e-12):
    """Smallest kmax whose sphere keeps every term with exp(-pi^2 m^2 / beta^2) > tol."""
    mcut = beta * math.sqrt(-math.log(tol)) / math.pi
    return int(math.ceil(mcut * min(box)))
