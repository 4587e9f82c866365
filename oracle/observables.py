"""Test infrastructure: the oracle of the cycle observables, a numpy restatement of gtdgl's measurement functions on a
host State (only tests may import this module).

Each function follows the cited reference lines, with its loop order and its sequential sums (`sumlin`,
observables.jl:8-14), and works on the State arrays as the reference does (1-based indices in the docstrings,
0-based slices in the code).
"""
from __future__ import annotations

import math

import numpy as np

TWO_PI = 2 * math.pi


def sumlin(values) -> float:
    s = 0.0
    for x in values:
        s += float(x)
    return s


def path_phase(G, Vx, gr, vi, vo):
    """_path_phase! (protocol.jl:168-179): per line (j, k) over y1..y2+1 × z1..z2+1, Σ_{vi ≤ i < vo}
    angle((conj(G[i]) Vx[i]) G[i+1])."""
    ys, zs = range(gr.y1, gr.y2 + 2), range(gr.z1, gr.z2 + 2)
    D = np.zeros((len(ys), len(zs)), order="F")
    for kk, k in enumerate(zs):
        for jj, j in enumerate(ys):
            acc = 0.0
            for i in range(vi, vo):
                w = (np.conj(G[i - 1, j - 1, k - 1]) * Vx[i - 1, j - 1, k - 1]) * G[i, j - 1, k - 1]
                acc += math.atan2(w.imag, w.real)
            D[jj, kk] = acc
    return D


def plane_sum(phx, gr, plane, M):
    """_plane_sum (protocol.jl:148-155): Σ over (j, k) with M of φx[plane, j, k], k outer, j inner."""
    tot = 0.0
    for kk, k in enumerate(range(gr.z1, gr.z2 + 2)):
        for jj, j in enumerate(range(gr.y1, gr.y2 + 2)):
            if M[jj, kk]:
                tot += phx[plane - 1, j - 1, k - 1]
    return tot


def theta_A_sum(phx, gr, vi, vo, line_ok):
    """_theta_A (protocol.jl:157-166) before its division: Σ over line_ok lines of Σ_{vi ≤ i < vo} φx."""
    tot = 0.0
    for kk, k in enumerate(range(gr.z1, gr.z2 + 2)):
        for jj, j in enumerate(range(gr.y1, gr.y2 + 2)):
            if not line_ok[jj, kk]:
                continue
            for i in range(vi, vo):
                tot += phx[i - 1, j - 1, k - 1]
    return tot


def block_abs(X, gr):
    """|X| on the block x1..x2+1 × y1..y2+1 × z1..z2+1 (protocol.jl:360, :433-436)."""
    return np.abs(X[gr.x1 - 1:gr.x2 + 1, gr.y1 - 1:gr.y2 + 1, gr.z1 - 1:gr.z2 + 1])


def nanmax(a) -> float:
    """Julia's max over an array: NaN wins."""
    a = np.asarray(a, dtype=float)
    return float("nan") if np.isnan(a).any() else float(a.max())


def cooper_residual(F, cooper0, gr):
    """protocol.jl:432-440 for one band: max over the block of | |F| − Cooper0 |, and |F| (the next Cooper0)."""
    a = block_abs(F, gr)
    return nanmax(np.abs(a - cooper0)), a


def midplane_current(hy, hz, gr, kappa2):
    """midplane_current (observables.jl:102-114): (Itot·dy·dz, Isam·dy·dz) through the plane ii = oround(Nx/2)."""
    ii = int(math.floor(abs(gr.Nx / 2) + 0.5))
    itot = isam = 0.0
    for kk in range(2, gr.Nz + 1):
        for jj in range(2, gr.Ny + 1):
            jx = kappa2 * ((hz[ii - 1, jj - 1, kk - 1] - hz[ii - 1, jj - 2, kk - 1]) / gr.dy -
                           (hy[ii - 1, jj - 1, kk - 1] - hy[ii - 1, jj - 1, kk - 2]) / gr.dz)
            itot += jx
            if gr.y1 <= jj <= gr.y2 + 1 and gr.z1 <= kk <= gr.z2 + 1:
                isam += jx
    return itot * gr.dy * gr.dz, isam * gr.dy * gr.dz


def oround(x: float) -> int:
    a = math.floor(abs(x) + 0.5)
    return int(a if x >= 0 else -a)


def count_vortices(psi, Vx, Vy, hz, f, gr, kc):
    """count_vortices (observables.jl:48-74): (Nv, nmap, Nv_loop, loop_ok) on the plane z = kc."""
    x1, x2, y1, y2 = gr.x1, gr.x2, gr.y1, gr.y2
    P = psi[x1 - 1:x2 + 1, y1 - 1:y2 + 1, kc - 1]
    Ux = Vx[x1 - 1:x2, y1 - 1:y2 + 1, kc - 1]
    Uy = Vy[x1 - 1:x2 + 1, y1 - 1:y2, kc - 1]
    nx, ny = P.shape
    ang = lambda w: math.atan2(w.imag, w.real)
    Dx = np.array([[ang((np.conj(P[i, j]) * Ux[i, j]) * P[i + 1, j]) for j in range(ny)] for i in range(nx - 1)])
    Dy = np.array([[ang((np.conj(P[i, j]) * Uy[i, j]) * P[i, j + 1]) for j in range(ny - 1)] for i in range(nx)])
    Fm = f[x1 - 1:x2 + 1, y1 - 1:y2 + 1, kc - 1]
    mat = (Fm > 1e-6) & (np.abs(P) > 1e-12)
    nmap = np.zeros((nx - 1, ny - 1), dtype=np.int32)
    for j in range(ny - 1):
        for i in range(nx - 1):
            circ = Dx[i, j] + Dy[i + 1, j] - Dx[i, j + 1] - Dy[i, j]
            phi = hz[x1 - 2 + i + 1, y1 - 2 + j + 1, kc - 1] * gr.dx * gr.dy
            good = mat[i, j] and mat[i + 1, j] and mat[i, j + 1] and mat[i + 1, j + 1]
            w = (circ + phi) / TWO_PI
            nmap[i, j] = oround(w) if good and math.isfinite(w) else 0
    Nv = int(nmap.sum())
    loop = sumlin(Dx[:, 0]) + sumlin(Dy[-1, :]) - sumlin(Dx[:, -1]) - sumlin(Dy[0, :])
    phi_enc = sumlin(hz[x1 - 1:x2, y1 - 1:y2, kc - 1].ravel(order="F")) * gr.dx * gr.dy
    wl = (loop + phi_enc) / TWO_PI
    Nv_loop = oround(wl) if math.isfinite(wl) else 0
    per = np.concatenate([mat[:, 0], mat[-1, :], mat[:, -1], mat[0, :]])
    return Nv, nmap, Nv_loop, bool(per.all())
