"""Bands and models of the N-band TDGL functional (host side).

Restates ``gtdgl/src/model.jl``: ``Band`` (model.jl:26-48), ``Model`` (:64-88) with its validation (symmetric
Josephson matrix with a zero diagonal, model.jl:84-87), ``two_band`` (:101-109) and ``equilibrium`` (:119-141).
Every scalar expression keeps the reference's order of operations, so that the step and the coefficients
derived from these values are the reference's to the bit.
"""
from __future__ import annotations

import math

import numpy as np
from dataclasses import dataclass
from typing import Sequence, Tuple

U_DIRTY = math.pi ** 4 / (14 * 1.2020569031595942)


@dataclass(frozen=True)
class Band:
    """One band (model.jl:26-33): mass ratio m (stiffness 1/m), Γ, a, β, the KWT factor γ̃ and the masses per axis."""
    m: float = 1.0
    Γ: float = 1.0
    a: float = 1.0
    β: float = 1.0
    γkwt: float = 0.0
    ma: Tuple[float, float, float] = None

    def __post_init__(self):
        if self.ma is None:
            object.__setattr__(self, "ma", (self.m, self.m, self.m))

    @staticmethod
    def make(m=1.0, g=None, Γ=1.0, a=1.0, β=1.0, γkwt=0.0, m_axes=None):
        """The keyword constructor of model.jl:37-46 (``g`` gives the stiffness instead of m)."""
        mm = float(m) if g is None else 1 / float(g)
        ma = (mm, mm, mm) if m_axes is None else tuple(float(x) for x in m_axes)
        if len(ma) != 3:
            raise ValueError("Band: m_axes is (m_x, m_y, m_z)")
        if m_axes is not None:
            mm = ma[0]
        if not (mm > 0 and all(x > 0 for x in ma) and Γ > 0 and β > 0):
            raise ValueError("Band: m (or g, m_axes), Γ and β must be positive")
        if γkwt < 0:
            raise ValueError("Band: γkwt must be >= 0")
        return Band(mm, float(Γ), float(a), float(β), float(γkwt), ma)


def stiffness(b: Band, i: int | None = None) -> float:
    """1/m, or 1/m_i along axis i (1, 2, 3) (model.jl:50-52)."""
    return 1 / b.m if i is None else 1 / b.ma[i - 1]


def isotropic(b: Band) -> bool:
    return b.ma[0] == b.ma[1] == b.ma[2] == b.m


def sigma_dirty(bands) -> float:
    s = 0.0
    for k, b in enumerate(bands):
        v = stiffness(b) * b.Γ / b.β
        s = v if k == 0 else s + v
    return s / U_DIRTY


@dataclass(frozen=True)
class Model:
    """N bands, the interband Josephson matrix γ, κ, σn and the bath temperature T (model.jl:64-70)."""
    bands: Tuple[Band, ...]
    γ: Tuple[Tuple[float, ...], ...]
    κ: float
    σn: float = 1.0
    T: float = 0.0

    @staticmethod
    def make(bands: Sequence[Band], γ, κ, σn=1.0, T=0.0):
        """model.jl:72-88: validates the coupling (real, symmetric, zero diagonal) and κ, σn > 0."""
        bands = tuple(bands)
        N = len(bands)
        if isinstance(σn, str):
            if σn != "dirty":
                raise ValueError("Model: σn is a number or :dirty")
            σn = sigma_dirty(bands)
        g = [[float(γ[m][n]) for n in range(N)] for m in range(N)]
        if len(γ) != N or any(len(r) != N for r in γ):
            raise ValueError(f"Model: γ must be {N}×{N}")
        for m in range(N):
            for n in range(N):
                if g[m][n] != g[n][m]:
                    raise ValueError("Model: γ must be symmetric")
                if m == n and g[m][m] != 0:
                    raise ValueError("Model: the diagonal of γ must be zero")
        if not (κ > 0 and σn > 0):
            raise ValueError("Model: κ and σn must be positive")
        return Model(bands, tuple(tuple(r) for r in g), float(κ), float(σn), float(T))

    @property
    def N(self) -> int:
        return len(self.bands)


def nbands(md: Model) -> int:
    return md.N


def eps_band(md: Model, µ: int) -> float:
    """ε_µ = a_µ − T (model.jl:93); µ is 1-based as in the reference."""
    return md.bands[µ - 1].a - md.T


def two_band(*, xi_ratio, a2n=0.59, gamma12=1e-3, gamma_ratio=1.0, κ, σn=1.0, T=0.0, beta2=1.0, gamma_kwt=0.0):
    """The two-band model of release 1.x (model.jl:101-109)."""
    mr = 1 / ((xi_ratio * xi_ratio) * (a2n / beta2))
    gk = (gamma_kwt, gamma_kwt) if not isinstance(gamma_kwt, tuple) else gamma_kwt
    return Model.make((Band.make(γkwt=gk[0]), Band.make(m=mr, Γ=gamma_ratio, a=a2n, β=beta2, γkwt=gk[1])),
                      [[0.0, gamma12], [gamma12, 0.0]], κ=κ, σn=σn, T=T)


def equilibrium(md: Model):
    """Amplitudes of the coupled homogeneous equilibrium (model.jl:119-141): Gauss–Seidel over the bands,
    Newton from above on each cubic."""
    b = md.bands
    N = md.N
    p = [math.sqrt(max(eps_band(md, µ + 1), 0.0) / b[µ].β) for µ in range(N)]
    for _ in range(100_000):
        dmax = 0.0
        for µ in range(N):
            ε = eps_band(md, µ + 1)
            β = b[µ].β
            c = 0.0
            for ν in range(N):
                term = 0.0 if ν == µ else abs(md.γ[µ][ν]) * p[ν]
                c = term if ν == 0 else c + term
            x = math.sqrt(max(ε, 0.0) / β) + float(np.cbrt(c / β))
            for _ in range(200):
                f = β * (x * x * x) - ε * x - c
                df = 3 * β * (x * x) - ε
                if f <= 0 or df <= 0:
                    break
                dx = f / df
                x -= dx
                if dx <= 1e-15 * x:
                    break
            dmax = max(dmax, abs(x - p[µ]))
            p[µ] = x
        if dmax < 1e-14:
            break
    return tuple(p)
