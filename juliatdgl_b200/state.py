"""The state of a step (host side): every field of ``gtdgl/src/state.jl``'s ``State`` (:13-22).

Ψ_µ on nodes (G this step, F the next), the link phases θ (this step) and φ (the next), the links
V = e^{−iθ} and U = e^{−iφ}, the supercurrent J on links and the field h on plaquettes.  numpy arrays in
Fortran order with the reference's shapes (``Grid.node`` etc.), complex128 for Ψ and the links.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List

import numpy as np

from .grid import Grid, Masks, slab_thickness
from .model import Model, eps_band

LINK_FIELDS = ("θx", "θy", "θz", "φx", "φy", "φz", "Ux", "Uy", "Uz", "Vx", "Vy", "Vz",
               "Jx", "Jy", "Jz", "hx", "hy", "hz")


def emiphi(φ: np.ndarray) -> np.ndarray:
    """cis(−φ) elementwise (state.jl:24)."""
    out = np.empty(φ.shape, dtype=np.complex128, order="F")
    out.real = np.cos(φ)
    out.imag = -np.sin(φ)
    return out


def _fcopy(a, dtype=None):
    return np.array(a, dtype=dtype if dtype is not None else a.dtype, order="F", copy=True)


@dataclass
class State:
    G: List[np.ndarray]
    F: List[np.ndarray]
    θx: np.ndarray
    θy: np.ndarray
    θz: np.ndarray
    φx: np.ndarray
    φy: np.ndarray
    φz: np.ndarray
    Ux: np.ndarray
    Uy: np.ndarray
    Uz: np.ndarray
    Vx: np.ndarray
    Vy: np.ndarray
    Vz: np.ndarray
    Jx: np.ndarray
    Jy: np.ndarray
    Jz: np.ndarray
    hx: np.ndarray
    hy: np.ndarray
    hz: np.ndarray

    @property
    def N(self) -> int:
        return len(self.G)

    @staticmethod
    def from_fields(gr: Grid, G, θ, θprev, h) -> "State":
        """state.jl:31-46: V = e^{−iθ}, U = e^{−iθprev}, J = 0, F = copy of G."""
        θx, θy, θz = (_fcopy(a, np.float64) for a in θ)
        φx, φy, φz = (_fcopy(a, np.float64) for a in θprev)
        G = [_fcopy(g, np.complex128) for g in G]
        return State(G, [g.copy(order="F") for g in G], θx, θy, θz, φx, φy, φz,
                     emiphi(φx), emiphi(φy), emiphi(φz), emiphi(θx), emiphi(θy), emiphi(θz),
                     np.zeros(gr.xlink, order="F"), np.zeros(gr.ylink, order="F"), np.zeros(gr.zlink, order="F"),
                     _fcopy(h[0], np.float64), _fcopy(h[1], np.float64), _fcopy(h[2], np.float64))

    def copy(self) -> "State":
        return State([g.copy(order="F") for g in self.G], [f.copy(order="F") for f in self.F],
                     *(getattr(self, k).copy(order="F") for k in LINK_FIELDS))

    def fields(self):
        """(name, array) of every field, bands first."""
        out = [(f"G{µ + 1}", g) for µ, g in enumerate(self.G)] + [(f"F{µ + 1}", f) for µ, f in enumerate(self.F)]
        return out + [(k, getattr(self, k)) for k in LINK_FIELDS]


def initial_state(md: Model, gr: Grid, mk: Masks, H: float, materials=None) -> State:
    """Meissner seed (state.jl:48-63): Ψ_µ = τψ √(ε_µ/β_µ), A = 0, h_z = H on the z faces; with `materials` (every
    model, the first is md) and a material map, each node at the uncoupled equilibrium of its own material."""
    G = []
    for µ in range(md.N):
        v = math.sqrt(max(eps_band(md, µ + 1), 0.0) / md.bands[µ].β)
        G.append(np.asarray(mk.τψ * v, dtype=np.complex128, order="F"))
    if materials is not None and mk.mat is not None:
        for µ in range(md.N):
            vm = np.array([math.sqrt(max(eps_band(m, µ + 1), 0.0) / m.bands[µ].β) for m in materials])
            G[µ] = np.asarray(mk.τψ * vm[mk.mat.astype(np.int64) - 1], dtype=np.complex128, order="F")
    θ = (np.zeros(gr.xlink, order="F"), np.zeros(gr.ylink, order="F"), np.zeros(gr.zlink, order="F"))
    hx = np.zeros(gr.hx_shape, order="F")
    hy = np.zeros(gr.hy_shape, order="F")
    hz = np.zeros(gr.hz_shape, order="F")
    hz[:, :, 0] = H
    hz[:, :, gr.Nz] = H
    return State.from_fields(gr, G, θ, θ, (hx, hy, hz))


def seeded_state(md: Model, gr: Grid, mk: Masks, H: float, *, seed: int = 0, amp: float = 1e-3,
                 base: float | None = None) -> State:
    """A perturbed start: Ψ_µ = τψ·(b_µ + amp·(n₁ + i n₂)) from numpy's seeded normal generator, A = 0.

    ``base`` is b_µ for every band (1 by default: the unit-amplitude start of the two-band parity case);
    with ``base=None`` and a model, b_µ = √(ε_µ/β_µ) as in ``initial_state``."""
    rng = np.random.default_rng(seed)
    s = initial_state(md, gr, mk, H)
    for µ in range(md.N):
        b = 1.0 if base is None else base
        n = rng.standard_normal(gr.node + (2,))
        g = mk.τψ * (b + amp * (n[..., 0] + 1j * n[..., 1]))
        s.G[µ][...] = g
        s.F[µ][...] = g
    return s
