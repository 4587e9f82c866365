"""The synthetic ladder workloads the benchmark times and the parity tests check, built with the host mirror.

``ramp`` is one ladder run of a three-band KWT sample: by default 256×128×32 cells at h = 0.5ξ with an 8-cell
insulating padding (σvac = 0.01 selects the PCG field solve; FP32 separable preconditioner, tolerance 1e-10), a
WEDGE notch 40 cells deep on the y1 face (wedge_depth = 40/128), the open-boundary FFT self-field recomputed every
1 t_GL, κ = 25, H = 0.03, and the transport current ramped as Jx = ±0.06·step/20000 (HJ updated every step).  Model:
the σ and π bands of gtdgl's mgb2_model_II (ξπ/ξσ = 4) and a third, heavier band, KWT γ̃ = 10 on all three,
off-diagonal Josephson couplings drawn from U[−0.1, 0] with seed 1.  Synthetic state: the model's Meissner seed.
The same scheme on a smaller grid (nx, ny, nz, buf) is the bounded sample the parity tests and the CPU baseline use.
"""
from __future__ import annotations

import numpy as np

from .grid import GeomSpec, Grid, build_masks
from .model import Band, Model
from .scheme import Stepper, selffield
from .state import initial_state

RAMP_H = 0.03
RAMP_JMAX = 0.06
RAMP_STEPS = 20000


def ramp_model() -> Model:
    rng = np.random.default_rng(1)
    g = -0.1 * rng.random(3)           # off-diagonal Josephson couplings ~ U[-0.1, 0], seed 1
    γ = [[0.0, g[0], g[1]], [g[0], 0.0, g[2]], [g[1], g[2], 0.0]]
    bands = (Band.make(m=1.0, Γ=1.0, a=1.0, γkwt=10.0),                 # σ of mgb2_model_II, KWT 10
             Band.make(m=1 / (16 * 0.59), Γ=1.0, a=0.59, γkwt=10.0),    # π (ξπ/ξσ = 4), KWT 10
             Band.make(m=2.0, Γ=1.2, a=0.8, γkwt=10.0))                 # a third, heavier band, KWT 10
    return Model.make(bands, γ, κ=25.0)


def ramp(nx=256, ny=128, nz=32, buf=8, open_bc=True, bar_tables=None, bar_backend="auto"):
    """(Stepper, State, H) of the ramp workload on an nx×ny×nz grid with a buf-cell insulating padding."""
    md = ramp_model()
    gr = Grid.make(nx, ny, nz, dx=0.5, buf=buf)
    mk = build_masks(GeomSpec(GEOM_MODE="WEDGE", wedge_depth=40 / 128), gr)
    st = Stepper.make(md, gr, mk, σvac=0.01, pcg_tol=1e-10, pcg_fast=True, pcg_f32=True,
                      selffield_bc="open" if open_bc else "bar", open_every=1.0, bar_tables=bar_tables,
                      bar_backend=bar_backend)
    return st, initial_state(md, gr, mk, RAMP_H), RAMP_H


def ramp_hj(st: Stepper, polarity: int = 1):
    """HJ of step q of the current ramp Jx = ±0.06·q/20000."""
    return lambda q: selffield(st, polarity * RAMP_JMAX * q / RAMP_STEPS)
