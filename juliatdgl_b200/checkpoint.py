"""Checkpoints of a run on the device: the state, the solver carry and the noise stream index in one file, so that a
stopped run resumes in a new context (another process, another GPU) where it stopped.

The file is a numpy ``.npz`` archive written atomically (a temporary file, then a rename), with the key names of
gtdgl's checkpoints: ``nbands``, ``G1``…``GN``, ``thetax/y/z``, ``thetax_prev/y/z`` (φ: after the swap of advance!
these are the link phases of the previous step), ``hx/hy/hz`` (``save_state``, gtdgl/src/io.jl:131-154); the open
boundary's ramp ``open_count``, ``open_old_x/y/z``, ``open_new_x/y/z`` (``open_extra``, io.jl:156-171); the PCG
warm start ``pcg_x1..3`` and, for pcg_fast's extrapolation, ``pcg_p1..3`` (the solution of the step before), each
on its link range (``_save_ladder``, gtdgl/src/protocol.jl:656-658).  Three differences, each so that a resume
continues the run to the bit:

* the derived fields are stored too (``F1``…, ``Ux``…, ``Vx``…, ``Jx``…): the reference rebuilds them on load
  (V = e^{−iθ} with the host's cos and sin, state.jl:31-46), which differs in the last bit from the device's;
* the noise is a counter-based stream, so its state is one integer, ``noise_step`` (the stream index of the next
  step), where the reference keeps its generator's state (``noise_rng``);
* ``open_theta_x/y/z``, the open boundary's link-phase term of the current ramp, which the device keeps between
  recomputations.

``load`` also takes a file with only the reference's keys: the derived fields are then rebuilt as the reference
does (`State.from_fields`) and the run continues close to, not equal to, the uninterrupted one.  That includes the
reference's own JLD2 checkpoints (``save_state`` with ``compress=true``; read by `juliatdgl_b200.jld2`), with the
heat model's temperature field ``Temp`` (protocol.jl:654) going into the carry.
"""
from __future__ import annotations

import dataclasses
import warnings
import os

import numpy as np

from . import gpu, jld2
from .abi import Carry
from .scheme import Stepper, sep_ranges
from .state import LINK_FIELDS, State

FORMAT = "juliatdgl_b200 checkpoint 1"

# the State's link fields under the reference's names (θ and φ) or under their own (the derived fields)
_REF_NAMES = {"θx": "thetax", "θy": "thetay", "θz": "thetaz", "φx": "thetax_prev", "φy": "thetay_prev",
              "φz": "thetaz_prev", "hx": "hx", "hy": "hy", "hz": "hz"}
_DERIVED = ("Ux", "Uy", "Uz", "Vx", "Vy", "Vz", "Jx", "Jy", "Jz")


def _range_shapes(st_or_grid):
    gr = st_or_grid.grid if isinstance(st_or_grid, Stepper) else st_or_grid
    return [tuple(b - a + 1 for a, b in r) for r in sep_ranges(gr)]


def save(path: str, s: State, carry: Carry | None = None, *, grid=None, steps: int = 0,
         noise_step: int | None = None, extra: dict | None = None) -> str:
    """Writes state `s` (and the carry, with `grid` for the shapes of the PCG ranges) to `path`, atomically."""
    out = {"format": np.array(FORMAT), "nbands": np.array(s.N), "steps": np.array(int(steps))}
    for µ, (g, f) in enumerate(zip(s.G, s.F)):
        out[f"G{µ + 1}"] = g
        out[f"F{µ + 1}"] = f
    for k in LINK_FIELDS:
        out[_REF_NAMES.get(k, k)] = getattr(s, k)
    if noise_step is not None:
        out["noise_step"] = np.array(int(noise_step), dtype=np.int64)
    if carry is not None:
        if carry.pcg_warm:
            shapes = _range_shapes(grid)
            o = 0
            for c, shp in enumerate(shapes):
                m = int(np.prod(shp))
                out[f"pcg_x{c + 1}"] = carry.pcg_x[o:o + m].reshape(shp, order="F")
                if carry.pcg_have2:
                    out[f"pcg_p{c + 1}"] = carry.pcg_xprev[o:o + m].reshape(shp, order="F")
                o += m
        if carry.open_count >= 0:
            out["open_count"] = np.array(int(carry.open_count))
            for ax, x in enumerate("xyz"):
                out[f"open_old_{x}"] = carry.open_old[ax]
                out[f"open_new_{x}"] = carry.open_new[ax]
                out[f"open_theta_{x}"] = carry.open_theta[ax]
    for k, v in (extra or {}).items():
        out[k] = np.asarray(v)
    tmp = path + ".tmp.npz"
    with open(tmp, "wb") as fh:
        np.savez_compressed(fh, **out)
    os.replace(tmp, path)
    return path


def _read(path: str, group):
    if path.endswith(".jld2"):   # a file gtdgl wrote (save_state, io.jl:131-154)
        d = jld2.load(path)
        if group is not None:
            d = d[group]
        return {k: (v if isinstance(v, (str, bytes, dict)) else np.asarray(v)) for k, v in d.items()}
    if group is not None:
        raise ValueError("a group is read from a JLD2 file only")
    with np.load(path, allow_pickle=False) as w:
        return {k: w[k] for k in w.files}


def load(path: str, st: Stepper, *, group: str | None = None, prev: str = "thetax_prev"):
    """(State, Carry, info) from a checkpoint for Stepper `st` (its grid and band count must match); info holds
    ``steps``, ``noise_step`` (None if absent) and every other key of the file.

    `path` is this library's ``.npz`` or one of gtdgl's ``.jld2`` files (`group`: read the keys of that group, e.g.
    a golden file's ``ini``).  `prev` names the previous link phases φ: ``thetax_prev`` (…y, …z) as save_state writes
    them; without them φ = θ, as load_state does (io.jl:181-191).  Release 1.2's state dumps call them ``phix``."""
    gr = st.grid
    d = _read(path, group)
    N = int(d["nbands"]) if "nbands" in d else 2
    if N != st.model.N:
        raise ValueError(f"{path}: {N} bands, the Stepper has {st.model.N}")
    G = [np.asfortranarray(d[f"G{µ + 1}"], dtype=np.complex128) for µ in range(N)]
    if G[0].shape != gr.node:
        raise ValueError(f"{path}: Ψ is {G[0].shape}, the grid needs {gr.node}")
    th = [d[n] for n in ("thetax", "thetay", "thetaz")]
    if prev.endswith("x_prev"):
        px = (prev, prev.replace("x_prev", "y_prev"), prev.replace("x_prev", "z_prev"))
    else:
        px = (prev, prev[:-1] + "y", prev[:-1] + "z")
    ph = [d[n] for n in px] if px[0] in d else th
    h = [d[n] for n in ("hx", "hy", "hz")]
    s = State.from_fields(gr, G, th, ph, h)
    if all(k in d for k in _DERIVED) and all(f"F{µ + 1}" in d for µ in range(N)):   # the exact state
        for µ in range(N):
            s.F[µ][...] = d[f"F{µ + 1}"]
        for k in _DERIVED:
            getattr(s, k)[...] = d[k]
    carry = Carry(st)
    if "pcg_x1" in d:
        carry.pcg_x[:] = np.concatenate([np.ravel(d[f"pcg_x{c + 1}"], order="F") for c in range(3)])
        carry.pcg_warm = 1
        if "pcg_p1" in d:
            carry.pcg_xprev[:] = np.concatenate([np.ravel(d[f"pcg_p{c + 1}"], order="F") for c in range(3)])
            carry.pcg_have2 = 1
    if "open_count" in d:
        carry.open_count = int(d["open_count"])
        for ax, x in enumerate("xyz"):
            carry.open_old[ax][...] = d[f"open_old_{x}"]
            carry.open_new[ax][...] = d[f"open_new_{x}"]
            if f"open_theta_{x}" in d:
                carry.open_theta[ax][...] = d[f"open_theta_{x}"]
    if st.heat is not None and "Temp" in d:   # the heat model's temperature field (protocol.jl:654)
        carry.heat_theta[...] = d["Temp"]
    info = dict(d)
    info["steps"] = int(d["steps"]) if "steps" in d else 0
    info["noise_step"] = int(d["noise_step"]) if "noise_step" in d else None
    if st.noise_T is not None and info["noise_step"] is None and "noise_rng" in d:
        # a file written by the reference carries its host generator (Xoshiro) but no index into this library's
        # counter-based stream: resuming would restart the stream at the Stepper's noise_step0 and repeat kicks
        warnings.warn("checkpoint: the file holds the reference's noise generator but no noise_step; the device's "
                      "noise stream restarts at the Stepper's noise_step0 (its first draws are repeated)",
                      RuntimeWarning, stacklevel=2)
    return s, carry, info


def save_run(path: str, gs: "gpu.GPUStepper", st: Stepper, like: State, *, extra: dict | None = None) -> str:
    """Checkpoints the run on context `gs` (Stepper `st`; `like` gives the host arrays' shapes): its device state,
    its carry, its step count and its noise stream index."""
    s = gs.download(like.copy())
    carry = gs.get_carry(Carry(st))
    steps = int(gs.stats().steps)
    noise = st.noise_step0 + steps if st.noise_T is not None else None
    return save(path, s, carry, grid=st.grid, steps=steps, noise_step=noise, extra=extra)


def resume(path: str, st: Stepper, *, group: str | None = None,
           prev: str = "thetax_prev") -> "tuple[gpu.GPUStepper, Stepper, dict]":
    """A new context continuing the run checkpointed in `path` (`group`, `prev` as `load`): the state and the carry
    uploaded, the noise stream continued from its index.  Returns (context, the Stepper it runs, info)."""
    s, carry, info = load(path, st, group=group, prev=prev)
    if info["noise_step"] is not None:
        st = dataclasses.replace(st, noise_step0=info["noise_step"])
    gs = gpu.GPUStepper(st)
    gs.upload(s)
    gs.set_carry(carry)
    return gs, st, info
