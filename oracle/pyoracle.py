"""Python binding of the CPU oracle (liboracle_tdgl.so).

TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
It drives the C++ restatement of gtdgl's step (oracle.cpp) through the same tdgl_params / tdgl_state_view
structures as the product library, so that both are fed identical inputs.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from juliatdgl_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle_tdgl.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "oracle.cpp")
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
            build()
        L = C.CDLL(LIB)
        vp = C.c_void_p
        L.oracle_ctx_create.argtypes = [C.POINTER(abi.Params_t), C.POINTER(vp)]
        L.oracle_ctx_destroy.argtypes = [vp]
        L.oracle_upload_state.argtypes = [vp, C.POINTER(abi.StateView_t)]
        L.oracle_download_state.argtypes = [vp, C.POINTER(abi.StateView_t)]
        L.oracle_set_carry.argtypes = [vp, C.POINTER(abi.CarryView_t)]
        L.oracle_get_carry.argtypes = [vp, C.POINTER(abi.CarryView_t)]
        L.oracle_steps.argtypes = [vp, C.c_int, C.c_double, C.c_double]
        L.oracle_steps_ramp.argtypes = [vp, C.c_int, C.c_double, abi.dptr]
        L.oracle_get_stats.argtypes = [vp, C.POINTER(abi.Stats_t)]
        L.oracle_last_error.restype = C.c_char_p
        L.oracle_sep_apply.argtypes = [vp, abi.dptr, C.c_int]
        L.oracle_bar_field.argtypes = [C.POINTER(abi.Grid_t), C.c_int] + [abi.dptr] * 6
        L.oracle_field_solve.argtypes = [vp]
        L.oracle_qp_delta.argtypes = [vp, abi.dptr]
        L.oracle_qp_mu.argtypes = [vp, abi.dptr]
        L.oracle_qp_iters.argtypes = [vp]
        L.oracle_set_threads.argtypes = [C.c_int]
        L.oracle_link_rotations.argtypes = [C.c_int] * 4 + [C.POINTER(C.c_int32), C.c_int] + [abi.dptr] * 3 + \
            [C.c_double, abi.dptr, abi.dptr]
        L.oracle_cis_short.argtypes = [C.c_double, abi.dptr]
        L.oracle_kwt_update.argtypes = [abi.dptr, abi.dptr, C.c_double, abi.dptr]
        _lib = L
    return _lib


class OracleStepper:
    """The oracle's context for one Stepper: upload a State, take n steps, download it."""

    def __init__(self, st):
        self.st = st
        self.p, self._keep = abi.pack_params(st)
        self.h = C.c_void_p()
        rc = lib().oracle_ctx_create(C.byref(self.p), C.byref(self.h))
        if rc != 0:
            raise RuntimeError(f"oracle_ctx_create: {rc} {lib().oracle_last_error().decode()}")

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.oracle_ctx_destroy(self.h)
            self.h = None

    def upload(self, s):
        v = abi.state_view(s)
        lib().oracle_upload_state(self.h, C.byref(v))

    def download(self, s):
        v = abi.state_view(s)
        lib().oracle_download_state(self.h, C.byref(v))
        return s

    def steps(self, n, H, HJ):
        return lib().oracle_steps(self.h, int(n), float(H), float(HJ))

    def steps_ramp(self, H, HJ):
        HJ = np.ascontiguousarray(HJ, dtype=np.float64)
        return lib().oracle_steps_ramp(self.h, len(HJ), float(H), HJ.ctypes.data_as(abi.dptr))

    def get_carry(self, carry):
        v = carry.view()
        lib().oracle_get_carry(self.h, C.byref(v))
        carry.absorb(v)
        return carry

    def set_carry(self, carry):
        v = carry.view()
        lib().oracle_set_carry(self.h, C.byref(v))

    def stats(self):
        s = abi.Stats_t()
        lib().oracle_get_stats(self.h, C.byref(s))
        return s

    def field_solve(self):
        """The field solve of step! alone on the uploaded θ, φ (implicit_curl! / scale_increment!)."""
        return lib().oracle_field_solve(self.h)

    def qp_delta(self):
        """δ = μ_π − μ_σ of the two normal fluids (qp_potential!) from the current state, node-shaped."""
        gr = self.st.grid
        out = np.zeros((gr.Nx + 1, gr.Ny + 1, gr.Nz + 1), order="F")
        rc = lib().oracle_qp_delta(self.h, out.ctypes.data_as(abi.dptr))
        if rc:
            raise RuntimeError(f"oracle_qp_delta: {rc}")
        return out

    def qp_iters(self):
        """Conjugate-gradient iterations of the last δ solve of a sculpted sample."""
        return lib().oracle_qp_iters(self.h)

    def qp_mu(self):
        """The potentials μ_µ of N normal fluids (QPExchangeN's qp_potential!) from the current state."""
        gr = self.st.grid
        out = np.zeros((self.st.N, gr.Nx + 1, gr.Ny + 1, gr.Nz + 1))
        flat = np.zeros(out.size)
        rc = lib().oracle_qp_mu(self.h, flat.ctypes.data_as(abi.dptr))
        if rc:
            raise RuntimeError(f"oracle_qp_mu: {rc}")
        n = (gr.Nx + 1) * (gr.Ny + 1) * (gr.Nz + 1)
        return [flat[mu * n:(mu + 1) * n].reshape((gr.Nx + 1, gr.Ny + 1, gr.Nz + 1), order="F") for mu in range(self.st.N)]

    def sep_apply(self, b, f32=False):
        b = np.ascontiguousarray(b, dtype=np.float64).copy()
        rc = lib().oracle_sep_apply(self.h, b.ctypes.data_as(abi.dptr), int(f32))
        if rc != 0:
            raise RuntimeError("sep_apply needs a SEP or PCG stepper")
        return b


def bar_field(gr, nq=8):
    """The oracle's own restatement of field.jl:151-180 (for cross-checking the host mirror)."""
    g = abi.Grid_t(gr.Nx, gr.Ny, gr.Nz, gr.x1, gr.x2, gr.y1, gr.y2, gr.z1, gr.z2, gr.dx, gr.dy, gr.dz)
    Ny, Nz = gr.Ny, gr.Nz
    out = [np.zeros((Ny + 1, 2), order="F"), np.zeros((2, Nz), order="F"), np.zeros((Ny, 2), order="F"),
           np.zeros((2, Nz + 1), order="F"), np.zeros((Ny, Nz + 1), order="F"), np.zeros((Ny + 1, Nz), order="F")]
    lib().oracle_bar_field(C.byref(g), nq, *[o.ctypes.data_as(abi.dptr) for o in out])
    return out


def run(st, s, n, H, HJ):
    """n oracle steps from a copy of s; returns the new state."""
    o = OracleStepper(st)
    s2 = s.copy()
    o.upload(s2)
    rc = o.steps(n, H, HJ)
    if rc not in (0, abi.E_NOCONV):
        raise RuntimeError(f"oracle_steps: {rc}")
    o.download(s2)
    return s2


def link_rotations(op, V, U, rng, par, ax=0, Om=None):
    """The oracle's _rot! (op 0 → (L, R)), _rotfrac! (op 1 → L) and _link_rate! (op 2 → R) on arrays."""
    from juliatdgl_b200.gpu import _rotations
    return _rotations(lib().oracle_link_rotations, op, V, U, rng, par, ax, Om)


def cis_short(a):
    out = np.zeros(2)
    lib().oracle_cis_short(float(a), out.ctypes.data_as(abi.dptr))
    return complex(out[0], out[1])


def kwt_update(g, d, g2):
    gg = np.array([g.real, g.imag])
    dd = np.array([d.real, d.imag])
    out = np.zeros(2)
    lib().oracle_kwt_update(gg.ctypes.data_as(abi.dptr), dd.ctypes.data_as(abi.dptr), float(g2), out.ctypes.data_as(abi.dptr))
    return complex(out[0], out[1])
