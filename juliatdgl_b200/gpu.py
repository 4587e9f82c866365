"""The accelerator interface of the reference's TDGLGPU module, on the B200 library (libtdgl_b200.so).

Mirrors gpu/TDGLGPU/src/TDGLGPU.jl: ``supported(st)`` (:39-44), ``GPUStepper(st)`` (the device copy of a Stepper),
``device_state`` / ``device_state_`` (:63-74), ``gpu_steps_`` (:2065-2071), ``host_state_`` (:77-82), and the ladder
hook ``enable_`` / ``disable_`` / ``execution_stats`` (:2076-2144) with ``cycle_steps`` in the role of gtdgl's
``_cycle_steps!`` (gtdgl/src/protocol.jl:305-316).  There is no CPU fallback: every call runs the CUDA library, and a
missing library or GPU is an error.
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from . import abi
from .scheme import Stepper
from .state import State

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libtdgl_b200.so")
_lib = None


class TDGLError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{abi.ERRNAMES.get(code, code)}: {msg}")
        self.code = code


def lib():
    """The loaded CUDA library (built in-tree by ``python -m juliatdgl_b200.build``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise RuntimeError(f"{LIB} is missing: build it with `python -m juliatdgl_b200.build`")
        L = C.CDLL(LIB)
        vp = C.c_void_p
        L.tdgl_ctx_create.argtypes = [C.POINTER(abi.Params_t), C.POINTER(vp)]
        L.tdgl_ctx_destroy.argtypes = [vp]
        L.tdgl_upload_state.argtypes = [vp, C.POINTER(abi.StateView_t)]
        L.tdgl_download_state.argtypes = [vp, C.POINTER(abi.StateView_t)]
        L.tdgl_set_carry.argtypes = [vp, C.POINTER(abi.CarryView_t)]
        L.tdgl_get_carry.argtypes = [vp, C.POINTER(abi.CarryView_t)]
        L.tdgl_steps.argtypes = [vp, C.c_int32, C.c_double, C.c_double]
        L.tdgl_steps_ramp.argtypes = [vp, C.c_int32, C.c_double, abi.dptr]
        L.tdgl_steps_async.argtypes = [vp, C.c_int32, C.c_double, C.c_double]
        L.tdgl_sync.argtypes = [vp]
        L.tdgl_set_graphs.argtypes = [vp, C.c_int32]
        L.tdgl_set_branches.argtypes = [vp, C.c_int32]
        for f in ("tdgl_snapshot_take", "tdgl_snapshot_restore", "tdgl_snapshot_free"):
            getattr(L, f).argtypes = [vp, C.c_int32]
        L.tdgl_device_bytes.argtypes = [vp]
        L.tdgl_device_bytes.restype = C.c_int64
        L.tdgl_batch_create.argtypes = [C.POINTER(vp), C.c_int32, C.POINTER(vp)]
        L.tdgl_batch_steps.argtypes = [vp, C.c_int32, abi.dptr, abi.dptr, C.c_int32]
        L.tdgl_batch_info.argtypes = [vp, C.POINTER(C.c_int32)]
        L.tdgl_batch_set_merge.argtypes = [vp, C.c_int32, C.c_double]
        L.tdgl_batch_merge_info.argtypes = [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.tdgl_batch_destroy.argtypes = [vp]
        L.tdgl_stream.argtypes = [vp]
        L.tdgl_stream.restype = vp
        L.tdgl_device_state.argtypes = [vp, C.POINTER(abi.StateView_t)]
        L.tdgl_get_stats.argtypes = [vp, C.POINTER(abi.Stats_t)]
        L.tdgl_last_error.argtypes = [vp]
        L.tdgl_last_error.restype = C.c_char_p
        L.tdgl_supported.argtypes = [C.POINTER(abi.Params_t), C.c_char_p, C.c_int32]
        L.tdgl_sep_apply.argtypes = [vp, abi.dptr, abi.dptr, C.c_int32]
        L.tdgl_field_solve.argtypes = [vp]
        L.tdgl_link_rotations.argtypes = [C.c_int32] * 4 + [C.POINTER(C.c_int32), C.c_int32] + [abi.dptr] * 3 + \
            [C.c_double, abi.dptr, abi.dptr]
        L.tdgl_meter_set.argtypes = [vp, C.POINTER(abi.Meter_t)]
        L.tdgl_measure.argtypes = [vp, C.POINTER(abi.Obs_t)]
        ip = C.POINTER(C.c_int32)
        L.tdgl_vortices.argtypes = [vp, C.c_int32, C.c_int32, ip, ip, ip, ip]
        L.tdgl_profile.argtypes = [vp, C.c_int32]
        L.tdgl_profile_read.argtypes = [vp, C.c_int32, C.POINTER(C.c_char_p), C.POINTER(C.c_int64),
                                        C.POINTER(C.c_double), C.POINTER(C.c_double)]
        _lib = L
    return _lib


def _check(rc, h=None):
    if rc != 0:
        raise TDGLError(rc, lib().tdgl_last_error(h).decode())
    return rc


def supported(st: Stepper):
    """(ok, why): whether the library runs this Stepper's step (TDGLGPU.jl:39-44)."""
    try:
        p, keep = abi.pack_params(st)
    except (ValueError, NotImplementedError) as e:
        return (False, str(e))
    buf = C.create_string_buffer(256)
    ok = lib().tdgl_supported(C.byref(p), buf, 256)
    return (bool(ok), buf.value.decode())


class GPUStepper:
    """The device copy of a Stepper: coefficients, masks, tables and workspaces (TDGLGPU.jl GPUStepper)."""

    def __init__(self, st: Stepper):
        self.st = st
        self.params, self._keep = abi.pack_params(st)
        self.h = C.c_void_p()
        _check(lib().tdgl_ctx_create(C.byref(self.params), C.byref(self.h)))
        self.carry = abi.Carry(st)
        self._state_id = None

    def close(self):
        if getattr(self, "h", None) and self.h.value and _lib is not None:
            _lib.tdgl_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        self.close()

    # -- the state
    def upload(self, s: State):
        v = abi.state_view(s)
        _check(lib().tdgl_upload_state(self.h, C.byref(v)), self.h)

    def download(self, s: State) -> State:
        v = abi.state_view(s)
        _check(lib().tdgl_download_state(self.h, C.byref(v)), self.h)
        return s

    # -- the carry (PCG warm start, open ramp)
    def set_carry(self, carry: abi.Carry | None = None):
        carry = carry or self.carry
        v = carry.view()
        _check(lib().tdgl_set_carry(self.h, C.byref(v)), self.h)

    def get_carry(self, carry: abi.Carry | None = None) -> abi.Carry:
        carry = carry or self.carry
        v = carry.view()
        _check(lib().tdgl_get_carry(self.h, C.byref(v)), self.h)
        carry.absorb(v)
        return carry

    # -- stepping
    def steps(self, n: int, H: float, HJ: float, *, wait=True):
        f = lib().tdgl_steps if wait else lib().tdgl_steps_async
        rc = f(self.h, int(n), float(H), float(HJ))
        if rc not in (0, abi.E_NOCONV):
            _check(rc, self.h)
        return rc

    def steps_ramp(self, H: float, HJ):
        HJ = np.ascontiguousarray(HJ, dtype=np.float64)
        rc = lib().tdgl_steps_ramp(self.h, len(HJ), float(H), HJ.ctypes.data_as(abi.dptr))
        if rc not in (0, abi.E_NOCONV):
            _check(rc, self.h)
        return rc

    def sync(self):
        """Waits for the enqueued steps; returns E_NOCONV if a PCG solve among them reached maxit."""
        rc = lib().tdgl_sync(self.h)
        if rc not in (0, abi.E_NOCONV):
            _check(rc, self.h)
        return rc

    def snapshot(self, slot: int = 0):
        """Keeps the resident state, carry and step count in device slot `slot` (protocol.jl:222-236)."""
        _check(lib().tdgl_snapshot_take(self.h, int(slot)), self.h)

    def restore(self, slot: int = 0):
        _check(lib().tdgl_snapshot_restore(self.h, int(slot)), self.h)

    def free_snapshot(self, slot: int = 0):
        _check(lib().tdgl_snapshot_free(self.h, int(slot)), self.h)

    @property
    def device_bytes(self) -> int:
        return int(lib().tdgl_device_bytes(self.h))

    def set_graphs(self, on: bool = True):
        """Steps as CUDA graphs once they repeat (on by default); off: every kernel launched from the host."""
        _check(lib().tdgl_set_graphs(self.h, int(on)), self.h)

    def set_branches(self, on: bool = True):
        """Parallel branches inside a step (on by default: the bands side by side, the PCG's work beside its
        preconditioner); off for many contexts in flight at once.  Results are identical either way."""
        _check(lib().tdgl_set_branches(self.h, int(on)), self.h)

    @property
    def stream(self) -> int:
        return lib().tdgl_stream(self.h) or 0

    def sep_apply(self, b, f32=False):
        """(I + aK)^{-1} b on the packed ranges (implicit.jl _sep_solve! / _precond32!)."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        z = np.empty_like(b)
        _check(lib().tdgl_sep_apply(self.h, b.ctypes.data_as(abi.dptr), z.ctypes.data_as(abi.dptr), int(f32)), self.h)
        return z

    def field_solve(self):
        """The field solve of step! alone on the resident θ, φ (implicit_curl! / scale_increment!)."""
        return _check(lib().tdgl_field_solve(self.h), self.h)

    def profile(self, on=True):
        _check(lib().tdgl_profile(self.h, int(on)), self.h)

    def profile_read(self):
        n = lib().tdgl_profile_read(self.h, -1, None, None, None, None)
        rows = []
        for cat in range(n):
            name, launches, ms, by = C.c_char_p(), C.c_int64(), C.c_double(), C.c_double()
            lib().tdgl_profile_read(self.h, cat, C.byref(name), C.byref(launches), C.byref(ms), C.byref(by))
            if launches.value:
                rows.append({"kernel": name.value.decode(), "launches": launches.value, "ms": ms.value,
                             "bytes": by.value})
        return rows

    # -- the cycle observables (protocol.jl:148-189, :409-451; observables.jl:48-114)
    def meter_set(self, vm, nphase: int | None = None):
        """Sets the voltmeter (a protocol.Voltmeter) and takes the baselines from the current device state."""
        self._vm = vm
        self._nphase = self.st.model.N if nphase is None else int(nphase)
        self._vm_keep = [np.asfortranarray(a.astype(np.uint8)) for a in (vm.Min, vm.Mou, vm.line_ok)]
        u8 = C.POINTER(C.c_uint8)
        m = abi.Meter_t(vm.vi, vm.vo, self._nphase, *(a.ctypes.data_as(u8) for a in self._vm_keep))
        _check(lib().tdgl_meter_set(self.h, C.byref(m)), self.h)

    def measure(self):
        """The observables of the current device state (and the baselines move to it): a dict with the path phases
        D[µ] (line grid, µ < nphase), vsum_in, vsum_out, ta_sum, res[µ], amax, diffh, Itot, Isam."""
        vm = self._vm
        D = [np.zeros(vm.Min.shape, order="F") for _ in range(self._nphase)]
        o = abi.Obs_t()
        for mu, d in enumerate(D):
            o.D[mu] = d.ctypes.data_as(abi.dptr)
        _check(lib().tdgl_measure(self.h, C.byref(o)), self.h)
        N = self.st.model.N
        return {"D": D, "vsum_in": o.vsum_in, "vsum_out": o.vsum_out, "ta_sum": o.ta_sum,
                "res": [o.res[mu] for mu in range(N)], "amax": o.amax, "diffh": o.diffh, "Itot": o.Itot,
                "Isam": o.Isam}

    def vortices(self, band: int, kc: int, with_map: bool = False):
        """count_vortices of band `band` (0-based) on the plane kc (1-based): (Nv, nmap or None, Nv_loop, loop_ok)."""
        gr = self.st.grid
        a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
        nmap = np.zeros((gr.x2 - gr.x1 + 1, gr.y2 - gr.y1 + 1), dtype=np.int32, order="F") if with_map else None
        mp = nmap.ctypes.data_as(C.POINTER(C.c_int32)) if with_map else None
        _check(lib().tdgl_vortices(self.h, band, kc, C.byref(a), C.byref(b), C.byref(c), mp), self.h)
        return a.value, nmap, b.value, bool(c.value)

    def stats(self) -> abi.Stats_t:
        s = abi.Stats_t()
        _check(lib().tdgl_get_stats(self.h, C.byref(s)), self.h)
        return s


class Batch:
    """Independent contexts stepped in lockstep, one graph launch per step once their steps are captured
    (tdgl_batch_*); contexts whose steps launch the same kernels share one launch per kernel (merged).  The contexts
    stay usable on their own (upload, download, measure) between calls."""

    def __init__(self, steppers, *, merge=True, blocks_per_sm=0.0):
        self.gs = list(steppers)
        hs = (C.c_void_p * len(self.gs))(*[g.h.value for g in self.gs])
        self.h = C.c_void_p()
        _check(lib().tdgl_batch_create(hs, len(self.gs), C.byref(self.h)))
        if not merge or blocks_per_sm:
            self.set_merge(merge, blocks_per_sm)

    def set_merge(self, on: bool, blocks_per_sm: float = 0.0):
        """Merging on or off, and the merged x-grid of the plane transforms in blocks per SM (0: unchanged)."""
        _check(lib().tdgl_batch_set_merge(self.h, int(bool(on)), float(blocks_per_sm)))

    def tune(self, H, HJ, candidates=(1.0, 2.0, 4.0, 8.0, 16.0), steps: int = 4) -> dict:
        """Autotunes the merged launch shape: the x-grid of the plane transforms, in blocks per SM over the whole
        merged launch.  Each candidate captures the step again and times `steps` steps on the host clock (after the
        two steps that capture both parities); the fastest stays set.  The steps are the runs' own steps (every
        candidate gives the same bits): 2 + steps per candidate.  Returns {candidate: seconds}."""
        times = {}
        for c in candidates:
            self.set_merge(True, c)
            self.steps(2, H, HJ)
            t0 = time.perf_counter()
            self.steps(steps, H, HJ)
            times[float(c)] = time.perf_counter() - t0
        self.set_merge(True, min(times, key=times.get))
        return times

    @property
    def merge_info(self) -> dict:
        """Of the captured step: contexts served by merged launches, chains of merged launches, kernel launches of
        a batch step in all."""
        v = [C.c_int32(0) for _ in range(3)]
        _check(lib().tdgl_batch_merge_info(self.h, *[C.byref(x) for x in v]))
        return {"contexts": v[0].value, "chains": v[1].value, "launches": v[2].value}

    def steps(self, n: int, H, HJ, *, wait=True):
        """n steps of every context with H[i], HJ[i]; returns E_NOCONV if a PCG solve reached maxit."""
        H = np.ascontiguousarray(np.broadcast_to(np.asarray(H, dtype=np.float64), (len(self.gs),)))
        HJ = np.ascontiguousarray(np.broadcast_to(np.asarray(HJ, dtype=np.float64), (len(self.gs),)))
        rc = lib().tdgl_batch_steps(self.h, int(n), H.ctypes.data_as(abi.dptr), HJ.ctypes.data_as(abi.dptr), int(wait))
        if rc not in (0, abi.E_NOCONV):
            _check(rc)
        return rc

    @property
    def one_graph(self) -> bool:
        v = C.c_int32(0)
        _check(lib().tdgl_batch_info(self.h, C.byref(v)))
        return bool(v.value)

    def close(self):
        if self.h:
            lib().tdgl_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GState:
    """A state resident on the device (TDGLGPU.jl GState), owned by its GPUStepper."""

    def __init__(self, gs: GPUStepper):
        self.gs = gs


def device_state(gs: GPUStepper, s: State) -> GState:
    """The state `s` copied to the device (TDGLGPU.jl:63-67)."""
    gs.upload(s)
    return GState(gs)


def device_state_(g: GState, s: State) -> GState:
    """The state `s` copied into the device state `g` (TDGLGPU.jl:69-74)."""
    g.gs.upload(s)
    return g


def gpu_steps_(g: GState, gs: GPUStepper, n: int, *, H: float, HJ: float) -> GState:
    """`n` steps of step!(s, st; H, HJ) on the device, then a synchronisation (TDGLGPU.jl:2065-2071)."""
    gs.steps(n, H, HJ)
    return g


def host_state_(s: State, g: GState) -> State:
    """The device state copied back into `s`, every field (TDGLGPU.jl:77-82)."""
    return g.gs.download(s)


# ---------------------------------------------------------------------------------------------- the ladder hook
STEPS = None          # the accelerator closure, as gtdgl's `STEPS = Ref{Any}(nothing)` (protocol.jl:305)
_LAST = None          # (Stepper, GPUStepper)
_DEV = None           # (State, GState)
_STATS = {"backend": "", "backend_cycles": 0, "backend_steps": 0, "cpu_fallback_cycles": 0, "cpu_fallback_steps": 0}


def execution_stats():
    return dict(_STATS)


def enable_(fallback: str = "error"):
    """Every cycle of a ladder steps on the B200 (TDGLGPU.jl:2103-2111).  Only ``fallback="error"`` exists here:
    the library has no CPU path, so an unsupported Stepper raises instead of stepping on the host."""
    global STEPS, _LAST, _DEV
    if fallback not in ("error", "cpu"):
        raise ValueError("fallback must be 'cpu' or 'error'")
    if fallback == "cpu":
        raise ValueError("this backend has no CPU fallback; use fallback='error'")
    _LAST = None
    _DEV = None
    _STATS.update(backend="B200 (libtdgl_b200)", backend_cycles=0, backend_steps=0, cpu_fallback_cycles=0,
                  cpu_fallback_steps=0)
    STEPS = _gpu_cycle


def disable_():
    global STEPS, _LAST, _DEV
    if _LAST is not None:
        _LAST[1].close()
    STEPS = None
    _LAST = None
    _DEV = None


def _gpu_cycle(s: State, st: Stepper, n: int, *, H: float, HJ: float):
    """One protocol cycle (TDGLGPU.jl:2114-2144): the state and the solver carry up, n steps, everything back."""
    global _LAST, _DEV
    if _LAST is None or _LAST[0] is not st:
        ok, why = supported(st)
        if not ok:
            raise ValueError(f"B200 backend: {why} is unsupported; CPU fallback is disabled")
        if _LAST is not None:
            _LAST[1].close()
        _LAST = (st, GPUStepper(st))
        _DEV = None
    gs = _LAST[1]
    carry = getattr(st, "carry", None)
    if carry is None:
        carry = st.carry = abi.Carry(st)
    if _DEV is None or _DEV[0] is not s:
        _DEV = (s, device_state(gs, s))
    else:
        device_state_(_DEV[1], s)
    gs.set_carry(carry)
    gpu_steps_(_DEV[1], gs, n, H=H, HJ=HJ)
    gs.get_carry(carry)
    host_state_(s, _DEV[1])
    _STATS["backend_cycles"] += 1
    _STATS["backend_steps"] += n
    return s


def cycle_steps(s: State, st: Stepper, n: int, *, H: float, HJ: float):
    """gtdgl's `_cycle_steps!` (protocol.jl:306-316) for hosts that drive ladders from Python: the hook when it is
    set; without it there is nothing to step on (this package has no CPU stepper)."""
    if STEPS is None:
        raise RuntimeError("no accelerator enabled: call enable_() (this package has no CPU stepper)")
    return STEPS(s, st, n, H=H, HJ=HJ)


def link_rotations(op: int, V, U, rng, par: float, ax: int = 0, Om=None):
    """The step's temporal link rotations on arrays (tdgl_link_rotations): op 0 = _rot! → (L, R), 1 = _rotfrac! → L,
    2 = _link_rate! along ax → R (real).  V, U complex (n1, n2, n3) arrays; rng = (i0, i1, j0, j1, k0, k1), 1-based."""
    return _rotations(lib().tdgl_link_rotations, op, V, U, rng, par, ax, Om)


def _rotations(fn, op, V, U, rng, par, ax, Om):
    V = np.asfortranarray(V, dtype=np.complex128)
    U = np.asfortranarray(U, dtype=np.complex128)
    n1, n2, n3 = V.shape
    r = (C.c_int32 * 6)(*[int(x) for x in rng])
    L = np.zeros_like(V) if op != 2 else None
    R = np.zeros_like(V) if op == 0 else (np.zeros(V.shape, order="F") if op == 2 else None)
    Om = np.asfortranarray(Om, dtype=np.float64) if Om is not None else None
    ptr = lambda a: a.ctypes.data_as(abi.dptr) if a is not None else None
    rc = fn(int(op), n1, n2, n3, r, int(ax), ptr(V), ptr(U), ptr(Om), float(par), ptr(L), ptr(R))
    if rc != 0:
        raise TDGLError(rc, "link rotations")
    return (L, R) if op == 0 else (L if op == 1 else R)
