"""The C-ABI boundary without a GPU: the library loads, exports every entry point include/tdgl_b200.h declares, its
structures have the layout the ctypes mirror (and a Julia NTuple/struct mirror) assumes, the host-side parameter
check accepts what the step supports and names what it refuses, and context creation on a machine without a GPU
fails with an error code and a message instead of falling back to the host.
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import cases
from conftest import have_gpu
from juliatdgl_b200 import abi, gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "tdgl_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = []
    for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(tdgl_\w+)\s*\(", src, flags=re.M):
        if not m.group(0).lstrip().startswith(("typedef", "#")):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_the_entry_points():
    names = declared_functions()
    for must in ("tdgl_ctx_create", "tdgl_ctx_destroy", "tdgl_upload_state", "tdgl_download_state", "tdgl_set_carry",
                 "tdgl_get_carry", "tdgl_steps", "tdgl_steps_ramp", "tdgl_supported", "tdgl_last_error",
                 "tdgl_sep_apply_noalloc", "tdgl_meter_set", "tdgl_measure", "tdgl_vortices"):
        assert must in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    L = gpu.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_abi_version_matches_header():
    L = gpu.lib()
    L.tdgl_abi_version.restype = C.c_int
    want = int(re.search(r"#define TDGL_ABI_VERSION (\d+)", open(HEADER).read()).group(1))
    assert L.tdgl_abi_version() == want == abi.ABI_VERSION


STRUCTS = {"tdgl_grid": abi.Grid_t, "tdgl_bandcoef": abi.BandCoef_t, "tdgl_params": abi.Params_t,
           "tdgl_state_view": abi.StateView_t, "tdgl_carry_view": abi.CarryView_t, "tdgl_stats": abi.Stats_t,
           "tdgl_meter": abi.Meter_t, "tdgl_obs": abi.Obs_t}


def test_struct_layout_matches_ctypes(tmp_path):
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "tdgl_b200.h"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln.strip():
            s, f, v = ln.split()
            got[(s, f)] = int(v)
    for cname, py in STRUCTS.items():
        assert got[(cname, "sizeof")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


@pytest.mark.parametrize("kind", cases.SMALL_KINDS)
def test_supported_accepts_every_parity_case(kind):
    st, s, H, HJ = cases.small(kind)
    ok, why = gpu.supported(st)
    assert ok, why


@pytest.mark.parametrize("kind", list(cases.NOISY))
def test_supported_accepts_the_noisy_cases(kind):
    st, s, H, HJ = cases.small(kind, **cases.NOISY[kind])
    ok, why = gpu.supported(st)
    assert ok, why
    p, keep = abi.pack_params(st)
    assert p.noise_on == 1 and p.noise_T == st.noise_T and p.noise_seed == st.noise_seed
    assert p.noise_field == int(st.noise_field) and p.noise_step0 == st.noise_step0
    assert [p.noise_gamma[mu] for mu in range(st.model.N)] == [b.Γ for b in st.model.bands]


def test_supported_refuses_bad_noise_with_a_reason():
    st, s, H, HJ = cases.small("rkc_kwt_rotframe", noise=1e-3)
    st.noise_T = -0.05
    ok, why = gpu.supported(st)
    assert not ok and "noise" in why.lower()


def test_packed_parameters_follow_the_stepper():
    st, s, H, HJ = cases.small("pcg")
    p, keep = abi.pack_params(st)
    assert p.abi_version == abi.ABI_VERSION and p.nbands == st.model.N
    assert p.dt == st.dt and p.solver == st.solver
    g = st.grid
    assert (p.grid.Nx, p.grid.Ny, p.grid.Nz) == (g.Nx, g.Ny, g.Nz)
    assert (p.grid.x1, p.grid.x2, p.grid.z1, p.grid.z2) == (g.x1, g.x2, g.z1, g.z2)
    assert p.pcg_tol == st.pcg.tol and p.a_imp == st.fc.a
    f = np.ctypeslib.as_array(p.f, shape=((g.Nx + 1) * (g.Ny + 1) * (g.Nz + 1),))
    assert np.array_equal(f, np.asarray(st.masks.f).ravel(order="F"))


@pytest.mark.skipif(have_gpu(), reason="checks the behaviour on a host without a GPU")
def test_context_creation_without_a_gpu_fails_loudly():
    st, s, H, HJ = cases.small("euler_substeps")
    p, keep = abi.pack_params(st)
    L = gpu.lib()
    h = C.c_void_p()
    rc = L.tdgl_ctx_create(C.byref(p), C.byref(h))
    assert rc == abi.E_CUDA and not h.value
    assert L.tdgl_last_error(None)
    with pytest.raises(gpu.TDGLError):
        gpu.GPUStepper(st)


def test_hook_has_no_host_fallback():
    with pytest.raises(ValueError):
        gpu.enable_(fallback="cpu")
    gpu.disable_()
