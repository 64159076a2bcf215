"""CPU checks of the C-ABI library: it loads, exports every entry point the
header declares, and reports errors without a GPU (no compute calls)."""
import ctypes as C
import os
import re

import pytest

from olam_b200 import abi, lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "olamgpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(olamgpu_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_header_symbols():
    L = lib.load()
    names = _declared()
    assert names, "header parse found no entry points"
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(lib.EXPORTS)


def test_fortran_interfaces_name_header_symbols():
    # every bind(C) interface of the Fortran module binds an entry point the
    # header declares
    src = open(os.path.join(ROOT, "olam_b200", "fortran", "olamgpu.f90")).read()
    bound = set(re.findall(r'bind\(C,\s*name="(olamgpu_[a-z0-9_]+)"\)', src))
    assert len(bound) >= 20
    assert not bound - set(_declared()), sorted(bound - set(_declared()))


def test_struct_sizes_match_header():
    # field counts of the ctypes mirror follow the header's declarations
    txt = open(os.path.join(ROOT, "include", "olamgpu.h")).read()
    assert "typedef struct olamgpu_grid" in txt
    assert C.sizeof(abi.CflDiag) == 36


def test_strerror_and_state_errors():
    L = lib.load()
    assert L.olamgpu_strerror(0) == b"ok"
    assert b"unsupported" in L.olamgpu_strerror(3)
    # hot-path calls before init are state errors, not crashes
    rc = L.olamgpu_scalar_transport_rk(None, None)
    assert rc == abi.E_STATE
    assert L.olamgpu_sync_to_host(abi.F_ALL) == abi.E_STATE
    assert L.olamgpu_set_coherence(7) == abi.E_ARG
    assert L.olamgpu_update_scalar_noalloc(None, None, None, None, None, None, C.c_float(1.0),
                                           None, None) == abi.E_STATE
    assert L.olamgpu_scalar_transport_rk_adjoint(None, None, None) == abi.E_STATE
    # the eddy and long-step entries too
    assert L.olamgpu_set_eddy(None) == abi.E_STATE
    assert L.olamgpu_comp_horiz_k() == abi.E_STATE
    assert L.olamgpu_set_scalars_bottom() == abi.E_STATE
    assert L.olamgpu_diagvel_t3d() == abi.E_STATE
    assert L.olamgpu_tracer_maxmin(None) == abi.E_STATE
    assert L.olamgpu_mass_sums(0, None, None) == abi.E_STATE
    assert L.olamgpu_timestep(0, 0, None) == abi.E_STATE
    assert L.olamgpu_timestep_diag(None, None) == abi.E_STATE
    assert L.olamgpu_set_halo(None) == abi.E_STATE
    assert L.olamgpu_set_surface_emission(None) == abi.E_STATE
    assert L.olamgpu_window_forward(2, 1, 0) == abi.E_STATE
    assert L.olamgpu_window_adjoint(None, None) == abi.E_STATE
    assert L.olamgpu_window_memory(1, 0, 4, 2) == abi.E_STATE
    assert L.olamgpu_window_rewind() == abi.E_STATE


def test_null_arguments_rejected():
    L = lib.load()
    assert L.olamgpu_init(None, None, None) == abi.E_ARG


def _header_constants():
    txt = open(os.path.join(ROOT, "include", "olamgpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    out = {}
    for name, expr in re.findall(r"\b(OLAMGPU_(?:F|TS|WIN)_[A-Z0-9_]+)\s*=\s*([0-9xXa-fA-Fu<\s]+?)\s*[,}\n]", txt):
        parts = [int(x.strip().rstrip("uU"), 0) for x in expr.split("<<")]   # N, 0xN or N << k
        out[name] = parts[0] << parts[1] if len(parts) == 2 else parts[0]
    return out


def test_flag_constants_agree_across_bindings():
    # the flag words of the header, the Python binding and the Fortran module
    h = _header_constants()
    assert {"OLAMGPU_F_ALL", "OLAMGPU_TS_GRAPH", "OLAMGPU_WIN_HOST", "OLAMGPU_WIN_LEAN"} <= set(h)
    for name, v in h.items():
        assert getattr(abi, name[len("OLAMGPU_"):]) == v, name
    src = open(os.path.join(ROOT, "olam_b200", "fortran", "olamgpu.f90")).read()
    fortran = {n: int(v) for n, v in re.findall(r"\b(OLAMGPU_(?:F|TS|WIN)_[A-Z0-9_]+)\s*=\s*(\d+)", src)}
    assert fortran, "no Fortran parameters found"
    for name, v in fortran.items():
        assert h[name] == v, name
