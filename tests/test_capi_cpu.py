"""CPU-side checks of the C ABI library: it loads, exports every declared symbol and fails
cleanly (error code + message, no crash) when no B200 is present."""
import ctypes as C
import os
import re

import pytest

from forte_b200 import build, capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "fcib.h")).read()
    return sorted(set(re.findall(r"\b(fcib_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def L():
    build.build()
    return capi.lib()


def test_exports_every_declared_symbol(L):
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(capi.SIGNATURES), "ctypes signatures must cover the header exactly"


def test_default_options_match_forte(L):
    o = capi.default_options()
    assert (o.maxiter, o.guess_per_root, o.dets_per_guess, o.collapse_per_root, o.subspace_per_root) == (100, 1, 50, 2, 10)
    assert o.e_convergence == 1e-9 and o.r_convergence == 1e-6


def test_null_arguments_are_rejected(L):
    assert L.fcib_create(None, 0) == capi.FCIB_ERR_ARG
    assert L.fcib_solve(None, None, None, None) == capi.FCIB_ERR_ARG
    assert b"null" in L.fcib_last_error()


def test_create_without_gpu_fails_cleanly(L):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    rc = L.fcib_create(C.byref(h), 0)
    assert rc in (capi.FCIB_ERR_CUDA, capi.FCIB_ERR_ARG)
    assert not h.value
    assert len(L.fcib_last_error()) > 0


def test_default_build_has_no_phase_clocks(L):
    """The batched solver's phase clocks exist only in the profiling build (-DFCIB_BATCH_PHASES)."""
    out = (C.c_ulonglong * 8)()
    assert L.fcib_batch_phase_cycles(out) == capi.FCIB_ERR_UNSUPPORTED
    assert b"FCIB_BATCH_PHASES" in L.fcib_last_error()
    assert L.fcib_batch_phase_cycles(None) == capi.FCIB_ERR_ARG


def test_default_options_select_the_blocked_layout(L):
    o = capi.default_options()
    assert o.sym_blocked == 1 and o.spin_adapt == 0
