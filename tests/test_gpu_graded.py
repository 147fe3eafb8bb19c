"""Parity at the workload sizes, through the C ABI.

* CAS(14,14) (11,778,624 determinants): FP64 and mixed sigma of a random unit vector against the
  whole oracle sigma (one oracle sigma, about half a minute on one core).
* CAS(16,16) (165,636,900 determinants, the headline workload's integrals): FP64 and mixed sigma
  of a random unit vector, checked on 258 rows against the oracle's Slater-rule rows
  (sigma_I = sum_J <I|H|J> C_J over every connected J), plus the mixed sigma against the FP64
  sigma over the whole vector.
* CAS(12,12) with three roots (853,776 determinants): FP64 and mixed Davidson energies against the
  oracle's Davidson-Liu on the same integrals and options (committed fixture, made by
  tests/golden/make_cas12_roots.py).
"""
import json
import os

import numpy as np
import pytest

from forte_b200 import FCISolver, StateInfo, synthetic
from oracle.oracle import Oracle, sigma_rows

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12   # relative to the largest element (whole vector) or row scale (sampled rows)
TOL_MIXED = 2e-5   # 3xTF32 products with FP32 accumulation, relative to the largest element
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def cas14():
    ints = synthetic(14, 42, 1)
    o = Oracle(14, 7, 7)
    o.set_integrals(ints)
    rng = np.random.default_rng(1414)
    c = rng.normal(size=o.ndet)
    c /= np.linalg.norm(c)
    ref = o.sigma(c)
    del o
    return ints, c, ref


@pytest.mark.parametrize("prec,same,tol", [("FP64", "TC", TOL_FP64), ("MIXED", "TC", TOL_MIXED),
                                           ("MIXED", "CUDA_CORES", TOL_MIXED)])
def test_cas14_sigma_matches_oracle(cas14, prec, same, tol):
    ints, c, ref = cas14
    s = FCISolver(StateInfo(7, 7, 0), 1, ints, {"FCI_PRECISION": prec, "FCI_SAME_SPIN": same})
    got = s.sigma(c)
    err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    assert err < tol, err


@pytest.fixture(scope="module")
def cas16():
    ints = synthetic(16, 48, 1, gap=0.3)
    s = FCISolver(StateInfo(8, 8, 0), 1, ints)
    N = s.size()
    assert N == 165636900
    rng = np.random.default_rng(1616)
    c = rng.standard_normal(N)
    c /= np.linalg.norm(c)
    rows = np.concatenate([[0, 1, N - 2, N - 1], np.sort(rng.choice(N, 254, replace=False))]).astype(np.int64)
    ref, scale = sigma_rows(ints, 8, 8, c, rows)
    fp64 = s.sigma(c)
    return ints, c, rows, ref, scale, fp64


def test_cas16_fp64_sigma_rows(cas16):
    ints, c, rows, ref, scale, fp64 = cas16
    err = np.max(np.abs(fp64[rows] - ref)) / np.max(scale)
    assert err < TOL_FP64, err
    # the rows are not trivially small: every one has many connected contributions
    assert np.min(scale) > 0.0


@pytest.mark.parametrize("mode", ["MIXED", "MIXED_CUDA_CORES"])
def test_cas16_mixed_sigma(cas16, mode):
    ints, c, rows, ref, scale, fp64 = cas16
    opts = {"FCI_PRECISION": "MIXED", "FCI_SAME_SPIN": "CUDA_CORES" if mode.endswith("CORES") else "TC"}
    s = FCISolver(StateInfo(8, 8, 0), 1, ints, opts)
    got = s.sigma(c)
    big = np.max(np.abs(fp64))
    assert np.max(np.abs(got[rows] - ref)) / big < TOL_MIXED
    assert np.max(np.abs(got - fp64)) / big < TOL_MIXED


def _cas12_fixture():
    with open(os.path.join(HERE, "golden", "cas12_roots.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("prec,tol", [("FP64", 1e-10), ("MIXED", 1e-8)])
def test_cas12_three_roots_match_oracle_davidson(prec, tol):
    g = _cas12_fixture()
    ints = synthetic(g["n"], g["L"], g["seed"])
    opts = dict(g["options"], FCI_PRECISION=prec)
    s = FCISolver(StateInfo(g["na"], g["nb"], 0), g["nroot"], ints, opts)
    s.compute_energy()
    assert np.max(np.abs(np.array(s.energies()) - np.array(g["energies"]))) < tol
