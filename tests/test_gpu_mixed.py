"""Mixed-precision path: tensor-core (tcgen05 kind::tf32) opposite-spin sigma with FP32 same-spin
terms, checked against the FP64 oracle; mixed Davidson energies checked against FP64 ones."""
import numpy as np
import pytest

import golden_cases
from forte_b200 import FCISolver, StateInfo, synthetic
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

# 3xTF32 split products with FP32 accumulation: ~FP32 accuracy of each sigma element relative
# to the largest one; single-pass TF32 keeps ~10 mantissa bits.
TOL_MIXED = 2e-5
TOL_TF32 = 5e-3


@pytest.mark.parametrize("n,na,nb", [(4, 2, 2), (6, 3, 3), (8, 4, 4), (7, 4, 2), (9, 3, 5), (10, 5, 5), (12, 6, 6),
                                     (6, 1, 1), (5, 2, 0)])
@pytest.mark.parametrize("mode,tol", [("MIXED", TOL_MIXED), ("MIXED_TF32", TOL_TF32)])
def test_mixed_sigma_matches_oracle(n, na, nb, mode, tol):
    ints = synthetic(n, 3 * n, 21)
    o = Oracle(n, na, nb)
    o.set_integrals(ints)
    s = FCISolver(StateInfo(na, nb, 0, na - nb), 1, ints, {"FCI_PRECISION": mode})
    rng = np.random.default_rng(7 * n + na)
    c = rng.normal(size=o.ndet)
    c /= np.linalg.norm(c)
    ref = o.sigma(c)
    got = s.sigma(c)
    err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    assert err < tol, err


@pytest.mark.parametrize("n,L", [(8, 24), (10, 30), (12, 36)])
def test_mixed_solve_matches_fp64(n, L):
    """North-star tolerance for mixed mode: 1e-8 Eh against the FP64 energy (one root; with
    several roots and no spin selection, exact FP64 arithmetic never leaves the spin sectors of
    the guess while low-precision noise can, so multi-root parity is checked on a
    symmetry-adapted golden system below)."""
    ints = synthetic(n, L, 3)
    opts = {"E_CONVERGENCE": 1e-10, "R_CONVERGENCE": 1e-6, "DL_MAXITER": 300}
    f = FCISolver(StateInfo(n // 2, n // 2, 0), 1, ints, opts)
    f.compute_energy()
    m = FCISolver(StateInfo(n // 2, n // 2, 0), 1, ints, dict(opts, FCI_PRECISION="MIXED"))
    m.compute_energy()
    assert abs(m.energies()[0] - f.energies()[0]) < 1e-8


def test_mixed_multiroot_golden():
    ints, na, nb, irrep, mult, ref = golden_cases.load(1)
    opts = {"E_CONVERGENCE": 1e-10, "R_CONVERGENCE": 1e-6}
    f = FCISolver(StateInfo(na, nb, mult, 0, irrep), 3, ints, opts)
    f.compute_energy()
    m = FCISolver(StateInfo(na, nb, mult, 0, irrep), 3, ints, dict(opts, FCI_PRECISION="MIXED"))
    m.compute_energy()
    assert np.max(np.abs(np.array(m.energies()) - np.array(f.energies()))) < 1e-8


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5])
def test_mixed_golden_fcidump(k):
    ints, na, nb, irrep, mult, ref = golden_cases.load(k)
    s = FCISolver(StateInfo(na, nb, mult, na - nb, irrep), 1, ints,
                  {"E_CONVERGENCE": 1e-10, "R_CONVERGENCE": 1e-6, "FCI_PRECISION": "MIXED"})
    assert abs(s.compute_energy() - ref) < 1e-8


@pytest.mark.parametrize("n,na,nb,oracle", [(8, 4, 4, True), (9, 3, 5, True), (12, 2, 3, True), (11, 5, 4, True),
                                            (10, 9, 2, True), (14, 7, 7, False)])
def test_same_spin_tensor_cores_match_cuda_cores(n, na, nb, oracle):
    """Mixed sigma with the same-spin groups on the tensor cores (3xTF32, FCI_SAME_SPIN=TC) against
    the FP32 CUDA-core groups and, where the oracle is quick, the FP64 oracle.  Group sizes
    C(n-k+2, 2), alpha / beta: (8,4,4) 15; (9,3,5) 28 / 15; (11,5,4) 28 / 36; (10,9,2) 3 / 45;
    (14,7,7) 36.  In (12,2,3)
    the alpha groups hold C(12,2) = 66 strings, more than the tensor-core layout takes, so that
    spin runs on the CUDA cores while beta (55 strings) runs on the tensor cores."""
    ints = synthetic(n, 3 * n, 23)
    rng = np.random.default_rng(11 * n + nb)
    got = {}
    for kern in ("TC", "CUDA_CORES"):
        s = FCISolver(StateInfo(na, nb, 0, na - nb), 1, ints, {"FCI_PRECISION": "MIXED", "FCI_SAME_SPIN": kern})
        if kern == "TC":
            c = rng.normal(size=s.size())
            c /= np.linalg.norm(c)
        got[kern] = s.sigma(c)
    scale = np.max(np.abs(got["CUDA_CORES"]))
    assert np.max(np.abs(got["TC"] - got["CUDA_CORES"])) / scale < TOL_MIXED
    if oracle:
        o = Oracle(n, na, nb)
        o.set_integrals(ints)
        ref = o.sigma(c)
        assert np.max(np.abs(got["TC"] - ref)) / np.max(np.abs(ref)) < TOL_MIXED


def test_same_spin_kernel_option_is_checked():
    ints = synthetic(6, 18, 1)
    with pytest.raises(KeyError):
        FCISolver(StateInfo(3, 3, 0), 1, ints, {"FCI_SAME_SPIN": "BOTH"})


@pytest.mark.parametrize("same", ["TC", "CUDA_CORES"])
@pytest.mark.parametrize("n,na,nb", [(10, 5, 5), (9, 5, 3), (12, 6, 6)])
def test_mixed_sigma_is_deterministic(n, na, nb, same):
    """The mixed sigma accumulates in integers on a fixed-point grid (opposite-spin scatter in shared
    memory, same-spin groups in global memory), so repeated builds of one vector agree bit for bit."""
    ints = synthetic(n, 3 * n, 5)
    s = FCISolver(StateInfo(na, nb, 0, na - nb), 1, ints, {"FCI_PRECISION": "MIXED", "FCI_SAME_SPIN": same})
    rng = np.random.default_rng(n + na)
    c = rng.normal(size=s.size())
    c /= np.linalg.norm(c)
    first = s.sigma(c)
    for _ in range(3):
        assert np.array_equal(s.sigma(c), first)
