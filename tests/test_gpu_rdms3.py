"""3-RDMs of the GPU engine (max_rdm_level = 3) against the oracle's restatement of
FCIVector::compute_3rdm_*_same_irrep (fci_vector_rdm.cc:395-565), which is pinned by brute force in
tests/test_rdm3_oracle.py.  Tolerance 1e-9 per element (FP64).  Also: the spin-free G3 sum of
fci_vector_rdm.cc:127-130, contractions to the 2-RDM, transition pairs and point-group symmetry."""
import numpy as np
import pytest

import golden_cases
from forte_b200 import FCISolver, StateInfo, synthetic
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
TOL = 1e-9
BLOCKS = ("g3aaa", "g3aab", "g3abb", "g3bbb")


def _rand_unit(rng, n):
    v = rng.normal(size=n)
    return v / np.linalg.norm(v)


def _spin_free(r):
    g = r["g3aaa"].copy()
    g += r["g3aab"] + np.einsum("prqsut->pqrstu", r["g3aab"]) + np.einsum("qrptus->pqrstu", r["g3aab"])
    g += r["g3abb"] + np.einsum("qprtsu->pqrstu", r["g3abb"]) + np.einsum("rpqust->pqrstu", r["g3abb"])
    return g + r["g3bbb"]


@pytest.mark.parametrize("n,na,nb", [(6, 3, 3), (7, 3, 2), (6, 2, 4), (7, 4, 3), (8, 4, 4), (6, 1, 2), (5, 3, 0),
                                     (9, 3, 3), (6, 5, 4)])
def test_rdms3_random_vectors_match_oracle(n, na, nb):
    ints = synthetic(n, 3 * n, 8)
    s = FCISolver(StateInfo(na, nb, 0, na - nb), 1, ints)
    o = Oracle(n, na, nb)
    o.set_integrals(ints)
    rng = np.random.default_rng(1000 * n + 10 * na + nb)
    left, right = _rand_unit(rng, s.size()), _rand_unit(rng, s.size())
    for lv, rv in ((left, None), (left, right)):
        got = s.compute_rdms(lv, rv, 3)
        ref = o.rdms3(lv, lv if rv is None else rv)
        for k in BLOCKS:
            d = float(np.max(np.abs(getattr(got, k) - ref[k])))
            assert d < TOL, (k, d)
        sf = s.compute_rdms(lv, rv, 3, "spin_free")
        assert float(np.max(np.abs(sf.g3 - _spin_free(ref)))) < TOL


def test_rdms3_of_solved_roots_contract_to_the_2rdm():
    n, na, nb = 8, 4, 3
    ints = synthetic(n, 24, 4)
    s = FCISolver(StateInfo(na, nb, 0, na - nb), 2, ints, {"E_CONVERGENCE": 1e-12, "R_CONVERGENCE": 1e-8})
    s.compute_energy()
    ev = s.evecs()
    o = Oracle(n, na, nb)
    o.set_integrals(ints)
    for (l, r) in ((0, 0), (1, 1), (0, 1)):
        g = s.rdms([(l, r)], 3)[0]
        ref = o.rdms3(ev[l], ev[r])
        for k in BLOCKS:
            assert float(np.max(np.abs(getattr(g, k) - ref[k]))) < TOL, k
        if l == r:
            # sum_r <a+p a+q a+r a_r a_t a_s> = (N_same - 2) g2, sum over the beta pair = N_beta g2
            assert float(np.max(np.abs(np.einsum("pqrstr->pqst", g.g3aaa) - (na - 2) * g.g2aa))) < TOL
            assert float(np.max(np.abs(np.einsum("pqrstr->pqst", g.g3aab) - nb * g.g2aa))) < TOL
            assert float(np.max(np.abs(np.einsum("pqrstr->pqst", g.g3bbb) - (nb - 2) * g.g2bb))) < TOL


def test_golden_fcidump1_rdms3_with_symmetry():
    from test_gpu_rdms import _flat_to_c1
    ints, na, nb, irrep, mult, ref_e = golden_cases.load(1)
    s = FCISolver(StateInfo(na, nb, mult, na - nb, irrep), 1, ints, {"E_CONVERGENCE": 1e-12, "R_CONVERGENCE": 1e-8})
    assert abs(s.compute_energy() - ref_e) < 1e-9
    c1 = _flat_to_c1(s, ints, irrep, s.evecs()[0])
    o = Oracle(ints.n, na, nb, ints.orbsym, irrep)
    o.set_integrals(ints)
    ref = o.rdms3(c1, c1)
    g = s.rdms([(0, 0)], 3)[0]
    for k in BLOCKS:
        assert float(np.max(np.abs(getattr(g, k) - ref[k]))) < TOL, k
