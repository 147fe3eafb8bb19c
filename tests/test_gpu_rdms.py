"""1- and 2-RDMs of the GPU engine against the CPU oracle (FCIVector::compute_rdms conventions).

Tolerance 1e-9 per element (FP64 path).  Besides element-wise parity: the energy rebuilt from the
spin-dependent RDMs equals the Davidson eigenvalue, and the spin-free sums follow the reference.
"""
import numpy as np
import pytest

import golden_cases
from forte_b200 import FCISolver, StateInfo, synthetic
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
TOL = 1e-9


def _rand_unit(rng, n):
    v = rng.normal(size=n)
    return v / np.linalg.norm(v)


def _max_diff(a, b):
    return float(np.max(np.abs(a - b))) if a.size else 0.0


def _check(eng, ref, tol=TOL):
    for k in ("g1a", "g1b", "g2aa", "g2ab", "g2bb"):
        d = _max_diff(getattr(eng, k), ref[k])
        assert d < tol, (k, d)


def _energy_from_rdms(ints, r):
    e = ints.scalar
    e += np.einsum("pq,pq", ints.oei_a, r.g1a) + np.einsum("pq,pq", ints.oei_b, r.g1b)
    e += 0.25 * np.einsum("pqrs,pqrs", ints.tei_aa, r.g2aa) + 0.25 * np.einsum("pqrs,pqrs", ints.tei_bb, r.g2bb)
    e += np.einsum("pqrs,pqrs", ints.tei_ab, r.g2ab)
    return e


def _flat_to_c1(s, ints, irrep, flat):
    """FCIVector flat order (alpha-irrep blocks) -> C1 row-major layout of the oracle."""
    sa, sb = s.strings(0), s.strings(1)
    osym = ints.orbsym

    def sym(x):
        h = 0
        for i in range(ints.n):
            if (int(x) >> i) & 1:
                h ^= osym[i]
        return h

    ha = np.array([sym(x) for x in sa])
    hb = np.array([sym(x) for x in sb])
    nirrep = max(osym) + 1
    nirrep = 1 << (nirrep - 1).bit_length() if nirrep > 1 else 1
    out = np.zeros(len(sa) * len(sb))
    pos = 0
    for h in range(nirrep):
        cols = np.nonzero(hb == (h ^ irrep))[0]
        for i in np.nonzero(ha == h)[0]:
            out[i * len(sb) + cols] = flat[pos:pos + len(cols)]
            pos += len(cols)
    assert pos == len(flat)
    return out


@pytest.mark.parametrize("n,na,nb", [(6, 3, 3), (7, 3, 2), (8, 4, 4), (6, 1, 0), (5, 0, 2), (6, 6, 6),
                                     (6, 1, 1), (8, 2, 1), (9, 4, 5)])
def test_rdms_random_vectors_match_oracle(n, na, nb):
    ints = synthetic(n, 3 * n, 5)
    s = FCISolver(StateInfo(na, nb, 0), 1, ints)
    o = Oracle(n, na, nb)
    o.set_integrals(ints)
    rng = np.random.default_rng(100 * n + 10 * na + nb)
    left, right = _rand_unit(rng, s.size()), _rand_unit(rng, s.size())
    _check(s.compute_rdms(left, right, 2), o.rdms(left, right, 2))
    _check(s.compute_rdms(left, None, 2), o.rdms(left, left, 2))
    # spin-free sums of FCIVector::compute_rdms
    ref = o.rdms(left, right, 2)
    sf = s.compute_rdms(left, right, 2, "spin_free")
    assert _max_diff(sf.g1, ref["g1a"] + ref["g1b"]) < TOL
    g2 = (ref["g2aa"] + (ref["g2ab"] + ref["g2ab"].transpose(1, 0, 3, 2))) + ref["g2bb"]
    assert _max_diff(sf.g2, g2) < TOL
    # level 1 leaves the two-body blocks out
    r1 = s.compute_rdms(left, right, 1)
    assert r1.g2aa is None and _max_diff(r1.g1a, ref["g1a"]) < TOL


def test_transition_rdms_of_three_roots_and_energies():
    n, na, nb = 8, 4, 4
    ints = synthetic(n, 24, 2)
    s = FCISolver(StateInfo(na, nb, 0), 3, ints, {"E_CONVERGENCE": 1e-12, "R_CONVERGENCE": 1e-8})
    s.compute_energy()
    ev = s.evecs()
    o = Oracle(n, na, nb)
    o.set_integrals(ints)
    pairs = [(0, 0), (0, 1), (1, 0), (2, 2), (1, 2)]
    got = s.rdms(pairs, 2)
    for (l, r), g in zip(pairs, got):
        _check(g, o.rdms(ev[l], ev[r], 2))
    for k in range(3):
        r = s.rdms([(k, k)], 2)[0]
        assert abs(_energy_from_rdms(ints, r) - s.energies()[k]) < 1e-9
        assert abs(np.trace(r.g1a) - na) < 1e-9 and abs(np.trace(r.g1b) - nb) < 1e-9


def test_golden_fcidump1_rdms_with_symmetry():
    ints, na, nb, irrep, mult, ref = golden_cases.load(1)
    s = FCISolver(StateInfo(na, nb, mult, na - nb, irrep), 1, ints, {"E_CONVERGENCE": 1e-12, "R_CONVERGENCE": 1e-8})
    e = s.compute_energy()
    assert abs(e - ref) < 1e-9
    c1 = _flat_to_c1(s, ints, irrep, s.evecs()[0])
    o = Oracle(ints.n, na, nb, ints.orbsym, irrep)
    o.set_integrals(ints)
    r = s.rdms([(0, 0)], 2)[0]
    _check(r, o.rdms(c1, c1, 2))
    assert abs(_energy_from_rdms(ints, r) - e) < 1e-9


def test_rdm_errors_like_reference():
    ints = synthetic(6, 18, 1)
    s = FCISolver(StateInfo(3, 3, 0), 2, ints)
    with pytest.raises(RuntimeError):
        s.rdms([(0, 0)], 2)  # no solution yet
    s.compute_energy()
    with pytest.raises(RuntimeError, match="because nroot = 2"):
        s.rdms([(0, 2)], 2)
    with pytest.raises(RuntimeError):
        s.rdms([(0, 0)], 4)
    empty = s.rdms([(0, 1)], 0)[0]
    assert not hasattr(empty, "g1a")


def test_cas1212_three_roots_mixed_vs_fp64_with_rdms():
    """CAS(12,12), 853,776 determinants, Ms = 0, 3 roots, synthetic integrals L = 36: the mixed
    path matches FP64 within 1e-8 Eh per root; RDMs of each root match the oracle at 1e-9 and
    rebuild the root's energy."""
    n = 12
    ints = synthetic(n, 36, 1)
    opts = {"E_CONVERGENCE": 1e-10, "R_CONVERGENCE": 1e-6, "DL_SUBSPACE_PER_ROOT": 8}
    f = FCISolver(StateInfo(6, 6, 0), 3, ints, dict(opts, FCI_PRECISION="FP64"))
    f.compute_energy()
    m = FCISolver(StateInfo(6, 6, 0), 3, ints, dict(opts, FCI_PRECISION="MIXED"))
    m.compute_energy()
    assert np.max(np.abs(np.array(m.energies()) - np.array(f.energies()))) < 1e-8
    o = Oracle(n, 6, 6)
    o.set_integrals(ints)
    ev = m.evecs()
    for k in range(3):
        r = m.rdms([(k, k)], 2)[0]
        _check(r, o.rdms(ev[k], ev[k], 2))
        assert abs(_energy_from_rdms(ints, r) - m.energies()[k]) < 1e-8
