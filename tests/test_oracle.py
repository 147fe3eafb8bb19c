"""The CPU oracle pinned against the reference's golden vectors and independent checks."""
import itertools

import numpy as np
import pytest

import golden_cases
from forte_b200 import integrals as I
from oracle.oracle import Oracle, dense_hamiltonian, make_strings


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5, 6])
def test_golden_fcidump_energy(k):
    """tests/methods/integrals-fcidump-k: compare_values(reffci, ..., 9)."""
    ints, na, nb, irrep, mult, ref = golden_cases.load(k)
    o = Oracle(ints.n, na, nb, ints.orbsym, irrep)
    o.set_integrals(ints)
    r = o.solve(nroot=1, multiplicity=mult, e_conv=1e-12)
    assert r["converged"]
    assert abs(r["energies"][0] - ref) < 1e-9


def test_golden_fcidump1_block_size():
    ints, na, nb, irrep, mult, ref = golden_cases.load(1)
    o = Oracle(ints.n, na, nb, ints.orbsym, irrep)
    assert int(o.mask().sum()) == 784  # A1 block of the C2v CAS(6,8)


@pytest.mark.parametrize("n,k", [(4, 2), (8, 4), (6, 1), (7, 3), (5, 0), (5, 5)])
def test_string_order(n, k):
    """Strings in std::next_permutation order starting from 0..01..1 (element 0 first)."""
    seqs = sorted(t for t in itertools.product([0, 1], repeat=n) if sum(t) == k)
    expect = [sum(1 << i for i in range(n) if t[i]) for t in seqs]
    got = [int(x) for x in make_strings(n, k)]
    assert got == expect
    if (n, k) == (8, 4):
        assert got[0] == 0b11110000  # string 0 = orbitals 4..7 occupied


def _synthetic(n, na, nb, seed=7):
    ints = I.synthetic(n, L=3 * n, seed=seed)
    o = Oracle(n, na, nb)
    o.set_integrals(ints)
    return ints, o


@pytest.mark.parametrize("n,na,nb", [(5, 2, 2), (6, 3, 2), (6, 1, 3), (5, 3, 0), (4, 4, 2)])
def test_sigma_vs_slater_rules(n, na, nb):
    ints, o = _synthetic(n, na, nb)
    H = dense_hamiltonian(o)
    rng = np.random.default_rng(1)
    c = rng.normal(size=o.ndet)
    assert np.max(np.abs(o.sigma(c) - H @ c)) < 1e-12
    assert np.max(np.abs(o.hdiag() - np.diag(H))) < 1e-12


def test_davidson_vs_eigh():
    """Lowest three eigenvalues of the Ms=0 space (guess without spin selection)."""
    ints, o = _synthetic(6, 3, 3)
    H = dense_hamiltonian(o)
    ev = np.linalg.eigvalsh(H)
    r = o.solve(nroot=3, multiplicity=0, e_conv=1e-12, r_conv=1e-8)
    assert r["converged"]
    assert np.max(np.abs(r["energies"] - ev[:3])) < 1e-10


def _apply(op_list, det, n):
    """Apply a product of (spin-orbital index, create?) ops (rightmost first) to a bit tuple."""
    occ = list(det)
    sign = 1
    for so, create in reversed(op_list):
        if occ[so] == create:
            return 0, None
        sign *= (-1) ** sum(occ[:so])
        occ[so] = 1 if create else 0
    return sign, tuple(occ)


def test_rdms_bruteforce():
    n, na, nb = 4, 2, 1
    ints, o = _synthetic(n, na, nb)
    r = o.solve(nroot=1, multiplicity=2, e_conv=1e-12, r_conv=1e-9)
    c = r["evecs"][0]
    sa, sb = o.strings(0), o.strings(1)
    # determinant -> spin-orbital occupation: alpha orbitals 0..n-1, beta n..2n-1
    dets = {}
    for ia, a in enumerate(sa):
        for ib, b in enumerate(sb):
            occ = tuple([(int(a) >> i) & 1 for i in range(n)] + [(int(b) >> i) & 1 for i in range(n)])
            dets[occ] = c[ia * len(sb) + ib]

    def expval(ops):
        tot = 0.0
        for occ, cv in dets.items():
            s, new = _apply(ops, occ, n)
            if s and new in dets:
                tot += dets[new] * s * cv
        return tot

    g = o.rdms(c, level=2)
    for p in range(n):
        for q in range(n):
            assert abs(g["g1a"][p, q] - expval([(p, 1), (q, 0)])) < 1e-12
            assert abs(g["g1b"][p, q] - expval([(n + p, 1), (n + q, 0)])) < 1e-12
    for p, q, rr, s in itertools.product(range(n), repeat=4):
        assert abs(g["g2aa"][p, q, rr, s] - expval([(p, 1), (q, 1), (s, 0), (rr, 0)])) < 1e-12
        assert abs(g["g2ab"][p, q, rr, s] - expval([(p, 1), (n + q, 1), (n + s, 0), (rr, 0)])) < 1e-12
    # energy from the RDMs reproduces the eigenvalue
    e = ints.scalar + np.sum(ints.oei_a * g["g1a"]) + np.sum(ints.oei_b * g["g1b"])
    e += 0.25 * np.sum(ints.tei_aa * g["g2aa"]) + 0.25 * np.sum(ints.tei_bb * g["g2bb"])
    e += np.sum(ints.tei_ab * g["g2ab"])
    assert abs(e - r["energies"][0]) < 1e-10


@pytest.mark.parametrize("n,na,nb", [(6, 3, 3), (7, 4, 2), (8, 4, 4), (6, 1, 0), (5, 0, 2)])
def test_sigma_rows_equal_list_sigma(n, na, nb):
    """Row-wise Slater-rule sigma (used to check CAS(16,16) rows) against the list-driven oracle
    sigma on every row, with a nonzero scalar energy."""
    from oracle.oracle import sigma_rows

    ints = I.synthetic(n, 3 * n, 11)
    ints.scalar = 0.37
    o = Oracle(n, na, nb)
    o.set_integrals(ints)
    rng = np.random.default_rng(n * 100 + na * 10 + nb)
    c = rng.normal(size=o.ndet)
    full = o.sigma(c)
    rows = np.arange(o.ndet)
    got, scale = sigma_rows(ints, na, nb, c, rows)
    assert np.all(scale >= np.abs(got) - 1e-12)
    np.testing.assert_allclose(got, full, rtol=0, atol=1e-12 * max(1.0, np.abs(full).max()))
