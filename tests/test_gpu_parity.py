"""Parity of the CUDA engine (through the C ABI) with the CPU oracle and the golden vectors."""
import numpy as np
import pytest

import golden_cases
from forte_b200 import FCISolver, StateInfo, build, synthetic
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib():
    build.build()


def _pair(n, na, nb, seed=11, L=None, mult=1):
    ints = synthetic(n, L or 3 * n, seed)
    o = Oracle(n, na, nb)
    o.set_integrals(ints)
    s = FCISolver(StateInfo(na, nb, mult, na - nb), 1, ints)
    return ints, o, s


@pytest.mark.parametrize("n,na,nb", [(6, 3, 3), (8, 4, 4), (7, 4, 2), (10, 3, 5), (12, 6, 6), (5, 5, 0), (4, 0, 2), (6, 1, 1)])
def test_strings_bit_exact(n, na, nb):
    ints, o, s = _pair(n, na, nb)
    assert np.array_equal(s.strings(0).astype(np.uint64), o.strings(0))
    assert np.array_equal(s.strings(1).astype(np.uint64), o.strings(1))


@pytest.mark.parametrize("n,k", [(6, 3), (7, 2), (8, 4), (9, 5)])
def test_substitution_lists_bit_exact(n, k):
    ints, o, s = _pair(n, k, k)
    for spin in (0, 1):
        for p in range(n):
            for q in range(n):
                a = s.string_list(spin, 0, p, q)
                b = o.list(spin, 0, p, q)
                assert np.array_equal(a[0], b[0].astype(np.int8)) and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
        for pq in range(n * (n - 1) // 2):
            a = s.string_list(spin, 1, pq)
            b = o.list(spin, 1, pq)
            assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]) and np.all(a[0] == 1)
        for p in range(n):
            for q in range(p):
                for r in range(n):
                    for t in range(r):
                        if (p, q) == (r, t):
                            continue
                        a = s.string_list(spin, 2, p, q, r, t)
                        b = o.list(spin, 2, p, q, r, t)
                        assert np.array_equal(a[0], b[0].astype(np.int8)), (p, q, r, t)
                        assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])


@pytest.mark.parametrize("n,na,nb", [(8, 4, 4), (9, 5, 3), (12, 6, 6)])
def test_hdiag_bit_exact(n, na, nb):
    ints, o, s = _pair(n, na, nb)
    assert np.array_equal(s.hdiag(), o.hdiag())


@pytest.mark.parametrize("n,na,nb", [(4, 2, 2), (6, 3, 3), (8, 4, 4), (7, 4, 2), (9, 3, 5), (6, 1, 1), (5, 2, 0),
                                     (6, 0, 3), (5, 1, 0), (10, 5, 5), (12, 6, 6), (6, 6, 6), (7, 6, 5)])
def test_sigma_matches_oracle(n, na, nb):
    ints, o, s = _pair(n, na, nb)
    rng = np.random.default_rng(n * 100 + na * 10 + nb)
    for _ in range(2):
        c = rng.normal(size=o.ndet)
        ref = o.sigma(c)
        got = s.sigma(c)
        scale = max(1.0, np.max(np.abs(ref)))
        assert np.max(np.abs(got - ref)) <= 1e-12 * scale


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5, 6])
def test_golden_fcidump_energies(k):
    ints, na, nb, irrep, mult, ref = golden_cases.load(k)
    s = FCISolver(StateInfo(na, nb, mult, na - nb, irrep), 1, ints, {"E_CONVERGENCE": 1e-12})
    e = s.compute_energy()
    assert abs(e - ref) < 1e-9
    o = Oracle(ints.n, na, nb, ints.orbsym, irrep)
    o.set_integrals(ints)
    r = o.solve(nroot=1, multiplicity=mult, e_conv=1e-12)
    assert abs(e - r["energies"][0]) < 1e-10
    assert abs(s.spin2()[0] - 0.25 * (mult * mult - 1)) < 1e-6


def test_cas88_multiroot_matches_oracle():
    """Config-0-style CAS(8,8), synthetic integrals L=24, three roots.  These integrals have an
    exchange-dominated (high-spin) spectrum, so the guess is not spin-selected
    (multiplicity 0); the roots have S^2 = 20, 12, 6."""
    ints = synthetic(8, 24, 0)
    o = Oracle(8, 4, 4)
    o.set_integrals(ints)
    r = o.solve(nroot=3, multiplicity=0, e_conv=1e-12, r_conv=1e-8)
    assert r["converged"]
    s = FCISolver(StateInfo(4, 4, 0), 3, ints, {"E_CONVERGENCE": 1e-12, "R_CONVERGENCE": 1e-8})
    s.compute_energy()
    assert np.max(np.abs(np.array(s.energies()) - r["energies"])) < 1e-10
    ev = s.evecs()
    for k in range(3):
        ov = abs(np.dot(ev[k], r["evecs"][k]))
        assert abs(ov - 1.0) < 1e-8
        assert abs(s.spin2()[k] - o.spin2(r["evecs"][k])) < 1e-8


def test_golden_fcidump1_three_roots():
    ints, na, nb, irrep, mult, ref = golden_cases.load(1)
    o = Oracle(ints.n, na, nb, ints.orbsym, irrep)
    o.set_integrals(ints)
    r = o.solve(nroot=3, multiplicity=mult, e_conv=1e-12, r_conv=1e-8)
    s = FCISolver(StateInfo(na, nb, mult, 0, irrep), 3, ints, {"E_CONVERGENCE": 1e-12, "R_CONVERGENCE": 1e-8})
    s.compute_energy()
    assert abs(s.energies()[0] - ref) < 1e-9
    assert np.max(np.abs(np.array(s.energies()) - r["energies"])) < 1e-10
    assert s.evecs().shape == (3, 784)


def test_spin2_matches_oracle():
    ints, o, s = _pair(7, 4, 3, mult=2)
    rng = np.random.default_rng(5)
    c = rng.normal(size=o.ndet)
    c /= np.linalg.norm(c)
    assert abs(s.compute_spin2(c) - o.spin2(c)) < 1e-12


def test_option_errors_like_reference():
    ints = synthetic(6, 18, 1)
    s = FCISolver(StateInfo(3, 3), 1, ints)
    with pytest.raises(RuntimeError):
        s.set_options({"DL_COLLAPSE_PER_ROOT": 0})
    with pytest.raises(RuntimeError):
        s.set_options({"DL_COLLAPSE_PER_ROOT": 3, "DL_SUBSPACE_PER_ROOT": 3})
    with pytest.raises(KeyError):
        s.set_options({"NOT_AN_OPTION": 1})


def test_non_convergence_raises_when_asked():
    ints = synthetic(8, 24, 2)
    s = FCISolver(StateInfo(4, 4), 1, ints, {"DL_MAXITER": 2, "E_CONVERGENCE": 1e-14, "R_CONVERGENCE": 1e-12})
    s.set_die_if_not_converged(True)
    with pytest.raises(RuntimeError):
        s.compute_energy()


def _block_addresses(s, orbsym, irrep):
    """(alpha irrep, alpha address, beta address) of every FCIVector flat position."""
    sa = s.strings(0).astype(np.int64)
    sb = s.strings(1).astype(np.int64)

    def sym(x):
        h = 0
        for i, o in enumerate(orbsym):
            if (x >> i) & 1:
                h ^= o
        return h

    ha = np.array([sym(int(x)) for x in sa])
    hb = np.array([sym(int(x)) for x in sb])
    out = []
    for h in range(8):
        na_h = int(np.sum(ha == h))
        nb_h = int(np.sum(hb == (h ^ irrep)))
        for ia in range(na_h):
            for ib in range(nb_h):
                out.append((h, ia, ib))
    return out


@pytest.mark.parametrize("case", ["golden1", "c1"])
def test_max_abs_elements_reference_order(case, capfd):
    """FCIVector::max_abs_elements: the largest |C| first, equal values in flat order (the reference's
    insertion keeps the first one found), each with its alpha irrep and string addresses; and the
    PRINT >= 1 listing of FCISolver::print_solutions."""
    if case == "golden1":
        ints, na, nb, irrep, mult, ref = golden_cases.load(1)
        state = StateInfo(na, nb, mult, na - nb, irrep)
    else:
        ints = synthetic(8, 24, 2)
        na, nb, irrep = 4, 4, 0
        state = StateInfo(4, 4, 1)
    s = FCISolver(state, 2, ints, {"E_CONVERGENCE": 1e-12, "PRINT": 1})
    s.compute_energy()
    out = capfd.readouterr().out
    assert "==> Root No. 0 <==" in out and "==> Root No. 1 <==" in out and "Total Energy:" in out
    addr = _block_addresses(s, ints.orbsym, irrep if case == "golden1" else 0)
    for root in (0, 1):
        c = s.evecs()[root]
        k = 40
        got = s.max_abs_elements(k, root)
        order = np.argsort(-np.abs(c), kind="stable")[:k]
        assert len(got) == min(k, c.size)
        for t, i in enumerate(order):
            a, v, h, ia, ib = got[t]
            assert a == abs(c[i]) and v == c[i]
            assert (h, ia, ib) == addr[i]


@pytest.mark.parametrize("n,na,nb", [(10, 5, 5), (9, 5, 3), (12, 6, 6), (6, 3, 0)])
def test_fp64_sigma_is_deterministic(n, na, nb):
    """The FP64 sigma sums in 64-bit fixed point (opposite-spin rows in shared memory, same-spin groups
    in global memory) on grids set from max|C|, so repeated builds of one vector are bit-identical."""
    ints = synthetic(n, 3 * n, 9)
    s = FCISolver(StateInfo(na, nb, 0, na - nb), 1, ints)
    rng = np.random.default_rng(n + 3 * na + nb)
    c = rng.normal(size=s.size())
    c /= np.linalg.norm(c)
    first = s.sigma(c)
    for _ in range(3):
        assert np.array_equal(s.sigma(c), first)


@pytest.mark.parametrize("prec", ["FP64", "MIXED"])
def test_solves_repeat_exactly(prec):
    """With every sigma summed in integers, a repeated Davidson solve from a fresh guess takes the
    same iterations to the same energies, bit for bit."""
    ints = synthetic(12, 36, 4)
    s = FCISolver(StateInfo(6, 6, 0), 2, ints, {"FCI_PRECISION": prec, "E_CONVERGENCE": 1e-10,
                                                 "R_CONVERGENCE": 1e-6, "DL_MAXITER": 300})
    s.compute_energy()
    e1, it1 = list(s.energies()), s.iterations()
    s.reset_guess()
    s.compute_energy()
    assert s.iterations() == it1 and list(s.energies()) == e1
