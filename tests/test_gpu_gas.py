"""GenCISolver: the generalized active space (GAS) -- the determinants whose electrons per orbital
space lie within bounds -- on the engine's masked layouts.  Checked against the GAS oracle (the
reference's determinant order, restated) and the CPU oracle (sigma, diagonal, RDMs, dense
Hamiltonian over the GAS determinants restricted to the target spin)."""
import numpy as np
import pytest

import golden_cases
from forte_b200 import GenCISolver, FCISolver, StateInfo, build, make_active_space_method, synthetic
from oracle import gas_oracle as G
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

D2H8 = [0, 1, 2, 3, 4, 5, 6, 7]
C2V9 = [0, 0, 0, 1, 1, 2, 2, 3, 3]
CS8 = [0, 0, 0, 0, 1, 1, 1, 1]
C2V7 = [0, 0, 1, 2, 3, 3, 0]

# (orbsym, na, nb, irrep, spaces, gas_min, gas_max)
CASES = [
    ([0] * 8, 4, 4, 0, [[0, 1, 2], [3, 4, 5, 6, 7]], [4, 0], [6, 4]),
    (D2H8, 4, 4, 0, [[0, 1, 2, 3], [4, 5, 6, 7]], [5, 0], [8, 3]),
    (C2V9, 4, 3, 2, [[0, 3, 5], [1, 4, 6, 7], [2, 8]], [2, 0, 0], [6, 5, 2]),
    (CS8, 3, 3, 1, [[0, 1, 4], [2, 3, 5, 6, 7]], [3, 0], [6, 3]),
    (C2V7, 0, 3, 1, [[0, 1, 2], [3, 4, 5, 6]], [1, 0], [3, 2]),
    ([0] * 10, 5, 5, 0, [[0, 1], [2, 3, 4], [5, 6, 7], [8, 9]], [3, 2, 0, 0], [4, 6, 4, 1]),
]


@pytest.fixture(scope="module", autouse=True)
def _lib():
    build.build()


def _nirrep(osym):
    m = max(osym)
    return 1 << m.bit_length() if m > 0 else 1


def _setup(case, opts=None, nroot=1, seed=4, mult=None):
    osym, na, nb, irrep, spaces, mn, mx = case
    n = len(osym)
    ints = synthetic(n, 3 * n, seed, orbsym=osym)
    st = StateInfo(na, nb, mult if mult is not None else abs(na - nb) + 1, na - nb, irrep, tuple(mn), tuple(mx))
    s = GenCISolver(st, nroot, ints, spaces, opts or {})
    o = orc.Oracle(n, na, nb, osym, irrep)
    o.set_integrals(ints)
    dets = G.determinants(n, osym, _nirrep(osym), irrep, na, nb, spaces, mn, mx)
    sa = {int(x): i for i, x in enumerate(o.strings(0))}
    sb = {int(x): i for i, x in enumerate(o.strings(1))}
    idx = np.array([sa[a] * o.nbs + sb[b] for a, b in dets], dtype=np.int64)
    return ints, s, o, dets, idx


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("blocked", [True, False])
def test_gas_flat_order_matches_oracle(case, blocked):
    ints, s, o, dets, idx = _setup(case, {"FCI_SYM_BLOCKED": blocked})
    assert s.size() == len(dets)
    a, b = s.determinants()
    assert [(int(x), int(y)) for x, y in zip(a, b)] == dets


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("prec,same,blocked,tol", [("FP64", "TC", True, 1e-12), ("FP64", "TC", False, 1e-12),
                                                   ("MIXED", "TC", True, 2e-5), ("MIXED", "CUDA_CORES", False, 2e-5)])
def test_gas_sigma_matches_oracle(case, prec, same, blocked, tol):
    ints, s, o, dets, idx = _setup(case, {"FCI_PRECISION": prec, "FCI_SAME_SPIN": same, "FCI_SYM_BLOCKED": blocked})
    rng = np.random.default_rng(len(dets))
    for _ in range(2):
        flat = rng.normal(size=len(dets))
        c1 = np.zeros(o.ndet)
        c1[idx] = flat
        ref = o.sigma(c1)[idx]  # P H P restricted to the GAS determinants
        got = s.sigma(flat)
        assert np.max(np.abs(got - ref)) <= tol * max(1.0, np.max(np.abs(ref)))


@pytest.mark.parametrize("case", CASES[:3])
def test_gas_hdiag_and_spin2_match_oracle(case):
    ints, s, o, dets, idx = _setup(case)
    assert np.array_equal(s.hdiag(), o.hdiag()[idx])
    rng = np.random.default_rng(9)
    flat = rng.normal(size=len(dets))
    flat /= np.linalg.norm(flat)
    c1 = np.zeros(o.ndet)
    c1[idx] = flat
    assert abs(s.compute_spin2(flat) - o.spin2(c1)) <= 1e-11


_EIGH = {}


def _gas_sector(key, o, dets, idx, mult, nroot):
    """Lowest nroot energies of the GAS Hamiltonian (columns from the oracle's sigma on unit
    vectors, diagonalized densely; cached per case) among its eigenvectors with <S^2> = S(S+1)."""
    N = len(dets)
    if key not in _EIGH:
        H = np.empty((N, N))
        for j in range(N):
            e = np.zeros(o.ndet)
            e[idx[j]] = 1.0
            H[:, j] = o.sigma(e)[idx]
        _EIGH[key] = np.linalg.eigh(0.5 * (H + H.T))
    w, V = _EIGH[key]
    S = (mult - 1) / 2
    out = []
    for k in range(N):
        c1 = np.zeros(o.ndet)
        c1[idx] = V[:, k]
        if abs(o.spin2(c1) - S * (S + 1)) < 1e-6:
            out.append(w[k])
        if len(out) == nroot:
            break
    return np.array(out)


def _num_csf(dets, mult):
    """CSFs of 2S + 1 = mult over the configurations of the determinants: f(N, S) per
    configuration with N open shells."""
    from math import comb
    S2 = mult - 1
    confs = {(a & b, a ^ b) for a, b in dets}
    tot = 0
    for d, o in confs:
        N = bin(o).count("1")
        if S2 > N or (N - S2) % 2:
            continue
        k = (N - S2) // 2
        tot += comb(N, k) - (comb(N, k - 1) if k >= 1 else 0)
    return tot


@pytest.mark.parametrize("case", [CASES[0], CASES[2], CASES[3], CASES[4]])
@pytest.mark.parametrize("prec,spin_adapt,tol", [("FP64", False, 1e-10), ("MIXED", False, 1e-8),
                                                 ("FP64", True, 1e-10)])
def test_gas_energies_match_dense_sector(case, prec, spin_adapt, tol):
    opts = {"FCI_PRECISION": prec, "E_CONVERGENCE": 1e-12, "R_CONVERGENCE": 1e-7, "CI_SPIN_ADAPT": spin_adapt,
            "DL_MAXITER": 200}
    ints, s, o, dets, idx = _setup(case, opts, nroot=2)
    s.set_die_if_not_converged(True)
    s.compute_energy()
    na, nb = case[1], case[2]
    mult = abs(na - nb) + 1
    ref = _gas_sector(repr(case), o, dets, idx, mult, 2)
    assert np.max(np.abs(np.array(s.energies()) - ref)) <= tol
    S = (mult - 1) / 2
    assert np.max(np.abs(np.array(s.spin2()) - S * (S + 1))) <= 1e-7
    if spin_adapt:
        assert s.ncsf() == _num_csf(dets, mult)


@pytest.mark.parametrize("case", [CASES[1], CASES[2]])
def test_gas_rdms_match_oracle(case):
    ints, s, o, dets, idx = _setup(case, {"E_CONVERGENCE": 1e-12, "R_CONVERGENCE": 1e-8}, nroot=2)
    s.compute_energy()
    v = s.evecs()
    c0 = np.zeros(o.ndet)
    c1 = np.zeros(o.ndet)
    c0[idx], c1[idx] = v[0], v[1]
    for (l, r), (cl, cr) in [((0, 0), (c0, c0)), ((0, 1), (c0, c1))]:
        got = s.rdms([(l, r)], 2)[0]
        ref = o.rdms(cl, cr, 2)
        for name in ("g1a", "g1b", "g2aa", "g2ab", "g2bb"):
            assert np.max(np.abs(getattr(got, name) - ref[name])) <= 1e-9, name


@pytest.mark.parametrize("k", [1, 2, 3])
def test_gas_with_open_bounds_is_fci(k):
    ints, na, nb, irrep, mult, ref = golden_cases.load(k)
    n = ints.n
    spaces = [list(range(n // 2)), list(range(n // 2, n))]
    st = StateInfo(na, nb, mult, na - nb, irrep)
    s = make_active_space_method("GENCI", st, 1, ints, {"E_CONVERGENCE": 1e-12}, gas_spaces=spaces)
    f = FCISolver(st, 1, ints, {"E_CONVERGENCE": 1e-12})
    assert s.size() == f.size()
    assert abs(s.compute_energy() - ref) <= 1e-9
    a, b = s.determinants()
    fa, fb = f.determinants()
    assert set(zip(a.tolist(), b.tolist())) == set(zip(fa.tolist(), fb.tolist()))


def test_gas_golden_lists():
    # tests/pytest/gas/test_lists.py (both cases), on the engine
    for osym, na, nb, spaces, mn, mx, golden in [
        ([0, 1, 1], 2, 2, [[0], [1, 2]], [0, 0], [2, 2], ["220", "202", "2+-", "2-+"]),
        ([0, 0, 1, 2, 2], 3, 3, [[0, 3], [1, 2, 4]], [3, 3], [3, 3],
         ["+-022", "220+-", "+-220", "202+-", "-+022", "220-+", "-+220", "202-+"]),
    ]:
        ints = synthetic(len(osym), 6, 1, orbsym=osym)
        s = GenCISolver(StateInfo(na, nb, 1, 0, 0, tuple(mn), tuple(mx)), 1, ints, spaces)
        a, b = s.determinants()
        assert sorted(zip(a.tolist(), b.tolist())) == sorted(G.det_from_occupation(t) for t in golden)


def test_gas_change_and_clear_rebuilds():
    case = CASES[0]
    opts = {"E_CONVERGENCE": 1e-12, "R_CONVERGENCE": 1e-8}
    ints, s, o, dets, idx = _setup(case, opts)
    e_gas = s.compute_energy()
    f = FCISolver(StateInfo(4, 4, 1), 1, ints, opts)
    e_fci = f.compute_energy()
    assert e_fci < e_gas - 1e-6  # the restricted space lies above
    s.set_gas([])  # back to the full space: a fresh guess, the FCI energy
    assert s.size() == f.size()
    assert abs(s.compute_energy() - e_fci) <= 1e-10
    s.set_gas(case[4], case[5], case[6])
    assert s.size() == len(dets)
    assert abs(s.compute_energy() - e_gas) <= 1e-10


def test_gas_rejects_bad_spaces():
    ints = synthetic(6, 12, 2)
    st = StateInfo(3, 3, 1)
    with pytest.raises(ValueError):
        GenCISolver(st, 1, ints, [[0, 1, 2], [3, 4]])  # orbital 5 in no space
    with pytest.raises(ValueError):
        GenCISolver(st, 1, ints, [[0, 1, 2], [], [3, 4, 5]])
    s = GenCISolver(st, 1, ints, [[0, 1, 2], [3, 4, 5]])
    s.set_gas([[0, 1, 2], [3, 4, 5]], [7, 0], [8, 6])  # no determinant satisfies the bounds
    assert s.size() == 0
    with pytest.raises(RuntimeError, match="dimension zero"):
        s.compute_energy()


def test_gas_rdms3_and_transition_rdm_match_oracle():
    # 3-RDMs of a GAS root and the transition 1-RDM between GAS states of two irreps
    case = CASES[2]
    opts = {"E_CONVERGENCE": 1e-12, "R_CONVERGENCE": 1e-8}
    ints, s, o, dets, idx = _setup(case, opts)
    s.compute_energy()
    c0 = np.zeros(o.ndet)
    c0[idx] = s.evecs()[0]
    got = s.rdms([(0, 0)], 3)[0]
    ref = o.rdms3(c0)
    for name in ("g3aaa", "g3aab", "g3abb", "g3bbb"):
        assert np.max(np.abs(getattr(got, name) - ref[name])) <= 1e-9, name
    osym, na, nb, irrep, spaces, mn, mx = case
    irrep2 = 1
    t = GenCISolver(StateInfo(na, nb, abs(na - nb) + 1, na - nb, irrep2, tuple(mn), tuple(mx)), 1, ints, spaces, opts)
    t.compute_energy()
    dets2 = G.determinants(len(osym), osym, _nirrep(osym), irrep2, na, nb, spaces, mn, mx)
    sa = {int(x): i for i, x in enumerate(o.strings(0))}
    sb = {int(x): i for i, x in enumerate(o.strings(1))}
    cr = np.zeros(o.ndet)
    cr[[sa[a] * o.nbs + sb[b] for a, b in dets2]] = t.evecs()[0]
    tr = s.transition_rdms([(0, 0)], t, 1)[0]
    rt = o.rdms(c0, cr, 1)
    assert max(np.max(np.abs(rt["g1a"])), np.max(np.abs(rt["g1b"]))) > 1e-6
    assert np.max(np.abs(tr.g1a - rt["g1a"])) <= 1e-9
    assert np.max(np.abs(tr.g1b - rt["g1b"])) <= 1e-9


def test_gas_learned_preconditioner_converges_to_the_same_energy():
    case = CASES[0]
    opts = {"E_CONVERGENCE": 1e-11, "R_CONVERGENCE": 1e-7, "DL_MAXITER": 200}
    ints, s, o, dets, idx = _setup(case, opts)
    e = s.compute_energy()
    m = GenCISolver(StateInfo(4, 4, 1, 0, 0, tuple(case[5]), tuple(case[6])), 1, ints, case[4],
                    dict(opts, FCI_PRECONDITIONER="MLP"))
    assert abs(m.compute_energy() - e) <= 1e-9


def test_gas_restart_with_new_integrals_matches_a_fresh_solver():
    # repeated solves restart from the previous roots (here in the GAS flat basis) with the new
    # integrals of a nearby Hamiltonian, as FCISolver keeps its Davidson-Liu solver between calls
    from forte_b200.integrals import ActiveSpaceIntegrals
    case = CASES[0]
    opts = {"E_CONVERGENCE": 1e-12, "R_CONVERGENCE": 1e-8, "DL_MAXITER": 200}
    ints, s, o, dets, idx = _setup(case, opts, nroot=2)
    s.compute_energy()
    h = ints.oei_a + 0.02 * np.eye(ints.n) * np.linspace(-1.0, 1.0, ints.n)
    ints2 = ActiveSpaceIntegrals(ints.n, ints.scalar, h, h, 1.03 * ints.tei_aa, 1.03 * ints.tei_ab,
                                 1.03 * ints.tei_bb, ints.orbsym)
    s.set_integrals(ints2)
    s.compute_energy()
    f = GenCISolver(StateInfo(case[1], case[2], 1, 0, case[3], tuple(case[5]), tuple(case[6])), 2, ints2, case[4],
                    opts)
    f.compute_energy()
    assert np.max(np.abs(np.array(s.energies()) - np.array(f.energies()))) <= 1e-10
    assert s.iterations() < f.iterations()
