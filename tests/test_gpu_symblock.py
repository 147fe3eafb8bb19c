"""The irrep-blocked layout: with point-group symmetry the engine's vectors and sigma cover only the
target irrep's determinants (FCIVector flat order).  Checked against the CPU oracle (sigma on the C1
layout, restricted to the target irrep) and against the engine's masked C1 mode (FCI_SYM_BLOCKED
off), which the blocked mode replaces."""
import ctypes as C

import numpy as np
import pytest

import golden_cases
from forte_b200 import FCISolver, StateInfo, build, capi, synthetic
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

D2H8 = [0, 1, 2, 3, 4, 5, 6, 7]
D2H10 = [0, 0, 1, 2, 3, 4, 5, 6, 7, 3]
C2V9 = [0, 0, 0, 1, 1, 2, 2, 3, 3]
CS8 = [0, 0, 0, 0, 1, 1, 1, 1]
C2V7 = [0, 0, 1, 2, 3, 3, 0]
C2V6 = [0, 1, 2, 3, 0, 1]

# (orbsym, na, nb, target irrep): D2h / C2v / Cs; the folded one-body path (na, nb >= 1), the
# unfolded one (na = 0 or nb = 0), single electrons, a full alpha shell
CASES = [
    (D2H8, 4, 4, 0), (D2H8, 4, 3, 5), (D2H10, 5, 5, 0), (D2H10, 4, 5, 3), (C2V9, 4, 3, 2), (CS8, 3, 3, 1),
    (C2V7, 0, 3, 1), (C2V7, 2, 0, 3), (C2V6, 1, 1, 0), (C2V6, 6, 5, 1), (C2V7, 2, 2, 2),
]


@pytest.fixture(scope="module", autouse=True)
def _lib():
    build.build()


def _irrep(x, osym):
    h = 0
    for i, o in enumerate(osym):
        if (int(x) >> i) & 1:
            h ^= o
    return h


def flat_to_c1_index(s, osym, irrep):
    """C1 position (alpha string * nb_str + beta string) of every FCIVector flat position."""
    sa, sb = s.strings(0), s.strings(1)
    ha = np.array([_irrep(x, osym) for x in sa])
    hb = np.array([_irrep(x, osym) for x in sb])
    nirrep = 1 << (max(osym)).bit_length() if max(osym) > 0 else 1
    idx = []
    for h in range(nirrep):
        cols = np.nonzero(hb == (h ^ irrep))[0]
        for i in np.nonzero(ha == h)[0]:
            idx.append(i * len(sb) + cols)
    return np.concatenate(idx) if idx else np.zeros(0, dtype=np.int64)


def _case(osym, na, nb, irrep, opts, seed=3):
    n = len(osym)
    ints = synthetic(n, 3 * n, seed, orbsym=osym)
    s = FCISolver(StateInfo(na, nb, abs(na - nb) + 1, na - nb, irrep), 1, ints, opts)
    o = Oracle(n, na, nb, osym, irrep)
    o.set_integrals(ints)
    return ints, s, o


@pytest.mark.parametrize("osym,na,nb,irrep", CASES)
@pytest.mark.parametrize("prec,same,tol", [("FP64", "TC", 1e-12), ("MIXED", "TC", 2e-5), ("MIXED", "CUDA_CORES", 2e-5)])
def test_blocked_sigma_matches_oracle(osym, na, nb, irrep, prec, same, tol):
    ints, s, o = _case(osym, na, nb, irrep, {"FCI_PRECISION": prec, "FCI_SAME_SPIN": same})
    idx = flat_to_c1_index(s, osym, irrep)
    assert s.size() == len(idx)
    rng = np.random.default_rng(len(osym) * 1000 + na * 10 + nb)
    for _ in range(2):
        flat = rng.normal(size=len(idx))
        c1 = np.zeros(o.ndet)
        c1[idx] = flat
        ref = o.sigma(c1)
        # nothing leaks outside the target irrep
        mask = np.zeros(o.ndet, dtype=bool)
        mask[idx] = True
        assert np.max(np.abs(ref[~mask]), initial=0.0) <= 1e-12 * max(1.0, np.max(np.abs(ref)))
        got = s.sigma(flat)
        scale = max(1.0, np.max(np.abs(ref)))
        assert np.max(np.abs(got - ref[idx])) <= tol * scale


@pytest.mark.parametrize("osym,na,nb,irrep", [(D2H10, 5, 5, 0), (C2V9, 4, 3, 2), (C2V7, 0, 3, 1)])
def test_blocked_hdiag_and_spin2_match_oracle(osym, na, nb, irrep):
    ints, s, o = _case(osym, na, nb, irrep, {})
    idx = flat_to_c1_index(s, osym, irrep)
    assert np.array_equal(s.hdiag(), o.hdiag()[idx])
    rng = np.random.default_rng(7)
    flat = rng.normal(size=len(idx))
    flat /= np.linalg.norm(flat)
    c1 = np.zeros(o.ndet)
    c1[idx] = flat
    assert abs(s.compute_spin2(flat) - o.spin2(c1)) <= 1e-11


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("prec", ["FP64", "MIXED"])
def test_blocked_solve_equals_masked(k, prec):
    ints, na, nb, irrep, mult, ref = golden_cases.load(k)
    opts = {"E_CONVERGENCE": 1e-12, "R_CONVERGENCE": 1e-8, "FCI_PRECISION": prec}
    state = StateInfo(na, nb, mult, na - nb, irrep)
    b = FCISolver(state, 1, ints, dict(opts, FCI_SYM_BLOCKED=True))
    m = FCISolver(state, 1, ints, dict(opts, FCI_SYM_BLOCKED=False))
    eb, em = b.compute_energy(), m.compute_energy()
    assert abs(eb - ref) <= 1e-9
    assert abs(eb - em) <= 1e-10
    assert b.size() == m.size()
    vb, vm = b.evecs()[0], m.evecs()[0]
    assert min(np.max(np.abs(vb - vm)), np.max(np.abs(vb + vm))) <= 1e-6
    # two valid mixed trajectories agree to the residual threshold, not bit for bit
    rb, rm = b.rdms([(0, 0)], 2)[0], m.rdms([(0, 0)], 2)[0]
    tol = 1e-9 if prec == "FP64" else 1e-7
    for name in ("g1a", "g1b", "g2aa", "g2ab", "g2bb"):
        assert np.max(np.abs(getattr(rb, name) - getattr(rm, name))) <= tol


def test_blocked_three_roots_and_rdms3_equal_masked():
    ints, na, nb, irrep, mult, ref = golden_cases.load(1)
    opts = {"E_CONVERGENCE": 1e-12, "R_CONVERGENCE": 1e-8}
    state = StateInfo(na, nb, mult, 0, irrep)
    b = FCISolver(state, 3, ints, dict(opts, FCI_SYM_BLOCKED=True))
    m = FCISolver(state, 3, ints, dict(opts, FCI_SYM_BLOCKED=False))
    b.compute_energy()
    m.compute_energy()
    assert np.max(np.abs(np.array(b.energies()) - np.array(m.energies()))) <= 1e-10
    rb, rm = b.rdms([(0, 1), (2, 2)], 3)[1], m.rdms([(0, 1), (2, 2)], 3)[1]
    for name in ("g1a", "g2ab", "g3aab", "g3bbb"):
        assert np.max(np.abs(getattr(rb, name) - getattr(rm, name))) <= 1e-9


def test_blocked_spin_adapted_solve_equals_masked():
    ints, na, nb, irrep, mult, ref = golden_cases.load(1)
    opts = {"E_CONVERGENCE": 1e-12, "R_CONVERGENCE": 1e-8, "CI_SPIN_ADAPT": True}
    state = StateInfo(na, nb, mult, na - nb, irrep)
    b = FCISolver(state, 2, ints, dict(opts, FCI_SYM_BLOCKED=True))
    m = FCISolver(state, 2, ints, dict(opts, FCI_SYM_BLOCKED=False))
    b.compute_energy()
    m.compute_energy()
    assert np.max(np.abs(np.array(b.energies()) - np.array(m.energies()))) <= 1e-10
    assert np.max(np.abs(np.array(b.spin2()) - np.array(m.spin2()))) <= 1e-8


def test_blocked_device_entry_points_use_flat_order():
    torch = pytest.importorskip("torch")
    ints, s, o = _case(C2V9, 4, 3, 2, {})
    N = s.size()
    rng = np.random.default_rng(5)
    flat = rng.normal(size=N)
    flat /= np.linalg.norm(flat)
    ref = s.sigma(flat)
    d_b = torch.tensor(flat, dtype=torch.float64, device="cuda")
    d_s = torch.empty_like(d_b)
    L = capi.lib()
    capi.check(L.fcib_sigma_device(s._h, C.c_void_p(d_b.data_ptr()), C.c_void_p(d_s.data_ptr()), capi.PREC_FP64,
                                   None))
    torch.cuda.synchronize()
    assert np.max(np.abs(d_s.cpu().numpy() - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref)))
    s2 = C.c_double()
    capi.check(L.fcib_spin2_device_noalloc(s._h, C.c_void_p(d_b.data_ptr()), C.byref(s2), None))
    assert abs(s2.value - s.compute_spin2(flat)) <= 1e-12


def test_blocked_layout_toggle_rebuilds():
    ints, na, nb, irrep, mult, ref = golden_cases.load(2)
    s = FCISolver(StateInfo(na, nb, mult, na - nb, irrep), 1, ints, {"E_CONVERGENCE": 1e-12})
    e1 = s.compute_energy()
    s.set_options({"FCI_SYM_BLOCKED": False})
    e2 = s.compute_energy()
    s.set_options({"FCI_SYM_BLOCKED": True})
    e3 = s.compute_energy()
    assert abs(e1 - ref) <= 1e-9 and abs(e2 - e1) <= 1e-10 and abs(e3 - e1) <= 1e-10
