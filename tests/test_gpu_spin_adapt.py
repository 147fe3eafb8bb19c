"""CI_SPIN_ADAPT: the Davidson solver works in the CSF basis of the state's multiplicity, like the
reference (sigma through P^T H P, CSF diagonal, lowest-CSF guess).  Energies are checked against
the dense Hamiltonian of the oracle restricted to the S^2 = S(S+1) sector, the CSF count against
that sector's dimension, <S^2> of the roots against S(S+1), and the golden C2v singlet; FP64
tolerance 1e-9 Eh, mixed precision 1e-8 Eh."""
import numpy as np
import pytest

import golden_cases
from forte_b200 import FCISolver, StateInfo, synthetic
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
OPTS = {"E_CONVERGENCE": 1e-11, "R_CONVERGENCE": 1e-7, "CI_SPIN_ADAPT": True, "DL_MAXITER": 200}


def _sector(n, na, nb, ints, mult, nroot):
    """(lowest nroot energies, dimension) of the S^2 = S(S+1) sector of the dense Hamiltonian."""
    o = orc.Oracle(n, na, nb)
    o.set_integrals(ints)
    H = orc.dense_hamiltonian(o)
    L = orc.lib()
    dets = [(int(a), int(b)) for a in o.strings(0) for b in o.strings(1)]
    S2 = np.array([[L.orc_det_spin2(a, b, c, d, n) for (c, d) in dets] for (a, b) in dets])
    w, V = np.linalg.eigh(S2)
    S = (mult - 1) / 2
    Q = V[:, np.abs(w - S * (S + 1)) < 1e-8]
    return np.linalg.eigvalsh(Q.T @ H @ Q)[:nroot], Q.shape[1]


def _sector_energies(n, na, nb, ints, mult, nroot):
    return _sector(n, na, nb, ints, mult, nroot)[0]


@pytest.mark.parametrize("n,na,nb,mult", [(6, 3, 3, 1), (6, 3, 3, 3), (6, 3, 3, 5), (7, 4, 3, 2), (7, 4, 3, 4),
                                          (6, 4, 2, 3)])
def test_spin_adapted_roots_match_the_spin_sector(n, na, nb, mult):
    ints = synthetic(n, 3 * n, 12)
    s = FCISolver(StateInfo(na, nb, mult, na - nb), 3, ints, OPTS)
    s.set_die_if_not_converged(True)
    s.compute_energy()
    ref, dim = _sector(n, na, nb, ints, mult, 3)
    assert s.ncsf() == dim
    assert np.max(np.abs(np.array(s.energies()) - ref)) < 1e-9
    S = (mult - 1) / 2
    assert np.max(np.abs(np.array(s.spin2()) - S * (S + 1))) < 1e-8


def test_spin_adapted_golden_c2v_singlet():
    ints, na, nb, irrep, mult, ref = golden_cases.load(1)
    s = FCISolver(StateInfo(na, nb, mult, na - nb, irrep), 1, ints, dict(OPTS, E_CONVERGENCE=1e-12))
    assert abs(s.compute_energy() - ref) < 1e-9
    assert abs(s.spin2()[0]) < 1e-8


def test_spin_adapted_mixed_precision_matches_fp64():
    ints = synthetic(8, 24, 5)
    st = StateInfo(4, 4, 1)
    opts = dict(OPTS, E_CONVERGENCE=1e-10, R_CONVERGENCE=1e-6)
    f = FCISolver(st, 2, ints, opts)
    f.compute_energy()
    m = FCISolver(st, 2, ints, dict(opts, FCI_PRECISION="MIXED"))
    m.compute_energy()
    assert np.max(np.abs(np.array(m.energies()) - np.array(f.energies()))) < 1e-8
    assert max(abs(x) for x in m.spin2()) < 1e-7


def test_spin_adaptation_needs_a_multiplicity():
    ints = synthetic(6, 18, 1)
    s = FCISolver(StateInfo(3, 3, 0), 1, ints, OPTS)
    with pytest.raises(RuntimeError, match="multiplicity"):
        s.compute_energy()


def _flat_index(s, osym, irrep):
    """C1 position of every FCIVector flat position (C1 cases: the identity)."""
    sa, sb = s.strings(0), s.strings(1)
    if not osym:
        return np.arange(len(sa) * len(sb))

    def irr(x):
        h = 0
        for i, o in enumerate(osym):
            if (int(x) >> i) & 1:
                h ^= o
        return h

    ha, hb = np.array([irr(x) for x in sa]), np.array([irr(x) for x in sb])
    nirrep = 1 << max(osym).bit_length()
    return np.concatenate([i * len(sb) + np.nonzero(hb == (h ^ irrep))[0] for h in range(nirrep)
                           for i in np.nonzero(ha == h)[0]])


@pytest.mark.parametrize("n,na,nb,mult,osym,irrep", [(6, 3, 3, 1, None, 0), (6, 3, 3, 3, None, 0),
                                                    (7, 4, 3, 2, None, 0), (6, 3, 3, 1, [0, 1, 2, 3, 0, 1], 1),
                                                    (6, 4, 2, 3, [0, 0, 1, 1, 0, 1], 0)])
def test_csf_transforms_and_diagonals_match_the_dense_hamiltonian(n, na, nb, mult, osym, irrep):
    """csf_C_to_det_C / det_C_to_csf_C are an isometry and its transpose; the CSF diagonal equals
    sum_m O_im^2 H_mm, and the full preconditioner's diagonal equals <CSF_i|H|CSF_i> from the dense
    oracle Hamiltonian (form_Hdiag_csf, fci_solver_initial_guess.cc:111-149)."""
    ints = synthetic(n, 3 * n, 21, orbsym=osym)
    s = FCISolver(StateInfo(na, nb, mult, na - nb, irrep), 1, ints, dict(OPTS))
    nc = s.ncsf()
    P = np.stack([s.csf_to_det(e) for e in np.eye(nc)], axis=1)
    assert np.max(np.abs(P.T @ P - np.eye(nc))) < 1e-12
    z = np.random.default_rng(3).normal(size=nc)
    assert np.max(np.abs(s.det_to_csf(P @ z) - z)) < 1e-12
    o = orc.Oracle(n, na, nb, osym, irrep)
    o.set_integrals(ints)
    idx = _flat_index(s, osym, irrep)
    Hf = orc.dense_hamiltonian(o)[np.ix_(idx, idx)]
    plain = (P ** 2).T @ np.diag(Hf)
    full = np.einsum("mi,mn,ni->i", P, Hf, P)
    assert np.max(np.abs(s.csf_hdiag(False) - plain)) < 1e-10
    assert np.max(np.abs(s.csf_hdiag(True) - full)) < 1e-10


def test_full_preconditioner_converges_to_the_same_roots():
    ints = synthetic(7, 21, 8)
    st = StateInfo(4, 3, 2, 1)
    a = FCISolver(st, 2, ints, dict(OPTS))
    b = FCISolver(st, 2, ints, dict(OPTS, CI_SPIN_ADAPT_FULL_PRECONDITIONER=True))
    a.compute_energy()
    b.compute_energy()
    assert np.max(np.abs(np.array(a.energies()) - np.array(b.energies()))) < 1e-9
