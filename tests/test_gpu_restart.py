"""Repeated compute_energy on one solver (FCISolver::compute_energy, fci_solver.cc:205-233, and
DavidsonLiuSolver::setup_guesses, davidson_liu_solver.cc:312-316): after the first run the solver
restarts from its previous eigenvectors with the current integrals instead of a fresh guess, unless
the guess space covers the whole determinant space.  The restarted energies must equal those of a
fresh solver on the same integrals (FP64 tolerance 1e-10 Eh; mixed 1e-8 Eh)."""
import numpy as np
import pytest

from forte_b200 import FCISolver, StateInfo, synthetic
from forte_b200.integrals import ActiveSpaceIntegrals

pytestmark = pytest.mark.gpu

OPTS = {"E_CONVERGENCE": 1e-11, "R_CONVERGENCE": 1e-7}


def _perturbed(ints, scale_2e, shift_1e):
    """The same orbital space with rescaled two-electron and shifted one-electron integrals (still
    8-fold symmetric), as in a macro-iteration of an orbital optimisation."""
    h = ints.oei_a + shift_1e * np.eye(ints.n) * np.linspace(-1.0, 1.0, ints.n)
    return ActiveSpaceIntegrals(ints.n, ints.scalar, h, h, scale_2e * ints.tei_aa, scale_2e * ints.tei_ab,
                                scale_2e * ints.tei_bb, ints.orbsym)


@pytest.mark.parametrize("precision,tol,opts", [("FP64", 1e-10, OPTS),
                                                ("MIXED", 1e-8, {"E_CONVERGENCE": 1e-10, "R_CONVERGENCE": 1e-6})])
def test_restart_after_integral_update_matches_fresh_solver(precision, tol, opts):
    n = 10
    a = synthetic(n, 30, 4)
    b = _perturbed(a, 1.03, 0.02)
    opts = dict(opts, FCI_PRECISION=precision, DL_MAXITER=200)
    s = FCISolver(StateInfo(5, 5, 0), 2, a, opts)
    s.compute_energy()
    s.set_integrals(b)
    s.compute_energy()
    restarted, it_restart = s.energies(), s.iterations()
    f = FCISolver(StateInfo(5, 5, 0), 2, b, opts)
    f.compute_energy()
    assert f.iterations() < 200
    assert np.max(np.abs(np.array(restarted) - np.array(f.energies()))) < tol
    assert it_restart < 200
    # starting from the previous eigenvectors of a nearby Hamiltonian saves iterations (FP64; the
    # mixed path's FP32 reductions are not deterministic, so its iteration counts vary by run)
    if precision == "FP64":
        assert it_restart < f.iterations(), (it_restart, f.iterations())


def test_restart_with_unchanged_integrals_converges_at_once():
    n = 8
    ints = synthetic(n, 24, 2)
    s = FCISolver(StateInfo(4, 4, 0), 3, ints, OPTS)
    s.compute_energy()
    e1 = np.array(s.energies())
    s.compute_energy()
    assert np.max(np.abs(np.array(s.energies()) - e1)) < 1e-10
    # the previous eigenvalues are kept as lambda_old, so the first iteration already passes both tests
    assert s.iterations() <= 2


def test_no_restart_when_the_guess_covers_the_space():
    """CAS(4,4): 36 determinants <= 1 guess x 50 determinants, so every run starts from a fresh
    guess and repeats the first run exactly."""
    ints = synthetic(4, 12, 3)
    s = FCISolver(StateInfo(2, 2, 0), 1, ints, OPTS)
    s.compute_energy()
    e1, it1 = s.energies(), s.iterations()
    s.compute_energy()
    assert s.energies() == e1 and s.iterations() == it1


def test_state_change_starts_fresh():
    n = 8
    ints = synthetic(n, 24, 6)
    s = FCISolver(StateInfo(4, 4, 0), 1, ints, OPTS)
    s.compute_energy()
    s.state = StateInfo(4, 3, 0, 1)
    s._push_state()
    e = s.compute_energy()
    f = FCISolver(StateInfo(4, 3, 0, 1), 1, ints, OPTS)
    assert abs(e - f.compute_energy()) < 1e-10
    assert s.iterations() == f.iterations()


def test_reset_guess_repeats_a_fresh_solve():
    ints = synthetic(8, 24, 9)
    s = FCISolver(StateInfo(4, 4, 0), 2, ints, OPTS)
    s.compute_energy()
    e1, it1 = np.array(s.energies()), s.iterations()
    s.reset_guess()
    s.compute_energy()
    assert s.iterations() == it1
    assert np.max(np.abs(np.array(s.energies()) - e1)) < 1e-10
