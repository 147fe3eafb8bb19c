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
