"""Batched persistent Davidson against per-instance FCISolver solves and the CPU oracle."""
import numpy as np
import pytest

from forte_b200 import FCISolver, StateInfo, synthetic
from forte_b200.batch import BatchSolver
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
OPTS = {"E_CONVERGENCE": 1e-10, "R_CONVERGENCE": 1e-6, "DL_SUBSPACE_PER_ROOT": 8, "DL_COLLAPSE_PER_ROOT": 2,
        "DL_MAXITER": 200}


def _instances(sizes, seed0):
    out = []
    for i, n in enumerate(sizes):
        out.append((synthetic(n, 3 * n, seed0 + i), (n + 1) // 2, n // 2))
    return out


def test_batch_matches_single_instance_solver():
    inst = _instances([6, 8, 7, 6, 9, 10, 7, 8], 500)
    b = BatchSolver(inst, nroot=4, options=OPTS)
    e, it, cv, ms = b.solve()
    assert cv.all(), it
    for i, (ints, na, nb) in enumerate(inst):
        s = FCISolver(StateInfo(na, nb, 0), 4, ints, dict(OPTS, E_CONVERGENCE=1e-12, R_CONVERGENCE=1e-8))
        s.compute_energy()
        ref = np.array(s.energies())
        assert np.max(np.abs(e[i] - ref)) < 1e-8, (i, e[i], ref)
    # the captured graph replays to the same answer
    e2, it2, cv2, _ = b.solve()
    assert np.max(np.abs(e2 - e)) < 1e-12 and cv2.all()


def test_batch_small_instances_match_oracle():
    inst = _instances([6, 6, 7, 5, 4], 900)
    b = BatchSolver(inst, nroot=3, options=OPTS)
    e, it, cv, _ = b.solve()
    assert cv.all()
    for i, (ints, na, nb) in enumerate(inst):
        o = Oracle(ints.n, na, nb)
        o.set_integrals(ints)
        r = o.solve(nroot=3, multiplicity=0, e_conv=1e-12, r_conv=1e-8)
        assert np.max(np.abs(e[i] - np.array(r["energies"]))) < 1e-8


def test_batch_autotuner_keeps_a_valid_shape():
    inst = _instances([8, 7, 9, 6] * 8, 700)
    b = BatchSolver(inst, nroot=4, options=OPTS)
    e0, _, cv0, _ = b.solve()
    t = b.tune()
    assert t["threads"] in (256, 512) and t["ctas_per_sm"] == 1 and t["pair_tile"] in (8, 16, 32)
    assert t["cluster"] in (1, 2, 4)
    assert any(v > 0 for v in t["times_ms"].values())
    e1, _, cv1, _ = b.solve()
    assert cv0.all() and cv1.all() and np.max(np.abs(e1 - e0)) < 1e-8


def test_batch_rejects_unsupported_instances():
    with pytest.raises(RuntimeError):
        BatchSolver([(synthetic(13, 39, 1), 6, 6)], nroot=2, options=OPTS)
    with pytest.raises(RuntimeError):
        BatchSolver([(synthetic(6, 18, 1), 3, 0)], nroot=2, options=OPTS)


@pytest.mark.parametrize("tile_seed", [0, 1])
def test_batch_mixed_precision_matches_fp64(tile_seed):
    """FP32 sigma with FP64 subspace and residuals, then the FP64 restart: the energies agree with the
    FP64 batch and with the single-instance FP64 solver at the mixed tolerance (1e-8 Eh)."""
    inst = _instances([6, 8, 7, 10, 9, 6, 8, 10], 300 + 17 * tile_seed)
    f = BatchSolver(inst, nroot=4, options=dict(OPTS, FCI_PRECISION="FP64"))
    m = BatchSolver(inst, nroot=4, options=dict(OPTS, FCI_PRECISION="MIXED"))
    ef, _, cf, _ = f.solve()
    em, itm, cm, _ = m.solve()
    assert cf.all() and cm.all(), itm
    assert np.max(np.abs(em - ef)) < 1e-8
    for i in (0, 3):
        ints, na, nb = inst[i]
        s = FCISolver(StateInfo(na, nb, 0), 4, ints, dict(OPTS, E_CONVERGENCE=1e-12, R_CONVERGENCE=1e-8))
        s.compute_energy()
        assert np.max(np.abs(em[i] - np.array(s.energies()))) < 1e-8


@pytest.mark.parametrize("cluster,prec", [(2, "FP64"), (2, "MIXED"), (4, "FP64")])
def test_batch_cluster_matches_single_cta(cluster, prec):
    """Instances shared by a thread-block cluster (rows, lines and vector elements split across its
    CTAs, partial sums combined through distributed shared memory) give the single-CTA energies."""
    inst = _instances([10, 6, 9, 7, 8, 5, 10], 1200)
    one = BatchSolver(inst, nroot=4, options=dict(OPTS, FCI_PRECISION=prec))
    many = BatchSolver(inst, nroot=4, options=dict(OPTS, FCI_PRECISION=prec))
    one.set_shape(512, 16, 1)
    many.set_shape(512, 16, cluster)
    e1, it1, c1, _ = one.solve()
    e2, it2, c2, _ = many.solve()
    assert c1.all() and c2.all(), (it1, it2)
    assert np.max(np.abs(e2 - e1)) < 1e-9
    # the graph replays to the same answer
    e3, _, c3, _ = many.solve()
    assert c3.all() and np.max(np.abs(e3 - e2)) < 1e-12
