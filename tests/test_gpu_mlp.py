"""Learned preconditioner on the GPU: inference and training kernels against the CPU oracle,
training reduces the loss, and Davidson with the network converges to the FP64 energy."""
import ctypes as C

import numpy as np
import pytest

from forte_b200 import FCISolver, StateInfo, capi, synthetic
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def _eval(w, s):
    f = np.zeros(len(s["u"]), np.float32)
    capi.check(capi.lib().fcib_mlp_eval(0, len(f), capi.uptr(s["ea"]), capi.uptr(s["eb"]), capi.fptr(s["u"]),
                                        capi.fptr(s["r"]), capi.fptr(w), capi.fptr(f)))
    return f


def _grad(w, s):
    g = np.zeros(M.NW, np.float32)
    loss = C.c_double()
    capi.check(capi.lib().fcib_mlp_grad(0, len(s["u"]), capi.uptr(s["ea"]), capi.uptr(s["eb"]), capi.fptr(s["u"]),
                                        capi.fptr(s["r"]), capi.fptr(s["tgt"]), capi.fptr(s["wgt"]), capi.fptr(w), capi.fptr(g),
                                        C.byref(loss)))
    return loss.value, g


def test_inference_kernel_matches_oracle():
    """mma.sync BF16 inference vs the numpy forward with the same rounding points.  Accumulation
    order can move an activation across a BF16 rounding boundary, so the bound is loose at the
    tail and tight in the median."""
    w = M.random_weights(11)
    s = M.random_samples(5003, 12)  # not a multiple of the 16-row tile
    got = _eval(w, s)
    ref = M.factor(w, s["ea"], s["eb"], s["u"], s["r"])
    d = np.abs(got - ref)
    assert np.median(d) < 1e-5 and np.max(d) < 2e-2, (np.median(d), np.max(d))
    assert np.all(_eval(np.zeros(M.NW, np.float32), s) == 1.0)


def test_gradient_kernel_matches_oracle():
    w = M.random_weights(21)
    s = M.random_samples(3000, 22)
    loss, g = _grad(w, s)
    lref, gref = M.loss_grad(w, s["ea"], s["eb"], s["u"], s["r"], s["tgt"], wgt=s["wgt"])
    assert abs(loss - lref) <= 1e-4 * lref
    assert np.linalg.norm(g - gref) <= 2e-3 * np.linalg.norm(gref), np.linalg.norm(g - gref) / np.linalg.norm(gref)
    for off, end in ((M.OFF_W1, M.OFF_B1), (M.OFF_W2, M.OFF_B2), (M.OFF_W3, M.OFF_B3), (M.OFF_W4, M.OFF_B4)):
        assert np.linalg.norm(g[off:end] - gref[off:end]) <= 5e-3 * np.linalg.norm(gref[off:end]) + 1e-12


def test_training_reduces_loss():
    s = M.random_samples(40000, 31)
    w = np.zeros(M.NW, np.float32)
    l0, _ = _grad(w, s)
    hist = np.zeros(8)
    capi.check(capi.lib().fcib_mlp_train(0, len(s["u"]), capi.uptr(s["ea"]), capi.uptr(s["eb"]), capi.fptr(s["u"]),
                                         capi.fptr(s["r"]), capi.fptr(s["tgt"]), capi.fptr(s["wgt"]), 8, 1024, 2e-3, 5, 1,
                                         capi.fptr(w),
                                         capi.dptr(hist)))
    l1, _ = _grad(w, s)
    assert np.all(np.isfinite(w)) and l1 < 0.5 * l0, (l0, l1, hist)


def test_trained_network_improves_corrections_on_unseen_instance():
    """What the committed network gains: on an instance outside its training set (CAS(10,10),
    seed 4242) the learned corrections are closer in direction to the exact corrections
    -(H - E0)^+ r than the diagonal rule's, measured by the training objective."""
    from forte_b200.learned_precond import generate_samples, load_weights, loss_of
    samples, ncorr, _ = generate_samples([(10, 4242)], per_correction=20000, max_corrections=40, log=lambda *a: None)
    assert ncorr >= 10
    l_diag, _ = loss_of(samples, np.zeros(M.NW, np.float32))
    l_mlp, _ = loss_of(samples, load_weights())
    print(f"direction loss on unseen CAS(10,10): diagonal {l_diag:.4e}, learned {l_mlp:.4e}")
    assert l_mlp < l_diag


def test_davidson_with_learned_preconditioner_reaches_fp64_energy():
    """Same energy as the diagonal preconditioner (every converged energy is certified by the FP64
    sigma); the iteration counts of both are printed -- on these synthetic instances the learned
    factor does not reduce them."""
    ints = synthetic(10, 30, 4242)
    opts = {"E_CONVERGENCE": 1e-10, "R_CONVERGENCE": 1e-6, "DL_SUBSPACE_PER_ROOT": 8, "DL_MAXITER": 300}
    d = FCISolver(StateInfo(5, 5, 0), 1, ints, opts)
    e_diag = d.compute_energy()
    m = FCISolver(StateInfo(5, 5, 0), 1, ints, dict(opts, FCI_PRECONDITIONER="MLP"))
    e_mlp = m.compute_energy()
    assert abs(e_mlp - e_diag) < 1e-8
    mm = FCISolver(StateInfo(5, 5, 0), 1, ints, dict(opts, FCI_PRECONDITIONER="MLP", FCI_PRECISION="MIXED"))
    assert abs(mm.compute_energy() - e_diag) < 1e-8
    assert m.iterations() <= 1.1 * d.iterations() + 2
    print(f"iterations: diagonal {d.iterations()}, learned {m.iterations()}, learned+mixed {mm.iterations()}")


def test_engine_preconditioner_step_matches_sample_kernel():
    """fcib_precondition (engine path: features from the string tables) against the sample-mode
    inference kernel on the same determinants."""
    from forte_b200.learned_precond import det_excitations, load_weights
    ints = synthetic(8, 24, 9)
    s = FCISolver(StateInfo(4, 4, 0), 1, ints)
    w = load_weights()
    s.set_mlp_weights(w)
    s.set_options({"FCI_PRECONDITIONER": "MLP"})
    hd = s.hdiag()
    rng = np.random.default_rng(3)
    r = rng.normal(size=len(hd)) * 10.0 ** rng.uniform(-4, 0, len(hd))
    r[: len(r) // 3] *= 1e-6  # a block of tiny residuals that the skip rule leaves alone
    lam = float(np.min(hd)) - 0.2
    out = np.zeros_like(r)
    capi.check(capi.lib().fcib_precondition(s._h, capi.dptr(r), lam, capi.dptr(out)))
    ea, eb = det_excitations(s, 4, 4)
    smp = {"ea": ea, "eb": eb, "u": (hd - lam).astype(np.float32), "r": (r / np.linalg.norm(r)).astype(np.float32)}
    f = _eval(w, smp)
    t = r / (lam - hd)
    # tiles of 16 determinants whose |t| are all below 1e-4 ||t|| keep the diagonal rule
    tau = np.float32(1e-4 * np.linalg.norm(t))
    pad = (-len(t)) % 16
    small = np.concatenate([np.abs(t) < tau, np.ones(pad, bool)]).reshape(-1, 16).all(axis=1)
    keep = np.repeat(small, 16)[:len(t)]
    expect = np.where(keep, t, t * f)
    assert keep.any() and not keep.all()
    assert np.max(np.abs(out - expect)) <= 1e-3 * np.max(np.abs(t))
