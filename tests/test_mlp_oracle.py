"""The CPU oracle of the learned preconditioner, pinned by finite differences (CPU only)."""
import numpy as np

from oracle import mlp_oracle as M


def test_backprop_matches_finite_differences():
    s = M.random_samples(64, 3)
    w = M.random_weights(5).astype(np.float64)
    loss, g = M.loss_grad(w, s["ea"], s["eb"], s["u"], s["r"], s["tgt"], rounding=False, dtype=np.float64,
                           wgt=s["wgt"])
    rng = np.random.default_rng(0)
    idx = np.concatenate([rng.choice(np.arange(M.OFF_W1, M.OFF_B1), 6), rng.choice(np.arange(M.OFF_W2, M.OFF_B2), 6),
                          rng.choice(np.arange(M.OFF_W3, M.OFF_B3), 6), np.arange(M.OFF_W4, M.OFF_W4 + 4),
                          [M.OFF_B1 + 3, M.OFF_B2 + 5, M.OFF_B3 + 7, M.OFF_B4]])
    h = 1e-6
    for i in idx:
        wp = w.copy(); wp[i] += h
        wm = w.copy(); wm[i] -= h
        lp, _ = M.loss_grad(wp, s["ea"], s["eb"], s["u"], s["r"], s["tgt"], rounding=False, dtype=np.float64,
                           wgt=s["wgt"])
        lm, _ = M.loss_grad(wm, s["ea"], s["eb"], s["u"], s["r"], s["tgt"], rounding=False, dtype=np.float64,
                           wgt=s["wgt"])
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-8, (i, fd, g[i])


def test_bf16_rounding_and_zero_network():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.0], dtype=np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == np.float32(1.0078125)
    assert abs(r[3] - (-3.140625)) < 1e-7
    s = M.random_samples(16, 1)
    f = M.factor(np.zeros(M.NW, np.float32), s["ea"], s["eb"], s["u"], s["r"])
    assert np.all(f == 1.0)  # zero network = the diagonal rule


def test_excitation_window():
    from forte_b200.learned_precond import excitation_window
    # 8 electrons in 16 orbitals: the aufbau string has no excitations
    assert excitation_window(np.array([0xFF], np.uint32), 8)[0] == 0
    # 8 -> orbital 8: hole at 7 (slot 7) and particle at 8 (slot 8)
    assert excitation_window(np.array([0x17F], np.uint32), 8)[0] == (1 << 7) | (1 << 8)
    # 4 electrons: window starts at orbital -4, orbital 0 is slot 4
    assert excitation_window(np.array([0b10111], np.uint32), 4)[0] == (1 << (3 + 4)) | (1 << (4 + 4))
