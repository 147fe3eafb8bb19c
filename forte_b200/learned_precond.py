"""Learned Davidson preconditioner: training data, GPU training and the default weights.

The network (kernels in csrc/mlp.cu) rescales each element of the diagonal correction
r_I / (lambda - H_II) by 1 + 0.25 tanh m(x_I).  Its training data comes from the engine's own
Davidson runs:

* seeded synthetic CAS(n,n) instances, n = 8..10, integrals ``synthetic(n, 3n, seed)``
  (alpha electrons ceil(n/2), beta floor(n/2));
* each instance is solved once tightly (E0, x0), then once more with the diagonal
  preconditioner while the engine keeps the residual r and Ritz value lambda of root 0 at
  every iteration (``fcib_set_residual_capture``);
* for each residual the exact correction d = -(H - E0)^+ r (pseudo-inverse on the complement
  of x0; the sign of the diagonal rule) is solved by preconditioned conjugate gradients with
  the engine's FP64 sigma;
* per-determinant samples of a seeded random subset of determinants feed ``fcib_mlp_train``
  (Adam, forward and backward on the GPU).  The objective is the direction of each correction,
  || t (1 + 0.25 tanh m) / ||t|| - d / ||d|| ||^2 with t the diagonal correction, written per
  sample as wgt (t_I/||r|| (1 + 0.25 tanh m) - tgt)^2 with tgt = d_I/||d|| * ||t||/||r|| and
  wgt = (||r|| / ||t||)^2 (features use r_I / ||r||).

``python -m forte_b200.learned_precond`` regenerates ``data/mlp_precond.npz``.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import time

import numpy as np

from . import capi
from .fci_solver import FCISolver, StateInfo
from .integrals import synthetic

WEIGHTS_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "mlp_precond.npz")


def excitation_window(strings: np.ndarray, k: int) -> np.ndarray:
    """Occupation XOR aufbau string of k electrons, orbitals k-8 .. k+7 -> 16 bits."""
    d = strings.astype(np.uint64) ^ np.uint64((1 << k) - 1)
    w = (d >> np.uint64(k - 8)) if k >= 8 else (d << np.uint64(8 - k))
    return (w & np.uint64(0xFFFF)).astype(np.uint32)


def det_excitations(solver: FCISolver, na: int, nb: int):
    """Excitation-window bits of every determinant of a C1 space (row-major alpha x beta)."""
    sa, sb = solver.strings(0), solver.strings(1)
    return np.repeat(excitation_window(sa, na), len(sb)), np.tile(excitation_window(sb, nb), len(sa))


def exact_correction(solver: FCISolver, x0: np.ndarray, e0: float, r: np.ndarray, hd: np.ndarray,
                     tol: float = 1e-9, maxit: int = 2000):
    """d = -(H - E0)^+ r on the complement of x0, by conjugate gradients preconditioned with
    diag(H - E0), H applied by the engine's FP64 sigma."""
    import torch
    L = capi.lib()
    dev = torch.device("cuda")
    x0t = torch.from_numpy(np.ascontiguousarray(x0)).to(dev)
    dinv = torch.from_numpy(1.0 / np.maximum(hd - e0, 1e-3)).to(dev)

    def proj(v):
        return v - (x0t @ v) * x0t

    def apply_a(v):
        out = torch.empty_like(v)
        torch.cuda.synchronize()
        capi.check(L.fcib_sigma_device(solver._h, C.c_void_p(v.data_ptr()), C.c_void_p(out.data_ptr()),
                                       capi.PREC_FP64, None))
        return proj(out - e0 * v)

    b = proj(-torch.from_numpy(np.ascontiguousarray(r)).to(dev))
    x = torch.zeros_like(b)
    res = b.clone()
    z = proj(res * dinv)
    p = z.clone()
    rz = res @ z
    bn = float(b.norm())
    it = 0
    for it in range(maxit):
        ap = apply_a(p)
        alpha = rz / (p @ ap)
        x += alpha * p
        res -= alpha * ap
        if float(res.norm()) < tol * bn:
            break
        z = proj(res * dinv)
        rz_new = res @ z
        p = z + (rz_new / rz) * p
        rz = rz_new
    return x.cpu().numpy(), it + 1


def default_instances(count: int = 90, first_seed: int = 1000):
    return [(8 + i % 3, first_seed + i) for i in range(count)]


def generate_samples(instances, per_correction=8192, max_corrections=2000, seed=0, log=print):
    """Training samples from the engine's own Davidson residuals (see the module docstring)."""
    L = capi.lib()
    rng = np.random.default_rng(seed)
    cols = {k: [] for k in ("ea", "eb", "u", "r", "tgt", "wgt")}
    ncorr = 0
    cg_iters = []
    for (n, s) in instances:
        if ncorr >= max_corrections:
            break
        na, nb = (n + 1) // 2, n // 2
        ints = synthetic(n, 3 * n, s)
        ex = FCISolver(StateInfo(na, nb, 0), 1, ints, {"E_CONVERGENCE": 1e-12, "R_CONVERGENCE": 1e-9,
                                                      "DL_MAXITER": 400})
        e0 = ex.compute_energy()
        x0 = ex.evecs()[0]
        hd = ex.hdiag()
        ea_all, eb_all = det_excitations(ex, na, nb)
        dv = FCISolver(StateInfo(na, nb, 0), 1, ints, {"E_CONVERGENCE": 1e-10, "R_CONVERGENCE": 1e-6,
                                                      "DL_SUBSPACE_PER_ROOT": 8, "DL_MAXITER": 400})
        capi.check(L.fcib_set_residual_capture(dv._h, 400))
        dv.compute_energy()
        cnt = C.c_int()
        capi.check(L.fcib_captured_residual(dv._h, -1, None, None, C.byref(cnt)))
        N = len(hd)
        r = np.zeros(N)
        lam = C.c_double()
        for i in range(cnt.value):
            if ncorr >= max_corrections:
                break
            capi.check(L.fcib_captured_residual(dv._h, i, capi.dptr(r), C.byref(lam), None))
            rn = float(np.linalg.norm(r))
            if rn < 1e-12:
                continue
            d, its = exact_correction(ex, x0, e0, r, hd)
            cg_iters.append(its)
            den = lam.value - hd
            t_full = np.where(np.abs(den) > 1e-6, r / np.where(np.abs(den) > 1e-6, den, 1.0), 0.0)
            tn, dn = float(np.linalg.norm(t_full)), float(np.linalg.norm(d))
            if tn < 1e-300 or dn < 1e-300:
                continue
            pick = np.sort(rng.choice(N, size=min(per_correction, N), replace=False))
            cols["ea"].append(ea_all[pick])
            cols["eb"].append(eb_all[pick])
            cols["u"].append((hd[pick] - lam.value).astype(np.float32))
            cols["r"].append((r[pick] / rn).astype(np.float32))
            cols["tgt"].append((d[pick] / dn * (tn / rn)).astype(np.float32))
            cols["wgt"].append(np.full(len(pick), (rn / tn) ** 2, dtype=np.float32))
            ncorr += 1
        log(f"  CAS({n},{n}) seed {s}: {cnt.value} residuals, {ncorr} corrections so far")
        del ex, dv
    out = {k: np.ascontiguousarray(np.concatenate(v)) for k, v in cols.items()}
    return out, ncorr, cg_iters


def train(samples, epochs=6, batch=4096, lr=1e-3, seed=7, weights=None, device=0):
    w = np.zeros(capi.MLP_NWEIGHTS, dtype=np.float32) if weights is None else np.array(weights, dtype=np.float32)
    loss = np.zeros(epochs)
    n = len(samples["u"])
    capi.check(capi.lib().fcib_mlp_train(device, n, capi.uptr(samples["ea"]), capi.uptr(samples["eb"]),
                                         capi.fptr(samples["u"]), capi.fptr(samples["r"]), capi.fptr(samples["tgt"]),
                                         capi.fptr(samples["wgt"]), epochs, batch, lr, seed, 1 if weights is None else 0, capi.fptr(w),
                                         capi.dptr(loss)))
    return w, loss


def loss_of(samples, w, device=0):
    g = np.zeros(capi.MLP_NWEIGHTS, dtype=np.float32)
    loss = C.c_double()
    capi.check(capi.lib().fcib_mlp_grad(device, len(samples["u"]), capi.uptr(samples["ea"]), capi.uptr(samples["eb"]),
                                        capi.fptr(samples["u"]), capi.fptr(samples["r"]), capi.fptr(samples["tgt"]),
                                        capi.fptr(samples["wgt"]), capi.fptr(np.ascontiguousarray(w, dtype=np.float32)),
                                        capi.fptr(g),
                                        C.byref(loss)))
    return loss.value, g


def load_weights(path: str = WEIGHTS_PATH) -> np.ndarray:
    with np.load(path) as f:
        return np.ascontiguousarray(f["weights"], dtype=np.float32)


def main():
    ap = argparse.ArgumentParser(description="regenerate the learned-preconditioner weights")
    ap.add_argument("--corrections", type=int, default=2000)
    ap.add_argument("--per-correction", type=int, default=8192)
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--out", default=WEIGHTS_PATH)
    args = ap.parse_args()
    from . import build
    build.build()
    t0 = time.time()
    samples, ncorr, cg = generate_samples(default_instances(), args.per_correction, args.corrections)
    t1 = time.time()
    zero_loss, _ = loss_of(samples, np.zeros(capi.MLP_NWEIGHTS, dtype=np.float32))
    w, losses = train(samples, args.epochs, args.batch, args.lr)
    final_loss, _ = loss_of(samples, w)
    t2 = time.time()
    meta = {"corrections": ncorr, "samples": int(len(samples["u"])), "cg_iterations_mean": float(np.mean(cg)),
            "epochs": args.epochs, "batch": args.batch, "lr": args.lr, "epoch_loss": [float(x) for x in losses],
            "loss_diagonal_rule": zero_loss, "loss_trained": final_loss,
            "data_seconds": t1 - t0, "train_seconds": t2 - t1}
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    np.savez(args.out, weights=w, meta=json.dumps(meta))
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
