"""Batched CASCI: many independent small instances solved in one persistent GPU launch.

Mirrors what a caller of Forte would do with one FCISolver per instance (same options and
integral layouts), but the engine runs every instance's Davidson-Liu on the device at once
(``fcib_batch_*``; kernel ``k_batch_dl`` in csrc/batch.cu).  No spin selection: the lowest
``nroot`` eigenvalues of each instance's determinant space (Ms = (na - nb)/2, C1).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .fci_solver import DEFAULT_OPTIONS


class BatchSolver:
    def __init__(self, instances, nroot=4, options=None, device=0):
        """instances: list of (ActiveSpaceIntegrals, na, nb)."""
        L = capi.lib()
        opts = dict(DEFAULT_OPTIONS)
        opts.update({k.upper(): v for k, v in (options or {}).items()})
        o = capi.default_options()
        o.maxiter = int(opts["DL_MAXITER"])
        o.e_convergence = float(opts["E_CONVERGENCE"])
        o.r_convergence = float(opts["R_CONVERGENCE"])
        o.subspace_per_root = int(opts["DL_SUBSPACE_PER_ROOT"])
        o.collapse_per_root = int(opts["DL_COLLAPSE_PER_ROOT"])
        o.precision = capi.PREC_FP64 if str(opts.get("FCI_PRECISION", "FP64")).upper() == "FP64" else capi.PREC_MIXED
        self.ninst = len(instances)
        self.nroot = nroot
        k = self.ninst
        self._keep = []
        arrs = {name: (C.POINTER(C.c_double) * k)() for name in ("oei_a", "oei_b", "tei_aa", "tei_ab", "tei_bb")}
        n = (C.c_int * k)()
        na = (C.c_int * k)()
        nb = (C.c_int * k)()
        sc = np.zeros(k)
        for i, (ints, a, b) in enumerate(instances):
            n[i], na[i], nb[i] = ints.n, a, b
            sc[i] = ints.scalar
            for name in arrs:
                x = np.ascontiguousarray(getattr(ints, name), dtype=np.float64)
                self._keep.append(x)
                arrs[name][i] = capi.dptr(x)
        h = C.c_void_p()
        capi.check(L.fcib_batch_create(C.byref(h), device, k, n, na, nb, capi.dptr(sc), arrs["oei_a"], arrs["oei_b"],
                                       arrs["tei_aa"], arrs["tei_ab"], arrs["tei_bb"], nroot, C.byref(o)))
        self._h = h
        self._keep = None

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                capi.lib().fcib_batch_destroy(self._h)
                self._h = None
        except Exception:
            pass

    def solve(self):
        """Returns (energies [ninst, nroot], iterations [ninst], converged [ninst], device ms)."""
        e = np.zeros((self.ninst, self.nroot))
        it = np.zeros(self.ninst, dtype=np.int32)
        cv = np.zeros(self.ninst, dtype=np.int32)
        ms = C.c_double()
        capi.check(capi.lib().fcib_batch_solve(self._h, capi.dptr(e), it.ctypes.data_as(C.POINTER(C.c_int)),
                                               cv.ctypes.data_as(C.POINTER(C.c_int)), C.byref(ms)))
        return e, it, cv.astype(bool), ms.value

    def set_shape(self, threads=512, pair_tile=32, cluster=2):
        """Launch shape of later solves: threads per CTA, opposite-spin sigma tile, CTAs per instance."""
        capi.check(capi.lib().fcib_batch_set_shape(self._h, threads, pair_tile, cluster))

    def tune(self):
        """Autotuner: opposite-spin sigma tile (pairs per work item) x launch shape (threads per CTA x
        CTAs per instance, a thread-block cluster); keeps the fastest."""
        t = C.c_int()
        c = C.c_int()
        p = C.c_int()
        cl = C.c_int()
        times = np.zeros(12)
        capi.check(capi.lib().fcib_batch_tune(self._h, C.byref(t), C.byref(c), C.byref(p), C.byref(cl),
                                              capi.dptr(times)))
        names = [f"tile{tile}_{shape}" for tile in (8, 16, 32) for shape in ("512x1", "256x2", "512x2", "512x4")]
        return {"threads": t.value, "ctas_per_sm": c.value, "pair_tile": p.value, "cluster": cl.value,
                "times_ms": dict(zip(names, times.tolist()))}
