"""ctypes wrapper around liboracle.so -- the CPU ORACLE (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs may import this module.  It is the
parity checker for the CUDA engine, never part of the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        vp = C.c_void_p
        dp = C.POINTER(C.c_double)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_int]
        L.orc_destroy.argtypes = [vp]
        L.orc_ndet.restype = C.c_int64
        L.orc_ndet.argtypes = [vp]
        L.orc_nstr.restype = C.c_int64
        L.orc_nstr.argtypes = [vp, C.c_int]
        L.orc_strings.argtypes = [vp, C.c_int, C.POINTER(C.c_uint64)]
        L.orc_mask.argtypes = [vp, C.POINTER(C.c_uint8)]
        L.orc_num_strings.restype = C.c_int64
        L.orc_make_strings.restype = C.c_int64
        L.orc_make_strings.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_uint64)]
        L.orc_list_len.restype = C.c_int64
        L.orc_list_len.argtypes = [vp] + [C.c_int] * 6
        L.orc_list_get.argtypes = [vp] + [C.c_int] * 6 + [dp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.orc_set_integrals.argtypes = [vp, C.c_double, dp, dp, dp, dp, dp]
        L.orc_sigma.argtypes = [vp, dp, dp]
        L.orc_sigma_terms.argtypes = [vp, dp, dp, C.c_int]
        L.orc_hdiag.argtypes = [vp, dp]
        L.orc_slater_rules.restype = C.c_double
        L.orc_slater_rules.argtypes = [vp, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64]
        L.orc_det_spin2.restype = C.c_double
        L.orc_det_spin2.argtypes = [C.c_uint64] * 4 + [C.c_int]
        L.orc_jacobi.argtypes = [C.c_int, dp, dp, dp]
        L.orc_solve.argtypes = [vp, C.POINTER(C.c_int), dp, dp, dp, C.POINTER(C.c_int)]
        L.orc_spin2.restype = C.c_double
        L.orc_spin2.argtypes = [vp, dp]
        L.orc_rdms.argtypes = [vp, dp, dp, C.c_int, dp, dp, dp, dp, dp]
        L.orc_sigma_rows.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, dp, dp, dp, dp, dp, dp, C.c_int64,
                                     C.POINTER(C.c_int64), dp, dp]
        L.orc_rdms3.argtypes = [vp, dp, dp, dp, dp, dp, dp]
        L.orc_last_error.restype = C.c_char_p
        _LIB = L
    return _LIB


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def make_strings(n: int, k: int) -> np.ndarray:
    L = lib()
    cnt = L.orc_num_strings(n, k)
    out = np.zeros(max(cnt, 1), dtype=np.uint64)
    L.orc_make_strings(n, k, out.ctypes.data_as(C.POINTER(C.c_uint64)))
    return out[:cnt]


class Oracle:
    """Forte FCI restated on the CPU for one (n, na, nb, symmetry) problem."""

    def __init__(self, n, na, nb, orbsym=None, irrep=0):
        L = lib()
        self.n, self.na, self.nb = n, na, nb
        osym = (C.c_int * n)(*(orbsym if orbsym is not None else [0] * n))
        self.h = L.orc_create(n, na, nb, osym, irrep)
        if not self.h:
            raise RuntimeError(L.orc_last_error().decode())
        self.ndet = L.orc_ndet(self.h)
        self.nas = L.orc_nstr(self.h, 0)
        self.nbs = L.orc_nstr(self.h, 1)

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().orc_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def strings(self, spin):
        out = np.zeros(self.nbs if spin else self.nas, dtype=np.uint64)
        lib().orc_strings(self.h, spin, out.ctypes.data_as(C.POINTER(C.c_uint64)))
        return out

    def mask(self):
        out = np.zeros(self.ndet, dtype=np.uint8)
        lib().orc_mask(self.h, out.ctypes.data_as(C.POINTER(C.c_uint8)))
        return out

    def list(self, spin, kind, p=0, q=0, r=0, s=0):
        L = lib()
        n = L.orc_list_len(self.h, spin, kind, p, q, r, s)
        sign = np.zeros(max(n, 1))
        I = np.zeros(max(n, 1), dtype=np.uint32)
        J = np.zeros(max(n, 1), dtype=np.uint32)
        L.orc_list_get(self.h, spin, kind, p, q, r, s, _dp(sign),
                       I.ctypes.data_as(C.POINTER(C.c_uint32)), J.ctypes.data_as(C.POINTER(C.c_uint32)))
        return sign[:n], I[:n], J[:n]

    def set_integrals(self, ints):
        self.ints = ints
        self._keep = [np.ascontiguousarray(x, dtype=np.float64) for x in
                      (ints.oei_a, ints.oei_b, ints.tei_aa, ints.tei_ab, ints.tei_bb)]
        lib().orc_set_integrals(self.h, float(ints.scalar), *[_dp(x) for x in self._keep])

    def sigma(self, c, terms=63):
        c = np.ascontiguousarray(c, dtype=np.float64)
        s = np.zeros_like(c)
        if lib().orc_sigma_terms(self.h, _dp(c), _dp(s), terms) != 0:
            raise RuntimeError(lib().orc_last_error().decode())
        return s

    def hdiag(self):
        out = np.zeros(self.ndet)
        if lib().orc_hdiag(self.h, _dp(out)) != 0:
            raise RuntimeError(lib().orc_last_error().decode())
        return out

    def slater_rules(self, la, lb, ra, rb):
        return lib().orc_slater_rules(self.h, la, lb, ra, rb)

    def solve(self, nroot=1, maxiter=100, collapse_per_root=2, subspace_per_root=10,
              guess_per_root=1, dets_per_guess=50, multiplicity=1, e_conv=1e-9, r_conv=1e-6):
        io = (C.c_int * 7)(nroot, maxiter, collapse_per_root, subspace_per_root, guess_per_root,
                           dets_per_guess, multiplicity)
        do = np.array([e_conv, r_conv])
        en = np.zeros(nroot)
        ev = np.zeros((nroot, self.ndet))
        it = C.c_int(0)
        ret = lib().orc_solve(self.h, io, _dp(do), _dp(en), _dp(ev), C.byref(it))
        if ret < 0:
            raise RuntimeError(lib().orc_last_error().decode())
        return {"energies": en, "evecs": ev, "converged": bool(ret), "iterations": it.value}

    def spin2(self, c):
        c = np.ascontiguousarray(c, dtype=np.float64)
        return lib().orc_spin2(self.h, _dp(c))

    def rdms(self, cl, cr=None, level=2):
        cl = np.ascontiguousarray(cl, dtype=np.float64)
        cr = cl if cr is None else np.ascontiguousarray(cr, dtype=np.float64)
        n = self.n
        g1a = np.zeros((n, n)); g1b = np.zeros((n, n))
        g2aa = np.zeros((n,) * 4); g2ab = np.zeros((n,) * 4); g2bb = np.zeros((n,) * 4)
        lib().orc_rdms(self.h, _dp(cl), _dp(cr), level, _dp(g1a), _dp(g1b), _dp(g2aa), _dp(g2ab), _dp(g2bb))
        return {"g1a": g1a, "g1b": g1b, "g2aa": g2aa, "g2ab": g2ab, "g2bb": g2bb}

    def rdms3(self, cl, cr=None):
        """3-RDM blocks g3aaa, g3aab, g3abb, g3bbb (n^6 each) in the reference's index order and
        orientation (FCIVector::compute_3rdm_*_same_irrep)."""
        cr = cl if cr is None else cr
        cl = np.ascontiguousarray(cl, dtype=np.float64)
        cr = np.ascontiguousarray(cr, dtype=np.float64)
        n = self.n
        out = {k: np.zeros((n,) * 6) for k in ("g3aaa", "g3aab", "g3abb", "g3bbb")}
        if lib().orc_rdms3(self.h, _dp(cl), _dp(cr), *[_dp(out[k]) for k in ("g3aaa", "g3aab", "g3abb", "g3bbb")]) < 0:
            raise RuntimeError(lib().orc_last_error().decode())
        return out


def sigma_rows(ints, na, nb, c, rows):
    """Rows ``rows`` (C1 determinant indices) of sigma = H c from the Slater rules over each row's
    connected determinants; returns (sigma rows, sum of |H_IJ c_J| per row).  Works at any size the
    vector fits in host memory (no substitution lists)."""
    c = np.ascontiguousarray(c, dtype=np.float64)
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in
            (ints.oei_a, ints.oei_b, ints.tei_aa, ints.tei_ab, ints.tei_bb)]
    out = np.zeros(len(rows))
    aout = np.zeros(len(rows))
    L = lib()
    if L.orc_sigma_rows(int(ints.n), na, nb, float(ints.scalar), *[_dp(x) for x in arrs], _dp(c), len(rows),
                        rows.ctypes.data_as(C.POINTER(C.c_int64)), _dp(out), _dp(aout)) != 0:
        raise RuntimeError(L.orc_last_error().decode())
    return out, aout


def jacobi(A):
    A = np.ascontiguousarray(A, dtype=np.float64)
    n = A.shape[0]
    ev = np.zeros(n)
    V = np.zeros((n, n))
    lib().orc_jacobi(n, _dp(A), _dp(ev), _dp(V))
    return ev, V


def dense_hamiltonian(orc: Oracle):
    """Dense H over the C1 determinant space from slater_rules (tiny cases only)."""
    sa = orc.strings(0)
    sb = orc.strings(1)
    dets = [(int(a), int(b)) for a in sa for b in sb]
    N = len(dets)
    H = np.zeros((N, N))
    for i in range(N):
        for j in range(i, N):
            v = orc.slater_rules(dets[i][0], dets[i][1], dets[j][0], dets[j][1])
            H[i, j] = H[j, i] = v
    H[np.diag_indices(N)] += orc.ints.scalar
    return H
