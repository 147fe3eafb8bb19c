"""Spin-adaptation couplings (host entry point fcib_csf_coupling, no device needed) checked against
the oracle's determinant S^2 matrix elements (FCIVector::compute_spin2 conventions): the CSFs of a
configuration are orthonormal, their number is the branching-diagram count, and each one is an
eigenvector of S^2 with eigenvalue S(S+1) in this engine's determinant phase convention, also with
doubly occupied orbitals between the open shells.  CPU only."""
import ctypes as C
from math import comb

import numpy as np
import pytest

from forte_b200 import capi
from oracle import oracle as orc


def _coupling(N, twoS, twoMs):
    cap = 1 << 20
    O = np.zeros(cap)
    pats = np.zeros(cap, dtype=np.uint32)
    f, nd = C.c_int(), C.c_int()
    rc = capi.lib().fcib_csf_coupling(N, twoS, twoMs, cap, capi.dptr(O), pats.ctypes.data_as(C.POINTER(C.c_uint32)),
                                       C.byref(f), C.byref(nd))
    assert rc == 0
    return O[: f.value * nd.value].reshape(f.value, nd.value), pats[: nd.value]


def _dets(D, opens, pat):
    a = b = D
    for k, o in enumerate(opens):
        if pat >> k & 1:
            a |= 1 << o
        else:
            b |= 1 << o
    return a, b


@pytest.mark.parametrize("N,twoS,twoMs", [(2, 0, 0), (2, 2, 0), (3, 1, 1), (4, 0, 0), (4, 2, 0), (4, 2, 2),
                                          (5, 1, -1), (5, 3, 1), (6, 0, 0), (6, 2, 0), (6, 4, 2), (7, 1, 1)])
def test_csfs_are_orthonormal_spin_eigenfunctions(N, twoS, twoMs):
    O, pats = _coupling(N, twoS, twoMs)
    f = comb(N, (N - twoS) // 2) - (comb(N, (N - twoS) // 2 - 1) if (N - twoS) // 2 >= 1 else 0)
    assert O.shape[0] == f
    assert np.max(np.abs(O @ O.T - np.eye(f))) < 1e-13
    S = twoS / 2
    L = orc.lib()
    # open shells alone, then with closed shells interleaved (orbitals 1 and 4 doubly occupied)
    for D, opens in ((0, list(range(N))), (0b10010, [o for o in range(N + 3) if o not in (1, 4)][:N])):
        nmo = max(opens + [4]) + 1
        dets = [_dets(D, opens, int(p)) for p in pats]
        S2 = np.array([[L.orc_det_spin2(a, b, c, d, nmo) for (c, d) in dets] for (a, b) in dets])
        assert np.max(np.abs(S2 @ O.T - S * (S + 1) * O.T)) < 1e-12


def test_coupling_rejects_too_many_open_shells():
    f, nd = C.c_int(), C.c_int()
    assert capi.lib().fcib_csf_coupling(25, 1, 1, 0, None, None, C.byref(f), C.byref(nd)) != 0


def _projector(o, twoS):
    """The engine's spin projector restated over the C1 determinant space of the oracle: for every
    configuration (doubly occupied D, open shells O in orbital order) P_conf = O_N^T O_N."""
    n = o.n
    sa, sb = [int(x) for x in o.strings(0)], [int(x) for x in o.strings(1)]
    ia, ib = {s: i for i, s in enumerate(sa)}, {s: i for i, s in enumerate(sb)}
    nb_ = len(sb)
    P = np.zeros((o.ndet, o.ndet))
    na, nb = o.na, o.nb
    for a in sa:
        for b in sb:
            D, Om = a & b, a ^ b
            # visit each configuration once: from its pattern with the lowest alpha mask
            opens = [p for p in range(n) if Om >> p & 1]
            N = len(opens)
            Oc, pats = _coupling(N, twoS, na - nb)
            idx = [ia[x] * nb_ + ib[y] for x, y in (_dets(D, opens, int(p)) for p in pats)]
            if idx[0] != ia[a] * nb_ + ib[b] and min(idx) != ia[a] * nb_ + ib[b]:
                continue
            if Oc.size:
                P[np.ix_(idx, idx)] = Oc.T @ Oc
    return P


@pytest.mark.parametrize("n,na,nb,mult", [(4, 2, 2, 1), (4, 2, 2, 3), (5, 3, 2, 2), (5, 3, 2, 4), (5, 2, 2, 5)])
def test_projector_is_the_spin_sector_projector(n, na, nb, mult):
    o = orc.Oracle(n, na, nb)
    L = orc.lib()
    sa, sb = [int(x) for x in o.strings(0)], [int(x) for x in o.strings(1)]
    dets = [(a, b) for a in sa for b in sb]
    S2 = np.array([[L.orc_det_spin2(a, b, c, d, n) for (c, d) in dets] for (a, b) in dets])
    w, V = np.linalg.eigh(S2)
    S = (mult - 1) / 2
    sel = np.abs(w - S * (S + 1)) < 1e-8
    ref = V[:, sel] @ V[:, sel].T
    assert np.max(np.abs(_projector(o, mult - 1) - ref)) < 1e-12
