"""fcib_spin2_device_noalloc against fcib_spin2 (same kernels, static scratch instead of buffers).

The no-alloc entry point serves callers that cannot allocate device memory (their own pool owns
the GPU, or an allocation's device sync is not acceptable); its scratch is one static array per
device that every call reuses, so two calls in a row must both match the allocating entry point.
Collected last (file name) so it also runs after every other GPU test in the same process.
"""
import ctypes as C

import numpy as np
import pytest

from forte_b200 import FCISolver, StateInfo, capi, synthetic

pytestmark = pytest.mark.gpu


def _noalloc(solver, dev_tensor):
    s2 = C.c_double()
    capi.check(capi.lib().fcib_spin2_device_noalloc(solver._h, C.c_void_p(dev_tensor.data_ptr()),
                                                    C.byref(s2), None))
    return s2.value


@pytest.mark.parametrize("n,na,nb", [(6, 3, 3), (8, 4, 3), (10, 5, 5)])
def test_noalloc_spin2_matches_twice(n, na, nb):
    import torch

    ints = synthetic(n, 3 * n, 7)
    s = FCISolver(StateInfo(na, nb, 0), 1, ints)
    N = s.size()
    rng = np.random.default_rng(n + na + nb)
    vecs = [rng.normal(size=N) for _ in range(2)]
    for c in vecs:
        c /= np.linalg.norm(c)
    ref = [s.compute_spin2(c) for c in vecs]
    # two calls in a row through the static scratch, each on a different vector
    got = [_noalloc(s, torch.from_numpy(c).cuda()) for c in vecs]
    assert got == ref
    # and the same vector again: the scratch left by the previous call must not leak in
    again = _noalloc(s, torch.from_numpy(vecs[0]).cuda())
    assert again == ref[0]


def test_noalloc_requires_tables():
    import torch

    L = capi.lib()
    h = C.c_void_p()
    capi.check(L.fcib_create(C.byref(h), 0))
    try:
        x = torch.zeros(4, dtype=torch.float64, device="cuda")
        s2 = C.c_double()
        rc = L.fcib_spin2_device_noalloc(h, C.c_void_p(x.data_ptr()), C.byref(s2), None)
        assert rc == capi.FCIB_ERR_STATE
        assert b"string tables" in L.fcib_last_error()
        rc = L.fcib_spin2_device_noalloc(h, None, C.byref(s2), None)
        assert rc == capi.FCIB_ERR_ARG
    finally:
        L.fcib_destroy(h)
