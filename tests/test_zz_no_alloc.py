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


def _noalloc(solver, dev_tensor, stream=None):
    s2 = C.c_double()
    capi.check(capi.lib().fcib_spin2_device_noalloc(solver._h, C.c_void_p(dev_tensor.data_ptr()),
                                                    C.byref(s2), None if stream is None else C.c_void_p(stream)))
    return s2.value


def _c1_from_flat(solver, orbsym, irrep, flat):
    """FCIVector flat order (alpha irrep blocks) -> the engine's C1 layout, zero outside the
    target irrep, as a device vector must be laid out for the *_device entry points."""
    sa = solver.strings(0).astype(np.int64)
    sb = solver.strings(1).astype(np.int64)

    def sym(s):
        h = 0
        for i, o in enumerate(orbsym):
            if (s >> i) & 1:
                h ^= o
        return h

    ha = np.array([sym(int(x)) for x in sa])
    hb = np.array([sym(int(x)) for x in sb])
    full = np.zeros(len(sa) * len(sb))
    pos = 0
    for h in range(8):
        rows = np.nonzero(ha == h)[0]
        cols = np.nonzero(hb == (h ^ irrep))[0]
        for i in rows:
            full[i * len(sb) + cols] = flat[pos:pos + len(cols)]
            pos += len(cols)
    assert pos == len(flat)
    return full


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


def test_noalloc_on_caller_stream():
    """The caller passes the stream that produced the vector (here torch's current stream, a
    non-default one), so the reduction is ordered after the copy that filled it."""
    import torch

    ints = synthetic(8, 24, 5)
    s = FCISolver(StateInfo(4, 4, 0), 1, ints)
    rng = np.random.default_rng(3)
    c = rng.normal(size=s.size())
    c /= np.linalg.norm(c)
    ref = s.compute_spin2(c)
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        d = torch.from_numpy(c).pin_memory().to("cuda", non_blocking=True)
        got = [_noalloc(s, d, torch.cuda.current_stream().cuda_stream) for _ in range(2)]
    assert got == [ref, ref]


def test_noalloc_with_symmetry_golden_c2v():
    """C2v golden CAS (784 determinants in the A1 block): with the blocked layout (the default) the
    device vector is the flat-order vector itself; with FCI_SYM_BLOCKED off it is in the C1 layout
    with zeros outside the target irrep.  Both equal fcib_spin2 on the flat-order vector."""
    import torch

    import golden_cases

    ints, na, nb, irrep, mult, ref_e = golden_cases.load(1)
    for blocked in (True, False):
        s = FCISolver(StateInfo(na, nb, mult, na - nb, irrep), 1, ints, {"FCI_SYM_BLOCKED": blocked})
        s.compute_energy()
        flat = s.evecs()[0]
        assert flat.size == 784
        ref = s.compute_spin2(flat)
        dev = flat if blocked else _c1_from_flat(s, ints.orbsym, irrep, flat)
        d = torch.from_numpy(np.ascontiguousarray(dev)).cuda()
        torch.cuda.synchronize()
        got = [_noalloc(s, d) for _ in range(2)]
        assert got == [ref, ref]
        assert abs(ref - 0.25 * (mult * mult - 1)) < 1e-6