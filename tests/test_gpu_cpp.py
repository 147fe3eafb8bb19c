"""The engine driven from C++ (tests/cpp/fcib_solver_main.cpp through include/fcib_solver.hpp, built
with g++ and linked to libfcib200.so), as a Forte-side adapter would: the golden C2v case
integrals-fcidump-1 (784 determinants in A1) solved to the reference energy, its RDMs equal to the
oracle's, and the transition 1-RDM to a state of another irrep equal to the oracle's."""
import os
import subprocess
import sys

import numpy as np
import pytest

import golden_cases
from oracle.oracle import Oracle

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "cpp"))
pytestmark = pytest.mark.gpu


def _c1(o, orbsym, irrep, flat):
    """FCIVector flat order (alpha irrep blocks) -> C1 layout over all strings."""
    sa = o.strings(0).astype(np.int64)
    sb = o.strings(1).astype(np.int64)

    def sym(s):
        h = 0
        for i, x in enumerate(orbsym):
            if (s >> i) & 1:
                h ^= x
        return h

    ha = np.array([sym(int(x)) for x in sa])
    hb = np.array([sym(int(x)) for x in sb])
    full = np.zeros(len(sa) * len(sb))
    pos = 0
    for h in range(8):
        cols = np.nonzero(hb == (h ^ irrep))[0]
        for i in np.nonzero(ha == h)[0]:
            full[i * len(sb) + cols] = flat[pos:pos + len(cols)]
            pos += len(cols)
    assert pos == len(flat)
    return full


def test_cpp_driver_golden_c2v(tmp_path):
    import build as cpp_build
    from forte_b200 import FCISolver, StateInfo, build

    build.build()
    exe = cpp_build.build(str(tmp_path))
    ints, na, nb, irrep, mult, ref = golden_cases.load(1)
    assert irrep == 0
    n = ints.n
    irrep2 = 3
    nirrep = 1 + max(ints.orbsym)
    nirrep = 1 << (nirrep - 1).bit_length() if nirrep > 1 else 1
    assert np.array_equal(ints.oei_a, ints.oei_b) and np.array_equal(ints.tei_aa, ints.tei_bb)
    hdr = np.array([n, nirrep, na, nb, mult, 2, irrep2, 0], dtype=np.int32)
    with open(tmp_path / "in.bin", "wb") as f:
        f.write(hdr.tobytes())
        f.write(np.array(ints.orbsym, dtype=np.int32).tobytes())
        f.write(np.array([ints.scalar], dtype=np.float64).tobytes())
        for a in (ints.oei_a, ints.tei_aa, ints.tei_ab):
            f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    r = subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    out = np.fromfile(tmp_path / "out.bin", dtype=np.float64)
    n2, n4 = n * n, n ** 4
    pos = 0

    def take(k):
        nonlocal pos
        v = out[pos:pos + k]
        pos += k
        return v

    energies, spin2, iters = take(2), take(2), take(1)
    g1a, g1b, g2aa, g2ab, g2bb = take(n2), take(n2), take(n4), take(n4), take(n4)
    sf1, sf2 = take(n2), take(n4)
    e2, t1a, t1b, refused = take(1), take(n2), take(n2), take(1)
    e_gas, n_gas = take(2)
    assert pos == out.size
    assert abs(energies[0] - ref) < 1e-9
    assert refused[0] == 1.0

    # the same solves through the Python mirror give the vectors for the oracle
    s = FCISolver(StateInfo(na, nb, mult, na - nb, irrep), 2, ints, {"E_CONVERGENCE": 1e-12, "R_CONVERGENCE": 1e-8})
    s.compute_energy()
    assert np.max(np.abs(np.array(s.energies()) - energies)) < 1e-10
    t = FCISolver(StateInfo(na, nb, mult, na - nb, irrep2), 1, ints, {"E_CONVERGENCE": 1e-12, "R_CONVERGENCE": 1e-8})
    t.compute_energy()
    assert abs(t.energies()[0] - e2[0]) < 1e-10

    o = Oracle(n, na, nb, ints.orbsym, irrep)
    o.set_integrals(ints)
    cl = _c1(o, ints.orbsym, irrep, s.evecs()[0])
    cr = _c1(o, ints.orbsym, irrep2, t.evecs()[0])
    ro = o.rdms(cl, cl, 2)
    for got, key in ((g1a, "g1a"), (g1b, "g1b"), (g2aa, "g2aa"), (g2ab, "g2ab"), (g2bb, "g2bb")):
        assert np.max(np.abs(got - ro[key].ravel())) < 1e-9, key
    assert np.max(np.abs(sf1 - (ro["g1a"] + ro["g1b"]).ravel())) < 1e-9
    g2sf = ro["g2aa"] + ro["g2ab"] + np.transpose(ro["g2ab"], (1, 0, 3, 2)) + ro["g2bb"]
    assert np.max(np.abs(sf2 - g2sf.ravel())) < 1e-9
    # transition 1-RDM between the A1 state and the irrep2 state; the eigenvector sign of each state
    # is arbitrary, so compare up to the overall sign fixed by the largest element
    rt = o.rdms(cl, cr, 1)
    ref_t = np.concatenate([rt["g1a"].ravel(), rt["g1b"].ravel()])
    got_t = np.concatenate([t1a, t1b])
    assert np.max(np.abs(ref_t)) > 1e-3
    k = np.argmax(np.abs(ref_t))
    sgn = np.sign(got_t[k]) * np.sign(ref_t[k])
    assert np.max(np.abs(sgn * got_t - ref_t)) < 1e-9
    # and the Python mirror of FCISolver::transition_rdms, on the very vectors given to the oracle
    tp = s.transition_rdms([(0, 0)], t, 1)[0]
    assert np.max(np.abs(np.concatenate([tp.g1a.ravel(), tp.g1b.ravel()]) - ref_t)) < 1e-9
    sfp = s.transition_rdms([(0, 0)], t, 1, "spin_free")[0]
    assert np.max(np.abs(sfp.g1.ravel() - (rt["g1a"] + rt["g1b"]).ravel())) < 1e-9
    # the GAS solve of the driver (at most two electrons in the upper half) through the Python mirror
    from forte_b200 import GenCISolver
    g = GenCISolver(StateInfo(na, nb, mult, na - nb, irrep, (na + nb - 2, 0), (2 * (n // 2), 2)), 1, ints,
                    [list(range(n // 2)), list(range(n // 2, n))], {"E_CONVERGENCE": 1e-12, "R_CONVERGENCE": 1e-8})
    assert g.size() == int(n_gas) and 0 < g.size() < s.size()
    assert abs(g.compute_energy() - e_gas) < 1e-10 and e_gas > energies[0]
    with pytest.raises(Exception):
        s.transition_rdms([(0, 0)], t, 2)
    with pytest.raises(Exception):
        s.transition_rdms([(0, 1)], t, 1)
