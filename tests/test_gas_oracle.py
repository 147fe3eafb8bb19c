"""The GAS oracle (GenCISolver's determinant space restated) pinned on the CPU: the reference's
golden determinant lists (tests/pytest/gas/test_lists.py, compared as sets there too) and the
equivalence of the occupation-pattern construction with the per-space electron bounds; also the
host-side validation of GAS spaces in the Python mirror."""
import itertools

import numpy as np
import pytest

from oracle import gas_oracle as G


def _det_set(texts):
    return sorted(G.det_from_occupation(t) for t in texts)


def test_golden_lists1():
    # tests/pytest/gas/test_lists.py::test_gas_lists1: C2v, nmopi [1, 2, 0, 0],
    # GAS1 = [1, 0, 0, 0], GAS2 = [0, 2, 0, 0]; na = nb = 2, gas_min [0, 0], gas_max [2, 2], A1
    orbsym = [0, 1, 1]
    dets = G.determinants(3, orbsym, 4, 0, 2, 2, [[0], [1, 2]], [0, 0], [2, 2])
    assert len(dets) == 4
    assert sorted(dets) == _det_set(["220", "202", "2+-", "2-+"])


def test_golden_lists2():
    # tests/pytest/gas/test_lists.py::test_gas_lists2: C2v, nmopi [2, 1, 2, 0],
    # GAS1 = [1, 0, 1, 0], GAS2 = [1, 1, 1, 0]; ACTIVE groups by irrep, then by space:
    # orbitals 0 (A1, GAS1), 1 (A1, GAS2), 2 (A2, GAS2), 3 (B1, GAS1), 4 (B1, GAS2)
    orbsym = [0, 0, 1, 2, 2]
    dets = G.determinants(5, orbsym, 4, 0, 3, 3, [[0, 3], [1, 2, 4]], [3, 3], [3, 3])
    golden = ["+-022", "220+-", "+-220", "202+-", "-+022", "220-+", "-+220", "202-+"]
    assert len(dets) == 8
    assert sorted(dets) == _det_set(golden)


def _all_strings(n, k):
    return [sum(1 << p for p in c) for c in itertools.combinations(range(n), k)]


CASES = [
    # n, orbsym, nirrep, irrep, na, nb, spaces, min, max
    (6, [0] * 6, 1, 0, 3, 3, [[0, 1], [2, 3], [4, 5]], [2, 0, 0], [4, 4, 2]),
    (7, [0, 1, 2, 3, 0, 1, 2], 4, 1, 3, 2, [[0, 1, 2], [3, 4, 5, 6]], [3, 0], [6, 3]),
    (8, [0, 0, 1, 1, 2, 2, 3, 3], 4, 0, 4, 4, [[0, 2, 4, 6], [1, 3], [5, 7]], [6, 0, 0], [8, 3, 2]),
    (6, [0] * 6, 1, 0, 0, 3, [[0, 1, 2], [3, 4, 5]], [1, 0], [3, 1]),
    (5, [0, 1, 0, 1, 0], 2, 1, 2, 1, [[1, 3], [0, 2, 4]], [0, 0], [1, 3]),
    (6, [0] * 6, 1, 0, 3, 3, [[0, 1, 2], [3, 4, 5]], [6, 0], [6, 0]),  # one determinant
    (6, [0] * 6, 1, 0, 3, 3, [[0, 1, 2], [3, 4, 5]], [0, 4], [2, 6]),  # at most 2 electrons in space 0
]


@pytest.mark.parametrize("case", CASES)
def test_patterns_equal_bounds(case):
    n, orbsym, nirrep, irrep, na, nb, spaces, mn, mx = case
    dets = G.determinants(n, orbsym, nirrep, irrep, na, nb, spaces, mn, mx)
    assert len(set(dets)) == len(dets)  # each determinant once
    ref = set()
    for a in _all_strings(n, na):
        for b in _all_strings(n, nb):
            if G._irrep(a ^ b, orbsym) == irrep and G.in_gas(a, b, spaces, mn, mx):
                ref.add((a, b))
    assert set(dets) == ref


def test_trivial_bounds_are_the_fci_space():
    n, orbsym = 6, [0, 1, 0, 1, 0, 1]
    dets = G.determinants(n, orbsym, 2, 1, 3, 2, [[0, 1, 2], [3, 4, 5]], [0, 0], [6, 6])
    fci = {(a, b) for a in _all_strings(n, 3) for b in _all_strings(n, 2) if G._irrep(a ^ b, orbsym) == 1}
    assert set(dets) == fci


def test_pattern_order_follows_the_walk():
    # two spaces of 2 orbitals, 2 + 2 electrons, space 1 holds at most 2: alpha count of space 0
    # ascending, then its beta count ascending
    alfa, beta, pairs = G.occupation_patterns(2, 2, [2, 2], [0, 0], [4, 2])
    walk = [(alfa[i][0], beta[j][0]) for i, j in pairs]
    assert walk == sorted(walk)
    assert all(a + b >= 2 for a, b in walk)
    assert np.all(np.array([alfa[i][0] + alfa[i][1] for i, _ in pairs]) == 2)


def test_gas_layout_host_validation():
    # the Python mirror's checks of the GAS spaces, before anything reaches the engine
    from forte_b200.fci_solver import gas_layout
    spaces, owner, mn, mx = gas_layout([[3, 0, 1], [2, 4, 5], []], 6, (2,))
    assert spaces == [[0, 1, 3], [2, 4, 5]] and owner == [0, 0, 1, 0, 1, 1]
    assert mn == [2, 0] and mx == [6, 6]
    assert gas_layout([], 4) == ([], [-1] * 4, [], [])
    # orbital 5 in no space, an empty space inside, orbital 2 twice, orbital 6 outside 0..5
    for bad in ([[0, 1, 2], [3, 4]], [[0, 1, 2], [], [3, 4, 5]], [[0, 1, 2], [2, 3, 4, 5]], [[0, 1, 2, 3, 4, 5, 6]]):
        with pytest.raises(ValueError):
            gas_layout(bad, 6)
    with pytest.raises(ValueError):
        gas_layout([[0], [1], [2], [3], [4], [5], [6]], 7)  # seven spaces


@pytest.mark.parametrize("nirrep,ngas", [(8, 3), (2, 6)])
def test_patterns_equal_bounds_many_spaces(nirrep, ngas):
    # up to six spaces and eight irreps: the pattern construction still equals the bounds filter
    n = 10
    rng = np.random.default_rng(nirrep * 10 + ngas)
    orbsym = [int(x) for x in rng.integers(0, nirrep, n)]
    cuts = sorted(rng.choice(np.arange(1, n), ngas - 1, replace=False))
    spaces = [list(range(a, b)) for a, b in zip([0] + list(cuts), list(cuts) + [n])]
    mn = [max(0, len(sp) - 1) if k == 0 else 0 for k, sp in enumerate(spaces)]
    mx = [2 * len(sp) if k == 0 else min(2 * len(sp), 3) for k, sp in enumerate(spaces)]
    irrep = int(rng.integers(0, nirrep))
    dets = G.determinants(n, orbsym, nirrep, irrep, 4, 3, spaces, mn, mx)
    assert len(set(dets)) == len(dets)
    ref = {(a, b) for a in _all_strings(n, 4) for b in _all_strings(n, 3)
           if G._irrep(a ^ b, orbsym) == irrep and G.in_gas(a, b, spaces, mn, mx)}
    assert set(dets) == ref and len(ref) > 0
