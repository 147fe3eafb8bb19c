"""GAS determinant space of Forte's GenCISolver restated in plain Python -- CPU ORACLE (test
infrastructure only; only tests/ may use it, as the checker of the engine's GAS layout).

Restates, for small cases:
  - the occupation patterns: get_ci_occupation_patterns / recursive_ormas_generation
    (forte/genci/ci_occupation.cc:66-170);
  - the strings of each (pattern, irrep) class: make_strings_with_occupation
    (forte/genci/string_lists_makers.cc:65-127) with the classes of StringClass
    (forte/genci/genci_string_address.cc:81-133);
  - the determinant order of GenCIVector: GenCIStringLists::make_determinants
    (forte/genci/genci_string_lists.cc:276-291).

Parity of the determinant SETS is pinned by the reference's tests/pytest/gas/test_lists.py (golden
determinant lists, compared as sets there); the ORDER inside the flat vector has no golden vector in
the reference and rests on this restatement.
"""
from __future__ import annotations

import itertools

import numpy as np


def occupation_patterns(na, nb, sizes, gas_min, gas_max):
    """(alpha patterns, beta patterns, pattern pairs) in the reference's order: a depth-first walk
    over the spaces; alpha count, then beta count ascending in each space but the last, which takes
    the remaining electrons (ci_occupation.cc:66-121); bounds clamped like :131-170."""
    ns = len(sizes)
    mx = [min(gas_max[k], 2 * sizes[k], na + nb) for k in range(ns)]
    mn = [gas_min[k] for k in range(ns)]
    alfa, beta, pairs = [], [], []

    def index(lst, occ):
        if occ not in lst:
            lst.append(occ)
        return lst.index(occ)

    def rec(k, ra, rb, oa, ob):
        if k == ns - 1:
            if mn[k] <= ra + rb <= mx[k] and max(ra, rb) <= sizes[k] and min(ra, rb) >= 0:
                pa, pb = tuple(oa + [ra]), tuple(ob + [rb])
                pairs.append((index(alfa, pa), index(beta, pb)))
            return
        for a in range(max(mn[k] - sizes[k], 0), min(mx[k], sizes[k]) + 1):
            for b in range(max(mn[k] - a, 0), min(mx[k] - a, sizes[k]) + 1):
                if mn[k] <= a + b <= mx[k]:
                    rec(k + 1, ra - a, rb - b, oa + [a], ob + [b])

    rec(0, na, nb, [], [])
    return alfa, beta, pairs


def _irrep(s, orbsym):
    h = 0
    for p, o in enumerate(orbsym):
        if s >> p & 1:
            h ^= o
    return h


def class_strings(spaces, patterns, orbsym, nirrep):
    """Strings of each class (pattern index * nirrep + irrep): per space the 0/1 sequences over its
    orbitals (ascending) with the pattern's count, in increasing lexicographic order (the
    std::next_permutation walk from 0..01..1); the product over the spaces with the first space
    varying slowest; split by irrep in that order."""
    out = []
    for pat in patterns:
        per_space = []
        for orbs, e in zip(spaces, pat):
            seqs = sorted(t for t in itertools.product((0, 1), repeat=len(orbs)) if sum(t) == e)
            per_space.append([sum(1 << orbs[i] for i, x in enumerate(t) if x) for t in seqs])
        byh = [[] for _ in range(nirrep)]
        for combo in itertools.product(*per_space):
            s = 0
            for x in combo:
                s |= x
            byh[_irrep(s, orbsym)].append(s)
        out.extend(byh)
    return out


def determinants(n, orbsym, nirrep, irrep, na, nb, spaces, gas_min, gas_max):
    """(alpha string, beta string) of every GenCIVector flat position."""
    sizes = [len(sp) for sp in spaces]
    alfa, beta, pairs = occupation_patterns(na, nb, sizes, gas_min, gas_max)
    ca = class_strings(spaces, alfa, orbsym, nirrep)
    cb = class_strings(spaces, beta, orbsym, nirrep)
    dets = []
    for pa, pb in pairs:
        for h in range(nirrep):
            for a in ca[pa * nirrep + h]:
                for b in cb[pb * nirrep + (h ^ irrep)]:
                    dets.append((a, b))
    return dets


def in_gas(a, b, spaces, gas_min, gas_max):
    """The determinant's electrons per space lie within the bounds."""
    for k, orbs in enumerate(spaces):
        m = sum(1 << p for p in orbs)
        e = bin(a & m).count("1") + bin(b & m).count("1")
        if not gas_min[k] <= e <= gas_max[k]:
            return False
    return True


def det_from_occupation(text):
    """Forte's occupation notation, orbital 0 first: 2 = both, + = alpha, - = beta, 0 = empty."""
    a = b = 0
    for p, ch in enumerate(text):
        if ch in "2+":
            a |= 1 << p
        if ch in "2-":
            b |= 1 << p
    return a, b


def dense_hamiltonian(orc, dets):
    """H over the given determinants from the oracle's slater_rules, scalar energy on the diagonal."""
    N = len(dets)
    H = np.zeros((N, N))
    for i in range(N):
        for j in range(i, N):
            v = orc.slater_rules(dets[i][0], dets[i][1], dets[j][0], dets[j][1])
            H[i, j] = H[j, i] = v
    H[np.diag_indices(N)] += orc.ints.scalar
    return H
