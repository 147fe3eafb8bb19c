"""Active-space integral inputs for the FCI engine (host side, numpy).

Three ways in, all producing Forte's ``ActiveSpaceIntegrals`` layout
(forte/integrals/active_space_integrals.h:103-120):

* ``oei_a[p*n+q]``, ``oei_b`` -- one-electron integrals h_pq;
* ``tei_ab[p,q,r,s] = <pq|rs> = (pr|qs)``;
* ``tei_aa[p,q,r,s] = tei_bb = <pq||rs> = (pr|qs) - (ps|qr)``;
* ``scalar`` -- nuclear repulsion + scalar + frozen-core energy.

``from_chemist`` does the chemist -> physicist conversion the reference applies to FCIDUMP
input (forte/modules/objects_factory_fcidump.py:16-44).  ``read_fcidump`` parses the FCIDUMP
text format (forte/proc/fcidump.py:262-312).  ``dress_core`` folds doubly occupied core
orbitals into the scalar and one-electron terms, as CustomIntegrals' frozen-core operator
(forte/integrals/custom_integrals.cc:193-337) and the restricted-docc dressing of
make_active_space_ints (forte/integrals/active_space_integrals.cc:50-165) do.
``synthetic`` builds the seeded Cholesky-style integrals used by the benchmarks.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class ActiveSpaceIntegrals:
    n: int
    scalar: float
    oei_a: np.ndarray  # (n, n)
    oei_b: np.ndarray
    tei_aa: np.ndarray  # (n, n, n, n)
    tei_ab: np.ndarray
    tei_bb: np.ndarray
    orbsym: list = field(default_factory=list)

    def __post_init__(self):
        if not self.orbsym:
            self.orbsym = [0] * self.n


def from_chemist(h: np.ndarray, eri: np.ndarray, scalar: float = 0.0, orbsym=None) -> ActiveSpaceIntegrals:
    """Chemist-notation (pq|rs) -> Forte's <pq|rs>/<pq||rs> layout."""
    n = h.shape[0]
    tab = np.ascontiguousarray(np.einsum("ikjl->ijkl", eri))
    taa = np.ascontiguousarray(tab - np.einsum("iljk->ijkl", eri))
    h = np.ascontiguousarray(h, dtype=np.float64)
    return ActiveSpaceIntegrals(n, float(scalar), h.copy(), h.copy(), taa, tab, taa.copy(),
                                list(orbsym) if orbsym is not None else [0] * n)


def synthetic(n: int, L: int, seed: int, gap: float = 0.0, orbsym=None) -> ActiveSpaceIntegrals:
    """Seeded synthetic integrals.

    h: symmetric, diagonal ~ U[-2, +1] Eh, off-diagonal ~ N(0, 0.1).
    (pq|rs) = sum_L B^L_pq B^L_rs with symmetric B^L ~ N(0, 0.15): 8-fold symmetric, PSD.
    ``gap`` > 0: the diagonal of h is sorted ascending and ``gap`` is added to h_pp for
    p >= n/2, opening a gap between orbitals n/2-1 and n/2.  Generator: numpy PCG64(seed).
    ``orbsym`` (irreps of an abelian point group, XOR products): h_pq is kept only when p and q
    share an irrep, and each B^L carries an irrep g_L = L mod 8 and keeps B^L_pq only when
    orbsym[p] ^ orbsym[q] = g_L, so (pq|rs) vanishes unless the four irreps multiply to the
    totally symmetric one; the draws are the same as without symmetry.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    h = rng.normal(0.0, 0.1, size=(n, n))
    h = np.triu(h, 1)
    h = h + h.T
    d = rng.uniform(-2.0, 1.0, size=n)
    if gap > 0.0:
        d = np.sort(d)
        d[n // 2:] += gap
    h[np.diag_indices(n)] = d
    B = rng.normal(0.0, 0.15, size=(L, n, n))
    B = np.triu(B)
    B = B + np.transpose(np.triu(B, 1), (0, 2, 1))
    if orbsym is not None:
        sym = np.asarray(orbsym, dtype=np.int64)
        pair = sym[:, None] ^ sym[None, :]
        h = np.where(pair == 0, h, 0.0)
        for l in range(L):
            B[l] = np.where(pair == (l % 8), B[l], 0.0)
    eri = np.einsum("lpq,lrs->pqrs", B, B)
    return from_chemist(h, eri, 0.0, orbsym)


def read_fcidump(path: str) -> dict:
    """Parse an FCIDUMP file into {'norb','nelec','ms2','isym','orbsym','enuc','hcore','eri'}."""
    hdr = {}
    with open(path) as f:
        lines = f.read().splitlines()
    i = 0
    assert lines[0].strip().startswith("&FCI")
    text = []
    while True:
        i += 1
        ln = lines[i]
        if "END" in ln or ln.strip() == "/":
            break
        text.append(ln)
    i += 1
    joined = " ".join(text)
    # split "KEY=value," groups (values may contain commas, e.g. ORBSYM)
    import re

    for m in re.finditer(r"([A-Za-z0-9_]+)\s*=\s*([^=]*?)(?=(?:[A-Za-z0-9_]+\s*=)|$)", joined):
        key = m.group(1).lower()
        val = m.group(2).strip().rstrip(",").strip()
        if key == "orbsym":
            hdr[key] = [int(x) for x in val.replace(",", " ").split()]
        elif key == "uhf":
            hdr[key] = "TRUE" in val.upper()
        elif key == "pntgrp":
            hdr[key] = val
        else:
            hdr[key] = int(val.replace(",", ""))
    data = np.array([list(map(float, ln.split())) for ln in lines[i:] if ln.strip()])
    n = hdr["norb"]
    eri = np.zeros((n, n, n, n))
    h = np.zeros((n, n))
    enuc = 0.0
    for v, a, b, c, d in data:
        a, b, c, d = int(a), int(b), int(c), int(d)
        if a > 0 and c > 0:
            p, q, r, s = a - 1, b - 1, c - 1, d - 1
            for (w, x, y, z) in ((p, q, r, s), (q, p, r, s), (p, q, s, r), (q, p, s, r),
                                 (r, s, p, q), (s, r, p, q), (r, s, q, p), (s, r, q, p)):
                eri[w, x, y, z] = v
        elif a > 0 and b > 0:
            h[a - 1, b - 1] = v
            h[b - 1, a - 1] = v
        elif a == 0 and b == 0:
            enuc = v
    hdr["enuc"] = enuc
    hdr["hcore"] = h
    hdr["eri"] = eri
    return hdr


#: FCIDUMP (Molpro) irrep label -> psi4 irrep index, per point group
#: (the mapping of forte/proc/fcidump.py:244-256).
DUMP2PSI = {
    "c1": [-1, 0], "ci": [-1, 0, 1], "c2": [-1, 0, 1], "cs": [-1, 0, 1],
    "d2": [-1, 0, 3, 2, 1], "c2v": [-1, 0, 2, 3, 1], "c2h": [-1, 0, 2, 3, 1],
    "d2h": [-1, 0, 7, 6, 1, 5, 2, 3, 4],
}


def fcidump_from_entries(header: str, values: np.ndarray, index: np.ndarray) -> dict:
    """Same result as ``read_fcidump`` from an already split FCIDUMP: header text (between
    &FCI and &END) plus the value column and the four index columns."""
    import re

    hdr = {}
    for m in re.finditer(r"([A-Za-z0-9_]+)\s*=\s*([^=]*?)(?=(?:[A-Za-z0-9_]+\s*=)|$)", " ".join(header.split("\n"))):
        key = m.group(1).lower()
        val = m.group(2).strip().rstrip(",").strip()
        if key == "orbsym":
            hdr[key] = [int(x) for x in val.replace(",", " ").split()]
        elif key == "uhf":
            hdr[key] = "TRUE" in val.upper()
        elif key == "pntgrp":
            hdr[key] = val
        else:
            hdr[key] = int(val.replace(",", ""))
    n = hdr["norb"]
    eri = np.zeros((n, n, n, n))
    h = np.zeros((n, n))
    enuc = 0.0
    for v, (a, b, c, d) in zip(values, index.astype(int)):
        if a > 0 and c > 0:
            p, q, r, s = a - 1, b - 1, c - 1, d - 1
            for (w, x, y, z) in ((p, q, r, s), (q, p, r, s), (p, q, s, r), (q, p, s, r),
                                 (r, s, p, q), (s, r, p, q), (r, s, q, p), (s, r, q, p)):
                eri[w, x, y, z] = v
        elif a > 0 and b > 0:
            h[a - 1, b - 1] = v
            h[b - 1, a - 1] = v
        elif a == 0 and b == 0:
            enuc = v
    hdr["enuc"] = enuc
    hdr["hcore"] = h
    hdr["eri"] = eri
    return hdr


def active_space_from_fcidump(d: dict, frozen_docc=None, restricted_docc=None, active=None,
                              nel=None, multiplicity=None):
    """FCIDUMP dict -> (ActiveSpaceIntegrals, na, nb, target irrep, multiplicity).

    Orbitals are grouped by psi4 irrep (FCIDUMP order kept inside an irrep); per irrep the
    first frozen_docc + restricted_docc orbitals are core, the next ``active`` are active.
    The electron count and spin default to the FCIDUMP header (twice_ms = multiplicity - 1,
    the lowest non-negative Ms, as forte/modules/objects_factory_fcidump.py:47-77 does).
    """
    n = d["norb"]
    pg = d.get("pntgrp", "c1").lower() if "pntgrp" in d else "c1"
    mp = DUMP2PSI.get(pg, DUMP2PSI["c1"])
    orbsym = [mp[x] if pg in DUMP2PSI and pg != "c1" else 0 for x in d.get("orbsym", [1] * n)]
    isym = mp[d.get("isym", 1)] if pg != "c1" else 0
    nirrep = max(orbsym) + 1
    byirrep = [[i for i in range(n) if orbsym[i] == h] for h in range(nirrep)]
    nel = d["nelec"] if nel is None or nel < 0 else nel
    mult = d.get("ms2", 0) + 1 if multiplicity is None or multiplicity < 0 else multiplicity
    if active is None or len(active) == 0:
        core, act = [], list(range(n))
    else:
        fz = list(frozen_docc) if frozen_docc is not None and len(frozen_docc) else [0] * nirrep
        rd = list(restricted_docc) if restricted_docc is not None and len(restricted_docc) else [0] * nirrep
        core, act = [], []
        for h in range(nirrep):
            core += byirrep[h][: fz[h] + rd[h]]
            act += byirrep[h][fz[h] + rd[h]: fz[h] + rd[h] + active[h]]
    ints = dress_core(d["hcore"], d["eri"], d["enuc"], core, act, orbsym)
    nact = nel - 2 * len(core)
    tms = mult - 1
    na = (nact + tms) // 2
    nb = nact - na
    return ints, na, nb, isym, mult


def dress_core(h: np.ndarray, eri: np.ndarray, enuc: float, core: list, active: list,
               orbsym=None) -> ActiveSpaceIntegrals:
    """Fold doubly occupied core orbitals into scalar and one-electron terms.

    E = E_nuc + sum_i 2 h_ii + sum_ij [2 (ii|jj) - (ij|ji)],
    h^eff_pq = h_pq + sum_i [2 (pq|ii) - (pi|iq)]   (i, j in core; p, q active).
    """
    core = list(core)
    act = list(active)
    e = enuc
    for i in core:
        e += 2.0 * h[i, i]
    for i in core:
        for j in core:
            e += 2.0 * eri[i, i, j, j] - eri[i, j, j, i]
    hc = h.copy()
    for i in core:
        hc += 2.0 * eri[:, :, i, i] - eri[:, i, i, :]
    ha = hc[np.ix_(act, act)]
    ea = eri[np.ix_(act, act, act, act)]
    syms = [orbsym[a] for a in act] if orbsym is not None else None
    return from_chemist(ha, ea, e, syms)


def symmetry_check(ints: ActiveSpaceIntegrals, tol: float = 1e-10) -> float:
    """Largest violation of the real-orbital symmetries the pair-symmetrised sigma relies on:
    h_pq = h_qp, (pq|rs) = (qp|rs) = (rs|pq).  Returns the max absolute deviation."""
    tab = ints.tei_ab  # tab[p,q,r,s] = (pr|qs)
    eri = np.einsum("prqs->pqrs", tab)
    dev = max(
        float(np.max(np.abs(ints.oei_a - ints.oei_a.T))),
        float(np.max(np.abs(ints.oei_b - ints.oei_b.T))),
        float(np.max(np.abs(eri - np.transpose(eri, (1, 0, 2, 3))))),
        float(np.max(np.abs(eri - np.transpose(eri, (2, 3, 0, 1))))),
    )
    return dev
