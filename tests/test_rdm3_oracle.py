"""The oracle's 3-RDMs (a restatement of FCIVector::compute_3rdm_*_same_irrep over the hole
lists) pinned by brute force, as FCIVector::test_rdms does it (fci_vector_rdm.cc:808-930):
g3[p,q,r,s,t,u] = <bra| a+_p a+_q a+_r a_u a_t a_s |ket> evaluated on determinants (spin orbitals
alpha 0..n-1 then beta n..2n-1), as the Gram matrix <a_r a_q a_p bra, a_u a_t a_s ket>.

For two different vectors the reference loops take the creation indices from the right vector's
list entries, so its tensor for (left, right) is the one with bra = right and ket = left; the
transition case pins that orientation.  CPU only."""
import itertools

import numpy as np
import pytest

from oracle.oracle import Oracle


def _annihilate(vec, x):
    out = {}
    for d, cf in vec.items():
        if d >> x & 1:
            sign = -1.0 if bin(d & ((1 << x) - 1)).count("1") & 1 else 1.0
            e = d ^ (1 << x)
            out[e] = out.get(e, 0.0) + sign * cf
    return out


def _as_dets(o, c):
    sa, sb = o.strings(0), o.strings(1)
    nbs = len(sb)
    return {int(a) | int(b) << o.n: float(c[i * nbs + j]) for i, a in enumerate(sa) for j, b in enumerate(sb)}


def _brute(o, bra, ket, spins):
    """<bra| a+_p a+_q a+_r a_u a_t a_s |ket> for orbital spins (sp, sq, sr) of (p, s), (q, t), (r, u)."""
    n = o.n
    B, K = _as_dets(o, bra), _as_dets(o, ket)
    off = [0 if s == "a" else n for s in spins]
    W, V = {}, {}
    for p, q, r in itertools.product(range(n), repeat=3):
        W[p, q, r] = _annihilate(_annihilate(_annihilate(B, p + off[0]), q + off[1]), r + off[2])
        V[p, q, r] = _annihilate(_annihilate(_annihilate(K, p + off[0]), q + off[1]), r + off[2])
    keys = sorted({d for v in list(W.values()) + list(V.values()) for d in v})
    idx = {d: i for i, d in enumerate(keys)}
    triples = list(itertools.product(range(n), repeat=3))

    def dense(D):
        m = np.zeros((len(triples), len(keys)))
        for t, tr in enumerate(triples):
            for d, cf in D[tr].items():
                m[t, idx[d]] = cf
        return m

    return (dense(W) @ dense(V).T).reshape((n,) * 6)


def _rand(o, seed):
    v = np.random.default_rng(seed).normal(size=o.ndet)
    return v / np.linalg.norm(v)


@pytest.mark.parametrize("n,na,nb", [(5, 3, 2), (5, 2, 3), (6, 3, 3), (5, 4, 1)])
def test_oracle_rdms3_match_brute_force(n, na, nb):
    o = Oracle(n, na, nb)
    c = _rand(o, 10 * n + na)
    g = o.rdms3(c)
    for blk, spins in (("g3aaa", "aaa"), ("g3aab", "aab"), ("g3abb", "abb"), ("g3bbb", "bbb")):
        ref = _brute(o, c, c, spins)
        assert np.max(np.abs(g[blk] - ref)) < 1e-12, blk


def test_oracle_transition_rdms3_orientation():
    o = Oracle(5, 3, 2)
    left, right = _rand(o, 1), _rand(o, 2)
    g = o.rdms3(left, right)
    for blk, spins in (("g3aaa", "aaa"), ("g3aab", "aab"), ("g3abb", "abb")):
        assert np.max(np.abs(g[blk] - _brute(o, right, left, spins))) < 1e-12, blk
