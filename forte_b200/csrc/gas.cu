// Layout maps of the engine's vectors and the generalized active space (GAS) restriction.
//
// The engine's device layout is the C1 layout (nas x nbs) or, with point-group symmetry, the
// target irrep's blocks (symblock.cu).  Two kinds of restriction sit on top of it as a byte mask
// over the layout plus a host map from the caller's flat order to layout positions:
//   - the masked C1 layout with symmetry (sym_blocked = 0): determinants of the target irrep,
//     host vectors in FCIVector flat order (forte/fci/fci_string_lists.cc:318-331);
//   - GAS (GenCISolver, forte/genci/genci_solver.h): determinants whose number of electrons
//     (alpha + beta) in each orbital space k lies in [emin[k], emax[k]], host vectors in
//     GenCIVector flat order.
// Sigma of a masked layout is P H P, P the projector on the kept determinants: on the kept
// space that is H itself, so energies, vectors and RDMs are those of the restricted space.
// With GAS spaces the blocked layout (symblock.cu, also without point-group symmetry) holds only
// the strings whose occupation pattern some GAS determinant has: its blocks are the products of
// those strings, a superset of the GAS space, and a sigma costs what those blocks cost.  The
// masked C1 layout (sym_blocked = 0) keeps every string and costs the full sigma.
//
// The GenCIVector flat order restated here, from the reference:
//   1. occupation patterns (get_ci_occupation_patterns and recursive_ormas_generation,
//      forte/genci/ci_occupation.cc:66-170): a depth-first walk over the spaces in order; in
//      every space but the last, alpha counts a then beta counts b ascending, with a <= size,
//      b <= size and emin <= a + b <= emax'; the last space takes the electrons that remain if
//      they fit.  emax' = min(emax, 2 size, na + nb).  Each leaf appends the pair (alpha
//      pattern, beta pattern); a pattern gets the index of its first appearance in its own list.
//   2. strings of an alpha (beta) pattern (make_strings_with_occupation,
//      forte/genci/string_lists_makers.cc:65-127): per space, the subsets of its orbitals with
//      the pattern's count, in lexicographic order of the 0/1 sequence over the space's orbitals
//      (ascending) starting from 0..01..1; the cartesian product over the spaces with the first
//      space varying slowest; then split by irrep keeping that order.  Class of a string =
//      pattern * nirrep + irrep (StringClass, forte/genci/genci_string_address.cc:81-133).
//   3. determinant blocks: for each pattern pair in order, for each alpha irrep h, the block
//      (alpha class (pa, h)) x (beta class (pb, h ^ symmetry)), row-major; the flat address is
//      the block offset + alpha address * beta class size + beta address
//      (GenCIStringLists::determinant_address, forte/genci/genci_string_lists.cc:293-305).
#include "fcib_internal.h"

#include <algorithm>
#include <array>

namespace fcib {

struct GasDev {
    int ngas = 0;
    int emin[kMaxGas] = {}, emax[kMaxGas] = {};
    uint32_t orbs[kMaxGas] = {};
    int check_irrep = 0;        // C1 layout with symmetry: keep only the target irrep
    uint32_t irrbit[3] = {0u, 0u, 0u};
    int irrep = 0;
};

__global__ void k_layout_mask(uint8_t* __restrict__ mask, int64_t nvec, SymDev d, int64_t nbs,
                              const uint32_t* __restrict__ sa, const uint32_t* __restrict__ sb, GasDev g) {
    for (int64_t I = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; I < nvec; I += (int64_t)gridDim.x * blockDim.x) {
        int ia, ib;
        if (d.on) {
            sym_decode(d, I, ia, ib);
        } else {
            ia = (int)(I / nbs);
            ib = (int)(I - (int64_t)ia * nbs);
        }
        const uint32_t a = sa[ia], b = sb[ib];
        bool ok = true;
        if (g.check_irrep) {
            // irrep(a) ^ irrep(b) = parities of the orbitals of a ^ b in each irrep bit
            const uint32_t x = a ^ b;
            const int h = (__popc(x & g.irrbit[0]) & 1) | ((__popc(x & g.irrbit[1]) & 1) << 1) |
                          ((__popc(x & g.irrbit[2]) & 1) << 2);
            ok = (h == g.irrep);
        }
        for (int k = 0; k < g.ngas; k++) {
            const int e = __popc(a & g.orbs[k]) + __popc(b & g.orbs[k]);
            ok = ok && e >= g.emin[k] && e <= g.emax[k];
        }
        mask[I] = ok ? 1 : 0;
    }
}

using Occ = std::array<int, kMaxGas>;

// step 1 above: the pattern lists and the ordered pattern pairs
static void gas_patterns(const Context& c, std::vector<Occ>& alfa, std::vector<Occ>& beta,
                         std::vector<std::pair<int, int>>& pairs) {
    const GasSpace& g = c.gas;
    const int ns = g.ngas;
    std::vector<int> size(ns), mn(ns), mx(ns);
    for (int k = 0; k < ns; k++) {
        size[k] = __builtin_popcount(g.orbs[k]);
        mn[k] = g.emin[k];
        mx[k] = std::min(g.emax[k], std::min(2 * size[k], c.na + c.nb));
    }
    alfa.clear();
    beta.clear();
    pairs.clear();
    auto index_of = [](std::vector<Occ>& list, const Occ& o) {
        auto it = std::find(list.begin(), list.end(), o);
        if (it != list.end()) return (int)(it - list.begin());
        list.push_back(o);
        return (int)list.size() - 1;
    };
    Occ oa{}, ob{};
    // depth-first over the spaces; ra, rb: electrons not yet placed
    auto walk = [&](auto&& self, int k, int ra, int rb) -> void {
        if (k == ns - 1) {
            const int tot = ra + rb;
            if (tot <= mx[k] && tot >= mn[k] && std::max(ra, rb) <= size[k] && std::min(ra, rb) >= 0) {
                oa[k] = ra;
                ob[k] = rb;
                const int ia = index_of(alfa, oa);
                const int ib = index_of(beta, ob);
                pairs.emplace_back(ia, ib);
            }
            return;
        }
        for (int a = std::max(mn[k] - size[k], 0); a <= std::min(mx[k], size[k]); a++)
            for (int b = std::max(mn[k] - a, 0); b <= std::min(mx[k] - a, size[k]); b++) {
                if (a + b > mx[k] || a + b < mn[k]) continue;
                oa[k] = a;
                ob[k] = b;
                self(self, k + 1, ra - a, rb - b);
            }
    };
    walk(walk, 0, c.na, c.nb);
}

void gas_string_patterns(const Context& c, const std::vector<uint32_t>& sa, const std::vector<uint32_t>& sb,
                         std::vector<int>& pat_a, std::vector<int>& pat_b, int& npa, int& npb,
                         std::vector<uint8_t>& allowed, std::vector<uint8_t>& reach_a, std::vector<uint8_t>& reach_b) {
    std::vector<Occ> pa, pb;
    std::vector<std::pair<int, int>> pairs;
    gas_patterns(c, pa, pb, pairs);
    npa = (int)pa.size();
    npb = (int)pb.size();
    // a string is used by some GAS determinant when its occupation pattern is in its spin's list
    auto mark = [&](const std::vector<uint32_t>& s, const std::vector<Occ>& pats, std::vector<int>& pat) {
        pat.assign(s.size(), -1);
        for (size_t i = 0; i < s.size(); i++) {
            Occ o{};
            for (int k = 0; k < c.gas.ngas; k++) o[k] = __builtin_popcount(s[i] & c.gas.orbs[k]);
            auto it = std::find(pats.begin(), pats.end(), o);
            if (it != pats.end()) pat[i] = (int)(it - pats.begin());
        }
    };
    mark(sa, pa, pat_a);
    mark(sb, pb, pat_b);
    allowed.assign((size_t)npa * npb, 0);
    for (auto& pr : pairs) allowed[(size_t)pr.first * npb + pr.second] = 1;
    // one replacement moves one electron: the patterns are equal or differ by +1 and -1 in two spaces
    auto reach = [&](const std::vector<Occ>& pats, std::vector<uint8_t>& r) {
        const size_t np = pats.size();
        r.assign(np * np, 0);
        for (size_t x = 0; x < np; x++)
            for (size_t y = 0; y < np; y++) {
                int up = 0, down = 0, other = 0;
                for (int k = 0; k < c.gas.ngas; k++) {
                    const int d = pats[y][k] - pats[x][k];
                    if (d == 1) up++;
                    else if (d == -1) down++;
                    else if (d != 0) other++;
                }
                r[x * np + y] = (other == 0 && up == down && up <= 1) ? 1 : 0;
            }
    };
    reach(pa, reach_a);
    reach(pb, reach_b);
}

// step 2 above: the strings of every class, as C1 string indices, for one spin
static void gas_classes(const Context& c, const std::vector<Occ>& pats, int nelec,
                        std::vector<std::vector<int32_t>>& cls) {
    const GasSpace& g = c.gas;
    const int ns = g.ngas, nh = std::max(1, c.nirrep);
    cls.assign(pats.size() * nh, {});
    std::vector<std::vector<int>> mos(ns);
    for (int k = 0; k < ns; k++)
        for (int p = 0; p < c.n; p++)
            if (g.orbs[k] >> p & 1u) mos[k].push_back(p);
    for (size_t ip = 0; ip < pats.size(); ip++) {
        // per space, the subsets in next-permutation order of the 0/1 sequence
        std::vector<std::vector<uint32_t>> part(ns);
        bool empty = false;
        for (int k = 0; k < ns; k++) {
            const int m = (int)mos[k].size(), e = pats[ip][k];
            if (e < 0 || e > m) {
                empty = true;
                continue;
            }
            std::vector<char> seq(m, 0);
            for (int i = m - e; i < m; i++) seq[i] = 1;
            do {
                uint32_t s = 0;
                for (int i = 0; i < m; i++)
                    if (seq[i]) s |= 1u << mos[k][i];
                part[k].push_back(s);
            } while (std::next_permutation(seq.begin(), seq.end()));
        }
        if (empty) continue;
        // cartesian product, first space slowest
        std::vector<size_t> idx(ns, 0);
        while (true) {
            uint32_t s = 0;
            for (int k = 0; k < ns; k++) s |= part[k][idx[k]];
            int h = 0;
            if (c.nirrep > 1)
                for (int p = 0; p < c.n; p++)
                    if (s >> p & 1u) h ^= c.orbsym[p];
            if (__builtin_popcount(s) == nelec) cls[ip * nh + h].push_back((int32_t)host_rank(s, c.n));
            int k = ns - 1;
            while (k >= 0 && ++idx[k] == part[k].size()) idx[k--] = 0;
            if (k < 0) break;
        }
    }
}

// mask and flat map of the current layout; nothing when the layout is the flat order itself
void build_layout_maps(Context& c) {
    c.flat_map.clear();
    c.gas.ndet = 0;
    c.gas.acls.clear();
    c.gas.bcls.clear();
    const bool masked_sym = c.nirrep > 1 && !c.sym.on;
    const bool gas = c.gas.ngas > 0;
    if (!masked_sym && !gas) {
        c.mask.release();
        return;
    }
    // the mask, on the device
    GasDev gd;
    gd.ngas = c.gas.ngas;
    for (int k = 0; k < gd.ngas; k++) {
        gd.orbs[k] = c.gas.orbs[k];
        gd.emin[k] = c.gas.emin[k];
        gd.emax[k] = c.gas.emax[k];
    }
    gd.check_irrep = masked_sym ? 1 : 0;
    gd.irrep = c.irrep;
    for (int b = 0; b < 3; b++)
        for (int p = 0; p < c.n; p++)
            if (c.orbsym[p] >> b & 1) gd.irrbit[b] |= 1u << p;
    c.mask.alloc((size_t)c.nvec);
    const int grid = (int)std::min<int64_t>((c.nvec + 255) / 256, 16 * (int64_t)c.num_sms);
    k_layout_mask<<<std::max(grid, 1), 256, 0, c.stream>>>(c.mask.p, c.nvec, sym_dev(c), c.nbs, c.A.str.p, c.B.str.p,
                                                           gd);
    FCIB_KCHECK();
    std::vector<uint32_t> sa(c.nas), sb(c.nbs);
    FCIB_CUDA(cudaMemcpy(sa.data(), c.A.str.p, 4 * c.nas, cudaMemcpyDeviceToHost));
    FCIB_CUDA(cudaMemcpy(sb.data(), c.B.str.p, 4 * c.nbs, cudaMemcpyDeviceToHost));
    auto irrep_of = [&](uint32_t s) {
        int h = 0;
        for (int i = 0; i < c.n; i++)
            if (s >> i & 1u) h ^= c.orbsym[i];
        return h;
    };
    auto pos = [&](int64_t ia, int64_t ib) { return c.sym.on ? sym_host_encode(c, ia, ib) : ia * c.nbs + ib; };
    if (!gas) {
        // FCIVector flat order: alpha irrep blocks h, rows = alpha strings of irrep h in string
        // order, columns = beta strings of irrep h ^ symmetry (forte/fci/fci_string_lists.cc:318-331)
        std::vector<int> ha(c.nas), hb(c.nbs);
        for (int64_t i = 0; i < c.nas; i++) ha[i] = irrep_of(sa[i]);
        for (int64_t i = 0; i < c.nbs; i++) hb[i] = irrep_of(sb[i]);
        for (int h = 0; h < c.nirrep; h++)
            for (int64_t i = 0; i < c.nas; i++) {
                if (ha[i] != h) continue;
                for (int64_t j = 0; j < c.nbs; j++)
                    if (hb[j] == (h ^ c.irrep)) c.flat_map.push_back(pos(i, j));
            }
        return;
    }
    // GenCIVector flat order
    GasSpace& g = c.gas;
    std::vector<Occ> pa, pb;
    std::vector<std::pair<int, int>> pairs;
    gas_patterns(c, pa, pb, pairs);
    std::vector<std::vector<int32_t>> ca, cb;
    gas_classes(c, pa, c.na, ca);
    gas_classes(c, pb, c.nb, cb);
    const int nh = std::max(1, c.nirrep);
    const int irrep = c.nirrep > 1 ? c.irrep : 0;
    g.acls.assign(c.nas, -1);
    g.bcls.assign(c.nbs, -1);
    g.aadd.assign(c.nas, 0);
    g.badd.assign(c.nbs, 0);
    g.acnt.assign(ca.size(), 0);
    g.bcnt.assign(cb.size(), 0);
    for (size_t k = 0; k < ca.size(); k++) {
        g.acnt[k] = (int64_t)ca[k].size();
        for (size_t t = 0; t < ca[k].size(); t++) {
            g.acls[ca[k][t]] = (int32_t)k;
            g.aadd[ca[k][t]] = (int64_t)t;
        }
    }
    for (size_t k = 0; k < cb.size(); k++) {
        g.bcnt[k] = (int64_t)cb[k].size();
        for (size_t t = 0; t < cb[k].size(); t++) {
            g.bcls[cb[k][t]] = (int32_t)k;
            g.badd[cb[k][t]] = (int64_t)t;
        }
    }
    g.ncb = (int)cb.size();
    g.blk_off.assign(ca.size() * cb.size(), -1);
    int64_t off = 0;
    for (auto& pr : pairs)
        for (int h = 0; h < nh; h++) {
            const int ka = pr.first * nh + h, kb = pr.second * nh + (h ^ irrep);
            g.blk_off[(size_t)ka * g.ncb + kb] = off;
            for (int32_t ia : ca[ka])
                for (int32_t ib : cb[kb]) c.flat_map.push_back(pos(ia, ib));
            off += (int64_t)ca[ka].size() * cb[kb].size();
        }
    g.ndet = off;
    // every kept determinant appears once in the blocks
    std::vector<uint8_t> hm((size_t)c.nvec);
    FCIB_CUDA(cudaMemcpyAsync(hm.data(), c.mask.p, (size_t)c.nvec, cudaMemcpyDeviceToHost, c.stream));
    FCIB_CUDA(cudaStreamSynchronize(c.stream));
    int64_t kept = 0;
    for (auto x : hm) kept += x;
    bool ok = kept == g.ndet;
    for (size_t i = 0; ok && i < c.flat_map.size(); i++) ok = hm[(size_t)c.flat_map[i]] == 1;
    FCIB_CHECK(ok, FCIB_ERR_NUMERIC, "GAS layout: the determinant blocks do not match the occupation bounds");
}

// GenCIVector flat position of the determinant at layout index I, -1 outside the GAS space
int64_t gas_flat_position(const Context& c, int64_t I) {
    int64_t ia, ib;
    if (c.sym.on) {
        sym_host_decode(c, I, ia, ib);
    } else {
        ia = I / c.nbs;
        ib = I % c.nbs;
    }
    const GasSpace& g = c.gas;
    const int ka = g.acls[ia], kb = g.bcls[ib];
    if (ka < 0 || kb < 0) return -1;
    const int64_t o = g.blk_off[(size_t)ka * g.ncb + kb];
    if (o < 0) return -1;
    return o + g.aadd[ia] * g.bcnt[kb] + g.badd[ib];
}

}  // namespace fcib
