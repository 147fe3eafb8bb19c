// Irrep-blocked determinant space: the target irrep's determinants only, in FCIVector flat order.
//
// Reference: FCIVector keeps one block per alpha irrep h, the alpha strings of irrep h by the beta
// strings of irrep h ^ symmetry (forte/fci/fci_vector.cc:86-169; string addresses per irrep,
// forte/fci/fci_string_address.cc:36-75), and FCIVector::Hamiltonian loops over those blocks and
// over the substitutions that symmetry allows (forte/fci/fci_vector_hamiltonian.cc:125-272).
// Here the dense sigma kernels of the C1 layout run on sub-problems whose tables are the C1 tables
// restricted by irrep:
//
// * opposite spin, for every target alpha irrep ha and pair irrep g: rows = the alpha strings of
//   irrep ha, their connections through pairs of irrep g (which reach alpha irrep ha ^ g), the
//   pair-matrix columns of irrep g ((pq|rs) vanishes unless both pairs have the same irrep), source
//   columns = beta strings of irrep ha ^ irrep ^ g, targets = beta strings of irrep ha ^ irrep.  The
//   g = 0 sub-problem of a block writes it (E0 C included); the others add to it.  Rows with fewer
//   connections than the longest are padded with the zero pair (a pair-matrix row of zeros).
// * same spin: an (N-2)-electron group splits by irrep (its strings of one irrep couple only among
//   themselves through <pq||rs>); every part is a group of its own in that irrep's block, padded to
//   the irrep's largest part with empty members (kNullRow).
//
// Each sub-problem is smaller than the C1 problem by about the irrep count in rows or columns and
// in connections or pairs, so a sigma costs ~1/nirrep of the masked C1 sigma and a vector
// 1/nirrep of its memory.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "fcib_internal.h"

namespace fcib {

static int sb_pad8(int x) { return (x + 7) / 8 * 8; }

// same-spin groups of one spin and kind, split by the irrep of their strings
static void build_group_subs(Context& c, const SpinTables& t, bool alpha, bool one_body, std::vector<GroupSub>& out,
                             std::vector<uint32_t>& rows_all, std::vector<uint16_t>& labs_all) {
    SymSpace& y = c.sym;
    out.clear();
    const int ng = one_body ? t.ng1 : t.ng2, G = one_body ? t.g1 : t.g2;
    if (ng == 0 || G == 0) return;
    std::vector<uint32_t> rows((size_t)ng * G);
    std::vector<uint16_t> labs((size_t)ng * G);
    FCIB_CUDA(cudaMemcpy(rows.data(), (one_body ? t.g1row.p : t.g2row.p), 4 * rows.size(), cudaMemcpyDeviceToHost));
    FCIB_CUDA(cudaMemcpy(labs.data(), (one_body ? t.g1lab.p : t.g2lab.p), 2 * labs.size(), cudaMemcpyDeviceToHost));
    const std::vector<int>& irr = alpha ? y.airr : y.birr;
    const std::vector<int32_t>& loc = alpha ? y.aloc_h : y.bloc_h;
    const int nh = c.nirrep, S = c.irrep;
    std::vector<std::vector<std::vector<std::pair<uint32_t, uint16_t>>>> parts(nh);
    std::vector<std::vector<std::pair<uint32_t, uint16_t>>> bucket(nh);
    for (int gi = 0; gi < ng; gi++) {
        for (auto& b : bucket) b.clear();
        for (int m = 0; m < G; m++) {
            const uint32_t e = rows[(size_t)gi * G + m];
            if (e == kNullRow) continue;
            const uint32_t I = e & kConnIdxMask;
            if (loc[I] < 0) continue;  // a string no GAS determinant uses: its rows and columns are absent
            bucket[irr[I]].push_back({(uint32_t)loc[I] | (e & kSignBit), labs[(size_t)gi * G + m]});
        }
        for (int h = 0; h < nh; h++)
            if (!bucket[h].empty()) parts[h].push_back(bucket[h]);
    }
    for (int h = 0; h < nh; h++) {
        const int ncols = alpha ? y.bcnt[h ^ S] : y.acnt[h ^ S];
        if (parts[h].empty() || ncols == 0) continue;
        GroupSub s;
        s.ngroups = (int)parts[h].size();
        for (auto& p : parts[h]) s.G = std::max(s.G, (int)p.size());
        s.ncols = ncols;
        s.blk = alpha ? y.d.blk[h] : y.blkT[h];
        s.off = rows_all.size();
        for (auto& p : parts[h])
            for (int m = 0; m < s.G; m++) {
                rows_all.push_back(m < (int)p.size() ? p[m].first : kNullRow);
                labs_all.push_back(m < (int)p.size() ? p[m].second : (uint16_t)0);
            }
        out.push_back(s);
    }
}

// opposite-spin sub-problem tables (needs the folded one-body terms: na >= 1 and nb >= 1)
static void build_ab_subs(Context& c, const std::vector<uint32_t>& sb) {
    SymSpace& y = c.sym;
    const int nh = c.nirrep, S = c.irrep, n = c.n;
    const int s1 = c.A.s1, npp = c.A.npair_pad, npair = c.A.npair;
    FCIB_CHECK(c.B.npair_pad == npp && npp + 1 <= 1023, FCIB_ERR_UNSUPPORTED, "blocked sigma: pair index range");
    std::vector<uint32_t> conn((size_t)c.nas * s1);
    std::vector<int32_t> tgt((size_t)c.nbs * npp);
    std::vector<double> V((size_t)npp * npp);
    FCIB_CUDA(cudaMemcpy(conn.data(), c.A.conn.p, 4 * conn.size(), cudaMemcpyDeviceToHost));
    FCIB_CUDA(cudaMemcpy(tgt.data(), c.B.tgt.p, 4 * tgt.size(), cudaMemcpyDeviceToHost));
    FCIB_CUDA(cudaMemcpy(V.data(), c.V.p, 8 * V.size(), cudaMemcpyDeviceToHost));
    std::vector<int> pirr(npair), pp(npair), pq(npair);
    for (int p = 0; p < n; p++)
        for (int q = 0; q <= p; q++) {
            const int P = p * (p + 1) / 2 + q;
            pirr[P] = c.orbsym[p] ^ c.orbsym[q];
            pp[P] = p;
            pq[P] = q;
        }
    y.npp = npp;
    const uint32_t Pz = (uint32_t)npp;  // the zero pair
    std::vector<std::vector<int>> plist(nh);
    std::vector<int> perm_all;
    y.np_g.assign(nh, 0);
    y.npg.assign(nh, 0);
    y.noff8_g.assign(nh, 0);
    y.ndiag_g.assign(nh, 0);
    y.vg_off.assign(nh, 0);
    y.perm_off.assign(nh, 0);
    std::vector<double> vg_all;
    for (int g = 0; g < nh; g++) {
        for (int P = 0; P < npair; P++)
            if (pirr[P] == g) plist[g].push_back(P);
        y.np_g[g] = (int)plist[g].size();
        y.npg[g] = sb_pad8(y.np_g[g]);
        // FP64 columns: the pairs of irrep g; row Pz stays zero
        y.vg_off[g] = vg_all.size();
        vg_all.resize(vg_all.size() + (size_t)(npp + 1) * y.npg[g], 0.0);
        double* vg = vg_all.data() + y.vg_off[g];
        for (int P = 0; P < npp; P++)
            for (int j = 0; j < y.np_g[g]; j++) vg[(size_t)P * y.npg[g] + j] = V[(size_t)P * npp + plist[g][j]];
        // tensor-core columns: off-diagonal pairs of irrep g (padded to 8), then every diagonal pair for g = 0
        std::vector<int> off;
        for (int P : plist[g])
            if (pp[P] != pq[P]) off.push_back(P);
        y.noff8_g[g] = sb_pad8((int)off.size());
        y.ndiag_g[g] = g == 0 ? n : 0;
        const int ncol = y.noff8_g[g] + y.ndiag_g[g];
        const int npad = (ncol + 15) / 16 * 16;
        y.perm_off[g] = perm_all.size();
        std::vector<int> pm(npad, -1);
        for (size_t i = 0; i < off.size(); i++) pm[i] = off[i];
        for (int r = 0; r < y.ndiag_g[g]; r++) pm[y.noff8_g[g] + r] = r * (r + 1) / 2 + r;
        perm_all.insert(perm_all.end(), pm.begin(), pm.end());
    }
    y.Vg.upload(vg_all, c.stream);
    std::vector<double> vz((size_t)(npp + 1) * npp, 0.0);
    std::copy(V.begin(), V.end(), vz.begin());
    y.Vz.upload(vz, c.stream);
    y.perm.upload(perm_all, c.stream);

    std::vector<uint32_t> conn_all;
    std::vector<int32_t> tgt32_all;
    std::vector<uint16_t> tgt16_all;
    std::vector<uint8_t> mag_all;
    y.ab.clear();
    for (int ha = 0; ha < nh; ha++) {
        const int hb = ha ^ S;
        if (y.acnt[ha] == 0 || y.bcnt[hb] == 0) continue;
        for (int g = 0; g < nh; g++) {
            const int src = ha ^ g, hjb = hb ^ g;
            if (y.np_g[g] == 0 || y.acnt[src] == 0 || y.bcnt[hjb] == 0) continue;
            AbSub u;
            u.ha = ha;
            u.g = g;
            u.src = src;
            u.rows = y.acnt[ha];
            u.ns = y.bcnt[hjb];
            u.nt = y.bcnt[hb];
            std::vector<std::vector<uint32_t>> lists(u.rows);
            for (int i = 0; i < u.rows; i++) {
                const int Ia = y.asrc_h[y.d.aoff[ha] + i];
                for (int k = 0; k < s1; k++) {
                    const uint32_t e = conn[(size_t)Ia * s1 + k];
                    const int P = (int)((e >> 21) & 1023u);
                    if (P >= npair || pirr[P] != g) continue;
                    const uint32_t J = e & kConnIdxMask;
                    FCIB_CHECK(y.airr[J] == src, FCIB_ERR_NUMERIC, "blocked sigma: connection irrep mismatch");
                    if (y.aloc_h[J] < 0) continue;  // a source string no GAS determinant uses
                    lists[i].push_back((uint32_t)y.aloc_h[J] | ((uint32_t)P << 21) | (e & kSignBit));
                }
                u.kmax = std::max(u.kmax, (int)lists[i].size());
            }
            if (u.kmax == 0) {
                if (g != 0) continue;
                u.kmax = 1;  // the g = 0 launch writes the block (E0 C) even without connections
            }
            u.conn = conn_all.size();
            for (int i = 0; i < u.rows; i++)
                for (int k = 0; k < u.kmax; k++)
                    conn_all.push_back(k < (int)lists[i].size() ? lists[i][k] : (Pz << 21));
            // FP64 targets [ns][npg]: local target | sign, or kNoTarget
            u.tgt32 = tgt32_all.size();
            for (int j = 0; j < u.ns; j++) {
                const int Jb = y.bsrc_h[y.d.boff[hjb] + j];
                for (int col = 0; col < y.npg[g]; col++) {
                    int32_t v = kNoTarget;
                    if (col < y.np_g[g]) {
                        const int32_t e = tgt[(size_t)Jb * npp + plist[g][col]];
                        if (e != kNoTarget) {
                            const uint32_t I = (uint32_t)e & kConnIdxMask;
                            FCIB_CHECK(y.birr[I] == hb, FCIB_ERR_NUMERIC, "blocked sigma: target irrep mismatch");
                            if (y.bloc_h[I] >= 0) v = (int32_t)((uint32_t)y.bloc_h[I] | ((uint32_t)e & kSignBit));
                        }
                    }
                    tgt32_all.push_back(v);
                }
            }
            // tensor-core targets [noff8/8][ns padded to 128][8]: local target * 4 | sign, 0xFFFF none
            u.tgt16 = tgt16_all.size();
            if (u.nt <= kMaxBetaStrings) {
                const int ldp = (u.ns + kTcM - 1) / kTcM * kTcM;
                const int* pm = perm_all.data() + y.perm_off[g];
                for (int c8 = 0; c8 < y.noff8_g[g] / 8; c8++)
                    for (int j = 0; j < ldp; j++)
                        for (int uu = 0; uu < 8; uu++) {
                            uint16_t v = 0xFFFFu;
                            const int R = pm[8 * c8 + uu];
                            if (R >= 0 && j < u.ns) {
                                const int Jb = y.bsrc_h[y.d.boff[hjb] + j];
                                const int32_t e = tgt[(size_t)Jb * npp + R];
                                if (e != kNoTarget && y.bloc_h[(uint32_t)e & kConnIdxMask] >= 0)
                                    v = (uint16_t)(((uint32_t)y.bloc_h[(uint32_t)e & kConnIdxMask] << 2) |
                                                   ((uint32_t)e >> 31));
                            }
                            tgt16_all.push_back(v);
                        }
            }
            // contributions per target element of the tensor-core scatter: one per off-diagonal pair of
            // irrep g with exactly one orbital occupied whose source string (the other orbital occupied)
            // is in the blocks, plus the diagonal sum when g = 0
            u.mag = mag_all.size();
            for (int j = 0; j < u.nt; j++) {
                const uint32_t s = sb[y.bsrc_h[y.d.boff[hb] + j]];
                int cnt = g == 0 ? 1 : 0;
                for (int P : plist[g]) {
                    if (pp[P] == pq[P] || !(((s >> pp[P]) ^ (s >> pq[P])) & 1u)) continue;
                    const uint32_t J = s ^ (1u << pp[P]) ^ (1u << pq[P]);
                    cnt += y.bkeep[host_rank(J, n)] ? 1 : 0;
                }
                mag_all.push_back((uint8_t)cnt);
            }
            y.ab.push_back(u);
        }
    }
    y.conn.upload(conn_all, c.stream);
    y.tgt32.upload(tgt32_all, c.stream);
    y.tgt16.upload(tgt16_all, c.stream);
    y.mag.upload(mag_all, c.stream);
    FCIB_CUDA(cudaStreamSynchronize(c.stream));  // the host tables go out of scope
    // TF32 planes of the mixed sigma: alpha block h with rows padded to whole tiles
    y.plane_off.assign(nh, 0);
    y.ldp.assign(nh, 0);
    y.plane_total = 0;
    for (int h = 0; h < nh; h++) {
        y.ldp[h] = (y.bcnt[h ^ S] + kTcM - 1) / kTcM * kTcM;
        y.plane_off[h] = y.plane_total;
        FCIB_CHECK((uint64_t)y.acnt[h] * y.ldp[h] * sizeof(float2) < (1ull << 32), FCIB_ERR_UNSUPPORTED,
                   "blocked sigma: TF32 plane exceeds the 32-bit gather offsets");
        y.plane_total += (size_t)y.acnt[h] * y.ldp[h];
    }
}

void build_sym_space(Context& c) {
    SymSpace& y = c.sym;
    y.on = false;
    y.ab.clear();
    y.a2.clear();
    y.a1.clear();
    y.b2.clear();
    y.b1.clear();
    c.nvec = c.ndet;
    // blocks with point-group symmetry, and with GAS spaces (blocks of the kept strings) even in C1
    if (!c.opt.sym_blocked || (c.nirrep <= 1 && c.gas.ngas == 0)) return;
    const int nh = c.nirrep, S = c.irrep, n = c.n;
    std::vector<uint32_t> sa(c.nas), sb(c.nbs);
    FCIB_CUDA(cudaMemcpy(sa.data(), c.A.str.p, 4 * c.nas, cudaMemcpyDeviceToHost));
    FCIB_CUDA(cudaMemcpy(sb.data(), c.B.str.p, 4 * c.nbs, cudaMemcpyDeviceToHost));
    std::vector<uint8_t> keep_a(c.nas, 1), keep_b(c.nbs, 1);
    if (c.gas.ngas > 0) gas_keep_strings(c, sa, sb, keep_a, keep_b);
    SymDev& d = y.d;
    d = SymDev{};
    d.on = 1;
    d.nirrep = nh;
    d.irrep = S;
    for (int b = 0; b < 3; b++)
        for (int p = 0; p < n; p++)
            if (c.orbsym[p] >> b & 1) d.irrbit[b] |= 1u << p;
    // kept strings sorted by irrep (string order within an irrep); loc = -1 for the others
    auto sort_strings = [&](const std::vector<uint32_t>& s, const std::vector<uint8_t>& keep, std::vector<int>& irr,
                            int* cnt, int32_t* off, std::vector<int32_t>& src, std::vector<int32_t>& loc) {
        const size_t ns = s.size();
        irr.resize(ns);
        loc.assign(ns, -1);
        for (int h = 0; h < 8; h++) cnt[h] = 0;
        for (size_t i = 0; i < ns; i++) {
            irr[i] = sym_irrep_of(d, s[i]);
            if (keep[i]) loc[i] = cnt[irr[i]]++;
        }
        int32_t o = 0;
        for (int h = 0; h < 8; h++) {
            off[h] = o;
            o += cnt[h];
        }
        src.assign((size_t)o, 0);
        for (size_t i = 0; i < ns; i++)
            if (loc[i] >= 0) src[off[irr[i]] + loc[i]] = (int32_t)i;
    };
    sort_strings(sa, keep_a, y.airr, y.acnt, d.aoff, y.asrc_h, y.aloc_h);
    sort_strings(sb, keep_b, y.birr, y.bcnt, d.boff, y.bsrc_h, y.bloc_h);
    y.bkeep = keep_b;
    d.blk[0] = 0;
    y.blkT[0] = 0;
    for (int h = 0; h < 8; h++) {
        const bool in = h < nh;
        d.blk[h + 1] = d.blk[h] + (in ? (int64_t)y.acnt[h] * y.bcnt[h ^ S] : 0);
        y.blkT[h + 1] = y.blkT[h] + (in ? (int64_t)y.bcnt[h] * y.acnt[h ^ S] : 0);
        d.bcol[h] = in ? y.bcnt[h ^ S] : 0;
    }
    y.asrc.upload(y.asrc_h, c.stream);
    y.bsrc.upload(y.bsrc_h, c.stream);
    y.aloc.upload(y.aloc_h, c.stream);
    y.bloc.upload(y.bloc_h, c.stream);
    d.asrc = y.asrc.p;
    d.bsrc = y.bsrc.p;
    d.aloc = y.aloc.p;
    d.bloc = y.bloc.p;
    std::vector<uint32_t> bsorted(y.bsrc_h.size());
    for (size_t i = 0; i < bsorted.size(); i++) bsorted[i] = sb[y.bsrc_h[i]];
    y.bstr_sorted.upload(bsorted, c.stream);
    c.nvec = d.blk[nh];
    y.on = true;
    if (c.fold_h) build_ab_subs(c, sb);
    std::vector<uint32_t> rows_all;
    std::vector<uint16_t> labs_all;
    build_group_subs(c, c.A, true, false, y.a2, rows_all, labs_all);
    build_group_subs(c, c.B, false, false, y.b2, rows_all, labs_all);
    if (!c.fold_h) {
        build_group_subs(c, c.A, true, true, y.a1, rows_all, labs_all);
        build_group_subs(c, c.B, false, true, y.b1, rows_all, labs_all);
    }
    y.grow.upload(rows_all, c.stream);
    y.glab.upload(labs_all, c.stream);
    FCIB_CUDA(cudaStreamSynchronize(c.stream));
}

void sym_host_locate(const Context& c, int64_t I, int& h, int64_t& ia_loc, int64_t& ib_loc) {
    const SymDev& d = c.sym.d;
    h = 0;
    for (int x = 1; x < d.nirrep; x++)
        if (I >= d.blk[x]) h = x;
    const int64_t r = I - d.blk[h];
    ia_loc = r / d.bcol[h];
    ib_loc = r - ia_loc * d.bcol[h];
}

void sym_host_decode(const Context& c, int64_t I, int64_t& ia, int64_t& ib) {
    int h;
    int64_t i, j;
    sym_host_locate(c, I, h, i, j);
    ia = c.sym.asrc_h[c.sym.d.aoff[h] + i];
    ib = c.sym.bsrc_h[c.sym.d.boff[h ^ c.irrep] + j];
}

int64_t sym_host_encode(const Context& c, int64_t ia, int64_t ib) {
    const int h = c.sym.airr[ia];
    return c.sym.d.blk[h] + (int64_t)c.sym.aloc_h[ia] * c.sym.d.bcol[h] + c.sym.bloc_h[ib];
}

// ------------------------------------------------------------------------------------------
// blocked <-> C1 layout
// ------------------------------------------------------------------------------------------
__global__ void k_sym_expand(const double* __restrict__ v, double* __restrict__ c1, SymDev d, int64_t nvec, int nbs) {
    for (int64_t I = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; I < nvec; I += (int64_t)gridDim.x * blockDim.x) {
        int ia, ib;
        sym_decode(d, I, ia, ib);
        c1[(size_t)ia * nbs + ib] = v[I];
    }
}
__global__ void k_sym_compress(const double* __restrict__ c1, double* __restrict__ v, SymDev d, int64_t nvec,
                               int nbs) {
    for (int64_t I = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; I < nvec; I += (int64_t)gridDim.x * blockDim.x) {
        int ia, ib;
        sym_decode(d, I, ia, ib);
        v[I] = c1[(size_t)ia * nbs + ib];
    }
}

const double* c1_view(Context& c, const double* v, DBuf<double>& buf) {
    if (!c.sym.on) return v;
    buf.alloc((size_t)c.ndet);
    FCIB_CUDA(cudaMemsetAsync(buf.p, 0, sizeof(double) * c.ndet, c.stream));
    k_sym_expand<<<4 * c.num_sms, 256, 0, c.stream>>>(v, buf.p, c.sym.d, c.nvec, (int)c.nbs);
    FCIB_KCHECK();
    return buf.p;
}

void from_c1(Context& c, const double* c1, double* v) {
    if (!c.sym.on) {
        if (c1 != v) FCIB_CUDA(cudaMemcpyAsync(v, c1, sizeof(double) * c.ndet, cudaMemcpyDeviceToDevice, c.stream));
        return;
    }
    k_sym_compress<<<4 * c.num_sms, 256, 0, c.stream>>>(c1, v, c.sym.d, c.nvec, (int)c.nbs);
    FCIB_KCHECK();
}

}  // namespace fcib
