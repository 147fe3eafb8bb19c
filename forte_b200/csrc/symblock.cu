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
//
// With GAS spaces (gas.cu) the blocks hold the strings of the GAS determinants only, sorted within
// an irrep by occupation pattern, so each pattern is a run of rows (alpha) or columns (beta).  The
// sub-problems then also split by the pattern run of the target rows and of the source columns,
// and keep only those through which a GAS determinant receives a contribution: source columns one
// replacement away from a column pattern that the rows pair with, and connections to source rows
// whose pattern pairs with the source columns.  Same-spin groups split by the column run and keep
// the members whose pattern pairs with it.  The first sub-problem of a row run writes it; elements
// outside the GAS space are left to the mask.  The work then follows the GAS determinants rather
// than the products of their strings.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "fcib_internal.h"

namespace fcib {

static int sb_pad8(int x) { return (x + 7) / 8 * 8; }

// same-spin groups of one spin and kind, split by the irrep of their strings and, per column
// pattern run of the block (one run without GAS), restricted to the members whose pattern some GAS
// determinant pairs with that run's pattern (the others meet zeros there and are masked there)
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
    const std::vector<int>& pat = alpha ? y.apat : y.bpat;
    const int nh = c.nirrep, S = c.irrep;
    // parts[h][r]: the groups of rows of irrep h for column run r of the block
    std::vector<std::vector<std::vector<std::vector<std::pair<uint32_t, uint16_t>>>>> parts(nh);
    for (int h = 0; h < nh; h++) parts[h].resize((alpha ? y.brun[h ^ S] : y.arun[h ^ S]).size());
    struct Member {
        uint32_t e;
        uint16_t lab;
        int pat;
    };
    std::vector<std::vector<Member>> bucket(nh);
    for (int gi = 0; gi < ng; gi++) {
        for (auto& b : bucket) b.clear();
        for (int m = 0; m < G; m++) {
            const uint32_t e = rows[(size_t)gi * G + m];
            if (e == kNullRow) continue;
            const uint32_t I = e & kConnIdxMask;
            if (loc[I] < 0) continue;  // a string no GAS determinant uses: its rows and columns are absent
            bucket[irr[I]].push_back({(uint32_t)loc[I] | (e & kSignBit), labs[(size_t)gi * G + m], pat[I]});
        }
        for (int h = 0; h < nh; h++) {
            if (bucket[h].empty()) continue;
            const std::vector<PatRange>& cr = alpha ? y.brun[h ^ S] : y.arun[h ^ S];
            for (size_t r = 0; r < cr.size(); r++) {
                std::vector<std::pair<uint32_t, uint16_t>> part;
                for (const Member& x : bucket[h]) {
                    const int pa = alpha ? x.pat : cr[r].pat, pb = alpha ? cr[r].pat : x.pat;
                    if (y.allowed[(size_t)pa * y.npb + pb]) part.push_back({x.e, x.lab});
                }
                if (!part.empty()) parts[h][r].push_back(std::move(part));
            }
        }
    }
    for (int h = 0; h < nh; h++) {
        const std::vector<PatRange>& cr = alpha ? y.brun[h ^ S] : y.arun[h ^ S];
        const int ld = alpha ? y.bcnt[h ^ S] : y.acnt[h ^ S];
        for (size_t r = 0; r < cr.size(); r++) {
            if (parts[h][r].empty()) continue;
            GroupSub s;
            s.ngroups = (int)parts[h][r].size();
            for (auto& p : parts[h][r]) s.G = std::max(s.G, (int)p.size());
            s.ncols = cr[r].count;
            s.ld = ld;
            s.blk = (alpha ? y.d.blk[h] : y.blkT[h]) + cr[r].start;
            s.off = rows_all.size();
            for (auto& p : parts[h][r])
                for (int m = 0; m < s.G; m++) {
                    rows_all.push_back(m < (int)p.size() ? p[m].first : kNullRow);
                    labs_all.push_back(m < (int)p.size() ? p[m].second : (uint16_t)0);
                }
            out.push_back(s);
        }
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
    auto allowed = [&](int pa, int pb) { return y.allowed[(size_t)pa * y.npb + pb] != 0; };
    for (int ha = 0; ha < nh; ha++) {
        const int hb = ha ^ S;
        if (y.acnt[ha] == 0 || y.bcnt[hb] == 0) continue;
        // target rows: one alpha pattern run at a time (the whole block without GAS)
        for (const PatRange& ar : y.arun[ha]) {
            bool written = false;  // the first sub-problem of these rows writes them
            // patterns of target columns that GAS determinants pair with these rows
            std::vector<int> tcols;
            for (const PatRange& br : y.brun[hb])
                if (allowed(ar.pat, br.pat)) tcols.push_back(br.pat);
            for (int g = 0; g < nh; g++) {
                const int src = ha ^ g, hjb = hb ^ g;
                if (y.np_g[g] == 0 || y.acnt[src] == 0 || y.bcnt[hjb] == 0) continue;
                for (const PatRange& sr : y.brun[hjb]) {
                    // useful when the source columns reach a column pattern of these rows and some
                    // alpha pattern one replacement away from the rows' pairs with the source columns
                    bool reach_t = false, reach_s = false;
                    for (int pb : tcols) reach_t = reach_t || y.breach[(size_t)sr.pat * y.npb + pb];
                    for (int pa = 0; pa < y.npa; pa++)
                        reach_s = reach_s || (y.areach[(size_t)ar.pat * y.npa + pa] && allowed(pa, sr.pat));
                    const bool writer = !written && g == 0;
                    if (!(reach_t && reach_s) && !writer) continue;
                    AbSub u;
                    u.ha = ha;
                    u.g = g;
                    u.src = src;
                    u.row0 = ar.start;
                    u.rows = ar.count;
                    u.col0 = sr.start;
                    u.ns = sr.count;
                    u.lds = y.bcnt[hjb];
                    u.nt = y.bcnt[hb];
                    u.diag_off = g == 0 ? sr.start : 0;
                    // connections of the rows through pairs of irrep g to sources whose pattern the
                    // source columns pair with (other sources hold zeros there)
                    std::vector<std::vector<uint32_t>> lists(u.rows);
                    for (int i = 0; i < u.rows; i++) {
                        const int Ia = y.asrc_h[y.d.aoff[ha] + ar.start + i];
                        for (int k = 0; k < s1; k++) {
                            const uint32_t e = conn[(size_t)Ia * s1 + k];
                            const int P = (int)((e >> 21) & 1023u);
                            if (P >= npair || pirr[P] != g) continue;
                            const uint32_t J = e & kConnIdxMask;
                            FCIB_CHECK(y.airr[J] == src, FCIB_ERR_NUMERIC, "blocked sigma: connection irrep mismatch");
                            if (y.aloc_h[J] < 0 || !allowed(y.apat[J], sr.pat)) continue;
                            lists[i].push_back((uint32_t)y.aloc_h[J] | ((uint32_t)P << 21) | (e & kSignBit));
                        }
                        u.kmax = std::max(u.kmax, (int)lists[i].size());
                    }
                    if (u.kmax == 0) {
                        if (!writer) continue;
                        u.kmax = 1;  // the writer writes its rows (E0 C) even without connections
                    }
                    u.accumulate = written ? 1 : 0;
                    written = true;
                    u.conn = conn_all.size();
                    for (int i = 0; i < u.rows; i++)
                        for (int k = 0; k < u.kmax; k++)
                            conn_all.push_back(k < (int)lists[i].size() ? lists[i][k] : (Pz << 21));
                    // FP64 targets [ns][npg]: target column in the whole row | sign, or kNoTarget
                    u.tgt32 = tgt32_all.size();
                    for (int j = 0; j < u.ns; j++) {
                        const int Jb = y.bsrc_h[y.d.boff[hjb] + sr.start + j];
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
                    // tensor-core targets [noff8/8][ns padded to 128][8]: target column * 4 | sign, 0xFFFF none
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
                                        const int Jb = y.bsrc_h[y.d.boff[hjb] + sr.start + j];
                                        const int32_t e = tgt[(size_t)Jb * npp + R];
                                        if (e != kNoTarget && y.bloc_h[(uint32_t)e & kConnIdxMask] >= 0)
                                            v = (uint16_t)(((uint32_t)y.bloc_h[(uint32_t)e & kConnIdxMask] << 2) |
                                                           ((uint32_t)e >> 31));
                                    }
                                    tgt16_all.push_back(v);
                                }
                    }
                    // contributions per target element of the tensor-core scatter: one per off-diagonal
                    // pair of irrep g with exactly one orbital occupied whose source string (the other
                    // orbital occupied) is in the source columns, plus the diagonal sum when g = 0 and
                    // the element's own string is a source column
                    u.mag = mag_all.size();
                    for (int j = 0; j < u.nt; j++) {
                        const int Ib = y.bsrc_h[y.d.boff[hb] + j];
                        const uint32_t s = sb[Ib];
                        int cnt = (g == 0 && y.bpat[Ib] == sr.pat) ? 1 : 0;
                        for (int P : plist[g]) {
                            if (pp[P] == pq[P] || !(((s >> pp[P]) ^ (s >> pq[P])) & 1u)) continue;
                            const uint32_t J = s ^ (1u << pp[P]) ^ (1u << pq[P]);
                            cnt += y.bpat[host_rank(J, n)] == sr.pat ? 1 : 0;
                        }
                        mag_all.push_back((uint8_t)cnt);
                    }
                    y.ab.push_back(u);
                }
            }
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
    // occupation patterns: with GAS spaces those of the GAS determinants (strings of no GAS
    // determinant are dropped), otherwise one pattern 0 for every string
    y.apat.assign(c.nas, 0);
    y.bpat.assign(c.nbs, 0);
    y.npa = y.npb = 1;
    y.allowed.assign(1, 1);
    y.areach.assign(1, 1);
    y.breach.assign(1, 1);
    if (c.gas.ngas > 0)
        gas_string_patterns(c, sa, sb, y.apat, y.bpat, y.npa, y.npb, y.allowed, y.areach, y.breach);
    SymDev& d = y.d;
    d = SymDev{};
    d.on = 1;
    d.nirrep = nh;
    d.irrep = S;
    for (int b = 0; b < 3; b++)
        for (int p = 0; p < n; p++)
            if (c.orbsym[p] >> b & 1) d.irrbit[b] |= 1u << p;
    // kept strings sorted by irrep, then by pattern, then in string order; loc = -1 for the others
    auto sort_strings = [&](const std::vector<uint32_t>& s, const std::vector<int>& pat, int npat, std::vector<int>& irr,
                            int* cnt, int32_t* off, std::vector<int32_t>& src, std::vector<int32_t>& loc,
                            std::vector<PatRange>* run) {
        const size_t ns = s.size();
        irr.resize(ns);
        loc.assign(ns, -1);
        std::vector<std::vector<std::vector<int32_t>>> by(8, std::vector<std::vector<int32_t>>(npat));
        for (size_t i = 0; i < ns; i++) {
            irr[i] = sym_irrep_of(d, s[i]);
            if (pat[i] >= 0) by[irr[i]][pat[i]].push_back((int32_t)i);
        }
        int32_t o = 0;
        src.clear();
        for (int h = 0; h < 8; h++) {
            off[h] = o;
            cnt[h] = 0;
            run[h].clear();
            for (int q = 0; q < npat; q++) {
                if (by[h][q].empty()) continue;
                run[h].push_back(PatRange{q, cnt[h], (int)by[h][q].size()});
                for (int32_t i : by[h][q]) {
                    loc[i] = cnt[h]++;
                    src.push_back(i);
                }
            }
            o += cnt[h];
        }
    };
    sort_strings(sa, y.apat, y.npa, y.airr, y.acnt, d.aoff, y.asrc_h, y.aloc_h, y.arun);
    sort_strings(sb, y.bpat, y.npb, y.birr, y.bcnt, d.boff, y.bsrc_h, y.bloc_h, y.brun);
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
