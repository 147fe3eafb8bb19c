// 3-particle reduced density matrices between two CI vectors (FP64): max_rdm_level = 3 of
// FCIVector::compute_rdms (forte/fci/fci_vector_rdm.cc:70-137; blocks :395-565).
//
// Index order and orientation follow the reference's loops, which take the creation indices from
// the list entries of the right vector.  For vectors (left, right):
//   g3aaa[p][q][r][s][t][u] = <right| a+_p a+_q a+_r a_u a_t a_s |left>        (all alpha)
//   g3aab: p, q, s, t alpha and r, u beta;   g3abb: p, s alpha and q, r, t, u beta;   g3bbb: beta
// so for one vector these are the usual 3-RDMs, and for two different vectors the tensor is the
// one with bra = right.  Below X is the bra (right) and Y the ket (left).
//
// Same-spin blocks: k_rdm_pairs<true> over (N-3)-electron groups.  A group K holds the strings
//   I_i = s_i a+_p a+_q a+_r K (p > q > r outside K, triple label lab_i); the Gram block
//   <X[I_i], Y[I_j]> over the other spin's strings, times s_i s_j, accumulates into
//   M[lab_i][lab_j], and the host writes each canonical element to its 36 antisymmetric positions.
// Mixed blocks: k_rdm3_pair_vo over (N-2)-electron groups of the pair spin.  For rows I_i, I_j of a
//   group, the one-body transition density of the other spin between the two rows,
//     gamma[r][u] = sum_Ic X[I_i][Ic] sum_{Ic = sgn a+_r a_u Jc} sgn Y[I_j][Jc],
//   accumulates into H[lab_i][r][lab_j][u] with the sign s_i s_j; the host expands the pair labels
//   to both orders.  abb and bbb run the same kernels on the transposed vectors (the operators
//   hold an even number of each spin's operators, so no phase appears).
#include "fcib_internal.h"

namespace fcib {

// (N-3)-electron groups of the k-electron strings of n orbitals: rows I | sign << 31 and triple
// labels lab(p, q, r) = C(p,3) + C(q,2) + r for p > q > r
static void triple_groups(int n, int k, std::vector<uint32_t>& rows, std::vector<uint16_t>& labs, int& ng, int& m) {
    const Binom& B = host_binom();
    ng = (int)B.c[n][k - 3];
    m = (int)B.c[n - k + 3][3];
    rows.assign((size_t)ng * m, 0u);
    labs.assign((size_t)ng * m, 0);
    for (int g = 0; g < ng; g++) {
        const uint32_t K = host_unrank((uint32_t)g, n, k - 3);
        int e = 0;
        for (int p = 0; p < n; p++) {
            if (K >> p & 1u) continue;
            for (int q = 0; q < p; q++) {
                if (K >> q & 1u) continue;
                for (int r = 0; r < q; r++) {
                    if (K >> r & 1u) continue;
                    // a+_p a+_q a+_r K: r first, then q (one more electron below it), then p (two more)
                    const int below = __builtin_popcount(K & ((1u << r) - 1u)) + __builtin_popcount(K & ((1u << q) - 1u)) +
                                      __builtin_popcount(K & ((1u << p) - 1u)) + 3;
                    const uint32_t I = host_rank(K | 1u << p | 1u << q | 1u << r, n);
                    rows[(size_t)g * m + e] = I | ((uint32_t)(below & 1) << 31);
                    labs[(size_t)g * m + e] = (uint16_t)(B.c[p][3] + B.c[q][2] + r);
                    e++;
                }
            }
        }
    }
}

// One CTA per (group, bra row i): the bra row X[I_i][:] sits in shared memory; for every ket row
// j of the group the column-spin transition density is accumulated in shared memory (FP64
// shared atomics) and added to H[lab_i][r][lab_j][u] with the sign s_i s_j.
__global__ void __launch_bounds__(kRdmThreads)
    k_rdm3_pair_vo(const double* __restrict__ X, const double* __restrict__ Y, int ncol,
                   const uint32_t* __restrict__ rows, const uint16_t* __restrict__ labs, int ng, int m, int npl,
                   const uint32_t* __restrict__ strC, const uint32_t* __restrict__ connC, int s1c, int n,
                   double* __restrict__ H) {
    extern __shared__ __align__(16) unsigned char rdm3_smem[];
    double* xrow = reinterpret_cast<double*>(rdm3_smem);  // [ncol]
    double* gam = xrow + ncol;                             // [n * n]
    int* ptab = reinterpret_cast<int*>(gam + n * n);       // [n (n + 1) / 2]
    fill_pair_table(ptab, n);
    const int nn = n * n;
    for (int item = blockIdx.x; item < ng * m; item += gridDim.x) {
        const int g = item / m, i = item - g * m;
        const uint32_t rI = rows[(size_t)g * m + i];
        const int li = labs[(size_t)g * m + i];
        __syncthreads();
        const double* xsrc = X + (size_t)(rI & 0x7FFFFFFFu) * ncol;
        for (int x = threadIdx.x; x < ncol; x += blockDim.x) xrow[x] = xsrc[x];
        for (int j = 0; j < m; j++) {
            const uint32_t rJ = rows[(size_t)g * m + j];
            const int lj = labs[(size_t)g * m + j];
            const double* yrow = Y + (size_t)(rJ & 0x7FFFFFFFu) * ncol;
            for (int x = threadIdx.x; x < nn; x += blockDim.x) gam[x] = 0.0;
            __syncthreads();
            for (int ic = threadIdx.x; ic < ncol; ic += blockDim.x) {
                const double xv = xrow[ic];
                if (xv == 0.0) continue;
                const uint32_t sI = strC[ic];
                const uint32_t* cn = connC + (size_t)ic * s1c;
                for (int kk = 0; kk < s1c; kk++) {
                    const uint32_t e = cn[kk];
                    int r, u;
                    created_annihilated(sI, ptab[(e >> 21) & 1023u], r, u);
                    const double v = xv * yrow[e & kConnIdxMask];
                    atomicAdd(&gam[r * n + u], (e & kSignBit) ? -v : v);
                }
            }
            __syncthreads();
            const double sg = ((rI ^ rJ) >> 31) ? -1.0 : 1.0;
            for (int x = threadIdx.x; x < nn; x += blockDim.x) {
                const double v = gam[x];
                if (v == 0.0) continue;
                const int r = x / n, u = x - r * n;
                atomicAdd(H + (((size_t)li * n + r) * npl + lj) * n + u, sg * v);
            }
            __syncthreads();
        }
    }
}

// Same-spin block on the row spin of X, Y (rows x ncol): M[lab][lab'] over triple labels
static void rdm3_same(Context& c, const double* X, const double* Y, int ncol, int k, double* M, int nl3) {
    if (k < 3 || ncol == 0) return;
    std::vector<uint32_t> hr;
    std::vector<uint16_t> hl;
    int ng = 0, m = 0;
    triple_groups(c.n, k, hr, hl, ng, m);
    DBuf<uint32_t> rows;
    DBuf<uint16_t> labs;
    rows.upload(hr, c.stream);
    labs.upload(hl, c.stream);
    const size_t smem = 2 * (size_t)m * (kPairTB + 1) * 8 + (size_t)m * 8;
    FCIB_CHECK(smem + 1024 <= (size_t)c.smem_optin, FCIB_ERR_UNSUPPORTED, "3-RDMs: triple group exceeds shared memory");
    FCIB_CUDA(cudaFuncSetAttribute(k_rdm_pairs<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int per_sm = std::max(1, std::min(8, (int)(c.smem_per_sm / (smem + 1024))));
    const int grid = std::min(ng, per_sm * c.num_sms);
    k_rdm_pairs<true><<<grid, kRdmThreads, smem, c.stream>>>(X, Y, ncol, rows.p, labs.p, ng, m, nl3, M);
    FCIB_KCHECK();
    FCIB_CUDA(cudaStreamSynchronize(c.stream));  // the tables are freed on return
}

// Mixed block: pair groups T of the row spin, column-spin tables Tc; H[npl][n][npl][n]
static void rdm3_mixed(Context& c, const double* X, const double* Y, int ncol, const SpinTables& T,
                       const SpinTables& Tc, double* H) {
    if (T.ng2 == 0 || Tc.s1 == 0 || ncol == 0) return;
    const int n = c.n, npl = n * (n - 1) / 2, npair = n * (n + 1) / 2;
    const size_t smem = (size_t)ncol * 8 + (size_t)n * n * 8 + (size_t)npair * 4;
    FCIB_CHECK(smem + 1024 <= (size_t)c.smem_optin, FCIB_ERR_UNSUPPORTED, "3-RDMs: CI row exceeds shared memory");
    FCIB_CUDA(cudaFuncSetAttribute(k_rdm3_pair_vo, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int per_sm = std::max(1, std::min(8, (int)(c.smem_per_sm / (smem + 1024))));
    const int items = T.ng2 * T.g2;
    const int grid = std::min(items, per_sm * c.num_sms);
    k_rdm3_pair_vo<<<grid, kRdmThreads, smem, c.stream>>>(X, Y, ncol, T.g2row.p, T.g2lab.p, T.ng2, T.g2, npl,
                                                         Tc.str.p, Tc.conn.p, Tc.s1, n, H);
    FCIB_KCHECK();
}

// sign of the permutation taking (a, b, c) to descending order, and the sorted label
static inline int triple_key(int a, int b, int c, const Binom& B, int& lab) {
    if (a == b || b == c || a == c) return 0;
    int s = 1;
    if (a < b) { std::swap(a, b); s = -s; }
    if (b < c) { std::swap(b, c); s = -s; }
    if (a < b) { std::swap(a, b); s = -s; }
    lab = (int)(B.c[a][3] + B.c[b][2] + c);
    return s;
}
static inline int pair_key(int a, int b, int& lab) {
    if (a == b) return 0;
    if (a > b) { lab = a * (a - 1) / 2 + b; return 1; }
    lab = b * (b - 1) / 2 + a;
    return -1;
}

// 3-RDM blocks between device vectors in C1 layout: left = Lv, right = Rv (reference orientation)
void compute_rdms3(Context& c, const double* Lv, const double* Rv, Rdm3Blocks& out) {
    const int n = c.n, nas = (int)c.nas, nbs = (int)c.nbs;
    const int npl = n * (n - 1) / 2;
    const Binom& B = host_binom();
    const int nl3 = (int)B.c[n][3];
    const size_t n6 = (size_t)n * n * n * n * n * n;
    const size_t sz3 = (size_t)nl3 * nl3, szm = (size_t)npl * n * npl * n;
    DBuf<double> acc;
    acc.alloc(2 * sz3 + 2 * szm);
    FCIB_CUDA(cudaMemsetAsync(acc.p, 0, sizeof(double) * (2 * sz3 + 2 * szm), c.stream));
    double* m3a = acc.p;
    double* m3b = m3a + sz3;
    double* haab = m3b + sz3;
    double* habb = haab + szm;
    const double* X = Rv;  // bra
    const double* Y = Lv;  // ket
    rdm3_same(c, X, Y, nbs, c.na, m3a, nl3);
    if (c.na >= 2 && c.nb >= 1) rdm3_mixed(c, X, Y, nbs, c.A, c.B, haab);
    if ((c.nb >= 3) || (c.nb >= 2 && c.na >= 1)) {
        DBuf<double> xt, yt;
        xt.alloc((size_t)c.ndet);
        transpose(c, X, xt.p, nas, nbs);
        const double* ytp = xt.p;
        if (Y != X) {
            yt.alloc((size_t)c.ndet);
            transpose(c, Y, yt.p, nas, nbs);
            ytp = yt.p;
        }
        rdm3_same(c, xt.p, ytp, nas, c.nb, m3b, nl3);
        if (c.nb >= 2 && c.na >= 1) rdm3_mixed(c, xt.p, ytp, nas, c.B, c.A, habb);
        FCIB_CUDA(cudaStreamSynchronize(c.stream));
    }
    std::vector<double> h(2 * sz3 + 2 * szm);
    FCIB_CUDA(cudaMemcpyAsync(h.data(), acc.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c.stream));
    FCIB_CUDA(cudaStreamSynchronize(c.stream));
    const double* Ma = h.data();
    const double* Mb = Ma + sz3;
    const double* Ha = Mb + sz3;
    const double* Hb = Ha + szm;
    out.n = n;
    out.aaa.assign(n6, 0.0);
    out.aab.assign(n6, 0.0);
    out.abb.assign(n6, 0.0);
    out.bbb.assign(n6, 0.0);
    auto six = [n](int p, int q, int r, int s, int t, int u) {
        return (((((size_t)p * n + q) * n + r) * n + s) * n + t) * n + u;
    };
    auto hidx = [n, npl](int li, int r, int lj, int u) { return (((size_t)li * n + r) * npl + lj) * n + u; };
    for (int p = 0; p < n; p++)
        for (int q = 0; q < n; q++)
            for (int r = 0; r < n; r++) {
                int l1 = 0, lpq = 0, lqr = 0;
                const int e1 = triple_key(p, q, r, B, l1);
                const int epq = pair_key(p, q, lpq);
                const int eqr = pair_key(q, r, lqr);
                for (int s = 0; s < n; s++)
                    for (int t = 0; t < n; t++)
                        for (int u = 0; u < n; u++) {
                            const size_t o = six(p, q, r, s, t, u);
                            if (e1) {
                                int l2 = 0;
                                const int e2 = triple_key(s, t, u, B, l2);
                                if (e2) {
                                    out.aaa[o] = e1 * e2 * Ma[(size_t)l1 * nl3 + l2];
                                    out.bbb[o] = e1 * e2 * Mb[(size_t)l1 * nl3 + l2];
                                }
                            }
                            // aab: <a+_p a+_q (alpha) a+_r a_u (beta) a_t a_s (alpha)>
                            if (epq) {
                                int lst = 0;
                                const int est = pair_key(s, t, lst);
                                if (est) out.aab[o] = epq * est * Ha[hidx(lpq, r, lst, u)];
                            }
                            // abb: <a+_p (alpha) a+_q a+_r a_u a_t (beta) a_s (alpha)>
                            if (eqr) {
                                int ltu = 0;
                                const int etu = pair_key(t, u, ltu);
                                if (etu) out.abb[o] = eqr * etu * Hb[hidx(lqr, p, ltu, s)];
                            }
                        }
            }
}

}  // namespace fcib
