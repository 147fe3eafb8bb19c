// 1- and 2-particle reduced density matrices between two CI vectors (FP64).
//
// Conventions are those of FCIVector::compute_rdms (forte/fci/fci_vector_rdm.cc:43-145):
//   g1[p][q]         = <L| a+_p a_q |R>                                       (:151-200)
//   g2aa[p][q][r][s] = <L| a+_p a+_q a_s a_r |R>, from the (pq) >= (rs) pair elements only,
//                      written to the 4 / 8 antisymmetric positions            (:206-306)
//   g2ab[p][q][r][s] = <L| a+_{p alpha} a+_{q beta} a_{s beta} a_{r alpha} |R> (:308-393)
//
// k_rdm_vo: one CTA per bra string J of the row spin.  The bra row L[J][:] sits in shared memory;
//   for each single replacement J = +-a+_p a_q I (the connection table of J) the CTA forms the
//   dot <L[J], R[I]> (1-RDM) and, for the alpha-beta 2-RDM, scatters
//   L[J][Jc] * R[I][Ic] * signs over the column-spin replacements Jc = +-a+_r a_s Ic into a
//   shared-memory block acc[k][r*n+s] (FP64 shared atomics), flushed once per chunk of
//   connections with global atomics.  Work: N_det * s1 dot terms and N_det * s1^2 scatter terms.
// k_rdm_pairs: one CTA per (N-2)-electron group K.  Its m rows I_i = s_i a+_p a+_q K give all
//   double replacements inside the group: <I_i| a+_p a+_q a_s a_r |I_j> = s_i s_j.  The CTA
//   forms the Gram block G[i][j] = <L[I_i], R[I_j]> over the column spin (tiles of 32 columns in
//   shared memory) for lab_i >= lab_j and adds s_i s_j G[i][j] to M[lab_i][lab_j].
//   Work: 2 * N_str * d2 * N_col FLOP, like the same-spin sigma term.

namespace fcib {

constexpr int kRdmThreads = 256;
constexpr int kPairTB = 32;   // columns per shared-memory tile in k_rdm_pairs
constexpr int kPairPer = 8;   // (i, j) elements per thread per pass in k_rdm_pairs

// pair index P = p(p+1)/2 + q (p >= q) -> p << 8 | q, built in shared memory by each CTA
__device__ __forceinline__ void fill_pair_table(int* ptab, int n) {
    const int npair = n * (n + 1) / 2;
    for (int P = threadIdx.x; P < npair; P += blockDim.x) {
        int r = 0;
        while ((r + 1) * (r + 2) / 2 <= P) r++;
        ptab[P] = r << 8 | (P - r * (r + 1) / 2);
    }
}

// Orbitals (p, q) of a connection-table entry of string sJ: J = +-a+_p a_q I, p occupied in J
// only, q in I only; a diagonal entry (J == I) is the number operator of p = q.
__device__ __forceinline__ void created_annihilated(uint32_t sJ, int code, int& p, int& q) {
    const int hi = code >> 8, lo = code & 0xFF;
    if (hi == lo) {
        p = q = hi;
    } else if (sJ >> hi & 1u) {
        p = hi;
        q = lo;
    } else {
        p = lo;
        q = hi;
    }
}

template <bool AB>
__global__ void __launch_bounds__(kRdmThreads)
    k_rdm_vo(const double* __restrict__ L, const double* __restrict__ R, int nrow, int ncol,
             const uint32_t* __restrict__ strR, const uint32_t* __restrict__ connR, int s1r,
             const uint32_t* __restrict__ strC, const uint32_t* __restrict__ connC, int s1c, int n, int kc,
             double* __restrict__ g1, double* __restrict__ g2) {
    extern __shared__ __align__(16) unsigned char rdm_smem[];
    double* lrow = reinterpret_cast<double*>(rdm_smem);  // [ncol]
    double* d1 = lrow + ncol;                             // [kc]
    double* acc = d1 + kc;                                // [kc][n*n] (alpha-beta only)
    int* ptab = reinterpret_cast<int*>(acc + (AB ? (size_t)kc * n * n : 0));
    fill_pair_table(ptab, n);
    const int nn = n * n;
    for (int J = blockIdx.x; J < nrow; J += gridDim.x) {
        __syncthreads();
        for (int i = threadIdx.x; i < ncol; i += blockDim.x) lrow[i] = L[(size_t)J * ncol + i];
        const uint32_t sJ = strR[J];
        for (int k0 = 0; k0 < s1r; k0 += kc) {
            const int kn = min(kc, s1r - k0);
            for (int i = threadIdx.x; i < kn; i += blockDim.x) d1[i] = 0.0;
            if (AB)
                for (int i = threadIdx.x; i < kn * nn; i += blockDim.x) acc[i] = 0.0;
            __syncthreads();
            for (int kk = 0; kk < kn; kk++) {
                const uint32_t e = connR[(size_t)J * s1r + k0 + kk];
                const double* rrow = R + (size_t)(e & 0x1FFFFFu) * ncol;
                const bool neg = e >> 31;
                double* ak = acc + (size_t)kk * nn;
                double dot = 0.0;
                for (int Ic = threadIdx.x; Ic < ncol; Ic += blockDim.x) {
                    double cr = rrow[Ic];
                    if (neg) cr = -cr;
                    dot = fma(lrow[Ic], cr, dot);
                    if (AB && cr != 0.0) {
                        // column replacements Jc = +-a+_r a_s Ic: the entries of Ic's table, with
                        // s occupied in Ic and r in Jc (same sign in both directions)
                        const uint32_t sIc = strC[Ic];
                        const uint32_t* cc = connC + (size_t)Ic * s1c;
                        for (int m = 0; m < s1c; m++) {
                            const uint32_t f = cc[m];
                            double v = lrow[f & 0x1FFFFFu];
                            if (v == 0.0) continue;
                            if (f >> 31) v = -v;
                            const int code = ptab[(f >> 21) & 0x3FFu];
                            const int hi = code >> 8, lo = code & 0xFF;
                            int r = hi, s = hi;
                            if (hi != lo) {
                                if (sIc >> hi & 1u) {
                                    r = lo;
                                    s = hi;
                                } else {
                                    r = hi;
                                    s = lo;
                                }
                            }
                            atomicAdd(ak + r * n + s, v * cr);
                        }
                    }
                }
                for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
                if ((threadIdx.x & 31) == 0 && dot != 0.0) atomicAdd(d1 + kk, dot);
            }
            __syncthreads();
            for (int i = threadIdx.x; i < kn; i += blockDim.x) {
                if (d1[i] == 0.0) continue;
                const uint32_t e = connR[(size_t)J * s1r + k0 + i];
                int p, q;
                created_annihilated(sJ, ptab[(e >> 21) & 0x3FFu], p, q);
                atomicAdd(g1 + p * n + q, d1[i]);
            }
            if (AB) {
                for (int i = threadIdx.x; i < kn * nn; i += blockDim.x) {
                    const double v = acc[i];
                    if (v == 0.0) continue;
                    const int kk = i / nn, rs = i - kk * nn, r = rs / n, s = rs - r * n;
                    const uint32_t e = connR[(size_t)J * s1r + k0 + kk];
                    int p, q;
                    created_annihilated(sJ, ptab[(e >> 21) & 0x3FFu], p, q);
                    atomicAdd(g2 + (((size_t)p * n + r) * n + q) * n + s, v);
                }
            }
            __syncthreads();
        }
    }
}

// FULL: every (i, j) element (the 3-RDM triple groups); otherwise only lab_i >= lab_j, the half the
// reference's 2-RDM loops form
template <bool FULL>
__global__ void __launch_bounds__(kRdmThreads)
    k_rdm_pairs(const double* __restrict__ L, const double* __restrict__ R, int ncol,
                const uint32_t* __restrict__ rows, const uint16_t* __restrict__ labs, int ng, int m, int npl,
                double* __restrict__ M) {
    extern __shared__ __align__(16) unsigned char rdm_smem[];
    constexpr int LD = kPairTB + 1;
    double* Lt = reinterpret_cast<double*>(rdm_smem);  // [m][LD]
    double* Rt = Lt + (size_t)m * LD;                   // [m][LD]
    uint32_t* rI = reinterpret_cast<uint32_t*>(Rt + (size_t)m * LD);
    int* lab = reinterpret_cast<int*>(rI + m);
    const int mm = m * m;
    for (int g = blockIdx.x; g < ng; g += gridDim.x) {
        __syncthreads();
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            rI[i] = rows[(size_t)g * m + i];
            lab[i] = labs[(size_t)g * m + i];
        }
        for (int t0 = 0; t0 < mm; t0 += kRdmThreads * kPairPer) {
            double acc[kPairPer];
#pragma unroll
            for (int u = 0; u < kPairPer; u++) acc[u] = 0.0;
            for (int c0 = 0; c0 < ncol; c0 += kPairTB) {
                const int cn = min(kPairTB, ncol - c0);
                __syncthreads();
                for (int x = threadIdx.x; x < m * kPairTB; x += blockDim.x) {
                    const int i = x / kPairTB, cidx = x - i * kPairTB;
                    double lv = 0.0, rv = 0.0;
                    if (cidx < cn) {
                        const size_t base = (size_t)(rI[i] & 0x7FFFFFFFu) * ncol + c0 + cidx;
                        lv = L[base];
                        rv = R[base];
                    }
                    Lt[i * LD + cidx] = lv;
                    Rt[i * LD + cidx] = rv;
                }
                __syncthreads();
#pragma unroll
                for (int u = 0; u < kPairPer; u++) {
                    const int t = t0 + u * kRdmThreads + threadIdx.x;
                    if (t >= mm) continue;
                    const int i = t / m, j = t - i * m;
                    if (!FULL && lab[i] < lab[j]) continue;
                    const double* li = Lt + i * LD;
                    const double* rj = Rt + j * LD;
                    double a = acc[u];
#pragma unroll 8
                    for (int cidx = 0; cidx < kPairTB; cidx++) a = fma(li[cidx], rj[cidx], a);
                    acc[u] = a;
                }
            }
#pragma unroll
            for (int u = 0; u < kPairPer; u++) {
                const int t = t0 + u * kRdmThreads + threadIdx.x;
                if (t >= mm) continue;
                const int i = t / m, j = t - i * m;
                if ((!FULL && lab[i] < lab[j]) || acc[u] == 0.0) continue;
                const double sg = ((rI[i] ^ rI[j]) >> 31) ? -1.0 : 1.0;
                atomicAdd(M + (size_t)lab[i] * npl + lab[j], sg * acc[u]);
            }
        }
    }
}

static void rdm_vo(Context& c, const double* L, const double* R, int nrow, int ncol, const SpinTables& Tr,
                   const SpinTables& Tc, bool ab, double* g1, double* g2) {
    if (Tr.s1 == 0 || nrow == 0 || ncol == 0) return;
    const int n = c.n, nn = n * n, npair = n * (n + 1) / 2;
    const size_t budget = (size_t)c.smem_optin - 1024;
    const size_t fixed = (size_t)ncol * 8 + (size_t)npair * 4 + 64;
    int kc = Tr.s1;
    if (ab) {
        FCIB_CHECK(fixed + 8 * (size_t)(nn + 1) <= budget, FCIB_ERR_UNSUPPORTED,
                   "RDMs: a CI row and one accumulator block exceed shared memory");
        kc = (int)std::min<size_t>(Tr.s1, (budget - fixed) / (8 * (size_t)(nn + 1)));
    }
    const size_t smem = (size_t)ncol * 8 + (size_t)kc * 8 + (ab ? (size_t)kc * nn * 8 : 0) + (size_t)npair * 4;
    FCIB_CHECK(smem <= budget, FCIB_ERR_UNSUPPORTED, "RDMs: CI row exceeds shared memory");
    auto kern = ab ? k_rdm_vo<true> : k_rdm_vo<false>;
    FCIB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int per_sm = std::max(1, std::min(8, (int)(c.smem_per_sm / (smem + 1024))));
    const int grid = std::min(nrow, per_sm * c.num_sms);
    kern<<<grid, kRdmThreads, smem, c.stream>>>(L, R, nrow, ncol, Tr.str.p, Tr.conn.p, Tr.s1, Tc.str.p,
                                                Tc.s1 > 0 ? Tc.conn.p : nullptr, Tc.s1, n, kc, g1, g2);
    FCIB_KCHECK();
}

static void rdm_pairs(Context& c, const double* L, const double* R, int ncol, const SpinTables& T, double* M) {
    if (T.ng2 == 0 || ncol == 0) return;
    const int m = T.g2, npl = c.n * (c.n - 1) / 2;
    const size_t smem = 2 * (size_t)m * (kPairTB + 1) * 8 + (size_t)m * 8;
    FCIB_CHECK(smem + 1024 <= (size_t)c.smem_optin, FCIB_ERR_UNSUPPORTED, "RDMs: pair group exceeds shared memory");
    FCIB_CUDA(cudaFuncSetAttribute(k_rdm_pairs<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int per_sm = std::max(1, std::min(8, (int)(c.smem_per_sm / (smem + 1024))));
    const int grid = std::min(T.ng2, per_sm * c.num_sms);
    k_rdm_pairs<false><<<grid, kRdmThreads, smem, c.stream>>>(L, R, ncol, T.g2row.p, T.g2lab.p, T.ng2, m, npl, M);
    FCIB_KCHECK();
}

// Device pass over C1-layout vectors L, R (nas x nbs); fills the host RdmBlocks.
void compute_rdms(Context& c, const double* L, const double* R, int level, RdmBlocks& out) {
    const int n = c.n, nn = n * n, npl = n * (n - 1) / 2;
    const int nas = (int)c.nas, nbs = (int)c.nbs;
    const size_t n4 = (size_t)nn * nn;
    const bool two = level >= 2;
    const size_t total = 2 * (size_t)nn + (two ? n4 + 2 * (size_t)npl * npl : 0);
    DBuf<double> acc;
    acc.alloc(total);
    FCIB_CUDA(cudaMemsetAsync(acc.p, 0, sizeof(double) * total, c.stream));
    double* g1a = acc.p;
    double* g1b = g1a + nn;
    double* g2ab = g1b + nn;
    double* maa = g2ab + n4;
    double* mbb = maa + (size_t)npl * npl;
    // alpha rows (and the alpha-beta two-body block)
    rdm_vo(c, L, R, nas, nbs, c.A, c.B, two && c.na >= 1 && c.nb >= 1, g1a, two ? g2ab : nullptr);
    if (two && c.na >= 2) rdm_pairs(c, L, R, nbs, c.A, maa);
    // beta rows on the transposed vectors
    if (c.nb >= 1) {
        DBuf<double> lt, rt;
        lt.alloc((size_t)c.ndet);
        transpose(c, L, lt.p, nas, nbs);
        const double* rtp = lt.p;
        if (R != L) {
            rt.alloc((size_t)c.ndet);
            transpose(c, R, rt.p, nas, nbs);
            rtp = rt.p;
        }
        rdm_vo(c, lt.p, rtp, nbs, nas, c.B, c.A, false, g1b, nullptr);
        if (two && c.nb >= 2) rdm_pairs(c, lt.p, rtp, nas, c.B, mbb);
        FCIB_CUDA(cudaStreamSynchronize(c.stream));
    }
    std::vector<double> h(total);
    FCIB_CUDA(cudaMemcpyAsync(h.data(), acc.p, sizeof(double) * total, cudaMemcpyDeviceToHost, c.stream));
    FCIB_CUDA(cudaStreamSynchronize(c.stream));
    out.n = n;
    out.g1a.assign(h.begin(), h.begin() + nn);
    out.g1b.assign(h.begin() + nn, h.begin() + 2 * nn);
    if (two) {
        out.g2ab.assign(h.begin() + 2 * nn, h.begin() + 2 * nn + n4);
        const double* ha = h.data() + 2 * nn + n4;
        const double* hb = ha + (size_t)npl * npl;
        out.g2aa.assign(n4, 0.0);
        out.g2bb.assign(n4, 0.0);
        // pair label a = p(p-1)/2 + q, p > q; elements with a >= b give the 4 (a == b) or 8
        // antisymmetric positions, like the reference's OO and VVOO loops
        std::vector<int> lp(npl), lq(npl);
        for (int p = 0, a = 0; p < n; p++)
            for (int q = 0; q < p; q++, a++) {
                lp[a] = p;
                lq[a] = q;
            }
        auto T = [n](int p, int q, int r, int s) { return (((size_t)p * n + q) * n + r) * n + s; };
        for (int pass = 0; pass < 2; pass++) {
            const double* Mx = pass ? hb : ha;
            std::vector<double>& g = pass ? out.g2bb : out.g2aa;
            for (int a = 0; a < npl; a++) {
                const int p = lp[a], q = lq[a];
                for (int b = 0; b <= a; b++) {
                    const double el = Mx[(size_t)a * npl + b];
                    if (el == 0.0) continue;
                    const int r = lp[b], s = lq[b];
                    g[T(p, q, r, s)] += el;
                    g[T(q, p, r, s)] -= el;
                    g[T(p, q, s, r)] -= el;
                    g[T(q, p, s, r)] += el;
                    if (b == a) continue;
                    g[T(r, s, p, q)] += el;
                    g[T(r, s, q, p)] -= el;
                    g[T(s, r, p, q)] -= el;
                    g[T(s, r, q, p)] += el;
                }
            }
        }
    }
}

}  // namespace fcib
