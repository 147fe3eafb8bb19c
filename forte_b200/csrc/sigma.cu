// FP64 sigma = H C on the device, plus the Hamiltonian diagonal.
//
// Reference: FCIVector::Hamiltonian (forte/fci/fci_vector_hamiltonian.cc:46-272) builds
// sigma as H0 + H1a + H1b + H2ab + H2aa + H2bb with BLAS-1 loops over substitution lists.
// Here the same operator is regrouped into dense blocks:
//
// * opposite spin (+ both one-body terms folded in, + H0):  for a target alpha row Ia,
//       sigma[Ia, Ib] = sum_{P in conn(Ia)} sgn_P sum_R V[P,R] sum_{Jb} <Ib|F_R|Jb> C[Ja(P), Jb]
//   with unordered orbital pairs P=(p>=q), F_P = E_pq + E_qp (E_pp on the diagonal) and
//   V[P,R] = (pq|rs).  One CTA owns a row: it gathers the connected C rows, multiplies the
//   tile by V[P(Ia), :] and scatters the result over beta single replacements into a sigma
//   row held in shared memory.  The one-body terms are exact parts of V: on strings with nb
//   beta electrons sum_r E^b_rr = nb, so h^a_pq E^a_pq = (1/nb) sum_r h^a_pq E^a_pq E^b_rr.
// * same spin:  a+_p a+_q a_s a_r = sum_K a+_p a+_q |K><K| a_s a_r over (N-2)-electron
//   strings K, so for each K the 45 (n=16) strings K+{p,q} couple through the dense block
//   <pq||rs> restricted to the orbitals K leaves empty.  One CTA applies that block to a
//   column chunk of the gathered rows and adds the result back with atomics.  The beta term
//   runs on the transposed vector.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <type_traits>

#include "fcib_internal.h"

namespace fcib {

// ------------------------------------------------------------------------------------------
// host-side integral preparation
// ------------------------------------------------------------------------------------------
void prepare_integrals(Context& c) {
    const int n = c.n;
    const size_t n2 = (size_t)n * n, n3 = n2 * n;
    auto tab = [&](int p, int q, int r, int s) { return c.tei_ab[p * n3 + q * n2 + r * n + s]; };
    const int np = n * (n + 1) / 2, npp = (np + 7) / 8 * 8;
    c.fold_h = (c.na >= 1 && c.nb >= 1);
    std::vector<double> V((size_t)npp * npp, 0.0);
    for (int p = 0; p < n; p++)
        for (int q = 0; q <= p; q++)
            for (int r = 0; r < n; r++)
                for (int s = 0; s <= r; s++) {
                    int P = p * (p + 1) / 2 + q, R = r * (r + 1) / 2 + s;
                    double v = tab(p, r, q, s);  // <pr|qs> = (pq|rs)
                    if (c.fold_h) {
                        if (r == s) v += c.oei_a[p * n + q] / c.nb;
                        if (p == q) v += c.oei_b[r * n + s] / c.na;
                    }
                    V[(size_t)P * npp + R] = v;
                }
    c.V.upload(V, c.stream);
    const int np2 = n * (n - 1) / 2;
    if (np2 > 0) {
        std::vector<double> Ma((size_t)np2 * np2), Mb((size_t)np2 * np2);
        for (int p = 0; p < n; p++)
            for (int q = 0; q < p; q++)
                for (int r = 0; r < n; r++)
                    for (int s = 0; s < r; s++) {
                        int PQ = p * (p - 1) / 2 + q, RS = r * (r - 1) / 2 + s;
                        size_t idx = (size_t)p * n3 + q * n2 + r * n + s;
                        Ma[(size_t)PQ * np2 + RS] = c.tei_aa[idx];
                        Mb[(size_t)PQ * np2 + RS] = c.tei_bb[idx];
                    }
        c.M2a.upload(Ma, c.stream);
        c.M2b.upload(Mb, c.stream);
    }
    c.Ha.upload(c.oei_a, c.stream);
    c.Hb.upload(c.oei_b, c.stream);
    // largest same-spin block element (the mixed same-spin fixed-point grid); the one-body blocks
    // count only when they are not folded into the opposite-spin pair matrix
    double mm = 0.0;
    for (int p = 0; p < n; p++)
        for (int q = 0; q < n; q++)
            for (int r = 0; r < n; r++)
                for (int t = 0; t < n; t++) {
                    const size_t idx = (size_t)p * n3 + q * n2 + r * n + t;
                    mm = std::max(mm, std::max(std::fabs(c.tei_aa[idx]), std::fabs(c.tei_bb[idx])));
                }
    if (!c.fold_h)
        for (size_t i = 0; i < n2; i++) mm = std::max(mm, std::max(std::fabs(c.oei_a[i]), std::fabs(c.oei_b[i])));
    c.same_mmax = mm * (1.0 + 1e-6) + 1e-300;
}

// ------------------------------------------------------------------------------------------
// opposite-spin kernel (FP64 on the tensor cores: mma.sync m8n8k4 f64)
// ------------------------------------------------------------------------------------------
// One CTA per SM, persistent over target alpha rows Ia.  Per row: B[k][R] = sgn_k V[P_k][R]
// (FP64) and the sigma row (initialised to E0 * C row) stay in shared memory; per tile of 64 beta
// strings the connected C rows are gathered into A[k][Jb] (coalesced, one tile ahead in
// registers), T = A^T B is formed with FP64 tensor-core MMAs (16 warps: 8 strings x 72 pairs each,
// 9 independent 8x8 accumulators per warp, the fragments of the next k step loaded while the
// current step's MMAs run), and T[Jb][R] is scattered over the beta single replacements F_R Jb with
// FP64 shared-memory atomics.  A and B rows are stored with an XOR swizzle of bit 3 of the column by
// the parity of k, so the fragment loads (4 rows x 8 consecutive columns) and the gather stores take
// two wavefronts, the minimum for 256 bytes.
constexpr int kDmTM = 64;              // beta rows per tile
constexpr int kDmThreads = 512;        // 16 warps: row tile mt = warp & 7 (8 strings), pair half h = warp >> 3
constexpr int kDmNT = 9;               // n8 pair tiles per warp: 2 halves x 9 x 8 = 144 >= npair (n <= 16)
constexpr int kDmLdB = 2 * kDmNT * 8;  // B row stride in doubles (1152 bytes, a multiple of 128)
constexpr int kDmMaxK = 72;            // connections per string (n <= 16)
constexpr int kDmG = kDmMaxK * kDmTM / kDmThreads;  // gathered elements per thread per tile

size_t ab_fp64_smem(int nbs, int s1a, int npp) {
    (void)npp;
    const int kpad = (s1a + 7) / 8 * 8;
    return (size_t)((nbs + 1) & ~1) * 8 + (size_t)kpad * kDmLdB * 8 + (size_t)kpad * kDmTM * 8 + (size_t)kpad * 4 + 16;
}

// D (8x8) += A (8x4, row) B (4x8, col); lane holds A[lane/4][lane%4], B[lane%4][lane/4] and
// D[lane/4][2 (lane%4) + {0,1}]
__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
        : "+d"(d[0]), "+d"(d[1])
        : "d"(a), "d"(b));
}

// One FP64 value rounded to the fixed-point grid 2^-el (scale = 2^el) as a two's-complement u64
__device__ __forceinline__ unsigned long long fixed64d(double v, double scale) {
    return (unsigned long long)__double2ll_rn(v * scale);
}

// the FP64 sigma's 62-bit grids from max|C| (bits in *cmax_bits): the opposite-spin row sums are at
// most |e0| max|C| + s1b kpad max|C| max|V|, so 2^el of that stays below 2^62
__device__ __forceinline__ int grid_el_fp64(const unsigned int* cmax_bits, double bound_per_c) {
    const double b = fmax(1.01 * bound_per_c * (double)__uint_as_float(*cmax_bits), 1e-300);
    return min(1000, (int)floor(62.0 - log2(b)));
}

// Source rows (the connected strings J) are rows of Csrc with ns columns (row stride lds); target rows
// Ia have nt columns (C for the E0 term and S, row stride nt).  tgtB rows hold the targets of the
// source columns (row stride ldt), V rows the pair-matrix columns (row stride ldv).  accumulate = 1
// adds to S instead of writing E0 C + the product (the blocked sigma's later pair irreps).  In the C1
// layout Csrc = C, ns = lds = nt = nbs.
__global__ void __launch_bounds__(kDmThreads, 1) k_ab_fp64(
    const double* __restrict__ Csrc, int lds, int ns, const double* __restrict__ C, double* __restrict__ S, int nt,
    int accumulate, const uint32_t* __restrict__ connA, int s1a, int kpad, const int32_t* __restrict__ tgtB, int ldt,
    int npair, const double* __restrict__ V, int ldv, int nas, double e0, int* __restrict__ row_counter,
    const unsigned int* __restrict__ cmax_bits, double bound_per_c) {
    extern __shared__ __align__(16) unsigned char smem[];
    // the sigma row in 64-bit fixed point: every product is rounded once to the grid and the integer
    // sum does not depend on the order of the atomics (a repeated sigma is bit-identical)
    unsigned long long* srow = reinterpret_cast<unsigned long long*>(smem);
    const int el = grid_el_fp64(cmax_bits, bound_per_c);
    const double scale = ldexp(1.0, el), inv_scale = ldexp(1.0, -el);
    double* Bs = reinterpret_cast<double*>(srow + ((nt + 1) & ~1));  // [kpad][kDmLdB]: (k, R) at k*kDmLdB + (R ^ ((k & 1) << 3))
    double* As = Bs + (size_t)kpad * kDmLdB;        // [kpad][kDmTM]: (k, Jb) at k*kDmTM + (Jb ^ ((k & 1) << 3))
    uint32_t* cs = reinterpret_cast<uint32_t*>(As + (size_t)kpad * kDmTM);
    __shared__ int s_row;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int mt = warp & 7, h = warp >> 3;
    const int nnt = (npair + 7) / 8;        // pair tiles holding at least one pair
    const int nks = kpad / 4;
    const int ng = kpad * kDmTM / kDmThreads;  // gathered elements per thread (kpad is a multiple of 8)
    const int fr = lane >> 2, fk = lane & 3;   // fragment row / k of this lane
    double g[kDmG];

    while (true) {
        if (tid == 0) s_row = atomicAdd(row_counter, 1);
        __syncthreads();
        const int Ia = s_row;
        if (Ia >= nas) break;
        for (int k = tid; k < kpad; k += kDmThreads) cs[k] = k < s1a ? connA[(size_t)Ia * s1a + k] : 0u;
        const double* Crow = C + (size_t)Ia * nt;
        double* Srow = S + (size_t)Ia * nt;
        for (int j = tid; j < nt; j += kDmThreads) srow[j] = fixed64d(accumulate ? Srow[j] : e0 * Crow[j], scale);
        __syncthreads();
        for (int idx = tid; idx < kpad * kDmLdB; idx += kDmThreads) {
            const int k = idx / kDmLdB, R = idx - k * kDmLdB;
            double v = 0.0;
            if (k < s1a && R < npair) {
                const uint32_t e = cs[k];
                v = V[(size_t)((e >> 21) & 1023) * ldv + R];
                if (e & kSignBit) v = -v;
            }
            Bs[(size_t)k * kDmLdB + (R ^ ((k & 1) << 3))] = v;
        }
        // element e = it * kDmThreads + tid of the [kpad][kDmTM] tile: k = e / kDmTM, Jb = e % kDmTM
        auto gather = [&](int jb0) {
#pragma unroll
            for (int it = 0; it < kDmG; it++) {
                if (it < ng) {
                    const int e = it * kDmThreads + tid;
                    const int k = e / kDmTM, jb = jb0 + (e % kDmTM);
                    g[it] = (jb < ns && k < s1a) ? Csrc[(size_t)(cs[k] & kConnIdxMask) * lds + jb] : 0.0;
                }
            }
        };
        gather(0);
        for (int jb0 = 0; jb0 < ns; jb0 += kDmTM) {
            __syncthreads();  // the previous tile's fragment loads are done; B and cs are visible
#pragma unroll
            for (int it = 0; it < kDmG; it++) {
                if (it < ng) {
                    const int e = it * kDmThreads + tid;
                    const int k = e / kDmTM, c = e % kDmTM;
                    As[(size_t)k * kDmTM + (c ^ ((k & 1) << 3))] = g[it];
                }
            }
            __syncthreads();
            if (jb0 + kDmTM < ns) gather(jb0 + kDmTM);
            double acc[kDmNT][2];
#pragma unroll
            for (int j = 0; j < kDmNT; j++) acc[j][0] = acc[j][1] = 0.0;
            // fragments of k step ks: A[mt*8 + fr][4 ks + fk] and B[4 ks + fk][nt*8 + fr]
            double fa[2], fb[2][kDmNT];
            auto load_frag = [&](int ks, int buf) {
                const int k = 4 * ks + fk;
                const int sw = (k & 1) << 3;
                fa[buf] = As[(size_t)k * kDmTM + ((mt * 8 + fr) ^ sw)];
                const double* br = Bs + (size_t)k * kDmLdB;
#pragma unroll
                for (int j = 0; j < kDmNT; j++) {
                    const int nt = h * kDmNT + j;
                    fb[buf][j] = nt < nnt ? br[(nt * 8 + fr) ^ sw] : 0.0;
                }
            };
            load_frag(0, 0);
            for (int ks = 0; ks < nks; ks += 2) {
                if (ks + 1 < nks) load_frag(ks + 1, 1);
#pragma unroll
                for (int j = 0; j < kDmNT; j++)
                    if (h * kDmNT + j < nnt) dmma_8x8x4(acc[j], fa[0], fb[0][j]);
                if (ks + 1 < nks) {
                    if (ks + 2 < nks) load_frag(ks + 2, 0);
#pragma unroll
                    for (int j = 0; j < kDmNT; j++)
                        if (h * kDmNT + j < nnt) dmma_8x8x4(acc[j], fa[1], fb[1][j]);
                }
            }
            // scatter T[Jb][R] over the beta single replacements into the sigma row
            const int jb = jb0 + mt * 8 + fr;
            if (jb < ns) {
#pragma unroll
                for (int j = 0; j < kDmNT; j++) {
                    const int ntile = h * kDmNT + j;
                    if (ntile < nnt) {
                        const int R = ntile * 8 + 2 * fk;
                        const int2 tg = *reinterpret_cast<const int2*>(tgtB + (size_t)jb * ldt + R);
                        if (tg.x != kNoTarget) {
                            const double v = acc[j][0];
                            atomicAdd(&srow[tg.x & kConnIdxMask], fixed64d((tg.x & (int)kSignBit) ? -v : v, scale));
                        }
                        if (tg.y != kNoTarget) {
                            const double v = acc[j][1];
                            atomicAdd(&srow[tg.y & kConnIdxMask], fixed64d((tg.y & (int)kSignBit) ? -v : v, scale));
                        }
                    }
                }
            }
        }
        __syncthreads();
        for (int j = tid; j < nt; j += kDmThreads) Srow[j] = (double)(long long)srow[j] * inv_scale;
    }
}

// bits of max|C| (rounded up) into *cmax_bits (zeroed before the launch)
__global__ void k_absmax(const double* __restrict__ C, size_t n, unsigned int* __restrict__ cmax_bits) {
    float mx = 0.f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        mx = fmaxf(mx, (float)fabs(C[i]));
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    // non-negative floats order like their bit patterns; two ulps up cover the rounding to float
    if ((threadIdx.x & 31) == 0) atomicMax(cmax_bits, mx > 0.f ? __float_as_uint(mx) + 2u : 0u);
}

// ------------------------------------------------------------------------------------------
// group kernel: sigma[row_i, :] += sgn_i sum_j M[lab_i, lab_j] sgn_j C[row_j, :]  (FP64)
// one CTA per (group, column chunk)
// ------------------------------------------------------------------------------------------
constexpr int kGrTN = 128;   // columns per CTA
constexpr int kGrRows = 8;   // rows per thread

// Persistent CTAs take (group, column chunk) work items in chunk-major order, so the columns of
// C and sigma a chunk touches stay L2-resident while every group of that chunk is processed.
// The pair-pair block M stays in shared memory; W = M[lab_i][lab_j] is rebuilt per item from it.
// T = double (FP64 path: FP64 in, FP64 atomics) or float (mixed path: an FP32 copy of C in, FP32
// accumulation, each result rounded to the sigma's fixed-point grid 2^-el and added with 64-bit
// integer reductions into an int64 buffer, so the sum does not depend on the order of the groups).
constexpr int kGrLoads = 16;  // X elements per thread per item (G*kGrTN/threads <= 16 by construction)

template <typename T>
struct GroupOut {
    using type = unsigned long long;
};

// one FP32 same-spin result -> its fixed-point integer on the grid 2^-el (two's complement in a u64)
__device__ __forceinline__ unsigned long long fixed64(float v, float scale) {
    return (unsigned long long)__float2ll_rn(v * scale);
}

template <typename T>
__global__ void __launch_bounds__(1024) k_group(
    const T* __restrict__ C, typename GroupOut<T>::type* __restrict__ S, int ncols, int ld,
    const uint32_t* __restrict__ rows, const uint16_t* __restrict__ labs, int G, int Gp,
    const double* __restrict__ M, int ldm, int ngroups, int nchunks, int* __restrict__ counter, int m_in_smem,
    const int* __restrict__ grid_el) {
    const T scale = (T)ldexp(1.0, *grid_el);
    using T2 = typename std::conditional<std::is_same<T, double>::value, double2, float2>::type;
    extern __shared__ __align__(16) unsigned char smem[];
    T* Ms = reinterpret_cast<T*>(smem);       // [ldm][ldm] when m_in_smem (else M is read from L2)
    // W must start 16-byte aligned for its vector loads: round the M region to 128 bytes
    const size_t m_elems = m_in_smem ? ((size_t)ldm * ldm * sizeof(T) + 127) / 128 * 128 / sizeof(T) : 0;
    T* Wt = Ms + m_elems;                     // [G][Gp]  Wt[j][i] = M[lab_i][lab_j]
    T* X = Wt + (size_t)G * Gp;               // [G][kGrTN]
    uint32_t* rs = reinterpret_cast<uint32_t*>(X + (size_t)G * kGrTN);
    uint16_t* ls = reinterpret_cast<uint16_t*>(rs + Gp);
    __shared__ int s_item;
    const int tid = threadIdx.x, nth = blockDim.x;
    if (m_in_smem)
        for (int idx = tid; idx < ldm * ldm; idx += nth) Ms[idx] = (T)M[idx];
    const int npairs = kGrTN / 2;
    const int cp = tid % npairs, rc = tid / npairs;
    const int i0 = rc * kGrRows;
    const int total = ngroups * nchunks;
    while (true) {
        __syncthreads();
        if (tid == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= total) break;
        const int chunk = item / ngroups, g = item - chunk * ngroups;
        const int c0 = chunk * kGrTN;
        for (int i = tid; i < Gp; i += nth) {
            rs[i] = i < G ? rows[(size_t)g * G + i] : 0u;
            ls[i] = i < G ? labs[(size_t)g * G + i] : 0;
        }
        __syncthreads();
        // gather the G rows (this chunk's columns) with all loads in flight at once
        T xv[kGrLoads];
#pragma unroll
        for (int r = 0; r < kGrLoads; r++) {
            const int idx = tid + r * nth;
            T v = (T)0;
            if (idx < G * kGrTN) {
                const int j = idx / kGrTN, col = c0 + (idx - j * kGrTN);
                if (col < ncols && rs[j] != kNullRow) v = C[(size_t)(rs[j] & kConnIdxMask) * ld + col];
            }
            xv[r] = v;
        }
        for (int idx = tid; idx < G * Gp; idx += nth) {
            int j = idx / Gp, i = idx - j * Gp;
            const size_t mi = (size_t)ls[i] * ldm + ls[j];
            Wt[idx] = i < G ? (m_in_smem ? Ms[mi] : (T)M[mi]) : (T)0;
        }
#pragma unroll
        for (int r = 0; r < kGrLoads; r++) {
            const int idx = tid + r * nth;
            if (idx < G * kGrTN) {
                const int j = idx / kGrTN;
                X[idx] = (T)((rs[j] & kSignBit) ? -xv[r] : xv[r]);
            }
        }
        __syncthreads();
        if (i0 < G) {
            T acc[kGrRows][2];
#pragma unroll
            for (int i = 0; i < kGrRows; i++) acc[i][0] = acc[i][1] = (T)0;
            for (int j = 0; j < G; j++) {
                T w[kGrRows];
                if (std::is_same<T, double>::value) {
                    const double2* w2 = reinterpret_cast<const double2*>(Wt + (size_t)j * Gp + i0);
#pragma unroll
                    for (int i = 0; i < kGrRows / 2; i++) {
                        double2 t = w2[i];
                        w[2 * i] = (T)t.x;
                        w[2 * i + 1] = (T)t.y;
                    }
                } else {
                    const float4* w4 = reinterpret_cast<const float4*>(Wt + (size_t)j * Gp + i0);
#pragma unroll
                    for (int i = 0; i < kGrRows / 4; i++) {
                        float4 t = w4[i];
                        w[4 * i] = (T)t.x; w[4 * i + 1] = (T)t.y; w[4 * i + 2] = (T)t.z; w[4 * i + 3] = (T)t.w;
                    }
                }
                T2 x = *reinterpret_cast<const T2*>(X + (size_t)j * kGrTN + 2 * cp);
#pragma unroll
                for (int i = 0; i < kGrRows; i++) {
                    acc[i][0] = fma(w[i], x.x, acc[i][0]);
                    acc[i][1] = fma(w[i], x.y, acc[i][1]);
                }
            }
            const int col = c0 + 2 * cp;
#pragma unroll
            for (int i = 0; i < kGrRows; i++) {
                int ii = i0 + i;
                if (ii < G && rs[ii] != kNullRow) {
                    uint32_t e = rs[ii];
                    const size_t off = (size_t)(e & kConnIdxMask) * ld + col;
                    auto* dst = S + off;
                    const T a0 = (e & kSignBit) ? -acc[i][0] : acc[i][0];
                    const T a1 = (e & kSignBit) ? -acc[i][1] : acc[i][1];
                    if constexpr (std::is_same<T, double>::value) {
                        if (col < ncols) atomicAdd(dst, fixed64d(a0, scale));
                        if (col + 1 < ncols) atomicAdd(dst + 1, fixed64d(a1, scale));
                    } else {
                        if (col < ncols) atomicAdd(dst, fixed64(a0, scale));
                        if (col + 1 < ncols) atomicAdd(dst + 1, fixed64(a1, scale));
                    }
                }
            }
        }
    }
}

// ------------------------------------------------------------------------------------------
// FP64 same-spin groups on the FP64 tensor cores (mma.sync m8n8k4 f64).  Persistent CTAs take
// (group, 128-column chunk) items in chunk-major order like k_group; per item
//     D[i][col] = sum_j W[i][j] X[j][col],  W[i][j] = M[lab_i][lab_j],  X[j][col] = s_j C[row_j][c0 + col],
// then s_i D[i][col] is rounded to the sigma's same-spin grid 2^-el and added to S[row_i][c0 + col]
// (an int64 buffer) with 64-bit integer reductions, so the sum does not depend on the group order.  8 warps: warp w owns columns
// 16w..16w+15 (two n8 tiles) for all G rows (up to six m8 tiles), so an item is 12 accumulators per
// warp over K = G padded to 4.  W rows are 52 doubles apart (416 B, 32 B past a multiple of 128) and
// X columns are XOR-swizzled by the parity of the row, so fragment loads take two wavefronts.
// ------------------------------------------------------------------------------------------
constexpr int kGdTN = 128;
constexpr int kGdThreads = 256;
constexpr int kGdMaxG = 48;
constexpr int kGdLdW = 52;

__global__ void __launch_bounds__(kGdThreads) k_group_dmma(
    const double* __restrict__ C, unsigned long long* __restrict__ S, int ncols, int ld,
    const uint32_t* __restrict__ rows, const uint16_t* __restrict__ labs, int G, const double* __restrict__ M, int ldm,
    int ngroups, int nchunks, int* __restrict__ counter, const int* __restrict__ grid_el) {
    const double scale = ldexp(1.0, *grid_el);  // the sigma's same-spin fixed-point grid
    extern __shared__ __align__(16) unsigned char gd_smem[];
    double* Ws = reinterpret_cast<double*>(gd_smem);      // W[i][j] at i*kGdLdW + j
    double* Xs = Ws + kGdMaxG * kGdLdW;                    // X[j][col] at j*kGdTN + (col ^ ((j & 1) << 3))
    uint32_t* rs = reinterpret_cast<uint32_t*>(Xs + kGdMaxG * kGdTN);
    uint16_t* ls = reinterpret_cast<uint16_t*>(rs + kGdMaxG);
    __shared__ int s_item;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int fr = lane >> 2, fk = lane & 3;
    const int Gp = (G + 7) / 8 * 8;       // rows padded to whole m8 tiles
    const int Kp = (G + 3) / 4 * 4;       // K padded to whole k4 steps
    const int nmt = Gp / 8, nks = Kp / 4;
    const int total = ngroups * nchunks;
    while (true) {
        __syncthreads();
        if (tid == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= total) break;
        const int chunk = item / ngroups, g = item - chunk * ngroups;
        const int c0 = chunk * kGdTN;
        for (int i = tid; i < kGdMaxG; i += kGdThreads) {
            rs[i] = i < G ? rows[(size_t)g * G + i] : 0u;
            ls[i] = i < G ? labs[(size_t)g * G + i] : (uint16_t)0;
        }
        __syncthreads();
        for (int idx = tid; idx < Gp * Kp; idx += kGdThreads) {
            const int i = idx / Kp, j = idx - i * Kp;
            Ws[i * kGdLdW + j] = (i < G && j < G) ? M[(size_t)ls[i] * ldm + ls[j]] : 0.0;
        }
        for (int idx = tid; idx < Kp * kGdTN; idx += kGdThreads) {
            const int j = idx / kGdTN, col = idx - j * kGdTN;
            double v = 0.0;
            if (j < G && c0 + col < ncols && rs[j] != kNullRow) {
                const uint32_t r = rs[j];
                v = C[(size_t)(r & kConnIdxMask) * ld + c0 + col];
                if (r & kSignBit) v = -v;
            }
            Xs[j * kGdTN + (col ^ ((j & 1) << 3))] = v;
        }
        __syncthreads();
        double acc[6][2][2];
#pragma unroll
        for (int m = 0; m < 6; m++)
#pragma unroll
            for (int t = 0; t < 2; t++) acc[m][t][0] = acc[m][t][1] = 0.0;
        for (int ks = 0; ks < nks; ks++) {
            const int k = 4 * ks + fk;
            const int sw = (k & 1) << 3;
            double b[2];
#pragma unroll
            for (int t = 0; t < 2; t++) b[t] = Xs[k * kGdTN + (((2 * warp + t) * 8 + fr) ^ sw)];
#pragma unroll
            for (int m = 0; m < 6; m++) {
                if (m < nmt) {
                    const double a = Ws[(m * 8 + fr) * kGdLdW + k];
                    dmma_8x8x4(acc[m][0], a, b[0]);
                    dmma_8x8x4(acc[m][1], a, b[1]);
                }
            }
        }
#pragma unroll
        for (int m = 0; m < 6; m++) {
            const int i = m * 8 + fr;
            if (m < nmt && i < G && rs[i] != kNullRow) {
                const uint32_t r = rs[i];
                unsigned long long* srow = S + (size_t)(r & kConnIdxMask) * ld;
#pragma unroll
                for (int t = 0; t < 2; t++) {
                    const int col = c0 + (2 * warp + t) * 8 + 2 * fk;
                    const double d0 = (r & kSignBit) ? -acc[m][t][0] : acc[m][t][0];
                    const double d1 = (r & kSignBit) ? -acc[m][t][1] : acc[m][t][1];
                    if (col < ncols) atomicAdd(srow + col, fixed64d(d0, scale));
                    if (col + 1 < ncols) atomicAdd(srow + col + 1, fixed64d(d1, scale));
                }
            }
        }
    }
}

template <typename T>
static void launch_group_t(Context& c, const T* C, typename GroupOut<T>::type* S, int ncols, int ld, int ngroups, int G,
                           const uint32_t* rows, const uint16_t* labs, const double* M, int ldm,
                           const int* grid_el) {
    if (ngroups == 0 || G == 0) return;
    int Gp = (G + kGrRows - 1) / kGrRows * kGrRows;
    size_t smem_tiles = (size_t)G * Gp * sizeof(T) + (size_t)G * kGrTN * sizeof(T) + (size_t)Gp * 4 + (size_t)Gp * 2 + 16;
    size_t smem_m = ((size_t)ldm * ldm * sizeof(T) + 127) / 128 * 128;
    int m_in_smem = (smem_tiles + smem_m + 1024 <= (size_t)c.smem_optin) ? 1 : 0;
    size_t smem = smem_tiles + (m_in_smem ? smem_m : 0);
    FCIB_CHECK(smem + 1024 <= (size_t)c.smem_optin, FCIB_ERR_UNSUPPORTED, "same-spin group block exceeds shared memory");
    int threads = (kGrTN / 2) * (Gp / kGrRows);
    threads = (threads + 31) / 32 * 32;
    FCIB_CHECK(threads <= 1024, FCIB_ERR_UNSUPPORTED, "same-spin group block too large");
    FCIB_CHECK((size_t)G * kGrTN <= (size_t)kGrLoads * threads, FCIB_ERR_UNSUPPORTED, "same-spin gather tile too large");
    FCIB_CUDA(cudaFuncSetAttribute(k_group<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int nchunks = (ncols + kGrTN - 1) / kGrTN;
    int per_sm = std::max(1, std::min((int)(c.smem_per_sm / (smem + 1024)), 2048 / threads));
    int grid = std::min(ngroups * nchunks, per_sm * c.num_sms);
    ensure_counter(c);
    FCIB_CUDA(cudaMemsetAsync(c.counter.p + 2, 0, sizeof(int), c.stream));
    k_group<T><<<grid, threads, smem, c.stream>>>(C, S, ncols, ld, rows, labs, G, Gp, M, ldm, ngroups, nchunks, c.counter.p + 2,
                                                  m_in_smem, grid_el);
    FCIB_KCHECK();
}

// ld: row stride of C and S (ncols, or the row length of the block when the columns are a sub-range)
static void launch_group(Context& c, const double* C, unsigned long long* S, int ncols, int ld, int ngroups, int G,
                         const uint32_t* rows, const uint16_t* labs, const double* M, int ldm) {
    if (ngroups == 0 || G == 0) return;
    if (G <= kGdMaxG) {
        // FP64 tensor cores; three CTAs per SM (69 KB of shared memory each)
        const int nchunks = (ncols + kGdTN - 1) / kGdTN;
        const int grid = std::min(ngroups * nchunks, 3 * c.num_sms);
        const size_t smem = sizeof(double) * (kGdMaxG * kGdLdW + kGdMaxG * kGdTN) + kGdMaxG * 6;
        FCIB_CUDA(cudaFuncSetAttribute(k_group_dmma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        ensure_counter(c);
        FCIB_CUDA(cudaMemsetAsync(c.counter.p + 2, 0, sizeof(int), c.stream));
        k_group_dmma<<<grid, kGdThreads, smem, c.stream>>>(C, S, ncols, ld, rows, labs, G, M, ldm, ngroups, nchunks,
                                                           c.counter.p + 2, c.counter.p + kSlotSameGrid);
        FCIB_KCHECK();
        return;
    }
    launch_group_t<double>(c, C, S, ncols, ld, ngroups, G, rows, labs, M, ldm, c.counter.p + kSlotSameGrid);
}
static void launch_group(Context& c, const float* C, unsigned long long* S, int ncols, int ld, int ngroups, int G,
                         const uint32_t* rows, const uint16_t* labs, const double* M, int ldm) {
    launch_group_t<float>(c, C, S, ncols, ld, ngroups, G, rows, labs, M, ldm, c.counter.p + kSlotSameGrid);
}

// ------------------------------------------------------------------------------------------
// small helpers
// ------------------------------------------------------------------------------------------
__global__ void k_transpose(const double* __restrict__ in, double* __restrict__ out, int rows, int cols) {
    __shared__ double tile[32][33];
    int x = blockIdx.x * 32 + threadIdx.x;
    int y0 = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        int y = y0 + j;
        if (x < cols && y < rows) tile[j][threadIdx.x] = in[(size_t)y * cols + x];
    }
    __syncthreads();
    int ox = y0 + threadIdx.x;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        int oy = blockIdx.x * 32 + j;
        if (ox < rows && oy < cols) out[(size_t)oy * rows + ox] = tile[threadIdx.x][j];
    }
}

__global__ void k_transpose_f32(const float* __restrict__ in, float* __restrict__ out, int rows, int cols) {
    __shared__ float tile[32][33];
    int x = blockIdx.x * 32 + threadIdx.x;
    int y0 = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        int y = y0 + j;
        if (x < cols && y < rows) tile[j][threadIdx.x] = in[(size_t)y * cols + x];
    }
    __syncthreads();
    int ox = y0 + threadIdx.x;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        int oy = blockIdx.x * 32 + j;
        if (ox < rows && oy < cols) out[(size_t)oy * rows + ox] = tile[threadIdx.x][j];
    }
}

// S[r][c] += (A[r][c] + Bt[c][r]) 2^-el: the alpha (row-major) and beta (transposed) same-spin parts,
// exact integers on the fixed-point grid 2^-el of this sigma (each part below 2^62 in magnitude)
__global__ void k_add_same_fixed(double* __restrict__ S, const unsigned long long* __restrict__ A,
                                 const unsigned long long* __restrict__ Bt, int rows, int cols,
                                 const int* __restrict__ grid_el) {
    __shared__ long long tile[32][33];
    const double inv = ldexp(1.0, -*grid_el);
    int x = blockIdx.x * 32 + threadIdx.x;  // Bt column = S row
    int y0 = blockIdx.y * 32;               // Bt row = S column
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        int y = y0 + j;
        if (x < rows && y < cols) tile[j][threadIdx.x] = (long long)Bt[(size_t)y * rows + x];
    }
    __syncthreads();
    int oc = y0 + threadIdx.x;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        int orow = blockIdx.x * 32 + j;
        if (orow < rows && oc < cols) {
            const size_t o = (size_t)orow * cols + oc;
            S[o] += (double)((long long)A[o] + tile[threadIdx.x][j]) * inv;
        }
    }
}

// fixed-point grid of the mixed same-spin sums: every |element| <= kbound * max|C| * max|M|, so
// 2^el times that stays below 2^62
__global__ void k_same_grid(const unsigned int* __restrict__ cmax_bits, float kbound_mmax, int* __restrict__ el) {
    const float b = fmaxf(1.01f * kbound_mmax * __uint_as_float(*cmax_bits), 1e-30f);
    *el = min(100, (int)floorf(62.0f - log2f(b)));
}

// FP32 copy of the sigma input and bits of max|C| rounded up (when the tensor-core split did not run)
__global__ void k_to_f32(const double* __restrict__ in, float* __restrict__ out, size_t n,
                         unsigned int* __restrict__ cmax_bits) {
    float mx = 0.f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        out[i] = (float)in[i];
        mx = fmaxf(mx, fabsf(out[i]));
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(cmax_bits, __float_as_uint(mx) + 1u);
}

__global__ void k_scale_copy(const double* __restrict__ in, double* __restrict__ out, double a, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = a * in[i];
}

__global__ void k_apply_mask(double* __restrict__ v, const uint8_t* __restrict__ m, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (!m[i]) v[i] = 0.0;
}

static void transpose(Context& c, const double* in, double* out, int rows, int cols) {
    dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
    k_transpose<<<grid, block, 0, c.stream>>>(in, out, rows, cols);
    FCIB_KCHECK();
}
void apply_mask(Context& c, double* v) {
    if (!c.mask.p || c.sigma_unmasked) return;
    k_apply_mask<<<4 * c.num_sms, 256, 0, c.stream>>>(v, c.mask.p, (size_t)c.nvec);
    FCIB_KCHECK();
}

// ------------------------------------------------------------------------------------------
// sigma orchestration
// ------------------------------------------------------------------------------------------
bool launch_group_tc(Context& c, const float* C, unsigned long long* S, int ncols, int ld, int ngroups, int G,
                     const uint32_t* rows, const uint16_t* labs, const double* M, int ldm);

// mixed same-spin two-body groups: tensor cores unless disabled or the groups are too large
static void launch_group_same_f32(Context& c, const float* C, unsigned long long* S, int ncols, int ld, int ngroups,
                                  int G, const uint32_t* rows, const uint16_t* labs, const double* M, int ldm) {
    if (c.opt.same_spin_kernel == FCIB_SAME_TC && launch_group_tc(c, C, S, ncols, ld, ngroups, G, rows, labs, M, ldm))
        return;
    launch_group(c, C, S, ncols, ld, ngroups, G, rows, labs, M, ldm);
}

// same-spin (and, when not folded into the opposite-spin block, one-body) terms added to S
static void sigma_same_spin(Context& c, const double* C, double* S, bool fp32) {
    const int nas = (int)c.nas, nbs = (int)c.nbs;
    const size_t N = (size_t)c.nvec;
    const int np2 = c.n * (c.n - 1) / 2;
    const bool a_g1 = !c.fold_h && c.A.ng1, b_g1 = !c.fold_h && c.B.ng1;
    const bool any_a = a_g1 || c.A.ng2, any_b = b_g1 || c.B.ng2;
    if (!any_a && !any_b) return;
    ensure_counter(c);
    const SymSpace& y = c.sym;
    // both precisions sum the same-spin results in int64 on a per-sigma fixed-point grid (the alpha
    // part row-major, the beta part transposed) and add them to S at the end
    auto same_grid = [&](const unsigned int* cmax_bits) {
        auto kb = [&](const SpinTables& t, bool g1, int ne) {
            double v = (double)t.ng2 > 0 ? (double)ne * (ne - 1) / 2 * ((t.g2 + 15) / 16 * 16) : 0.0;
            if (g1 && t.ng1) v += (double)ne * ((t.g1 + 15) / 16 * 16);
            return v;
        };
        const double kbound = std::max(kb(c.A, a_g1, c.na), kb(c.B, b_g1, c.nb));
        k_same_grid<<<1, 1, 0, c.stream>>>(cmax_bits, (float)(kbound * c.same_mmax), c.counter.p + kSlotSameGrid);
        FCIB_KCHECK();
        c.s64a.alloc(N);
        c.st64.alloc(N);
        FCIB_CUDA(cudaMemsetAsync(c.s64a.p, 0, N * sizeof(unsigned long long), c.stream));
        FCIB_CUDA(cudaMemsetAsync(c.st64.p, 0, N * sizeof(unsigned long long), c.stream));
    };
    // C -> its transpose: one matrix in the C1 layout, one per alpha block in the blocked layout
    auto transpose_all = [&](const auto* in, auto* out, auto&& tr) {
        if (!y.on) {
            tr(in, out, nas, nbs);
            return;
        }
        for (int ha = 0; ha < c.nirrep; ha++) {
            const int hb = ha ^ c.irrep;
            if (y.acnt[ha] && y.bcnt[hb]) tr(in + y.d.blk[ha], out + y.blkT[hb], y.acnt[ha], y.bcnt[hb]);
        }
    };
    auto add_same = [&]() {
        auto add = [&](double* Sx, const unsigned long long* A, const unsigned long long* Bt, int rows, int cols) {
            dim3 grid2((rows + 31) / 32, (cols + 31) / 32), block2(32, 8);
            k_add_same_fixed<<<grid2, block2, 0, c.stream>>>(Sx, A, Bt, rows, cols, c.counter.p + kSlotSameGrid);
            FCIB_KCHECK();
        };
        if (!y.on) {
            add(S, c.s64a.p, c.st64.p, nas, nbs);
            return;
        }
        for (int ha = 0; ha < c.nirrep; ha++) {
            const int hb = ha ^ c.irrep;
            if (y.acnt[ha] && y.bcnt[hb])
                add(S + y.d.blk[ha], c.s64a.p + y.d.blk[ha], c.st64.p + y.blkT[hb], y.acnt[ha], y.bcnt[hb]);
        }
    };
    if (!fp32) {
        same_grid(reinterpret_cast<unsigned int*>(c.counter.p + kSlotCmax64));  // max|C| from sigma_fp64
        auto groups = [&](const double* X, unsigned long long* out, const std::vector<GroupSub>& subs, const SpinTables& t,
                          bool one_body, int ncols, const double* M, int ldm) {
            if (!y.on) {
                if (one_body) launch_group(c, X, out, ncols, ncols, t.ng1, t.g1, t.g1row.p, t.g1lab.p, M, ldm);
                else launch_group(c, X, out, ncols, ncols, t.ng2, t.g2, t.g2row.p, t.g2lab.p, M, ldm);
                return;
            }
            for (const GroupSub& g : subs)
                launch_group(c, X + g.blk, out + g.blk, g.ncols, g.ld, g.ngroups, g.G, y.grow.p + g.off, y.glab.p + g.off,
                             M, ldm);
        };
        if (a_g1) groups(C, c.s64a.p, y.a1, c.A, true, nbs, c.Ha.p, c.n);
        if (c.A.ng2) groups(C, c.s64a.p, y.a2, c.A, false, nbs, c.M2a.p, np2);
        if (any_b) {
            c.ct.alloc(N);
            transpose_all(C, c.ct.p, [&](const double* in, double* out, int r, int cc) { transpose(c, in, out, r, cc); });
            if (b_g1) groups(c.ct.p, c.st64.p, y.b1, c.B, true, nas, c.Hb.p, c.n);
            if (c.B.ng2) groups(c.ct.p, c.st64.p, y.b2, c.B, false, nas, c.M2b.p, np2);
        }
        add_same();
        return;
    }
    // mixed: FP32 copy of C (written by the tensor-core split when it ran), FP32 accumulation
    unsigned int* cmax_bits = reinterpret_cast<unsigned int*>(c.counter.p + kSlotCmax);
    if (!c.c32_ready) {
        c.c32.alloc(N);
        FCIB_CUDA(cudaMemsetAsync(cmax_bits, 0, sizeof(unsigned int), c.stream));
        k_to_f32<<<4 * c.num_sms, 256, 0, c.stream>>>(C, c.c32.p, N, cmax_bits);
        FCIB_KCHECK();
    }
    c.c32_ready = false;
    // fixed-point grid from max|C| (just computed on the device) and the host bound kbound * max|M|
    same_grid(cmax_bits);
    FCIB_CUDA(cudaMemsetAsync(c.counter.p + 5, 0, sizeof(int), c.stream));  // tensor-core group timeout flag
    auto groups32 = [&](const float* X, unsigned long long* out, const std::vector<GroupSub>& subs, const SpinTables& t,
                        bool one_body, int ncols, const double* M, int ldm) {
        auto one = [&](const float* Xb, unsigned long long* Ob, int nc, int ld, int ng, int G, const uint32_t* rows,
                       const uint16_t* labs) {
            if (one_body) launch_group(c, Xb, Ob, nc, ld, ng, G, rows, labs, M, ldm);
            else launch_group_same_f32(c, Xb, Ob, nc, ld, ng, G, rows, labs, M, ldm);
        };
        if (!y.on) {
            if (one_body) one(X, out, ncols, ncols, t.ng1, t.g1, t.g1row.p, t.g1lab.p);
            else one(X, out, ncols, ncols, t.ng2, t.g2, t.g2row.p, t.g2lab.p);
            return;
        }
        for (const GroupSub& g : subs)
            one(X + g.blk, out + g.blk, g.ncols, g.ld, g.ngroups, g.G, y.grow.p + g.off, y.glab.p + g.off);
    };
    if (a_g1) groups32(c.c32.p, c.s64a.p, y.a1, c.A, true, nbs, c.Ha.p, c.n);
    if (c.A.ng2) groups32(c.c32.p, c.s64a.p, y.a2, c.A, false, nbs, c.M2a.p, np2);
    if (any_b) {
        c.ct32.alloc(N);
        transpose_all(c.c32.p, c.ct32.p, [&](const float* in, float* out, int r, int cc) {
            dim3 gridt((cc + 31) / 32, (r + 31) / 32), blockt(32, 8);
            k_transpose_f32<<<gridt, blockt, 0, c.stream>>>(in, out, r, cc);
            FCIB_KCHECK();
        });
        if (b_g1) groups32(c.ct32.p, c.st64.p, y.b1, c.B, true, nas, c.Hb.p, c.n);
        if (c.B.ng2) groups32(c.ct32.p, c.st64.p, y.b2, c.B, false, nas, c.M2b.p, np2);
    }
    add_same();
}

// events bracketing the opposite-spin and same-spin parts of a sigma build
struct SigmaEvents {
    cudaEvent_t e[3];
    SigmaEvents() { for (auto& x : e) cudaEventCreate(&x); }
    ~SigmaEvents() { for (auto& x : e) cudaEventDestroy(x); }
};
static void sigma_timing(Context& c, SigmaEvents& ev, bool fp64) {
    FCIB_CUDA(cudaEventSynchronize(ev.e[2]));
    float a = 0.f, b = 0.f;
    cudaEventElapsedTime(&a, ev.e[0], ev.e[1]);
    cudaEventElapsedTime(&b, ev.e[1], ev.e[2]);
    if (fp64) {
        c.t_ab64_ms += a;
        c.t_same64_ms += b;
        c.n_ab64++;
    } else {
        c.t_ab_ms += a;
        c.t_same_ms += b;
        c.n_ab++;
        if (c.tc_recorded) {
            float t = 0.f;
            cudaEventElapsedTime(&t, c.tc_ev.e[0], c.tc_ev.e[1]);
            c.t_tc_ms += t;
            c.tc_recorded = false;
        }
    }
}

void sigma_fp64(Context& c, const double* C, double* S) {
    const int nas = (int)c.nas, nbs = (int)c.nbs;
    const size_t N = (size_t)c.nvec;
    ensure_counter(c);
    SigmaEvents ev;
    FCIB_CUDA(cudaEventRecord(ev.e[0], c.stream));
    // max|C| for the fixed-point grids of the opposite-spin rows and the same-spin groups
    unsigned int* cmax64 = reinterpret_cast<unsigned int*>(c.counter.p + kSlotCmax64);
    FCIB_CUDA(cudaMemsetAsync(cmax64, 0, sizeof(unsigned int), c.stream));
    k_absmax<<<4 * c.num_sms, 256, 0, c.stream>>>(C, N, cmax64);
    FCIB_KCHECK();
    if (c.fold_h) {
        const int s1a = c.A.s1, npp = c.A.npair_pad;
        const int kpad = (s1a + 7) / 8 * 8;
        FCIB_CHECK(kpad <= kDmMaxK && c.A.npair <= 2 * kDmNT * 8 && c.B.npair_pad == npp, FCIB_ERR_UNSUPPORTED,
                   "too many orbitals for the FP64 opposite-spin kernel");
        if (c.vmax <= 0.0f) c.vmax = host_vmax(c);
        // one grid for every launch of this sigma (the blocked sub-problems have fewer connections)
        const double bound = std::fabs(c.scalar) + (double)c.B.s1 * kpad * (double)c.vmax;
        int attr_smem = -1;  // the kernel's dynamic shared memory limit, raised only when a launch needs more
        auto launch = [&](const double* Csrc, int lds, int ns, const double* Ct, double* St, int nt, int acc,
                          const uint32_t* conn, int s1, const int32_t* tgt, int ldt, int npair, const double* V,
                          int ldv, int rows, int* ctr) {
            const size_t smem = ab_fp64_smem(nt, s1, 0);
            FCIB_CHECK(smem + 1024 <= (size_t)c.smem_optin, FCIB_ERR_UNSUPPORTED,
                       "opposite-spin row block exceeds shared memory (beta string count too large)");
            if ((int)smem > attr_smem) {
                FCIB_CUDA(cudaFuncSetAttribute(k_ab_fp64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                attr_smem = (int)smem;
            }
            int per_sm = std::max(1, (int)(c.smem_per_sm / (smem + 1024)));
            per_sm = std::min(per_sm, 2048 / kDmThreads);
            const int grid = std::min(rows, per_sm * c.num_sms);
            k_ab_fp64<<<grid, kDmThreads, smem, c.stream>>>(Csrc, lds, ns, Ct, St, nt, acc, conn, s1, (s1 + 7) / 8 * 8,
                                                            tgt, ldt, npair, V, ldv, rows, c.scalar, ctr, cmax64,
                                                            bound);
            FCIB_KCHECK();
        };
        if (c.sym.on) {
            // per target rows: the first sub-problem writes them, the others add to them; each
            // sub-problem has its own row counter, all zeroed at once
            const SymSpace& y = c.sym;
            c.subctr.alloc(std::max<size_t>(y.ab.size(), 1));
            FCIB_CUDA(cudaMemsetAsync(c.subctr.p, 0, sizeof(int) * c.subctr.n, c.stream));
            for (size_t i = 0; i < y.ab.size(); i++) {
                const AbSub& u = y.ab[i];
                // source columns: a run of the source block's rows; target rows: a run of the target block
                const int64_t sb = y.d.blk[u.src] + u.col0, tb = y.d.blk[u.ha] + (int64_t)u.row0 * u.nt;
                launch(C + sb, u.lds, u.ns, C + tb, S + tb, u.nt, u.accumulate, y.conn.p + u.conn, u.kmax,
                       y.tgt32.p + u.tgt32, y.npg[u.g], y.np_g[u.g], y.Vg.p + y.vg_off[u.g], y.npg[u.g], u.rows,
                       c.subctr.p + i);
            }
        } else {
            FCIB_CUDA(cudaMemsetAsync(c.counter.p, 0, sizeof(int), c.stream));
            launch(C, nbs, nbs, C, S, nbs, 0, c.A.conn.p, s1a, c.B.tgt.p, npp, c.A.npair, c.V.p, npp, nas, c.counter.p);
        }
    } else {
        k_scale_copy<<<4 * c.num_sms, 256, 0, c.stream>>>(C, S, c.scalar, N);
        FCIB_KCHECK();
    }
    FCIB_CUDA(cudaEventRecord(ev.e[1], c.stream));
    sigma_same_spin(c, C, S, false);
    FCIB_CUDA(cudaEventRecord(ev.e[2], c.stream));
    sigma_timing(c, ev, true);
    apply_mask(c, S);
}

void ab_tc(Context& c, const double* C, double* S, bool three);
int tc_check_error(Context& c, bool opposite_spin);

void sigma_mixed(Context& c, const double* C, double* S, bool three) {
    const size_t N = (size_t)c.nvec;
    SigmaEvents ev;
    FCIB_CUDA(cudaEventRecord(ev.e[0], c.stream));
    if (c.fold_h) {
        ab_tc(c, C, S, three);
    } else {
        k_scale_copy<<<4 * c.num_sms, 256, 0, c.stream>>>(C, S, c.scalar, N);
        FCIB_KCHECK();
    }
    FCIB_CUDA(cudaEventRecord(ev.e[1], c.stream));
    sigma_same_spin(c, C, S, true);
    FCIB_CUDA(cudaEventRecord(ev.e[2], c.stream));
    sigma_timing(c, ev, false);
    apply_mask(c, S);
    const int e = tc_check_error(c, c.fold_h);
    FCIB_CHECK(e == 0, FCIB_ERR_NUMERIC, "tensor-core sigma kernel reported a timeout (code " + std::to_string(e) + ")");
}

// ------------------------------------------------------------------------------------------
// Hamiltonian diagonal, summed in the order of ActiveSpaceIntegrals::energy
// (forte/integrals/active_space_integrals.cc:206-245) starting from the scalar energy
// ------------------------------------------------------------------------------------------
struct DiagInts {
    double ha[kMaxOrb], hb[kMaxOrb];
    double aa[kMaxOrb * kMaxOrb], ab[kMaxOrb * kMaxOrb], bb[kMaxOrb * kMaxOrb];
};
__constant__ DiagInts d_diag;

// out in the engine layout: C1 (sd.on = 0) or the blocked layout of sd
__global__ void k_hdiag(const uint32_t* __restrict__ sa, const uint32_t* __restrict__ sb, int nas,
                        int nbs, int n, double e0, double* __restrict__ out, size_t N, SymDev sd) {
    for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < N; I += (size_t)gridDim.x * blockDim.x) {
        int ia, ib;
        if (sd.on) {
            sym_decode(sd, (int64_t)I, ia, ib);
        } else {
            ia = (int)(I / nbs);
            ib = (int)(I % nbs);
        }
        uint32_t Ia = sa[ia], Ib = sb[ib];
        double e = e0;
        uint32_t a = Ia;
        while (a) {
            int p = __ffs(a) - 1;
            a &= a - 1;
            e = __dadd_rn(e, d_diag.ha[p]);
            uint32_t ac = a;
            while (ac) {
                int q = __ffs(ac) - 1;
                ac &= ac - 1;
                e = __dadd_rn(e, d_diag.aa[p * n + q]);
            }
            uint32_t bc = Ib;
            while (bc) {
                int q = __ffs(bc) - 1;
                bc &= bc - 1;
                e = __dadd_rn(e, d_diag.ab[p * n + q]);
            }
        }
        uint32_t b = Ib;
        while (b) {
            int p = __ffs(b) - 1;
            b &= b - 1;
            e = __dadd_rn(e, d_diag.hb[p]);
            uint32_t bc = b;
            while (bc) {
                int q = __ffs(bc) - 1;
                bc &= bc - 1;
                e = __dadd_rn(e, d_diag.bb[p * n + q]);
            }
        }
        out[I] = e;
    }
}

void compute_hdiag(Context& c, double* out) {
    DiagInts d;
    memset(&d, 0, sizeof(d));
    const int n = c.n;
    const size_t n2 = (size_t)n * n, n3 = n2 * n;
    for (int p = 0; p < n; p++) {
        d.ha[p] = c.oei_a[p * n + p];
        d.hb[p] = c.oei_b[p * n + p];
        for (int q = 0; q < n; q++) {
            size_t idx = p * n3 + q * n2 + p * n + q;
            d.aa[p * n + q] = c.tei_aa[idx];
            d.ab[p * n + q] = c.tei_ab[idx];
            d.bb[p * n + q] = c.tei_bb[idx];
        }
    }
    FCIB_CUDA(cudaMemcpyToSymbolAsync(d_diag, &d, sizeof(d), 0, cudaMemcpyHostToDevice, c.stream));
    k_hdiag<<<8 * c.num_sms, 256, 0, c.stream>>>(c.A.str.p, c.B.str.p, (int)c.nas, (int)c.nbs, n,
                                                c.scalar, out, (size_t)c.nvec, sym_dev(c));
    FCIB_KCHECK();
}

}  // namespace fcib
