// Batched Davidson-Liu: many small CAS instances of uneven size solved in one persistent launch
// (no counterpart in the reference, whose FCISolver handles one instance per call).
//
// k_batch_dl is persistent: each CTA takes the next instance from an atomic counter (instances
// are ordered largest first) and runs the whole Davidson-Liu solve for it.  All of an instance's
// iterations run inside this one kernel:
//   sigma:   opposite-spin + one-body (folded into the pair matrix V, the engine's formulation),
//            one target alpha row at a time: B[k][R] = s_k V[P_k][R] in shared memory, every
//            (beta string, pair tile) work item forms T[Jb][R] = sum_k c[J_k][Jb] B[k][R] in
//            registers and adds it to the row at the beta replacement F_R Jb (FP64 shared-memory
//            atomics); then the alpha and beta same-spin terms over the (N-2)-electron groups,
//              s[I_i] += s_i sum_j W[i][j] s_j c[I_j],   W[i][j] = M[lab_i][lab_j] in shared memory,
//            with one thread owning each column (alpha) or row (beta), so no atomics are needed.
//            Products and sums in FP32 (mixed phase) or FP64; vectors always FP64.  The pair tile
//            (8, 16 or 32 pairs per work item) and the launch shape are autotuned.
//   subspace: G = B S^T (FP64), eigenpairs by a warp-parallel cyclic Jacobi in shared memory;
//   residuals r_k = sum_j a_jk (s_j - lambda_k b_j), diagonal corrections r/(lambda - H_II)
//            (0 when |lambda - H_II| <= 1e-6), normalised, two-pass Gram-Schmidt, discarded
//            below 1e-7 (the reference's thresholds, davidson_liu_solver.cc:432-687);
//   collapse to collapse_per_root * nroot Ritz vectors when the subspace is full.
// Convergence needs |dlambda| < e_convergence and ||r|| < r_convergence for every root; in mixed
// precision the FP32 iteration's convergence triggers a restart from the nroot Ritz vectors with
// FP64 sigma, and only the FP64 iteration's convergence ends the solve.
// Guess: unit vectors on the 2 * nroot lowest diagonal elements (no spin selection).
// Several CTAs can share an instance as a thread-block cluster (csize CTAs, autotuned 1 or 2): CTA
// crank owns the vector elements I = crank * nth + tid (mod csize * nth), every csize-th sigma row
// and a contiguous share of the same-spin lines; partial sums are combined through distributed
// shared memory in rank order, so every CTA of the cluster holds the same reduced values and takes
// the same branches.  Cluster barriers separate the phases whose data cross CTAs: before each sigma
// (basis vectors written by all CTAs), between its opposite-spin, alpha and beta same-spin parts,
// and at every partial-sum combination.
#include <cooperative_groups.h>

#include <algorithm>
#include <memory>

namespace fcib {

// Phase clocks (profiling builds only, compiled with -DFCIB_BATCH_PHASES, see forte_b200/build.py):
// thread 0 of every CTA adds the clock cycles of each phase of its solves to g_bphase, read back by
// fcib_batch_phase_cycles.  Phases: 0 opposite-spin sigma, 1 same-spin sigma, 2 G update, 3 subspace
// eigenproblem, 4 residuals, 5 preconditioner, 6 collapse, 7 Gram-Schmidt.
#ifdef FCIB_BATCH_PHASES
__device__ unsigned long long g_bphase[8];
__device__ __forceinline__ void bphase_mark(int ph, long long& t) {
    if (threadIdx.x == 0) {
        const long long now = clock64();
        atomicAdd(&g_bphase[ph], (unsigned long long)(now - t));
        t = now;
    }
}
#define FCIB_PHASE(ph) bphase_mark((ph), pt)
#else
#define FCIB_PHASE(ph) ((void)pt)
#endif

constexpr int kBMaxOrb = 12;
constexpr int kBMaxRoot = 8;
constexpr int kBMaxSub = 32;   // subspace dimension cap
constexpr int kBMaxG = 28;     // rows per same-spin group held in registers
constexpr int kBMaxThreads = 512;
constexpr int kBKC = 8;        // alpha connections per register chunk in the opposite-spin build

struct BatchInst {
    int n, na, nb, nas, nbs, s1a, s1b, ng2a, g2a, ng2b, g2b, npp, npl, msub, ncol;
    long long ndet;
    double scalar;
    const uint32_t *stra, *strb, *conna, *connb, *g2ra, *g2rb;
    const uint16_t *g2la, *g2lb;
    const int32_t* tgtb;              // beta F_R J -> I | sign << 31 (kNoTarget: none), row stride nppb
    int nppb;
    const double *V, *Ma, *Mb, *dg;  // dg: da[n] db[n] Aaa[n*n] Abb[n*n] Aab[n*n]
    double* vec;                      // hd[N] | B[msub][N] | S[msub][N] | R[nroot][N]
};

struct BatchOpts {
    int nroot, maxiter;
    double e_conv, r_conv;
    int mixed;  // FP32 sigma until converged, then FP64 sigma from the Ritz vectors to convergence
};

struct BatchShared {  // per-CTA shared scalars
    double G[kBMaxSub * kBMaxSub];
    double Ev[kBMaxSub * kBMaxSub];
    double lam[kBMaxSub];
    double lam_old[kBMaxRoot];
    double out[kBMaxSub];
    double red[(kBMaxThreads / 32) * kBMaxSub];
    int chosen[2 * kBMaxRoot];
    int inst, nb, nsig, added;
    double part[2][kBMaxSub];  // this CTA's partial sums, read by the cluster's other CTAs
};

// the cluster sharing an instance: size CTAs, this CTA's rank, the partial-sum buffer in turn
struct CInfo {
    int size, rank, pb;
};
// every thread of every CTA of the cluster (a block barrier when the cluster is one CTA)
__device__ __forceinline__ void csync(const CInfo& ci) {
    if (ci.size > 1) cooperative_groups::this_cluster().sync();
    else __syncthreads();
}

// sum over the cluster of v[0..K) (K <= kBMaxSub); results in S.out of every CTA.  The partial
// buffers alternate between calls: a CTA writes a buffer again only after the barrier of the next
// call, which every other CTA reaches after reading it.
__device__ __forceinline__ void bsum(double (&v)[kBMaxSub], int K, BatchShared& S, CInfo& ci) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < kBMaxSub; k++) {
        if (k < K) {
            double x = v[k];
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            if (lane == 0) S.red[w * kBMaxSub + k] = x;
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        double s = 0.0;
        for (int i = 0; i < nw; i++) s += S.red[i * kBMaxSub + k];
        if (ci.size == 1) S.out[k] = s;
        else S.part[ci.pb][k] = s;
    }
    if (ci.size > 1) {
        auto cl = cooperative_groups::this_cluster();
        cl.sync();
        for (int k = threadIdx.x; k < K; k += blockDim.x) {
            double t = 0.0;
            for (int r = 0; r < ci.size; r++) t += cl.map_shared_rank(&S.part[ci.pb][0], r)[k];
            S.out[k] = t;
        }
        ci.pb ^= 1;
    }
    __syncthreads();
}

// S.out[j] = <x, B_j> for j < nb.  x may be a sigma vector that other CTAs of the cluster wrote, so
// its loads stay coherent (not __restrict__).
__device__ void bdots(const double* x, const double* __restrict__ B, size_t N, int nb, BatchShared& S, CInfo& ci) {
    double acc[kBMaxSub];
#pragma unroll
    for (int j = 0; j < kBMaxSub; j++) acc[j] = 0.0;
    for (size_t I = (size_t)ci.rank * blockDim.x + threadIdx.x; I < N; I += (size_t)ci.size * blockDim.x) {
        const double xi = x[I];
#pragma unroll
        for (int j = 0; j < kBMaxSub; j++)
            if (j < nb) acc[j] = fma(B[(size_t)j * N + I], xi, acc[j]);
    }
    bsum(acc, nb, S, ci);
}

// c is not __restrict__: the other CTAs of a cluster write it during the kernel, so its loads must
// stay coherent (no read-only cache path).
// sigma of one instance by the whole CTA, FP64 in and out, products and sums in T (float in the
// mixed phase, double otherwise).  scratch: shared memory for the pair block B[k][R] (T), the sigma
// row (double) and the row's connections; grp: a same-spin group's rows and labels.
//   opposite spin + folded one-body terms, one target alpha row Ia at a time:
//     B[k][R] = s_k V[P_k][R] for the row's connections k;  every (Jb, 16-pair chunk) work item forms
//     T[Jb][R] = sum_k c[J_k][Jb] B[k][R] in registers and adds s_R T[Jb][R] to the sigma row at
//     F_R Jb (FP64 shared-memory atomics); the row then goes to global memory.
//   same spin: per (N-2)-electron group, W[i][j] = M[lab_i][lab_j] in shared memory, every thread
//     owns a column (alpha) or row (beta) line and applies W to the group's rows of its line.
// RC: pairs per work item in the opposite-spin term (the autotuned sigma tile: 8, 16 or 32)
template <typename T, int RC>
__device__ void bsigma(const BatchInst& P, const double* __restrict__ V, const double* __restrict__ Ma,
                       const double* __restrict__ Mb, const double* c, double* __restrict__ s,
                       unsigned char* __restrict__ scratch, int* __restrict__ grp, const CInfo& ci,
                       long long& pt) {
    const int nbs = P.nbs, nas = P.nas, npp = P.npp, npl = P.npl, s1a = P.s1a;
    const int tid = threadIdx.x, nth = blockDim.x;
    const int nch = (npp + RC - 1) / RC;
    const int ldb = nch * RC;  // B rows padded to whole chunks (zeros)
    T* Bt = reinterpret_cast<T*>(scratch);
    double* srow = reinterpret_cast<double*>(scratch + (((size_t)s1a * ldb * sizeof(T) + 15) / 16) * 16);
    uint32_t* cs = reinterpret_cast<uint32_t*>(srow + nbs);
    for (int ia = ci.rank; ia < nas; ia += ci.size) {  // every csize-th row
        for (int k = tid; k < s1a; k += nth) cs[k] = P.conna[(size_t)ia * s1a + k];
        for (int j = tid; j < nbs; j += nth) srow[j] = P.scalar * c[(size_t)ia * nbs + j];
        __syncthreads();
        for (int idx = tid; idx < s1a * ldb; idx += nth) {
            const int k = idx / ldb, R = idx - k * ldb;
            double v = 0.0;
            if (R < npp) {
                const uint32_t e = cs[k];
                v = V[(size_t)((e >> 21) & 0x3FFu) * npp + R];
                if (e >> 31) v = -v;
            }
            Bt[idx] = (T)v;
        }
        __syncthreads();
        for (int item = tid; item < nbs * nch; item += nth) {
            const int ch = item / nbs, jb = item - ch * nbs;
            T acc[RC];
#pragma unroll
            for (int r = 0; r < RC; r++) acc[r] = (T)0;
            const T* br = Bt + ch * RC;
            // the gathered elements of 8 connections are loaded together, then used
            for (int k0 = 0; k0 < s1a; k0 += 8) {
                T a[8];
#pragma unroll
                for (int u = 0; u < 8; u++)
                    a[u] = (k0 + u < s1a) ? (T)c[(size_t)(cs[k0 + u] & kConnIdxMask) * nbs + jb] : (T)0;
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    if (k0 + u < s1a) {
#pragma unroll
                        for (int r = 0; r < RC; r++) acc[r] = fma(a[u], br[(size_t)(k0 + u) * ldb + r], acc[r]);
                    }
                }
            }
            const int32_t* tg = P.tgtb + (size_t)jb * P.nppb + ch * RC;
#pragma unroll
            for (int r = 0; r < RC; r++) {
                if (ch * RC + r < npp) {
                    const int32_t t = tg[r];
                    if (t != kNoTarget) {
                        const double v = (double)acc[r];
                        atomicAdd(&srow[t & kConnIdxMask], (t & (int32_t)kSignBit) ? -v : v);
                    }
                }
            }
        }
        __syncthreads();
        for (int j = tid; j < nbs; j += nth) s[(size_t)ia * nbs + j] = srow[j];
        __syncthreads();
    }
    csync(ci);  // every row written before the same-spin terms add to them
    FCIB_PHASE(0);
    // same-spin terms over the (N-2)-electron groups
    T* W = reinterpret_cast<T*>(scratch);  // [kBMaxG][kBMaxG], reuses the opposite-spin scratch
    for (int spin = 0; spin < 2; spin++) {
        const int ng = spin ? P.ng2b : P.ng2a;
        if (!ng) {
            csync(ci);
            continue;
        }
        const int m = spin ? P.g2b : P.g2a;
        const uint32_t* growp = spin ? P.g2rb : P.g2ra;
        const uint16_t* glabp = spin ? P.g2lb : P.g2la;
        const double* M = spin ? Mb : Ma;
        const int nlines = spin ? nas : nbs;   // columns (alpha) or rows (beta) owned by threads
        const size_t stride = spin ? 1 : (size_t)nbs;  // distance between consecutive strings
        const size_t lstep = spin ? (size_t)nbs : 1;   // distance between consecutive lines
        int* rows_s = grp;
        int* labs_s = grp + kBMaxG;
        for (int g = 0; g < ng; g++) {
            if (tid < m) {
                rows_s[tid] = (int)growp[(size_t)g * m + tid];
                labs_s[tid] = glabp[(size_t)g * m + tid];
            }
            __syncthreads();
            for (int idx = tid; idx < m * m; idx += nth) {
                const int i = idx / m, j = idx - i * m;
                W[i * kBMaxG + j] = (T)M[(size_t)labs_s[i] * npl + labs_s[j]];
            }
            __syncthreads();
            // this CTA's contiguous share of the lines
            const int l0 = (int)((long long)ci.rank * nlines / ci.size);
            const int l1 = (int)((long long)(ci.rank + 1) * nlines / ci.size);
            for (int line = l0 + tid; line < l1; line += nth) {
                const double* cl = c + (size_t)line * lstep;
                double* sl = s + (size_t)line * lstep;
                T x[kBMaxG];
#pragma unroll
                for (int j = 0; j < kBMaxG; j++) {
                    x[j] = (T)0;
                    if (j < m) {
                        const uint32_t r = (uint32_t)rows_s[j];
                        const T v = (T)cl[(size_t)(r & kConnIdxMask) * stride];
                        x[j] = (r >> 31) ? -v : v;
                    }
                }
                for (int i = 0; i < m; i++) {
                    const T* wr = W + i * kBMaxG;
                    T a = (T)0;
#pragma unroll
                    for (int j = 0; j < kBMaxG; j++)
                        if (j < m) a = fma(wr[j], x[j], a);
                    const uint32_t r = (uint32_t)rows_s[i];
                    const double ad = (double)a;
                    sl[(size_t)(r & kConnIdxMask) * stride] += (r >> 31) ? -ad : ad;
                }
            }
            __syncthreads();
        }
        csync(ci);  // alpha lines (columns) done before the beta lines (rows); sigma complete at the end
    }
    FCIB_PHASE(1);
}

// shared-memory scratch of bsigma in bytes (the larger of the opposite-spin block and the group W),
// for the largest pair tile (32)
__host__ __device__ inline size_t bsigma_scratch(int s1a, int npp, int nbs) {
    const int ldb = (npp + 31) / 32 * 32;
    const size_t opp = ((size_t)s1a * ldb * sizeof(double) + 15) / 16 * 16 + (size_t)nbs * 8 + (size_t)s1a * 4;
    const size_t grp = (size_t)kBMaxG * kBMaxG * sizeof(double);
    return opp > grp ? opp : grp;
}

// eigenpairs of the symmetric n x n matrix S.G (leading dimension kBMaxSub) by cyclic Jacobi
// on warp 0: S.lam ascending, S.Ev columns = eigenvectors
__device__ void bjacobi(BatchShared& S, int n) {
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        double* A = S.G;  // destroyed; the caller keeps a copy
        double* Vv = S.Ev;
        for (int i = lane; i < n * kBMaxSub; i += 32) Vv[i] = 0.0;
        __syncwarp();
        for (int i = lane; i < n; i += 32) Vv[i * kBMaxSub + i] = 1.0;
        __syncwarp();
        for (int sweep = 0; sweep < 30; sweep++) {
            double off = 0.0, dia = 0.0;
            for (int i = lane; i < n * n; i += 32) {
                const int p = i / n, q = i - p * n;
                const double a = A[p * kBMaxSub + q];
                if (p != q) off += a * a; else dia += a * a;
            }
            for (int o = 16; o > 0; o >>= 1) {
                off += __shfl_xor_sync(0xffffffffu, off, o);
                dia += __shfl_xor_sync(0xffffffffu, dia, o);
            }
            if (off <= 1e-26 * dia || off == 0.0) break;
            for (int p = 0; p < n - 1; p++)
                for (int q = p + 1; q < n; q++) {
                    const double apq = A[p * kBMaxSub + q];
                    const double app = A[p * kBMaxSub + p], aqq = A[q * kBMaxSub + q];
                    if (fabs(apq) <= 1e-15 * sqrt(fabs(app * aqq)) || fabs(apq) < 1e-300) continue;
                    const double theta = (aqq - app) / (2.0 * apq);
                    const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                    const double cs = 1.0 / sqrt(t * t + 1.0), sn = t * cs;
                    __syncwarp();
                    for (int k = lane; k < n; k += 32) {
                        const double akp = A[k * kBMaxSub + p], akq = A[k * kBMaxSub + q];
                        A[k * kBMaxSub + p] = cs * akp - sn * akq;
                        A[k * kBMaxSub + q] = sn * akp + cs * akq;
                        const double vkp = Vv[k * kBMaxSub + p], vkq = Vv[k * kBMaxSub + q];
                        Vv[k * kBMaxSub + p] = cs * vkp - sn * vkq;
                        Vv[k * kBMaxSub + q] = sn * vkp + cs * vkq;
                    }
                    __syncwarp();
                    for (int k = lane; k < n; k += 32) {
                        const double apk = A[p * kBMaxSub + k], aqk = A[q * kBMaxSub + k];
                        A[p * kBMaxSub + k] = cs * apk - sn * aqk;
                        A[q * kBMaxSub + k] = sn * apk + cs * aqk;
                    }
                    __syncwarp();
                }
        }
        if (lane == 0) {
            for (int i = 0; i < n; i++) S.lam[i] = A[i * kBMaxSub + i];
            // selection sort, ascending, with the eigenvector columns
            for (int i = 0; i < n; i++) {
                int b = i;
                for (int j = i + 1; j < n; j++)
                    if (S.lam[j] < S.lam[b]) b = j;
                if (b != i) {
                    const double t = S.lam[i];
                    S.lam[i] = S.lam[b];
                    S.lam[b] = t;
                    for (int k = 0; k < n; k++) {
                        const double u = Vv[k * kBMaxSub + i];
                        Vv[k * kBMaxSub + i] = Vv[k * kBMaxSub + b];
                        Vv[k * kBMaxSub + b] = u;
                    }
                }
            }
        }
    }
    __syncthreads();
}

template <int RC>
__global__ void __launch_bounds__(kBMaxThreads, 1)
    k_batch_dl(const BatchInst* __restrict__ insts, const int* __restrict__ order, int ninst, int* __restrict__ counter,
               BatchOpts o, double* __restrict__ energies, int* __restrict__ iters, int* __restrict__ conv, int npp_max,
               int npl_max, int xcap, int csize) {
    extern __shared__ __align__(16) unsigned char batch_smem[];
    BatchShared& S = *reinterpret_cast<BatchShared*>(batch_smem);
    double* Vs = reinterpret_cast<double*>(batch_smem + sizeof(BatchShared));
    double* Mas = Vs + (size_t)npp_max * npp_max;
    double* Mbs = Mas + (size_t)npl_max * npl_max;
    unsigned char* Xs = reinterpret_cast<unsigned char*>(Mbs + (size_t)npl_max * npl_max);
    __shared__ double Gkeep[kBMaxSub * kBMaxSub];
    __shared__ int grp[2 * kBMaxG];
    __shared__ BatchInst sP;  // one copy per CTA (a per-thread copy would live in local memory)
    const int tid = threadIdx.x, nth = blockDim.x;
    CInfo ci{csize, csize > 1 ? (int)cooperative_groups::this_cluster().block_rank() : 0, 0};
    // this CTA's share of an instance's vector elements
#define BFOR(I) for (size_t I = (size_t)ci.rank * nth + tid; I < N; I += (size_t)ci.size * nth)
    for (;;) {
        // rank 0 takes the next instance for the cluster; the others read it from its shared memory
        if (tid == 0 && ci.rank == 0) S.inst = atomicAdd(counter, 1);
        csync(ci);
        const int slot = ci.size > 1 ? *cooperative_groups::this_cluster().map_shared_rank(&S.inst, 0) : S.inst;
        if (slot >= ninst) break;
        const int id = order[slot];
        if (tid == 0) sP = insts[id];
        __syncthreads();
        const BatchInst& P = sP;
        const size_t N = (size_t)P.ndet;
        const int nroot = o.nroot, msub = P.msub;
        double* hd = P.vec;
        double* B = hd + N;
        double* Sg = B + (size_t)msub * N;
        double* R = Sg + (size_t)msub * N;
        for (int i = tid; i < P.npp * P.npp; i += nth) Vs[i] = P.V[i];
        for (int i = tid; i < P.npl * P.npl; i += nth) {
            Mas[i] = P.Ma[i];
            Mbs[i] = P.Mb[i];
        }
        // diagonal
        {
            const int n = P.n;
            const double* da = P.dg;
            const double* db = da + n;
            const double* Aaa = db + n;
            const double* Abb = Aaa + n * n;
            const double* Aab = Abb + n * n;
            BFOR(e) {
                const int ia = (int)(e / P.nbs), ib = (int)(e - (size_t)ia * P.nbs);
                const uint32_t sa = P.stra[ia], sb = P.strb[ib];
                double h = P.scalar;
                for (uint32_t x = sa; x; x &= x - 1) {
                    const int p = __ffs(x) - 1;
                    h += da[p];
                    for (uint32_t y = x & (x - 1); y; y &= y - 1) h += Aaa[p * n + __ffs(y) - 1];
                    for (uint32_t y = sb; y; y &= y - 1) h += Aab[p * n + __ffs(y) - 1];
                }
                for (uint32_t x = sb; x; x &= x - 1) {
                    const int p = __ffs(x) - 1;
                    h += db[p];
                    for (uint32_t y = x & (x - 1); y; y &= y - 1) h += Abb[p * n + __ffs(y) - 1];
                }
                hd[e] = h;
            }
        }
        csync(ci);  // the guess reads every diagonal element
        // guess: unit vectors on the lowest diagonal elements
        const int nguess = min(min(2 * nroot, msub), (int)N);
        for (int g = 0; g < nguess; g++) {
            double best = 1e300;
            long long bi = -1;
            for (size_t e = tid; e < N; e += nth) {
                bool used = false;
                for (int q = 0; q < g; q++) used |= (S.chosen[q] == (int)e);
                if (!used && (hd[e] < best || (hd[e] == best && (long long)e < bi))) {
                    best = hd[e];
                    bi = (long long)e;
                }
            }
            for (int off = 16; off > 0; off >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, off);
                const long long oi = __shfl_xor_sync(0xffffffffu, bi, off);
                if (ob < best || (ob == best && oi >= 0 && (bi < 0 || oi < bi))) {
                    best = ob;
                    bi = oi;
                }
            }
            if ((tid & 31) == 0) {
                S.red[(tid >> 5) * 2] = best;
                S.red[(tid >> 5) * 2 + 1] = (double)bi;
            }
            __syncthreads();
            if (tid == 0) {
                double b0 = 1e300;
                long long i0 = -1;
                for (int w = 0; w < nth / 32; w++) {
                    const double bv = S.red[2 * w];
                    const long long iv = (long long)S.red[2 * w + 1];
                    if (iv >= 0 && (bv < b0 || (bv == b0 && iv < i0))) {
                        b0 = bv;
                        i0 = iv;
                    }
                }
                S.chosen[g] = (int)i0;
            }
            __syncthreads();
        }
        for (int g = 0; g < nguess; g++) {
            double* bg = B + (size_t)g * N;
            BFOR(e) bg[e] = ((int)e == S.chosen[g]) ? 1.0 : 0.0;
        }
        if (tid == 0) {
            S.nb = nguess;
            S.nsig = 0;
        }
        for (int k = tid; k < kBMaxRoot; k += nth) S.lam_old[k] = 0.0;
        __syncthreads();
        int it = 0;
        long long pt = 0;
#ifdef FCIB_BATCH_PHASES
        pt = clock64();
#endif
        bool done = false;
        bool fp64_phase = !o.mixed;  // mixed: FP32 sigma first, FP64 sigma from the restart on
        while (it < o.maxiter) {
            const int nb = S.nb;
            csync(ci);  // the new basis vectors, written by every CTA, are read whole by sigma
            // sigma of the new basis vectors and the new columns of G
            for (int j = S.nsig; j < nb; j++) {
                if (o.mixed && !fp64_phase)
                    bsigma<float, RC>(P, Vs, Mas, Mbs, B + (size_t)j * N, Sg + (size_t)j * N, Xs, grp, ci, pt);
                else
                    bsigma<double, RC>(P, Vs, Mas, Mbs, B + (size_t)j * N, Sg + (size_t)j * N, Xs, grp, ci, pt);
                bdots(Sg + (size_t)j * N, B, N, nb, S, ci);
                for (int i = tid; i < nb; i += nth) {
                    Gkeep[i * kBMaxSub + j] = S.out[i];
                    Gkeep[j * kBMaxSub + i] = S.out[i];
                }
                __syncthreads();
                FCIB_PHASE(2);
            }
            if (tid == 0) S.nsig = nb;
            for (int i = tid; i < nb * kBMaxSub; i += nth) {
                const int r = i / kBMaxSub, cc = i - r * kBMaxSub;
                S.G[i] = (cc < nb) ? 0.5 * (Gkeep[r * kBMaxSub + cc] + Gkeep[cc * kBMaxSub + r]) : 0.0;
            }
            __syncthreads();
            bjacobi(S, nb);
            FCIB_PHASE(3);
            // residuals and their norms
            {
                double acc[kBMaxSub];
#pragma unroll
                for (int k = 0; k < kBMaxSub; k++) acc[k] = 0.0;
                BFOR(I) {
                    double rs[kBMaxRoot], rb[kBMaxRoot];
#pragma unroll
                    for (int k = 0; k < kBMaxRoot; k++) rs[k] = rb[k] = 0.0;
                    for (int j = 0; j < nb; j++) {
                        const double sj = Sg[(size_t)j * N + I], bj = B[(size_t)j * N + I];
#pragma unroll
                        for (int k = 0; k < kBMaxRoot; k++)
                            if (k < nroot) {
                                const double a = S.Ev[j * kBMaxSub + k];
                                rs[k] = fma(a, sj, rs[k]);
                                rb[k] = fma(a, bj, rb[k]);
                            }
                    }
#pragma unroll
                    for (int k = 0; k < kBMaxRoot; k++)
                        if (k < nroot) {
                            const double r = rs[k] - S.lam[k] * rb[k];
                            R[(size_t)k * N + I] = r;
                            acc[k] = fma(r, r, acc[k]);
                        }
                }
                bsum(acc, nroot, S, ci);
            }
            FCIB_PHASE(4);
            it++;
            bool ok = true;
            for (int k = 0; k < nroot; k++)
                ok = ok && fabs(S.lam[k] - S.lam_old[k]) < o.e_conv && sqrt(S.out[k]) < o.r_conv;
            if ((size_t)nb >= N) ok = true;  // the basis spans the space: the Ritz values are exact
            if (ok && fp64_phase) {
                done = true;
                break;
            }
            if (ok) {
                // mixed: the FP32 iteration has converged; restart from the nroot Ritz vectors and
                // recompute their sigma in FP64, which alone decides convergence from here on
                BFOR(I) {
                    double tb[kBMaxRoot];
#pragma unroll
                    for (int k = 0; k < kBMaxRoot; k++) tb[k] = 0.0;
                    for (int j = 0; j < nb; j++) {
                        const double bj = B[(size_t)j * N + I];
#pragma unroll
                        for (int k = 0; k < kBMaxRoot; k++)
                            if (k < nroot) tb[k] = fma(S.Ev[j * kBMaxSub + k], bj, tb[k]);
                    }
#pragma unroll
                    for (int k = 0; k < kBMaxRoot; k++)
                        if (k < nroot) B[(size_t)k * N + I] = tb[k];
                }
                __syncthreads();
                for (int i = tid; i < kBMaxSub * kBMaxSub; i += nth) Gkeep[i] = 0.0;
                for (int k = tid; k < nroot; k += nth) S.lam_old[k] = S.lam[k];
                if (tid == 0) {
                    S.nb = nroot;
                    S.nsig = 0;
                }
                fp64_phase = true;
                __syncthreads();
                continue;
            }
            __syncthreads();
            for (int k = tid; k < nroot; k += nth) S.lam_old[k] = S.lam[k];
            // diagonal corrections
            BFOR(I) {
                const double h = hd[I];
                for (int k = 0; k < nroot; k++) {
                    const double den = S.lam[k] - h;
                    double* r = R + (size_t)k * N + I;
                    *r = (fabs(den) > 1.0e-6) ? *r / den : 0.0;
                }
            }
            __syncthreads();
            FCIB_PHASE(5);
            // collapse when the subspace would overflow
            if (nb + nroot > msub) {
                const int ncol = min(P.ncol, nb);
                BFOR(I) {
                    double tb[2 * kBMaxRoot], ts[2 * kBMaxRoot];
#pragma unroll
                    for (int k = 0; k < 2 * kBMaxRoot; k++) tb[k] = ts[k] = 0.0;
                    for (int j = 0; j < nb; j++) {
                        const double bj = B[(size_t)j * N + I], sj = Sg[(size_t)j * N + I];
#pragma unroll
                        for (int k = 0; k < 2 * kBMaxRoot; k++)
                            if (k < ncol) {
                                tb[k] = fma(S.Ev[j * kBMaxSub + k], bj, tb[k]);
                                ts[k] = fma(S.Ev[j * kBMaxSub + k], sj, ts[k]);
                            }
                    }
#pragma unroll
                    for (int k = 0; k < 2 * kBMaxRoot; k++)
                        if (k < ncol) {
                            B[(size_t)k * N + I] = tb[k];
                            Sg[(size_t)k * N + I] = ts[k];
                        }
                }
                __syncthreads();
                for (int i = tid; i < kBMaxSub * kBMaxSub; i += nth) {
                    const int r = i / kBMaxSub, cc = i - r * kBMaxSub;
                    Gkeep[i] = (r == cc && r < ncol) ? S.lam[r] : 0.0;
                }
                if (tid == 0) {
                    S.nb = ncol;
                    S.nsig = ncol;
                }
                __syncthreads();
            }
            FCIB_PHASE(6);
            // add the normalised, orthogonalised corrections
            if (tid == 0) S.added = 0;
            __syncthreads();
            for (int k = 0; k < nroot; k++) {
                const int nbk = S.nb;
                if (nbk >= msub) break;
                double* r = R + (size_t)k * N;
                {
                    double a[kBMaxSub];
#pragma unroll
                    for (int j = 0; j < kBMaxSub; j++) a[j] = 0.0;
                    BFOR(I) a[0] = fma(r[I], r[I], a[0]);
                    bsum(a, 1, S, ci);
                }
                const double nrm0 = sqrt(S.out[0]);
                if (!(nrm0 > 0.0)) continue;
                BFOR(I) r[I] /= nrm0;
                __syncthreads();
                for (int pass = 0; pass < 2; pass++) {
                    bdots(r, B, N, nbk, S, ci);
                    BFOR(I) {
                        double v = r[I];
                        for (int j = 0; j < nbk; j++) v -= S.out[j] * B[(size_t)j * N + I];
                        r[I] = v;
                    }
                    __syncthreads();
                }
                {
                    double a[kBMaxSub];
#pragma unroll
                    for (int j = 0; j < kBMaxSub; j++) a[j] = 0.0;
                    BFOR(I) a[0] = fma(r[I], r[I], a[0]);
                    bsum(a, 1, S, ci);
                }
                const double nrm = sqrt(S.out[0]);
                if (!(nrm >= 1.0e-7)) continue;
                double* bn = B + (size_t)nbk * N;
                BFOR(I) bn[I] = r[I] / nrm;
                __syncthreads();
                if (tid == 0) {
                    S.nb = nbk + 1;
                    S.added++;
                }
                __syncthreads();
            }
            FCIB_PHASE(7);
            if (S.added == 0) break;
        }
        if (ci.rank == 0) {
            if (tid < nroot) energies[(size_t)id * nroot + tid] = S.lam[tid];
            if (tid == 0) {
                iters[id] = it;
                conv[id] = done ? 1 : 0;
            }
        }
        __syncthreads();
    }
#undef BFOR
    // no CTA leaves while another may still read its shared memory
    if (ci.size > 1) cooperative_groups::this_cluster().sync();
}

}  // namespace fcib

// ------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------
struct fcib_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    int num_sms = 0, smem_optin = 0;
    int ninst = 0, nroot = 0;
    fcib::BatchOpts opts{};
    std::vector<std::unique_ptr<fcib::SpinTables>> tables;
    fcib::DBuf<double> pool, vec, energies;
    fcib::DBuf<fcib::BatchInst> insts;
    fcib::DBuf<int> order, counter, iters, conv;
    int npp_max = 0, npl_max = 0, xcap = 0;
    size_t smem = 0;
    int threads = 512, ctas_per_sm = 1, pair_tile = 32, cluster = 1;  // the default shape (see fcib_batch_create)
    cudaGraphExec_t graph = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double last_ms = 0.0;
    ~fcib_batch() {
        if (graph) cudaGraphExecDestroy(graph);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace fcib {

static void batch_capture(fcib_batch* b) {
    if (b->graph) {
        FCIB_CUDA(cudaGraphExecDestroy(b->graph));
        b->graph = nullptr;
    }
    // clusters of b->cluster CTAs, one cluster per instance at a time, at most one cluster slot per
    // (ctas_per_sm x SMs / cluster) and never more clusters than instances
    const int cl = b->cluster;
    const int grid = std::min(b->ninst, b->ctas_per_sm * b->num_sms / cl) * cl;
    cudaGraph_t g;
    FCIB_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(b->counter.p, 0, sizeof(int), b->stream);
    auto kern = b->pair_tile == 8 ? k_batch_dl<8> : b->pair_tile == 32 ? k_batch_dl<32> : k_batch_dl<16>;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(b->threads);
    cfg.dynamicSmemBytes = b->smem;
    cfg.stream = b->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = cl > 1 ? 1 : 0;
    cudaError_t le = cudaLaunchKernelEx(&cfg, kern, (const BatchInst*)b->insts.p, (const int*)b->order.p, b->ninst,
                                        b->counter.p, b->opts, b->energies.p, b->iters.p, b->conv.p, b->npp_max,
                                        b->npl_max, b->xcap, cl);
    if (le == cudaSuccess) le = cudaGetLastError();
    cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
    FCIB_CUDA(le);
    FCIB_CUDA(ce);
    cudaError_t ie = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    FCIB_CUDA(ie);
}

static double batch_run(fcib_batch* b) {
    if (!b->graph) batch_capture(b);
    FCIB_CUDA(cudaEventRecord(b->e0, b->stream));
    FCIB_CUDA(cudaGraphLaunch(b->graph, b->stream));
    FCIB_CUDA(cudaEventRecord(b->e1, b->stream));
    FCIB_CUDA(cudaEventSynchronize(b->e1));
    g_launch_count++;
    float ms = 0.f;
    FCIB_CUDA(cudaEventElapsedTime(&ms, b->e0, b->e1));
    b->last_ms = ms;
    return ms;
}

}  // namespace fcib

extern "C" {

int fcib_batch_create(fcib_batch** out, int device, int ninst, const int* n, const int* na, const int* nb,
                      const double* scalar, const double* const* oei_a, const double* const* oei_b,
                      const double* const* tei_aa, const double* const* tei_ab, const double* const* tei_bb,
                      int nroot, const fcib_options* opt) {
    using namespace fcib;
    if (!out || ninst <= 0 || !n || !na || !nb || !scalar || !oei_a || !oei_b || !tei_aa || !tei_ab || !tei_bb || !opt) {
        set_error("fcib_batch_create: null or empty argument");
        return FCIB_ERR_ARG;
    }
    *out = nullptr;
    auto* b = new fcib_batch();
    int rc = guarded(nullptr, [&] {
        FCIB_CHECK(nroot >= 1 && nroot <= kBMaxRoot, FCIB_ERR_UNSUPPORTED, "fcib_batch_create: 1..8 roots per instance");
        FCIB_CHECK(opt->maxiter >= 1 && opt->subspace_per_root >= 2 && opt->collapse_per_root >= 1 &&
                       opt->collapse_per_root < opt->subspace_per_root,
                   FCIB_ERR_ARG, "fcib_batch_create: bad Davidson options");
        b->device = device;
        FCIB_CUDA(cudaSetDevice(device));
        FCIB_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        FCIB_CUDA(cudaEventCreate(&b->e0));
        FCIB_CUDA(cudaEventCreate(&b->e1));
        cudaDeviceProp prop;
        FCIB_CUDA(cudaGetDeviceProperties(&prop, device));
        b->num_sms = prop.multiProcessorCount;
        b->smem_optin = (int)prop.sharedMemPerBlockOptin;
        b->ninst = ninst;
        b->nroot = nroot;
        const int msub = std::min(kBMaxSub, opt->subspace_per_root * nroot);
        b->opts = BatchOpts{nroot, opt->maxiter, opt->e_convergence, opt->r_convergence,
                            opt->precision != FCIB_PREC_FP64 ? 1 : 0};
        std::vector<BatchInst> hi(ninst);
        std::vector<double> pool;
        std::vector<size_t> off_V(ninst), off_Ma(ninst), off_Mb(ninst), off_dg(ninst);
        size_t vec_total = 0;
        std::vector<size_t> off_vec(ninst);
        for (int i = 0; i < ninst; i++) {
            const int ni = n[i], a = na[i], bb = nb[i];
            FCIB_CHECK(ni >= 2 && ni <= kBMaxOrb && a >= 1 && bb >= 1 && a <= ni && bb <= ni, FCIB_ERR_UNSUPPORTED,
                       "fcib_batch_create: instances need 2..12 orbitals and at least one electron of each spin");
            auto ta = std::make_unique<SpinTables>();
            build_spin_tables(*ta, ni, a, false, b->stream);
            SpinTables* tb = ta.get();
            std::unique_ptr<SpinTables> tbo;
            if (bb != a) {
                tbo = std::make_unique<SpinTables>();
                build_spin_tables(*tbo, ni, bb, false, b->stream);
                tb = tbo.get();
            }
            FCIB_CHECK(ta->g2 <= kBMaxG && tb->g2 <= kBMaxG, FCIB_ERR_UNSUPPORTED,
                       "fcib_batch_create: same-spin groups larger than 28 rows (too few electrons for the orbitals)");
            BatchInst& P = hi[i];
            P.n = ni;
            P.na = a;
            P.nb = bb;
            P.nas = ta->nstr;
            P.nbs = tb->nstr;
            P.s1a = ta->s1;
            P.s1b = tb->s1;
            P.ng2a = ta->ng2;
            P.g2a = ta->g2;
            P.ng2b = tb->ng2;
            P.g2b = tb->g2;
            P.npp = ni * (ni + 1) / 2;
            P.npl = ni * (ni - 1) / 2;
            P.ndet = (long long)P.nas * P.nbs;
            P.msub = (int)std::min<long long>(msub, P.ndet);
            P.ncol = std::min(opt->collapse_per_root * nroot, P.msub);
            FCIB_CHECK(nroot <= P.ndet, FCIB_ERR_ARG, "fcib_batch_create: more roots than determinants");
            FCIB_CHECK(P.msub >= std::min<long long>(2 * nroot, P.ndet) && P.msub > nroot, FCIB_ERR_ARG,
                       "fcib_batch_create: subspace smaller than two vectors per root");
            P.scalar = scalar[i];
            P.stra = ta->str.p;
            P.strb = tb->str.p;
            P.conna = ta->conn.p;
            P.connb = tb->conn.p;
            P.g2ra = ta->g2row.p;
            P.g2la = ta->g2lab.p;
            P.g2rb = tb->g2row.p;
            P.g2lb = tb->g2lab.p;
            P.tgtb = tb->tgt.p;
            P.nppb = tb->npair_pad;
            b->tables.push_back(std::move(ta));
            if (tbo) b->tables.push_back(std::move(tbo));
            // integrals: pair matrix with folded one-body terms, same-spin pair matrices, diagonal pieces
            const size_t n2 = (size_t)ni * ni, n3 = n2 * ni;
            const double* tab = tei_ab[i];
            const double* taa = tei_aa[i];
            const double* tbbp = tei_bb[i];
            const double* ha = oei_a[i];
            const double* hb = oei_b[i];
            off_V[i] = pool.size();
            pool.resize(pool.size() + (size_t)P.npp * P.npp);
            for (int p = 0; p < ni; p++)
                for (int q = 0; q <= p; q++)
                    for (int r = 0; r < ni; r++)
                        for (int s = 0; s <= r; s++) {
                            const int PP = p * (p + 1) / 2 + q, RR = r * (r + 1) / 2 + s;
                            double v = tab[p * n3 + r * n2 + q * ni + s];
                            if (r == s) v += ha[p * ni + q] / bb;
                            if (p == q) v += hb[r * ni + s] / a;
                            pool[off_V[i] + (size_t)PP * P.npp + RR] = v;
                        }
            off_Ma[i] = pool.size();
            pool.resize(pool.size() + 2 * (size_t)P.npl * P.npl);
            off_Mb[i] = off_Ma[i] + (size_t)P.npl * P.npl;
            for (int p = 0; p < ni; p++)
                for (int q = 0; q < p; q++)
                    for (int r = 0; r < ni; r++)
                        for (int s = 0; s < r; s++) {
                            const size_t PQ = p * (p - 1) / 2 + q, RS = r * (r - 1) / 2 + s;
                            const size_t idx = p * n3 + q * n2 + r * ni + s;
                            pool[off_Ma[i] + PQ * P.npl + RS] = taa[idx];
                            pool[off_Mb[i] + PQ * P.npl + RS] = tbbp[idx];
                        }
            off_dg[i] = pool.size();
            pool.resize(pool.size() + 2 * ni + 3 * n2);
            double* dg = pool.data() + off_dg[i];
            for (int p = 0; p < ni; p++) {
                dg[p] = ha[p * ni + p];
                dg[ni + p] = hb[p * ni + p];
                for (int q = 0; q < ni; q++) {
                    const size_t pqpq = p * n3 + q * n2 + p * ni + q;
                    dg[2 * ni + p * ni + q] = taa[pqpq];
                    dg[2 * ni + n2 + p * ni + q] = tbbp[pqpq];
                    dg[2 * ni + 2 * n2 + p * ni + q] = tab[pqpq];
                }
            }
            b->npp_max = std::max(b->npp_max, P.npp);
            b->npl_max = std::max(b->npl_max, P.npl);
            off_vec[i] = vec_total;
            vec_total += (size_t)(1 + 2 * P.msub + nroot) * P.ndet;
        }
        b->pool.upload(pool, b->stream);
        b->vec.alloc(vec_total);
        for (int i = 0; i < ninst; i++) {
            hi[i].V = b->pool.p + off_V[i];
            hi[i].Ma = b->pool.p + off_Ma[i];
            hi[i].Mb = b->pool.p + off_Mb[i];
            hi[i].dg = b->pool.p + off_dg[i];
            hi[i].vec = b->vec.p + off_vec[i];
        }
        b->insts.upload(hi, b->stream);
        std::vector<int> ord(ninst);
        for (int i = 0; i < ninst; i++) ord[i] = i;
        std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return hi[x].ndet > hi[y].ndet; });
        b->order.upload(ord, b->stream);
        b->counter.alloc(1);
        b->iters.alloc(ninst);
        b->conv.alloc(ninst);
        b->energies.alloc((size_t)ninst * nroot);
        const size_t fixed = sizeof(BatchShared) + 8 * ((size_t)b->npp_max * b->npp_max + 2 * (size_t)b->npl_max * b->npl_max);
        const size_t statics = sizeof(double) * kBMaxSub * kBMaxSub + sizeof(int) * 2 * kBMaxG + 1024;
        FCIB_CHECK(fixed + statics + 8 * 2048 <= (size_t)b->smem_optin, FCIB_ERR_UNSUPPORTED,
                   "fcib_batch_create: integral blocks exceed shared memory");
        // sigma scratch: the largest instance's pair block, sigma row and connections
        size_t want = 0;
        for (const BatchInst& P : hi) want = std::max(want, bsigma_scratch(P.s1a, P.npp, P.nbs));
        FCIB_CHECK(fixed + statics + want <= (size_t)b->smem_optin, FCIB_ERR_UNSUPPORTED,
                   "fcib_batch_create: sigma scratch exceeds shared memory");
        b->xcap = (int)((want + 7) / 8);
        b->smem = fixed + 8 * (size_t)b->xcap;
        FCIB_CUDA(cudaFuncSetAttribute(k_batch_dl<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem));
        FCIB_CUDA(cudaFuncSetAttribute(k_batch_dl<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem));
        FCIB_CUDA(cudaFuncSetAttribute(k_batch_dl<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem));
        // default shape: 512 threads, 32-pair tiles, instances shared by clusters of two CTAs when two
        // such CTAs can be co-scheduled (the fastest shape measured on the 256-instance batch)
        {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(b->num_sms / 2 * 2);
            cfg.blockDim = dim3(512);
            cfg.dynamicSmemBytes = b->smem;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = 2;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            int nclusters = 0;
            if (cudaOccupancyMaxActiveClusters(&nclusters, k_batch_dl<32>, &cfg) == cudaSuccess && nclusters >= 1)
                b->cluster = 2;
            cudaGetLastError();
        }
        FCIB_CUDA(cudaStreamSynchronize(b->stream));
    });
    if (rc != FCIB_OK) {
        delete b;
        return rc;
    }
    *out = b;
    return FCIB_OK;
}

int fcib_batch_destroy(fcib_batch* b) {
    if (!b) return FCIB_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    delete b;
    return FCIB_OK;
}

int fcib_batch_solve(fcib_batch* b, double* energies, int* iterations, int* converged, double* device_ms) {
    if (!b) { fcib::set_error("null batch"); return FCIB_ERR_ARG; }
    return fcib::guarded(nullptr, [&] {
        FCIB_CUDA(cudaSetDevice(b->device));
        const double ms = fcib::batch_run(b);
        if (device_ms) *device_ms = ms;
        if (energies)
            FCIB_CUDA(cudaMemcpy(energies, b->energies.p, sizeof(double) * b->ninst * b->nroot, cudaMemcpyDeviceToHost));
        if (iterations) FCIB_CUDA(cudaMemcpy(iterations, b->iters.p, sizeof(int) * b->ninst, cudaMemcpyDeviceToHost));
        if (converged) FCIB_CUDA(cudaMemcpy(converged, b->conv.p, sizeof(int) * b->ninst, cudaMemcpyDeviceToHost));
    });
}

// Clock cycles of each phase summed over all CTAs since the last call (then zeroed); only builds
// compiled with -DFCIB_BATCH_PHASES count them.
int fcib_batch_phase_cycles(unsigned long long* cycles) {
    if (!cycles) { fcib::set_error("null argument"); return FCIB_ERR_ARG; }
#ifdef FCIB_BATCH_PHASES
    return fcib::guarded(nullptr, [&] {
        FCIB_CUDA(cudaMemcpyFromSymbol(cycles, fcib::g_bphase, 8 * sizeof(unsigned long long)));
        const unsigned long long z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        FCIB_CUDA(cudaMemcpyToSymbol(fcib::g_bphase, z, sizeof(z)));
    });
#else
    fcib::set_error("fcib_batch_phase_cycles: this build has no phase clocks (build with -DFCIB_BATCH_PHASES)");
    return FCIB_ERR_UNSUPPORTED;
#endif
}

// Launch shape for later solves: threads per CTA (256 or 512), opposite-spin sigma tile (8, 16 or
// 32 pairs per work item) and CTAs per instance (a thread-block cluster of 1, 2 or 4).
int fcib_batch_set_shape(fcib_batch* b, int threads, int pair_tile, int cluster) {
    if (!b) { fcib::set_error("null batch"); return FCIB_ERR_ARG; }
    return fcib::guarded(nullptr, [&] {
        FCIB_CHECK(threads == 256 || threads == 512, FCIB_ERR_ARG, "fcib_batch_set_shape: 256 or 512 threads");
        FCIB_CHECK(pair_tile == 8 || pair_tile == 16 || pair_tile == 32, FCIB_ERR_ARG,
                   "fcib_batch_set_shape: pair tile 8, 16 or 32");
        FCIB_CHECK(cluster == 1 || cluster == 2 || cluster == 4, FCIB_ERR_ARG, "fcib_batch_set_shape: cluster 1, 2 or 4");
        FCIB_CUDA(cudaSetDevice(b->device));
        b->threads = threads;
        b->ctas_per_sm = 1;
        b->pair_tile = pair_tile;
        b->cluster = cluster;
        if (b->graph) {
            cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
        }
    });
}

// Autotuner: times the whole batch for each launch shape (threads per CTA x CTAs per instance, the
// cluster size) and opposite-spin sigma tile, keeps the fastest and re-captures it into the solve
// graph.  times_ms[12] (may be NULL) receives each candidate's time (0 when a shape does not fit),
// tile-major: tiles 8, 16, 32 x shapes 512x1, 256 in clusters of 2, 512 in clusters of 2 and of 4.
int fcib_batch_tune(fcib_batch* b, int* threads, int* ctas_per_sm, int* pair_tile, int* cluster, double* times_ms) {
    if (!b) { fcib::set_error("null batch"); return FCIB_ERR_ARG; }
    return fcib::guarded(nullptr, [&] {
        FCIB_CUDA(cudaSetDevice(b->device));
        const int cand[4][2] = {{512, 1}, {256, 2}, {512, 2}, {512, 4}};  // threads, cluster size
        const int tiles[3] = {8, 16, 32};
        double best = 1e300;
        int bt = b->threads, bp = b->pair_tile, bcl = b->cluster;
        for (int ti = 0; ti < 3; ti++) {
            auto kern = tiles[ti] == 8 ? fcib::k_batch_dl<8> : tiles[ti] == 32 ? fcib::k_batch_dl<32> : fcib::k_batch_dl<16>;
            for (int i = 0; i < 4; i++) {
                if (times_ms) times_ms[ti * 4 + i] = 0.0;
                int per_sm = 0;
                FCIB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, cand[i][0], b->smem));
                if (per_sm < 1) continue;
                if (cand[i][1] > 1) {
                    cudaLaunchConfig_t cfg = {};
                    cfg.gridDim = dim3(b->num_sms / cand[i][1] * cand[i][1]);
                    cfg.blockDim = dim3(cand[i][0]);
                    cfg.dynamicSmemBytes = b->smem;
                    cudaLaunchAttribute attr[1];
                    attr[0].id = cudaLaunchAttributeClusterDimension;
                    attr[0].val.clusterDim.x = cand[i][1];
                    attr[0].val.clusterDim.y = 1;
                    attr[0].val.clusterDim.z = 1;
                    cfg.attrs = attr;
                    cfg.numAttrs = 1;
                    int nclusters = 0;
                    if (cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg) != cudaSuccess || nclusters < 1) {
                        cudaGetLastError();
                        continue;
                    }
                }
                b->threads = cand[i][0];
                b->ctas_per_sm = 1;
                b->cluster = cand[i][1];
                b->pair_tile = tiles[ti];
                if (b->graph) {
                    cudaGraphExecDestroy(b->graph);
                    b->graph = nullptr;
                }
                fcib::batch_run(b);  // capture + warm
                const double ms = fcib::batch_run(b);
                if (times_ms) times_ms[ti * 4 + i] = ms;
                if (ms < best) {
                    best = ms;
                    bt = cand[i][0];
                    bcl = cand[i][1];
                    bp = tiles[ti];
                }
            }
        }
        b->threads = bt;
        b->ctas_per_sm = 1;
        b->cluster = bcl;
        b->pair_tile = bp;
        if (b->graph) {
            cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
        }
        if (threads) *threads = bt;
        if (ctas_per_sm) *ctas_per_sm = 1;
        if (pair_tile) *pair_tile = bp;
        if (cluster) *cluster = bcl;
    });
}

}  // extern "C"
