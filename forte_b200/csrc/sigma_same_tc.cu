// Mixed-precision sigma: the same-spin two-body term on the 5th-generation tensor cores.
//
// The (N-2)-electron group formulation of the CUDA-core kernel k_group: a group g holds the G
// strings I_i = g + {p_i, q_i} (pair label lab_i, sign s_i), and
//     sigma[I_i][col] += sum_j s_i s_j M[lab_i][lab_j] C[I_j][col]      for every column col.
// Per group this is one small dense product, mapped onto tcgen05 as
//     D[col][i] = sum_j X[col][j] W[i][j],   X[col][j] = C[I_j][col],   W[i][j] = s_i s_j M[lab_i][lab_j]
// with 128 columns per tile in the MMA's M dimension (one TMEM lane per column), N = G padded to 16
// and K = G padded to 8:
// * a CTA takes a whole group (dynamic counter) and sweeps its 128-column tiles; W is split into
//   TF32 hi/lo planes in shared memory once per group (K-major, no swizzle);
// * the gathered tile X (the FP32 copy of C, coalesced across lanes) is split into TF32 hi/lo in
//   registers and written to tensor memory with tcgen05.st; the three 3xTF32 products
//   Xlo Whi + Xhi Wlo + Xhi Whi accumulate in FP32 in TMEM;
// * two accumulators are double buffered, so the MMAs of tile t overlap the epilogue of tile t-1,
//   and the gather of tile t+1 is in flight during both;
// * the epilogue reads the accumulator with tcgen05.ld and adds each element to the FP32 sigma
//   buffer with a global reduction (a warp covers 32 consecutive columns of one row); each sigma
//   element receives one addition per group that holds its row, C(k,2) in all.
// Groups of more than 64 strings (few electrons in many orbitals) keep the CUDA-core kernel.
//
// Every mbarrier wait is bounded; on timeout the kernel records an error code, waits (bounded)
// for its outstanding MMAs, frees tensor memory and exits.
#include "fcib_internal.h"

namespace fcib {

constexpr int kGtM = 128;             // columns per tile (MMA M, TMEM lanes)
constexpr int kGtThreads = 256;       // 8 warps: lane quarter q = warp % 4, column group warp / 4
constexpr uint32_t kGtTmemCols = 256; // two CTAs per SM
constexpr uint32_t kGtColAcc = 64, kGtColAhi = 128, kGtColAlo = 192;  // accumulators at 0 and 64
constexpr int kGtMaxG = 64;
constexpr int kGtChunks = 4;          // 8-column chunks per thread: at most 8 chunks over 2 column groups
constexpr int kErrTimeoutGroupMma = 2;

struct GtLayout {
    int kp, np;  // K (source strings) padded to 8, N (target strings) padded to 16
    uint32_t b_bytes, off_bhi, off_blo, off_rows, off_labs, off_bar, total;
};

__host__ __device__ inline GtLayout gt_layout(int G) {
    GtLayout L;
    L.kp = (G + 7) / 8 * 8;
    L.np = (G + 15) / 16 * 16;
    L.b_bytes = (uint32_t)L.np * L.kp * 4;  // a multiple of 512 bytes
    uint32_t o = 0;
    L.off_bhi = o; o += L.b_bytes;
    L.off_blo = o; o += L.b_bytes;
    L.off_rows = o; o += kGtMaxG * 4;
    L.off_labs = o; o += kGtMaxG * 2;
    o = (o + 127) / 128 * 128;
    L.off_bar = o; o += 128;
    L.total = o;
    return L;
}

__global__ void __launch_bounds__(kGtThreads, 2)
    k_group_tc(const float* __restrict__ C, float* __restrict__ S, int ncols, const uint32_t* __restrict__ rows,
               const uint16_t* __restrict__ labs, int G, const double* __restrict__ M, int ldm, int ngroups,
               int* __restrict__ counter, int* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char smem[];
    const GtLayout L = gt_layout(G);
    unsigned char* Bhi = smem + L.off_bhi;
    unsigned char* Blo = smem + L.off_blo;
    uint32_t* rs = reinterpret_cast<uint32_t*>(smem + L.off_rows);
    uint16_t* ls = reinterpret_cast<uint16_t*>(smem + L.off_labs);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L.off_bar);  // [0],[1]: MMA done per accumulator
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + L.off_bar + 64);
    __shared__ int s_group;
    __shared__ int s_abort;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int q = warp & 3, cg = warp >> 2;
    const int kp = L.kp, np = L.np, nk8 = kp / 8, nn8 = np / 8;

    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kGtTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const uint32_t tlane = (uint32_t)(32 * q) << 16;

    // instruction descriptor: D f32, A/B tf32, both K-major, N = np, M = 128
    const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(np >> 3) << 17) | ((uint32_t)(kGtM >> 4) << 24);
    const uint32_t lbo_b = (uint32_t)(np / 8) * 128;
    const uint32_t sb_hi = smem_u32(Bhi), sb_lo = smem_u32(Blo);

    uint32_t mma_count[2] = {0u, 0u};  // commits issued per accumulator (parity tracking)
    const int ntiles = (ncols + kGtM - 1) / kGtM;

    while (true) {
        if (tid == 0) s_group = atomicAdd(counter, 1);
        __syncthreads();
        const int g = s_group;
        if (g >= ngroups || s_abort) break;
        for (int i = tid; i < kGtMaxG; i += blockDim.x) {
            rs[i] = i < G ? rows[(size_t)g * G + i] : 0u;
            ls[i] = i < G ? labs[(size_t)g * G + i] : (uint16_t)0;
        }
        __syncthreads();
        // W[i][j] = s_i s_j M[lab_i][lab_j], split into tf32 hi/lo (zero outside G x G)
        for (int idx = tid; idx < np * kp; idx += blockDim.x) {
            const int i = idx / kp, j = idx - i * kp;
            float hi = 0.f, lo = 0.f;
            if (i < G && j < G) {
                double v = M[(size_t)ls[i] * ldm + ls[j]];
                if ((rs[i] ^ rs[j]) & kSignBit) v = -v;
                hi = __uint_as_float(to_tf32((float)v));
                lo = __uint_as_float(to_tf32((float)(v - (double)hi)));
            }
            const uint32_t off = kmaj_off(i, j, np);
            *reinterpret_cast<float*>(Bhi + off) = hi;
            *reinterpret_cast<float*>(Blo + off) = lo;
        }
        fence_proxy_async();  // W (generic-proxy stores) becomes visible to the tensor core's reads
        // X-tile gather: the thread owning tile row m = 32q + lane (column c0 + m) loads the source
        // strings j of its 8-column chunks c8 = cg + 2 jj; one tile ahead in registers
        float xv[kGtChunks][8];
        auto prefetch = [&](int tt) {
            const int col = tt * kGtM + 32 * q + lane;
#pragma unroll
            for (int jj = 0; jj < kGtChunks; jj++) {
                const int c8 = cg + 2 * jj;
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    const int j = 8 * c8 + u;
                    float x = 0.f;
                    if (c8 < nk8 && j < G && col < ncols) x = __ldg(C + (size_t)(rs[j] & kConnIdxMask) * ncols + col);
                    xv[jj][u] = x;
                }
            }
        };
        prefetch(0);
        for (int t = 0; t <= ntiles; t++) {
            const int cur = t & 1, prv = cur ^ 1;
            // (a) the TMEM X buffer is free once the previous tile's MMAs completed (one waiter)
            if (t >= 1 && tid == 0) {
                if (!mbar_wait_bounded(&bars[prv], (mma_count[prv] - 1) & 1)) {
                    atomicCAS(err, 0, kErrTimeoutGroupMma);
                    s_abort = 1;
                }
            }
            __syncthreads();
            if (s_abort) break;
            tc_fence_after();
            // (b) registers -> X hi/lo in tensor memory
            if (t < ntiles) {
#pragma unroll
                for (int jj = 0; jj < kGtChunks; jj++) {
                    const int c8 = cg + 2 * jj;
                    if (c8 < nk8) {
                        float h[8], l[8];
#pragma unroll
                        for (int u = 0; u < 8; u++) {
                            h[u] = __uint_as_float(to_tf32(xv[jj][u]));
                            l[u] = __uint_as_float(to_tf32(xv[jj][u] - h[u]));
                        }
                        tmem_st8(tmem_base + tlane + kGtColAhi + 8 * c8, h);
                        tmem_st8(tmem_base + tlane + kGtColAlo + 8 * c8, l);
                    }
                }
                asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            }
            tc_fence_before();
            __syncthreads();
            tc_fence_after();
            // (c) one thread issues the tile's MMAs into accumulator `cur`
            if (t < ntiles && tid == 0) {
                const uint32_t dt = tmem_base + (uint32_t)cur * kGtColAcc;
                uint32_t acc = 0;
                for (int ks = 0; ks < nk8; ks++) {
                    const uint32_t ah = tmem_base + kGtColAhi + 8 * ks;
                    const uint32_t al = tmem_base + kGtColAlo + 8 * ks;
                    const uint64_t bh = make_desc(sb_hi + ks * 2 * lbo_b, lbo_b, 128);
                    const uint64_t bl = make_desc(sb_lo + ks * 2 * lbo_b, lbo_b, 128);
                    mma_tf32_ta(dt, al, bh, idesc, acc);
                    acc = 1;
                    mma_tf32_ta(dt, ah, bl, idesc, acc);
                    mma_tf32_ta(dt, ah, bh, idesc, acc);
                }
                mma_commit(&bars[cur]);
            }
            if (t < ntiles) mma_count[cur]++;
            // (b') next tile's loads overlap the MMAs above and the epilogue below
            if (t + 1 < ntiles) prefetch(t + 1);
            // (d) epilogue of tile t-1: reductions into the FP32 sigma buffer
            if (t >= 1) {
                const uint32_t tbase = tmem_base + (uint32_t)prv * kGtColAcc + tlane;
                uint32_t rv[kGtChunks][8];
#pragma unroll
                for (int i = 0; i < kGtChunks; i++) {
                    const int c8 = cg + 2 * i;
                    if (c8 < nn8) tmem_ld8_async(tbase + (uint32_t)(c8 * 8), rv[i]);
                }
                tmem_wait_ld8(rv[0]);
#pragma unroll
                for (int i = 1; i < kGtChunks; i++) reg_after(rv[i]);
                const int col = (t - 1) * kGtM + 32 * q + lane;
                if (col < ncols) {
#pragma unroll
                    for (int i = 0; i < kGtChunks; i++) {
                        const int c8 = cg + 2 * i;
                        if (c8 < nn8) {
#pragma unroll
                            for (int u = 0; u < 8; u++) {
                                const int r = 8 * c8 + u;
                                if (r < G)
                                    atomicAdd(S + (size_t)(rs[r] & kConnIdxMask) * ncols + col, __uint_as_float(rv[i][u]));
                            }
                        }
                    }
                }
                tc_fence_before();
            }
        }
        if (s_abort) break;
        __syncthreads();  // the next group overwrites the row list and W
    }
    // drain: wait (bounded) for any MMA still in flight before releasing tensor memory
    __syncthreads();
    if (tid == 0) {
        for (int b = 0; b < 2; b++)
            if (mma_count[b] > 0) mbar_wait_bounded(&bars[b], (mma_count[b] - 1) & 1);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(kGtTmemCols)
                     : "memory");
}

// Same-spin groups of FP32 sigma on the tensor cores.  Returns false (nothing launched) when the
// groups are too large for the kernel's tensor-memory layout; the caller then uses k_group<float>.
// The group counter and the timeout flag live in counter slots 4 and 5; the flag is cleared by
// the caller once per sigma and read back by tc_check_error.
bool launch_group_tc(Context& c, const float* C, float* S, int ncols, int ngroups, int G, const uint32_t* rows,
                     const uint16_t* labs, const double* M, int ldm) {
    if (G < 1 || G > kGtMaxG) return false;
    if (ngroups == 0) return true;
    const GtLayout L = gt_layout(G);
    // at least 80 KB so that no more than two CTAs (2 x 256 TMEM columns) share an SM
    const size_t smem = std::max<size_t>(L.total, 80 * 1024);
    if (smem + 1024 > (size_t)c.smem_optin) return false;
    FCIB_CUDA(cudaFuncSetAttribute(k_group_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    ensure_counter(c);
    FCIB_CUDA(cudaMemsetAsync(c.counter.p + 4, 0, sizeof(int), c.stream));
    const int grid = std::min(ngroups, 2 * c.num_sms);
    k_group_tc<<<grid, kGtThreads, smem, c.stream>>>(C, S, ncols, rows, labs, G, M, ldm, ngroups, c.counter.p + 4,
                                                     c.counter.p + 5);
    FCIB_KCHECK();
    return true;
}

}  // namespace fcib
