// Mixed-precision sigma: the same-spin two-body term on the 5th-generation tensor cores.
//
// The (N-2)-electron group formulation of the CUDA-core kernel k_group: a group g holds the G
// strings I_i = g + {p_i, q_i} (pair label lab_i, sign s_i), and
//     sigma[I_i][col] += sum_j s_i s_j M[lab_i][lab_j] C[I_j][col]      for every column col.
// Per group this is one small dense product, mapped onto tcgen05 as
//     D[col][i] = sum_j X[col][j] W[i][j],   X[col][j] = C[I_j][col],   W[i][j] = s_i s_j M[lab_i][lab_j]
// with 128 columns per tile in the MMA's M dimension (one TMEM lane per column) and N = K = G
// padded to a multiple of 16:
// * a CTA takes a whole group (dynamic counter) and sweeps its 128-column tiles; W is split into
//   TF32 hi/lo planes in shared memory once per group (K-major, no swizzle);
// * the gathered tile X (the FP32 copy of C, coalesced across lanes) is split into TF32 hi/lo in
//   registers and written to tensor memory with tcgen05.st; the three 3xTF32 products
//   Xlo Whi + Xhi Wlo + Xhi Whi accumulate in FP32 in TMEM;
// * two accumulators are double buffered, so the MMAs of tile t overlap the epilogue of tile t-1,
//   and the gather of tile t+1 is in flight during both;
// * the epilogue reads the accumulator with tcgen05.ld, rounds each element to the sigma's
//   fixed-point grid 2^-el and adds it to an int64 sigma buffer with a 64-bit integer reduction
//   (a warp covers 32 consecutive columns of one row); each sigma element receives one addition
//   per group that holds its row, C(k,2) in all, and the integer sum does not depend on their order.
// Groups of more than 64 strings (few electrons in many orbitals) keep the CUDA-core kernel.
//
// Every mbarrier wait is bounded; on timeout the kernel records an error code, waits (bounded)
// for its outstanding MMAs, frees tensor memory and exits.
#include "fcib_internal.h"

namespace fcib {

constexpr int kGtM = 128;             // columns per tile (MMA M, TMEM lanes)
constexpr int kGtThreads = 512;       // 16 warps: lane quarter q = warp % 4, column group cg = warp / 4
constexpr uint32_t kGtTmemCols = 256; // two CTAs per SM
constexpr uint32_t kGtColAcc = 64, kGtColAhi = 128, kGtColAlo = 192;  // accumulators at 0 and 64
constexpr int kGtMaxG = 64;
constexpr int kErrTimeoutGroupMma = 2;
constexpr uint32_t kGtNoRow = 0xFFFFFFFFu;

// K (source strings) and N (target strings) are both G padded to P = 16 Q; thread (q, lane, cg)
// owns column c0 + 32 q + lane and the Q quads of strings 4 (cg + 4 i) .. +3, i < Q, for the
// gather and the epilogue alike
struct GtLayout {
    int P;
    uint32_t b_bytes, off_bhi, off_blo, off_rows, off_labs, off_bar, total;
};

__host__ __device__ inline GtLayout gt_layout(int G) {
    GtLayout L;
    L.P = (G + 15) / 16 * 16;
    L.b_bytes = (uint32_t)L.P * L.P * 4;  // a multiple of 1 KB
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

__device__ __forceinline__ void tmem_st4(uint32_t taddr, const float (&v)[4]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1,%2,%3,%4};" ::"r"(taddr), "r"(__float_as_uint(v[0])),
                 "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3]))
                 : "memory");
}
__device__ __forceinline__ void tmem_ld4_async(uint32_t taddr, uint32_t (&r)[4]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld4(uint32_t (&r)[4]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3])::"memory");
}
__device__ __forceinline__ void reg_after4(uint32_t (&r)[4]) {
    asm volatile("" : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]));
}

template <int Q>
__global__ void __launch_bounds__(kGtThreads, 2)
    k_group_tc(const float* __restrict__ C, unsigned long long* __restrict__ S, int ncols, int ld,
               const uint32_t* __restrict__ rows, const uint16_t* __restrict__ labs, int G,
               const double* __restrict__ M, int ldm, int ngroups, int* __restrict__ counter,
               int* __restrict__ err, const int* __restrict__ grid_el) {
    const float scale = ldexpf(1.0f, *grid_el);  // fixed-point grid 2^-el of this sigma
    extern __shared__ __align__(128) unsigned char gt_smem[];
    unsigned char* smem = gt_smem;
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
    constexpr int P = 16 * Q;

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

    // instruction descriptor: D f32, A/B tf32, both K-major, N = P, M = 128
    const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(P >> 3) << 17) | ((uint32_t)(kGtM >> 4) << 24);
    const uint32_t lbo_b = (uint32_t)(P / 8) * 128;
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
        for (int idx = tid; idx < P * P; idx += blockDim.x) {
            const int i = idx / P, j = idx - i * P;
            float hi = 0.f, lo = 0.f;
            if (i < G && j < G) {
                double v = M[(size_t)ls[i] * ldm + ls[j]];
                if ((rs[i] ^ rs[j]) & kSignBit) v = -v;
                hi = __uint_as_float(to_tf32((float)v));
                lo = __uint_as_float(to_tf32((float)(v - (double)hi)));
            }
            const uint32_t off = kmaj_off(i, j, P);
            *reinterpret_cast<float*>(Bhi + off) = hi;
            *reinterpret_cast<float*>(Blo + off) = lo;
        }
        fence_proxy_async();  // W (generic-proxy stores) becomes visible to the tensor core's reads
        // row offsets (string index * ld) of this thread's quads, shared by gather and epilogue
        uint32_t off[Q][4];
#pragma unroll
        for (int i = 0; i < Q; i++)
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int j = 4 * (cg + 4 * i) + u;
                off[i][u] = (j < G && rs[j] != kNullRow) ? (rs[j] & kConnIdxMask) * (uint32_t)ld : kGtNoRow;
            }
        // X-tile gather, one tile ahead in registers (coalesced across lanes)
        float xv[Q][4];
        auto prefetch = [&](int tt) {
            const int col = tt * kGtM + 32 * q + lane;
            const bool in = col < ncols;
#pragma unroll
            for (int i = 0; i < Q; i++)
#pragma unroll
                for (int u = 0; u < 4; u++)
                    xv[i][u] = (in && off[i][u] != kGtNoRow) ? __ldg(C + (size_t)(off[i][u] + (uint32_t)col)) : 0.f;
        };
        prefetch(0);
        for (int t = 0; t <= ntiles; t++) {
            const int cur = t & 1, prv = cur ^ 1;
            // (a) the TMEM X buffer and accumulator prv are ready once the previous tile's MMAs
            // completed; every thread waits on the barrier itself (no block barrier here)
            if (t >= 1 && !mbar_wait_bounded(&bars[prv], (mma_count[prv] - 1) & 1)) {
                atomicCAS(err, 0, kErrTimeoutGroupMma);
                s_abort = 1;
            }
            tc_fence_after();
            // (b) registers -> X hi/lo in tensor memory
            if (t < ntiles) {
#pragma unroll
                for (int i = 0; i < Q; i++) {
                    float h[4], l[4];
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        h[u] = __uint_as_float(to_tf32(xv[i][u]));
                        l[u] = __uint_as_float(to_tf32(xv[i][u] - h[u]));
                    }
                    const uint32_t c4 = 4 * (uint32_t)(cg + 4 * i);
                    tmem_st4(tmem_base + tlane + kGtColAhi + c4, h);
                    tmem_st4(tmem_base + tlane + kGtColAlo + c4, l);
                }
                asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            }
            tc_fence_before();
            __syncthreads();
            if (s_abort) break;
            tc_fence_after();
            // (c) one thread issues the tile's MMAs into accumulator `cur`
            if (t < ntiles && tid == 0) {
                const uint32_t dt = tmem_base + (uint32_t)cur * kGtColAcc;
                uint32_t acc = 0;
#pragma unroll
                for (int ks = 0; ks < P / 8; ks++) {
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
                uint32_t rv[Q][4];
#pragma unroll
                for (int i = 0; i < Q; i++) tmem_ld4_async(tbase + 4 * (uint32_t)(cg + 4 * i), rv[i]);
                tmem_wait_ld4(rv[0]);
#pragma unroll
                for (int i = 1; i < Q; i++) reg_after4(rv[i]);
                const int col = (t - 1) * kGtM + 32 * q + lane;
                if (col < ncols) {
#pragma unroll
                    for (int i = 0; i < Q; i++)
#pragma unroll
                        for (int u = 0; u < 4; u++)
                            if (off[i][u] != kGtNoRow)
                                atomicAdd(S + (size_t)(off[i][u] + (uint32_t)col),
                                          fixed64(__uint_as_float(rv[i][u]), scale));
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
// groups are too large for the kernel's tensor-memory layout or the vectors too long for its
// 32-bit element offsets; the caller then uses k_group<float>.  The group counter and the timeout
// flag live in counter slots 4 and 5; the flag is cleared by the caller once per sigma and read
// back by tc_check_error.
bool launch_group_tc(Context& c, const float* C, unsigned long long* S, int ncols, int ld, int ngroups, int G,
                     const uint32_t* rows, const uint16_t* labs, const double* M, int ldm) {
    if (G < 1 || G > kGtMaxG || (uint64_t)c.nas * (uint64_t)c.nbs >= (1ull << 32) - kGtM) return false;
    if (ngroups == 0) return true;
    const GtLayout L = gt_layout(G);
    // at least 80 KB so that no more than two CTAs (2 x 256 TMEM columns) share an SM
    const size_t smem = std::max<size_t>(L.total, 80 * 1024);
    if (smem + 1024 > (size_t)c.smem_optin) return false;
    auto kern = L.P == 16 ? k_group_tc<1> : L.P == 32 ? k_group_tc<2> : L.P == 48 ? k_group_tc<3> : k_group_tc<4>;
    FCIB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    ensure_counter(c);
    FCIB_CUDA(cudaMemsetAsync(c.counter.p + 4, 0, sizeof(int), c.stream));
    const int grid = std::min(ngroups, 2 * c.num_sms);
    kern<<<grid, kGtThreads, smem, c.stream>>>(C, S, ncols, ld, rows, labs, G, M, ldm, ngroups, c.counter.p + 4,
                                               c.counter.p + 5, c.counter.p + kSlotSameGrid);
    FCIB_KCHECK();
    return true;
}

}  // namespace fcib
