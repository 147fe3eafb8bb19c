// Mixed-precision sigma: the opposite-spin contraction on the 5th-generation tensor cores.
//
// Same regrouping as the FP64 kernel (one CTA owns a target alpha row Ia; the C rows
// connected to Ia by a single alpha replacement are gathered into a tile A[Jb, k] and
// multiplied by the pair-integral block B[k, R] = sgn_k V[P_k, R]; the product is scattered
// over beta single replacements into a sigma row held on chip), mapped onto Blackwell:
//
// * the input vector is split once per sigma into tf32 hi/lo planes (3xTF32: A*B ~ Ahi*Bhi +
//   Ahi*Blo + Alo*Bhi with FP32 accumulation);
// * the gathered tile A (128 beta strings x K connections) is written straight into tensor
//   memory with tcgen05.st and multiplied from there (tcgen05.mma kind::tf32 with the A operand
//   in TMEM); B (Npad x K) lives in shared memory in the K-major no-swizzle core-matrix layout
//   (element (row, k) at (k/4)*LBO + (row/8)*128 + (row%8)*16 + (k%4)*4 bytes);
// * two 144-column accumulators in TMEM are double buffered, so the MMAs of tile t overlap the
//   epilogue of tile t-1;
// * the epilogue accumulates the sigma row exactly in two-word fixed point with native 32-bit
//   shared-memory integer atomics: each contribution y is scaled, exactly and in FP32, to the
//   grid 2^-el chosen per sigma from max|C| * max|V| (so |y| 2^el < 2^44) and rounded to the
//   integer X = hi 2^22 + lo with |hi| < 2^22 and |lo| <= 2^21 (FP32 adds of 1.5 * 2^23 do the
//   rounding; no FP64 or conversion instructions); every sigma element receives at most
//   s1 (<= 72) contributions, so neither 32-bit word can overflow.  The row is converted back to
//   FP64 and added to E0*C when it is written.
//
// Every mbarrier wait is bounded; on timeout the kernel records an error code, waits (bounded)
// for its outstanding MMAs, frees tensor memory and exits.
#include "fcib_internal.h"

namespace fcib {

constexpr int kTcM = 128;          // beta rows per tile (MMA M)
constexpr int kTcWarps = 16;       // warps of the opposite-spin kernel: all gather, one thread issues MMAs, all scatter
constexpr uint32_t kTmemCols = 512;
constexpr long long kWaitLimit = 1ll << 24;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (long long i = 0; i < kWaitLimit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// K-major, no-swizzle shared-memory matrix descriptor (sm_100 version 1)
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for sm_100
    // base offset 0, lbo mode 0, layout type 0 (no swizzle)
    return d;
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 8 columns of the accumulator without waiting; tmem_wait_ld8 must follow before any use
__device__ __forceinline__ void tmem_ld8_async(uint32_t taddr, uint32_t (&r)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}
// waits for every outstanding tcgen05.ld of the thread; the "+r" operands keep the compiler from
// moving uses of those registers above the wait
__device__ __forceinline__ void tmem_wait_ld8(uint32_t (&r)[8]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7])
                 :: "memory");
}
// orders later uses of r after a preceding volatile wait (emits no instruction)
__device__ __forceinline__ void reg_after(uint32_t (&r)[8]) {
    asm volatile(""
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]));
}

// ------------------------------------------------------------------------------------------
// k_ab_tc layout.  Dynamic shared memory of the one CTA per SM:
//   [0, 4 nbs)                   acc_hi: signed high words of the sigma row's fixed-point sums
//   [kAccLoOff, kAccLoOff+4 nbs) acc_lo: low words, at a fixed distance from acc_hi so that one
//                                address register serves both reductions (immediate offset)
//   B hi, B lo                   Npad x Kpad TF32 planes, K-major core matrices, no swizzle
//   cs[Kpad], koff[Kpad]         the row's connections and the byte offsets of their plane rows
//   barriers, TMEM address
// ------------------------------------------------------------------------------------------
constexpr uint32_t kAccLoOff = 65536;
constexpr int kMaxBetaStrings = 16383;  // Ib * 4 and a sign bit fit the 16-bit target entries

struct TcLayout {
    int kpad, npad;          // K (connections) and N (pairs) padded to 8 / 16
    uint32_t b_bytes;        // one B plane
    uint32_t off_bhi, off_blo, off_cs, off_koff, off_bar, total;
};

__host__ __device__ inline TcLayout tc_layout(int s1a, int npair, int nbs, bool three) {
    TcLayout L;
    L.kpad = (s1a + 7) / 8 * 8;
    L.npad = (npair + 15) / 16 * 16;
    L.b_bytes = (uint32_t)L.npad * L.kpad * 4;
    uint32_t o = kAccLoOff + ((uint32_t)nbs * 4 + 127) / 128 * 128;
    L.off_bhi = o; o += L.b_bytes;
    L.off_blo = o; o += three ? L.b_bytes : 0;
    L.off_cs = o; o += ((uint32_t)L.kpad * 4 + 127) / 128 * 128;
    L.off_koff = o; o += ((uint32_t)L.kpad * 4 + 127) / 128 * 128;
    L.off_bar = o; o += 128;
    L.total = o;
    return L;
}

// B plane (N x K, K-major interleaved): element (row, k) at (k/4)*(rows/8)*128 + (row/8)*128 + (row%8)*16 + (k%4)*4
__device__ __forceinline__ uint32_t kmaj_off(int row, int k, int rows) {
    return (uint32_t)((k >> 2) * (rows / 8) * 128 + (row >> 3) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

// no "memory" clobber: the accumulator is read only after a __syncthreads, which orders it
__device__ __forceinline__ void red_add_u32(uint32_t saddr, uint32_t v) {
    asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(saddr), "r"(v));
}
// both words of one fixed-point contribution (the low word kAccLoOff bytes above the high word), for
// target entries g that hold a target (g != 0xFFFF)
__device__ __forceinline__ void red_pair(uint32_t saddr, uint32_t hi, uint32_t lo, uint32_t g) {
    if (g != 0xFFFFu) {
        asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(saddr), "r"(hi));
        asm volatile("red.shared.add.u32 [%0+65536], %1;" ::"r"(saddr), "r"(lo));
    }
}

// Two fixed-point splits at once with the paired FP32 instructions of sm_100 (f32x2): for each y
// (|y| < 2^44, the grid already folded in), hi = round(y 2^-22) as the bits of 1.5 * 2^23 + hi and
// lo = y - hi 2^22 (exact) as the bits of 1.5 * 2^23 + round(lo)
__device__ __forceinline__ void split_fixed2(float y0, float y1, uint32_t& h0, uint32_t& h1, uint32_t& l0,
                                             uint32_t& l1) {
    asm("{\n .reg .b64 y, t, h, l;\n mov.b64 y, {%4, %5};\n"
        " fma.rn.f32x2 t, y, %6, %7;\n sub.rn.f32x2 h, t, %7;\n"
        " fma.rn.f32x2 l, h, %8, y;\n add.rn.f32x2 l, l, %7;\n"
        " mov.b64 {%0, %1}, t;\n mov.b64 {%2, %3}, l;\n}"
        : "=r"(h0), "=r"(h1), "=r"(l0), "=r"(l1)
        : "f"(y0), "f"(y1), "l"(0x3480000034800000ull),  // (2^-22, 2^-22)
          "l"(0x4B4000004B400000ull),                     // (1.5 * 2^23, 1.5 * 2^23)
          "l"(0xCA800000CA800000ull));                    // (-2^22, -2^22)
}

__device__ __forceinline__ void mma_tf32_ta(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n}\n" ::"r"(d_tmem),
        "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void tmem_st8(uint32_t taddr, const float (&v)[8]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr),
                 "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
                 "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
                 "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7]))
                 : "memory");
}

// Error codes written to *err (first one wins)
constexpr int kErrTimeoutMma = 1;

// TMEM columns: accumulators at 0 and 256 (npad <= 144), A hi at 160, A lo at 416 (kpad <= 72)
constexpr uint32_t kColAccStride = 256, kColAhi = 160, kColAlo = 416;
constexpr int kTcMmaThread = 5 * 32;  // issues the MMAs (warp 5: two gather chunks, four epilogue chunks)
constexpr int kFixLoBits = 22;
constexpr float kMagic = 12582912.0f;       // 1.5 * 2^23: x + kMagic rounds |x| < 2^22 to an integer
constexpr int kMagicBits = 0x4B400000;      // bit pattern of kMagic

// One CTA per SM, persistent over target alpha rows Ia (dynamic counter).  Per row: the s1a
// connections (J_k, P_k, sign_k) and B[R][k] = sign_k V[P_k][R] 2^el (TF32 hi/lo, the fixed-point
// grid folded in exactly) are staged in shared memory; per tile of 128 beta strings Jb:
//   gather   A[Jb][k] = plane[J_k][Jb] (interleaved TF32 hi/lo pairs; one coalesced 8-byte load per
//            element, address = tile base + koff[k]) into registers, one tile ahead;
//   store    registers -> A in TMEM (tcgen05.st), after the previous tile's MMAs released it;
//   MMA      T = A B, 3xTF32, FP32 accumulator in TMEM (two accumulators, double buffered);
//   scatter  the previous tile's T[Jb][R] to sigma[F_R Jb] in exact 2-word fixed point.
// Plane rows are padded to whole tiles (zeros) and the target table to whole tiles (no target), so
// neither the gather nor the scatter checks bounds.  Per tile: one mbarrier wait and one block
// barrier.
// Source rows (plane, ns beta strings) and target rows (C, S: nt beta strings) have their own
// lengths, so one launch also serves a sub-problem of the irrep-blocked layout; ndiag = 0 drops the
// diagonal pairs and accumulate = 1 adds the row to S instead of writing E0 C + the product.  The
// source strings may be a sub-range of the target row's strings (GAS sub-problems): their own
// elements, which the diagonal pairs add to, start at target column diag_off.
// NW warps: NW / 4 column groups per TMEM lane quarter.  Gather chunks of column group cg: cg + NCG j
// (at 16 warps the third round goes to group 3 - cg, which holds one epilogue chunk fewer);
// off-diagonal epilogue chunks: (NCG - 1 - cg) + NCG i; the diagonal chunks go to group 0.
template <int NW>
__device__ __forceinline__ int tc_gather_chunk(int cg, int j) {
    constexpr int NCG = NW / 4;
    return (NCG == 4 && j == 2) ? 8 + (3 - cg) : cg + NCG * j;
}

template <bool THREE, int NW>
__global__ void __launch_bounds__(NW * 32, 1)
    k_ab_tc(const float2* __restrict__ Phl, int ldp, int ns, const double* __restrict__ C, double* __restrict__ S,
            int nt, int accumulate, const uint32_t* __restrict__ connA, int s1a, const uint16_t* __restrict__ tgtR,
            int npair, const int* __restrict__ perm, int noff8, int ndiag, int diag_off,
            const uint32_t* __restrict__ bstr, int kb,
            const double* __restrict__ V, int ldv, float vmax, const unsigned int* __restrict__ cmax_bits,
            int nas, int ncontrib, const uint8_t* __restrict__ mag, double e0, int* __restrict__ row_counter,
            int* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char tc_smem[];
    unsigned char* smem = tc_smem;
    const TcLayout L = tc_layout(s1a, npair, nt, THREE);
    unsigned char* Bhi = smem + L.off_bhi;
    unsigned char* Blo = smem + L.off_blo;
    int* acc_hi = reinterpret_cast<int*>(smem);
    unsigned int* acc_lo = reinterpret_cast<unsigned int*>(smem + kAccLoOff);
    uint32_t* cs = reinterpret_cast<uint32_t*>(smem + L.off_cs);
    uint32_t* koff = reinterpret_cast<uint32_t*>(smem + L.off_koff);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L.off_bar);  // [0],[1]: MMA done per accumulator
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + L.off_bar + 64);
    __shared__ int s_row;
    __shared__ int s_abort;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int kpad = L.kpad, npad = L.npad;
    const int q = warp & 3, cg = warp >> 2;  // TMEM lane quarter and column group of this warp
    constexpr int NCG = NW / 4;
    constexpr int GJ = (9 + NCG - 1) / NCG;        // gather chunks per warp (kpad <= 72)
    constexpr int EI = (15 + NCG - 1) / NCG;       // off-diagonal epilogue chunks per warp (n <= 16)
    constexpr int EB = EI < 3 ? EI : 3;            // chunks of the first epilogue batch
    const int ec0 = NCG - 1 - cg;                  // first epilogue chunk of this warp

    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const uint32_t tlane = (uint32_t)(32 * q) << 16;

    // fixed-point grid: every contribution, the sum of a string's kb diagonal-pair products included,
    // is at most kb * kpad * max|C| * max|V| < 2^44 * 2^-el
    const float cmax = __uint_as_float(*cmax_bits);
    const float ybound = fmaxf(1.01f * (float)max(kb, 1) * (float)kpad * cmax * vmax, 1e-30f);
    const int el = min(60, (int)floorf(44.0f - log2f(ybound)));
    const double inv_grid = ldexp(1.0, -el);
    const double grid = ldexp(1.0, el);
    // every element receives exactly ncontrib contributions (C1 layout: kb (n - kb) off-diagonal ones and
    // the diagonal sum of its own string; blocked sub-problems: mag[element]); that many kMagicBits are
    // removed once per element (mod 2^32)
    const unsigned magic_total = (unsigned)ncontrib * (unsigned)kMagicBits;

    // instruction descriptor: D f32, A/B tf32, both K-major, N = npad, M = 128
    const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(npad >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);
    const uint32_t lbo_b = (uint32_t)(npad / 8) * 128;
    const uint32_t sb_hi = smem_u32(Bhi), sb_lo = smem_u32(Blo);
    const uint32_t acc_s = smem_u32(acc_hi);

    uint32_t mma_count[2] = {0u, 0u};  // commits issued per accumulator (parity tracking)
    const int ntiles = (ns + kTcM - 1) / kTcM;
    const int nk8 = kpad / 8;
    const int nn8 = noff8 / 8;        // accumulator chunks of off-diagonal pairs
    const int ndc = (ndiag + 7) / 8;  // accumulator chunks of the diagonal pairs (r,r), after them
    const unsigned char* pbase = reinterpret_cast<const unsigned char*>(Phl);

    float gh[GJ][8], gl[GJ][8];
    // A-tile gather: the thread owning tile row m = 32q + lane loads A[m][k] = plane[J_k][jb0 + m] for
    // the 8-column chunks c8 = cg + 4j (coalesced across lanes)
    auto gather = [&](int tt) {
        const unsigned char* pj = pbase + (size_t)(tt * kTcM + 32 * q + lane) * sizeof(float2);
#pragma unroll
        for (int j = 0; j < GJ; j++) {
            const int c8 = tc_gather_chunk<NW>(cg, j);
            if (c8 < nk8) {
                const uint4 o0 = *reinterpret_cast<const uint4*>(koff + 8 * c8);
                const uint4 o1 = *reinterpret_cast<const uint4*>(koff + 8 * c8 + 4);
                const uint32_t o[8] = {o0.x, o0.y, o0.z, o0.w, o1.x, o1.y, o1.z, o1.w};
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    const float2 x = __ldg(reinterpret_cast<const float2*>(pj + o[u]));
                    gh[j][u] = x.x;
                    gl[j][u] = x.y;
                }
            }
        }
    };

    while (true) {
        if (tid == 0) s_row = atomicAdd(row_counter, 1);
        __syncthreads();
        const int Ia = s_row;
        if (Ia >= nas || s_abort) break;
        for (int k = tid; k < kpad; k += blockDim.x) {
            const uint32_t e = k < s1a ? connA[(size_t)Ia * s1a + k] : 0u;
            cs[k] = e;
            koff[k] = (e & kConnIdxMask) * (uint32_t)ldp * (uint32_t)sizeof(float2);
        }
        for (int j = tid; j < nt; j += blockDim.x) {
            acc_hi[j] = 0;
            acc_lo[j] = 0u;
        }
        __syncthreads();
        // B[c][k] = sgn_k V[P_k][perm[c]] 2^el, split into tf32 hi/lo; column c holds pair perm[c]
        // (off-diagonal pairs first, then the diagonal ones; -1 = padding)
        for (int idx = tid; idx < npad * kpad; idx += blockDim.x) {
            int R = idx / kpad, k = idx - R * kpad;
            float hi = 0.f, lo = 0.f;
            const int pr = perm[R];
            if (k < s1a && pr >= 0) {
                uint32_t e = cs[k];
                double v = V[(size_t)((e >> 21) & 1023) * ldv + pr] * grid;
                if (e & kSignBit) v = -v;
                hi = __uint_as_float(to_tf32((float)v));
                lo = __uint_as_float(to_tf32((float)(v - (double)hi)));
            }
            uint32_t off = kmaj_off(R, k, npad);
            *reinterpret_cast<float*>(Bhi + off) = hi;
            if (THREE) *reinterpret_cast<float*>(Blo + off) = lo;
        }
        fence_proxy_async();  // B (generic-proxy stores) becomes visible to the tensor core's reads
        gather(0);
        for (int t = 0; t <= ntiles; t++) {
            const int cur = t & 1, prv = cur ^ 1;
            // targets of the epilogue tile t-1, loaded early (consumed in (d)); rows past nbs and
            // pairs past npair hold no target
            const int jb_epi = (t - 1) * kTcM + 32 * q + lane;
            auto load_tg = [&](int i) {
                const int c8 = ec0 + NCG * i;
                return (t >= 1 && c8 < nn8)
                           ? __ldg(reinterpret_cast<const uint4*>(tgtR + ((size_t)c8 * ntiles * kTcM + jb_epi) * 8))
                           : make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);
            };
            uint4 tg[EB];
#pragma unroll
            for (int i = 0; i < EB; i++) tg[i] = load_tg(i);
            const uint32_t occ_epi = (cg == 0 && ndiag > 0 && t >= 1 && jb_epi < ns) ? __ldg(bstr + jb_epi) : 0u;
            // (a) the TMEM A buffer and accumulator prv are ready once tile t-1's MMAs completed
            if (t >= 1 && !mbar_wait_bounded(&bars[prv], (mma_count[prv] - 1) & 1)) {
                atomicCAS(err, 0, kErrTimeoutMma);
                s_abort = 1;
            }
            tc_fence_after();
            // (b) registers -> A in tensor memory
            if (t < ntiles) {
#pragma unroll
                for (int j = 0; j < GJ; j++) {
                    const int c8 = tc_gather_chunk<NW>(cg, j);
                    if (c8 < nk8) {
                        tmem_st8(tmem_base + tlane + kColAhi + 8 * c8, gh[j]);
                        if (THREE) tmem_st8(tmem_base + tlane + kColAlo + 8 * c8, gl[j]);
                    }
                }
                asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            }
            tc_fence_before();
            __syncthreads();
            if (s_abort) break;
            tc_fence_after();
            // (c) one thread issues the tile's MMAs into accumulator `cur`
            if (t < ntiles && tid == kTcMmaThread) {
                const uint32_t dt = tmem_base + (uint32_t)cur * kColAccStride;
                uint32_t acc = 0;
                for (int ks = 0; ks < nk8; ks++) {
                    const uint32_t ah = tmem_base + kColAhi + 8 * ks;
                    uint64_t bh = make_desc(sb_hi + ks * 2 * lbo_b, lbo_b, 128);
                    if (THREE) {
                        const uint32_t al = tmem_base + kColAlo + 8 * ks;
                        uint64_t bl = make_desc(sb_lo + ks * 2 * lbo_b, lbo_b, 128);
                        mma_tf32_ta(dt, al, bh, idesc, acc);
                        acc = 1;
                        mma_tf32_ta(dt, ah, bl, idesc, acc);
                    }
                    mma_tf32_ta(dt, ah, bh, idesc, acc);
                    acc = 1;
                }
                mma_commit(&bars[cur]);
            }
            if (t < ntiles) mma_count[cur]++;
            // (b') next tile's loads overlap the MMAs above and the epilogue below
            if (t + 1 < ntiles) gather(t + 1);
            // (d) epilogue of tile t-1: exact fixed-point scatter over beta replacements, in two
            // batches of accumulator chunks (fewer live registers)
            if (t >= 1) {
                const uint32_t tbase = tmem_base + (uint32_t)prv * kColAccStride + tlane;
                // y 2^el (grid folded into B) exactly in FP32 (|.| < 2^44), split as hi 2^22 + lo with
                // hi = round(y 2^(el-22)) and lo = round(y 2^el - hi 2^22), |lo| <= 2^21, both rounded by
                // adding 1.5 * 2^23; the raw bit patterns (integer + kMagicBits) are accumulated and
                // ncontrib * kMagicBits is removed per element when the row is written
                auto add_fixed = [&](float ys, uint32_t a, uint32_t g) {
                    const float t1 = fmaf(ys, 2.38418579e-7f, kMagic);
                    const float lf = fmaf(t1 - kMagic, -4194304.0f, ys);
                    red_pair(a, __float_as_uint(t1), __float_as_uint(lf + kMagic), g);
                };
                auto scatter = [&](const uint32_t (&rv)[8], const uint4& tw) {
                    const uint32_t w[4] = {tw.x, tw.y, tw.z, tw.w};
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        // two slots per 32-bit word; entry = Ib * 4 | sign (bit 0), 0xFFFF = no target
                        const uint32_t g0 = w[j] & 0xFFFFu, g1 = w[j] >> 16;
                        uint32_t h0, h1, l0, l1;
                        split_fixed2(__uint_as_float(rv[2 * j] ^ (g0 << 31)), __uint_as_float(rv[2 * j + 1] ^ (g1 << 31)),
                                     h0, h1, l0, l1);
                        red_pair(acc_s + (g0 & 0xFFFCu), h0, l0, g0);
                        red_pair(acc_s + (g1 & 0xFFFCu), h1, l1, g1);
                    }
                };
                uint4 tg2 = load_tg(EB);
                {
                    uint32_t rv[EB][8];
#pragma unroll
                    for (int i = 0; i < EB; i++) {
                        const int c8 = ec0 + NCG * i;
                        if (c8 < nn8) tmem_ld8_async(tbase + (uint32_t)(c8 * 8), rv[i]);
                    }
                    tmem_wait_ld8(rv[0]);
#pragma unroll
                    for (int i = 1; i < EB; i++) reg_after(rv[i]);
#pragma unroll
                    for (int i = 0; i < EB; i++)
                        if (ec0 + NCG * i < nn8) scatter(rv[i], tg[i]);
                }
                if (EB < EI && ec0 + NCG * EB < nn8) {
                    uint32_t rv[8];
                    tmem_ld8_async(tbase + (uint32_t)((ec0 + NCG * EB) * 8), rv);
                    tmem_wait_ld8(rv);
                    scatter(rv, tg2);
                }
                if (cg == 0 && ndiag > 0) {
                    // diagonal pairs (r,r): F_rr Jb = Jb for every occupied r, so the string's own
                    // element receives sum_{r occupied} T[Jb][(r,r)], added in FP32 in a fixed order
                    // and reduced as one contribution
                    uint32_t rd[2][8];
                    tmem_ld8_async(tbase + (uint32_t)(nn8 * 8), rd[0]);
                    if (ndc > 1) tmem_ld8_async(tbase + (uint32_t)((nn8 + 1) * 8), rd[1]);
                    tmem_wait_ld8(rd[0]);
                    reg_after(rd[1]);
                    const uint32_t occ = occ_epi;
                    float d = 0.f;
#pragma unroll
                    for (int r = 0; r < 16; r++)
                        if (r < ndiag && ((occ >> r) & 1u)) d += __uint_as_float(rd[r >> 3][r & 7]);
                    add_fixed(d, acc_s + (uint32_t)(jb_epi + diag_off) * 4u, jb_epi < ns ? 0u : 0xFFFFu);
                }
            }
            tc_fence_before();
        }
        if (s_abort) break;
        __syncthreads();
        // (e) sigma row = E0 * C row + opposite-spin part (exact fixed-point sum -> FP64)
        const double* Crow = C + (size_t)Ia * nt;
        double* Srow = S + (size_t)Ia * nt;
        for (int j = tid; j < nt; j += blockDim.x) {
            const unsigned mt = mag ? (unsigned)mag[j] * (unsigned)kMagicBits : magic_total;
            const int hi = (int)((unsigned)acc_hi[j] - mt), lo = (int)(acc_lo[j] - mt);
            const long long tot = ((long long)hi << kFixLoBits) + (long long)lo;
            Srow[j] = (accumulate ? Srow[j] : e0 * Crow[j]) + (double)tot * inv_grid;
        }
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
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(kTmemCols) : "memory");
}

// tgtR[c/8][Jb][c%8] = 16-bit scatter target of F_R Jb for the pair R = perm[c] of column c:
// Ib * 4 | sign (bit 0); no connection, padding columns, the diagonal-pair columns (c >= noff8) and rows
// past nstr (up to nrows, a whole number of tiles) -> 0xFFFF.  Chunk-major: the 8
// targets of one 8-pair chunk of consecutive Jb sit in consecutive 16-byte words, so a warp (32
// consecutive Jb) reads one chunk with fully coalesced loads.
__global__ void k_tgt_rows16(const int32_t* __restrict__ tgt, uint16_t* __restrict__ out, int nstr, int nrows,
                             int npp_in, const int* __restrict__ perm, int noff8, int npad_out) {
    size_t total = (size_t)npad_out * nrows;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int u = (int)(i & 7);
        const size_t cj = i >> 3;
        const int c8 = (int)(cj / nrows), J = (int)(cj - (size_t)c8 * nrows);
        const int col = 8 * c8 + u;
        const int R = col < noff8 ? perm[col] : -1;  // diagonal pairs are summed in registers, not scattered
        uint16_t v = 0xFFFFu;
        if (R >= 0 && J < nstr) {
            int32_t t = tgt[(size_t)J * npp_in + R];
            if (t != kNoTarget) v = (uint16_t)((((uint32_t)t & kConnIdxMask) << 2) | ((uint32_t)t >> 31));
        }
        out[i] = v;
    }
}

// C (FP64, nas x nbs) -> tf32 hi/lo planes with row stride ldp (zero padded); also max |C|
// hl[r][col] = (tf32 hi, tf32 lo) of C[r][col] (interleaved, row stride ldp), c32 = FP32 copy of C,
// cmax_bits = bits of max|C| rounded up
__global__ void k_split_tf32(const double* __restrict__ C, float2* __restrict__ hl, float* __restrict__ c32, int nas,
                             int nbs, int ldp, unsigned int* __restrict__ cmax_bits) {
    size_t total = (size_t)nas * ldp;
    float mx = 0.f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        int r = (int)(i / ldp), col = (int)(i % ldp);
        double v = col < nbs ? C[(size_t)r * nbs + col] : 0.0;
        const float h = __uint_as_float(to_tf32((float)v));
        hl[i] = make_float2(h, __uint_as_float(to_tf32((float)(v - (double)h))));
        if (col < nbs) c32[(size_t)r * nbs + col] = (float)v;
        mx = fmaxf(mx, fabsf((float)v));
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    // non-negative floats order like their bit patterns; round up by one ulp for safety
    if ((threadIdx.x & 31) == 0) atomicMax(cmax_bits, __float_as_uint(mx) + 1u);
}

size_t tc_smem_bytes(int s1a, int npair, int nbs, bool three) { return tc_layout(s1a, npair, nbs, three).total; }

float host_vmax(Context& c) {
    std::vector<double> hv(c.V.n);
    FCIB_CUDA(cudaMemcpy(hv.data(), c.V.p, sizeof(double) * c.V.n, cudaMemcpyDeviceToHost));
    double m = 0.0;
    for (double x : hv) m = std::max(m, std::fabs(x));
    return (float)(m * (1.0 + 1e-6)) + 1e-30f;
}

void ab_tc(Context& c, const double* C, double* S, bool three) {
    const int nas = (int)c.nas, nbs = (int)c.nbs;
    const int s1a = c.A.s1;
    const int n = c.n, kb = c.nb;
    const SymSpace& y = c.sym;
    if (c.vmax <= 0.0f) c.vmax = host_vmax(c);
    ensure_counter(c);
    FCIB_CUDA(cudaMemsetAsync(c.counter.p, 0, 3 * sizeof(int), c.stream));
    unsigned int* cmax_bits = reinterpret_cast<unsigned int*>(c.counter.p + 3);
    FCIB_CUDA(cudaMemsetAsync(cmax_bits, 0, sizeof(unsigned int), c.stream));
    auto kern = three ? k_ab_tc<true, kTcWarps> : k_ab_tc<false, kTcWarps>;
    // shared memory of one launch: one CTA per SM (it owns all tensor memory)
    int attr_smem = -1;  // the kernel's dynamic shared memory limit, raised only when a launch needs more
    auto smem_of = [&](int s1, int ncol, int nt, int noff8, int ndiag) {
        const TcLayout L = tc_layout(s1, ncol, nt, three);
        FCIB_CHECK(nt <= kMaxBetaStrings, FCIB_ERR_UNSUPPORTED, "tensor-core opposite-spin kernel: too many beta strings");
        FCIB_CHECK(L.npad <= 144 && L.kpad <= 72 && noff8 / 8 <= 15 && ndiag <= 16 && L.kpad / 8 <= 9,
                   FCIB_ERR_UNSUPPORTED, "tensor-core kernel: more than 16 active orbitals");
        const size_t smem = std::max<size_t>(L.total, 120 * 1024);
        FCIB_CHECK(smem + 2048 <= (size_t)c.smem_optin, FCIB_ERR_UNSUPPORTED,
                   "tensor-core kernel: sigma row and integral block exceed shared memory");
        if ((int)smem > attr_smem) {
            FCIB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            attr_smem = (int)smem;
        }
        return smem;
    };
    c.tc_ev.ensure();
    if (y.on) {
        // blocked layout: TF32 planes per alpha block, one launch per sub-problem
        // a sub-problem whose source columns start inside a row gathers up to 127 pairs past the
        // row's end; the planes carry that much (zeroed) slack at their end
        const size_t slack = kTcM;
        if (c.tf_hi.n != 2 * (y.plane_total + slack)) {
            c.tf_hi.alloc(2 * (y.plane_total + slack));
            FCIB_CUDA(cudaMemsetAsync(c.tf_hi.p, 0, sizeof(float) * c.tf_hi.n, c.stream));
        }
        c.c32.alloc((size_t)c.nvec);
        float2* hl = reinterpret_cast<float2*>(c.tf_hi.p);
        for (int h = 0; h < c.nirrep; h++) {
            const int nb_h = y.bcnt[h ^ c.irrep];
            if (y.acnt[h] == 0 || nb_h == 0) continue;
            k_split_tf32<<<8 * c.num_sms, 256, 0, c.stream>>>(C + y.d.blk[h], hl + y.plane_off[h], c.c32.p + y.d.blk[h],
                                                              y.acnt[h], nb_h, y.ldp[h], cmax_bits);
            FCIB_KCHECK();
        }
        c.c32_ready = true;
        FCIB_CUDA(cudaEventRecord(c.tc_ev.e[0], c.stream));
        // one row counter per sub-problem, all zeroed at once (the error flag in counter slot 1 stays)
        c.subctr.alloc(std::max<size_t>(y.ab.size(), 1));
        FCIB_CUDA(cudaMemsetAsync(c.subctr.p, 0, sizeof(int) * c.subctr.n, c.stream));
        for (size_t i = 0; i < y.ab.size(); i++) {
            const AbSub& u = y.ab[i];
            const int g = u.g, noff8 = y.noff8_g[g], ndiag = y.ndiag_g[g];
            const int ncol = noff8 + ndiag;
            const size_t smem = smem_of(u.kmax, ncol, u.nt, noff8, ndiag);
            const int64_t tb = y.d.blk[u.ha] + (int64_t)u.row0 * u.nt;
            kern<<<std::min(u.rows, c.num_sms), kTcWarps * 32, smem, c.stream>>>(
                hl + y.plane_off[u.src] + u.col0, y.ldp[u.src], u.ns, C + tb, S + tb, u.nt, u.accumulate,
                y.conn.p + u.conn, u.kmax, y.tgt16.p + u.tgt16, ncol, y.perm.p + y.perm_off[g], noff8, ndiag,
                u.diag_off, y.bstr_sorted.p + y.d.boff[u.ha ^ c.irrep ^ g] + u.col0, kb, y.Vz.p, y.npp, c.vmax,
                cmax_bits, u.rows, 0,
                y.mag.p + u.mag, c.scalar, c.subctr.p + i, c.counter.p + 1);
            FCIB_KCHECK();
        }
        FCIB_CUDA(cudaEventRecord(c.tc_ev.e[1], c.stream));
        c.tc_recorded = true;
        return;
    }
    // columns: the n(n-1)/2 off-diagonal pairs in pair order (padded to a multiple of 8), then the n
    // diagonal pairs (r,r)
    const int noff = n * (n - 1) / 2, noff8 = (noff + 7) / 8 * 8;
    const int ncol = noff8 + n;
    const size_t smem = smem_of(s1a, ncol, nbs, noff8, n);
    const TcLayout L = tc_layout(s1a, ncol, nbs, three);
    const int ntiles = (nbs + kTcM - 1) / kTcM;
    const int ldp = ntiles * kTcM;  // plane rows padded to whole tiles (zeros)
    FCIB_CHECK((uint64_t)nas * ldp * sizeof(float2) < (1ull << 32), FCIB_ERR_UNSUPPORTED,
               "tensor-core kernel: TF32 planes exceed the 32-bit gather offsets");
    if (!c.tgtR16.p) {
        std::vector<int> perm(L.npad, -1);
        for (int p = 0, col = 0; p < n; p++)
            for (int q = 0; q < p; q++) perm[col++] = p * (p + 1) / 2 + q;
        for (int r = 0; r < n; r++) perm[noff8 + r] = r * (r + 1) / 2 + r;
        c.tc_perm.upload(perm, c.stream);
        c.tgtR16.alloc((size_t)L.npad * ldp);
        k_tgt_rows16<<<4 * c.num_sms, 256, 0, c.stream>>>(c.B.tgt.p, c.tgtR16.p, nbs, ldp, c.B.npair_pad,
                                                          c.tc_perm.p, noff8, L.npad);
        FCIB_KCHECK();
    }
    c.tf_hi.alloc(2 * (size_t)nas * ldp);  // interleaved hi/lo pairs
    c.c32.alloc((size_t)nas * nbs);
    float2* hl = reinterpret_cast<float2*>(c.tf_hi.p);
    k_split_tf32<<<8 * c.num_sms, 256, 0, c.stream>>>(C, hl, c.c32.p, nas, nbs, ldp, cmax_bits);
    FCIB_KCHECK();
    c.c32_ready = true;
    const int grid = std::min(nas, c.num_sms);
    FCIB_CUDA(cudaEventRecord(c.tc_ev.e[0], c.stream));
    kern<<<grid, kTcWarps * 32, smem, c.stream>>>(hl, ldp, nbs, C, S, nbs, 0, c.A.conn.p, s1a, c.tgtR16.p, ncol,
                                                  c.tc_perm.p, noff8, n, 0, c.B.str.p, kb, c.V.p, c.A.npair_pad, c.vmax,
                                                  cmax_bits, nas, kb * (n - kb) + 1, nullptr, c.scalar, c.counter.p,
                                                  c.counter.p + 1);
    FCIB_KCHECK();
    FCIB_CUDA(cudaEventRecord(c.tc_ev.e[1], c.stream));
    c.tc_recorded = true;
}

// timeout flags of one mixed sigma: slot 1 (opposite-spin kernel, when it ran) and slot 5
// (tensor-core same-spin groups, cleared at the start of every mixed same-spin term)
int tc_check_error(Context& c, bool opposite_spin) {
    if (!c.counter.p) return 0;
    int h[6] = {0, 0, 0, 0, 0, 0};
    FCIB_CUDA(cudaMemcpyAsync(h, c.counter.p, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
    FCIB_CUDA(cudaStreamSynchronize(c.stream));
    if (opposite_spin && h[1]) return h[1];
    return h[5];
}

}  // namespace fcib
