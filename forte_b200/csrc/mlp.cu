// Learned per-determinant Davidson preconditioner (no counterpart in the reference).
//
// The reference's correction is t_I = r_I / (lambda - H_II), zero when |lambda - H_II| <= 1e-6
// (davidson_liu_solver.cc:432-448).  The learned correction keeps it and rescales every element:
//     t_I <- t_I * (1 + R tanh m(x_I)),  R = kMlpRange = 0.25,
// so a network with zero output is exactly the reference's preconditioner, and the factor stays
// in (1 - R, 1 + R).  (With R = 1 or 0.5 the trained network damped many determinants towards
// zero and Davidson needed more iterations; 0.25 keeps every component alive.)  m is a 35 -> 64 -> 64 -> 64 -> 1 ReLU network with BF16 weights and FP32
// accumulation.  Inputs x_I:
//   x[0..15]  alpha excitation bits: occupation XOR aufbau string, orbitals na-8 .. na+7
//   x[16..31] beta excitation bits, orbitals nb-8 .. nb+7
//   x[32] = u / (1 + |u|), x[33] = 0.05 / (0.05 + |u|), u = H_II - lambda (Eh)
//   x[34] = log2(|r_I| / ||r|| + 2^-30) / 30 + 1
// Activations entering layers 2 and 3 are rounded to BF16 (tensor-core operands); layer 1 and
// the output layer run in FP32.  Weight vector (FP32 master copy, FCIB_MLP_NWEIGHTS floats):
//   W1[64][35], b1[64], W2[64][64], b2[64], W3[64][64], b3[64], w4[64], b4.
//
// Kernels:
//   k_mlp_apply<Src>  inference, one warp per 16 determinants: layer 1 on CUDA cores, layers 2-3
//                     as mma.sync m16n8k16 BF16 tiles whose FP32 accumulators are re-packed
//                     in registers as the next layer's A fragments; in place on the correction.
//   k_mlp_grad        training forward + backward for 32 samples per CTA, shared-memory
//                     activations, FP32 gradient accumulation with global atomics.
//   k_adam            Adam update of the FP32 master weights.
#include <cuda_bf16.h>

#include <random>

namespace fcib {

constexpr int kMlpIn = 35;
constexpr int kMlpH = 64;
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpH * kMlpIn;
constexpr int kOffW2 = kOffB1 + kMlpH;
constexpr int kOffB2 = kOffW2 + kMlpH * kMlpH;
constexpr int kOffW3 = kOffB2 + kMlpH;
constexpr int kOffB3 = kOffW3 + kMlpH * kMlpH;
constexpr int kOffW4 = kOffB3 + kMlpH;
constexpr int kOffB4 = kOffW4 + kMlpH;
constexpr int kMlpNW = kOffB4 + 1;
static_assert(kMlpNW == FCIB_MLP_NWEIGHTS, "weight layout");
#ifndef FCIB_MLP_RANGE
#define FCIB_MLP_RANGE 0.25f
#endif
constexpr float kMlpRange = FCIB_MLP_RANGE;  // factor = 1 + kMlpRange * tanh(m)
constexpr int kW2Ld = 72;
// Tiles of 16 determinants whose diagonal corrections are all below kMlpSkip * ||t|| keep the
// diagonal rule (their elements change the correction by less than 1e-4 ||t|| each).
constexpr double kMlpSkip = 1.0e-4;  // padded bf16 row stride of W2/W3 in shared memory (conflict-free B fragments)

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__host__ __device__ __forceinline__ uint32_t excitation_window(uint32_t occ, int k) {
    const uint32_t ref = (k >= 32) ? 0xFFFFFFFFu : ((1u << k) - 1u);
    const uint32_t d = occ ^ ref;
    return (k >= 8 ? (d >> (k - 8)) : (d << (8 - k))) & 0xFFFFu;
}

// scalar inputs x[32..34] from u = H_II - lambda and rr = |r_I| / ||r||
__device__ __forceinline__ void scalar_features(float u, float rr, float& x32, float& x33, float& x34) {
    const float au = fabsf(u);
    x32 = u / (1.0f + au);
    x33 = 0.05f / (0.05f + au);
    x34 = log2f(rr + 9.3132257e-10f) * (1.0f / 30.0f) + 1.0f;
}

struct MlpDevice {
    const float* w;  // FP32 master copy (BF16-representable values where BF16 is used)
};

// ---- inference --------------------------------------------------------------------------
// Per-string layer-1 tables: tab[s][c] = sum over the excitation bits b of string s of
// W1[c][off + b] (BF16-rounded weights), so that layer 1 of determinant (Ia, Ib) is
// b1 + tabA[Ia] + tabB[Ib] + W1[:, 32..34] x[32..34].
__global__ void k_mlp_tables(const uint32_t* __restrict__ str, int nstr, int k, int off, const float* __restrict__ w,
                             float* __restrict__ tab) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= (size_t)nstr * kMlpH) return;
    const int s = (int)(i / kMlpH), c = (int)(i - (size_t)s * kMlpH);
    float acc = 0.0f;
    for (uint32_t e = excitation_window(str[s], k); e; e &= e - 1) acc += bf16r(w[kOffW1 + c * kMlpIn + off + __ffs(e) - 1]);
    tab[i] = acc;
}

struct MlpSmem {
    float w1[kMlpH][kMlpIn];
    float b1[kMlpH], b2[kMlpH], b3[kMlpH], w4[kMlpH];
    float b4;
    __nv_bfloat16 w2[kMlpH * kW2Ld];
    __nv_bfloat16 w3[kMlpH * kW2Ld];
};

struct EngineSource {  // determinant I of an engine-layout vector: diagonal correction t rescaled in place
    double* t;
    const double* hd;
    const float* tabA;  // [nas][64]
    const float* tabB;  // [nbs][64]
    unsigned nbs;
    double lambda;
    float inv_rnorm;
    float skip;  // tiles whose |t_I| are all below this keep the diagonal rule
    SymDev sd;   // the blocked layout (sd.on) or C1
    __device__ bool load(size_t I, uint32_t& a, uint32_t& b, float& u, float& rr, double& tv) const {
        if (sd.on) {
            int ia, ib;
            sym_decode(sd, (int64_t)I, ia, ib);
            a = (uint32_t)ia;
            b = (uint32_t)ib;
        } else {
            const unsigned Iu = (unsigned)I;
            a = Iu / nbs;
            b = Iu - a * nbs;
        }
        const double h = hd[I];
        tv = t[I];
        u = (float)(h - lambda);
        rr = (float)fabs(tv * (lambda - h)) * inv_rnorm;
        return fabs(tv) >= (double)skip;
    }
    __device__ float2 excite(uint32_t a, uint32_t b, int col, const MlpSmem&) const {
        const float2 x = *reinterpret_cast<const float2*>(tabA + (size_t)a * kMlpH + col);
        const float2 y = *reinterpret_cast<const float2*>(tabB + (size_t)b * kMlpH + col);
        return make_float2(x.x + y.x, x.y + y.y);
    }
    __device__ void store(size_t I, double tv, float f) const { t[I] = tv * (double)f; }
};

struct SampleSource {  // training-style samples: factor out
    const uint32_t* ea;
    const uint32_t* eb;
    const float* u;
    const float* r;
    float* factor;
    __device__ bool load(size_t I, uint32_t& a, uint32_t& b, float& uu, float& rr, double& tv) const {
        a = ea[I] | (eb[I] << 16);
        b = 0;
        uu = u[I];
        rr = fabsf(r[I]);
        tv = 0.0;
        return true;
    }
    __device__ float2 excite(uint32_t a, uint32_t, int col, const MlpSmem& S) const {
        float x = 0.0f, y = 0.0f;
        for (uint32_t e = a; e; e &= e - 1) {
            const int bit = __ffs(e) - 1;
            x += S.w1[col][bit];
            y += S.w1[col + 1][bit];
        }
        return make_float2(x, y);
    }
    __device__ void store(size_t I, double, float f) const { factor[I] = f; }
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// one hidden layer on the tensor cores: A fragments in, relu(A W^T + b) as FP32 C fragments
__device__ __forceinline__ void mma_layer(uint32_t (&a)[4][4], const __nv_bfloat16* W, const float* b, int g, int t4,
                                          float (&out)[8][4]) {
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        out[nt][0] = out[nt][1] = out[nt][2] = out[nt][3] = 0.0f;
        const __nv_bfloat16* wrow = W + (8 * nt + g) * kW2Ld + 2 * t4;
#pragma unroll
        for (int kt = 0; kt < 4; kt++) {
            const uint32_t b0 = *reinterpret_cast<const uint32_t*>(wrow + 16 * kt);
            const uint32_t b1 = *reinterpret_cast<const uint32_t*>(wrow + 16 * kt + 8);
            mma_bf16(out[nt], a[kt], b0, b1);
        }
        const float c0 = b[8 * nt + 2 * t4], c1 = b[8 * nt + 2 * t4 + 1];
        out[nt][0] = fmaxf(out[nt][0] + c0, 0.0f);
        out[nt][1] = fmaxf(out[nt][1] + c1, 0.0f);
        out[nt][2] = fmaxf(out[nt][2] + c0, 0.0f);
        out[nt][3] = fmaxf(out[nt][3] + c1, 0.0f);
    }
}

// One warp per tile of 16 consecutive determinants.  Lanes 0..15 load one determinant each and
// compute its scalar inputs; mma fragment lane (g, t4) works on rows g and g + 8, whose inputs
// arrive by shuffles; the factor goes back to the loading lane by a shuffle.
template <class Src>
__global__ void __launch_bounds__(256) k_mlp_apply(Src src, size_t N, MlpDevice P) {
    extern __shared__ __align__(16) unsigned char mlp_smem_raw[];
    MlpSmem& S = *reinterpret_cast<MlpSmem*>(mlp_smem_raw);
    for (int i = threadIdx.x; i < kMlpH * kMlpIn; i += blockDim.x) (&S.w1[0][0])[i] = bf16r(P.w[kOffW1 + i]);
    for (int i = threadIdx.x; i < kMlpH; i += blockDim.x) {
        S.b1[i] = P.w[kOffB1 + i];
        S.b2[i] = P.w[kOffB2 + i];
        S.b3[i] = P.w[kOffB3 + i];
        S.w4[i] = bf16r(P.w[kOffW4 + i]);
    }
    if (threadIdx.x == 0) S.b4 = P.w[kOffB4];
    for (int i = threadIdx.x; i < kMlpH * kMlpH; i += blockDim.x) {
        const int j = i / kMlpH, k = i - j * kMlpH;
        S.w2[j * kW2Ld + k] = __float2bfloat16_rn(P.w[kOffW2 + i]);
        S.w3[j * kW2Ld + k] = __float2bfloat16_rn(P.w[kOffW3 + i]);
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, g = lane >> 2, t4 = lane & 3;
    const size_t warp = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
    const size_t nwarps = (gridDim.x * (size_t)blockDim.x) >> 5;
    const size_t ntiles = (N + 15) / 16;
    for (size_t tile = warp; tile < ntiles; tile += nwarps) {
        const size_t I = tile * 16 + (lane & 15);
        const bool mine = lane < 16 && I < N;
        uint32_t ka = 0, kb = 0;
        float u = 0.0f, rr = 0.0f;
        double tv = 0.0;
        bool big = src.load(mine ? I : N - 1, ka, kb, u, rr, tv);
        if (!__any_sync(0xffffffffu, mine && big)) continue;
        float f0, f1, f2;
        scalar_features(u, rr, f0, f1, f2);
        uint32_t ra[2], rb[2];
        float x[2][3];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int srcl = g + 8 * h;
            ra[h] = __shfl_sync(0xffffffffu, ka, srcl);
            rb[h] = __shfl_sync(0xffffffffu, kb, srcl);
            x[h][0] = __shfl_sync(0xffffffffu, f0, srcl);
            x[h][1] = __shfl_sync(0xffffffffu, f1, srcl);
            x[h][2] = __shfl_sync(0xffffffffu, f2, srcl);
        }
        // layer 1 (FP32): columns 16kt + 2t4 + {0,1} and 16kt + 8 + 2t4 + {0,1} of rows g, g+8
        uint32_t a[4][4];
#pragma unroll
        for (int kt = 0; kt < 4; kt++) {
            float z[2][4];
#pragma unroll
            for (int half = 0; half < 2; half++) {
                const int col = 16 * kt + 8 * half + 2 * t4;
                const float* w0 = S.w1[col];
                const float* w1 = S.w1[col + 1];
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const float2 e = src.excite(ra[h], rb[h], col, S);
                    const float z0 = S.b1[col] + w0[32] * x[h][0] + w0[33] * x[h][1] + w0[34] * x[h][2] + e.x;
                    const float z1 = S.b1[col + 1] + w1[32] * x[h][0] + w1[33] * x[h][1] + w1[34] * x[h][2] + e.y;
                    z[h][2 * half] = fmaxf(z0, 0.0f);
                    z[h][2 * half + 1] = fmaxf(z1, 0.0f);
                }
            }
            a[kt][0] = pack_bf16(z[0][0], z[0][1]);
            a[kt][1] = pack_bf16(z[1][0], z[1][1]);
            a[kt][2] = pack_bf16(z[0][2], z[0][3]);
            a[kt][3] = pack_bf16(z[1][2], z[1][3]);
        }
        float c[8][4];
        mma_layer(a, S.w2, S.b2, g, t4, c);
#pragma unroll
        for (int kt = 0; kt < 4; kt++) {
            a[kt][0] = pack_bf16(c[2 * kt][0], c[2 * kt][1]);
            a[kt][1] = pack_bf16(c[2 * kt][2], c[2 * kt][3]);
            a[kt][2] = pack_bf16(c[2 * kt + 1][0], c[2 * kt + 1][1]);
            a[kt][3] = pack_bf16(c[2 * kt + 1][2], c[2 * kt + 1][3]);
        }
        mma_layer(a, S.w3, S.b3, g, t4, c);
        float m0 = 0.0f, m1 = 0.0f;
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            const float w0 = S.w4[8 * nt + 2 * t4], w1 = S.w4[8 * nt + 2 * t4 + 1];
            m0 += c[nt][0] * w0 + c[nt][1] * w1;
            m1 += c[nt][2] * w0 + c[nt][3] * w1;
        }
        m0 += __shfl_xor_sync(0xffffffffu, m0, 1);
        m0 += __shfl_xor_sync(0xffffffffu, m0, 2);
        m1 += __shfl_xor_sync(0xffffffffu, m1, 1);
        m1 += __shfl_xor_sync(0xffffffffu, m1, 2);
        // lane (g, t4): t4 == 0 holds row g, t4 == 1 row g + 8; the loader of row r is lane r
        const float fm = 1.0f + kMlpRange * tanhf((t4 ? m1 : m0) + S.b4);
        const int r = lane & 15;
        const float fr = __shfl_sync(0xffffffffu, fm, ((r & 7) << 2) | (r >> 3));
        if (mine) src.store(I, tv, fr);
    }
}

// ---- training ---------------------------------------------------------------------------
constexpr int kGradSB = 32;  // samples per CTA

struct TrainSamples {
    const uint32_t* ea;
    const uint32_t* eb;
    const float* u;
    const float* r;    // r_I / ||r||
    const float* tgt;  // target correction element (same scale as -r/u)
    const float* wgt;  // per-sample loss weight (NULL = 1)
    const int* idx;    // minibatch sample indices
    int count;
};

struct GradSmem {
    float W1[kMlpH][kMlpIn];
    float W2[kMlpH][kMlpH + 1];
    float W3[kMlpH][kMlpH + 1];
    float b1[kMlpH], b2[kMlpH], b3[kMlpH], w4[kMlpH];
    float b4;
    float X[kGradSB][kMlpIn];
    float H1[kGradSB][kMlpH + 1], H2[kGradSB][kMlpH + 1], H3[kGradSB][kMlpH + 1];
    float D3[kGradSB][kMlpH + 1], D2[kGradSB][kMlpH + 1], D1[kGradSB][kMlpH + 1];
    float dm[kGradSB];
};

// forward + backward for one CTA's samples; grad += dL/dw with L = scale * sum wgt (t f - tgt)^2
__global__ void __launch_bounds__(256) k_mlp_grad(TrainSamples d, const float* __restrict__ w, float* __restrict__ grad,
                                                  double* __restrict__ loss, float scale) {
    extern __shared__ __align__(16) unsigned char grad_smem_raw[];
    GradSmem& S = *reinterpret_cast<GradSmem*>(grad_smem_raw);
    const int tid = threadIdx.x;
    for (int i = tid; i < kMlpH * kMlpIn; i += blockDim.x) (&S.W1[0][0])[i] = bf16r(w[kOffW1 + i]);
    for (int i = tid; i < kMlpH * kMlpH; i += blockDim.x) {
        const int j = i / kMlpH, k = i - j * kMlpH;
        S.W2[j][k] = bf16r(w[kOffW2 + i]);
        S.W3[j][k] = bf16r(w[kOffW3 + i]);
    }
    for (int i = tid; i < kMlpH; i += blockDim.x) {
        S.b1[i] = w[kOffB1 + i];
        S.b2[i] = w[kOffB2 + i];
        S.b3[i] = w[kOffB3 + i];
        S.w4[i] = bf16r(w[kOffW4 + i]);
    }
    if (tid == 0) S.b4 = w[kOffB4];
    const int s0 = blockIdx.x * kGradSB;
    const int ns = min(kGradSB, d.count - s0);
    if (tid < kGradSB) {
        float* x = S.X[tid];
        for (int i = 0; i < kMlpIn; i++) x[i] = 0.0f;
        if (tid < ns) {
            const int I = d.idx[s0 + tid];
            const uint32_t e = d.ea[I] | (d.eb[I] << 16);
            for (int i = 0; i < 32; i++) x[i] = (float)(e >> i & 1u);
            scalar_features(d.u[I], fabsf(d.r[I]), x[32], x[33], x[34]);
        }
    }
    __syncthreads();
    const int j = tid & 63, sq = tid >> 6;  // hidden unit, sample quarter
    // forward
    for (int s = sq; s < kGradSB; s += 4) {
        float z = S.b1[j];
        for (int i = 0; i < kMlpIn; i++) z += S.W1[j][i] * S.X[s][i];
        S.H1[s][j] = bf16r(fmaxf(z, 0.0f));
    }
    __syncthreads();
    for (int s = sq; s < kGradSB; s += 4) {
        float z = S.b2[j];
        for (int k = 0; k < kMlpH; k++) z += S.W2[j][k] * S.H1[s][k];
        S.H2[s][j] = bf16r(fmaxf(z, 0.0f));
    }
    __syncthreads();
    for (int s = sq; s < kGradSB; s += 4) {
        float z = S.b3[j];
        for (int k = 0; k < kMlpH; k++) z += S.W3[j][k] * S.H2[s][k];
        S.H3[s][j] = fmaxf(z, 0.0f);
    }
    __syncthreads();
    if (tid < kGradSB) {
        float dm = 0.0f;
        if (tid < ns) {
            const int I = d.idx[s0 + tid];
            float m = S.b4;
            for (int k = 0; k < kMlpH; k++) m += S.w4[k] * S.H3[tid][k];
            const float th = tanhf(m);
            const float u = d.u[I];
            const float t = (fabsf(u) > 1.0e-6f) ? -d.r[I] / u : 0.0f;
            const float diff = t * (1.0f + kMlpRange * th) - d.tgt[I];
            const float ws = d.wgt ? d.wgt[I] : 1.0f;
            atomicAdd(loss, (double)(scale * ws * diff * diff));
            dm = 2.0f * scale * ws * diff * t * kMlpRange * (1.0f - th * th);
        }
        S.dm[tid] = dm;
    }
    __syncthreads();
    // output layer and layer-3 pre-activation gradients
    for (int s = sq; s < kGradSB; s += 4) S.D3[s][j] = (S.H3[s][j] > 0.0f) ? S.dm[s] * S.w4[j] : 0.0f;
    if (tid < kMlpH) {
        float gw = 0.0f;
        for (int s = 0; s < kGradSB; s++) gw += S.dm[s] * S.H3[s][tid];
        atomicAdd(grad + kOffW4 + tid, gw);
    }
    if (tid == 0) {
        float gb = 0.0f;
        for (int s = 0; s < kGradSB; s++) gb += S.dm[s];
        atomicAdd(grad + kOffB4, gb);
    }
    __syncthreads();
    // layer 3: dW3 = D3^T H2, db3, D2 = (D3 W3) * [H2 > 0]
    {
        const int jj = tid >> 2, k0 = (tid & 3) * 16;
        for (int k = k0; k < k0 + 16; k++) {
            float gsum = 0.0f;
            for (int s = 0; s < kGradSB; s++) gsum += S.D3[s][jj] * S.H2[s][k];
            atomicAdd(grad + kOffW3 + jj * kMlpH + k, gsum);
        }
    }
    if (tid < kMlpH) {
        float gb = 0.0f;
        for (int s = 0; s < kGradSB; s++) gb += S.D3[s][tid];
        atomicAdd(grad + kOffB3 + tid, gb);
    }
    for (int s = sq; s < kGradSB; s += 4) {
        float a = 0.0f;
        for (int jj = 0; jj < kMlpH; jj++) a += S.D3[s][jj] * S.W3[jj][j];
        S.D2[s][j] = (S.H2[s][j] > 0.0f) ? a : 0.0f;
    }
    __syncthreads();
    // layer 2
    {
        const int jj = tid >> 2, k0 = (tid & 3) * 16;
        for (int k = k0; k < k0 + 16; k++) {
            float gsum = 0.0f;
            for (int s = 0; s < kGradSB; s++) gsum += S.D2[s][jj] * S.H1[s][k];
            atomicAdd(grad + kOffW2 + jj * kMlpH + k, gsum);
        }
    }
    if (tid < kMlpH) {
        float gb = 0.0f;
        for (int s = 0; s < kGradSB; s++) gb += S.D2[s][tid];
        atomicAdd(grad + kOffB2 + tid, gb);
    }
    for (int s = sq; s < kGradSB; s += 4) {
        float a = 0.0f;
        for (int jj = 0; jj < kMlpH; jj++) a += S.D2[s][jj] * S.W2[jj][j];
        S.D1[s][j] = (S.H1[s][j] > 0.0f) ? a : 0.0f;
    }
    __syncthreads();
    // layer 1
    for (int e = tid; e < kMlpH * kMlpIn; e += blockDim.x) {
        const int jj = e / kMlpIn, i = e - jj * kMlpIn;
        float gsum = 0.0f;
        for (int s = 0; s < kGradSB; s++) gsum += S.D1[s][jj] * S.X[s][i];
        atomicAdd(grad + kOffW1 + e, gsum);
    }
    if (tid < kMlpH) {
        float gb = 0.0f;
        for (int s = 0; s < kGradSB; s++) gb += S.D1[s][tid];
        atomicAdd(grad + kOffB1 + tid, gb);
    }
}

__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v, const float* __restrict__ g,
                       int n, float lr, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = 0.9f * m[i] + 0.1f * gi;
    const float vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + 1.0e-8f);
}

// diagonal correction t = r / (lambda - H_II), 0 when |lambda - H_II| <= 1e-6
__global__ void k_diag_correction(double* __restrict__ t, const double* __restrict__ hd, double lambda, size_t N) {
    for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < N; I += (size_t)gridDim.x * blockDim.x) {
        const double den = lambda - hd[I];
        t[I] = (fabs(den) > 1.0e-6) ? t[I] / den : 0.0;
    }
}

// ---- host -------------------------------------------------------------------------------

void mlp_apply(Context& c, double* t, double lambda, double rnorm, double tnorm) {
    FCIB_CHECK(c.mlp_w.p, FCIB_ERR_STATE, "learned preconditioner selected but no MLP weights are loaded (fcib_set_mlp)");
    FCIB_CHECK(c.ndet < ((int64_t)1 << 32), FCIB_ERR_UNSUPPORTED, "learned preconditioner: determinant index above 2^32");
    if (!c.mlp_tables_ready) {
        c.mlp_tabA.alloc((size_t)c.nas * kMlpH);
        c.mlp_tabB.alloc((size_t)c.nbs * kMlpH);
        k_mlp_tables<<<(unsigned)((c.nas * kMlpH + 255) / 256), 256, 0, c.stream>>>(c.A.str.p, (int)c.nas, c.na, 0,
                                                                                  c.mlp_w.p, c.mlp_tabA.p);
        FCIB_KCHECK();
        k_mlp_tables<<<(unsigned)((c.nbs * kMlpH + 255) / 256), 256, 0, c.stream>>>(c.B.str.p, (int)c.nbs, c.nb, 16,
                                                                                  c.mlp_w.p, c.mlp_tabB.p);
        FCIB_KCHECK();
        c.mlp_tables_ready = true;
    }
    EngineSource src{t, c.hdiag.p, c.mlp_tabA.p, c.mlp_tabB.p, (unsigned)c.nbs, lambda,
                     (float)(rnorm > 0.0 ? 1.0 / rnorm : 0.0), (float)(kMlpSkip * tnorm), sym_dev(c)};
    const size_t smem = sizeof(MlpSmem);
    FCIB_CUDA(cudaFuncSetAttribute(k_mlp_apply<EngineSource>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const size_t N = (size_t)c.nvec;
    const int grid = (int)std::min<size_t>((size_t)6 * c.num_sms, (N + 127) / 128);
    k_mlp_apply<EngineSource><<<grid, 256, smem, c.stream>>>(src, N, MlpDevice{c.mlp_w.p});
    FCIB_KCHECK();
}

// Xavier-uniform hidden layers, zero output layer (the network starts as the diagonal rule)
static void mlp_init(std::vector<float>& w, uint64_t seed) {
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int fan_in, int fan_out) {
        const float a = std::sqrt(6.0f / (float)(fan_in + fan_out));
        std::uniform_real_distribution<float> U(-a, a);
        for (int i = 0; i < fan_in * fan_out; i++) w[off + i] = U(rng);
    };
    std::fill(w.begin(), w.end(), 0.0f);
    fill(kOffW1, kMlpIn, kMlpH);
    fill(kOffW2, kMlpH, kMlpH);
    fill(kOffW3, kMlpH, kMlpH);
}

struct DeviceSamples {
    DBuf<uint32_t> ea, eb;
    DBuf<float> u, r, tgt, wgt;
    void upload(int64_t n, const uint32_t* a, const uint32_t* b, const float* uu, const float* rr, const float* tt,
                cudaStream_t s, const float* ww = nullptr) {
        ea.alloc(n);
        eb.alloc(n);
        u.alloc(n);
        r.alloc(n);
        FCIB_CUDA(cudaMemcpyAsync(ea.p, a, 4 * n, cudaMemcpyHostToDevice, s));
        FCIB_CUDA(cudaMemcpyAsync(eb.p, b, 4 * n, cudaMemcpyHostToDevice, s));
        FCIB_CUDA(cudaMemcpyAsync(u.p, uu, 4 * n, cudaMemcpyHostToDevice, s));
        FCIB_CUDA(cudaMemcpyAsync(r.p, rr, 4 * n, cudaMemcpyHostToDevice, s));
        if (tt) {
            tgt.alloc(n);
            FCIB_CUDA(cudaMemcpyAsync(tgt.p, tt, 4 * n, cudaMemcpyHostToDevice, s));
        }
        if (ww) {
            wgt.alloc(n);
            FCIB_CUDA(cudaMemcpyAsync(wgt.p, ww, 4 * n, cudaMemcpyHostToDevice, s));
        }
    }
};

static void launch_grad(const DeviceSamples& ds, const int* idx, int count, const float* w, float* grad, double* loss,
                        float scale, cudaStream_t s) {
    TrainSamples d{ds.ea.p, ds.eb.p, ds.u.p, ds.r.p, ds.tgt.p, ds.wgt.p, idx, count};
    const size_t smem = sizeof(GradSmem);
    FCIB_CUDA(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_mlp_grad<<<(count + kGradSB - 1) / kGradSB, 256, smem, s>>>(d, w, grad, loss, scale);
    FCIB_KCHECK();
}

}  // namespace fcib

extern "C" {

int fcib_set_mlp(fcib_ctx* ctx, const float* weights, int nweights) {
    if (!ctx) { set_error("null context"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        ctx->c.mlp_tables_ready = false;
        if (!weights) {
            ctx->c.mlp_w.release();
            return;
        }
        FCIB_CHECK(nweights == kMlpNW, FCIB_ERR_ARG, "fcib_set_mlp: expected FCIB_MLP_NWEIGHTS weights");
        std::vector<float> w(weights, weights + nweights);
        for (float x : w) FCIB_CHECK(std::isfinite(x), FCIB_ERR_ARG, "fcib_set_mlp: non-finite weight");
        ctx->c.mlp_w.upload(w, ctx->c.stream);
        ctx->c.mlp_tables_ready = false;
        FCIB_CUDA(cudaStreamSynchronize(ctx->c.stream));
    });
}

int fcib_precondition(fcib_ctx* ctx, const double* r, double lambda, double* out) {
    if (!ctx || !r || !out) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        Context& c = ctx->c;
        ensure_setup(c);
        const int64_t nf = flat_size(c);
        double rn = 0.0;
        for (int64_t i = 0; i < nf; i++) rn += r[i] * r[i];
        rn = std::sqrt(rn);
        DBuf<double> d;
        d.alloc(c.nvec);
        upload_flat(c, r, d.p);
        k_diag_correction<<<4 * c.num_sms, 256, 0, c.stream>>>(d.p, c.hdiag.p, lambda, (size_t)c.nvec);
        FCIB_KCHECK();
        if (c.opt.preconditioner == FCIB_PRECOND_MLP) {
            std::vector<double> h((size_t)c.nvec);
            FCIB_CUDA(cudaMemcpyAsync(h.data(), d.p, sizeof(double) * c.nvec, cudaMemcpyDeviceToHost, c.stream));
            FCIB_CUDA(cudaStreamSynchronize(c.stream));
            double tn = 0.0;
            for (double x : h) tn += x * x;
            mlp_apply(c, d.p, lambda, rn, std::sqrt(tn));
        }
        download_flat(c, d.p, out);
    });
}

int fcib_mlp_eval(int device, int64_t n, const uint32_t* ea, const uint32_t* eb, const float* u, const float* r,
                  const float* weights, float* factor) {
    if (n < 0 || (n > 0 && (!ea || !eb || !u || !r || !weights || !factor))) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(nullptr, [&] {
        if (n == 0) return;
        FCIB_CUDA(cudaSetDevice(device));
        cudaStream_t s;
        FCIB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        try {
            DeviceSamples ds;
            ds.upload(n, ea, eb, u, r, nullptr, s);
            DBuf<float> w, f;
            w.alloc(kMlpNW);
            f.alloc(n);
            FCIB_CUDA(cudaMemcpyAsync(w.p, weights, 4 * kMlpNW, cudaMemcpyHostToDevice, s));
            SampleSource src{ds.ea.p, ds.eb.p, ds.u.p, ds.r.p, f.p};
            const size_t smem = sizeof(MlpSmem);
            FCIB_CUDA(cudaFuncSetAttribute(k_mlp_apply<SampleSource>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            const int grid = (int)std::min<int64_t>(1184, (n + 127) / 128);
            k_mlp_apply<SampleSource><<<grid, 256, smem, s>>>(src, (size_t)n, MlpDevice{w.p});
            FCIB_KCHECK();
            FCIB_CUDA(cudaMemcpyAsync(factor, f.p, 4 * n, cudaMemcpyDeviceToHost, s));
            FCIB_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            cudaStreamDestroy(s);
            throw;
        }
        cudaStreamDestroy(s);
    });
}

int fcib_mlp_grad(int device, int64_t n, const uint32_t* ea, const uint32_t* eb, const float* u, const float* r,
                  const float* tgt, const float* wgt, const float* weights, float* grad, double* loss) {
    if (n <= 0 || !ea || !eb || !u || !r || !tgt || !weights || !grad || !loss) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(nullptr, [&] {
        FCIB_CHECK(n <= (int64_t)1 << 30, FCIB_ERR_UNSUPPORTED, "fcib_mlp_grad: too many samples");
        FCIB_CUDA(cudaSetDevice(device));
        cudaStream_t s;
        FCIB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        try {
            DeviceSamples ds;
            ds.upload(n, ea, eb, u, r, tgt, s, wgt);
            std::vector<int> hidx(n);
            for (int64_t i = 0; i < n; i++) hidx[i] = (int)i;
            DBuf<int> idx;
            idx.upload(hidx, s);
            DBuf<float> w, g;
            w.alloc(kMlpNW);
            g.alloc(kMlpNW);
            DBuf<double> l;
            l.alloc(1);
            FCIB_CUDA(cudaMemcpyAsync(w.p, weights, 4 * kMlpNW, cudaMemcpyHostToDevice, s));
            FCIB_CUDA(cudaMemsetAsync(g.p, 0, 4 * kMlpNW, s));
            FCIB_CUDA(cudaMemsetAsync(l.p, 0, 8, s));
            launch_grad(ds, idx.p, (int)n, w.p, g.p, l.p, 1.0f / (float)n, s);
            FCIB_CUDA(cudaMemcpyAsync(grad, g.p, 4 * kMlpNW, cudaMemcpyDeviceToHost, s));
            FCIB_CUDA(cudaMemcpyAsync(loss, l.p, 8, cudaMemcpyDeviceToHost, s));
            FCIB_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            cudaStreamDestroy(s);
            throw;
        }
        cudaStreamDestroy(s);
    });
}

int fcib_mlp_train(int device, int64_t n, const uint32_t* ea, const uint32_t* eb, const float* u, const float* r,
                   const float* tgt, const float* wgt, int epochs, int batch, float lr, uint64_t seed, int init,
                   float* weights, double* epoch_loss) {
    if (n <= 0 || !ea || !eb || !u || !r || !tgt || !weights) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(nullptr, [&] {
        FCIB_CHECK(epochs >= 1 && batch >= kGradSB && lr > 0.0f, FCIB_ERR_ARG, "fcib_mlp_train: bad epochs/batch/lr");
        FCIB_CHECK(n <= (int64_t)1 << 30, FCIB_ERR_UNSUPPORTED, "fcib_mlp_train: too many samples");
        FCIB_CUDA(cudaSetDevice(device));
        cudaStream_t s;
        FCIB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        try {
            std::vector<float> hw(weights, weights + kMlpNW);
            if (init) mlp_init(hw, seed);
            DeviceSamples ds;
            ds.upload(n, ea, eb, u, r, tgt, s, wgt);
            DBuf<float> w, g, m1, m2;
            w.upload(hw, s);
            g.alloc(kMlpNW);
            m1.alloc(kMlpNW);
            m2.alloc(kMlpNW);
            FCIB_CUDA(cudaMemsetAsync(m1.p, 0, 4 * kMlpNW, s));
            FCIB_CUDA(cudaMemsetAsync(m2.p, 0, 4 * kMlpNW, s));
            DBuf<double> l;
            l.alloc(1);
            DBuf<int> idx;
            std::vector<int> perm(n);
            for (int64_t i = 0; i < n; i++) perm[i] = (int)i;
            std::mt19937_64 rng(seed ^ 0x9E3779B97F4A7C15ull);
            int step = 0;
            for (int ep = 0; ep < epochs; ep++) {
                std::shuffle(perm.begin(), perm.end(), rng);
                idx.upload(perm, s);
                FCIB_CUDA(cudaMemsetAsync(l.p, 0, 8, s));
                for (int64_t b0 = 0; b0 + batch <= n || b0 == 0; b0 += batch) {
                    const int cnt = (int)std::min<int64_t>(batch, n - b0);
                    FCIB_CUDA(cudaMemsetAsync(g.p, 0, 4 * kMlpNW, s));
                    launch_grad(ds, idx.p + b0, cnt, w.p, g.p, l.p, 1.0f / (float)cnt, s);
                    step++;
                    const float c1 = 1.0f / (1.0f - std::pow(0.9f, (float)step));
                    const float c2 = 1.0f / (1.0f - std::pow(0.999f, (float)step));
                    k_adam<<<(kMlpNW + 255) / 256, 256, 0, s>>>(w.p, m1.p, m2.p, g.p, kMlpNW, lr, c1, c2);
                    FCIB_KCHECK();
                    if (cnt < batch) break;
                }
                double el = 0.0;
                FCIB_CUDA(cudaMemcpyAsync(&el, l.p, 8, cudaMemcpyDeviceToHost, s));
                FCIB_CUDA(cudaStreamSynchronize(s));
                if (epoch_loss) epoch_loss[ep] = el / std::max<int64_t>(1, n / batch);
            }
            FCIB_CUDA(cudaMemcpyAsync(weights, w.p, 4 * kMlpNW, cudaMemcpyDeviceToHost, s));
            FCIB_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            cudaStreamDestroy(s);
            throw;
        }
        cudaStreamDestroy(s);
    });
}

}  // extern "C"
