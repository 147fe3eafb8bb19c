// Davidson-Liu on the device (FP64 vectors in HBM, small subspace algebra on the host).
//
// Follows DavidsonLiuSolver::solve (forte/helpers/davidson_liu_solver.cc:180-273): sigma of
// new basis vectors, subspace Hamiltonian G = b sigma^T (symmetrised) and its
// diagonalisation, residuals r_k = sum_j alpha_jk (sigma_j - lambda_k b_j), diagonal
// preconditioner r/(lambda - H_II) zeroed when |lambda - H_II| <= 1e-6, projection of
// unwanted roots, normalisation, convergence on |delta lambda| and ||r||, collapse, and
// Gram-Schmidt with the reference's discard (1e-7) and orthogonality (1e-12) thresholds.
// G is updated incrementally (new rows/columns only) instead of the full b sigma^T GEMM of
// every iteration; after a collapse it is rebuilt from the collapsed vectors.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <stdexcept>

#include "fcib_internal.h"
#include "guess.h"

namespace fcib {

constexpr int kRedThreads = 256;
constexpr int kMaxIn = 64;     // input vectors per fused pass
constexpr int kMaxOut = 4;     // output vectors per fused pass
constexpr int kSlots = 2 * kMaxOut + kMaxIn + 1;  // partial sums per block

// d_j = V_j . (sel_j ? x1 : x0) for j < nv, plus x0 . x0 when self != 0 (slot kMaxIn)
struct DotArgs {
    const double* v[kMaxIn];
    unsigned long long sel;
    int nv, self;
    const double* x0;
    const double* x1;
};

template <int NV>
__global__ void __launch_bounds__(kRedThreads) k_dots(DotArgs a, size_t N, double* __restrict__ partial) {
    double acc[NV + 1];
#pragma unroll
    for (int j = 0; j <= NV; j++) acc[j] = 0.0;
    const size_t G = (size_t)gridDim.x * blockDim.x;
    size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    // four elements per thread per step, all loads issued before the FMAs
    for (; I + 3 * G < N; I += 4 * G) {
        double x0[4], x1[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            x0[u] = a.x0[I + u * G];
            x1[u] = a.x1 ? a.x1[I + u * G] : 0.0;
        }
#pragma unroll
        for (int j = 0; j < NV; j++) {
            if (j < a.nv) {
                double v[4];
#pragma unroll
                for (int u = 0; u < 4; u++) v[u] = a.v[j][I + u * G];
                const bool s1 = (a.sel >> j) & 1ull;
#pragma unroll
                for (int u = 0; u < 4; u++) acc[j] = fma(v[u], s1 ? x1[u] : x0[u], acc[j]);
            }
        }
        if (a.self)
#pragma unroll
            for (int u = 0; u < 4; u++) acc[NV] = fma(x0[u], x0[u], acc[NV]);
    }
    for (; I < N; I += G) {
        double x0 = a.x0[I];
        double x1 = a.x1 ? a.x1[I] : 0.0;
#pragma unroll
        for (int j = 0; j < NV; j++)
            if (j < a.nv) acc[j] = fma(a.v[j][I], ((a.sel >> j) & 1ull) ? x1 : x0, acc[j]);
        if (a.self) acc[NV] = fma(x0, x0, acc[NV]);
    }
    __shared__ double red[kRedThreads / 32][NV + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j <= NV; j++) {
        if (j < a.nv || (j == NV && a.self)) {
            double v = acc[j];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) red[warp][j] = v;
        }
    }
    __syncthreads();
    for (int j = threadIdx.x; j <= NV; j += blockDim.x) {
        if (j < a.nv || (j == NV && a.self)) {
            double t = 0.0;
            for (int w = 0; w < kRedThreads / 32; w++) t += red[w][j];
            partial[(size_t)blockIdx.x * kSlots + (j < NV ? j : kMaxIn)] = t;
        }
    }
}

// out_k = beta*out_k + sum_j coef[k][j] V_j (k < nout); optional diagonal preconditioning
// corr_k = out_k / (lambda_k - hd) (0 when |lambda_k - hd| <= 1e-6) written instead of out_k.
// partial slots: 2k = out_k.out_k (before preconditioning), 2k+1 = corr_k.corr_k
struct ComboArgs {
    const double* v[kMaxIn];
    double coef[kMaxOut][kMaxIn];
    double* out[kMaxOut];
    double lambda[kMaxOut];
    const double* hd;
    int nv, nout, precond;
    double beta;
};

template <int NV, int NO>
__device__ __forceinline__ void combo_elem(const ComboArgs& a, size_t I, double hd, double (&acc)[2 * NO],
                                           const double (&o)[NO]) {
#pragma unroll
    for (int k = 0; k < NO; k++) {
        if (k < a.nout) {
            acc[2 * k] = fma(o[k], o[k], acc[2 * k]);
            double w = o[k];
            if (a.precond) {
                double den = a.lambda[k] - hd;
                w = (fabs(den) > 1.0e-6) ? o[k] / den : 0.0;
            }
            a.out[k][I] = w;
            acc[2 * k + 1] = fma(w, w, acc[2 * k + 1]);
        }
    }
}

template <int NV, int NO>
__global__ void __launch_bounds__(kRedThreads) k_combo(ComboArgs a, size_t N, double* __restrict__ partial) {
    double acc[2 * NO];
#pragma unroll
    for (int k = 0; k < 2 * NO; k++) acc[k] = 0.0;
    const size_t G = (size_t)gridDim.x * blockDim.x;
    size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    for (; I + 3 * G < N; I += 4 * G) {
        double o[4][NO];
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
            for (int k = 0; k < NO; k++) o[u][k] = (k < a.nout && a.beta != 0.0) ? a.beta * a.out[k][I + u * G] : 0.0;
#pragma unroll
        for (int j = 0; j < NV; j++) {
            if (j < a.nv) {
                double v[4];
#pragma unroll
                for (int u = 0; u < 4; u++) v[u] = a.v[j][I + u * G];
#pragma unroll
                for (int u = 0; u < 4; u++)
#pragma unroll
                    for (int k = 0; k < NO; k++) o[u][k] = fma(a.coef[k][j], v[u], o[u][k]);
            }
        }
        double hd[4];
#pragma unroll
        for (int u = 0; u < 4; u++) hd[u] = a.precond ? a.hd[I + u * G] : 0.0;
#pragma unroll
        for (int u = 0; u < 4; u++) combo_elem<NV, NO>(a, I + u * G, hd[u], acc, o[u]);
    }
    for (; I < N; I += G) {
        double o[NO];
#pragma unroll
        for (int k = 0; k < NO; k++) o[k] = (k < a.nout && a.beta != 0.0) ? a.beta * a.out[k][I] : 0.0;
#pragma unroll
        for (int j = 0; j < NV; j++) {
            if (j < a.nv) {
                double v = a.v[j][I];
#pragma unroll
                for (int k = 0; k < NO; k++) o[k] = fma(a.coef[k][j], v, o[k]);
            }
        }
        combo_elem<NV, NO>(a, I, a.precond ? a.hd[I] : 0.0, acc, o);
    }
    __shared__ double red[kRedThreads / 32][2 * NO];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < 2 * NO; j++) {
        if (j < 2 * a.nout) {
            double v = acc[j];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) red[warp][j] = v;
        }
    }
    __syncthreads();
    for (int j = threadIdx.x; j < 2 * a.nout; j += blockDim.x) {
        double t = 0.0;
        for (int w = 0; w < kRedThreads / 32; w++) t += red[w][j];
        partial[(size_t)blockIdx.x * kSlots + j] = t;
    }
}

// Fused projection + check: out = rho * (a * x - sum_j coef_j V_j) and, in the same pass,
// partial sums of V_j . out (slots j < nv) and out . out (slot kMaxIn).  out may alias x.
struct OrthArgs {
    const double* v[kMaxIn];
    double coef[kMaxIn];
    const double* x;
    double* out;
    double a, rho;
    int nv;
};

template <int NV>
__global__ void __launch_bounds__(kRedThreads) k_orth(OrthArgs a, size_t N, double* __restrict__ partial) {
    double acc[NV + 1];
#pragma unroll
    for (int j = 0; j <= NV; j++) acc[j] = 0.0;
    const size_t G = (size_t)gridDim.x * blockDim.x;
    size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    for (; I + G < N; I += 2 * G) {
        double o[2];
#pragma unroll
        for (int u = 0; u < 2; u++) o[u] = a.a * a.x[I + u * G];
#pragma unroll
        for (int j = 0; j < NV; j++)
            if (j < a.nv)
#pragma unroll
                for (int u = 0; u < 2; u++) o[u] = fma(-a.coef[j], a.v[j][I + u * G], o[u]);
#pragma unroll
        for (int u = 0; u < 2; u++) {
            o[u] *= a.rho;
            a.out[I + u * G] = o[u];
            acc[NV] = fma(o[u], o[u], acc[NV]);
        }
        // the V_j elements were just read: these loads hit L1
#pragma unroll
        for (int j = 0; j < NV; j++)
            if (j < a.nv)
#pragma unroll
                for (int u = 0; u < 2; u++) acc[j] = fma(a.v[j][I + u * G], o[u], acc[j]);
    }
    for (; I < N; I += G) {
        double o = a.a * a.x[I];
#pragma unroll
        for (int j = 0; j < NV; j++)
            if (j < a.nv) o = fma(-a.coef[j], a.v[j][I], o);
        o *= a.rho;
        a.out[I] = o;
        acc[NV] = fma(o, o, acc[NV]);
#pragma unroll
        for (int j = 0; j < NV; j++)
            if (j < a.nv) acc[j] = fma(a.v[j][I], o, acc[j]);
    }
    __shared__ double red[kRedThreads / 32][NV + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j <= NV; j++) {
        if (j < a.nv || j == NV) {
            double v = acc[j];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) red[warp][j] = v;
        }
    }
    __syncthreads();
    for (int j = threadIdx.x; j <= NV; j += blockDim.x) {
        if (j < a.nv || j == NV) {
            double t = 0.0;
            for (int w = 0; w < kRedThreads / 32; w++) t += red[w][j];
            partial[(size_t)blockIdx.x * kSlots + (j < NV ? j : kMaxIn)] = t;
        }
    }
}

// out[j] = sum_b partial[b][j] for j < nslots (one block per slot, deterministic order)
__global__ void k_final_reduce(const double* __restrict__ partial, int nblocks, double* __restrict__ out) {
    const int j = blockIdx.x;
    double s = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += partial[(size_t)b * kSlots + j];
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)blockDim.x / 32; w++) t += red[w];
        out[j] = t;
    }
}

__global__ void k_scale(double* __restrict__ v, double a, size_t N) {
    for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < N; I += (size_t)gridDim.x * blockDim.x) v[I] *= a;
}

// v[I] += scale * u(I) with u uniform in [-1, 1) from a counter-based hash of (seed, I)
__global__ void k_add_random(double* __restrict__ v, size_t N, unsigned long long seed, double scale) {
    for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < N; I += (size_t)gridDim.x * blockDim.x) {
        unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (I + 1);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        v[I] += scale * ((double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0);
    }
}

__global__ void k_fill_sparse(double* __restrict__ v, const int64_t* __restrict__ idx, const double* __restrict__ val, int cnt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < cnt) v[idx[i]] = val[i];
}

// v -= (v . u_b) u_b for the sparse vectors u_0, u_1, ... in order (one block; entries of u_b at
// off[b] .. off[b + 1] of idx/val)
__global__ void k_project_sparse(double* __restrict__ v, const int64_t* __restrict__ idx, const double* __restrict__ val,
                                 const int* __restrict__ off, int nb) {
    __shared__ double red[32];
    for (int b = 0; b < nb; b++) {
        const int o0 = off[b], cnt = off[b + 1] - o0;
        double s = 0.0;
        for (int i = threadIdx.x; i < cnt; i += blockDim.x) s = fma(v[idx[o0 + i]], val[o0 + i], s);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < (int)(blockDim.x + 31) / 32; w++) t += red[w];
            red[0] = t;
        }
        __syncthreads();
        double ov = red[0];
        __syncthreads();
        for (int i = threadIdx.x; i < cnt; i += blockDim.x) v[idx[o0 + i]] -= ov * val[o0 + i];
        __syncthreads();  // the next vector's dot reads these updates
    }
}

// ------------------------------------------------------------------------------------------
// top-k of the diagonal: radix select on order-preserving 64-bit keys, 8 bits per pass
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ uint64_t dkey(double d) {
    uint64_t u = __double_as_longlong(d);
    return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}

__global__ void k_radix_hist(const double* __restrict__ hd, const uint8_t* __restrict__ mask, size_t N,
                             uint64_t prefix, uint64_t pmask, int shift, unsigned int* __restrict__ hist) {
    __shared__ unsigned int h[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < N; I += (size_t)gridDim.x * blockDim.x) {
        if (mask && !mask[I]) continue;
        uint64_t k = dkey(hd[I]);
        if ((k & pmask) == prefix) atomicAdd(&h[(k >> shift) & 255], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (h[i]) atomicAdd(&hist[i], h[i]);
}

__global__ void k_collect_le(const double* __restrict__ hd, const uint8_t* __restrict__ mask, size_t N,
                             uint64_t thr, int cap, int* __restrict__ count, double* __restrict__ ev,
                             int64_t* __restrict__ ei) {
    for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < N; I += (size_t)gridDim.x * blockDim.x) {
        if (mask && !mask[I]) continue;
        double e = hd[I];
        if (dkey(e) <= thr) {
            int s = atomicAdd(count, 1);
            if (s < cap) {
                ev[s] = e;
                ei[s] = (int64_t)I;
            }
        }
    }
}

// ------------------------------------------------------------------------------------------
// <S^2> = -sum_rs <E^a_sr E^b_rs> + (na-nb)^2/4 + (na+nb)/2  (forte/fci/fci_vector_spin2.cc:38-75)
// per determinant: doubly occupied orbitals (r = s) and alpha/beta open-shell swaps.
// ------------------------------------------------------------------------------------------

// C in the engine layout: C1 (sd.on = 0, nas * nbs elements) or the blocked layout of sd (N elements)
__global__ void __launch_bounds__(kRedThreads) k_spin2(const double* __restrict__ C, const uint32_t* __restrict__ sa,
                                                       const uint32_t* __restrict__ sb, int nas, int nbs, int n,
                                                       double* __restrict__ partial, SymDev sd, size_t N) {
    double acc = 0.0;
    const bool blocked = sd.on;
    if (!blocked) N = (size_t)nas * nbs;
    for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < N; I += (size_t)gridDim.x * blockDim.x) {
        double ci = C[I];
        if (ci == 0.0) continue;
        int ia, ib;
        if (blocked) {
            sym_decode(sd, (int64_t)I, ia, ib);
        } else {
            ia = (int)(I / nbs);
            ib = (int)(I % nbs);
        }
        uint32_t Ia = sa[ia], Ib = sb[ib];
        double t = (double)__popc(Ia & Ib) * ci;
        uint32_t oa = Ia & ~Ib, ob = Ib & ~Ia;
        // alpha electron s -> r and beta electron r -> s with s in oa, r in ob
        for (uint32_t xs = oa; xs; xs &= xs - 1) {
            int s = __ffs(xs) - 1;
            for (uint32_t xr = ob; xr; xr &= xr - 1) {
                int r = __ffs(xr) - 1;
                uint32_t Ja = (Ia & ~(1u << s)) | (1u << r);
                uint32_t Jb = (Ib & ~(1u << r)) | (1u << s);
                int lo = r < s ? r : s, hi = r < s ? s : r;
                uint32_t m = (hi - lo < 2) ? 0u : (((1u << hi) - 1u) & ~((2u << lo) - 1u));
                int par = (__popc(Ia & m) + __popc(Ib & m)) & 1;
                const int ja = (int)d_rank(Ja, n), jb = (int)d_rank(Jb, n);
                // blocked: a swap may leave the kept strings of a GAS layout (no such determinant there)
                const int64_t J = blocked ? sym_encode_kept(sd, Ja, ja, jb) : (int64_t)ja * nbs + jb;
                if (J < 0) continue;
                const double cj = C[J];
                t += par ? -cj : cj;
            }
        }
        acc = fma(ci, t, acc);
    }
    __shared__ double red[kRedThreads / 32];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kRedThreads / 32; w++) s += red[w];
        partial[(size_t)blockIdx.x * kSlots] = s;
    }
}

// ------------------------------------------------------------------------------------------
// host helpers
// ------------------------------------------------------------------------------------------
struct Ops {
    Context& c;
    size_t N;
    const double* hd;  // diagonal of the preconditioner
    int nblk;
    DBuf<double> partial, out;
    std::vector<double> hout;
    explicit Ops(Context& cc) : Ops(cc, (size_t)cc.nvec, cc.hdiag.p) {}
    Ops(Context& cc, size_t n, const double* diag) : c(cc), hd(diag) {
        N = n;
        nblk = std::max(1, std::min(4 * c.num_sms, (int)((N + kRedThreads - 1) / kRedThreads)));
        partial.alloc((size_t)nblk * kSlots);
        out.alloc(kSlots);
        hout.resize(kSlots);
    }
    void fetch(int nslots) {
        k_final_reduce<<<nslots, 256, 0, c.stream>>>(partial.p, nblk, out.p);
        FCIB_KCHECK();
        FCIB_CUDA(cudaMemcpyAsync(hout.data(), out.p, sizeof(double) * nslots, cudaMemcpyDeviceToHost, c.stream));
        FCIB_CUDA(cudaStreamSynchronize(c.stream));
    }
    // d[j] = V[j] . (sel[j] ? x1 : x0); optionally *self = x0 . x0
    void dots(const std::vector<const double*>& V, const std::vector<int>& sel, const double* x0, const double* x1,
              std::vector<double>& d, double* self = nullptr) {
        d.assign(V.size(), 0.0);
        size_t done = 0;
        bool first = true;
        while (first || done < V.size()) {
            DotArgs a;
            int nv = (int)std::min<size_t>(kMaxIn, V.size() - done);
            a.sel = 0;
            for (int j = 0; j < nv; j++) {
                a.v[j] = V[done + j];
                if (!sel.empty() && sel[done + j]) a.sel |= 1ull << j;
            }
            a.nv = nv;
            a.self = (self && first) ? 1 : 0;
            a.x0 = x0;
            a.x1 = x1;
            if (nv <= 8) k_dots<8><<<nblk, kRedThreads, 0, c.stream>>>(a, N, partial.p);
            else if (nv <= 16) k_dots<16><<<nblk, kRedThreads, 0, c.stream>>>(a, N, partial.p);
            else if (nv <= 32) k_dots<32><<<nblk, kRedThreads, 0, c.stream>>>(a, N, partial.p);
            else k_dots<64><<<nblk, kRedThreads, 0, c.stream>>>(a, N, partial.p);
            FCIB_KCHECK();
            fetch(kMaxIn + 1);
            for (int j = 0; j < nv; j++) d[done + j] = hout[j];
            if (a.self) *self = hout[kMaxIn];
            done += nv;
            first = false;
        }
    }
    // out = rho * (a * x - sum_j coef[j] V[j]) with d[j] = V[j] . out and *self = out . out, one
    // pass (V.size() <= kMaxIn)
    void orth(const std::vector<const double*>& V, const std::vector<double>& coef, const double* x, double a_x,
              double rho, double* out, std::vector<double>& d, double* self) {
        FCIB_CHECK(V.size() <= (size_t)kMaxIn, FCIB_ERR_UNSUPPORTED, "subspace larger than 64 vectors");
        OrthArgs a;
        const int nv = (int)V.size();
        for (int j = 0; j < nv; j++) {
            a.v[j] = V[j];
            a.coef[j] = coef[j];
        }
        a.x = x;
        a.out = out;
        a.a = a_x;
        a.rho = rho;
        a.nv = nv;
        if (nv <= 8) k_orth<8><<<nblk, kRedThreads, 0, c.stream>>>(a, N, partial.p);
        else if (nv <= 16) k_orth<16><<<nblk, kRedThreads, 0, c.stream>>>(a, N, partial.p);
        else if (nv <= 32) k_orth<32><<<nblk, kRedThreads, 0, c.stream>>>(a, N, partial.p);
        else k_orth<64><<<nblk, kRedThreads, 0, c.stream>>>(a, N, partial.p);
        FCIB_KCHECK();
        fetch(kMaxIn + 1);
        d.assign(hout.begin(), hout.begin() + nv);
        *self = hout[kMaxIn];
    }
    double norm2(const double* x) {
        std::vector<double> d;
        double s = 0.0;
        dots({}, {}, x, nullptr, d, &s);
        return s;
    }
    // outs[k] = beta*outs[k] + sum_j coef[k][j] V[j];  optional diagonal preconditioning with
    // lambda[k].  Returns (out.out, corr.corr) per output of the last chunk.
    std::vector<std::pair<double, double>> combo(const std::vector<const double*>& V,
                                                 const std::vector<std::vector<double>>& coef,
                                                 const std::vector<double*>& outs, double beta,
                                                 const double* lambda = nullptr) {
        const int nout_all = (int)outs.size();
        std::vector<std::pair<double, double>> res(nout_all, {0.0, 0.0});
        for (int k0 = 0; k0 < nout_all; k0 += kMaxOut) {
            int nout = std::min(kMaxOut, nout_all - k0);
            size_t done = 0;
            do {
                ComboArgs a;
                int nv = (int)std::min<size_t>(kMaxIn, V.size() - done);
                bool last = done + nv >= V.size();
                for (int j = 0; j < nv; j++) a.v[j] = V[done + j];
                for (int k = 0; k < nout; k++) {
                    for (int j = 0; j < nv; j++) a.coef[k][j] = coef[k0 + k][done + j];
                    a.out[k] = outs[k0 + k];
                    a.lambda[k] = lambda ? lambda[k0 + k] : 0.0;
                }
                a.hd = hd;
                a.nv = nv;
                a.nout = nout;
                a.precond = (lambda && last) ? 1 : 0;
                a.beta = (done == 0) ? beta : 1.0;
#define FCIB_COMBO(NVv, NOv) k_combo<NVv, NOv><<<nblk, kRedThreads, 0, c.stream>>>(a, N, partial.p)
                if (nout == 1) {
                    if (nv <= 8) FCIB_COMBO(8, 1); else if (nv <= 16) FCIB_COMBO(16, 1);
                    else if (nv <= 32) FCIB_COMBO(32, 1); else FCIB_COMBO(64, 1);
                } else if (nout == 2) {
                    if (nv <= 8) FCIB_COMBO(8, 2); else if (nv <= 16) FCIB_COMBO(16, 2);
                    else if (nv <= 32) FCIB_COMBO(32, 2); else FCIB_COMBO(64, 2);
                } else {
                    if (nv <= 8) FCIB_COMBO(8, 4); else if (nv <= 16) FCIB_COMBO(16, 4);
                    else if (nv <= 32) FCIB_COMBO(32, 4); else FCIB_COMBO(64, 4);
                }
#undef FCIB_COMBO
                FCIB_KCHECK();
                done += nv;
                if (last) {
                    fetch(2 * nout);
                    for (int k = 0; k < nout; k++) res[k0 + k] = {hout[2 * k], hout[2 * k + 1]};
                }
            } while (done < V.size());
        }
        return res;
    }
    void scale(double* v, double a) {
        k_scale<<<nblk, kRedThreads, 0, c.stream>>>(v, a, N);
        FCIB_KCHECK();
    }
    void copy(double* dst, const double* src) {
        FCIB_CUDA(cudaMemcpyAsync(dst, src, N * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
    }
};

struct SparseDev {
    DBuf<int64_t> idx;
    DBuf<double> val;
    int cnt = 0;
};
// the unwanted roots of the guess, packed: root b holds entries off[b] .. off[b + 1]
struct BadRoots {
    DBuf<int64_t> idx;
    DBuf<double> val;
    DBuf<int> off;
    int nb = 0;
    bool empty() const { return nb == 0; }
};

// add_row_and_orthonormalize (davidson_liu_solver.cc:634-687): A[rowsA] <- s*src Gram-Schmidt
// orthonormalised against A[0..rowsA); false if discarded (norm < 1e-7 after projection).
// Classical Gram-Schmidt with the reference's thresholds.  After one dots pass, each projection
// is one fused pass that also returns the dots of the result with A and its norm (k_orth): the
// result is scaled by the norm predicted from the dots, and the exact sums decide between
// accept (orthogonal to 1e-12 and unit norm to 1e-12), discard (projected norm < 1e-7), a
// corrective projection or a rescale.
static bool add_row_orth(Ops& ops, std::vector<double*>& A, int rowsA, const double* src, double s = 1.0) {
    double* w = A[rowsA];
    std::vector<const double*> B(A.begin(), A.begin() + rowsA);
    std::vector<double> d;
    double vv = 0.0;
    ops.dots(B, {}, src, nullptr, d, &vv);
    // first projection: w = rho * s * (src - sum d_i B_i), rho from the predicted norm
    std::vector<double> coef(rowsA);
    for (int i = 0; i < rowsA; i++) coef[i] = s * d[i];
    double p2 = vv;
    for (int i = 0; i < rowsA; i++) p2 -= d[i] * d[i];
    double rho = (p2 > 0.0 && s != 0.0) ? 1.0 / (std::fabs(s) * std::sqrt(p2)) : 1.0;
    const double* in = src;
    double a_in = s;
    for (int cycle = 0; cycle < 10; cycle++) {
        std::vector<double> dw;
        double ww = 0.0;
        ops.orth(B, coef, in, a_in, rho, w, dw, &ww);
        const double nw = std::sqrt(ww);
        if (!(nw / rho >= 1.0e-7)) return false;  // projected norm (also rejects NaN)
        double mo = 0.0;
        for (int i = 0; i < rowsA; i++) mo = std::max(mo, std::fabs(dw[i] / nw));
        if (mo < 1.0e-12) {
            if (std::fabs(ww - 1.0) >= 1.0e-12) ops.scale(w, 1.0 / nw);
            return true;
        }
        // re-orthogonalise: w <- (w - sum dw_i B_i) / ||.||, norm predicted from the sums
        double q2 = ww;
        for (int i = 0; i < rowsA; i++) q2 -= dw[i] * dw[i];
        for (int i = 0; i < rowsA; i++) coef[i] = dw[i];
        in = w;
        a_in = 1.0;
        rho = q2 > 0.0 ? 1.0 / std::sqrt(q2) : 1.0 / nw;
    }
    return false;
}

static int add_rows_orth(Ops& ops, std::vector<double*>& A, int rowsA, const std::vector<double*>& Bv, int rowsB,
                         const std::vector<double>* scales = nullptr) {
    int added = 0;
    for (int j = 0; j < rowsB; j++)
        if (add_row_orth(ops, A, rowsA + added, Bv[j], scales ? (*scales)[j] : 1.0)) added++;
    return added;
}

static void project_out(Context& c, BadRoots& bad, std::vector<double*>& V, int nvec) {
    if (bad.empty()) return;
    for (int k = 0; k < nvec; k++) {
        k_project_sparse<<<1, 256, 0, c.stream>>>(V[k], bad.idx.p, bad.val.p, bad.off.p, bad.nb);
        FCIB_KCHECK();
    }
}

const double* root_vector(Context& c, int root) {
    return c.roots_in_evdet ? c.evdet.p + (size_t)root * c.nvec : c.b.p + (size_t)root * c.nvec;
}

double spin2_device(Context& c, const double* C) {
    Ops ops(c);
    k_spin2<<<ops.nblk, kRedThreads, 0, c.stream>>>(C, c.A.str.p, c.B.str.p, (int)c.nas, (int)c.nbs, c.n, ops.partial.p,
                                                    sym_dev(c), (size_t)c.nvec);
    FCIB_KCHECK();
    ops.fetch(1);
    double s = ops.hout[0];
    double na = c.na, nb = c.nb;
    return -s + 0.25 * (na - nb) * (na - nb) + 0.5 * (na + nb);
}

// lowest `count` diagonal entries ordered by (value, address), like the insertion list of
// FCISolver::initial_guess_generate_dets (fci_solver_initial_guess.cc:44-69)
// the `count` smallest keys[] of the determinants in the target irrep with their C1 indices, sorted by
// (key, index); ties at the boundary are resolved by the index
std::vector<std::pair<double, int64_t>> lowest_keys(Context& c, const double* keys, int count) {
    return lowest_keys(c, keys, count, (size_t)c.nvec, c.mask.p);
}
std::vector<std::pair<double, int64_t>> lowest_keys(Context& c, const double* keys, int count, size_t N,
                                                    const uint8_t* mask) {
    DBuf<unsigned int> hist;
    hist.alloc(256);
    uint64_t prefix = 0, pmask = 0;
    uint64_t need = count;
    int grid = 4 * c.num_sms;
    for (int shift = 56; shift >= 0; shift -= 8) {
        FCIB_CUDA(cudaMemsetAsync(hist.p, 0, 256 * sizeof(unsigned int), c.stream));
        k_radix_hist<<<grid, 256, 0, c.stream>>>(keys, mask, N, prefix, pmask, shift, hist.p);
        FCIB_KCHECK();
        unsigned int h[256];
        FCIB_CUDA(cudaMemcpyAsync(h, hist.p, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
        FCIB_CUDA(cudaStreamSynchronize(c.stream));
        uint64_t cum = 0;
        int bin = 255;
        for (int i = 0; i < 256; i++) {
            if (cum + h[i] >= need) { bin = i; break; }
            cum += h[i];
        }
        need -= cum;
        prefix |= (uint64_t)bin << shift;
        pmask |= 255ull << shift;
    }
    // prefix is now the key of the count-th smallest entry; collect all keys <= it
    int cap = count + 65536;
    DBuf<int> cnt;
    DBuf<double> ev;
    DBuf<int64_t> ei;
    cnt.alloc(1);
    ev.alloc(cap);
    ei.alloc(cap);
    FCIB_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int), c.stream));
    k_collect_le<<<grid, 256, 0, c.stream>>>(keys, mask, N, prefix, cap, cnt.p, ev.p, ei.p);
    FCIB_KCHECK();
    int hc = 0;
    FCIB_CUDA(cudaMemcpyAsync(&hc, cnt.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    FCIB_CUDA(cudaStreamSynchronize(c.stream));
    FCIB_CHECK(hc <= cap, FCIB_ERR_NUMERIC, "too many degenerate entries for the lowest-k selection");
    std::vector<double> he(hc);
    std::vector<int64_t> hi(hc);
    FCIB_CUDA(cudaMemcpy(he.data(), ev.p, sizeof(double) * hc, cudaMemcpyDeviceToHost));
    FCIB_CUDA(cudaMemcpy(hi.data(), ei.p, sizeof(int64_t) * hc, cudaMemcpyDeviceToHost));
    std::vector<std::pair<double, int64_t>> v(hc);
    for (int i = 0; i < hc; i++) v[i] = {he[i], hi[i]};
    std::sort(v.begin(), v.end());
    if ((int)v.size() > count) v.resize(count);
    return v;
}
static std::vector<std::pair<double, int64_t>> lowest_diagonal(Context& c, int count) {
    return lowest_keys(c, c.hdiag.p, count);
}

// out[i] = in[idx[i]] and out[idx[i]] = in[i] (flat order <-> engine layout)
__global__ void k_gather_idx(double* __restrict__ out, const double* __restrict__ in, const int64_t* __restrict__ idx,
                             size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = in[idx[i]];
}
__global__ void k_scatter_idx(double* __restrict__ out, const double* __restrict__ in, const int64_t* __restrict__ idx,
                              size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[idx[i]] = in[i];
}
static void gather_flat(Context& c, const double* layout, double* flat) {
    const size_t nf = c.flat_map.size();
    k_gather_idx<<<(int)std::min<size_t>((nf + 255) / 256, 8 * (size_t)c.num_sms), 256, 0, c.stream>>>(
        flat, layout, c.flat_map_d.p, nf);
    FCIB_KCHECK();
}
static void scatter_flat(Context& c, const double* flat, double* layout) {
    const size_t nf = c.flat_map.size();
    k_scatter_idx<<<(int)std::min<size_t>((nf + 255) / 256, 8 * (size_t)c.num_sms), 256, 0, c.stream>>>(
        layout, flat, c.flat_map_d.p, nf);
    FCIB_KCHECK();
}

__global__ void k_neg_abs(const double* __restrict__ x, double* __restrict__ out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = -fabs(x[i]);
}

static double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Precision of the sigma build for a new basis vector in each solver phase.
enum class Phase { LowPrecision, Refine, FP64Only };

void dl_solve(Context& c) {
    // spin adaptation: the Davidson space is the CSF basis of the target multiplicity
    // (fci_solver.cc:186-262); otherwise the engine's determinant layout
    const bool csf_basis = c.opt.spin_adapt != 0;
    if (csf_basis) {
        FCIB_CHECK(c.opt.preconditioner != FCIB_PRECOND_MLP, FCIB_ERR_UNSUPPORTED,
                   "the learned preconditioner works in the determinant basis (not with spin adaptation)");
        ensure_csf(c);
        FCIB_CHECK(c.ncsf > 0, FCIB_ERR_ARG, "Found zero FCI guesses with the requested multiplicity.");
        c.hd_csf.alloc((size_t)c.ncsf);
        csf_hdiag(c, c.hd_csf.p);
        c.csf_x.alloc((size_t)c.nvec);
        c.csf_s.alloc((size_t)c.nvec);
    }
    // GAS spaces: the Davidson space is the GAS determinants themselves (GenCIVector flat order),
    // so the vector work follows them and not the layout's string products; sigma scatters its
    // input into the layout and gathers its output back.  The learned preconditioner and the
    // residual capture work on layout vectors, so they keep the layout.
    const bool gas_basis = !csf_basis && c.gas.ngas > 0 && c.opt.preconditioner != FCIB_PRECOND_MLP &&
                           c.capture_max == 0 && !c.flat_map.empty();
    if (gas_basis) {
        const size_t nf = c.flat_map.size();
        c.flat_map_d.upload(c.flat_map, c.stream);
        c.gas_x.alloc((size_t)c.nvec);
        FCIB_CUDA(cudaMemsetAsync(c.gas_x.p, 0, sizeof(double) * c.nvec, c.stream));  // scatters write GAS positions only
        c.gas_s.alloc((size_t)c.nvec);
        c.hd_gas.alloc(nf);
        gather_flat(c, c.hdiag.p, c.hd_gas.p);
    }
    const int64_t N = csf_basis ? c.ncsf : gas_basis ? (int64_t)c.flat_map.size() : c.nvec;
    int64_t Neff = N;
    if (!csf_basis && !gas_basis && c.mask.p) {
        std::vector<uint8_t> hm(N);
        FCIB_CUDA(cudaMemcpy(hm.data(), c.mask.p, N, cudaMemcpyDeviceToHost));
        Neff = 0;
        for (auto x : hm) Neff += x;
    }
    const fcib_options& o = c.opt;
    FCIB_CHECK(Neff > 0, FCIB_ERR_ARG, "DavidsonLiuSolver called with space of dimension zero.");
    FCIB_CHECK(c.nroot >= 1, FCIB_ERR_ARG, "DavidsonLiuSolver called with zero roots.");
    FCIB_CHECK(o.collapse_per_root >= 1, FCIB_ERR_ARG, "DavidsonLiuSolver: collapse_per_root must be >= 1");
    FCIB_CHECK(o.subspace_per_root >= o.collapse_per_root + 1, FCIB_ERR_ARG,
               "DavidsonLiuSolver: subspace_per_root must be >= collapse_per_root + 1");
    const int nroot = c.nroot;
    FCIB_CHECK(nroot <= kMaxOut * 8, FCIB_ERR_UNSUPPORTED, "too many roots");
    const int collapse = (int)std::min<int64_t>((int64_t)o.collapse_per_root * nroot, Neff);
    const int m = (int)std::min<int64_t>((int64_t)o.subspace_per_root * nroot, Neff);
    FCIB_CHECK(nroot <= m, FCIB_ERR_ARG, "more roots than determinants");
    FCIB_CHECK(2 * m <= kMaxIn * 4, FCIB_ERR_UNSUPPORTED, "Davidson subspace too large");
    c.subspace = m;
    c.b.alloc((size_t)m * N);
    c.sig.alloc((size_t)m * N);
    c.tmp.alloc((size_t)m * N);
    c.r.alloc((size_t)nroot * N);
    std::vector<double*> b(m), sg(m), tmp(m), r(nroot);
    for (int i = 0; i < m; i++) {
        b[i] = c.b.p + (size_t)i * N;
        sg[i] = c.sig.p + (size_t)i * N;
        tmp[i] = c.tmp.p + (size_t)i * N;
    }
    for (int k = 0; k < nroot; k++) r[k] = c.r.p + (size_t)k * N;
    Ops ops(c, (size_t)N, csf_basis ? c.hd_csf.p : gas_basis ? c.hd_gas.p : c.hdiag.p);
    // sigma of a vector of the Davidson space: in the CSF basis z -> P z -> H P z -> P^T H P z
    // (fci_solver.cc:247-254)
    auto space_sigma = [&](const double* bj, double* sj, int prec) {
        if (gas_basis) {
            scatter_flat(c, bj, c.gas_x.p);
            // only the GAS positions of the output are gathered, so the mask pass is skipped
            struct Unmasked {
                Context& c;
                explicit Unmasked(Context& cc) : c(cc) { c.sigma_unmasked = true; }
                ~Unmasked() { c.sigma_unmasked = false; }
            } guard(c);
            sigma_dispatch(c, c.gas_x.p, c.gas_s.p, prec);
            gather_flat(c, c.gas_s.p, sj);
            return;
        }
        if (!csf_basis) {
            sigma_dispatch(c, bj, sj, prec);
            return;
        }
        csf_to_det(c, bj, c.csf_x.p);
        sigma_dispatch(c, c.csf_x.p, c.csf_s.p, prec);
        det_to_csf(c, c.csf_s.p, sj);
    };
    cudaEvent_t ev_start, e0, e1;
    FCIB_CUDA(cudaEventCreate(&ev_start));
    FCIB_CUDA(cudaEventCreate(&e0));
    FCIB_CUDA(cudaEventCreate(&e1));
    FCIB_CUDA(cudaEventRecord(ev_start, c.stream));
    double t_start = now_ms();
    c.t_sigma_ms = 0.0;
    c.n_sigma = 0;
    c.n_sigma_fp64 = 0;
    c.t_ab_ms = c.t_same_ms = c.t_tc_ms = 0.0;
    c.n_ab = 0;
    c.t_ab64_ms = c.t_same64_ms = 0.0;
    c.n_ab64 = 0;
    c.trace.clear();

    // ---- initial guess, or restart from the previous solution ----
    // FCISolver::compute_energy (fci_solver.cc:205-233) keeps its Davidson-Liu solver between
    // calls and resets it with a fresh guess only on the first run or when the guess space
    // covers the whole space; otherwise DavidsonLiuSolver::setup_guesses (davidson_liu_solver.cc:
    // 312-316) restarts from the first nroot vectors, recomputing their sigma with the current
    // integrals, and keeps projecting out the first run's unwanted roots.
    int num_guess_states = (int)std::min<int64_t>((int64_t)o.guess_per_root * nroot, Neff);
    // the spin sector is part of the space: with spin adaptation the previous vectors must come
    // from a solve of the same multiplicity that was itself spin adapted
    std::vector<int64_t> space = {c.n, c.na, c.nb, c.irrep, c.nirrep, (int64_t)N, Neff, nroot, m,
                                  o.spin_adapt ? c.multiplicity : -1};
    for (int x : c.orbsym) space.push_back(x);
    space.push_back(c.gas.ngas);  // the GAS restriction is part of the space too
    for (int k = 0; k < c.gas.ngas; k++) {
        space.push_back(c.gas.orbs[k]);
        space.push_back(c.gas.emin[k]);
        space.push_back(c.gas.emax[k]);
    }
    const bool restart = c.dl_prev && c.dl_prev_space == space &&
                         (int64_t)num_guess_states * o.dets_per_guess < Neff;
    c.dl_prev = false;  // set again when this solve completes
    if (restart) {
        if (o.print) printf("\n  Davidson-Liu solver: restarting from previous calculation.\n");
        c.restarted = true;
    } else {
        c.restarted = false;
    }
    int ng = (int)std::min<int64_t>((int64_t)num_guess_states * o.dets_per_guess, Neff);
    double t_guess0 = now_ms();
    int basis = 0;
    BadRoots bad;
    auto upload_bad = [&](const std::vector<std::vector<std::pair<int64_t, double>>>& src) {
        std::vector<int64_t> ix;
        std::vector<double> vv;
        std::vector<int> off(1, 0);
        for (auto& r : src) {
            for (auto& e : r) { ix.push_back(e.first); vv.push_back(e.second); }
            off.push_back((int)ix.size());
        }
        bad.nb = (int)src.size();
        bad.idx.upload(ix, c.stream);
        bad.val.upload(vv, c.stream);
        bad.off.upload(off, c.stream);
        FCIB_CUDA(cudaStreamSynchronize(c.stream));  // the host index vectors go out of scope
    };
    // a fresh guess (FCISolver::initial_guess_det): lowest diagonal determinants, spin-adapted
    // guess vectors and the unwanted roots to project out
    // a fresh guess in the CSF basis (FCISolver::initial_guess_csf, find_initial_guess_csf in
    // sparse_initial_guess.cc:266-327): unit vectors on the num_guess_states lowest CSF diagonal
    // elements, ordered by (value, index); no roots to project out
    auto fresh_guess_csf = [&]() -> int {
        auto lowest = lowest_keys(c, c.hd_csf.p, num_guess_states, (size_t)N, nullptr);
        const int nguess = (int)lowest.size();
        c.t_guess_ms = now_ms() - t_guess0;
        c.guess_dets = nguess;
        FCIB_CHECK(nguess >= 1, FCIB_ERR_ARG, "Found zero FCI guesses with the requested multiplicity.");
        FCIB_CHECK(nguess >= nroot && nguess <= m, FCIB_ERR_ARG,
                   "DavidsonLiuSolver: number of guess vectors must be between nroot and the subspace size");
        c.dl_bad.clear();
        upload_bad(c.dl_bad);
        FCIB_CUDA(cudaMemsetAsync(c.tmp.p, 0, sizeof(double) * (size_t)m * N, c.stream));
        std::vector<int64_t> ix(nguess);
        std::vector<double> one(nguess, 1.0);
        for (int g = 0; g < nguess; g++) ix[g] = (int64_t)g * N + lowest[g].second;  // tmp[g][csf]
        SparseDev sd;
        sd.idx.upload(ix, c.stream);
        sd.val.upload(one, c.stream);
        k_fill_sparse<<<(nguess + 255) / 256, 256, 0, c.stream>>>(c.tmp.p, sd.idx.p, sd.val.p, nguess);
        FCIB_KCHECK();
        FCIB_CUDA(cudaStreamSynchronize(c.stream));
        const int added = add_rows_orth(ops, b, 0, std::vector<double*>(tmp.begin(), tmp.begin() + nguess), nguess);
        FCIB_CHECK(added == nguess, FCIB_ERR_NUMERIC, "DavidsonLiuSolver: guess vectors are zero or linearly dependent");
        return added;
    };
    auto fresh_guess = [&]() -> int {
        // lowest diagonal elements (GAS basis: over the flat order, ties by flat position)
        auto lowest = gas_basis ? lowest_keys(c, c.hd_gas.p, ng, (size_t)N, nullptr) : lowest_diagonal(c, ng);
        std::vector<uint32_t> sa(c.nas), sbv(c.nbs);
        FCIB_CUDA(cudaMemcpy(sa.data(), c.A.str.p, 4 * c.nas, cudaMemcpyDeviceToHost));
        FCIB_CUDA(cudaMemcpy(sbv.data(), c.B.str.p, 4 * c.nbs, cudaMemcpyDeviceToHost));
        HostInts hi;
        hi.n = c.n;
        hi.oa = &c.oei_a; hi.ob = &c.oei_b; hi.taa = &c.tei_aa; hi.tab = &c.tei_ab; hi.tbb = &c.tei_bb;
        const int64_t nbs = c.nbs;
        const int n = c.n;
        GuessResult gr;
        try {
            // vector index <-> determinant in the engine layout (C1 or the target irrep's blocks), or
            // in the GAS flat order
            gr = make_guess(
                hi, lowest,
                [&](int64_t I) {
                    if (gas_basis) I = c.flat_map[I];
                    if (!c.sym.on) return Det{sa[I / nbs], sbv[I % nbs]};
                    int64_t ia, ib;
                    sym_host_decode(c, I, ia, ib);
                    return Det{sa[ia], sbv[ib]};
                },
                [&](const Det& d) {
                    const int64_t ia = host_rank((uint32_t)d.a, n), ib = host_rank((uint32_t)d.b, n);
                    const int64_t I = c.sym.on ? sym_host_encode(c, ia, ib) : ia * nbs + ib;
                    if (!gas_basis) return I;
                    // spin partners of GAS determinants are GAS determinants (same electrons per space)
                    const int64_t f = gas_flat_position(c, I);
                    if (f < 0) throw std::runtime_error("initial guess: a determinant outside the GAS space");
                    return f;
                },
                num_guess_states, c.multiplicity);
        } catch (std::exception& e) {
            throw Error{FCIB_ERR_ARG, e.what()};
        }
        int nguess = (int)gr.guesses.size();
        c.t_guess_ms = now_ms() - t_guess0;
        c.guess_dets = gr.guesses.empty() ? 0 : (int)gr.guesses[0].size();
        FCIB_CHECK(nguess >= nroot && nguess <= m, FCIB_ERR_ARG,
                   "DavidsonLiuSolver: number of guess vectors must be between nroot and the subspace size");
        c.dl_bad = gr.bad_roots;
        upload_bad(c.dl_bad);
        FCIB_CUDA(cudaMemsetAsync(c.tmp.p, 0, sizeof(double) * (size_t)m * N, c.stream));
        for (int g = 0; g < nguess; g++) {
            SparseDev sd;
            std::vector<int64_t> ix;
            std::vector<double> vv;
            for (auto& e : gr.guesses[g]) { ix.push_back(e.first); vv.push_back(e.second); }
            sd.idx.upload(ix, c.stream);
            sd.val.upload(vv, c.stream);
            k_fill_sparse<<<((int)ix.size() + 255) / 256, 256, 0, c.stream>>>(tmp[g], sd.idx.p, sd.val.p, (int)ix.size());
            FCIB_KCHECK();
            FCIB_CUDA(cudaStreamSynchronize(c.stream));
        }
        if (gr.perturb) {
            // Without spin selection the lowest state may lie in a spin sector the guess space does
            // not contain; exact FP64 iterations never leave the sectors of the guess, so every
            // guess gets a seeded pseudo-random component of norm ~1e-3 over all determinants.
            for (int k = 0; k < nguess; k++) {
                k_add_random<<<ops.nblk, kRedThreads, 0, c.stream>>>(tmp[k], N, 0x9E3779B97F4A7C15ull * (k + 1),
                                                                     1.0e-3 * std::sqrt(3.0 / (double)N));
                FCIB_KCHECK();
                if (!gas_basis) apply_mask(c, tmp[k]);
            }
        }
        project_out(c, bad, tmp, std::min(nroot, nguess));
        int should = std::max(nroot, nguess);
        const int added = add_rows_orth(ops, b, 0, std::vector<double*>(tmp.begin(), tmp.begin() + should), should);
        FCIB_CHECK(added == should, FCIB_ERR_NUMERIC, "DavidsonLiuSolver: guess vectors are zero or linearly dependent");
        return added;
    };
    if (restart) {
        upload_bad(c.dl_bad);
        basis = nroot;  // rows 0..nroot-1 of b hold the previous eigenvectors
        c.t_guess_ms = 0.0;
    } else {
        basis = csf_basis ? fresh_guess_csf() : fresh_guess();
    }

    const bool mixed = (o.precision != FCIB_PREC_FP64);
    const int lowp = o.precision;
    Phase phase = mixed ? Phase::LowPrecision : Phase::FP64Only;
    std::vector<int> sig_fp64(m, 0);  // sigma of basis vector j computed in FP64
    int restarts = 0;
    double best_r = 1e300;
    int stall = 0;

    int nsig = 0;
    std::vector<double> G((size_t)m * m, 0.0), alpha((size_t)m * m, 0.0), lambda(m, 0.0), lambda_old(m, 0.0);
    if (restart && (int)c.dl_lambda_old.size() == m) lambda_old = c.dl_lambda_old;  // a member of the reference solver
    std::vector<double> rnorm(nroot, 0.0), cnorm(nroot, 0.0);
    int gvalid = 0;
    bool converged = false;
    int iter = 0;
    std::mt19937_64 rng(12345);
    if (o.print)
        printf("\n  Davidson-Liu (B200): %lld determinants, %d roots, subspace %d, collapse %d, precision %d\n",
               (long long)Neff, nroot, m, collapse, o.precision);

    // Restart the basis from the current Ritz vectors with FP64 sigma (mixed modes).
    auto restart_fp64 = [&]() {
        std::vector<const double*> Bp(b.begin(), b.begin() + basis);
        std::vector<std::vector<double>> coef(nroot, std::vector<double>(basis));
        for (int k = 0; k < nroot; k++)
            for (int j = 0; j < basis; j++) coef[k][j] = alpha[j * m + k];
        ops.combo(Bp, coef, std::vector<double*>(tmp.begin(), tmp.begin() + nroot), 0.0);
        int got = add_rows_orth(ops, b, 0, std::vector<double*>(tmp.begin(), tmp.begin() + nroot), nroot);
        FCIB_CHECK(got == nroot, FCIB_ERR_NUMERIC, "DavidsonLiuSolver: restart generated fewer vectors than expected");
        basis = nroot;
        nsig = 0;
        gvalid = 0;
        restarts++;
    };

    for (iter = 0; iter < o.maxiter; iter++) {
        // 1. sigma of the new basis vectors
        for (int j = nsig; j < basis; j++) {
            bool fp64 = (phase == Phase::FP64Only) || (phase == Phase::Refine && j < nroot && nsig == 0);
            FCIB_CUDA(cudaEventRecord(e0, c.stream));
            space_sigma(b[j], sg[j], fp64 ? FCIB_PREC_FP64 : lowp);
            FCIB_CUDA(cudaEventRecord(e1, c.stream));
            FCIB_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            c.t_sigma_ms += ms;
            c.n_sigma++;
            c.n_sigma_fp64 += fp64 ? 1 : 0;
            sig_fp64[j] = fp64 ? 1 : 0;
        }
        bool all_fp64 = true;
        for (int j = 0; j < basis; j++) all_fp64 = all_fp64 && sig_fp64[j];
        nsig = basis;
        // 2. new rows/columns of G = b sigma^T in one pass per new vector
        for (int j = gvalid; j < basis; j++) {
            std::vector<const double*> V;
            std::vector<int> sel;
            for (int i = 0; i < basis; i++) { V.push_back(b[i]); sel.push_back(0); }
            for (int i = 0; i < gvalid; i++) { V.push_back(sg[i]); sel.push_back(1); }
            std::vector<double> d;
            ops.dots(V, sel, sg[j], b[j], d);
            for (int i = 0; i < basis; i++) G[i * m + j] = d[i];
            for (int i = 0; i < gvalid; i++) G[j * m + i] = d[basis + i];
        }
        gvalid = basis;
        std::vector<double> Gb((size_t)basis * basis), ab((size_t)basis * basis), lb(basis);
        for (int i = 0; i < basis; i++)
            for (int j = 0; j < basis; j++) Gb[i * basis + j] = 0.5 * (G[i * m + j] + G[j * m + i]);
        sym_eigen(basis, Gb.data(), lb.data(), ab.data());
        std::fill(alpha.begin(), alpha.end(), 0.0);
        for (int i = 0; i < basis; i++)
            for (int j = 0; j < basis; j++) alpha[i * m + j] = ab[i * basis + j];
        for (int i = 0; i < m; i++) lambda[i] = i < basis ? lb[i] : 0.0;
        for (int i = 0; i < nroot; i++)
            FCIB_CHECK(std::isfinite(lambda[i]), FCIB_ERR_NUMERIC, "non-finite eigenvalue in the Davidson subspace");
        // 3. residuals r_k = sum_j alpha_jk (sigma_j - lambda_k b_j), norms and corrections
        {
            std::vector<const double*> V;
            for (int j = 0; j < basis; j++) V.push_back(sg[j]);
            for (int j = 0; j < basis; j++) V.push_back(b[j]);
            std::vector<std::vector<double>> coef(nroot, std::vector<double>(2 * basis));
            for (int k = 0; k < nroot; k++)
                for (int j = 0; j < basis; j++) {
                    coef[k][j] = alpha[j * m + k];
                    coef[k][basis + j] = -lambda[k] * alpha[j * m + k];
                }
            auto rc = ops.combo(V, coef, r, 0.0, lambda.data());
            for (int k = 0; k < nroot; k++) {
                rnorm[k] = std::sqrt(rc[k].first);
                cnorm[k] = std::sqrt(rc[k].second);
            }
            if (c.capture_max > (int)c.cap_r.size()) {
                // raw residual of root 0 (training data of the learned preconditioner)
                std::vector<std::vector<double>> c0(1, coef[0]);
                ops.combo(V, c0, {tmp[0]}, 0.0);
                std::vector<double> h(N);
                FCIB_CUDA(cudaMemcpyAsync(h.data(), tmp[0], sizeof(double) * N, cudaMemcpyDeviceToHost, c.stream));
                FCIB_CUDA(cudaStreamSynchronize(c.stream));
                c.cap_r.push_back(std::move(h));
                c.cap_lambda.push_back(lambda[0]);
            }
            if (o.preconditioner == FCIB_PRECOND_MLP) {
                // learned per-determinant rescaling of the diagonal corrections
                for (int k = 0; k < nroot; k++) {
                    mlp_apply(c, r[k], lambda[k], rnorm[k], cnorm[k]);
                    cnorm[k] = std::sqrt(ops.norm2(r[k]));
                }
            }
        }
        // 4. project out undesired roots; normalisation is folded into Gram-Schmidt
        project_out(c, bad, r, nroot);
        if (!bad.empty() || o.spin_adapt)
            for (int k = 0; k < nroot; k++) cnorm[k] = std::sqrt(ops.norm2(r[k]));
        // 5./6. convergence
        int ne = 0, nr = 0;
        double maxde = 0.0, maxr = 0.0;
        for (int k = 0; k < nroot; k++) {
            double de = std::fabs(lambda[k] - lambda_old[k]);
            maxde = std::max(maxde, de);
            maxr = std::max(maxr, rnorm[k]);
            ne += de < o.e_convergence;
            nr += rnorm[k] < o.r_convergence;
        }
        c.trace.push_back({(double)iter, now_ms() - t_start, lambda[0], maxr, all_fp64 ? 1.0 : 0.0});
        if (o.print) {
            double avg = 0.0;
            for (int k = 0; k < nroot; k++) avg += lambda[k] / nroot;
            printf("  %4d  %20.12f  %12.3e  %12.3e  %3d %s\n", iter, avg, maxde, maxr, basis,
                   all_fp64 ? "fp64" : "low");
        }
        bool e_ok = ne == nroot, r_ok = nr == nroot;
        if ((e_ok && r_ok) || basis == Neff) {
            if (!mixed || all_fp64) {
                converged = true;
                break;
            }
        }
        // mixed modes: restart from the Ritz vectors with FP64 sigma when the low-precision
        // residual reaches its floor or the low-precision iteration claims convergence
        if (mixed && phase != Phase::FP64Only) {
            if (maxr < 0.9 * best_r) { best_r = maxr; stall = 0; } else stall++;
            bool want = (e_ok && r_ok) || basis == Neff ||
                        (phase == Phase::LowPrecision && maxr < std::max(o.mixed_switch, o.r_convergence)) ||
                        (stall >= 4 && maxr < 1.0e-2);
            if (want) {
                if (restarts >= 6) phase = Phase::FP64Only;
                else phase = Phase::Refine;
                restart_fp64();
                best_r = 1e300;
                stall = 0;
                lambda_old = lambda;
                continue;
            }
        }
        // 7. collapse
        if (basis + nroot > m) {
            int cs = std::min(std::max(collapse, nroot), basis);
            std::vector<const double*> Bp(b.begin(), b.begin() + basis), Sp(sg.begin(), sg.begin() + basis);
            std::vector<std::vector<double>> coef(cs, std::vector<double>(basis));
            for (int k = 0; k < cs; k++)
                for (int j = 0; j < basis; j++) coef[k][j] = alpha[j * m + k];
            ops.combo(Bp, coef, std::vector<double*>(tmp.begin(), tmp.begin() + cs), 0.0);
            int a2 = add_rows_orth(ops, b, 0, std::vector<double*>(tmp.begin(), tmp.begin() + cs), cs);
            FCIB_CHECK(a2 == cs, FCIB_ERR_NUMERIC, "DavidsonLiuSolver: collapse generated fewer vectors than expected");
            ops.combo(Sp, coef, std::vector<double*>(tmp.begin(), tmp.begin() + cs), 0.0);
            bool f64 = true;
            for (int j = 0; j < basis; j++) f64 = f64 && sig_fp64[j];
            for (int k = 0; k < cs; k++) {
                std::swap(sg[k], tmp[k]);
                sig_fp64[k] = f64 ? 1 : 0;
            }
            basis = cs;
            nsig = cs;
            gvalid = 0;
        }
        // 8. add the normalised correction vectors
        int num_to_add = std::min(nroot, m - basis);
        std::vector<double> sc(nroot);
        for (int k = 0; k < nroot; k++) sc[k] = 1.0 / cnorm[k];
        int added = add_rows_orth(ops, b, basis, r, num_to_add, &sc);
        basis += added;
        int missing = num_to_add - added;
        if (missing > 0) {
            for (int k = 0; k < missing; k++) {
                FCIB_CUDA(cudaMemsetAsync(tmp[m - 1], 0, sizeof(double) * N, c.stream));
                k_add_random<<<ops.nblk, kRedThreads, 0, c.stream>>>(tmp[m - 1], N, 0xD1B54A32D192ED03ull + rng(), 1.0);
                FCIB_KCHECK();
                if (!csf_basis && !gas_basis) apply_mask(c, tmp[m - 1]);
                std::vector<double*> one{tmp[m - 1]};
                project_out(c, bad, one, 1);
                int ra = add_rows_orth(ops, b, basis, one, 1);
                basis += ra;
                added += ra;
            }
        }
        if (added == 0) {
            converged = r_ok && (!mixed || all_fp64);
            break;
        }
        lambda_old = lambda;
    }
    c.iterations = std::min(iter + 1, o.maxiter);
    // get_results (davidson_liu_solver.cc:488-501): final eigenvectors in b[0..nroot)
    {
        std::vector<const double*> Bp(b.begin(), b.begin() + basis);
        std::vector<std::vector<double>> coef(nroot, std::vector<double>(basis));
        for (int k = 0; k < nroot; k++)
            for (int j = 0; j < basis; j++) coef[k][j] = alpha[j * m + k];
        ops.combo(Bp, coef, std::vector<double*>(tmp.begin(), tmp.begin() + nroot), 0.0);
        int got = add_rows_orth(ops, b, 0, std::vector<double*>(tmp.begin(), tmp.begin() + nroot), nroot);
        FCIB_CHECK(got == nroot, FCIB_ERR_NUMERIC, "DavidsonLiuSolver: get_results generated fewer vectors than expected");
    }
    c.energies.assign(lambda.begin(), lambda.begin() + nroot);
    FCIB_CUDA(cudaEventRecord(e1, c.stream));
    FCIB_CUDA(cudaEventSynchronize(e1));
    float tot = 0.f;
    cudaEventElapsedTime(&tot, ev_start, e1);
    c.t_total_ms = tot;
    c.solved = true;
    c.converged = converged;
    c.dl_prev = true;
    c.dl_prev_space = space;
    c.dl_lambda_old = lambda;
    if (csf_basis || gas_basis) {
        // the roots in the determinant layout, for <S^2>, RDMs and the flat-order vectors
        c.evdet.alloc((size_t)nroot * c.nvec);
        if (gas_basis) FCIB_CUDA(cudaMemsetAsync(c.evdet.p, 0, sizeof(double) * nroot * c.nvec, c.stream));
        for (int k = 0; k < nroot; k++) {
            if (gas_basis) scatter_flat(c, c.b.p + (size_t)k * N, c.evdet.p + (size_t)k * c.nvec);
            else csf_to_det(c, c.b.p + (size_t)k * N, c.evdet.p + (size_t)k * c.nvec);
        }
    }
    c.roots_in_evdet = csf_basis || gas_basis;
    c.spin2.resize(nroot);
    for (int k = 0; k < nroot; k++) c.spin2[k] = spin2_device(c, root_vector(c, k));
    FCIB_CUDA(cudaStreamSynchronize(c.stream));
    cudaEventDestroy(ev_start);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

}  // namespace fcib
