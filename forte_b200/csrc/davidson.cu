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

#include "fcib_internal.h"
#include "guess.h"

namespace fcib {

constexpr int kMaxV = 32;
struct VecSet {
    const double* p[kMaxV];
    double coef[kMaxV];
};

constexpr int kRedThreads = 256;

// partial[block][j] = sum_I V_j[I] * x[I]   (j < nv); slot nv holds x.x when self != 0
__global__ void __launch_bounds__(kRedThreads) k_multidot(VecSet vs, int nv, const double* __restrict__ x,
                                                          size_t N, int self, double* __restrict__ partial) {
    double acc[kMaxV + 1];
#pragma unroll
    for (int j = 0; j <= kMaxV; j++) acc[j] = 0.0;
    for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < N; I += (size_t)gridDim.x * blockDim.x) {
        double xv = x[I];
#pragma unroll
        for (int j = 0; j < kMaxV; j++)
            if (j < nv) acc[j] = fma(vs.p[j][I], xv, acc[j]);
        if (self) acc[kMaxV] = fma(xv, xv, acc[kMaxV]);
    }
    __shared__ double red[kRedThreads / 32][kMaxV + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j <= kMaxV; j++) {
        if (j < nv || (j == kMaxV && self)) {
            double v = acc[j];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) red[warp][j] = v;
        }
    }
    __syncthreads();
    if (threadIdx.x <= kMaxV) {
        int j = threadIdx.x;
        if (j < nv || (j == kMaxV && self)) {
            double s = 0.0;
            for (int w = 0; w < kRedThreads / 32; w++) s += red[w][j];
            partial[(size_t)blockIdx.x * (kMaxV + 1) + j] = s;
        }
    }
}

__global__ void k_reduce_partials(const double* __restrict__ partial, int nblocks, int nv, int self,
                                  double* __restrict__ out) {
    int j = threadIdx.x;
    if (j <= kMaxV && (j < nv || (j == kMaxV && self))) {
        double s = 0.0;
        for (int b = 0; b < nblocks; b++) s += partial[(size_t)b * (kMaxV + 1) + j];
        out[j] = s;
    }
}

// out[I] = beta * out[I] + sum_j coef_j V_j[I]; optional partial sums of out^2
__global__ void __launch_bounds__(kRedThreads) k_lincomb(VecSet vs, int nv, double* __restrict__ out, double beta,
                                                         size_t N, double* __restrict__ partial) {
    double nrm = 0.0;
    for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < N; I += (size_t)gridDim.x * blockDim.x) {
        double v = (beta == 0.0) ? 0.0 : beta * out[I];
#pragma unroll
        for (int j = 0; j < kMaxV; j++)
            if (j < nv) v = fma(vs.coef[j], vs.p[j][I], v);
        out[I] = v;
        nrm = fma(v, v, nrm);
    }
    if (partial) {
        __shared__ double red[kRedThreads / 32];
        for (int o = 16; o > 0; o >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = nrm;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0.0;
            for (int w = 0; w < kRedThreads / 32; w++) s += red[w];
            partial[(size_t)blockIdx.x * (kMaxV + 1)] = s;
        }
    }
}

// corr = r / (lambda - H_II) (0 when |lambda - H_II| <= 1e-6); partial[b][0] = r.r, [1] = corr.corr
__global__ void __launch_bounds__(kRedThreads) k_precond_diag(double* __restrict__ r, const double* __restrict__ hd,
                                                              double lambda, size_t N, double* __restrict__ partial) {
    double rr = 0.0, cc = 0.0;
    for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < N; I += (size_t)gridDim.x * blockDim.x) {
        double v = r[I];
        rr = fma(v, v, rr);
        double den = lambda - hd[I];
        double c = (fabs(den) > 1.0e-6) ? v / den : 0.0;
        r[I] = c;
        cc = fma(c, c, cc);
    }
    __shared__ double red[2][kRedThreads / 32];
    for (int o = 16; o > 0; o >>= 1) {
        rr += __shfl_xor_sync(0xffffffffu, rr, o);
        cc += __shfl_xor_sync(0xffffffffu, cc, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = rr;
        red[1][threadIdx.x >> 5] = cc;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double s = 0.0;
        for (int w = 0; w < kRedThreads / 32; w++) s += red[threadIdx.x][w];
        partial[(size_t)blockIdx.x * (kMaxV + 1) + threadIdx.x] = s;
    }
}

__global__ void k_scale(double* __restrict__ v, double a, size_t N) {
    for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < N; I += (size_t)gridDim.x * blockDim.x) v[I] *= a;
}

__global__ void k_fill_sparse(double* __restrict__ v, const int64_t* __restrict__ idx, const double* __restrict__ val, int cnt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < cnt) v[idx[i]] = val[i];
}

// v -= (v . u) u for a sparse vector u (one block)
__global__ void k_project_sparse(double* __restrict__ v, const int64_t* __restrict__ idx, const double* __restrict__ val, int cnt) {
    __shared__ double red[32];
    double s = 0.0;
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) s = fma(v[idx[i]], val[i], s);
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
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) v[idx[i]] -= ov * val[i];
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

__global__ void __launch_bounds__(kRedThreads) k_spin2(const double* __restrict__ C, const uint32_t* __restrict__ sa,
                                                       const uint32_t* __restrict__ sb, int nas, int nbs, int n,
                                                       double* __restrict__ partial) {
    double acc = 0.0;
    const size_t N = (size_t)nas * nbs;
    for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < N; I += (size_t)gridDim.x * blockDim.x) {
        double ci = C[I];
        if (ci == 0.0) continue;
        uint32_t Ia = sa[I / nbs], Ib = sb[I % nbs];
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
                double cj = C[(size_t)d_rank(Ja, n) * nbs + d_rank(Jb, n)];
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
        partial[(size_t)blockIdx.x * (kMaxV + 1)] = s;
    }
}

// ------------------------------------------------------------------------------------------
// host helpers
// ------------------------------------------------------------------------------------------
struct Ops {
    Context& c;
    size_t N;
    int nblk;
    DBuf<double> partial, out;
    std::vector<double> hout;
    explicit Ops(Context& cc) : c(cc) {
        N = (size_t)c.ndet;
        nblk = std::max(1, std::min(4 * c.num_sms, (int)((N + kRedThreads - 1) / kRedThreads)));
        partial.alloc((size_t)nblk * (kMaxV + 1));
        out.alloc(kMaxV + 1);
        hout.resize(kMaxV + 1);
    }
    // d[j] = V_j . x for j < nv (any nv), optionally x.x
    void dots(const std::vector<const double*>& V, const double* x, std::vector<double>& d, double* xx = nullptr) {
        d.assign(V.size(), 0.0);
        size_t done = 0;
        bool self = xx != nullptr;
        do {
            VecSet vs;
            int nv = (int)std::min<size_t>(kMaxV, V.size() - done);
            for (int j = 0; j < nv; j++) vs.p[j] = V[done + j];
            int want_self = (self && done == 0) ? 1 : 0;
            k_multidot<<<nblk, kRedThreads, 0, c.stream>>>(vs, nv, x, N, want_self, partial.p);
            FCIB_CUDA(cudaGetLastError());
            k_reduce_partials<<<1, 64, 0, c.stream>>>(partial.p, nblk, nv, want_self, out.p);
            FCIB_CUDA(cudaGetLastError());
            FCIB_CUDA(cudaMemcpyAsync(hout.data(), out.p, sizeof(double) * (kMaxV + 1), cudaMemcpyDeviceToHost, c.stream));
            FCIB_CUDA(cudaStreamSynchronize(c.stream));
            for (int j = 0; j < nv; j++) d[done + j] = hout[j];
            if (want_self) *xx = hout[kMaxV];
            done += nv;
        } while (done < V.size());
    }
    // out = beta*out + sum coef_j V_j ; returns out.out when want_norm
    double lincomb(const std::vector<const double*>& V, const std::vector<double>& coef, double* o, double beta,
                   bool want_norm) {
        size_t done = 0;
        double nrm = 0.0;
        if (V.empty()) {
            if (beta != 1.0) {
                k_scale<<<nblk, kRedThreads, 0, c.stream>>>(o, beta, N);
                FCIB_CUDA(cudaGetLastError());
            }
            if (want_norm) {
                std::vector<double> dd;
                dots({}, o, dd, &nrm);
            }
            return nrm;
        }
        while (done < V.size()) {
            VecSet vs;
            int nv = (int)std::min<size_t>(kMaxV, V.size() - done);
            for (int j = 0; j < nv; j++) {
                vs.p[j] = V[done + j];
                vs.coef[j] = coef[done + j];
            }
            bool last = done + nv == V.size();
            k_lincomb<<<nblk, kRedThreads, 0, c.stream>>>(vs, nv, o, done == 0 ? beta : 1.0, N,
                                                          (last && want_norm) ? partial.p : nullptr);
            FCIB_CUDA(cudaGetLastError());
            done += nv;
        }
        if (want_norm) {
            k_reduce_partials<<<1, 64, 0, c.stream>>>(partial.p, nblk, 1, 0, out.p);
            FCIB_CUDA(cudaMemcpyAsync(hout.data(), out.p, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
            FCIB_CUDA(cudaStreamSynchronize(c.stream));
            nrm = hout[0];
        }
        return nrm;
    }
    void scale(double* v, double a) {
        k_scale<<<nblk, kRedThreads, 0, c.stream>>>(v, a, N);
        FCIB_CUDA(cudaGetLastError());
    }
    void copy(double* dst, const double* src) {
        FCIB_CUDA(cudaMemcpyAsync(dst, src, N * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
    }
    // returns (r.r, corr.corr)
    std::pair<double, double> precond(double* r, double lambda) {
        k_precond_diag<<<nblk, kRedThreads, 0, c.stream>>>(r, c.hdiag.p, lambda, N, partial.p);
        FCIB_CUDA(cudaGetLastError());
        k_reduce_partials<<<1, 64, 0, c.stream>>>(partial.p, nblk, 2, 0, out.p);
        FCIB_CUDA(cudaMemcpyAsync(hout.data(), out.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        FCIB_CUDA(cudaStreamSynchronize(c.stream));
        return {hout[0], hout[1]};
    }
};

struct SparseDev {
    DBuf<int64_t> idx;
    DBuf<double> val;
    int cnt = 0;
};

// add_row_and_orthonormalize (davidson_liu_solver.cc:634-687): copy v into A[rowsA] and
// Gram-Schmidt it against A[0..rowsA); false if discarded.
static bool add_row_orth(Ops& ops, std::vector<double*>& A, int rowsA, const double* v) {
    double* w = A[rowsA];
    if (w != v) ops.copy(w, v);
    std::vector<const double*> B(A.begin(), A.begin() + rowsA);
    std::vector<double> d;
    double vv = 0.0;
    ops.dots(B, w, d, &vv);
    for (int cycle = 0; cycle < 10; cycle++) {
        std::vector<double> coef(rowsA);
        for (int i = 0; i < rowsA; i++) coef[i] = -d[i];
        double nn = ops.lincomb(B, coef, w, 1.0, true);
        double nv = std::sqrt(nn);
        if (nv < 1.0e-7) return false;
        ops.scale(w, 1.0 / nv);
        ops.dots(B, w, d, &vv);
        double mo = 0.0;
        for (int i = 0; i < rowsA; i++) mo = std::max(mo, std::fabs(d[i]));
        if (mo < 1.0e-12 && std::fabs(vv - 1.0) < 1.0e-12) return true;
    }
    return false;
}

static int add_rows_orth(Ops& ops, std::vector<double*>& A, int rowsA, const std::vector<double*>& Bv, int rowsB) {
    int added = 0;
    for (int j = 0; j < rowsB; j++)
        if (add_row_orth(ops, A, rowsA + added, Bv[j])) added++;
    return added;
}

static void project_out(Context& c, std::vector<SparseDev>& bad, std::vector<double*>& V, int nvec) {
    for (int k = 0; k < nvec; k++)
        for (auto& b : bad) {
            k_project_sparse<<<1, 256, 0, c.stream>>>(V[k], b.idx.p, b.val.p, b.cnt);
            FCIB_CUDA(cudaGetLastError());
        }
}

double spin2_device(Context& c, const double* C) {
    Ops ops(c);
    k_spin2<<<ops.nblk, kRedThreads, 0, c.stream>>>(C, c.A.str.p, c.B.str.p, (int)c.nas, (int)c.nbs, c.n, ops.partial.p);
    FCIB_CUDA(cudaGetLastError());
    k_reduce_partials<<<1, 64, 0, c.stream>>>(ops.partial.p, ops.nblk, 1, 0, ops.out.p);
    double s = 0.0;
    FCIB_CUDA(cudaMemcpyAsync(&s, ops.out.p, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    FCIB_CUDA(cudaStreamSynchronize(c.stream));
    double na = c.na, nb = c.nb;
    return -s + 0.25 * (na - nb) * (na - nb) + 0.5 * (na + nb);
}

// lowest `count` diagonal entries ordered by (value, address), like the insertion list of
// FCISolver::initial_guess_generate_dets (fci_solver_initial_guess.cc:44-69)
static std::vector<std::pair<double, int64_t>> lowest_diagonal(Context& c, int count) {
    const size_t N = (size_t)c.ndet;
    const uint8_t* mask = (c.nirrep > 1) ? c.mask.p : nullptr;
    DBuf<unsigned int> hist;
    hist.alloc(256);
    uint64_t prefix = 0, pmask = 0;
    uint64_t need = count;
    int grid = 4 * c.num_sms;
    for (int shift = 56; shift >= 0; shift -= 8) {
        FCIB_CUDA(cudaMemsetAsync(hist.p, 0, 256 * sizeof(unsigned int), c.stream));
        k_radix_hist<<<grid, 256, 0, c.stream>>>(c.hdiag.p, mask, N, prefix, pmask, shift, hist.p);
        FCIB_CUDA(cudaGetLastError());
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
    k_collect_le<<<grid, 256, 0, c.stream>>>(c.hdiag.p, mask, N, prefix, cap, cnt.p, ev.p, ei.p);
    FCIB_CUDA(cudaGetLastError());
    int hc = 0;
    FCIB_CUDA(cudaMemcpyAsync(&hc, cnt.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    FCIB_CUDA(cudaStreamSynchronize(c.stream));
    FCIB_CHECK(hc <= cap, FCIB_ERR_NUMERIC, "too many degenerate diagonal entries for the guess selection");
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

static double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void dl_solve(Context& c) {
    const int64_t N = c.ndet;
    int64_t Neff = N;
    if (c.nirrep > 1) {
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
    const int collapse = (int)std::min<int64_t>((int64_t)o.collapse_per_root * nroot, Neff);
    const int m = (int)std::min<int64_t>((int64_t)o.subspace_per_root * nroot, Neff);
    FCIB_CHECK(nroot <= m, FCIB_ERR_ARG, "more roots than determinants");
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
    Ops ops(c);
    double t_start = now_ms();
    c.t_sigma_ms = 0.0;
    c.n_sigma = 0;

    // ---- initial guess ----
    int num_guess_states = (int)std::min<int64_t>((int64_t)o.guess_per_root * nroot, Neff);
    int ng = (int)std::min<int64_t>((int64_t)num_guess_states * o.dets_per_guess, Neff);
    auto lowest = lowest_diagonal(c, ng);
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
        gr = make_guess(
            hi, lowest, [&](int64_t I) { return Det{sa[I / nbs], sbv[I % nbs]}; },
            [&](const Det& d) { return (int64_t)host_rank((uint32_t)d.a, n) * nbs + host_rank((uint32_t)d.b, n); },
            num_guess_states, c.multiplicity);
    } catch (std::exception& e) {
        throw Error{FCIB_ERR_ARG, e.what()};
    }
    int nguess = (int)gr.guesses.size();
    FCIB_CHECK(nguess >= nroot && nguess <= m, FCIB_ERR_ARG,
               "DavidsonLiuSolver: number of guess vectors must be between nroot and the subspace size");
    std::vector<SparseDev> bad(gr.bad_roots.size());
    for (size_t i = 0; i < bad.size(); i++) {
        std::vector<int64_t> ix;
        std::vector<double> vv;
        for (auto& e : gr.bad_roots[i]) { ix.push_back(e.first); vv.push_back(e.second); }
        bad[i].idx.upload(ix, c.stream);
        bad[i].val.upload(vv, c.stream);
        bad[i].cnt = (int)ix.size();
    }
    // guesses -> tmp rows
    FCIB_CUDA(cudaMemsetAsync(c.tmp.p, 0, sizeof(double) * (size_t)m * N, c.stream));
    for (int g = 0; g < nguess; g++) {
        SparseDev sd;
        std::vector<int64_t> ix;
        std::vector<double> vv;
        for (auto& e : gr.guesses[g]) { ix.push_back(e.first); vv.push_back(e.second); }
        sd.idx.upload(ix, c.stream);
        sd.val.upload(vv, c.stream);
        k_fill_sparse<<<((int)ix.size() + 255) / 256, 256, 0, c.stream>>>(tmp[g], sd.idx.p, sd.val.p, (int)ix.size());
        FCIB_CUDA(cudaGetLastError());
        FCIB_CUDA(cudaStreamSynchronize(c.stream));
    }
    project_out(c, bad, tmp, std::min(nroot, nguess));
    int should = std::max(nroot, nguess);
    int basis = add_rows_orth(ops, b, 0, std::vector<double*>(tmp.begin(), tmp.begin() + should), should);
    FCIB_CHECK(basis == should, FCIB_ERR_NUMERIC, "DavidsonLiuSolver: guess vectors are zero or linearly dependent");
    int nsig = 0;
    std::vector<double> G((size_t)m * m, 0.0), alpha((size_t)m * m, 0.0), lambda(m, 0.0), lambda_old(m, 0.0);
    std::vector<double> rnorm(nroot, 0.0);
    int gvalid = 0;  // G[i][j] valid for i, j < gvalid
    bool converged = false;
    int iter = 0;
    std::mt19937_64 rng(12345);
    if (o.print)
        printf("\n  Davidson-Liu (B200): %lld determinants, %d roots, subspace %d, collapse %d\n",
               (long long)Neff, nroot, m, collapse);
    for (iter = 0; iter < o.maxiter; iter++) {
        // 1. sigma of the new basis vectors
        for (int j = nsig; j < basis; j++) {
            cudaEvent_t e0, e1;
            FCIB_CUDA(cudaEventCreate(&e0));
            FCIB_CUDA(cudaEventCreate(&e1));
            FCIB_CUDA(cudaEventRecord(e0, c.stream));
            sigma_dispatch(c, b[j], sg[j], FCIB_PREC_FP64);
            FCIB_CUDA(cudaEventRecord(e1, c.stream));
            FCIB_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            c.t_sigma_ms += ms;
            c.n_sigma++;
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
        }
        nsig = basis;
        // 2. subspace matrix: new rows and columns of G = b sigma^T
        {
            std::vector<double> d;
            std::vector<const double*> Bp(b.begin(), b.begin() + basis), Sp(sg.begin(), sg.begin() + basis);
            for (int j = gvalid; j < basis; j++) {
                ops.dots(Bp, sg[j], d);
                for (int i = 0; i < basis; i++) G[i * m + j] = d[i];
                std::vector<const double*> So(sg.begin(), sg.begin() + gvalid);
                ops.dots(So, b[j], d);
                for (int i = 0; i < gvalid; i++) G[j * m + i] = d[i];
            }
            gvalid = basis;
        }
        std::vector<double> Gb((size_t)basis * basis), ab((size_t)basis * basis), lb(basis);
        for (int i = 0; i < basis; i++)
            for (int j = 0; j < basis; j++) Gb[i * basis + j] = 0.5 * (G[i * m + j] + G[j * m + i]);
        sym_eigen(basis, Gb.data(), lb.data(), ab.data());
        std::fill(alpha.begin(), alpha.end(), 0.0);
        for (int i = 0; i < basis; i++)
            for (int j = 0; j < basis; j++) alpha[i * m + j] = ab[i * basis + j];
        for (int i = 0; i < m; i++) lambda[i] = i < basis ? lb[i] : 0.0;
        // 3. residuals, norms and corrections
        std::vector<double> cnorm(nroot);
        for (int k = 0; k < nroot; k++) {
            std::vector<const double*> V;
            std::vector<double> coef;
            for (int j = 0; j < basis; j++) {
                V.push_back(sg[j]);
                coef.push_back(alpha[j * m + k]);
                V.push_back(b[j]);
                coef.push_back(-lambda[k] * alpha[j * m + k]);
            }
            ops.lincomb(V, coef, r[k], 0.0, false);
            auto rc = ops.precond(r[k], lambda[k]);
            rnorm[k] = std::sqrt(rc.first);
            cnorm[k] = std::sqrt(rc.second);
        }
        // 4. project out undesired roots, normalize
        project_out(c, bad, r, nroot);
        for (int k = 0; k < nroot; k++) {
            double nn = cnorm[k];
            if (!bad.empty()) {
                std::vector<double> dd;
                double xx = 0.0;
                ops.dots({}, r[k], dd, &xx);
                nn = std::sqrt(xx);
            }
            ops.scale(r[k], 1.0 / nn);
        }
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
        if (o.print) {
            double avg = 0.0;
            for (int k = 0; k < nroot; k++) avg += lambda[k] / nroot;
            printf("  %4d  %20.12f  %12.3e  %12.3e  %3d\n", iter, avg, maxde, maxr, basis);
        }
        bool e_ok = ne == nroot, r_ok = nr == nroot;
        if ((e_ok && r_ok) || basis == Neff) {
            converged = true;
            break;
        }
        // 7. collapse
        if (basis + nroot > m) {
            int cs = std::min(std::max(collapse, nroot), basis);
            std::vector<const double*> Bp(b.begin(), b.begin() + basis), Sp(sg.begin(), sg.begin() + basis);
            for (int k = 0; k < cs; k++) {
                std::vector<double> coef(basis);
                for (int j = 0; j < basis; j++) coef[j] = alpha[j * m + k];
                ops.lincomb(Bp, coef, tmp[k], 0.0, false);
            }
            int a2 = add_rows_orth(ops, b, 0, std::vector<double*>(tmp.begin(), tmp.begin() + cs), cs);
            FCIB_CHECK(a2 == cs, FCIB_ERR_NUMERIC, "DavidsonLiuSolver: collapse generated fewer vectors than expected");
            for (int k = 0; k < cs; k++) {
                std::vector<double> coef(basis);
                for (int j = 0; j < basis; j++) coef[j] = alpha[j * m + k];
                ops.lincomb(Sp, coef, tmp[k], 0.0, false);
            }
            for (int k = 0; k < cs; k++) std::swap(sg[k], tmp[k]);
            basis = cs;
            nsig = cs;
            gvalid = 0;
        }
        // 8. add correction vectors
        int num_to_add = std::min(nroot, m - basis);
        int added = add_rows_orth(ops, b, basis, r, num_to_add);
        basis += added;
        int missing = num_to_add - added;
        if (missing > 0) {
            std::vector<double> rv(N);
            std::uniform_real_distribution<double> dist(-1.0, 1.0);
            for (int k = 0; k < missing; k++) {
                for (auto& x : rv) x = dist(rng);
                FCIB_CUDA(cudaMemcpy(tmp[m - 1], rv.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
                apply_mask(c, tmp[m - 1]);
                std::vector<double*> one{tmp[m - 1]};
                project_out(c, bad, one, 1);
                int ra = add_rows_orth(ops, b, basis, one, 1);
                basis += ra;
                added += ra;
            }
        }
        if (added == 0) {
            converged = r_ok;
            break;
        }
        lambda_old = lambda;
    }
    c.iterations = std::min(iter + 1, o.maxiter);
    // get_results: final eigenvectors
    {
        std::vector<const double*> Bp(b.begin(), b.begin() + basis);
        for (int k = 0; k < nroot; k++) {
            std::vector<double> coef(basis);
            for (int j = 0; j < basis; j++) coef[j] = alpha[j * m + k];
            ops.lincomb(Bp, coef, tmp[k], 0.0, false);
        }
        int got = add_rows_orth(ops, b, 0, std::vector<double*>(tmp.begin(), tmp.begin() + nroot), nroot);
        FCIB_CHECK(got == nroot, FCIB_ERR_NUMERIC, "DavidsonLiuSolver: get_results generated fewer vectors than expected");
        // keep the eigenvectors at the start of the b buffer
        for (int k = 0; k < nroot; k++)
            if (b[k] != c.b.p + (size_t)k * N)
                ops.copy(c.b.p + (size_t)k * N, b[k]);
    }
    c.energies.assign(lambda.begin(), lambda.begin() + nroot);
    c.solved = true;
    c.spin2.resize(nroot);
    for (int k = 0; k < nroot; k++) c.spin2[k] = spin2_device(c, c.b.p + (size_t)k * N);
    FCIB_CUDA(cudaStreamSynchronize(c.stream));
    c.t_total_ms = now_ms() - t_start;
    c.converged = converged;
}

}  // namespace fcib
