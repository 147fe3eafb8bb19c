// Spin adaptation (option spin_adapt; Forte's CI_SPIN_ADAPT, SpinAdapter in
// forte/sparse_ci/ci_spin_adaptation.h:81-183, used by fci_solver.cc:136-141,186-262).
//
// Like the reference, the Davidson-Liu solver then works in a basis of configuration state
// functions (CSFs) of the target spin S: its vectors hold CSF coefficients z, and sigma is formed
// as z -> C = P z (determinants) -> H C -> P^T (H C) (fci_solver.cc:247-254), with the CSF
// diagonal sum_m O_im^2 H_mm as preconditioner (form_Hdiag_csf without the full-preconditioner
// option, fci_solver_initial_guess.cc:111-149) and unit vectors on the lowest CSF diagonal elements
// as guess (find_initial_guess_csf, sparse_initial_guess.cc:266-327).
//
// CSFs of a configuration (doubly occupied set D, open-shell set O, N = |O|) are the genealogical
// couplings of the N open shells taken in orbital order (the published construction that adds one
// spin 1/2 at a time with Clebsch-Gordan coefficients, e.g. Pauncz, "Spin Eigenfunctions"), times
// the closed-shell pairs, which commute with the spin operators and with any pair of fermion
// operators.  Written in this engine's determinants |D+Oa ; D+Ob> (alpha string, then beta string),
// the coefficient of the spin pattern m over O (bit k set: the k-th open shell is alpha) is
//     O_N[i][m] = (-1)^(number of beta open shells below an alpha open shell) * prod_k CG_k(i, m)
// up to a sign common to the configuration.  So P restricted to a configuration is O_N^T, the same
// matrix for every configuration with N open shells; configurations that cannot couple to S
// (N < 2S) hold no CSF.  CSF vector layout: groups of increasing N, configuration-major, the f
// couplings of a configuration consecutive.
#include "fcib_internal.h"

namespace fcib {

// <S' M-m; 1/2 m | S M> for adding one spin 1/2, in units of 1/2: twoS, twoM after the step,
// dS = +-1 the change of 2S, dm = +-1 the change of 2M
static double cg_half(int twoS, int twoM, int dS, int dm) {
    if (dS == 1) return std::sqrt(0.5 * (twoS + dm * twoM) / (double)twoS);
    return -dm * std::sqrt(0.5 * (twoS + 2 - dm * twoM) / (double)(twoS + 2));
}

// Coupling matrix of N open shells to 2S = twoS at 2Ms = twoMs: O[i * nd + m] for the f coupling
// paths i (bit k set: the spin rises at step k) and the nd spin patterns m in increasing mask order
static void csf_coupling(int N, int twoS, int twoMs, std::vector<double>& O, std::vector<uint32_t>& pats, int& f,
                         int& nd) {
    pats.clear();
    std::vector<uint32_t> paths;
    const int na_open = (N + twoMs) / 2;
    for (uint32_t m = 0; m < (1u << N); m++) {
        if (__builtin_popcount(m) == na_open) pats.push_back(m);
        if (twoS > N || (N - twoS) % 2) continue;
        int s = 0;
        bool ok = true;
        for (int k = 0; k < N && ok; k++) {
            s += (m >> k & 1u) ? 1 : -1;
            ok = s >= 0;
        }
        if (ok && s == twoS) paths.push_back(m);
    }
    f = (int)paths.size();
    nd = (int)pats.size();
    O.assign((size_t)f * nd, 0.0);
    for (int i = 0; i < f; i++)
        for (int j = 0; j < nd; j++) {
            const uint32_t p = paths[i], m = pats[j];
            double v = 1.0;
            int s = 0, mm = 0, betas = 0, inv = 0;
            for (int k = 0; k < N; k++) {
                const int dS = (p >> k & 1u) ? 1 : -1;
                const int dm = (m >> k & 1u) ? 1 : -1;
                s += dS;
                mm += dm;
                if (std::abs(mm) > s) { v = 0.0; break; }
                v *= cg_half(s, mm, dS, dm);
                if (dm > 0) inv += betas;  // beta open shells below this alpha one
                else betas++;
            }
            O[(size_t)i * nd + j] = (inv & 1) ? -v : v;
        }
}

// index in the engine layout (C1, or the target irrep's blocks) of the determinant with spin
// pattern pat (bit k: the k-th open shell in orbital order is alpha) of configuration (D, Om)
__device__ __forceinline__ int64_t csf_det_id(uint32_t D, uint32_t Om, uint32_t pat, int N, int n, int nbs,
                                              const SymDev& sd) {
    uint32_t a = D, b = D, rest = Om;
    for (int k = 0; k < N; k++) {
        const uint32_t bit = rest & (0u - rest);
        rest ^= bit;
        if (pat >> k & 1u) a |= bit;
        else b |= bit;
    }
    const uint32_t ra = d_rank(a, n), rb = d_rank(b, n);
    return sd.on ? sym_encode(sd, a, (int)ra, (int)rb) : (int64_t)ra * nbs + rb;
}

// One CTA per configuration (grid-stride) of a group with N open shells, nd spin patterns and f
// couplings; its CSF coefficients are z[zoff + cf * f + i].  Every determinant belongs to exactly
// one configuration, so the scatters have no conflicts.
//   mode 0: x[det m] = sum_i O[i][m] z_i        (CSF -> determinants; zeros when f = 0)
//   mode 1: z_i = sum_m O[i][m] x[det m]        (determinants -> CSF)
//   mode 2: z_i = sum_m O[i][m]^2 x[det m]      (the CSF diagonal from the determinant diagonal x)
template <int MODE>
__global__ void k_csf_map(const double* __restrict__ in, double* __restrict__ out, const uint32_t* __restrict__ conf,
                          int nconf, int N, int nd, int f, const uint32_t* __restrict__ pats,
                          const double* __restrict__ O, int n, int nbs, SymDev sd, int64_t zoff) {
    extern __shared__ __align__(16) unsigned char csf_smem[];
    double* xs = reinterpret_cast<double*>(csf_smem);  // [nd] determinant values (modes 1, 2)
    double* zs = xs + nd;                              // [f] CSF values (mode 0)
    int64_t* idx = reinterpret_cast<int64_t*>(zs + f); // [nd]
    for (int cf = blockIdx.x; cf < nconf; cf += gridDim.x) {
        const uint32_t D = conf[2 * (size_t)cf], Om = conf[2 * (size_t)cf + 1];
        const int64_t z0 = zoff + (int64_t)cf * f;
        __syncthreads();
        for (int m = threadIdx.x; m < nd; m += blockDim.x) {
            const int64_t id = csf_det_id(D, Om, pats[m], N, n, nbs, sd);
            idx[m] = id;
            if (MODE != 0) xs[m] = in[id];
        }
        if (MODE == 0)
            for (int i = threadIdx.x; i < f; i += blockDim.x) zs[i] = in[z0 + i];
        __syncthreads();
        if (MODE == 0) {
            for (int m = threadIdx.x; m < nd; m += blockDim.x) {
                double v = 0.0;
                for (int i = 0; i < f; i++) v = fma(O[(size_t)i * nd + m], zs[i], v);
                out[idx[m]] = v;
            }
        } else {
            for (int i = threadIdx.x; i < f; i += blockDim.x) {
                const double* row = O + (size_t)i * nd;
                double v = 0.0;
                for (int m = 0; m < nd; m++) v = fma(MODE == 2 ? row[m] * row[m] : row[m], xs[m], v);
                out[z0 + i] = v;
            }
        }
    }
}

// The full CSF diagonal (CI_SPIN_ADAPT_FULL_PRECONDITIONER; form_Hdiag_csf with the full
// preconditioner, fci_solver_initial_guess.cc:118-138):
//     E_i = sum_m O_im^2 H_mm + 2 sum_{m < m'} O_im O_im' H_mm'.
// Within a configuration the only off-diagonal elements join spin patterns m, m' that differ by one
// alpha <-> beta swap of two open shells at positions a (alpha in m) and b (beta in m), orbitals
// o_a, o_b: H_mm' = (-1)^(open shells strictly between a and b) * (o_a o_b | o_b o_a) (the doubly
// occupied orbitals between them contribute to both spins' parities and cancel).  Kx[p][q] =
// <pq|qp> of the alpha-beta block.  Patterns are in increasing mask order, so the index of m' is
// its colex rank.  One CTA per configuration; one thread per CSF.
__global__ void k_csf_full_diag(const double* __restrict__ hd, double* __restrict__ out,
                                const uint32_t* __restrict__ conf, int nconf, int N, int nd, int f,
                                const uint32_t* __restrict__ pats, const double* __restrict__ O, int n, int nbs,
                                SymDev sd, int64_t zoff, const double* __restrict__ Kx) {
    extern __shared__ __align__(16) unsigned char csf_smem[];
    double* xs = reinterpret_cast<double*>(csf_smem);  // [nd] determinant diagonal
    __shared__ int orb[32];                            // orbital of each open-shell position
    for (int cf = blockIdx.x; cf < nconf; cf += gridDim.x) {
        const uint32_t D = conf[2 * (size_t)cf], Om = conf[2 * (size_t)cf + 1];
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t rest = Om;
            for (int k = 0; k < N; k++) {
                orb[k] = __ffs(rest) - 1;
                rest &= rest - 1;
            }
        }
        for (int m = threadIdx.x; m < nd; m += blockDim.x) xs[m] = hd[csf_det_id(D, Om, pats[m], N, n, nbs, sd)];
        __syncthreads();
        for (int i = threadIdx.x; i < f; i += blockDim.x) {
            const double* Oi = O + (size_t)i * nd;
            double e = 0.0, off = 0.0;
            for (int m = 0; m < nd; m++) {
                const double om = Oi[m];
                e = fma(om * om, xs[m], e);
                if (om == 0.0) continue;
                const uint32_t pat = pats[m];
                for (uint32_t ra = pat; ra; ra &= ra - 1) {
                    const int a = __ffs(ra) - 1;
                    for (uint32_t rb = ~pat & ((N >= 32) ? 0xFFFFFFFFu : ((1u << N) - 1u)); rb; rb &= rb - 1) {
                        const int b = __ffs(rb) - 1;
                        const uint32_t mp = pat ^ (1u << a) ^ (1u << b);
                        if (mp <= pat) continue;  // each pair once
                        uint32_t j = 0, t = 1;    // colex rank of mp among the patterns
                        for (uint32_t x = mp; x; x &= x - 1) j += d_binom[__ffs(x) - 1][t++];
                        const int between = (a > b ? a - b : b - a) - 1;
                        const double h = ((between & 1) ? -1.0 : 1.0) * Kx[orb[a] * n + orb[b]];
                        off = fma(om * Oi[j], h, off);
                    }
                }
            }
            out[zoff + (int64_t)cf * f + i] = e + 2.0 * off;
        }
    }
}

// Configuration groups of the current state and target spin (rebuilt when either changes)
void ensure_csf(Context& c) {
    const int twoS = c.multiplicity - 1, twoMs = c.na - c.nb;
    if (c.csf_ready && c.csf_twoS == twoS) return;
    FCIB_CHECK(c.multiplicity >= 1, FCIB_ERR_ARG, "spin adaptation needs the multiplicity of the target state");
    FCIB_CHECK(twoS >= std::abs(twoMs) && (twoS - twoMs) % 2 == 0, FCIB_ERR_ARG,
               "spin adaptation: multiplicity incompatible with the number of alpha and beta electrons");
    const int n = c.n, nd_occ_max = std::min(c.na, c.nb);
    std::vector<std::vector<uint32_t>> byN(n + 1);
    for (int d = 0; d <= nd_occ_max; d++) {
        const int N = c.na + c.nb - 2 * d;
        if (N > n - d) continue;
        const uint32_t full = (n >= 32) ? 0xFFFFFFFFu : ((1u << n) - 1u);
        const int64_t nD = host_binom().c[n][d];
        for (int64_t di = 0; di < nD; di++) {
            const uint32_t D = host_unrank((uint32_t)di, n, d);
            const uint32_t free_m = full & ~D;
            const int64_t nO = host_binom().c[n - d][N];
            for (int64_t oi = 0; oi < nO; oi++) {
                // oi-th N-subset of the free orbitals
                const uint32_t sub = host_unrank((uint32_t)oi, n - d, N);
                uint32_t Om = 0, fm = free_m;
                for (int k = 0; k < n - d; k++) {
                    const uint32_t bit = fm & (0u - fm);
                    fm ^= bit;
                    if (sub >> k & 1u) Om |= bit;
                }
                int h = 0;
                for (int p = 0; p < n; p++)
                    if (Om >> p & 1u) h ^= c.orbsym[p];
                if (h != c.irrep) continue;
                // GAS: the electrons of a space are a function of the configuration
                bool in_gas = true;
                for (int k = 0; k < c.gas.ngas && in_gas; k++) {
                    const int e = 2 * __builtin_popcount(D & c.gas.orbs[k]) + __builtin_popcount(Om & c.gas.orbs[k]);
                    in_gas = e >= c.gas.emin[k] && e <= c.gas.emax[k];
                }
                if (!in_gas) continue;
                byN[N].push_back(D);
                byN[N].push_back(Om);
            }
        }
    }
    c.csf.clear();
    c.ncsf = 0;
    for (int N = 0; N <= n; N++) {
        if (byN[N].empty()) continue;
        c.csf.emplace_back(new CsfGroup());
        CsfGroup& g = *c.csf.back();
        std::vector<double> O;
        std::vector<uint32_t> pats;
        csf_coupling(N, twoS, twoMs, O, pats, g.f, g.nd);
        g.N = N;
        g.nconf = (int)(byN[N].size() / 2);
        g.zoff = c.ncsf;
        g.conf.upload(byN[N], c.stream);
        g.pats.upload(pats, c.stream);
        if (!O.empty()) g.O.upload(O, c.stream);
        c.ncsf += (int64_t)g.f * g.nconf;
    }
    FCIB_CUDA(cudaStreamSynchronize(c.stream));
    c.csf_ready = true;
    c.csf_twoS = twoS;
}

// one k_csf_map launch per configuration group
template <int MODE>
static void csf_map(Context& c, const double* in, double* out) {
    ensure_csf(c);
    for (auto& gp : c.csf) {
        CsfGroup& g = *gp;
        if (MODE != 0 && g.f == 0) continue;  // no CSF to write
        const size_t smem = (size_t)g.nd * 16 + (size_t)g.f * 8;
        FCIB_CHECK(smem + 1024 <= (size_t)c.smem_optin, FCIB_ERR_UNSUPPORTED, "spin adaptation: configuration too large");
        FCIB_CUDA(cudaFuncSetAttribute(k_csf_map<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const int grid = std::min(g.nconf, 8 * c.num_sms);
        k_csf_map<MODE><<<grid, g.nd > 64 ? 256 : 64, smem, c.stream>>>(
            in, out, g.conf.p, g.nconf, g.N, g.nd, g.f, g.pats.p, g.f > 0 ? g.O.p : nullptr, c.n, (int)c.nbs,
            sym_dev(c), g.zoff);
        FCIB_KCHECK();
    }
}

void csf_to_det(Context& c, const double* z, double* x) {
    // a masked layout also holds determinants that no configuration covers
    if (c.mask.p) FCIB_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * c.nvec, c.stream));
    csf_map<0>(c, z, x);
}
void det_to_csf(Context& c, const double* x, double* z) { csf_map<1>(c, x, z); }
void csf_hdiag(Context& c, double* out) {
    if (!c.opt.spin_adapt_full_preconditioner) {
        csf_map<2>(c, c.hdiag.p, out);
        return;
    }
    ensure_csf(c);
    const int n = c.n;
    std::vector<double> kx((size_t)n * n);
    const size_t n2 = (size_t)n * n, n3 = n2 * n;
    for (int p = 0; p < n; p++)
        for (int q = 0; q < n; q++) kx[(size_t)p * n + q] = c.tei_ab[p * n3 + q * n2 + q * n + p];  // <pq|qp>
    DBuf<double> Kx;
    Kx.upload(kx, c.stream);
    for (auto& gp : c.csf) {
        CsfGroup& g = *gp;
        if (g.f == 0) continue;
        const size_t smem = (size_t)g.nd * 8;
        FCIB_CHECK(smem + 1024 <= (size_t)c.smem_optin, FCIB_ERR_UNSUPPORTED, "spin adaptation: configuration too large");
        FCIB_CUDA(cudaFuncSetAttribute(k_csf_full_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const int grid = std::min(g.nconf, 8 * c.num_sms);
        k_csf_full_diag<<<grid, 128, smem, c.stream>>>(c.hdiag.p, out, g.conf.p, g.nconf, g.N, g.nd, g.f, g.pats.p,
                                                       g.O.p, n, (int)c.nbs, sym_dev(c), g.zoff, Kx.p);
        FCIB_KCHECK();
    }
    FCIB_CUDA(cudaStreamSynchronize(c.stream));  // Kx goes out of scope
}

}  // namespace fcib

// Host-only access to the coupling matrix (no device needed): O[f][nd] and the spin patterns.
// Returns FCIB_ERR_ARG when the sizes do not fit the caller's capacity cap (f * nd and nd).
extern "C" int fcib_csf_coupling(int N, int twoS, int twoMs, int cap, double* O, uint32_t* pats, int* f, int* nd) {
    if (N < 0 || N > 20 || !f || !nd) return FCIB_ERR_ARG;
    std::vector<double> o;
    std::vector<uint32_t> p;
    fcib::csf_coupling(N, twoS, twoMs, o, p, *f, *nd);
    if ((size_t)cap < o.size() || (size_t)cap < p.size()) return FCIB_ERR_ARG;
    if (O) std::copy(o.begin(), o.end(), O);
    if (pats) std::copy(p.begin(), p.end(), pats);
    return FCIB_OK;
}
