// extern "C" boundary of the engine (declared in include/fcib.h).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "fcib_internal.h"

struct fcib_ctx {
    fcib::Context c;
};

namespace fcib {

unsigned long long g_launch_count = 0;
static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }

template <typename F>
static int guarded(fcib_ctx* ctx, F&& f) {
    try {
        if (ctx) FCIB_CUDA(cudaSetDevice(ctx->c.device));
        f();
        return FCIB_OK;
    } catch (const Error& e) {
        set_error(e.msg);
        return e.code;
    } catch (const std::exception& e) {
        set_error(e.what());
        return FCIB_ERR_ARG;
    }
}

void ensure_setup(Context& c) {
    FCIB_CHECK(c.has_ints, FCIB_ERR_STATE, "integrals have not been set");
    FCIB_CHECK(c.has_state, FCIB_ERR_STATE, "state has not been set");
    if (c.tables_ready) return;
    c.mlp_tables_ready = false;
    c.csf_ready = false;
    FCIB_CHECK(c.na <= c.n && c.nb <= c.n, FCIB_ERR_ARG, "more electrons than orbitals");
    FCIB_CHECK(c.gas.ngas == 0 || (int)c.gas.space.size() == c.n, FCIB_ERR_STATE,
               "the GAS spaces were set for a different number of orbitals");
    bool fold = (c.na >= 1 && c.nb >= 1);
    c.tgtR16.release();
    c.vmax = 0.0f;
    build_spin_tables(c.A, c.n, c.na, !fold, c.stream);
    build_spin_tables(c.B, c.n, c.nb, !fold, c.stream);
    c.nas = c.A.nstr;
    c.nbs = c.B.nstr;
    c.ndet = c.nas * c.nbs;
    FCIB_CUDA(cudaStreamSynchronize(c.stream));
    prepare_integrals(c);
    build_sym_space(c);
    build_layout_maps(c);
    c.hdiag.alloc((size_t)c.nvec);
    compute_hdiag(c, c.hdiag.p);
    FCIB_CUDA(cudaStreamSynchronize(c.stream));
    c.tables_ready = true;
}

void sigma_dispatch(Context& c, const double* b, double* s, int precision) {
    if (precision == FCIB_PREC_FP64) sigma_fp64(c, b, s);
    else if (precision == FCIB_PREC_MIXED) sigma_mixed(c, b, s, true);
    else if (precision == FCIB_PREC_MIXED_TF32) sigma_mixed(c, b, s, false);
    else throw Error{FCIB_ERR_ARG, "unknown sigma precision"};
}

// host flat order (FCIVector, or GenCIVector with GAS) <-> device layout (C1, the blocked layout,
// or either with a mask; the flat map holds the layout index of every flat position)
static void upload_flat(Context& c, const double* flat, double* dev) {
    if (!c.mask.p) {
        FCIB_CUDA(cudaMemcpyAsync(dev, flat, sizeof(double) * c.nvec, cudaMemcpyHostToDevice, c.stream));
        return;
    }
    std::vector<double> full((size_t)c.nvec, 0.0);
    for (size_t i = 0; i < c.flat_map.size(); i++) full[c.flat_map[i]] = flat[i];
    FCIB_CUDA(cudaMemcpyAsync(dev, full.data(), sizeof(double) * c.nvec, cudaMemcpyHostToDevice, c.stream));
    FCIB_CUDA(cudaStreamSynchronize(c.stream));
}
static void download_flat(Context& c, const double* dev, double* flat) {
    if (!c.mask.p) {
        FCIB_CUDA(cudaMemcpyAsync(flat, dev, sizeof(double) * c.nvec, cudaMemcpyDeviceToHost, c.stream));
        FCIB_CUDA(cudaStreamSynchronize(c.stream));
        return;
    }
    std::vector<double> full((size_t)c.nvec);
    FCIB_CUDA(cudaMemcpyAsync(full.data(), dev, sizeof(double) * c.nvec, cudaMemcpyDeviceToHost, c.stream));
    FCIB_CUDA(cudaStreamSynchronize(c.stream));
    for (size_t i = 0; i < c.flat_map.size(); i++) flat[i] = full[c.flat_map[i]];
}
// RDM blocks -> caller buffers; spin-free sums follow FCIVector::compute_rdms
// (fci_vector_rdm.cc:120-126): G1 = g1a + g1b, G2 = (g2aa + (g2ab(pqrs) + g2ab(qpsr))) + g2bb.
static void rdms_to_outputs(const RdmBlocks& b, int level, int spin_free, double* g1a, double* g1b, double* g2aa,
                            double* g2ab, double* g2bb) {
    const int n = b.n;
    const size_t nn = (size_t)n * n, n4 = nn * nn;
    if (!spin_free) {
        if (g1a) std::copy(b.g1a.begin(), b.g1a.end(), g1a);
        if (g1b) std::copy(b.g1b.begin(), b.g1b.end(), g1b);
        if (level >= 2) {
            if (g2aa) std::copy(b.g2aa.begin(), b.g2aa.end(), g2aa);
            if (g2ab) std::copy(b.g2ab.begin(), b.g2ab.end(), g2ab);
            if (g2bb) std::copy(b.g2bb.begin(), b.g2bb.end(), g2bb);
        }
        return;
    }
    if (g1a)
        for (size_t i = 0; i < nn; i++) g1a[i] = b.g1a[i] + b.g1b[i];
    if (level >= 2 && g2aa) {
        for (int p = 0; p < n; p++)
            for (int q = 0; q < n; q++)
                for (int r = 0; r < n; r++)
                    for (int s = 0; s < n; s++) {
                        const size_t x = (((size_t)p * n + q) * n + r) * n + s;
                        const size_t y = (((size_t)q * n + p) * n + s) * n + r;
                        g2aa[x] = (b.g2aa[x] + (b.g2ab[x] + b.g2ab[y])) + b.g2bb[x];
                    }
    }
    (void)n4;
}
// masked layouts (a mask is allocated) map every flat position; otherwise the layout is the flat order
static int64_t flat_size(const Context& c) { return c.mask.p ? (int64_t)c.flat_map.size() : c.nvec; }

}  // namespace fcib

using namespace fcib;

extern "C" {

void fcib_default_options(fcib_options* o) {
    if (!o) return;
    o->maxiter = 100;
    o->e_convergence = 1.0e-9;
    o->r_convergence = 1.0e-6;
    o->guess_per_root = 1;
    o->dets_per_guess = 50;
    o->collapse_per_root = 2;
    o->subspace_per_root = 10;
    o->die_if_not_converged = 0;
    o->print = 0;
    o->precision = FCIB_PREC_FP64;
    o->preconditioner = FCIB_PRECOND_DIAG;
    o->mixed_switch = 1.0e-4;
    o->same_spin_kernel = FCIB_SAME_TC;
    o->spin_adapt = 0;
    o->sym_blocked = 1;
    o->spin_adapt_full_preconditioner = 0;
}

const char* fcib_last_error(void) { return g_last_error.c_str(); }
const char* fcib_version(void) { return "fcib 0.1 (sm_100a)"; }

int fcib_create(fcib_ctx** out, int device) {
    if (!out) {
        set_error("fcib_create: null output pointer");
        return FCIB_ERR_ARG;
    }
    *out = nullptr;
    fcib_ctx* ctx = new fcib_ctx();
    int rc = guarded(nullptr, [&] {
        int ndev = 0;
        FCIB_CUDA(cudaGetDeviceCount(&ndev));
        FCIB_CHECK(device >= 0 && device < ndev, FCIB_ERR_ARG, "fcib_create: no such CUDA device");
        FCIB_CUDA(cudaSetDevice(device));
        cudaDeviceProp prop;
        FCIB_CUDA(cudaGetDeviceProperties(&prop, device));
        FCIB_CHECK(prop.major == 10, FCIB_ERR_UNSUPPORTED, "fcib requires an sm_100 (B200) device");
        ctx->c.device = device;
        ctx->c.num_sms = prop.multiProcessorCount;
        ctx->c.smem_optin = (int)prop.sharedMemPerBlockOptin;
        ctx->c.smem_per_sm = (int)prop.sharedMemPerMultiprocessor;
        FCIB_CUDA(cudaStreamCreateWithFlags(&ctx->c.stream, cudaStreamNonBlocking));
        fcib_default_options(&ctx->c.opt);
    });
    if (rc != FCIB_OK) {
        delete ctx;
        return rc;
    }
    *out = ctx;
    return FCIB_OK;
}

int fcib_destroy(fcib_ctx* ctx) {
    if (!ctx) return FCIB_OK;
    cudaSetDevice(ctx->c.device);
    cudaStreamSynchronize(ctx->c.stream);
    cudaStream_t s = ctx->c.stream;
    delete ctx;
    if (s) cudaStreamDestroy(s);
    return FCIB_OK;
}

int fcib_set_integrals(fcib_ctx* ctx, int n, int nirrep, const int* orbsym, double scalar,
                       const double* oei_a, const double* oei_b, const double* tei_aa,
                       const double* tei_ab, const double* tei_bb) {
    if (!ctx) { set_error("null context"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        FCIB_CHECK(n >= 1 && n <= kMaxOrb, FCIB_ERR_UNSUPPORTED, "number of active orbitals must be 1..22");
        FCIB_CHECK(nirrep >= 1 && nirrep <= 8, FCIB_ERR_ARG, "nirrep must be 1..8");
        FCIB_CHECK(oei_a && oei_b && tei_aa && tei_ab && tei_bb, FCIB_ERR_ARG, "null integral pointer");
        FCIB_CHECK(std::isfinite(scalar), FCIB_ERR_NUMERIC, "scalar energy is not finite");
        Context& c = ctx->c;
        const size_t n2 = (size_t)n * n, n4 = n2 * n2;
        c.n = n;
        c.nirrep = nirrep;
        c.orbsym.assign(n, 0);
        if (orbsym)
            for (int i = 0; i < n; i++) {
                FCIB_CHECK(orbsym[i] >= 0 && orbsym[i] < nirrep, FCIB_ERR_ARG, "orbital irrep out of range");
                c.orbsym[i] = orbsym[i];
            }
        c.scalar = scalar;
        c.oei_a.assign(oei_a, oei_a + n2);
        c.oei_b.assign(oei_b, oei_b + n2);
        c.tei_aa.assign(tei_aa, tei_aa + n4);
        c.tei_ab.assign(tei_ab, tei_ab + n4);
        c.tei_bb.assign(tei_bb, tei_bb + n4);
        double mx = 0.0, dev = 0.0;
        for (size_t i = 0; i < n4; i++) {
            FCIB_CHECK(std::isfinite(c.tei_ab[i]) && std::isfinite(c.tei_aa[i]) && std::isfinite(c.tei_bb[i]),
                       FCIB_ERR_NUMERIC, "two-electron integrals contain non-finite values");
            mx = std::max(mx, std::fabs(c.tei_ab[i]));
        }
        for (size_t i = 0; i < n2; i++)
            FCIB_CHECK(std::isfinite(c.oei_a[i]) && std::isfinite(c.oei_b[i]), FCIB_ERR_NUMERIC,
                       "one-electron integrals contain non-finite values");
        // real-orbital symmetry used by the pair-symmetrised sigma: (pq|rs) = (qp|rs) = (rs|pq)
        auto tab = [&](int p, int q, int r, int s) { return c.tei_ab[((size_t)p * n + q) * n2 + r * n + s]; };
        for (int p = 0; p < n; p++)
            for (int q = 0; q < n; q++) {
                dev = std::max(dev, std::fabs(c.oei_a[p * n + q] - c.oei_a[q * n + p]));
                dev = std::max(dev, std::fabs(c.oei_b[p * n + q] - c.oei_b[q * n + p]));
                for (int r = 0; r < n; r++)
                    for (int s = 0; s < n; s++) {
                        double v = tab(p, r, q, s);  // (pq|rs)
                        dev = std::max(dev, std::fabs(v - tab(q, r, p, s)));
                        dev = std::max(dev, std::fabs(v - tab(r, p, s, q)));
                    }
            }
        FCIB_CHECK(dev <= 1e-10 * std::max(1.0, mx), FCIB_ERR_UNSUPPORTED,
                   "integrals must be real with 8-fold symmetry (h_pq = h_qp, (pq|rs) = (qp|rs) = (rs|pq))");
        c.has_ints = true;
        c.tables_ready = false;
        c.solved = false;
    });
}

int fcib_set_state(fcib_ctx* ctx, int na, int nb, int irrep, int multiplicity, int nroot, int root) {
    if (!ctx) { set_error("null context"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        Context& c = ctx->c;
        FCIB_CHECK(c.has_ints, FCIB_ERR_STATE, "set integrals before the state");
        FCIB_CHECK(na >= 0 && nb >= 0 && na <= c.n && nb <= c.n, FCIB_ERR_ARG, "electron counts out of range");
        FCIB_CHECK(irrep >= 0 && irrep < c.nirrep, FCIB_ERR_ARG, "target irrep out of range");
        FCIB_CHECK(multiplicity >= 0, FCIB_ERR_ARG, "multiplicity must be >= 1 (0 = no spin selection in the guess)");
        FCIB_CHECK(nroot >= 1, FCIB_ERR_ARG, "nroot must be >= 1");
        FCIB_CHECK(root >= 0 && root < nroot, FCIB_ERR_ARG, "root must be < nroot");
        bool same = (c.na == na && c.nb == nb && c.irrep == irrep);
        c.na = na; c.nb = nb; c.irrep = irrep; c.multiplicity = multiplicity;
        c.nroot = nroot; c.root = root;
        c.has_state = true;
        if (!same) c.tables_ready = false;
        c.solved = false;
    });
}

// GenCISolver's determinant space (forte/genci/genci_solver.h; the GAS spaces of MOSpaceInfo and the
// bounds of StateInfo::gas_min/gas_max)
int fcib_set_gas(fcib_ctx* ctx, int ngas, const int* space, const int* gas_min, const int* gas_max) {
    if (!ctx) { set_error("null context"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        Context& c = ctx->c;
        FCIB_CHECK(c.has_ints, FCIB_ERR_STATE, "set integrals before the GAS spaces");
        FCIB_CHECK(ngas >= 0 && ngas <= kMaxGas, FCIB_ERR_ARG, "the number of GAS spaces must be 0..6");
        GasSpace g;
        if (ngas > 0) {
            FCIB_CHECK(space && gas_min && gas_max, FCIB_ERR_ARG, "null argument");
            g.ngas = ngas;
            g.space.assign(space, space + c.n);
            for (int p = 0; p < c.n; p++) {
                FCIB_CHECK(space[p] >= 0 && space[p] < ngas, FCIB_ERR_ARG, "orbital GAS space out of range");
                g.orbs[space[p]] |= 1u << p;
            }
            for (int k = 0; k < ngas; k++) {
                FCIB_CHECK(g.orbs[k] != 0u, FCIB_ERR_ARG, "every GAS space needs at least one orbital");
                FCIB_CHECK(gas_min[k] >= 0 && gas_max[k] >= 0, FCIB_ERR_ARG, "GAS electron bounds must be >= 0");
                g.emin[k] = gas_min[k];
                g.emax[k] = gas_max[k];
            }
        }
        c.gas = std::move(g);
        c.tables_ready = false;  // the layout maps, stored vectors and the restart state go
        c.solved = false;
        c.dl_prev = false;
        c.csf_ready = false;
    });
}

// FCIStringLists / GenCIStringLists::make_determinants: the strings of every flat position
int fcib_determinants(fcib_ctx* ctx, uint32_t* alfa, uint32_t* beta) {
    if (!ctx || !alfa || !beta) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        Context& c = ctx->c;
        ensure_setup(c);
        std::vector<uint32_t> sa(c.nas), sb(c.nbs);
        FCIB_CUDA(cudaMemcpy(sa.data(), c.A.str.p, 4 * c.nas, cudaMemcpyDeviceToHost));
        FCIB_CUDA(cudaMemcpy(sb.data(), c.B.str.p, 4 * c.nbs, cudaMemcpyDeviceToHost));
        const int64_t nf = flat_size(c);
        for (int64_t f = 0; f < nf; f++) {
            const int64_t I = c.mask.p ? c.flat_map[f] : f;
            int64_t ia, ib;
            if (c.sym.on) {
                sym_host_decode(c, I, ia, ib);
            } else {
                ia = I / c.nbs;
                ib = I % c.nbs;
            }
            alfa[f] = sa[ia];
            beta[f] = sb[ib];
        }
    });
}

int fcib_set_options(fcib_ctx* ctx, const fcib_options* o) {
    if (!ctx || !o) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        FCIB_CHECK(o->maxiter >= 1, FCIB_ERR_ARG, "maxiter must be >= 1");
        FCIB_CHECK(o->e_convergence > 0 && o->r_convergence > 0, FCIB_ERR_ARG, "convergence thresholds must be > 0");
        FCIB_CHECK(o->guess_per_root >= 1 && o->dets_per_guess >= 1, FCIB_ERR_ARG, "guess options must be >= 1");
        FCIB_CHECK(o->collapse_per_root >= 1, FCIB_ERR_ARG,
                   "DavidsonLiuSolver: collapse_per_root must be greater or equal to one");
        FCIB_CHECK(o->subspace_per_root >= o->collapse_per_root + 1, FCIB_ERR_ARG,
                   "DavidsonLiuSolver: subspace_per_root must be greater or equal to collapse_per_root + 1");
        FCIB_CHECK(o->precision >= FCIB_PREC_FP64 && o->precision <= FCIB_PREC_MIXED_TF32, FCIB_ERR_ARG, "bad precision mode");
        FCIB_CHECK(o->preconditioner == FCIB_PRECOND_DIAG || o->preconditioner == FCIB_PRECOND_MLP, FCIB_ERR_ARG,
                   "bad preconditioner");
        FCIB_CHECK(o->same_spin_kernel == FCIB_SAME_TC || o->same_spin_kernel == FCIB_SAME_CUDA_CORES, FCIB_ERR_ARG,
                   "bad same-spin kernel");
        Context& c = ctx->c;
        if ((o->sym_blocked != 0) != (c.opt.sym_blocked != 0)) {
            // the vector layout changes: tables, stored vectors and the restart state go
            c.tables_ready = false;
            c.solved = false;
            c.dl_prev = false;
        }
        c.opt = *o;
    });
}

int fcib_size(fcib_ctx* ctx, int64_t* ndet) {
    if (!ctx || !ndet) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        ensure_setup(ctx->c);
        *ndet = flat_size(ctx->c);
    });
}

int fcib_layout_size(fcib_ctx* ctx, int64_t* n) {
    if (!ctx || !n) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        ensure_setup(ctx->c);
        *n = ctx->c.nvec;
    });
}

// SpinAdapter::ncsf (ci_spin_adaptation.h:81-183): CSFs of the state's multiplicity in the target irrep
int fcib_ncsf(fcib_ctx* ctx, int64_t* ncsf) {
    if (!ctx || !ncsf) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        ensure_setup(ctx->c);
        ensure_csf(ctx->c);
        *ncsf = ctx->c.ncsf;
    });
}

// CSF <-> determinant transforms and the CSF diagonal for host vectors (flat order)
int fcib_csf_to_det(fcib_ctx* ctx, const double* z, double* cv) {
    if (!ctx || !z || !cv) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        Context& c = ctx->c;
        ensure_setup(c);
        ensure_csf(c);
        DBuf<double> dz, dx;
        dz.upload(z, (size_t)c.ncsf, c.stream);
        dx.alloc((size_t)c.nvec);
        csf_to_det(c, dz.p, dx.p);
        download_flat(c, dx.p, cv);
    });
}

int fcib_det_to_csf(fcib_ctx* ctx, const double* cv, double* z) {
    if (!ctx || !cv || !z) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        Context& c = ctx->c;
        ensure_setup(c);
        ensure_csf(c);
        DBuf<double> dz, dx;
        dx.alloc((size_t)c.nvec);
        upload_flat(c, cv, dx.p);
        dz.alloc((size_t)c.ncsf);
        det_to_csf(c, dx.p, dz.p);
        FCIB_CUDA(cudaMemcpyAsync(z, dz.p, sizeof(double) * c.ncsf, cudaMemcpyDeviceToHost, c.stream));
        FCIB_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int fcib_csf_hdiag(fcib_ctx* ctx, int full, double* out) {
    if (!ctx || !out) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        Context& c = ctx->c;
        ensure_setup(c);
        ensure_csf(c);
        const int keep = c.opt.spin_adapt_full_preconditioner;
        c.opt.spin_adapt_full_preconditioner = full ? 1 : 0;
        DBuf<double> d;
        d.alloc((size_t)c.ncsf);
        try {
            csf_hdiag(c, d.p);
        } catch (...) {
            c.opt.spin_adapt_full_preconditioner = keep;
            throw;
        }
        c.opt.spin_adapt_full_preconditioner = keep;
        FCIB_CUDA(cudaMemcpyAsync(out, d.p, sizeof(double) * c.ncsf, cudaMemcpyDeviceToHost, c.stream));
        FCIB_CUDA(cudaStreamSynchronize(c.stream));
    });
}

static void print_solutions(Context& c);

int fcib_solve(fcib_ctx* ctx, double* energies, double* spin2, int* iterations) {
    if (!ctx) { set_error("null context"); return FCIB_ERR_ARG; }
    int rc = guarded(ctx, [&] {
        Context& c = ctx->c;
        ensure_setup(c);
        dl_solve(c);
        for (int k = 0; k < c.nroot; k++) {
            if (energies) energies[k] = c.energies[k];
            if (spin2) spin2[k] = c.spin2[k];
        }
        if (iterations) *iterations = c.iterations;
        if (c.opt.print >= 1 && (c.converged || !c.opt.die_if_not_converged)) print_solutions(c);
    });
    if (rc == FCIB_OK && !ctx->c.converged && ctx->c.opt.die_if_not_converged) {
        // the reference's message (forte/fci/fci_solver.cc:269-276)
        set_error("Davidson-Liu solver did not converge.\nPlease try to increase the number of "
                  "Davidson-Liu iterations (DL_MAXITER). You can also try to increase:\n - the "
                  "maximum "
                  "size of the subspace (DL_SUBSPACE_PER_ROOT)"
                  "\n - the number of guess states (DL_GUESS_PER_ROOT)");
        return FCIB_ERR_NOT_CONVERGED;
    }
    return rc;
}

// FCIVector::max_abs_elements (forte/fci/fci_vector_h_diag.cc:37-68): the num_dets largest |C| of a
// root in the reference's order (descending |C|; equal values in FCIVector flat order, which the
// reference's insertion keeps), each as (|C|, C, alpha irrep, alpha and beta string address within
// their irreps); slots past the nonzero elements hold zeros, as the reference's preset tuples do.
static void max_abs_elements(Context& c, int root, int num_dets, std::vector<double>& absv, std::vector<double>& val,
                             std::vector<int>& irr, std::vector<int64_t>& ia, std::vector<int64_t>& ib) {
    const int64_t N = c.nvec;
    const int64_t nflat = flat_size(c);
    num_dets = (int)std::min<int64_t>(num_dets, nflat);
    absv.assign(num_dets, 0.0);
    val.assign(num_dets, 0.0);
    irr.assign(num_dets, 0);
    ia.assign(num_dets, 0);
    ib.assign(num_dets, 0);
    if (num_dets <= 0) return;
    const double* x = root_vector(c, root);
    DBuf<double> kb;
    kb.alloc((size_t)N);
    double* keys = kb.p;
    k_neg_abs<<<4 * c.num_sms, 256, 0, c.stream>>>(x, keys, (size_t)N);
    FCIB_KCHECK();
    auto sel = lowest_keys(c, keys, num_dets);
    // C1 index -> (alpha irrep, addresses within the irrep blocks, FCIVector flat position)
    std::vector<uint32_t> sa(c.nas), sb(c.nbs);
    FCIB_CUDA(cudaMemcpy(sa.data(), c.A.str.p, 4 * c.nas, cudaMemcpyDeviceToHost));
    FCIB_CUDA(cudaMemcpy(sb.data(), c.B.str.p, 4 * c.nbs, cudaMemcpyDeviceToHost));
    auto sym = [&](uint32_t s) {
        int h = 0;
        for (int i = 0; i < c.n; i++)
            if (s >> i & 1u) h ^= c.orbsym[i];
        return h;
    };
    std::vector<int> ha(c.nas), hb(c.nbs);
    std::vector<int64_t> ra(c.nas), rb(c.nbs), pa(c.nas), pb(c.nbs);
    {
        std::vector<int64_t> cnta(8, 0), cntb(8, 0);
        for (int64_t i = 0; i < c.nas; i++) { ha[i] = c.nirrep > 1 ? sym(sa[i]) : 0; ra[i] = cnta[ha[i]]++; }
        for (int64_t i = 0; i < c.nbs; i++) { hb[i] = c.nirrep > 1 ? sym(sb[i]) : 0; rb[i] = cntb[hb[i]]++; }
        // start of each alpha irrep block in flat order
        std::vector<int64_t> blk(9, 0);
        for (int h = 0; h < 8; h++) blk[h + 1] = blk[h] + cnta[h] * cntb[h ^ (c.nirrep > 1 ? c.irrep : 0)];
        for (int64_t i = 0; i < c.nas; i++) pa[i] = blk[ha[i]] + ra[i] * cntb[ha[i] ^ (c.nirrep > 1 ? c.irrep : 0)];
    }
    // vector index -> (flat position, alpha irrep, addresses within the irrep blocks); the flat
    // position (FCIVector order, or GenCIVector order with GAS) orders equal |C|
    auto locate = [&](int64_t idx, int64_t& flat, int& h, int64_t& ai, int64_t& bi) {
        if (c.sym.on) {  // the blocked layout is the FCIVector flat order (without GAS spaces)
            flat = idx;
            int64_t i, j;  // string indices (the blocks of a GAS layout hold a subset of the strings)
            sym_host_decode(c, idx, i, j);
            h = ha[i];
            ai = ra[i];
            bi = rb[j];
        } else {
            const int64_t i = idx / c.nbs, j = idx % c.nbs;
            flat = pa[i] + rb[j];
            h = ha[i];
            ai = ra[i];
            bi = rb[j];
        }
        if (c.gas.ngas > 0) flat = gas_flat_position(c, idx);
    };
    std::vector<std::pair<std::pair<double, int64_t>, int64_t>> order;  // ((-|C|, flat), vector index)
    for (auto& e : sel) {
        int64_t flat, ai, bi;
        int h;
        locate(e.second, flat, h, ai, bi);
        order.push_back({{e.first, flat}, e.second});
    }
    std::sort(order.begin(), order.end());
    std::vector<double> h(order.size());
    for (size_t t = 0; t < order.size(); t++)
        FCIB_CUDA(cudaMemcpyAsync(&h[t], x + order[t].second, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    FCIB_CUDA(cudaStreamSynchronize(c.stream));
    for (int t = 0; t < num_dets && t < (int)order.size(); t++) {
        const double a = -order[t].first.first;
        if (!(a > 0.0)) break;
        int64_t flat, ai, bi;
        int hh;
        locate(order[t].second, flat, hh, ai, bi);
        absv[t] = a;
        val[t] = h[t];
        irr[t] = hh;
        ia[t] = ai;
        ib[t] = bi;
    }
}

// FCISolver::print_solutions (forte/fci/fci_solver.cc:316-367): per root, the determinants with
// |C| >= 0.01 among the 100 largest, as occupation strings per irrep block (2, a, b, 0), then the
// root's energy and <S^2>.
static void print_solutions(Context& c) {
    std::vector<double> absv, val;
    std::vector<int> irr;
    std::vector<int64_t> ia, ib;
    std::vector<uint32_t> sa(c.nas), sb(c.nbs);
    FCIB_CUDA(cudaMemcpy(sa.data(), c.A.str.p, 4 * c.nas, cudaMemcpyDeviceToHost));
    FCIB_CUDA(cudaMemcpy(sb.data(), c.B.str.p, 4 * c.nbs, cudaMemcpyDeviceToHost));
    // strings of each irrep in string order, to turn (irrep, address) back into a string
    auto sym = [&](uint32_t s) {
        int h = 0;
        for (int i = 0; i < c.n; i++)
            if (s >> i & 1u) h ^= c.orbsym[i];
        return h;
    };
    std::vector<std::vector<uint32_t>> bya(8), byb(8);
    for (auto s : sa) bya[c.nirrep > 1 ? sym(s) : 0].push_back(s);
    for (auto s : sb) byb[c.nirrep > 1 ? sym(s) : 0].push_back(s);
    for (int r = 0; r < c.nroot; r++) {
        printf("\n\n  ==> Root No. %d <==\n", r);
        max_abs_elements(c, r, 100, absv, val, irr, ia, ib);
        for (size_t t = 0; t < absv.size(); t++) {
            if (absv[t] < 0.01) continue;
            const uint32_t A = bya[irr[t]][ia[t]];
            const uint32_t B = byb[irr[t] ^ (c.nirrep > 1 ? c.irrep : 0)][ib[t]];
            printf("\n    ");
            for (int h = 0; h < std::max(1, c.nirrep); h++) {
                int cnt = 0;
                for (int i = 0; i < c.n; i++) {
                    if ((c.nirrep > 1 ? c.orbsym[i] : 0) != h) continue;
                    const bool a = A >> i & 1u, b = B >> i & 1u;
                    if (a == b) printf("%d", a ? 2 : 0);
                    else printf("%c", a ? 'a' : 'b');
                    cnt++;
                }
                if (cnt) printf(" ");
            }
            printf("%15.8f", val[t]);
        }
        printf("\n\n    Total Energy: %20.12f, <S^2>: %8.6f", c.energies[r], c.spin2[r]);
    }
    printf("\n");
    fflush(stdout);
}

int fcib_reset_guess(fcib_ctx* ctx) {
    if (!ctx) { set_error("null context"); return FCIB_ERR_ARG; }
    ctx->c.dl_prev = false;
    return FCIB_OK;
}

int fcib_max_abs_elements(fcib_ctx* ctx, int root, int num_dets, double* abs_c, double* c_out, int* alfa_irrep,
                          int64_t* alfa_address, int64_t* beta_address, int* count) {
    if (!ctx) { set_error("null context"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        Context& c = ctx->c;
        FCIB_CHECK(c.solved, FCIB_ERR_STATE, "no solution available");
        FCIB_CHECK(root >= 0 && root < c.nroot, FCIB_ERR_ARG, "root out of range");
        FCIB_CHECK(num_dets >= 0, FCIB_ERR_ARG, "negative determinant count");
        std::vector<double> a, v;
        std::vector<int> h;
        std::vector<int64_t> ia, ib;
        max_abs_elements(c, root, num_dets, a, v, h, ia, ib);
        for (size_t t = 0; t < a.size(); t++) {
            if (abs_c) abs_c[t] = a[t];
            if (c_out) c_out[t] = v[t];
            if (alfa_irrep) alfa_irrep[t] = h[t];
            if (alfa_address) alfa_address[t] = ia[t];
            if (beta_address) beta_address[t] = ib[t];
        }
        if (count) *count = (int)a.size();
    });
}

int fcib_get_vector(fcib_ctx* ctx, int root, double* out) {
    if (!ctx || !out) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        Context& c = ctx->c;
        FCIB_CHECK(c.solved, FCIB_ERR_STATE, "no solution available");
        FCIB_CHECK(root >= 0 && root < c.nroot, FCIB_ERR_ARG, "root out of range");
        download_flat(c, root_vector(c, root), out);
    });
}

int fcib_sigma(fcib_ctx* ctx, const double* b, double* sigma) {
    if (!ctx || !b || !sigma) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        Context& c = ctx->c;
        ensure_setup(c);
        DBuf<double> db, ds;
        db.alloc(c.nvec);
        ds.alloc(c.nvec);
        upload_flat(c, b, db.p);
        sigma_dispatch(c, db.p, ds.p, c.opt.precision);
        download_flat(c, ds.p, sigma);
    });
}

int fcib_sigma_device(fcib_ctx* ctx, const double* d_b, double* d_sigma, int precision, void* stream) {
    if (!ctx || !d_b || !d_sigma) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        Context& c = ctx->c;
        ensure_setup(c);
        cudaStream_t keep = c.stream;
        if (stream) c.stream = (cudaStream_t)stream;
        try {
            sigma_dispatch(c, d_b, d_sigma, precision);
        } catch (...) {
            c.stream = keep;
            throw;
        }
        c.stream = keep;
    });
}

int fcib_hdiag(fcib_ctx* ctx, double* out) {
    if (!ctx || !out) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        ensure_setup(ctx->c);
        download_flat(ctx->c, ctx->c.hdiag.p, out);
    });
}

int fcib_spin2(fcib_ctx* ctx, const double* cvec, double* s2) {
    if (!ctx || !cvec || !s2) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        Context& c = ctx->c;
        ensure_setup(c);
        DBuf<double> d;
        d.alloc(c.nvec);
        upload_flat(c, cvec, d.p);
        *s2 = spin2_device(c, d.p);
    });
}

int fcib_rdms(fcib_ctx* ctx, int root_left, int root_right, int level, int spin_free, double* g1a,
              double* g1b, double* g2aa, double* g2ab, double* g2bb) {
    if (!ctx) { set_error("null context"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        Context& c = ctx->c;
        FCIB_CHECK(c.solved, FCIB_ERR_STATE, "FCIVector is not assigned. Cannot compute RDMs.");
        FCIB_CHECK(root_left >= 0 && root_right >= 0, FCIB_ERR_ARG, "negative root index");
        if (std::max(root_left, root_right) >= c.nroot)
            throw Error{FCIB_ERR_ARG, "Cannot compute RDMs <" + std::to_string(root_left) + "| ... |" +
                                          std::to_string(root_right) + "> (0-based) because nroot = " +
                                          std::to_string(c.nroot)};
        FCIB_CHECK(level <= 3, FCIB_ERR_UNSUPPORTED, "RDMs of order higher than 3 are not available");
        if (level <= 0) return;
        level = std::min(level, 2);  // the three-body blocks come from fcib_rdms3
        RdmBlocks blk;
        DBuf<double> xl, xr;
        const double* L = c1_view(c, root_vector(c, root_left), xl);
        const double* R = root_right == root_left ? L : c1_view(c, root_vector(c, root_right), xr);
        compute_rdms(c, L, R, level, blk);
        rdms_to_outputs(blk, level, spin_free, g1a, g1b, g2aa, g2ab, g2bb);
    });
}

// FCISolver::transition_rdms(root_list, method2, max_rdm_level, type) for one pair
// (forte/fci/fci_solver_transition_rdms.cc:37-109) and compute_transition_rdms /
// compute_1rdm_different_irrep (fci_vector_transition_rdm.cc:43-165): <left root| a+_p a_q |right root>
// between the solutions of two contexts whose states may belong to different irreps.  Both vectors
// live on the device in the full C1 layout (zero outside each state's irrep), so the one kernel pass
// over the C1 space sums exactly the irrep blocks the reference loops over.
int fcib_transition_rdms(fcib_ctx* left, int root_left, fcib_ctx* right, int root_right, int level,
                         int spin_free, double* g1a, double* g1b) {
    if (!left || !right) { set_error("null context"); return FCIB_ERR_ARG; }
    return guarded(left, [&] {
        Context& c = left->c;
        Context& r = right->c;
        FCIB_CHECK(c.solved && r.solved, FCIB_ERR_STATE, "FCIVector is not assigned. Cannot compute RDMs.");
        FCIB_CHECK(level <= 3 && level >= 1, FCIB_ERR_ARG, "Invalid max_rdm_level, required 1 <= max_rdm_level <= 3.");
        FCIB_CHECK(root_left >= 0 && root_right >= 0, FCIB_ERR_ARG, "negative root index");
        if (root_left >= c.nroot || root_right >= r.nroot)
            throw Error{FCIB_ERR_ARG, "Cannot compute RDMs <" + std::to_string(root_left) + "| ... |" +
                                          std::to_string(root_right) + "> (0-based) because nroot_left = " +
                                          std::to_string(c.nroot) + " and nroot_right = " + std::to_string(r.nroot)};
        FCIB_CHECK(c.n == r.n, FCIB_ERR_ARG,
                   "FCI transition RDMs: The number of MOs must be the same in the two wave functions.");
        FCIB_CHECK(c.na == r.na && c.nb == r.nb, FCIB_ERR_ARG,
                   "FCI transition RDMs: The number of alfa and beta electrons must be the same in the two wave "
                   "functions.");
        FCIB_CHECK(c.device == r.device, FCIB_ERR_UNSUPPORTED, "transition RDMs: the two contexts use different devices");
        FCIB_CHECK(level < 2, FCIB_ERR_UNSUPPORTED,
                   "Transition RDMs of order 2 or higher are not implemented in FCISolver (and more generally in "
                   "Forte).");
        const int n = c.n;
        std::vector<double> a((size_t)n * n, 0.0), b((size_t)n * n, 0.0);
        // the reference returns empty blocks when the left state has no alpha electrons, for both
        // spins (compute_1rdm_different_irrep takes nb from the alpha address), and so does this call
        if (c.na >= 1) {
            // both vectors in the C1 layout, which does not depend on the irrep
            DBuf<double> xl, xr;
            const double* L = c1_view(c, root_vector(c, root_left), xl);
            const double* R = c1_view(r, root_vector(r, root_right), xr);
            FCIB_CUDA(cudaStreamSynchronize(r.stream));
            RdmBlocks blk;
            compute_rdms(c, L, R, 1, blk);
            a = blk.g1a;
            b = blk.g1b;
        }
        if (spin_free) {
            if (g1a)
                for (size_t i = 0; i < a.size(); i++) g1a[i] = a[i] + b[i];
        } else {
            if (g1a) std::copy(a.begin(), a.end(), g1a);
            if (g1b) std::copy(b.begin(), b.end(), g1b);
        }
    });
}

int fcib_compute_rdms(fcib_ctx* ctx, const double* left, const double* right, int level, int spin_free,
                      double* g1a, double* g1b, double* g2aa, double* g2ab, double* g2bb) {
    if (!ctx || !left) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        Context& c = ctx->c;
        ensure_setup(c);
        FCIB_CHECK(level <= 3, FCIB_ERR_UNSUPPORTED, "RDMs of order higher than 3 are not available");
        if (level <= 0) return;
        level = std::min(level, 2);  // the three-body blocks come from fcib_compute_rdms3
        DBuf<double> dl, dr, xl, xr;
        dl.alloc(c.nvec);
        upload_flat(c, left, dl.p);
        const double* L = c1_view(c, dl.p, xl);
        const double* R = L;
        if (right && right != left) {
            dr.alloc(c.nvec);
            upload_flat(c, right, dr.p);
            R = c1_view(c, dr.p, xr);
        }
        RdmBlocks blk;
        compute_rdms(c, L, R, level, blk);
        rdms_to_outputs(blk, level, spin_free, g1a, g1b, g2aa, g2ab, g2bb);
    });
}

// 3-RDM blocks -> caller's arrays; spin_free: G3 of FCIVector::compute_rdms (fci_vector_rdm.cc:127-130)
static void rdms3_to_outputs(const Rdm3Blocks& b, int spin_free, double* g3aaa, double* g3aab, double* g3abb,
                             double* g3bbb) {
    if (!spin_free) {
        if (g3aaa) std::copy(b.aaa.begin(), b.aaa.end(), g3aaa);
        if (g3aab) std::copy(b.aab.begin(), b.aab.end(), g3aab);
        if (g3abb) std::copy(b.abb.begin(), b.abb.end(), g3abb);
        if (g3bbb) std::copy(b.bbb.begin(), b.bbb.end(), g3bbb);
        return;
    }
    if (!g3aaa) return;
    const int n = b.n;
    auto six = [n](int p, int q, int r, int s, int t, int u) {
        return (((((size_t)p * n + q) * n + r) * n + s) * n + t) * n + u;
    };
    for (int p = 0; p < n; p++)
        for (int q = 0; q < n; q++)
            for (int r = 0; r < n; r++)
                for (int s = 0; s < n; s++)
                    for (int t = 0; t < n; t++)
                        for (int u = 0; u < n; u++) {
                            const size_t o = six(p, q, r, s, t, u);
                            double g = b.aaa[o];
                            g += b.aab[o] + b.aab[six(p, r, q, s, u, t)] + b.aab[six(q, r, p, t, u, s)];
                            g += b.abb[o] + b.abb[six(q, p, r, t, s, u)] + b.abb[six(r, p, q, u, s, t)];
                            g += b.bbb[o];
                            g3aaa[o] = g;
                        }
}

int fcib_rdms3(fcib_ctx* ctx, int root_left, int root_right, int spin_free, double* g3aaa, double* g3aab,
               double* g3abb, double* g3bbb) {
    if (!ctx) { set_error("null context"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        Context& c = ctx->c;
        FCIB_CHECK(c.solved, FCIB_ERR_STATE, "FCIVector is not assigned. Cannot compute RDMs.");
        FCIB_CHECK(root_left >= 0 && root_right >= 0, FCIB_ERR_ARG, "negative root index");
        if (std::max(root_left, root_right) >= c.nroot)
            throw Error{FCIB_ERR_ARG, "Cannot compute RDMs <" + std::to_string(root_left) + "| ... |" +
                                          std::to_string(root_right) + "> (0-based) because nroot = " +
                                          std::to_string(c.nroot)};
        Rdm3Blocks blk;
        DBuf<double> xl, xr;
        const double* L = c1_view(c, root_vector(c, root_left), xl);
        const double* R = root_right == root_left ? L : c1_view(c, root_vector(c, root_right), xr);
        compute_rdms3(c, L, R, blk);
        rdms3_to_outputs(blk, spin_free, g3aaa, g3aab, g3abb, g3bbb);
    });
}

int fcib_compute_rdms3(fcib_ctx* ctx, const double* left, const double* right, int spin_free, double* g3aaa,
                       double* g3aab, double* g3abb, double* g3bbb) {
    if (!ctx || !left) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        Context& c = ctx->c;
        ensure_setup(c);
        DBuf<double> dl, dr, xl, xr;
        dl.alloc(c.nvec);
        upload_flat(c, left, dl.p);
        const double* L = c1_view(c, dl.p, xl);
        const double* R = L;
        if (right && right != left) {
            dr.alloc(c.nvec);
            upload_flat(c, right, dr.p);
            R = c1_view(c, dr.p, xr);
        }
        Rdm3Blocks blk;
        compute_rdms3(c, L, R, blk);
        rdms3_to_outputs(blk, spin_free, g3aaa, g3aab, g3abb, g3bbb);
    });
}

int fcib_set_residual_capture(fcib_ctx* ctx, int max_vectors) {
    if (!ctx || max_vectors < 0) { set_error("bad argument"); return FCIB_ERR_ARG; }
    ctx->c.capture_max = max_vectors;
    ctx->c.cap_r.clear();
    ctx->c.cap_lambda.clear();
    return FCIB_OK;
}

int fcib_captured_residual(fcib_ctx* ctx, int index, double* r, double* lambda, int* count) {
    if (!ctx) { set_error("null context"); return FCIB_ERR_ARG; }
    const Context& c = ctx->c;
    if (count) *count = (int)c.cap_r.size();
    if (index < 0) return FCIB_OK;
    if (index >= (int)c.cap_r.size()) { set_error("captured residual index out of range"); return FCIB_ERR_ARG; }
    if (r) std::copy(c.cap_r[index].begin(), c.cap_r[index].end(), r);
    if (lambda) *lambda = c.cap_lambda[index];
    return FCIB_OK;
}

int fcib_num_strings(fcib_ctx* ctx, int spin, int64_t* count) {
    if (!ctx || !count) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        ensure_setup(ctx->c);
        *count = spin ? ctx->c.nbs : ctx->c.nas;
    });
}

int fcib_strings(fcib_ctx* ctx, int spin, uint32_t* out) {
    if (!ctx || !out) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        Context& c = ctx->c;
        ensure_setup(c);
        const SpinTables& t = spin ? c.B : c.A;
        FCIB_CUDA(cudaMemcpy(out, t.str.p, 4 * (size_t)t.nstr, cudaMemcpyDeviceToHost));
    });
}

int fcib_string_list(fcib_ctx* ctx, int spin, int kind, int p, int q, int r, int s, int64_t* len,
                     int8_t* sign, uint32_t* I, uint32_t* J) {
    if (!ctx || !len) { set_error("null argument"); return FCIB_ERR_ARG; }
    return guarded(ctx, [&] {
        Context& c = ctx->c;
        ensure_setup(c);
        int n = c.n;
        FCIB_CHECK(kind >= 0 && kind <= 2, FCIB_ERR_ARG, "kind must be 0 (VO), 1 (OO) or 2 (VVOO)");
        FCIB_CHECK(p >= 0 && q >= 0 && r >= 0 && s >= 0, FCIB_ERR_ARG, "negative orbital index");
        if (kind == 0) FCIB_CHECK(p < n && q < n, FCIB_ERR_ARG, "orbital index out of range");
        if (kind == 1) FCIB_CHECK(p < n * (n - 1) / 2, FCIB_ERR_ARG, "pair index out of range");
        if (kind == 2)
            FCIB_CHECK(p < n && q < n && r < n && s < n && p > q && r > s && !(p == r && q == s), FCIB_ERR_ARG,
                       "VVOO lists need p > q, r > s, (p,q) != (r,s)");
        std::vector<int8_t> hs;
        std::vector<uint32_t> hI, hJ;
        export_list(n, spin ? c.nb : c.na, kind, p, q, r, s, hs, hI, hJ, c.stream);
        *len = (int64_t)hs.size();
        if (sign) {
            std::copy(hs.begin(), hs.end(), sign);
            if (I) std::copy(hI.begin(), hI.end(), I);
            if (J) std::copy(hJ.begin(), hJ.end(), J);
        }
    });
}

int fcib_last_timing(fcib_ctx* ctx, double* sigma_ms, int* n_sigma, double* total_ms) {
    if (!ctx) { set_error("null context"); return FCIB_ERR_ARG; }
    if (sigma_ms) *sigma_ms = ctx->c.t_sigma_ms;
    if (n_sigma) *n_sigma = ctx->c.n_sigma;
    if (total_ms) *total_ms = ctx->c.t_total_ms;
    return FCIB_OK;
}

int fcib_get_profile(fcib_ctx* ctx, fcib_profile* o) {
    if (!ctx || !o) { set_error("null argument"); return FCIB_ERR_ARG; }
    const Context& c = ctx->c;
    o->total_ms = c.t_total_ms;
    o->sigma_ms = c.t_sigma_ms;
    o->ab_ms = c.t_ab_ms;
    o->same_ms = c.t_same_ms;
    o->ab64_ms = c.t_ab64_ms;
    o->same64_ms = c.t_same64_ms;
    o->n_ab64 = c.n_ab64;
    o->guess_ms = c.t_guess_ms;
    o->iterations = c.iterations;
    o->n_sigma = c.n_sigma;
    o->n_sigma_fp64 = c.n_sigma_fp64;
    o->n_ab = c.n_ab;
    o->launches = g_launch_count;
    o->tc_kernel_ms = c.t_tc_ms;
    return FCIB_OK;
}

int fcib_stream(fcib_ctx* ctx, void** stream) {
    if (!ctx || !stream) { set_error("null argument"); return FCIB_ERR_ARG; }
    *stream = (void*)ctx->c.stream;
    return FCIB_OK;
}

}  // extern "C"
