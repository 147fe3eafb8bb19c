/*
 * fcib.h -- C ABI of the B200 determinant-space FCI engine.
 *
 * Plain C types only (no CUDA or torch types).  Every function returns FCIB_OK (0) or a
 * negative error code; fcib_last_error() returns the calling thread's last message.
 * Host-buffer entry points take and return host memory; *_device entry points take device
 * pointers in the engine's layout and a CUDA stream handle passed as void*.  The engine's layout
 * is the C1 layout (na_str x nb_str row-major) without point-group symmetry; with symmetry it is
 * FCIVector flat order (fcib_size elements, the target irrep's blocks only) by default, or the C1
 * layout with zeros outside the target irrep when fcib_options.sym_blocked = 0.  With GAS spaces
 * (fcib_set_gas) host vectors follow GenCIVector flat order (fcib_size elements) and device
 * vectors keep the engine's layout with zeros outside the GAS space.
 *
 * Each entry point replaces a piece of Forte's FCISolver path (paths relative to the Forte
 * project root):
 *   fcib_create/destroy     -- FCISolver construction (forte/fci/fci_solver.cc:57-64)
 *   fcib_set_integrals      -- ActiveSpaceIntegrals input (forte/integrals/active_space_integrals.h:103-120,
 *                              make_active_space_ints active_space_integrals.cc:553-592)
 *   fcib_set_state          -- StateInfo / nroot / root (active_space_method.h:105, fci_solver.h:87-122)
 *   fcib_set_options        -- FCISolver::set_options (forte/fci/fci_solver.cc:156-172)
 *   fcib_solve              -- FCISolver::compute_energy (forte/fci/fci_solver.cc:177-314)
 *   fcib_get_vector         -- eigenvector rows of DavidsonLiuSolver::eigenvectors (davidson_liu_solver.h:86)
 *                              in FCIVector flat order (forte/fci/fci_vector.cc:139-169)
 *   fcib_sigma              -- the sigma builder FCIVector::Hamiltonian (fci_vector_hamiltonian.cc:46-82)
 *   fcib_hdiag              -- FCISolver::form_Hdiag_det (fci_solver_initial_guess.cc:151-172)
 *   fcib_rdms               -- FCISolver::rdms / FCIVector::compute_rdms (fci_solver_rdms.cc:40-104,
 *                              fci_vector_rdm.cc:43-393)
 *   fcib_spin2              -- FCIVector::compute_spin2 (fci_vector_spin2.cc:38-75)
 *   fcib_set_gas            -- GenCISolver's GAS space (forte/genci/genci_solver.h, genci_string_lists.cc:58-210)
 *   fcib_determinants       -- FCIStringLists / GenCIStringLists::make_determinants (genci_string_lists.cc:276-291)
 *   fcib_strings / fcib_string_list -- FCIStringLists strings and VO/OO/VVOO lists
 *                              (fci_string_lists.cc:52-205, fci_string_vo_list.cc:54-140,
 *                              fci_string_oo_list.cc:59-115, fci_string_vvoo_list.cc:56-187)
 */
#ifndef FCIB_H
#define FCIB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FCIB_OK 0
#define FCIB_ERR_ARG -1        /* invalid argument */
#define FCIB_ERR_STATE -2      /* call out of order (e.g. solve before set_integrals) */
#define FCIB_ERR_CUDA -3       /* CUDA runtime failure */
#define FCIB_ERR_UNSUPPORTED -4 /* size or feature outside the engine's range */
#define FCIB_ERR_NOT_CONVERGED -5 /* Davidson-Liu did not converge and die_if_not_converged */
#define FCIB_ERR_NUMERIC -6    /* non-finite values or a failed numerical invariant */

/* precision of the sigma build */
#define FCIB_PREC_FP64 0       /* everything in FP64 */
#define FCIB_PREC_MIXED 1      /* tensor-core TF32x3 sigma, FP64 subspace/residual/final energy */
#define FCIB_PREC_MIXED_TF32 2 /* single-pass TF32 sigma for the early iterations */

/* Davidson correction-vector preconditioner */
#define FCIB_PRECOND_DIAG 0    /* r_I / (lambda - H_II), the reference's */
#define FCIB_PRECOND_MLP 1     /* learned per-determinant MLP correction on top of the diagonal */
#define FCIB_SAME_TC 0         /* mixed same-spin term on the tensor cores (groups of <= 64 strings) */
#define FCIB_SAME_CUDA_CORES 1 /* mixed same-spin term in FP32 on the CUDA cores */

typedef struct fcib_options {
    int maxiter;               /* DL_MAXITER (default 100) */
    double e_convergence;      /* E_CONVERGENCE (default 1e-9) */
    double r_convergence;      /* R_CONVERGENCE (default 1e-6) */
    int guess_per_root;        /* DL_GUESS_PER_ROOT (default 1) */
    int dets_per_guess;        /* DL_DETS_PER_GUESS (default 50) */
    int collapse_per_root;     /* DL_COLLAPSE_PER_ROOT (default 2) */
    int subspace_per_root;     /* DL_SUBSPACE_PER_ROOT (default 10) */
    int die_if_not_converged;  /* throw on non-convergence (ActiveSpaceMethod::set_die_if_not_converged) */
    int print;                 /* PRINT level: 0 quiet, 1 iteration table to stdout */
    int precision;             /* FCIB_PREC_* */
    int preconditioner;        /* FCIB_PRECOND_* */
    double mixed_switch;       /* mixed modes: residual norm at which sigma switches to FP64 */
    int same_spin_kernel;      /* mixed modes: FCIB_SAME_TC (default) or FCIB_SAME_CUDA_CORES */
    int spin_adapt;            /* CI_SPIN_ADAPT: solve in the CSF basis of the state's multiplicity;
                                  default 0 */
    int sym_blocked;           /* nirrep > 1: vectors and sigma cover only the target irrep's blocks
                                  (FCIVector flat order, default 1); 0 = the full C1 space with a mask */
    int spin_adapt_full_preconditioner;  /* CI_SPIN_ADAPT_FULL_PRECONDITIONER: the CSF diagonal with
                                  the configuration's spin-exchange elements; default 0 */
} fcib_options;

typedef struct fcib_ctx fcib_ctx;

/* defaults of Forte's options.yaml for the FCI solver */
void fcib_default_options(fcib_options* opt);
const char* fcib_last_error(void);
const char* fcib_version(void);

int fcib_create(fcib_ctx** ctx, int device);
int fcib_destroy(fcib_ctx* ctx);

/* n active orbitals; orbsym[n] irreps (psi4 order, NULL = C1); scalar = nuclear repulsion +
 * scalar + frozen-core energy; oei_*[n*n]; tei_aa/bb[n^4] = <pq||rs>; tei_ab[n^4] = <pq|rs>
 * (row-major p,q,r,s).  The integrals must be real (8-fold symmetric two-electron block). */
int fcib_set_integrals(fcib_ctx* ctx, int n, int nirrep, const int* orbsym, double scalar,
                       const double* oei_a, const double* oei_b, const double* tei_aa,
                       const double* tei_ab, const double* tei_bb);
/* na/nb active alpha/beta electrons, target irrep, multiplicity (2S+1) used to select the
 * guess, number of roots and the root returned by the solver's energy.  StateInfo's twice_ms is
 * not a separate argument: the determinant space fixes 2 Ms = na - nb. */
int fcib_set_state(fcib_ctx* ctx, int na, int nb, int irrep, int multiplicity, int nroot, int root);
int fcib_set_options(fcib_ctx* ctx, const fcib_options* opt);
/* Generalized active spaces (GenCISolver, forte/genci/genci_solver.h): keep the determinants whose
 * number of electrons (alpha + beta) in each space k lies in [gas_min[k], gas_max[k]]
 * (StateInfo::gas_min/gas_max).  space[p] in 0..ngas-1 is the space of active orbital p (GAS1..GAS6
 * of MOSpaceInfo, each non-empty, ngas <= 6); ngas = 0 restores the full space.  Call after
 * fcib_set_integrals.  Host vectors then follow GenCIVector flat order: per occupation pair of
 * get_ci_occupation_patterns (ci_occupation.cc:131-170) and alpha irrep, the block of the alpha
 * and beta string classes (genci_string_address.cc:81-133, string_lists_makers.cc:65-127). */
int fcib_set_gas(fcib_ctx* ctx, int ngas, const int* space, const int* gas_min, const int* gas_max);

/* determinant-space size in flat order: FCIVector (sum over irrep blocks) or GenCIVector */
int fcib_size(fcib_ctx* ctx, int64_t* ndet);
/* length of device vectors in the engine's layout (the *_device entry points): fcib_size without
 * symmetry or GAS spaces and in the blocked layout; with GAS spaces the blocks of the strings some
 * GAS determinant uses (blocked) or the C1 space (sym_blocked = 0) */
int fcib_layout_size(fcib_ctx* ctx, int64_t* n);
/* alpha and beta strings (bit p = orbital p) of every flat position, fcib_size entries each
 * (FCIStringLists / GenCIStringLists::make_determinants, genci_string_lists.cc:276-291) */
int fcib_determinants(fcib_ctx* ctx, uint32_t* alfa, uint32_t* beta);
/* size of the CSF basis of the state's multiplicity in the target irrep, the Davidson space of
 * spin-adapted solves (SpinAdapter::ncsf, forte/sparse_ci/ci_spin_adaptation.h:81-183) */
int fcib_ncsf(fcib_ctx* ctx, int64_t* ncsf);
/* SpinAdapter::csf_C_to_det_C / det_C_to_csf_C (ci_spin_adaptation.h:81-183): CSF coefficients
 * z[ncsf] <-> a determinant vector c in FCIVector flat order (fcib_size elements) */
int fcib_csf_to_det(fcib_ctx* ctx, const double* z, double* c);
int fcib_det_to_csf(fcib_ctx* ctx, const double* c, double* z);
/* the CSF diagonal of H (FCISolver::form_Hdiag_csf, fci_solver_initial_guess.cc:111-149):
 * full = 0: sum_m O_im^2 H_mm; full = 1: <CSF_i|H|CSF_i> (the full preconditioner) */
int fcib_csf_hdiag(fcib_ctx* ctx, int full, double* out);

/* Runs the Davidson-Liu FCI.  energies[nroot], spin2[nroot] (either may be NULL), iterations
 * (may be NULL).  Returns FCIB_ERR_NOT_CONVERGED when the solver did not converge and
 * die_if_not_converged is set (the results are still stored). */
int fcib_solve(fcib_ctx* ctx, double* energies, double* spin2, int* iterations);
/* A context that solved before restarts the next fcib_solve from its previous eigenvectors
 * (FCISolver::compute_energy keeps its DavidsonLiuSolver, fci_solver.cc:205-233), as long as the
 * determinant space, nroot and subspace size are unchanged and the guess space does not cover the
 * whole space.  fcib_reset_guess forgets the previous solution, so that the next solve starts from
 * a fresh guess, as a newly constructed FCISolver would. */
int fcib_reset_guess(fcib_ctx* ctx);
/* eigenvector of a root in FCIVector flat order (size from fcib_size) */
int fcib_get_vector(fcib_ctx* ctx, int root, double* out);

/* FCIVector::max_abs_elements (forte/fci/fci_vector_h_diag.cc:37-68) of a root of the last solve:
 * the num_dets largest |C| in descending order (equal values in FCIVector flat order), each with its
 * signed value, alpha irrep and the alpha / beta string addresses within their irreps; slots past the
 * nonzero elements are zero, as in the reference.  *count = min(num_dets, size).  Any output may be
 * NULL.  With print >= 1, fcib_solve also prints these for the 100 largest elements of every root
 * (|C| >= 0.01), like FCISolver::print_solutions (fci_solver.cc:316-367). */
int fcib_max_abs_elements(fcib_ctx* ctx, int root, int num_dets, double* abs_c, double* c, int* alfa_irrep,
                          int64_t* alfa_address, int64_t* beta_address, int* count);
/* sigma = H b for a host vector in FCIVector flat order */
int fcib_sigma(fcib_ctx* ctx, const double* b, double* sigma);
/* sigma for device vectors in the engine's layout (see the top of this file), on a
 * stream (void* = cudaStream_t, NULL = the context's stream); precision = FCIB_PREC_* */
int fcib_sigma_device(fcib_ctx* ctx, const double* d_b, double* d_sigma, int precision, void* stream);
/* diagonal of H in FCIVector flat order */
int fcib_hdiag(fcib_ctx* ctx, double* out);
/* <S^2> of a host vector in FCIVector flat order */
int fcib_spin2(fcib_ctx* ctx, const double* c, double* s2);

/* Reduced density matrices between roots (root_left, root_right) of the last solve:
 * level 1 or 2.  spin_free = 0: g1a, g1b [n*n]; g2aa, g2ab, g2bb [n^4] (NULL to skip);
 * spin_free = 1: g1a <- g1a + g1b and g2aa <- g2aa + g2ab + g2ab(qpsr) + g2bb. */
int fcib_rdms(fcib_ctx* ctx, int root_left, int root_right, int level, int spin_free,
              double* g1a, double* g1b, double* g2aa, double* g2ab, double* g2bb);
/* The same RDMs between two host vectors in FCIVector flat order (right == NULL: right = left);
 * replaces FCIVector::compute_rdms(C_left, C_right, max_rdm_level, type) (fci_vector_rdm.cc:43-145). */
int fcib_compute_rdms(fcib_ctx* ctx, const double* left, const double* right, int level, int spin_free,
                      double* g1a, double* g1b, double* g2aa, double* g2ab, double* g2bb);
/* Transition 1-RDMs <left root| a+_p a_q |right root> between the solutions of two contexts, whose
 * states may belong to different irreps (FCISolver::transition_rdms(root_list, method2, max_rdm_level,
 * type), forte/fci/fci_solver_transition_rdms.cc:37-109, compute_1rdm_different_irrep
 * fci_vector_transition_rdm.cc:43-165).  Same orbitals, electrons and device in both contexts.
 * level 1..3 is accepted, but as in the reference only level 1 is implemented (FCIB_ERR_UNSUPPORTED
 * for 2 and 3).  spin_free = 0: g1a, g1b [n*n]; spin_free = 1: g1a <- g1a + g1b.  Like the reference,
 * both blocks are zero when the states have no alpha electrons. */
int fcib_transition_rdms(fcib_ctx* left, int root_left, fcib_ctx* right, int root_right, int level,
                         int spin_free, double* g1a, double* g1b);
/* 3-RDMs (max_rdm_level = 3 of FCISolver::rdms / FCIVector::compute_rdms, fci_vector_rdm.cc:70-137,
 * blocks compute_3rdm_aaa/aab/abb_same_irrep :395-565); fcib_rdms and fcib_compute_rdms accept
 * level 3 and return its one- and two-body parts.  Blocks are n^6 row-major in the reference's
 * index order and orientation (its loops take the creation indices from the right vector):
 *   g3aaa[p,q,r,s,t,u] = <right| a+_p a+_q a+_r a_u a_t a_s |left>, all alpha;
 *   g3aab: p, q, s, t alpha and r, u beta;  g3abb: p, s alpha and q, r, t, u beta;  g3bbb: beta.
 * For left == right these are the usual 3-RDMs.  spin_free: g3aaa receives the spin-free
 * G3 = aaa + aab + aab(prqsut) + aab(qrptus) + abb + abb(qprtsu) + abb(rpqust) + bbb (:127-130)
 * and the other pointers are ignored.  Any output may be NULL. */
/* Coupling coefficients of the spin adaptation (host only, no device): N open shells coupled to
 * 2S = twoS at 2Ms = twoMs; O[f][nd] for the f genealogical CSFs over the nd spin patterns pats[nd]
 * (bit k set: the k-th open shell in orbital order is alpha), in this engine's determinant phase
 * convention (alpha string, then beta string).  cap: capacity of O and pats in elements. */
int fcib_csf_coupling(int N, int twoS, int twoMs, int cap, double* O, uint32_t* pats, int* f, int* nd);
int fcib_rdms3(fcib_ctx* ctx, int root_left, int root_right, int spin_free, double* g3aaa, double* g3aab,
               double* g3abb, double* g3bbb);
int fcib_compute_rdms3(fcib_ctx* ctx, const double* left, const double* right, int spin_free, double* g3aaa,
                       double* g3aab, double* g3abb, double* g3bbb);

/* ---- learned preconditioner (no counterpart in the reference) ------------------------------
 * With preconditioner = FCIB_PRECOND_MLP each diagonal correction t_I = r_I / (lambda - H_II)
 * is rescaled by 1 + 0.25 tanh(m(x_I)), m a 35-64-64-64-1 ReLU network with BF16 weights; inputs
 * are the alpha/beta excitation bits of determinant I in a 16-orbital window around the Fermi
 * level, H_II - lambda and |r_I| / ||r||.  Weight vector (floats): W1[64][35], b1[64], W2[64][64],
 * b2[64], W3[64][64], b3[64], w4[64], b4.  Samples for eval/grad/train: ea/eb = excitation
 * window bits (16 each), u = H_II - lambda, r = r_I / ||r||, tgt = target correction element on
 * the scale of -r/u, wgt = per-sample loss weight. */
#define FCIB_MLP_NWEIGHTS 10689
/* load weights into a context (NULL unloads) */
int fcib_set_mlp(fcib_ctx* ctx, const float* weights, int nweights);
/* inference kernel on samples: factor[i] = 1 + 0.25 tanh(m(x_i)) */
int fcib_mlp_eval(int device, int64_t n, const uint32_t* ea, const uint32_t* eb, const float* u, const float* r,
                  const float* weights, float* factor);
/* loss = mean over samples of wgt (t (1 + 0.25 tanh m) - tgt)^2, t = -r/u (0 when |u| <= 1e-6), wgt
 * NULL = 1, and its gradient */
int fcib_mlp_grad(int device, int64_t n, const uint32_t* ea, const uint32_t* eb, const float* u, const float* r,
                  const float* tgt, const float* wgt, const float* weights, float* grad, double* loss);
/* Adam training on the GPU (init != 0: seeded Xavier init, zero output layer); weights in/out,
 * epoch_loss[epochs] (may be NULL) = mean minibatch loss of each epoch */
int fcib_mlp_train(int device, int64_t n, const uint32_t* ea, const uint32_t* eb, const float* u, const float* r,
                   const float* tgt, const float* wgt, int epochs, int batch, float lr, uint64_t seed, int init,
                   float* weights, double* epoch_loss);
/* the correction-vector step of DavidsonLiuSolver (davidson_liu_solver.cc:432-448) with the
 * context's preconditioner option: out = r / (lambda - H_II) (0 when |lambda - H_II| <= 1e-6),
 * rescaled by the network when preconditioner = FCIB_PRECOND_MLP; host vectors in flat order */
int fcib_precondition(fcib_ctx* ctx, const double* r, double lambda, double* out);
/* keep the raw residual of root 0 (engine layout) and its Ritz value at every Davidson iteration of
 * later solves, up to max_vectors (0 = off); read them back by index (index < 0: count only) */
int fcib_set_residual_capture(fcib_ctx* ctx, int max_vectors);
int fcib_captured_residual(fcib_ctx* ctx, int index, double* r, double* lambda, int* count);

/* ---- batched solver (no counterpart in the reference) ------------------------------------
 * Many independent CAS instances (2..12 orbitals, >= 1 electron of each spin, C1, no spin
 * selection) solved in one persistent launch: one CTA, or a thread-block cluster of CTAs sharing
 * its rows and vector elements, per instance at a time, largest first, every Davidson-Liu
 * iteration on the device.  Per instance: n, na, nb, scalar and the integral
 * arrays in the layouts of fcib_set_integrals.  Options used: maxiter, e_convergence,
 * r_convergence, subspace_per_root, collapse_per_root, precision (FCIB_PREC_FP64: FP64 sigma;
 * otherwise FP32 sigma with FP64 subspace, residuals and vectors until converged, then a restart
 * from the Ritz vectors with FP64 sigma, which alone decides convergence).  The launch is captured
 * in a CUDA graph on the first solve and replayed. */
typedef struct fcib_batch fcib_batch;
int fcib_batch_create(fcib_batch** batch, int device, int ninst, const int* n, const int* na, const int* nb,
                      const double* scalar, const double* const* oei_a, const double* const* oei_b,
                      const double* const* tei_aa, const double* const* tei_ab, const double* const* tei_bb,
                      int nroot, const fcib_options* opt);
int fcib_batch_destroy(fcib_batch* batch);
/* energies[ninst * nroot] (instance-major), iterations[ninst], converged[ninst], device_ms = device
 * time of the launch; any output may be NULL */
int fcib_batch_solve(fcib_batch* batch, double* energies, int* iterations, int* converged, double* device_ms);
/* clock cycles per phase of the batched solves since the last call (then reset), summed over all
 * CTAs: opposite-spin sigma, same-spin sigma, G update, subspace eigenproblem, residuals,
 * preconditioner, collapse, Gram-Schmidt (cycles[8]).  Only the profiling build of the library
 * (forte_b200.build.build(phases=True), compiled with -DFCIB_BATCH_PHASES) counts them; other
 * builds return FCIB_ERR_UNSUPPORTED. */
int fcib_batch_phase_cycles(unsigned long long* cycles);
/* launch shape of later solves: threads per CTA (256 or 512), opposite-spin sigma tile (8, 16 or 32
 * pairs per work item), CTAs per instance (a thread-block cluster of 1, 2 or 4).  The default is
 * 512 threads, 32-pair tiles and clusters of 2 (1 when two CTAs cannot be co-scheduled). */
int fcib_batch_set_shape(fcib_batch* batch, int threads, int pair_tile, int cluster);
/* autotuner: times the whole batch for each opposite-spin sigma tile (8, 16 or 32 pairs per work item)
 * and launch shape (threads per CTA x CTAs per instance, a thread-block cluster: 512x1, 256x2,
 * 512x2, 512x4), keeps the fastest for later solves; ctas_per_sm is 1; times_ms[12] (tile-major,
 * 0 for shapes that do not fit) may be NULL */
int fcib_batch_tune(fcib_batch* batch, int* threads, int* ctas_per_sm, int* pair_tile, int* cluster,
                    double* times_ms);

/* String tables for parity checks.  spin 0 = alpha, 1 = beta. */
int fcib_num_strings(fcib_ctx* ctx, int spin, int64_t* count);
int fcib_strings(fcib_ctx* ctx, int spin, uint32_t* out);
/* Substitution list in the reference's order: kind 0 = VO(p,q), 1 = OO(pair index p),
 * 2 = VVOO(p,q,r,s).  With sign == NULL only *len is written. */
int fcib_string_list(fcib_ctx* ctx, int spin, int kind, int p, int q, int r, int s,
                     int64_t* len, int8_t* sign, uint32_t* I, uint32_t* J);

/* timing of the last solve: total sigma milliseconds and number of sigma builds */
int fcib_last_timing(fcib_ctx* ctx, double* sigma_ms, int* n_sigma, double* total_ms);

/* Device-timed breakdown of the last solve (CUDA events on the engine's stream). */
typedef struct fcib_profile {
    double total_ms;        /* whole Davidson-Liu solve */
    double sigma_ms;        /* all sigma builds */
    double ab_ms;           /* tensor-core opposite-spin kernel inside mixed sigma builds */
    double same_ms;         /* same-spin kernels inside mixed sigma builds */
    double ab64_ms;         /* FP64 opposite-spin kernel inside FP64 sigma builds */
    double same64_ms;       /* same-spin kernels inside FP64 sigma builds */
    double guess_ms;        /* initial guess (host wall time) */
    int iterations;
    int n_sigma;            /* sigma builds */
    int n_sigma_fp64;       /* of which in FP64 */
    int n_ab;               /* launches timed in ab_ms */
    int n_ab64;             /* launches timed in ab64_ms */
    unsigned long long launches; /* kernel launches of this library since it was loaded */
    double tc_kernel_ms;    /* tensor-core contraction kernel alone (part of ab_ms) */
} fcib_profile;
int fcib_get_profile(fcib_ctx* ctx, fcib_profile* out);
/* the CUDA stream (cudaStream_t as void*) the engine launches on */
int fcib_stream(fcib_ctx* ctx, void** stream);

/* <S^2> of a device vector in the engine's layout, allocating nothing.  For callers that
 * cannot call cudaMalloc: a host whose memory pool already owns the GPU, or a loop that must
 * not pay for an allocation's device synchronisation or risk its failure.  No device or host
 * buffers are created; the reduction scratch is a static per-device array of 598,600 bytes
 * (1024 partial-sum blocks) that every call shares.  Same kernels and grid as fcib_spin2, so
 * the value matches it bit for bit.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress); make it before any stream capture.  The address is kept with
 * the ID of the device's CUDA context and looked up again when that changes (after
 * cudaDeviceReset the module is loaded at a new address), so make the first call after a reset
 * before any capture too.  The context's string tables must already exist (FCIB_ERR_STATE
 * otherwise); a launch needing more than 1024 blocks returns FCIB_ERR_UNSUPPORTED.  Calls on one
 * device that overlap on the GPU race on the shared scratch: serialise them.  d_c is in the
 * engine's layout (see the top of this file).  stream: cudaStream_t as
 * void*, NULL = the context's stream, which is a non-blocking stream and so is NOT ordered after
 * the legacy default stream or the caller's streams: either pass the stream that wrote d_c, or
 * make sure d_c is complete before the call.  The call synchronizes the stream it runs on.  No
 * counterpart in the reference. */
int fcib_spin2_device_noalloc(fcib_ctx* ctx, const double* d_c, double* s2, void* stream);

/* FP64 throughput of the GPU in TFLOP/s, measured with CUDA events (no setting changed):
 * dfma = CUDA-core FMA chains, dmma = FP64 tensor-core MMAs (mma.sync m8n8k4).  The
 * denominators of the FP64 sigma kernels' roofline fractions.  No counterpart in the reference. */
int fcib_fp64_peak(int device, double* dfma_tflops, double* dmma_tflops);

#ifdef __cplusplus
}
#endif
#endif /* FCIB_H */
