// Internal declarations shared by the engine's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <array>
#include <memory>
#include <string>
#include <vector>

#include "../../include/fcib.h"

namespace fcib {

// ------------------------------------------------------------------------------------------
// error handling: every public entry point returns FCIB_OK or an error code and sets a
// thread-local message readable with fcib_last_error().
// ------------------------------------------------------------------------------------------
struct Error {
    int code;
    std::string msg;
};
void set_error(const std::string& msg);

#define FCIB_CUDA(call)                                                                          \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            throw fcib::Error{FCIB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

// counts this engine's kernel launches (reported by fcib_profile) and checks the launch
extern unsigned long long g_launch_count;
#define FCIB_KCHECK()                           \
    do {                                        \
        ++fcib::g_launch_count;                 \
        FCIB_CUDA(cudaGetLastError());          \
    } while (0)

#define FCIB_CHECK(cond, code, msg)                   \
    do {                                              \
        if (!(cond)) throw fcib::Error{(code), (msg)}; \
    } while (0)

// ------------------------------------------------------------------------------------------
// device buffers
// ------------------------------------------------------------------------------------------
template <typename T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count) {
        if (count == n && p) return;
        release();
        if (count == 0) return;
        FCIB_CUDA(cudaMalloc((void**)&p, count * sizeof(T)));
        n = count;
    }
    void upload(const T* h, size_t count, cudaStream_t s = 0) {
        alloc(count);
        if (count) FCIB_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void upload(const std::vector<T>& v, cudaStream_t s = 0) { upload(v.data(), v.size(), s); }
};

// ------------------------------------------------------------------------------------------
// string machinery (strings.cu)
// ------------------------------------------------------------------------------------------
constexpr int kMaxOrb = 22;          // strings are uint32 masks; addresses fit in 21 bits
constexpr uint32_t kConnIdxMask = (1u << 21) - 1;
constexpr uint32_t kSignBit = 0x80000000u;
constexpr int32_t kNoTarget = 0x7FFFFFFF;

// Binomial table C(i, j) for i, j <= 32 (host and device copies)
struct Binom {
    uint32_t c[33][33];
};
const Binom& host_binom();
// rank of a string in the reference enumeration order (colex over reversed orbital positions)
uint32_t host_rank(uint32_t s, int n);
uint32_t host_unrank(uint32_t idx, int n, int k);

// Per-spin string tables resident in HBM.
struct SpinTables {
    int n = 0, k = 0;
    int nstr = 0;         // C(n,k)
    int s1 = 0;           // single-replacement connections per string (diagonal included)
    int npair = 0;        // unordered pairs with diagonal: n(n+1)/2
    int npair_pad = 0;    // padded to a multiple of 8
    DBuf<uint32_t> str;   // [nstr] bit masks in reference order
    DBuf<uint32_t> conn;  // [nstr * s1]: source J | pair P << 21 | sign << 31 (I = +-F_P J)
    DBuf<int32_t> tgt;    // [nstr * npair_pad]: F_R J = +-I -> I | sign << 31, or kNoTarget
    // (N-2)-electron groups for the same-spin two-body term
    int ng2 = 0, g2 = 0;  // number of groups, rows per group
    DBuf<uint32_t> g2row; // [ng2 * g2]: row I | sign << 31
    DBuf<uint16_t> g2lab; // [ng2 * g2]: pair label (p>q) index p(p-1)/2+q
    // (N-1)-electron groups for the one-body term when it is not folded
    int ng1 = 0, g1 = 0;
    DBuf<uint32_t> g1row;
    DBuf<uint16_t> g1lab;
};
void build_spin_tables(SpinTables& t, int n, int k, bool need_g1, cudaStream_t s);

// ------------------------------------------------------------------------------------------
// irrep-blocked determinant space (symblock.cu)
// ------------------------------------------------------------------------------------------
// With point-group symmetry the engine's vectors hold only the determinants of the target irrep,
// in FCIVector flat order (forte/fci/fci_vector.cc:86-169): alpha irrep blocks h, each the alpha
// strings of irrep h (string order) x the beta strings of irrep h ^ irrep.  The beta same-spin
// terms work on the transposed blocks: beta irrep h x the alpha strings of irrep h ^ irrep.
constexpr uint32_t kNullRow = 0x7FFFFFFFu;  // padding member of a same-spin group (no string)

// device view of the blocked layout, passed to kernels by value.  With GAS spaces the blocks hold
// only the strings that some GAS determinant uses (the kept strings); loc of any other string is -1.
struct SymDev {
    int on = 0;                         // 1: the blocked layout (0: the C1 layout)
    int nirrep = 1, irrep = 0;
    uint32_t irrbit[3] = {0u, 0u, 0u};  // orbitals whose irrep label has bit b set
    int64_t blk[9] = {};                // alpha-major block offsets
    int32_t bcol[8] = {};               // row length of alpha block h (beta strings of irrep h ^ irrep)
    int32_t aoff[8] = {}, boff[8] = {}; // first position of each irrep in the irrep-sorted string lists
    const int32_t* asrc = nullptr;      // irrep-sorted position -> string index
    const int32_t* bsrc = nullptr;
    const int32_t* aloc = nullptr;      // string index -> position among the strings of its irrep
    const int32_t* bloc = nullptr;
};

__host__ __device__ inline int sym_irrep_of(const SymDev& d, uint32_t s) {
#ifdef __CUDA_ARCH__
    return (__popc(s & d.irrbit[0]) & 1) | ((__popc(s & d.irrbit[1]) & 1) << 1) | ((__popc(s & d.irrbit[2]) & 1) << 2);
#else
    return (__builtin_popcount(s & d.irrbit[0]) & 1) | ((__builtin_popcount(s & d.irrbit[1]) & 1) << 1) |
           ((__builtin_popcount(s & d.irrbit[2]) & 1) << 2);
#endif
}
// blocked index -> (alpha string index, beta string index)
__device__ __forceinline__ void sym_decode(const SymDev& d, int64_t I, int& ia, int& ib) {
    int h = 0;
    for (int x = 1; x < d.nirrep; x++)
        if (I >= d.blk[x]) h = x;  // an empty block x shares its offset with x + 1, which wins
    const int64_t r = I - d.blk[h];
    const int64_t col = d.bcol[h];
    const int64_t i = r / col;
    ia = d.asrc[d.aoff[h] + i];
    ib = d.bsrc[d.boff[h ^ d.irrep] + (int)(r - i * col)];
}
// (alpha string sa with index ia, beta string index ib) of the target irrep -> blocked index
__device__ __forceinline__ int64_t sym_encode(const SymDev& d, uint32_t sa, int ia, int ib) {
    const int h = sym_irrep_of(d, sa);
    return d.blk[h] + (int64_t)d.aloc[ia] * d.bcol[h] + d.bloc[ib];
}
// the same, or -1 when either string is not in the blocks (GAS spaces)
__device__ __forceinline__ int64_t sym_encode_kept(const SymDev& d, uint32_t sa, int ia, int ib) {
    const int la = d.aloc[ia], lb = d.bloc[ib];
    if (la < 0 || lb < 0) return -1;
    const int h = sym_irrep_of(d, sa);
    return d.blk[h] + (int64_t)la * d.bcol[h] + lb;
}

// one opposite-spin sub-problem of the blocked sigma: target alpha irrep ha, pair irrep g.  Rows are
// the alpha strings of irrep ha; their connections through pairs of irrep g reach alpha strings of
// irrep ha ^ g, whose rows hold the beta strings of irrep ha ^ irrep ^ g (the source columns); the
// beta replacements of irrep g take those to the target columns (beta irrep ha ^ irrep).
// With GAS spaces a sub-problem covers one alpha pattern range of the target rows (row0, rows)
// and one beta pattern range of the source columns (col0, ns; the source row length is lds); its
// targets are the whole row of the target block (nt).  Without GAS both ranges are whole blocks.
struct AbSub {
    int ha = 0, g = 0, src = 0;  // target alpha irrep, pair irrep, source alpha irrep ha ^ g
    int rows = 0, ns = 0, nt = 0;
    int row0 = 0, col0 = 0, lds = 0;
    int diag_off = 0;            // target column of the first source string (g = 0 only)
    int accumulate = 0;          // 0: the first sub-problem of its rows (writes E0 C + its part)
    int kmax = 0;                // connections per row (short rows padded with the zero pair)
    size_t conn = 0, tgt32 = 0, tgt16 = 0, mag = 0;  // offsets into the SymSpace tables
};
// same-spin groups whose strings lie in one irrep (padded to G members with kNullRow), over a range
// of ncols columns of rows of length ld
struct GroupSub {
    int ngroups = 0, G = 0, ncols = 0, ld = 0;
    int64_t blk = 0;   // block offset (+ first column): alpha-major for alpha groups, transposed for beta groups
    size_t off = 0;    // into SymSpace::grow / glab
};
// a run of strings of one occupation pattern inside an irrep's kept strings
struct PatRange {
    int pat = 0, start = 0, count = 0;
};
struct SymSpace {
    bool on = false;
    SymDev d;
    int64_t blkT[9] = {};
    int acnt[8] = {}, bcnt[8] = {};
    std::vector<int> airr, birr;                      // irrep of each string
    std::vector<int32_t> asrc_h, bsrc_h, aloc_h, bloc_h;  // loc -1: string not in the blocks (GAS)
    // GAS occupation patterns (one pattern 0 covering everything without GAS): per string its
    // pattern (-1: not kept), per irrep the pattern runs of the kept strings, the pattern pairs
    // that GAS determinants have, and which patterns one electron replacement connects
    std::vector<int> apat, bpat;
    std::vector<PatRange> arun[8], brun[8];
    int npa = 1, npb = 1;
    std::vector<uint8_t> allowed;                     // [npa * npb]
    std::vector<uint8_t> areach, breach;              // [npa * npa], [npb * npb]
    DBuf<int32_t> asrc, bsrc, aloc, bloc;
    DBuf<uint32_t> bstr_sorted;                       // beta strings in irrep-sorted order
    // opposite spin
    std::vector<AbSub> ab;                            // per target irrep: g = 0 first
    int npp = 0;                                      // rows of V; the zero pair is row npp
    std::vector<int> np_g, npg, noff8_g, ndiag_g;     // per pair irrep: pairs, FP64 columns (x8), tensor-core layout
    std::vector<size_t> vg_off, perm_off;
    DBuf<double> Vg;    // per g: (npp + 1) x npg[g], column j = pair j of irrep g
    DBuf<double> Vz;    // the pair matrix with the zero pair row appended, (npp + 1) x npp
    DBuf<int> perm;     // per g: tensor-core columns -> pair (off-diagonal pairs, then the diagonal ones)
    DBuf<uint32_t> conn;
    DBuf<int32_t> tgt32;
    DBuf<uint16_t> tgt16;
    DBuf<uint8_t> mag;
    std::vector<size_t> plane_off;                    // TF32 plane of each alpha block (float2 units)
    std::vector<int> ldp;
    size_t plane_total = 0;
    // same spin
    std::vector<GroupSub> a2, a1, b2, b1;
    DBuf<uint32_t> grow;
    DBuf<uint16_t> glab;
};

// a pair of CUDA events owned by the context (created on first use)
struct EventPair {
    cudaEvent_t e[2] = {nullptr, nullptr};
    void ensure() {
        for (auto& x : e)
            if (!x) cudaEventCreate(&x);
    }
    ~EventPair() {
        for (auto& x : e)
            if (x) cudaEventDestroy(x);
    }
};

// ------------------------------------------------------------------------------------------
// engine context
// ------------------------------------------------------------------------------------------
// configurations with N open shells of the spin-adapted space (csf.cu)
struct CsfGroup {
    int N = 0, f = 0, nd = 0, nconf = 0;  // open shells, CSFs and determinants per configuration
    int64_t zoff = 0;                     // first CSF of the group in a CSF vector
    DBuf<uint32_t> conf;                  // [nconf][2]: doubly occupied mask, open-shell mask
    DBuf<uint32_t> pats;                  // [nd] spin patterns over the open shells (bit k: alpha)
    DBuf<double> O;                       // [f][nd] coupling coefficients
};

// generalized active spaces (gas.cu): bounds on the electrons in each orbital space
constexpr int kMaxGas = 6;
struct GasSpace {
    int ngas = 0;                          // 0: no restriction
    std::vector<int> space;                // [n] space of each orbital
    int emin[kMaxGas] = {}, emax[kMaxGas] = {};  // bounds on alpha + beta electrons per space
    uint32_t orbs[kMaxGas] = {};           // orbitals of each space
    // string classes of the current state (GenCIStringLists): per C1 string its class (-1: none)
    // and address in it; strings per class; flat offset of each (alpha class, beta class) block
    std::vector<int32_t> acls, bcls;
    std::vector<int64_t> aadd, badd, acnt, bcnt, blk_off;
    int ncb = 0;
    int64_t ndet = 0;                      // determinants of the GAS space
};

struct Context {
    int device = 0;
    cudaStream_t stream = nullptr;
    int num_sms = 0;
    int smem_optin = 0;   // max dynamic+static shared memory per block
    int smem_per_sm = 0;
    // problem
    int n = 0, nirrep = 1;
    std::vector<int> orbsym;
    double scalar = 0.0;
    std::vector<double> oei_a, oei_b, tei_aa, tei_ab, tei_bb;  // host copies (guess, checks)
    bool has_ints = false;
    int na = -1, nb = -1, irrep = 0, multiplicity = 1, nroot = 1, root = 0;
    bool has_state = false;
    fcib_options opt;
    // device tables
    SpinTables A, B;
    bool tables_ready = false;
    int64_t nas = 0, nbs = 0, ndet = 0;  // ndet = nas * nbs (the C1 layout)
    int64_t nvec = 0;     // length of the engine's vectors: ndet, or the target irrep's blocks
    SymSpace sym;         // the blocked layout (sym.on) when the state has point-group symmetry
    DBuf<double> V;       // [npair_pad_a x npair_pad_b] pair-pair (pq|rs) (+ folded h)
    DBuf<double> M2a, M2b;  // same-spin <pq||rs> over pairs p>q, r>s
    DBuf<double> Ha, Hb;  // one-body matrices (used when h is not folded)
    bool fold_h = true;
    DBuf<uint8_t> mask;   // kept determinants of a masked layout (gas.cu), else unallocated
    GasSpace gas;         // GAS restriction (ngas = 0: none)
    // work vectors
    DBuf<double> ct;      // transposed C for the beta same-spin terms
    DBuf<uint16_t> tgtR16; // beta replacement targets [column/8][string][column%8] for the tensor-core kernel
    DBuf<int> tc_perm;     // pair of each tensor-core column: off-diagonal pairs, then the diagonal ones
    DBuf<float> tf_hi;        // interleaved (tf32 hi, tf32 lo) pairs of the sigma input (mixed path)
    DBuf<float> c32, ct32;    // FP32 copy of the sigma input and its transpose (mixed same-spin)
    DBuf<unsigned long long> s64a, st64;  // mixed same-spin sigma parts, int64 fixed point: alpha
                                          // (row-major), beta (transposed)
    double same_mmax = 0.0;   // max |same-spin block element| (fixed-point grid of those sums)
    bool c32_ready = false;   // c32 holds the current sigma input (written by the tensor-core split)
    float vmax = 0.0f;    // max |V| (fixed-point grid of the tensor-core scatter)
    DBuf<double> hdiag;
    // solver storage
    DBuf<double> b, sig, r, tmp;
    int subspace = 0;
    std::vector<double> energies, spin2;
    int iterations = 0;
    bool solved = false;
    // masked layouts: layout index of every position of the caller's flat order (FCIVector or
    // GenCIVector order); empty when the layout is the flat order itself
    std::vector<int64_t> flat_map;
    DBuf<int> counter;    // work counters for persistent kernels
    DBuf<int> subctr;     // row counters of the blocked sigma's sub-problems (zeroed once per sigma)
    DBuf<double> red;     // reduction scratch
    // timers and status of the last solve
    double t_sigma_ms = 0.0;
    int n_sigma = 0;
    double t_total_ms = 0.0;
    int n_sigma_fp64 = 0;
    double t_guess_ms = 0.0;
    double t_ab_ms = 0.0, t_same_ms = 0.0;  // tensor-core opposite-spin / same-spin kernels (mixed sigma)
    int n_ab = 0;
    double t_ab64_ms = 0.0, t_same64_ms = 0.0;  // the same for FP64 sigma builds
    int n_ab64 = 0;
    EventPair tc_ev;      // brackets the last tensor-core contraction launch
    bool tc_recorded = false;
    double t_tc_ms = 0.0;  // tensor-core contraction kernel alone (mixed sigma)
    int guess_dets = 0;
    bool converged = false;
    // restart state of the Davidson-Liu solver (DavidsonLiuSolver::setup_guesses restarts a solver
    // that already ran from its first nroot vectors): the determinant space it ran on and the
    // vectors its first guess asked to project out
    bool dl_prev = false;
    bool restarted = false;  // the last solve restarted from the previous solution
    // spin adaptation (csf.cu): configuration groups of the current state and target spin
    std::vector<std::unique_ptr<CsfGroup>> csf;
    bool csf_ready = false;
    int csf_twoS = -1;
    int64_t ncsf = 0;
    DBuf<double> csf_x, csf_s;  // determinant-space scratch of the CSF-basis sigma
    DBuf<double> hd_csf;        // CSF diagonal of the last spin-adapted solve
    DBuf<double> evdet;         // spin-adapted solves: the roots in the engine's determinant layout
    bool roots_in_evdet = false;   // the last solve ran in the CSF basis or the GAS flat basis (roots in evdet)
    // GAS solves: the Davidson space is the GAS determinants in GenCIVector flat order
    DBuf<int64_t> flat_map_d;   // device copy of flat_map
    DBuf<double> gas_x, gas_s;  // layout-sized sigma input (zero outside the GAS space) and output
    DBuf<double> hd_gas;        // diagonal in flat order
    bool sigma_unmasked = false;  // the sigma being built is only gathered at GAS positions (no mask pass)
    std::vector<int64_t> dl_prev_space;
    std::vector<std::vector<std::pair<int64_t, double>>> dl_bad;
    std::vector<double> dl_lambda_old;  // eigenvalues of the previous solve's last iteration
    std::vector<std::array<double, 5>> trace;
    // learned preconditioner weights (FP32 master copy, BF16-rounded at use)
    DBuf<float> mlp_w;
    DBuf<float> mlp_tabA, mlp_tabB;  // per-string layer-1 sums of the loaded weights
    bool mlp_tables_ready = false;
    // residual capture of root 0 during solves (training data of the learned preconditioner)
    int capture_max = 0;
    std::vector<std::vector<double>> cap_r;
    std::vector<double> cap_lambda;  // iteration, ms, lambda_0, max residual, fp64 basis
};

// the blocked layout's device view for kernels that decode vector indices (nirrep = 1: C1 layout)
inline SymDev sym_dev(const Context& c) { return c.sym.on ? c.sym.d : SymDev{}; }

// counter slots: 0 opposite-spin row counter, 1 its timeout flag, 2 CUDA-core group counter,
// 3 bits of max|C| of the sigma input, 4 tensor-core group counter, 5 its timeout flag,
// 6 exponent el of the same-spin fixed-point grid 2^-el, 7 bits of max|C| of an FP64 sigma input
constexpr int kSlotCmax = 3;
constexpr int kSlotSameGrid = 6;
constexpr int kSlotCmax64 = 7;
// the work counters and error flags of the persistent kernels, zeroed when first allocated
inline void ensure_counter(Context& c) {
    if (c.counter.p) return;
    c.counter.alloc(16);
    FCIB_CUDA(cudaMemsetAsync(c.counter.p, 0, 16 * sizeof(int), c.stream));
}

// kernels / launchers (sigma.cu)
void prepare_integrals(Context& c);
// csf.cu: the CSF basis of the target multiplicity (the Davidson space of spin_adapt): configuration
// groups, x = P z (CSF coefficients -> engine-layout determinants), z = P^T x, the CSF diagonal
void ensure_csf(Context& c);
void csf_to_det(Context& c, const double* z, double* x);
void det_to_csf(Context& c, const double* x, double* z);
void csf_hdiag(Context& c, double* out);
void sigma_fp64(Context& c, const double* C, double* S);
float host_vmax(Context& c);  // max |V| (pair matrix) with a small margin, from a host copy
void sigma_mixed(Context& c, const double* C, double* S, bool three);
void apply_mask(Context& c, double* v);
// gas.cu: mask and flat map of the layout (masked C1 with symmetry, GAS); GenCIVector position
void build_layout_maps(Context& c);
int64_t gas_flat_position(const Context& c, int64_t I);
// GAS occupation pattern of every string of each spin (index into its spin's pattern list, -1 when
// no GAS determinant uses the string), the allowed pattern pairs [npa * npb] and, per spin, which
// patterns differ by one electron moved between spaces or not at all ([np * np])
void gas_string_patterns(const Context& c, const std::vector<uint32_t>& sa, const std::vector<uint32_t>& sb,
                         std::vector<int>& pat_a, std::vector<int>& pat_b, int& npa, int& npb,
                         std::vector<uint8_t>& allowed, std::vector<uint8_t>& reach_a, std::vector<uint8_t>& reach_b);
void export_list(int n, int k, int kind, int p, int q, int r, int s, std::vector<int8_t>& sign,
                 std::vector<uint32_t>& I, std::vector<uint32_t>& J, cudaStream_t st);
void compute_hdiag(Context& c, double* out);
void sigma_dispatch(Context& c, const double* b, double* s, int precision);
void ensure_setup(Context& c);
// rdms.cu: host copies of the RDM blocks (row-major, n^2 and n^4)
struct RdmBlocks {
    int n = 0;
    std::vector<double> g1a, g1b, g2aa, g2ab, g2bb;
};
void compute_rdms(Context& c, const double* L, const double* R, int level, RdmBlocks& out);
// rdms3.cu: host copies of the 3-RDM blocks (row-major n^6, reference index order and orientation)
struct Rdm3Blocks {
    int n = 0;
    std::vector<double> aaa, aab, abb, bbb;
};
void compute_rdms3(Context& c, const double* L, const double* R, Rdm3Blocks& out);
// mlp.cu: learned preconditioner, in place on a diagonal correction t
void mlp_apply(Context& c, double* t, double lambda, double rnorm, double tnorm);
// symblock.cu: blocked-layout tables of the target irrep (c.sym.on when nirrep > 1 and blocking is on)
void build_sym_space(Context& c);
// v (engine layout) in the C1 layout: v itself without blocking, else expanded into buf
const double* c1_view(Context& c, const double* v, DBuf<double>& buf);
// engine layout <- C1 layout (blocked: the target irrep's elements)
void from_c1(Context& c, const double* c1, double* v);
// host view of a blocked index: (alpha irrep, positions within the irrep blocks) / string indices
void sym_host_locate(const Context& c, int64_t I, int& h, int64_t& ia_loc, int64_t& ib_loc);
void sym_host_decode(const Context& c, int64_t I, int64_t& ia, int64_t& ib);
int64_t sym_host_encode(const Context& c, int64_t ia, int64_t ib);
// davidson.cu
void dl_solve(Context& c);
// a root of the last solve in the engine's determinant layout
const double* root_vector(Context& c, int root);
std::vector<std::pair<double, int64_t>> lowest_keys(Context& c, const double* keys, int count);
// the same over N keys with an optional mask (keys whose mask byte is 0 are skipped)
std::vector<std::pair<double, int64_t>> lowest_keys(Context& c, const double* keys, int count, size_t N,
                                                    const uint8_t* mask);
double spin2_device(Context& c, const double* C);

}  // namespace fcib
