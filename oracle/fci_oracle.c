/*
 * fci_oracle.c -- CPU ORACLE (test infrastructure only, never shipped or measured as product).
 *
 * A single-threaded C restatement of Forte's determinant-space FCI path, used as the parity
 * checker for the CUDA engine and as the timed CPU baseline ("port").  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU legs may load it.
 *
 * Each function cites the reference file:line it restates (paths are relative to the Forte
 * project root).  Point-group symmetry is handled by masking the C1 determinant space to the
 * target irrep (the reference stores one block per irrep instead); energies, vectors (on the
 * target block) and RDMs are identical because H is block diagonal by symmetry.
 *
 * Orbital strings are uint64 bit masks: bit i set <=> orbital i occupied (the reference's
 * BitArray<64> word 0).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MAXN 24

/* ------------------------------------------------------------------------------------------ */
/* error reporting                                                                             */
/* ------------------------------------------------------------------------------------------ */
static char orc_err[512];
const char* orc_last_error(void) { return orc_err; }
static int fail(const char* msg) {
    snprintf(orc_err, sizeof(orc_err), "%s", msg);
    return -1;
}

/* ------------------------------------------------------------------------------------------ */
/* permutations and strings                                                                    */
/* ------------------------------------------------------------------------------------------ */

/* std::next_permutation over a 0/1 sequence (lexicographic, element 0 most significant). */
static int next_perm(int8_t* a, int n) {
    if (n < 2) return 0;
    int i = n - 2;
    while (i >= 0 && !(a[i] < a[i + 1])) i--;
    if (i < 0) {
        for (int l = 0, r = n - 1; l < r; l++, r--) { int8_t t = a[l]; a[l] = a[r]; a[r] = t; }
        return 0;
    }
    int j = n - 1;
    while (!(a[i] < a[j])) j--;
    int8_t t = a[i]; a[i] = a[j]; a[j] = t;
    for (int l = i + 1, r = n - 1; l < r; l++, r--) { t = a[l]; a[l] = a[r]; a[r] = t; }
    return 1;
}

static int64_t binom(int n, int k) {
    if (k < 0 || k > n) return 0;
    int64_t r = 1;
    for (int i = 1; i <= k; i++) r = r * (n - k + i) / i;
    return r;
}

int64_t orc_num_strings(int n, int k) { return binom(n, k); }

/* FCIStringLists::make_fci_strings (forte/fci/fci_string_lists.cc:258-293), C1 case:
 * start from 0..01..1 (ones in the last k slots) and enumerate with next_permutation. */
int64_t orc_make_strings(int n, int k, uint64_t* out) {
    if (k < 0 || k > n || n > ORC_MAXN) return 0;
    int8_t b[64];
    for (int i = 0; i < n; i++) b[i] = (i >= n - k) ? 1 : 0;
    int64_t cnt = 0;
    do {
        uint64_t s = 0;
        for (int i = 0; i < n; i++)
            if (b[i]) s |= (1ull << i);
        out[cnt++] = s;
    } while (next_perm(b, n));
    return cnt;
}

static inline int popc(uint64_t x) { return __builtin_popcountll(x); }
/* BitArray::slater_sign(n): (-1)^(number of set bits below n) (forte/sparse_ci/bitarray.hpp:635) */
static inline double sgn_below(uint64_t s, int n) {
    return (popc(s & ((1ull << n) - 1ull)) & 1) ? -1.0 : 1.0;
}
/* ui64_sign(x, m, n): (-1)^(set bits strictly between m and n) (bitwise_operations.hpp:125) */
static inline double sgn_between(uint64_t s, int m, int n) {
    if (m > n) { int t = m; m = n; n = t; }
    if (n - m < 2) return 1.0;
    uint64_t mask = ((1ull << n) - 1ull) & ~((1ull << (m + 1)) - 1ull);
    return (popc(s & mask) & 1) ? -1.0 : 1.0;
}

/* ------------------------------------------------------------------------------------------ */
/* substitution lists (reference layout: sign, I, J; StringSubstitution in string_list_defs.h:40) */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
    int64_t len, cap;
    double* sign;
    uint32_t* I;
    uint32_t* J;
} sublist;

static void sl_push(sublist* l, double sign, uint32_t I, uint32_t J) {
    if (l->len == l->cap) {
        int64_t nc = l->cap ? 2 * l->cap : 16;
        l->sign = (double*)realloc(l->sign, nc * sizeof(double));
        l->I = (uint32_t*)realloc(l->I, nc * sizeof(uint32_t));
        l->J = (uint32_t*)realloc(l->J, nc * sizeof(uint32_t));
        l->cap = nc;
    }
    l->sign[l->len] = sign;
    l->I[l->len] = I;
    l->J[l->len] = J;
    l->len++;
}
static void sl_free(sublist* l) {
    free(l->sign); free(l->I); free(l->J);
    memset(l, 0, sizeof(*l));
}

typedef struct {
    int n, k;
    int64_t ns;
    uint64_t* str;   /* ns strings in reference order */
    int32_t* addr;   /* 1<<n lookup: string -> address, -1 if not a k-string */
    sublist* vo;     /* [p*n+q] : J = sign a+_p a_q I */
    sublist* oo;     /* [pq pair index] */
    sublist* vvoo;   /* [((p*n+q)*n+r)*n+s] : J = sign a+_p a+_q a_s a_r I */
} spinlists;

static int32_t addr_of(const spinlists* L, uint64_t s) { return L->addr[s]; }

/* FCIStringLists::make_vo (forte/fci/fci_string_vo_list.cc:90-140) */
static void make_vo(spinlists* L, int p, int q) {
    int n = L->n - 1 - (p == q ? 0 : 1);
    int k = L->k - 1;
    sublist* out = &L->vo[p * L->n + q];
    if (!(k >= 0 && k <= n)) return;
    int8_t b[64];
    for (int i = 0; i < n; i++) b[i] = (i >= n - k) ? 1 : 0;
    int lo = p < q ? p : q, hi = p < q ? q : p;
    do {
        uint64_t I = 0, J = 0;
        int kk = 0;
        double sign = 1.0;
        for (int i = 0; i < lo; i++, kk++)
            if (b[kk]) { I |= 1ull << i; J |= 1ull << i; }
        for (int i = lo + 1; i < hi; i++, kk++)
            if (b[kk]) { I |= 1ull << i; J |= 1ull << i; sign = -sign; }
        for (int i = hi + 1; i < L->n; i++, kk++)
            if (b[kk]) { I |= 1ull << i; J |= 1ull << i; }
        I &= ~(1ull << p); I |= 1ull << q;
        J &= ~(1ull << q); J |= 1ull << p;
        sl_push(out, sign, (uint32_t)addr_of(L, I), (uint32_t)addr_of(L, J));
    } while (next_perm(b, n));
}

/* FCIStringLists::make_oo (forte/fci/fci_string_oo_list.cc:69-115), pair (p>q) index pq */
static void make_oo(spinlists* L, int p, int q, int pq) {
    int k = L->k - 2;
    if (k < 0) return;
    int n = L->n - 2;
    sublist* out = &L->oo[pq];
    int8_t b[64];
    for (int i = 0; i < n; i++) b[i] = (i >= n - k) ? 1 : 0;
    do {
        uint64_t I = 0;
        int kk = 0;
        for (int i = 0; i < q; i++, kk++)
            if (b[kk]) I |= 1ull << i;
        for (int i = q + 1; i < p; i++, kk++)
            if (b[kk]) I |= 1ull << i;
        for (int i = p + 1; i < L->n; i++, kk++)
            if (b[kk]) I |= 1ull << i;
        I |= (1ull << p) | (1ull << q);
        uint32_t a = (uint32_t)addr_of(L, I);
        sl_push(out, 1.0, a, a);
    } while (next_perm(b, n));
}

/* FCIStringLists::make_vvoo (forte/fci/fci_string_vvoo_list.cc:88-187) */
static void make_vvoo(spinlists* L, int p, int q, int r, int s) {
    int a[4] = {s, r, q, p};
#define CSW(x, y) if (a[x] > a[y]) { int t_ = a[x]; a[x] = a[y]; a[y] = t_; }
    CSW(1, 2);
    CSW(0, 1); CSW(1, 2); CSW(2, 3);
    CSW(0, 1); CSW(1, 2); CSW(2, 3);
#undef CSW
    int overlap = (a[0] == a[1]) || (a[1] == a[2]) || (a[2] == a[3]);
    int n = L->n - 4 + (overlap ? 1 : 0);
    int k = L->k - 2;
    int N = L->n;
    sublist* out = &L->vvoo[((p * N + q) * N + r) * N + s];
    if (!(k >= 0 && n >= 0 && n >= k)) return;
    int8_t b[64];
    for (int i = 0; i < n; i++) b[i] = (i >= n - k) ? 1 : 0;
    do {
        uint64_t I = 0;
        I &= ~(1ull << p); I &= ~(1ull << q); I |= 1ull << s; I |= 1ull << r;
        int kk = 0;
        for (int i = 0; i < a[0]; i++, kk++) { if (b[kk]) I |= 1ull << i; else I &= ~(1ull << i); }
        for (int i = a[0] + 1; i < a[1]; i++, kk++) { if (b[kk]) I |= 1ull << i; else I &= ~(1ull << i); }
        for (int i = a[1] + 1; i < a[2]; i++, kk++) { if (b[kk]) I |= 1ull << i; else I &= ~(1ull << i); }
        for (int i = a[2] + 1; i < a[3]; i++, kk++) { if (b[kk]) I |= 1ull << i; else I &= ~(1ull << i); }
        for (int i = a[3] + 1; i < N; i++, kk++) { if (b[kk]) I |= 1ull << i; else I &= ~(1ull << i); }
        uint64_t J = I;
        double sign = 1.0;
        for (int i = s; i < r; i++)
            if (J & (1ull << i)) sign = -sign;
        J &= ~(1ull << r);
        J &= ~(1ull << s);
        if (!(J & (1ull << q))) {
            J |= 1ull << q;
            sign *= sgn_below(J, q);
            if (!(J & (1ull << p))) {
                J |= 1ull << p;
                sign *= sgn_below(J, p);
                sl_push(out, sign, (uint32_t)addr_of(L, I), (uint32_t)addr_of(L, J));
            }
        }
    } while (next_perm(b, n));
}

static int build_spinlists(spinlists* L, int n, int k) {
    memset(L, 0, sizeof(*L));
    L->n = n;
    L->k = k;
    L->ns = binom(n, k);
    L->str = (uint64_t*)malloc(sizeof(uint64_t) * (L->ns > 0 ? L->ns : 1));
    orc_make_strings(n, k, L->str);
    L->addr = (int32_t*)malloc(sizeof(int32_t) << n);
    for (int64_t i = 0; i < (1ll << n); i++) L->addr[i] = -1;
    for (int64_t i = 0; i < L->ns; i++) L->addr[L->str[i]] = (int32_t)i;
    L->vo = (sublist*)calloc((size_t)n * n, sizeof(sublist));
    int npair = n * (n - 1) / 2;
    L->oo = (sublist*)calloc(npair > 0 ? npair : 1, sizeof(sublist));
    L->vvoo = (sublist*)calloc((size_t)n * n * n * n, sizeof(sublist));
    /* make_vo_list order (fci_string_vo_list.cc:68-88): p outer, q inner (C1) */
    for (int p = 0; p < n; p++)
        for (int q = 0; q < n; q++) make_vo(L, p, q);
    /* make_pair_list (fci_string_lists.cc:211-229): pairs p>q, p outer, q inner */
    int pq = 0;
    for (int p = 0; p < n; p++)
        for (int q = 0; q < p; q++) make_oo(L, p, q, pq++);
    /* make_vvoo_list (fci_string_vvoo_list.cc:56-86) */
    for (int p = 0; p < n; p++)
        for (int q = 0; q < n; q++)
            for (int r = 0; r < n; r++)
                for (int s = 0; s < n; s++)
                    if (p > q && r > s && !(p == r && q == s)) make_vvoo(L, p, q, r, s);
    return 0;
}

static void free_spinlists(spinlists* L) {
    int n = L->n;
    if (L->vo)
        for (int i = 0; i < n * n; i++) sl_free(&L->vo[i]);
    if (L->oo)
        for (int i = 0; i < n * (n - 1) / 2; i++) sl_free(&L->oo[i]);
    if (L->vvoo)
        for (int i = 0; i < n * n * n * n; i++) sl_free(&L->vvoo[i]);
    free(L->vo); free(L->oo); free(L->vvoo); free(L->str); free(L->addr);
    memset(L, 0, sizeof(*L));
}

/* ------------------------------------------------------------------------------------------ */
/* context                                                                                     */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
    int n, na, nb;
    spinlists A, B;
    int64_t nas, nbs, ndet;
    double e0;
    double *oei_a, *oei_b, *tei_aa, *tei_ab, *tei_bb;
    int has_ints;
    int orbsym[ORC_MAXN];
    int target_irrep;
    uint8_t* mask; /* per determinant: 1 if its irrep is the target one */
    double* scratch1;
    double* scratch2;
} orc_ctx;

void* orc_create(int n, int na, int nb, const int* orbsym, int target_irrep) {
    if (n < 1 || n > ORC_MAXN || na < 0 || nb < 0 || na > n || nb > n) {
        fail("orc_create: bad sizes");
        return NULL;
    }
    orc_ctx* c = (orc_ctx*)calloc(1, sizeof(orc_ctx));
    c->n = n; c->na = na; c->nb = nb;
    build_spinlists(&c->A, n, na);
    build_spinlists(&c->B, n, nb);
    c->nas = c->A.ns; c->nbs = c->B.ns; c->ndet = c->nas * c->nbs;
    for (int i = 0; i < n; i++) c->orbsym[i] = orbsym ? orbsym[i] : 0;
    c->target_irrep = target_irrep;
    c->mask = (uint8_t*)malloc(c->ndet > 0 ? c->ndet : 1);
    for (int64_t ia = 0; ia < c->nas; ia++) {
        int sa = 0;
        for (int i = 0; i < n; i++) if (c->A.str[ia] >> i & 1) sa ^= c->orbsym[i];
        for (int64_t ib = 0; ib < c->nbs; ib++) {
            int sb = 0;
            for (int i = 0; i < n; i++) if (c->B.str[ib] >> i & 1) sb ^= c->orbsym[i];
            c->mask[ia * c->nbs + ib] = ((sa ^ sb) == target_irrep);
        }
    }
    int64_t mx = c->nas > c->nbs ? c->nas : c->nbs;
    c->scratch1 = (double*)malloc(sizeof(double) * mx * mx);
    c->scratch2 = (double*)malloc(sizeof(double) * mx * mx);
    return c;
}

void orc_destroy(void* h) {
    orc_ctx* c = (orc_ctx*)h;
    if (!c) return;
    free_spinlists(&c->A);
    free_spinlists(&c->B);
    free(c->oei_a); free(c->oei_b); free(c->tei_aa); free(c->tei_ab); free(c->tei_bb);
    free(c->mask); free(c->scratch1); free(c->scratch2);
    free(c);
}

int64_t orc_ndet(void* h) { return ((orc_ctx*)h)->ndet; }
int64_t orc_nstr(void* h, int spin) { orc_ctx* c = (orc_ctx*)h; return spin ? c->nbs : c->nas; }
void orc_strings(void* h, int spin, uint64_t* out) {
    orc_ctx* c = (orc_ctx*)h;
    spinlists* L = spin ? &c->B : &c->A;
    memcpy(out, L->str, sizeof(uint64_t) * L->ns);
}
void orc_mask(void* h, uint8_t* out) { orc_ctx* c = (orc_ctx*)h; memcpy(out, c->mask, c->ndet); }

/* list export: kind 0 = VO(p,q), 1 = OO(pq index in p), 2 = VVOO(p,q,r,s) */
static sublist* get_list(orc_ctx* c, int spin, int kind, int p, int q, int r, int s) {
    spinlists* L = spin ? &c->B : &c->A;
    int n = c->n;
    if (kind == 0) return &L->vo[p * n + q];
    if (kind == 1) return &L->oo[p];
    return &L->vvoo[((p * n + q) * n + r) * n + s];
}
int64_t orc_list_len(void* h, int spin, int kind, int p, int q, int r, int s) {
    return get_list((orc_ctx*)h, spin, kind, p, q, r, s)->len;
}
void orc_list_get(void* h, int spin, int kind, int p, int q, int r, int s, double* sign,
                  uint32_t* I, uint32_t* J) {
    sublist* l = get_list((orc_ctx*)h, spin, kind, p, q, r, s);
    memcpy(sign, l->sign, sizeof(double) * l->len);
    memcpy(I, l->I, sizeof(uint32_t) * l->len);
    memcpy(J, l->J, sizeof(uint32_t) * l->len);
}

int orc_set_integrals(void* h, double e0, const double* oei_a, const double* oei_b,
                      const double* tei_aa, const double* tei_ab, const double* tei_bb) {
    orc_ctx* c = (orc_ctx*)h;
    size_t n = c->n, n2 = n * n, n4 = n2 * n2;
    free(c->oei_a); free(c->oei_b); free(c->tei_aa); free(c->tei_ab); free(c->tei_bb);
    c->oei_a = (double*)malloc(n2 * 8); memcpy(c->oei_a, oei_a, n2 * 8);
    c->oei_b = (double*)malloc(n2 * 8); memcpy(c->oei_b, oei_b, n2 * 8);
    c->tei_aa = (double*)malloc(n4 * 8); memcpy(c->tei_aa, tei_aa, n4 * 8);
    c->tei_ab = (double*)malloc(n4 * 8); memcpy(c->tei_ab, tei_ab, n4 * 8);
    c->tei_bb = (double*)malloc(n4 * 8); memcpy(c->tei_bb, tei_bb, n4 * 8);
    c->e0 = e0;
    c->has_ints = 1;
    return 0;
}

#define OEI(a, p, q) (a)[(p) * n + (q)]
#define TEI(a, p, q, r, s) (a)[(((size_t)(p) * n + (q)) * n + (r)) * n + (s)]

/* ------------------------------------------------------------------------------------------ */
/* sigma = H C (forte/fci/fci_vector_hamiltonian.cc:46-272)                                   */
/* ------------------------------------------------------------------------------------------ */
static inline void daxpy(int64_t len, double a, const double* x, double* y) {
    for (int64_t i = 0; i < len; i++) y[i] += a * x[i];
}

/* gather_C_block (forte/fci/fci_vector.cc:239-278): for beta terms the block is transposed */
static void transpose(const double* in, double* out, int64_t rows, int64_t cols) {
    for (int64_t i = 0; i < rows; i++)
        for (int64_t j = 0; j < cols; j++) out[j * rows + i] = in[i * cols + j];
}

/* H1 (fci_vector_hamiltonian.cc:93-123) */
static void sigma_h1(orc_ctx* c, const double* C, double* S, int alfa) {
    int n = c->n;
    spinlists* L = alfa ? &c->A : &c->B;
    int64_t maxL = alfa ? c->nbs : c->nas;
    const double* Cr;
    double* Cl;
    if (alfa) {
        Cr = C; Cl = S;
    } else {
        transpose(C, c->scratch1, c->nas, c->nbs);
        transpose(S, c->scratch2, c->nas, c->nbs);
        Cr = c->scratch1; Cl = c->scratch2;
    }
    const double* oei = alfa ? c->oei_a : c->oei_b;
    for (int p = 0; p < n; p++)
        for (int q = 0; q < n; q++) {
            double hpq = OEI(oei, p, q);
            sublist* l = &L->vo[p * n + q];
            for (int64_t e = 0; e < l->len; e++)
                daxpy(maxL, l->sign[e] * hpq, Cr + (int64_t)l->I[e] * maxL, Cl + (int64_t)l->J[e] * maxL);
        }
    if (!alfa) transpose(c->scratch2, S, c->nbs, c->nas);
}

/* H2_aaaa2 (fci_vector_hamiltonian.cc:125-192) */
static void sigma_h2_same(orc_ctx* c, const double* C, double* S, int alfa) {
    int n = c->n;
    spinlists* L = alfa ? &c->A : &c->B;
    int64_t maxL = alfa ? c->nbs : c->nas;
    const double* Cr;
    double* Cl;
    if (alfa) {
        Cr = C; Cl = S;
    } else {
        transpose(C, c->scratch1, c->nas, c->nbs);
        transpose(S, c->scratch2, c->nas, c->nbs);
        Cr = c->scratch1; Cl = c->scratch2;
    }
    const double* tei = alfa ? c->tei_aa : c->tei_bb;
    /* pair list in order (make_pair_list) */
    int np = n * (n - 1) / 2;
    int* pp = (int*)malloc(sizeof(int) * (np + 1));
    int* pqv = (int*)malloc(sizeof(int) * (np + 1));
    int t = 0;
    for (int p = 0; p < n; p++)
        for (int q = 0; q < p; q++) { pp[t] = p; pqv[t] = q; t++; }
    for (int pq = 0; pq < np; pq++) {
        int p = pp[pq], q = pqv[pq];
        double integral = TEI(tei, p, q, p, q);
        sublist* l = &L->oo[pq];
        for (int64_t e = 0; e < l->len; e++)
            daxpy(maxL, l->sign[e] * integral, Cr + (int64_t)l->I[e] * maxL, Cl + (int64_t)l->J[e] * maxL);
    }
    for (int pq = 0; pq < np; pq++) {
        int p = pp[pq], q = pqv[pq];
        for (int rs = 0; rs < pq; rs++) {
            int r = pp[rs], s = pqv[rs];
            double integral = TEI(tei, p, q, r, s);
            sublist* l1 = &L->vvoo[((p * n + q) * n + r) * n + s];
            for (int64_t e = 0; e < l1->len; e++)
                daxpy(maxL, l1->sign[e] * integral, Cr + (int64_t)l1->I[e] * maxL, Cl + (int64_t)l1->J[e] * maxL);
            sublist* l2 = &L->vvoo[((r * n + s) * n + p) * n + q];
            for (int64_t e = 0; e < l2->len; e++)
                daxpy(maxL, l2->sign[e] * integral, Cr + (int64_t)l2->I[e] * maxL, Cl + (int64_t)l2->J[e] * maxL);
        }
    }
    free(pp); free(pqv);
    if (!alfa) transpose(c->scratch2, S, c->nbs, c->nas);
}

/* H2_aabb (fci_vector_hamiltonian.cc:194-272) */
static void sigma_h2_ab(orc_ctx* c, const double* C, double* S) {
    int n = c->n;
    int64_t nas = c->nas, nbs = c->nbs;
    double* CR = c->scratch1;
    double* CL = c->scratch2;
    for (int r = 0; r < n; r++)
        for (int s = 0; s < n; s++) {
            sublist* vb = &c->B.vo[r * n + s];
            int64_t maxSSb = vb->len;
            if (maxSSb == 0) continue;
            memset(CR, 0, sizeof(double) * nas * maxSSb);
            memset(CL, 0, sizeof(double) * nas * maxSSb);
            for (int64_t Ia = 0; Ia < nas; Ia++) {
                const double* cc = C + Ia * nbs;
                double* cr = CR + Ia * maxSSb;
                for (int64_t SSb = 0; SSb < maxSSb; SSb++) cr[SSb] = cc[vb->I[SSb]] * vb->sign[SSb];
            }
            for (int p = 0; p < n; p++)
                for (int q = 0; q < n; q++) {
                    double integral = TEI(c->tei_ab, p, r, q, s);
                    sublist* va = &c->A.vo[p * n + q];
                    for (int64_t e = 0; e < va->len; e++)
                        daxpy(maxSSb, integral * va->sign[e], CR + (int64_t)va->I[e] * maxSSb,
                              CL + (int64_t)va->J[e] * maxSSb);
                }
            for (int64_t Ja = 0; Ja < nas; Ja++) {
                double* hc = S + Ja * nbs;
                const double* cl = CL + Ja * maxSSb;
                for (int64_t SSb = 0; SSb < maxSSb; SSb++) hc[vb->J[SSb]] += cl[SSb];
            }
        }
}

/* FCIVector::Hamiltonian (fci_vector_hamiltonian.cc:46-82); S is overwritten. Terms can be
 * selected with a bit mask (1 = H0, 2 = H1a, 4 = H1b, 8 = H2ab, 16 = H2aa, 32 = H2bb). */
int orc_sigma_terms(void* h, const double* C, double* S, int terms) {
    orc_ctx* c = (orc_ctx*)h;
    if (!c->has_ints) return fail("orc_sigma: integrals not set");
    int64_t N = c->ndet;
    for (int64_t i = 0; i < N; i++) S[i] = (terms & 1) ? c->e0 * C[i] : 0.0;
    if (terms & 2) sigma_h1(c, C, S, 1);
    if (terms & 4) sigma_h1(c, C, S, 0);
    if (terms & 8) sigma_h2_ab(c, C, S);
    if (terms & 16) sigma_h2_same(c, C, S, 1);
    if (terms & 32) sigma_h2_same(c, C, S, 0);
    return 0;
}
int orc_sigma(void* h, const double* C, double* S) { return orc_sigma_terms(h, C, S, 63); }

/* ------------------------------------------------------------------------------------------ */
/* determinant-level helpers                                                                   */
/* ------------------------------------------------------------------------------------------ */

/* ActiveSpaceIntegrals::energy (forte/integrals/active_space_integrals.cc:206-245), plus the
 * E0 = nuclear + scalar added in form_Hdiag_det (fci_solver_initial_guess.cc:151-172).
 * e0 here is the total scalar (nuclear + scalar + frozen core). */
static double det_energy(orc_ctx* c, uint64_t Ia, uint64_t Ib) {
    int n = c->n;
    double energy = c->e0;
    uint64_t a = Ia;
    while (a) {
        int p = __builtin_ctzll(a);
        a &= a - 1;
        energy += OEI(c->oei_a, p, p);
        uint64_t ac = a;
        while (ac) {
            int q = __builtin_ctzll(ac);
            ac &= ac - 1;
            energy += TEI(c->tei_aa, p, q, p, q);
        }
        uint64_t bc = Ib;
        while (bc) {
            int q = __builtin_ctzll(bc);
            bc &= bc - 1;
            energy += TEI(c->tei_ab, p, q, p, q);
        }
    }
    uint64_t b = Ib;
    while (b) {
        int p = __builtin_ctzll(b);
        b &= b - 1;
        energy += OEI(c->oei_b, p, p);
        uint64_t bc = b;
        while (bc) {
            int q = __builtin_ctzll(bc);
            bc &= bc - 1;
            energy += TEI(c->tei_bb, p, q, p, q);
        }
    }
    return energy;
}

int orc_hdiag(void* h, double* out) {
    orc_ctx* c = (orc_ctx*)h;
    if (!c->has_ints) return fail("orc_hdiag: integrals not set");
    for (int64_t ia = 0; ia < c->nas; ia++)
        for (int64_t ib = 0; ib < c->nbs; ib++)
            out[ia * c->nbs + ib] = det_energy(c, c->A.str[ia], c->B.str[ib]);
    return 0;
}

/* DeterminantImpl::slater_sign_aaaa (forte/sparse_ci/determinant.hpp:391-406) */
static double sign_aaaa(uint64_t s, int i, int j, int a, int b) {
    if ((((i < a) && (j < a) && (i < b) && (j < b)) == 1) ||
        (((i < a) || (j < a) || (i < b) || (j < b)) == 0)) {
        if ((i < j) ^ (a < b))
            return -1.0 * sgn_between(s, i, j) * sgn_between(s, a, b);
        return sgn_between(s, i, j) * sgn_between(s, a, b);
    }
    if ((i < j) ^ (a < b)) return -1.0 * sgn_between(s, i, b) * sgn_between(s, j, a);
    return sgn_between(s, i, a) * sgn_between(s, j, b);
}

/* ActiveSpaceIntegrals::slater_rules (forte/integrals/active_space_integrals.cc:247-411);
 * the diagonal includes e0 like the guess Hamiltonian does through its energy shift. */
static double slater_rules(orc_ctx* c, uint64_t la, uint64_t lb, uint64_t ra, uint64_t rb) {
    int n = c->n;
    if (popc(la) != popc(ra) || popc(lb) != popc(rb)) return 0.0;
    int nadiff = popc(la ^ ra), nbdiff = popc(lb ^ rb);
    if (nadiff + nbdiff > 4) return 0.0;
    nadiff /= 2;
    nbdiff /= 2;
    double me = 0.0;
    if (nadiff == 0 && nbdiff == 0) {
        for (int p = 0; p < n; p++) {
            int ap = la >> p & 1, bp = lb >> p & 1;
            if (ap) me += OEI(c->oei_a, p, p);
            if (bp) me += OEI(c->oei_b, p, p);
            for (int q = 0; q < n; q++) {
                int aq = la >> q & 1, bq = lb >> q & 1;
                if (ap && aq) me += 0.5 * TEI(c->tei_aa, p, q, p, q);
                if (bp && bq) me += 0.5 * TEI(c->tei_bb, p, q, p, q);
                if (ap && bq) me += TEI(c->tei_ab, p, q, p, q);
            }
        }
    }
    if (nadiff == 1 && nbdiff == 0) {
        int i = 0, j = 0;
        for (int p = 0; p < n; p++) {
            if (((la ^ ra) >> p & 1) && (la >> p & 1)) i = p;
            if (((la ^ ra) >> p & 1) && (ra >> p & 1)) j = p;
        }
        double sign = sgn_between(la, i, j);
        me = sign * OEI(c->oei_a, i, j);
        for (int p = 0; p < n; p++) {
            if ((la >> p & 1) && (ra >> p & 1)) me += sign * TEI(c->tei_aa, i, p, j, p);
            if ((lb >> p & 1) && (rb >> p & 1)) me += sign * TEI(c->tei_ab, i, p, j, p);
        }
    }
    if (nadiff == 0 && nbdiff == 1) {
        int i = 0, j = 0;
        for (int p = 0; p < n; p++) {
            if (((lb ^ rb) >> p & 1) && (lb >> p & 1)) i = p;
            if (((lb ^ rb) >> p & 1) && (rb >> p & 1)) j = p;
        }
        double sign = sgn_between(lb, i, j);
        me = sign * OEI(c->oei_b, i, j);
        for (int p = 0; p < n; p++) {
            if ((la >> p & 1) && (ra >> p & 1)) me += sign * TEI(c->tei_ab, p, i, p, j);
            if ((lb >> p & 1) && (rb >> p & 1)) me += sign * TEI(c->tei_bb, i, p, j, p);
        }
    }
    if (nadiff == 2 && nbdiff == 0) {
        int i = -1, j = 0, k = -1, l = 0;
        for (int p = 0; p < n; p++) {
            if (((la ^ ra) >> p & 1) && (la >> p & 1)) { if (i == -1) i = p; else j = p; }
            if (((la ^ ra) >> p & 1) && (ra >> p & 1)) { if (k == -1) k = p; else l = p; }
        }
        me = sign_aaaa(la, i, j, k, l) * TEI(c->tei_aa, i, j, k, l);
    }
    if (nadiff == 0 && nbdiff == 2) {
        int i = -1, j = -1, k = -1, l = -1;
        for (int p = 0; p < n; p++) {
            if (((lb ^ rb) >> p & 1) && (lb >> p & 1)) { if (i == -1) i = p; else j = p; }
            if (((lb ^ rb) >> p & 1) && (rb >> p & 1)) { if (k == -1) k = p; else l = p; }
        }
        me = sign_aaaa(lb, i, j, k, l) * TEI(c->tei_bb, i, j, k, l);
    }
    if (nadiff == 1 && nbdiff == 1) {
        int i = -1, j = -1, k = -1, l = -1;
        for (int p = 0; p < n; p++) {
            if (((la ^ ra) >> p & 1) && (la >> p & 1)) i = p;
            if (((lb ^ rb) >> p & 1) && (lb >> p & 1)) j = p;
            if (((la ^ ra) >> p & 1) && (ra >> p & 1)) k = p;
            if (((lb ^ rb) >> p & 1) && (rb >> p & 1)) l = p;
        }
        me = sgn_between(la, i, k) * sgn_between(lb, j, l) * TEI(c->tei_ab, i, j, k, l);
    }
    return me;
}

double orc_slater_rules(void* h, uint64_t la, uint64_t lb, uint64_t ra, uint64_t rb) {
    return slater_rules((orc_ctx*)h, la, lb, ra, rb);
}

/* Selected rows of sigma = H C in the C1 determinant space, one row at a time from the Slater
 * rules: sigma_I = e0 C_I + sum_J <I|H|J> C_J over every J that differs from I by at most a
 * double replacement (ActiveSpaceIntegrals::slater_rules, forte/integrals/active_space_integrals.cc:
 * 247-411, for the same operator FCIVector::Hamiltonian applies, fci_vector_hamiltonian.cc:46-272).
 * Needs no substitution lists, so it reaches sizes where a whole oracle sigma would take hours.
 * C is the full vector in C1 flat order (alpha string index * nbs + beta string index, strings in
 * FCIStringLists order); rows[] are determinant indices; abs_out[i] (may be NULL) receives
 * sum_J |<I|H|J> C_J|, the scale of the row's rounding error. */
int orc_sigma_rows(int n, int na, int nb, double e0, const double* oei_a, const double* oei_b,
                   const double* tei_aa, const double* tei_ab, const double* tei_bb, const double* C,
                   int64_t nrows, const int64_t* rows, double* out, double* abs_out) {
    if (n < 1 || n > ORC_MAXN || na < 0 || nb < 0 || na > n || nb > n) return fail("orc_sigma_rows: bad sizes");
    orc_ctx c;
    memset(&c, 0, sizeof(c));
    c.n = n;
    c.oei_a = (double*)oei_a; c.oei_b = (double*)oei_b;
    c.tei_aa = (double*)tei_aa; c.tei_ab = (double*)tei_ab; c.tei_bb = (double*)tei_bb;
    const int64_t nas = binom(n, na), nbs = binom(n, nb);
    uint64_t* sa = (uint64_t*)malloc(sizeof(uint64_t) * (nas > 0 ? nas : 1));
    uint64_t* sb = (uint64_t*)malloc(sizeof(uint64_t) * (nbs > 0 ? nbs : 1));
    int32_t* addr = (int32_t*)malloc(sizeof(int32_t) * ((size_t)1 << n));
    if (!sa || !sb || !addr) { free(sa); free(sb); free(addr); return fail("orc_sigma_rows: out of memory"); }
    orc_make_strings(n, na, sa);
    orc_make_strings(n, nb, sb);
    /* string -> index within its spin (the alpha and beta lists are separate when na != nb) */
    int32_t* addr_b = NULL;
    for (int64_t i = 0; i < nas; i++) addr[sa[i]] = (int32_t)i;
    if (na != nb) {
        addr_b = (int32_t*)malloc(sizeof(int32_t) * ((size_t)1 << n));
        if (!addr_b) { free(sa); free(sb); free(addr); return fail("orc_sigma_rows: out of memory"); }
        for (int64_t i = 0; i < nbs; i++) addr_b[sb[i]] = (int32_t)i;
    }
    const int32_t* ab = addr_b ? addr_b : addr;
    const uint64_t full = (n == 64) ? ~0ull : ((1ull << n) - 1ull);
    for (int64_t t = 0; t < nrows; t++) {
        const int64_t I = rows[t];
        const uint64_t Ia = sa[I / nbs], Ib = sb[I % nbs];
        double acc = 0.0, aacc = 0.0;
#define ORC_ADD(Ja, Jb)                                                          \
        do {                                                                     \
            const int64_t J_ = (int64_t)addr[(Ja)] * nbs + ab[(Jb)];             \
            double h_ = slater_rules(&c, Ia, Ib, (Ja), (Jb));                    \
            if ((Ja) == Ia && (Jb) == Ib) h_ += e0;                              \
            const double v_ = h_ * C[J_];                                        \
            acc += v_;                                                           \
            aacc += fabs(v_);                                                    \
        } while (0)
        ORC_ADD(Ia, Ib);
        /* alpha replacements of rank 1 and 2, each combined with beta replacements of rank 0/1,
         * and beta replacements of rank 1 and 2 with the alpha string fixed */
        const uint64_t occa = Ia, vira = full & ~Ia, occb = Ib, virb = full & ~Ib;
        for (uint64_t oi = occa; oi; oi &= oi - 1) {
            const int i = __builtin_ctzll(oi);
            for (uint64_t va = vira; va; va &= va - 1) {
                const int a = __builtin_ctzll(va);
                const uint64_t Ja = (Ia & ~(1ull << i)) | (1ull << a);
                ORC_ADD(Ja, Ib);
                for (uint64_t oj = occb; oj; oj &= oj - 1) {
                    const int j = __builtin_ctzll(oj);
                    for (uint64_t vb = virb; vb; vb &= vb - 1) {
                        const int b = __builtin_ctzll(vb);
                        ORC_ADD(Ja, (Ib & ~(1ull << j)) | (1ull << b));
                    }
                }
                for (uint64_t oj = oi & (oi - 1); oj; oj &= oj - 1) {
                    const int j = __builtin_ctzll(oj);
                    for (uint64_t vb = va & (va - 1); vb; vb &= vb - 1) {
                        const int b = __builtin_ctzll(vb);
                        ORC_ADD((Ja & ~(1ull << j)) | (1ull << b), Ib);
                    }
                }
            }
        }
        for (uint64_t oi = occb; oi; oi &= oi - 1) {
            const int i = __builtin_ctzll(oi);
            for (uint64_t vb = virb; vb; vb &= vb - 1) {
                const int b = __builtin_ctzll(vb);
                const uint64_t Jb = (Ib & ~(1ull << i)) | (1ull << b);
                ORC_ADD(Ia, Jb);
                for (uint64_t oj = oi & (oi - 1); oj; oj &= oj - 1) {
                    const int j = __builtin_ctzll(oj);
                    for (uint64_t vc = vb & (vb - 1); vc; vc &= vc - 1) {
                        const int d = __builtin_ctzll(vc);
                        ORC_ADD(Ia, (Jb & ~(1ull << j)) | (1ull << d));
                    }
                }
            }
        }
#undef ORC_ADD
        out[t] = acc;
        if (abs_out) abs_out[t] = aacc;
    }
    free(sa); free(sb); free(addr); free(addr_b);
    return 0;
}

/* spin2(lhs, rhs) (forte/sparse_ci/determinant.hpp:910-958) */
static double det_spin2(uint64_t Ia, uint64_t Ib, uint64_t Ja, uint64_t Jb, int nmo) {
    if (popc(Ia) != popc(Ja) || popc(Ib) != popc(Jb)) return 0.0;
    int nadiff = popc(Ia ^ Ja) / 2, nbdiff = popc(Ib ^ Jb) / 2;
    int na = popc(Ia), nb = popc(Ib), npair = popc(Ia & Ib);
    double Ms = 0.5 * (double)(na - nb);
    double me = 0.0;
    if (nadiff == 0 && nbdiff == 0) me += Ms * (Ms + 1.0) + (double)nb - (double)npair;
    if (nadiff == 1 && nbdiff == 1) {
        int i = -1, j = -1;
        for (int p = 0; p < nmo; p++) {
            if ((Ja >> p & 1) && (Ib >> p & 1) && !(Jb >> p & 1) && !(Ia >> p & 1)) i = p;
            if ((Jb >> p & 1) && (Ia >> p & 1) && !(Ja >> p & 1) && !(Ib >> p & 1)) j = p;
        }
        if (i != j && i >= 0 && j >= 0) {
            /* slater_sign_a(i) counts alpha bits below i; slater_sign_b(j) counts all alpha bits
             * plus beta bits below j (the determinant's alpha word precedes the beta word). */
            double sign = sgn_below(Ja, i) * ((popc(Ja) & 1) ? -1.0 : 1.0) * sgn_below(Jb, j) *
                          sgn_below(Ia, j) * ((popc(Ia) & 1) ? -1.0 : 1.0) * sgn_below(Ib, i);
            me -= sign;
        }
    }
    return me;
}

double orc_det_spin2(uint64_t Ia, uint64_t Ib, uint64_t Ja, uint64_t Jb, int nmo) {
    return det_spin2(Ia, Ib, Ja, Jb, nmo);
}

/* ------------------------------------------------------------------------------------------ */
/* dense symmetric eigensolver (cyclic Jacobi; stands in for LAPACK dsyev in psi::Matrix::      */
/* diagonalize).  Eigenvalues ascending, eigenvectors in columns: V[i*n + k] = component i of  */
/* vector k; each vector's largest-magnitude component is made positive.                       */
/* ------------------------------------------------------------------------------------------ */
void orc_jacobi(int n, const double* Ain, double* evals, double* V) {
    double* A = (double*)malloc(sizeof(double) * n * n);
    memcpy(A, Ain, sizeof(double) * n * n);
    for (int i = 0; i < n * n; i++) V[i] = 0.0;
    for (int i = 0; i < n; i++) V[i * n + i] = 1.0;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0, tot = 0.0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                tot += A[i * n + j] * A[i * n + j];
                if (i != j) off += A[i * n + j] * A[i * n + j];
            }
        if (off <= 1e-30 * (tot > 0 ? tot : 1.0) || off < 1e-300) break;
        for (int p = 0; p < n - 1; p++)
            for (int q = p + 1; q < n; q++) {
                double apq = A[p * n + q];
                if (fabs(apq) < 1e-300) continue;
                double app = A[p * n + p], aqq = A[q * n + q];
                double theta = (aqq - app) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double cs = 1.0 / sqrt(t * t + 1.0), sn = t * cs;
                for (int k = 0; k < n; k++) {
                    double akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p] = cs * akp - sn * akq;
                    A[k * n + q] = sn * akp + cs * akq;
                }
                for (int k = 0; k < n; k++) {
                    double apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k] = cs * apk - sn * aqk;
                    A[q * n + k] = sn * apk + cs * aqk;
                }
                for (int k = 0; k < n; k++) {
                    double vkp = V[k * n + p], vkq = V[k * n + q];
                    V[k * n + p] = cs * vkp - sn * vkq;
                    V[k * n + q] = sn * vkp + cs * vkq;
                }
            }
    }
    for (int i = 0; i < n; i++) evals[i] = A[i * n + i];
    /* sort ascending (selection sort, stable for ties by index) */
    for (int i = 0; i < n; i++) {
        int m = i;
        for (int j = i + 1; j < n; j++)
            if (evals[j] < evals[m]) m = j;
        if (m != i) {
            double t = evals[i]; evals[i] = evals[m]; evals[m] = t;
            for (int k = 0; k < n; k++) { t = V[k * n + i]; V[k * n + i] = V[k * n + m]; V[k * n + m] = t; }
        }
    }
    for (int j = 0; j < n; j++) {
        int im = 0;
        for (int i = 1; i < n; i++)
            if (fabs(V[i * n + j]) > fabs(V[im * n + j]) + 1e-14) im = i;
        if (V[im * n + j] < 0)
            for (int i = 0; i < n; i++) V[i * n + j] = -V[i * n + j];
    }
    free(A);
}

/* ------------------------------------------------------------------------------------------ */
/* Davidson-Liu (forte/helpers/davidson_liu_solver.cc:45-730)                                  */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
    int nroot, maxiter, collapse_per_root, subspace_per_root, guess_per_root, dets_per_guess;
    int multiplicity;
    double e_conv, r_conv;
} orc_opts;

typedef struct {
    int64_t size;
    int nroot, collapse, subspace, basis, nsig;
    double *b, *sigma, *r, *temp; /* subspace x size row-major */
    double *G, *alpha, *lambda, *lambda_old, *rnorm;
    const double* hdiag;
    int nbad;
    int64_t* bad_len;
    int64_t** bad_idx;
    double** bad_val;
    double e_conv, r_conv;
    int maxiter;
} dlsolver;

static double ddot(int64_t n, const double* x, const double* y) {
    double s = 0.0;
    for (int64_t i = 0; i < n; i++) s += x[i] * y[i];
    return s;
}

/* add_row_and_orthonormalize (davidson_liu_solver.cc:634-687) */
static int add_row_orth(dlsolver* d, double* A, int rowsA, const double* v_in) {
    int64_t N = d->size;
    double* v = A + (int64_t)rowsA * N;
    memcpy(v, v_in, sizeof(double) * N);
    for (int cycle = 0; cycle < 10; cycle++) {
        for (int i = 0; i < rowsA; i++) {
            double* Ai = A + (int64_t)i * N;
            double dv = ddot(N, Ai, v);
            for (int64_t I = 0; I < N; I++) v[I] -= dv * Ai[I];
        }
        double nv = sqrt(ddot(N, v, v));
        if (nv < 1.0e-7) return 0;
        for (int64_t I = 0; I < N; I++) v[I] *= 1.0 / nv;
        double mo = 0.0;
        for (int i = 0; i < rowsA; i++) {
            double o = fabs(ddot(N, A + (int64_t)i * N, v));
            if (o > mo) mo = o;
        }
        double nrm = ddot(N, v, v);
        if (mo < 1.0e-12 && fabs(nrm - 1.0) < 1.0e-12) return 1;
    }
    return 0;
}

static int add_rows_orth(dlsolver* d, double* A, int rowsA, const double* B, int rowsB) {
    int added = 0;
    for (int j = 0; j < rowsB; j++)
        if (add_row_orth(d, A, rowsA + added, B + (int64_t)j * d->size)) added++;
    return added;
}

/* project_out_roots (davidson_liu_solver.cc:590-603) */
static void project_out(dlsolver* d, double* V) {
    for (int k = 0; k < d->nroot; k++) {
        double* vk = V + (int64_t)k * d->size;
        for (int b = 0; b < d->nbad; b++) {
            double ov = 0.0;
            for (int64_t e = 0; e < d->bad_len[b]; e++) ov += vk[d->bad_idx[b][e]] * d->bad_val[b][e];
            for (int64_t e = 0; e < d->bad_len[b]; e++) vk[d->bad_idx[b][e]] -= ov * d->bad_val[b][e];
        }
    }
}

typedef int (*sigma_fn)(void* ctx, const double* b, double* s);

static void dl_gemm_t(dlsolver* d, const double* coef, int nrow_in, int nrow_out, const double* in,
                      double* out) {
    /* out[k] = sum_j coef[j*subspace + k] * in[j] */
    int64_t N = d->size;
    memset(out, 0, sizeof(double) * N * nrow_out);
    for (int k = 0; k < nrow_out; k++)
        for (int j = 0; j < nrow_in; j++) {
            double a = coef[j * d->subspace + k];
            if (a != 0.0) daxpy(N, a, in + (int64_t)j * N, out + (int64_t)k * N);
        }
}

/* DavidsonLiuSolver::solve (davidson_liu_solver.cc:180-273). Returns 1 if converged. */
static int dl_solve(dlsolver* d, sigma_fn sig, void* sctx, const double* guesses, int nguess,
                    const uint8_t* mask, int* iters_out) {
    int64_t N = d->size;
    int m = d->subspace;
    /* setup_guesses */
    memset(d->temp, 0, sizeof(double) * m * N);
    memcpy(d->temp, guesses, sizeof(double) * N * nguess);
    project_out(d, d->temp);
    int should = nguess > d->nroot ? nguess : d->nroot;
    int added = add_rows_orth(d, d->b, 0, d->temp, should);
    if (added != should) { fail("DL: guess vectors are zero or linearly dependent"); return -1; }
    d->basis = added;
    d->nsig = 0;
    for (int k = 0; k < m; k++) d->lambda_old[k] = 0.0;
    int iter = 0;
    int converged = 0;
    for (iter = 0; iter < d->maxiter; iter++) {
        /* compute_sigma */
        for (int j = d->nsig; j < d->basis; j++) {
            sig(sctx, d->b + (int64_t)j * N, d->sigma + (int64_t)j * N);
            if (mask)
                for (int64_t I = 0; I < N; I++)
                    if (!mask[I]) d->sigma[(int64_t)j * N + I] = 0.0;
        }
        d->nsig = d->basis;
        /* form_and_diagonalize_effective_hamiltonian */
        int nb = d->basis;
        double* Gb = (double*)malloc(sizeof(double) * nb * nb);
        for (int i = 0; i < nb; i++)
            for (int j = 0; j < nb; j++) d->G[i * m + j] = ddot(N, d->b + (int64_t)i * N, d->sigma + (int64_t)j * N);
        for (int i = 0; i < nb; i++)
            for (int j = 0; j < nb; j++) Gb[i * nb + j] = 0.5 * (d->G[i * m + j] + d->G[j * m + i]);
        double* ab = (double*)malloc(sizeof(double) * nb * nb);
        double* lb = (double*)malloc(sizeof(double) * nb);
        orc_jacobi(nb, Gb, lb, ab);
        memset(d->alpha, 0, sizeof(double) * m * m);
        for (int i = 0; i < nb; i++)
            for (int j = 0; j < nb; j++) d->alpha[i * m + j] = ab[i * nb + j];
        for (int i = 0; i < m; i++) d->lambda[i] = i < nb ? lb[i] : 0.0;
        free(Gb); free(ab); free(lb);
        /* form_residual_vectors */
        dl_gemm_t(d, d->alpha, nb, d->nroot, d->sigma, d->r);
        dl_gemm_t(d, d->alpha, nb, d->nroot, d->b, d->temp);
        for (int k = 0; k < d->nroot; k++) {
            double lk = d->lambda[k];
            double* rk = d->r + (int64_t)k * N;
            double* tk = d->temp + (int64_t)k * N;
            for (int64_t I = 0; I < N; I++) rk[I] -= lk * tk[I];
        }
        /* compute_residual_norm */
        for (int k = 0; k < d->nroot; k++) {
            double* rk = d->r + (int64_t)k * N;
            d->rnorm[k] = sqrt(ddot(N, rk, rk));
        }
        /* form_correction_vectors */
        for (int k = 0; k < d->nroot; k++) {
            double lk = d->lambda[k];
            double* rk = d->r + (int64_t)k * N;
            for (int64_t I = 0; I < N; I++) {
                double den = lk - d->hdiag[I];
                if (fabs(den) > 1.0e-6) rk[I] /= den;
                else rk[I] = 0.0;
            }
        }
        project_out(d, d->r);
        /* normalize_vectors(r, nroot) */
        for (int k = 0; k < d->nroot; k++) {
            double* rk = d->r + (int64_t)k * N;
            double nv = sqrt(ddot(N, rk, rk));
            for (int64_t I = 0; I < N; I++) rk[I] /= nv;
        }
        /* check_convergence */
        int ne = 0, nr = 0;
        for (int k = 0; k < d->nroot; k++) {
            if (fabs(d->lambda[k] - d->lambda_old[k]) < d->e_conv) ne++;
            if (d->rnorm[k] < d->r_conv) nr++;
        }
        int e_ok = (ne == d->nroot), r_ok = (nr == d->nroot);
        if ((e_ok && r_ok) || d->basis == N) { converged = 1; break; }
        /* subspace_collapse */
        if (d->basis + d->nroot > m) {
            int cs = d->collapse > d->nroot ? d->collapse : d->nroot;
            if (cs > d->basis) cs = d->basis;
            dl_gemm_t(d, d->alpha, d->basis, cs, d->b, d->temp);
            memset(d->b, 0, sizeof(double) * m * N);
            int a2 = add_rows_orth(d, d->b, 0, d->temp, cs);
            dl_gemm_t(d, d->alpha, d->basis, cs, d->sigma, d->temp);
            memcpy(d->sigma, d->temp, sizeof(double) * cs * N);
            if (a2 != cs) { fail("DL: collapse generated fewer vectors than expected"); return -1; }
            d->basis = cs;
            d->nsig = cs;
        }
        int num_to_add = d->nroot < m - d->basis ? d->nroot : m - d->basis;
        int ad = add_rows_orth(d, d->b, d->basis, d->r, num_to_add);
        d->basis += ad;
        if (ad == 0) {
            converged = r_ok ? 1 : 0;
            break;
        }
        for (int k = 0; k < m; k++) d->lambda_old[k] = d->lambda[k];
    }
    if (iters_out) *iters_out = iter + 1;
    /* get_results */
    for (int k = 0; k < m; k++) d->lambda_old[k] = d->lambda[k];
    dl_gemm_t(d, d->alpha, d->basis, d->nroot, d->b, d->temp);
    memset(d->b, 0, sizeof(double) * m * N);
    add_rows_orth(d, d->b, 0, d->temp, d->nroot);
    return converged;
}

/* ------------------------------------------------------------------------------------------ */
/* initial guess (forte/fci/fci_solver_initial_guess.cc:44-103, sparse_initial_guess.cc:72-264) */
/* ------------------------------------------------------------------------------------------ */
typedef struct { uint64_t a, b; } det_t;

/* enforce_spin_completeness (forte/sparse_ci/determinant_functions.cc:133-190) */
static int spin_complete(det_t** dets_io, int ndet, int cap_hint, int nmo) {
    det_t* dets = *dets_io;
    int cap = cap_hint > ndet ? cap_hint : ndet;
    for (int I = 0; I < ndet; I++) {
        uint64_t a = dets[I].a, b = dets[I].b;
        uint64_t closed = a & b, oa = a & ~b, ob = b & ~a;
        int nao = popc(oa), nbo = popc(ob);
        if (nao + nbo == 0) continue;
        int open[64], no = 0;
        for (int i = 0; i < nmo; i++)
            if (((oa | ob) >> i) & 1) open[no++] = i;
        int8_t bits[64];
        for (int i = 0; i < no; i++) bits[i] = (i >= nbo) ? 1 : 0;
        do {
            uint64_t na_ = closed, nb_ = closed;
            for (int o = 0; o < no; o++) {
                if (bits[o]) na_ |= 1ull << open[o];
                else nb_ |= 1ull << open[o];
            }
            int found = 0;
            for (int J = 0; J < ndet; J++)
                if (dets[J].a == na_ && dets[J].b == nb_) { found = 1; break; }
            if (!found) {
                if (ndet == cap) {
                    cap = 2 * cap + 16;
                    dets = (det_t*)realloc(dets, sizeof(det_t) * cap);
                }
                dets[ndet].a = na_;
                dets[ndet].b = nb_;
                ndet++;
            }
        } while (next_perm(bits, no));
    }
    *dets_io = dets;
    return ndet;
}

/* find_integer_groups (forte/helpers/helpers.cc:237-263) */
static int near_int(double v, double t) { return fabs(v - round(v)) <= t; }
static int integer_groups(const double* v, int n, double tol, int* gm, int* gs, int* ge) {
    int ng = 0, it = 0;
    while (it < n) {
        while (it < n && !near_int(v[it], tol)) it++;
        if (it < n) {
            int start = it, end = -1;
            for (int k = it; k + 1 < n; k++)
                if (near_int(v[k], tol) && fabs(v[k] - v[k + 1]) > 2 * tol) { end = k; break; }
            if (end < 0) end = n - 1;
            gm[ng] = (int)llround(v[start]);
            gs[ng] = start;
            ge[ng] = end + 1;
            ng++;
            it = end + 1;
        }
    }
    return ng;
}

/* Builds guess vectors (dense, ndet each) and bad roots (dense).  Returns nguess or -1. */
static int make_guess(orc_ctx* c, const double* hdiag, int num_guess_states, int dets_per_guess,
                      int multiplicity, double** guesses_out, int* nbad_out, double** bad_out) {
    int64_t N = c->ndet;
    int64_t ng = (int64_t)num_guess_states * dets_per_guess;
    if (ng > N) ng = N;
    /* initial_guess_generate_dets: insertion into a sorted list of the lowest diagonals */
    double* ve = (double*)malloc(sizeof(double) * ng);
    int64_t* vi = (int64_t*)malloc(sizeof(int64_t) * ng);
    double emax = 1.7976931348623157e308;
    for (int64_t t = 0; t < ng; t++) { ve[t] = emax; vi[t] = 0; }
    int64_t added = 0;
    for (int64_t I = 0; I < N; I++) {
        if (c->mask && !c->mask[I]) continue;
        double e = hdiag[I];
        if (e < emax || added < num_guess_states) {
            int64_t pos = 0;
            while (pos < ng - 1 && !(e < ve[pos])) pos++;
            /* pop_back then insert at pos */
            for (int64_t t = ng - 1; t > pos; t--) { ve[t] = ve[t - 1]; vi[t] = vi[t - 1]; }
            ve[pos] = e;
            vi[pos] = I;
            emax = ve[ng - 1];
            added++;
        }
    }
    int nd = (int)ng;
    det_t* dets = (det_t*)malloc(sizeof(det_t) * nd);
    for (int t = 0; t < nd; t++) {
        int64_t I = vi[t];
        dets[t].a = c->A.str[I / c->nbs];
        dets[t].b = c->B.str[I % c->nbs];
    }
    nd = spin_complete(&dets, nd, nd, c->n);
    free(ve); free(vi);
    int64_t* pos = (int64_t*)malloc(sizeof(int64_t) * nd);
    for (int t = 0; t < nd; t++)
        pos[t] = (int64_t)c->A.addr[dets[t].a] * c->nbs + c->B.addr[dets[t].b];
    /* compute_s2_transformed_hamiltonian_matrix (sparse_initial_guess.cc:52-68) */
    double* S2 = (double*)malloc(sizeof(double) * nd * nd);
    double* S2v = (double*)malloc(sizeof(double) * nd * nd);
    double* S2e = (double*)malloc(sizeof(double) * nd);
    for (int i = 0; i < nd; i++)
        for (int j = i; j < nd; j++) {
            double v = det_spin2(dets[i].a, dets[i].b, dets[j].a, dets[j].b, c->n);
            S2[i * nd + j] = v;
            S2[j * nd + i] = v;
        }
    orc_jacobi(nd, S2, S2e, S2v);
    double* H = (double*)malloc(sizeof(double) * nd * nd);
    double esave = c->e0;
    c->e0 = 0.0;
    for (int i = 0; i < nd; i++)
        for (int j = i; j < nd; j++) {
            double v = slater_rules(c, dets[i].a, dets[i].b, dets[j].a, dets[j].b);
            H[i * nd + j] = v;
            H[j * nd + i] = v;
        }
    c->e0 = esave;
    /* H -> S2v^T H S2v */
    double* T1 = (double*)calloc((size_t)nd * nd, sizeof(double));
    double* HS = (double*)calloc((size_t)nd * nd, sizeof(double));
    for (int i = 0; i < nd; i++)
        for (int k = 0; k < nd; k++) {
            double a = H[i * nd + k];
            if (a == 0.0) continue;
            for (int j = 0; j < nd; j++) T1[i * nd + j] += a * S2v[k * nd + j];
        }
    for (int k = 0; k < nd; k++)
        for (int i = 0; i < nd; i++) {
            double a = S2v[k * nd + i];
            if (a == 0.0) continue;
            for (int j = 0; j < nd; j++) HS[i * nd + j] += a * T1[k * nd + j];
        }
    double* mult = (double*)malloc(sizeof(double) * nd);
    for (int i = 0; i < nd; i++) mult[i] = sqrt(1.0 + 4.0 * S2e[i]);
    int* gm = (int*)malloc(sizeof(int) * (nd + 1));
    int* gs = (int*)malloc(sizeof(int) * (nd + 1));
    int* ge = (int*)malloc(sizeof(int) * (nd + 1));
    int ngr = integer_groups(mult, nd, 1.0e-6, gm, gs, ge);
    /* per group: diagonalize the H block, C = S2v[:, block] * evecs */
    double** gE = (double**)calloc(ngr + 1, sizeof(double*));
    double** gC = (double**)calloc(ngr + 1, sizeof(double*));
    int* gsz = (int*)calloc(ngr + 1, sizeof(int));
    int target = -1;
    for (int g = 0; g < ngr; g++) {
        int bs = ge[g] - gs[g];
        gsz[g] = bs;
        double* Hb = (double*)malloc(sizeof(double) * bs * bs);
        for (int i = 0; i < bs; i++)
            for (int j = 0; j < bs; j++) Hb[i * bs + j] = HS[(gs[g] + i) * nd + gs[g] + j];
        double* ev = (double*)malloc(sizeof(double) * bs);
        double* evv = (double*)malloc(sizeof(double) * bs * bs);
        orc_jacobi(bs, Hb, ev, evv);
        gE[g] = ev;
        gC[g] = (double*)calloc((size_t)nd * bs, sizeof(double));
        for (int i = 0; i < nd; i++)
            for (int r = 0; r < bs; r++) {
                double s = 0.0;
                for (int k = 0; k < bs; k++) s += S2v[i * nd + gs[g] + k] * evv[k * bs + r];
                gC[g][i * bs + r] = s;
            }
        free(Hb); free(evv);
        if (gm[g] == multiplicity) target = g;
    }
    int ret = num_guess_states;
    if (multiplicity == 0) {
        /* extension used by the synthetic benchmarks: no spin selection, the lowest states of the
         * guess Hamiltonian of any multiplicity, nothing projected out */
        double* Hc = (double*)malloc(sizeof(double) * nd * nd);
        double* ev = (double*)malloc(sizeof(double) * nd);
        double* evv = (double*)malloc(sizeof(double) * nd * nd);
        memcpy(Hc, H, sizeof(double) * nd * nd);
        orc_jacobi(nd, Hc, ev, evv);
        if (nd < num_guess_states) { ret = fail("guess space smaller than the number of guess states"); }
        else {
            double* G = (double*)calloc((size_t)N * num_guess_states, sizeof(double));
            for (int r = 0; r < num_guess_states; r++)
                for (int i = 0; i < nd; i++) G[(int64_t)r * N + pos[i]] = evv[i * nd + r];
            *guesses_out = G;
            *nbad_out = 0;
            *bad_out = NULL;
        }
        free(Hc); free(ev); free(evv);
        goto done;
    }
    if (target < 0) { ret = fail("No guess with the requested multiplicity was found."); goto done; }
    if (gsz[target] < num_guess_states) {
        ret = fail("Found fewer guesses with the requested multiplicity than requested; increase DL_DETS_PER_GUESS");
        goto done;
    }
    {
        double* G = (double*)calloc((size_t)N * num_guess_states, sizeof(double));
        double gmax = -1.7976931348623157e308;
        for (int r = 0; r < num_guess_states; r++) {
            for (int i = 0; i < nd; i++) G[(int64_t)r * N + pos[i]] = gC[target][i * gsz[target] + r];
            if (gE[target][r] > gmax) gmax = gE[target][r];
        }
        *guesses_out = G;
        int nbad = 0;
        double* B = NULL;
        for (int g = 0; g < ngr; g++) {
            if (g == target) continue;
            for (int r = 0; r < gsz[g]; r++)
                if (gE[g][r] < gmax) {
                    B = (double*)realloc(B, sizeof(double) * N * (nbad + 1));
                    memset(B + (int64_t)nbad * N, 0, sizeof(double) * N);
                    for (int i = 0; i < nd; i++) B[(int64_t)nbad * N + pos[i]] = gC[g][i * gsz[g] + r];
                    nbad++;
                }
        }
        *nbad_out = nbad;
        *bad_out = B;
    }
done:
    for (int g = 0; g < ngr; g++) { free(gE[g]); free(gC[g]); }
    free(gE); free(gC); free(gsz); free(gm); free(gs); free(ge); free(mult);
    free(T1); free(HS); free(H); free(S2); free(S2v); free(S2e); free(pos); free(dets);
    return ret;
}

static int sigma_masked(void* h, const double* b, double* s) { return orc_sigma(h, b, s); }

/* FCISolver::compute_energy (forte/fci/fci_solver.cc:177-314), without printing.
 * energies[nroot]; evecs[nroot*ndet] (may be NULL); returns 1 converged, 0 not, -1 error. */
int orc_solve(void* h, const int* iopts, const double* dopts, double* energies, double* evecs,
              int* iters) {
    orc_ctx* c = (orc_ctx*)h;
    if (!c->has_ints) return fail("orc_solve: integrals not set");
    orc_opts o;
    o.nroot = iopts[0]; o.maxiter = iopts[1]; o.collapse_per_root = iopts[2];
    o.subspace_per_root = iopts[3]; o.guess_per_root = iopts[4]; o.dets_per_guess = iopts[5];
    o.multiplicity = iopts[6];
    o.e_conv = dopts[0]; o.r_conv = dopts[1];
    int64_t N = c->ndet;
    int64_t Neff = 0;
    for (int64_t I = 0; I < N; I++) Neff += c->mask[I];
    if (Neff == 0) return fail("DavidsonLiuSolver called with space of dimension zero.");
    if (o.nroot < 1) return fail("DavidsonLiuSolver called with zero roots.");
    if (o.collapse_per_root < 1) return fail("DavidsonLiuSolver: collapse_per_root must be >= 1");
    if (o.subspace_per_root < o.collapse_per_root + 1)
        return fail("DavidsonLiuSolver: subspace_per_root must be >= collapse_per_root + 1");
    dlsolver d;
    memset(&d, 0, sizeof(d));
    d.size = N;
    d.nroot = o.nroot;
    d.collapse = (int)(o.collapse_per_root * o.nroot < Neff ? o.collapse_per_root * o.nroot : Neff);
    d.subspace = (int)(o.subspace_per_root * o.nroot < Neff ? o.subspace_per_root * o.nroot : Neff);
    d.e_conv = o.e_conv; d.r_conv = o.r_conv; d.maxiter = o.maxiter;
    int m = d.subspace;
    d.b = (double*)calloc((size_t)m * N, 8);
    d.sigma = (double*)calloc((size_t)m * N, 8);
    d.r = (double*)calloc((size_t)m * N, 8);
    d.temp = (double*)calloc((size_t)m * N, 8);
    d.G = (double*)calloc((size_t)m * m, 8);
    d.alpha = (double*)calloc((size_t)m * m, 8);
    d.lambda = (double*)calloc(m, 8);
    d.lambda_old = (double*)calloc(m, 8);
    d.rnorm = (double*)calloc(o.nroot, 8);
    double* hd = (double*)malloc(sizeof(double) * N);
    orc_hdiag(h, hd);
    d.hdiag = hd;
    int num_guess_states = o.guess_per_root * o.nroot;
    if (num_guess_states > Neff) num_guess_states = (int)Neff;
    double* guesses = NULL;
    double* bad = NULL;
    int nbad = 0;
    int ng = make_guess(c, hd, num_guess_states, o.dets_per_guess, o.multiplicity, &guesses, &nbad, &bad);
    int ret;
    if (ng < 0) { ret = -1; goto out; }
    if (ng < o.nroot || ng > m) { ret = fail("DavidsonLiuSolver: bad number of guess vectors"); goto out; }
    d.nbad = nbad;
    d.bad_len = (int64_t*)calloc(nbad + 1, sizeof(int64_t));
    d.bad_idx = (int64_t**)calloc(nbad + 1, sizeof(int64_t*));
    d.bad_val = (double**)calloc(nbad + 1, sizeof(double*));
    for (int b = 0; b < nbad; b++) {
        int64_t cnt = 0;
        for (int64_t I = 0; I < N; I++) if (bad[(int64_t)b * N + I] != 0.0) cnt++;
        d.bad_len[b] = cnt;
        d.bad_idx[b] = (int64_t*)malloc(sizeof(int64_t) * (cnt + 1));
        d.bad_val[b] = (double*)malloc(sizeof(double) * (cnt + 1));
        cnt = 0;
        for (int64_t I = 0; I < N; I++)
            if (bad[(int64_t)b * N + I] != 0.0) { d.bad_idx[b][cnt] = I; d.bad_val[b][cnt] = bad[(int64_t)b * N + I]; cnt++; }
    }
    ret = dl_solve(&d, sigma_masked, c, guesses, ng, c->mask, iters);
    if (ret >= 0) {
        for (int k = 0; k < o.nroot; k++) energies[k] = d.lambda[k];
        if (evecs) memcpy(evecs, d.b, sizeof(double) * N * o.nroot);
    }
    for (int b = 0; b < nbad; b++) { free(d.bad_idx[b]); free(d.bad_val[b]); }
    free(d.bad_len); free(d.bad_idx); free(d.bad_val);
out:
    free(guesses); free(bad); free(hd);
    free(d.b); free(d.sigma); free(d.r); free(d.temp); free(d.G); free(d.alpha);
    free(d.lambda); free(d.lambda_old); free(d.rnorm);
    return ret;
}

/* ------------------------------------------------------------------------------------------ */
/* <S^2> (forte/fci/fci_vector_spin2.cc:38-75)                                                 */
/* ------------------------------------------------------------------------------------------ */
double orc_spin2(void* h, const double* C) {
    orc_ctx* c = (orc_ctx*)h;
    int n = c->n;
    int64_t nbs = c->nbs;
    double s2 = 0.0;
    for (int r = 0; r < n; r++)
        for (int s = 0; s < n; s++) {
            sublist* va = &c->A.vo[s * n + r];
            sublist* vb = &c->B.vo[r * n + s];
            for (int64_t x = 0; x < va->len; x++)
                for (int64_t y = 0; y < vb->len; y++)
                    s2 += C[(int64_t)va->J[x] * nbs + vb->J[y]] * C[(int64_t)va->I[x] * nbs + vb->I[y]] *
                          va->sign[x] * vb->sign[y];
        }
    double na = c->na, nb = c->nb;
    return -s2 + 0.25 * (na - nb) * (na - nb) + 0.5 * (na + nb);
}

/* ------------------------------------------------------------------------------------------ */
/* RDMs (forte/fci/fci_vector_rdm.cc:151-393).  g1[n*n], g2[n^4] row-major; g1[p*n+q] =        */
/* <L|a+_p a_q|R>, g2aa[pqrs] = <L|a+_p a+_q a_s a_r|R>, g2ab[pqrs] = <a+_pa a+_qb a_sb a_ra>.  */
/* ------------------------------------------------------------------------------------------ */
static void rdm1(orc_ctx* c, const double* L, const double* R, double* g, int alfa) {
    int n = c->n;
    spinlists* S = alfa ? &c->A : &c->B;
    memset(g, 0, sizeof(double) * n * n);
    if (S->k < 1) return;
    int64_t maxL = alfa ? c->nbs : c->nas;
    const double *Cl = L, *Cr = R;
    double *tl = NULL, *tr = NULL;
    if (!alfa) {
        tl = (double*)malloc(sizeof(double) * c->ndet);
        tr = (double*)malloc(sizeof(double) * c->ndet);
        transpose(L, tl, c->nas, c->nbs);
        transpose(R, tr, c->nas, c->nbs);
        Cl = tl; Cr = tr;
    }
    for (int p = 0; p < n; p++)
        for (int q = 0; q < n; q++) {
            sublist* l = &S->vo[p * n + q];
            double el = 0.0;
            for (int64_t e = 0; e < l->len; e++)
                el += l->sign[e] * ddot(maxL, Cl + (int64_t)l->J[e] * maxL, Cr + (int64_t)l->I[e] * maxL);
            g[p * n + q] += el;
        }
    free(tl); free(tr);
}

#define TIDX(p, q, r, s) ((((size_t)(p) * n + (q)) * n + (r)) * n + (s))
static void rdm2_same(orc_ctx* c, const double* L, const double* R, double* g, int alfa) {
    int n = c->n;
    spinlists* S = alfa ? &c->A : &c->B;
    memset(g, 0, sizeof(double) * n * n * n * n);
    if (S->k < 2) return;
    int64_t maxL = alfa ? c->nbs : c->nas;
    const double *Cl = L, *Cr = R;
    double *tl = NULL, *tr = NULL;
    if (!alfa) {
        tl = (double*)malloc(sizeof(double) * c->ndet);
        tr = (double*)malloc(sizeof(double) * c->ndet);
        transpose(L, tl, c->nas, c->nbs);
        transpose(R, tr, c->nas, c->nbs);
        Cl = tl; Cr = tr;
    }
    int np = n * (n - 1) / 2;
    int* pp = (int*)malloc(sizeof(int) * (np + 1));
    int* qq = (int*)malloc(sizeof(int) * (np + 1));
    int t = 0;
    for (int p = 0; p < n; p++)
        for (int q = 0; q < p; q++) { pp[t] = p; qq[t] = q; t++; }
    for (int pq = 0; pq < np; pq++) {
        int p = pp[pq], q = qq[pq];
        sublist* l = &S->oo[pq];
        double el = 0.0;
        for (int64_t e = 0; e < l->len; e++)
            el += l->sign[e] * ddot(maxL, Cl + (int64_t)l->J[e] * maxL, Cr + (int64_t)l->I[e] * maxL);
        g[TIDX(p, q, p, q)] += el;
        g[TIDX(p, q, q, p)] -= el;
        g[TIDX(q, p, p, q)] -= el;
        g[TIDX(q, p, q, p)] += el;
    }
    for (int pq = 0; pq < np; pq++) {
        int p = pp[pq], q = qq[pq];
        for (int rs = 0; rs < pq; rs++) {
            int r = pp[rs], s = qq[rs];
            sublist* l = &S->vvoo[((p * n + q) * n + r) * n + s];
            double el = 0.0;
            for (int64_t e = 0; e < l->len; e++)
                el += l->sign[e] * ddot(maxL, Cl + (int64_t)l->J[e] * maxL, Cr + (int64_t)l->I[e] * maxL);
            g[TIDX(p, q, r, s)] += el;
            g[TIDX(q, p, r, s)] -= el;
            g[TIDX(p, q, s, r)] -= el;
            g[TIDX(q, p, s, r)] += el;
            g[TIDX(r, s, p, q)] += el;
            g[TIDX(r, s, q, p)] -= el;
            g[TIDX(s, r, p, q)] -= el;
            g[TIDX(s, r, q, p)] += el;
        }
    }
    free(pp); free(qq); free(tl); free(tr);
}

static void rdm2_ab(orc_ctx* c, const double* L, const double* R, double* g) {
    int n = c->n;
    memset(g, 0, sizeof(double) * n * n * n * n);
    if (c->na < 1 || c->nb < 1) return;
    int64_t nbs = c->nbs;
    for (int r = 0; r < n; r++)
        for (int s = 0; s < n; s++) {
            sublist* vb = &c->B.vo[r * n + s];
            for (int p = 0; p < n; p++)
                for (int q = 0; q < n; q++) {
                    sublist* va = &c->A.vo[p * n + q];
                    double el = 0.0;
                    for (int64_t x = 0; x < va->len; x++) {
                        const double* cl = L + (int64_t)va->J[x] * nbs;
                        const double* cr = R + (int64_t)va->I[x] * nbs;
                        double sa = va->sign[x];
                        for (int64_t y = 0; y < vb->len; y++)
                            el += cl[vb->J[y]] * cr[vb->I[y]] * sa * vb->sign[y];
                    }
                    g[TIDX(p, r, q, s)] += el;
                }
        }
}

int orc_rdms(void* h, const double* L, const double* R, int level, double* g1a, double* g1b,
             double* g2aa, double* g2ab, double* g2bb) {
    orc_ctx* c = (orc_ctx*)h;
    if (level >= 1) { rdm1(c, L, R, g1a, 1); rdm1(c, L, R, g1b, 0); }
    if (level >= 2) { rdm2_same(c, L, R, g2aa, 1); rdm2_same(c, L, R, g2bb, 0); rdm2_ab(c, L, R, g2ab); }
    return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* 3-RDMs (FCIVector::compute_3rdm_aaa/aab/abb_same_irrep, forte/fci/fci_vector_rdm.cc:395-565), */
/* restated over the 1h/2h/3h string lists of FCIStringLists::make_1h/2h/3h_list               */
/* (fci_string_hole_list.cc:59-223).  An entry (sign, o1[, o2[, o3]], I) of the list of the    */
/* (k-h)-string K means <K| a_o1 [a_o2 [a_o3]] |I> = sign; the 2h and 3h lists hold every       */
/* ordering of the removed orbitals.  Blocks are n^6 row-major, filled with the reference's     */
/* loops: the first index triple comes from the entries of the right vector, the second from    */
/* those of the left vector.                                                                   */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
    double sign;
    int o[3];
    uint32_t I; /* address of the k-string */
} hentry;

#define SIX(p, q, r, s, t, u) \
    ((((((size_t)(p) * n + (q)) * n + (r)) * n + (s)) * n + (t)) * n + (u))

/* the h-hole list of the (k-h)-string K over the k-strings of S; returns the entry count */
static int hole_list(const spinlists* S, uint64_t K, int h, hentry* out) {
    int n = S->n, cnt = 0;
    if (h == 1) {
        for (int p = 0; p < n; p++) {
            if (K >> p & 1) continue;
            hentry e = {sgn_below(K, p), {p, 0, 0}, (uint32_t)addr_of(S, K | 1ull << p)};
            out[cnt++] = e;
        }
    } else if (h == 2) {
        for (int q = 0; q < n; q++)
            for (int p = q + 1; p < n; p++) {
                if ((K >> p & 1) || (K >> q & 1)) continue;
                /* make_2h_list: remove q, then p */
                double s = sgn_below(K | 1ull << p, q) * sgn_below(K, p);
                uint32_t I = (uint32_t)addr_of(S, K | 1ull << p | 1ull << q);
                hentry a = {s, {p, q, 0}, I}, b = {-s, {q, p, 0}, I};
                out[cnt++] = a;
                out[cnt++] = b;
            }
    } else {
        for (int r = 0; r < n; r++)
            for (int q = r + 1; q < n; q++)
                for (int p = q + 1; p < n; p++) {
                    if ((K >> p & 1) || (K >> q & 1) || (K >> r & 1)) continue;
                    /* make_3h_list: remove r, then q, then p */
                    double s = sgn_below(K | 1ull << p | 1ull << q, r) * sgn_below(K | 1ull << p, q) * sgn_below(K, p);
                    uint32_t I = (uint32_t)addr_of(S, K | 1ull << p | 1ull << q | 1ull << r);
                    hentry e[6] = {{+s, {p, q, r}, I}, {-s, {p, r, q}, I}, {-s, {q, p, r}, I},
                                   {+s, {q, r, p}, I}, {-s, {r, q, p}, I}, {+s, {r, p, q}, I}};
                    for (int x = 0; x < 6; x++) out[cnt++] = e[x];
                }
    }
    return cnt;
}

/* all (k-h)-strings of n orbitals, in any order; returns the count */
static int64_t hole_strings(int n, int kh, uint64_t** out) {
    int64_t ns = binom(n, kh);
    *out = (uint64_t*)malloc(sizeof(uint64_t) * (ns > 0 ? ns : 1));
    if (ns > 0) orc_make_strings(n, kh, *out);
    return ns;
}

/* compute_3rdm_aaa_same_irrep (fci_vector_rdm.cc:395-437): rdm[p,q,r,s,t,u] += sign_K sign_L
 * <Cl[J], Cr[I]> over the pairs of entries (sign_K, p, q, r, I), (sign_L, s, t, u, J) of one
 * 3h list; the dots are formed once per pair of strings */
static void rdm3_same(orc_ctx* c, const double* L, const double* R, double* g, int alfa) {
    int n = c->n;
    spinlists* S = alfa ? &c->A : &c->B;
    memset(g, 0, sizeof(double) * (size_t)n * n * n * n * n * n);
    if (S->k < 3) return;
    int64_t maxL = alfa ? c->nbs : c->nas;
    const double *Cl = L, *Cr = R;
    double *tl = NULL, *tr = NULL;
    if (!alfa) {
        tl = (double*)malloc(sizeof(double) * c->ndet);
        tr = (double*)malloc(sizeof(double) * c->ndet);
        transpose(L, tl, c->nas, c->nbs);
        transpose(R, tr, c->nas, c->nbs);
        Cl = tl; Cr = tr;
    }
    uint64_t* Ks = NULL;
    int64_t nK = hole_strings(n, S->k - 3, &Ks);
    hentry* e = (hentry*)malloc(sizeof(hentry) * 6 * (size_t)binom(n, 3));
    int m3 = (int)binom(n - S->k + 3, 3);
    double* D = (double*)malloc(sizeof(double) * (size_t)m3 * m3);
    for (int64_t k = 0; k < nK; k++) {
        int cnt = hole_list(S, Ks[k], 3, e);
        int nr = cnt / 6; /* distinct strings: entries 6x, 6x+1, ... share I */
        for (int a = 0; a < nr; a++)
            for (int b = 0; b < nr; b++)
                D[a * nr + b] = ddot(maxL, Cl + (int64_t)e[6 * b].I * maxL, Cr + (int64_t)e[6 * a].I * maxL);
        for (int x = 0; x < cnt; x++)
            for (int y = 0; y < cnt; y++) {
                const hentry* K = &e[x];
                const hentry* J = &e[y];
                g[SIX(K->o[0], K->o[1], K->o[2], J->o[0], J->o[1], J->o[2])] +=
                    K->sign * J->sign * D[(x / 6) * nr + (y / 6)];
            }
    }
    free(D); free(e); free(Ks); free(tl); free(tr);
}

/* compute_3rdm_aab_same_irrep (fci_vector_rdm.cc:439-502) */
static void rdm3_aab(orc_ctx* c, const double* L, const double* R, double* g) {
    int n = c->n;
    memset(g, 0, sizeof(double) * (size_t)n * n * n * n * n * n);
    if (c->A.k < 2 || c->B.k < 1) return;
    int64_t nbs = c->nbs;
    uint64_t *Ka = NULL, *Kb = NULL;
    int64_t nKa = hole_strings(n, c->A.k - 2, &Ka), nKb = hole_strings(n, c->B.k - 1, &Kb);
    hentry* I2 = (hentry*)malloc(sizeof(hentry) * 2 * (size_t)binom(n, 2));
    hentry* M1 = (hentry*)malloc(sizeof(hentry) * (size_t)n);
    for (int64_t ka = 0; ka < nKa; ka++) {
        int ni = hole_list(&c->A, Ka[ka], 2, I2);
        for (int64_t kb = 0; kb < nKb; kb++) {
            int nm = hole_list(&c->B, Kb[kb], 1, M1);
            for (int x = 0; x < ni; x++) {
                int q = I2[x].o[0], p = I2[x].o[1];
                const double* Cr = R + (int64_t)I2[x].I * nbs;
                for (int y = 0; y < ni; y++) {
                    int t = I2[y].o[0], s = I2[y].o[1];
                    const double* Cl = L + (int64_t)I2[y].I * nbs;
                    for (int u = 0; u < nm; u++) {
                        int r = M1[u].o[0];
                        double cr = Cr[M1[u].I];
                        if (cr == 0.0) continue;
                        for (int v = 0; v < nm; v++) {
                            int a = M1[v].o[0];
                            double sign = I2[x].sign * I2[y].sign * M1[u].sign * M1[v].sign;
                            g[SIX(p, q, r, s, t, a)] += sign * cr * Cl[M1[v].I];
                        }
                    }
                }
            }
        }
    }
    free(I2); free(M1); free(Ka); free(Kb);
}

/* compute_3rdm_abb_same_irrep (fci_vector_rdm.cc:504-565) */
static void rdm3_abb(orc_ctx* c, const double* L, const double* R, double* g) {
    int n = c->n;
    memset(g, 0, sizeof(double) * (size_t)n * n * n * n * n * n);
    if (c->A.k < 1 || c->B.k < 2) return;
    int64_t nbs = c->nbs;
    uint64_t *Ka = NULL, *Kb = NULL;
    int64_t nKa = hole_strings(n, c->A.k - 1, &Ka), nKb = hole_strings(n, c->B.k - 2, &Kb);
    hentry* I1 = (hentry*)malloc(sizeof(hentry) * (size_t)n);
    hentry* M2 = (hentry*)malloc(sizeof(hentry) * 2 * (size_t)binom(n, 2));
    for (int64_t ka = 0; ka < nKa; ka++) {
        int ni = hole_list(&c->A, Ka[ka], 1, I1);
        for (int64_t kb = 0; kb < nKb; kb++) {
            int nm = hole_list(&c->B, Kb[kb], 2, M2);
            for (int x = 0; x < ni; x++) {
                int p = I1[x].o[0];
                const double* Cr = R + (int64_t)I1[x].I * nbs;
                for (int u = 0; u < nm; u++) {
                    int q = M2[u].o[0], r = M2[u].o[1];
                    double cr = Cr[M2[u].I];
                    if (cr == 0.0) continue;
                    for (int y = 0; y < ni; y++) {
                        int s = I1[y].o[0];
                        const double* Cl = L + (int64_t)I1[y].I * nbs;
                        for (int v = 0; v < nm; v++) {
                            int t = M2[v].o[0], a = M2[v].o[1];
                            double sign = I1[x].sign * I1[y].sign * M2[u].sign * M2[v].sign;
                            g[SIX(p, q, r, s, t, a)] += sign * cr * Cl[M2[v].I];
                        }
                    }
                }
            }
        }
    }
    free(I1); free(M2); free(Ka); free(Kb);
}

int orc_rdms3(void* h, const double* L, const double* R, double* g3aaa, double* g3aab, double* g3abb,
              double* g3bbb) {
    orc_ctx* c = (orc_ctx*)h;
    if (c->n > 12) return fail("orc_rdms3: at most 12 orbitals");
    rdm3_same(c, L, R, g3aaa, 1);
    rdm3_aab(c, L, R, g3aab);
    rdm3_abb(c, L, R, g3abb);
    rdm3_same(c, L, R, g3bbb, 0);
    return 0;
}
