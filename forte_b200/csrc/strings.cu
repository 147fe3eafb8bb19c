// Device construction of the alpha/beta string tables (integer arithmetic only).
//
// Reference ordering (forte/fci/fci_string_lists.cc:258-293): strings of k electrons in n
// orbitals are enumerated with std::next_permutation over the occupation sequence
// (element 0 most significant) starting from 0..01..1.  That order is the colexicographic
// order of the occupied positions c = n-1-i, so the address of a string is
//     rank(S) = sum_t C(c_t, t),  c_1 < c_2 < ... < c_k,
// and unrank() inverts it.  This replaces FCIStringAddress's hash map
// (forte/fci/fci_string_address.cc:36-75) with closed-form integer arithmetic.
#include <algorithm>
#include <cstdio>

#include "fcib_internal.h"

namespace fcib {

__constant__ uint32_t d_binom[33][33];

static Binom make_binom() {
    Binom b;
    for (int i = 0; i <= 32; i++)
        for (int j = 0; j <= 32; j++) {
            if (j > i) b.c[i][j] = 0;
            else if (j == 0 || j == i) b.c[i][j] = 1;
            else b.c[i][j] = b.c[i - 1][j - 1] + b.c[i - 1][j];
        }
    return b;
}
const Binom& host_binom() {
    static Binom b = make_binom();
    return b;
}

uint32_t host_rank(uint32_t s, int n) {
    const Binom& B = host_binom();
    uint32_t r = 0;
    int t = 1;
    for (int i = n - 1; i >= 0; i--)
        if (s >> i & 1u) r += B.c[n - 1 - i][t++];
    return r;
}

uint32_t host_unrank(uint32_t idx, int n, int k) {
    const Binom& B = host_binom();
    uint32_t s = 0;
    int c = n - 1;
    for (int t = k; t >= 1; t--) {
        while (B.c[c][t] > idx) c--;
        idx -= B.c[c][t];
        s |= 1u << (n - 1 - c);
        c--;
    }
    return s;
}

__device__ __forceinline__ uint32_t d_rank(uint32_t s, int n) {
    uint32_t r = 0;
    int t = 1;
    while (s) {
        int i = 31 - __clz(s);
        s ^= 1u << i;
        r += d_binom[n - 1 - i][t++];
    }
    return r;
}

__device__ __forceinline__ uint32_t d_unrank(uint32_t idx, int n, int k) {
    uint32_t s = 0;
    int c = n - 1;
    for (int t = k; t >= 1; t--) {
        while (d_binom[c][t] > idx) c--;
        idx -= d_binom[c][t];
        s |= 1u << (n - 1 - c);
        c--;
    }
    return s;
}

// parity of the set bits strictly between orbitals a and b
__device__ __forceinline__ uint32_t d_between_parity(uint32_t s, int a, int b) {
    int lo = a < b ? a : b, hi = a < b ? b : a;
    uint32_t m = (hi - lo < 2) ? 0u : (((1u << hi) - 1u) & ~((2u << lo) - 1u));
    return __popc(s & m) & 1u;
}

__device__ __forceinline__ int pair_index(int p, int q) {  // p >= q, diagonal included
    return p * (p + 1) / 2 + q;
}

__global__ void k_unrank(uint32_t* out, int nstr, int n, int k) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nstr) out[i] = d_unrank(i, n, k);
}

// conn[I][e]: all (J, P, sign) with <I|F_P|J> = sign, F_P = E_pq + E_qp (p>q) or E_pp,
// emitted in increasing pair index P.
__global__ void k_conn(const uint32_t* str, uint32_t* conn, int nstr, int n, int s1) {
    int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= nstr) return;
    uint32_t s = str[I];
    int e = 0;
    for (int p = 0; p < n; p++)
        for (int q = 0; q <= p; q++) {
            uint32_t bp = s >> p & 1u, bq = s >> q & 1u;
            uint32_t J;
            uint32_t neg = 0;
            if (p == q) {
                if (!bp) continue;
                J = I;
            } else {
                if (bp == bq) continue;
                uint32_t js = s ^ (1u << p) ^ (1u << q);
                J = d_rank(js, n);
                neg = d_between_parity(s, p, q);
            }
            conn[(size_t)I * s1 + e] = J | ((uint32_t)pair_index(p, q) << 21) | (neg << 31);
            e++;
        }
}

// tgt[J][R]: F_R J = sign * I  ->  I | sign << 31, or kNoTarget when F_R J = 0.
__global__ void k_tgt(const uint32_t* str, int32_t* tgt, int nstr, int n, int npair_pad) {
    int J = blockIdx.x;
    if (J >= nstr) return;
    uint32_t s = str[J];
    for (int R = threadIdx.x; R < npair_pad; R += blockDim.x) {
        int32_t out = kNoTarget;
        if (R < n * (n + 1) / 2) {
            int r = (int)((sqrtf(8.0f * R + 1.0f) - 1.0f) * 0.5f);
            while (r * (r + 1) / 2 > R) r--;
            while ((r + 1) * (r + 2) / 2 <= R) r++;
            int q = R - r * (r + 1) / 2;
            uint32_t br = s >> r & 1u, bq = s >> q & 1u;
            if (r == q) {
                if (br) out = J;
            } else if (br != bq) {
                uint32_t is = s ^ (1u << r) ^ (1u << q);
                out = (int32_t)(d_rank(is, n) | (d_between_parity(s, r, q) << 31));
            }
        }
        tgt[(size_t)J * npair_pad + R] = out;
    }
}

// Groups of strings sharing an (N-h)-electron core K (h = 1 or 2).  For h = 2 the rows are
// I = K + {p, q} for particle pairs p > q (label p(p-1)/2 + q) with sign of a+_p a+_q |K>;
// for h = 1 the rows are I = K + {p} (label p) with sign of a+_p |K>.
__global__ void k_groups(uint32_t* rows, uint16_t* labs, int ngroups, int G, int n, int k, int h) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ngroups) return;
    uint32_t K = d_unrank(g, n, k - h);
    int e = 0;
    if (h == 2) {
        for (int p = 0; p < n; p++) {
            if (K >> p & 1u) continue;
            for (int q = 0; q < p; q++) {
                if (K >> q & 1u) continue;
                uint32_t below_q = __popc(K & ((1u << q) - 1u));
                uint32_t below_p = __popc(K & ((1u << p) - 1u));
                uint32_t neg = (below_q + below_p + 1u) & 1u;
                uint32_t I = d_rank(K | (1u << p) | (1u << q), n);
                rows[(size_t)g * G + e] = I | (neg << 31);
                labs[(size_t)g * G + e] = (uint16_t)(p * (p - 1) / 2 + q);
                e++;
            }
        }
    } else {
        for (int p = 0; p < n; p++) {
            if (K >> p & 1u) continue;
            uint32_t neg = __popc(K & ((1u << p) - 1u)) & 1u;
            uint32_t I = d_rank(K | (1u << p), n);
            rows[(size_t)g * G + e] = I | (neg << 31);
            labs[(size_t)g * G + e] = (uint16_t)p;
            e++;
        }
    }
}

static bool binom_uploaded_for_device[64] = {false};

static void upload_binom() {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && binom_uploaded_for_device[dev]) return;
    const Binom& b = host_binom();
    FCIB_CUDA(cudaMemcpyToSymbol(d_binom, b.c, sizeof(b.c)));
    if (dev >= 0 && dev < 64) binom_uploaded_for_device[dev] = true;
}

void build_spin_tables(SpinTables& t, int n, int k, bool need_g1, cudaStream_t s) {
    upload_binom();
    const Binom& B = host_binom();
    t.n = n;
    t.k = k;
    t.nstr = (int)B.c[n][k];
    t.s1 = k * (n - k) + k;
    t.npair = n * (n + 1) / 2;
    t.npair_pad = (t.npair + 7) / 8 * 8;
    t.str.alloc(t.nstr);
    k_unrank<<<(t.nstr + 255) / 256, 256, 0, s>>>(t.str.p, t.nstr, n, k);
    FCIB_KCHECK();
    if (t.s1 > 0) {
        t.conn.alloc((size_t)t.nstr * t.s1);
        k_conn<<<(t.nstr + 127) / 128, 128, 0, s>>>(t.str.p, t.conn.p, t.nstr, n, t.s1);
        FCIB_KCHECK();
    }
    t.tgt.alloc((size_t)t.nstr * t.npair_pad);
    k_tgt<<<t.nstr, 128, 0, s>>>(t.str.p, t.tgt.p, t.nstr, n, t.npair_pad);
    FCIB_KCHECK();
    t.ng2 = t.g2 = 0;
    if (k >= 2) {
        t.ng2 = (int)B.c[n][k - 2];
        t.g2 = (int)B.c[n - k + 2][2];
        t.g2row.alloc((size_t)t.ng2 * t.g2);
        t.g2lab.alloc((size_t)t.ng2 * t.g2);
        k_groups<<<(t.ng2 + 127) / 128, 128, 0, s>>>(t.g2row.p, t.g2lab.p, t.ng2, t.g2, n, k, 2);
        FCIB_KCHECK();
    }
    t.ng1 = t.g1 = 0;
    if (need_g1 && k >= 1) {
        t.ng1 = (int)B.c[n][k - 1];
        t.g1 = n - k + 1;
        t.g1row.alloc((size_t)t.ng1 * t.g1);
        t.g1lab.alloc((size_t)t.ng1 * t.g1);
        k_groups<<<(t.ng1 + 127) / 128, 128, 0, s>>>(t.g1row.p, t.g1lab.p, t.ng1, t.g1, n, k, 1);
        FCIB_KCHECK();
    }
}

// ------------------------------------------------------------------------------------------
// Substitution lists in the reference's own format and order, one thread per entry.
// Entry e of a list corresponds to the e-th occupation pattern b of the free orbitals in
// next_permutation order, i.e. b = unrank(e) over the free positions.
// ------------------------------------------------------------------------------------------

// VO (forte/fci/fci_string_vo_list.cc:90-140): J = sign a+_p a_q I
__global__ void k_vo_list(int n, int k, int p, int q, int len, int8_t* sign, uint32_t* I, uint32_t* J) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= len) return;
    int nf = n - 1 - (p == q ? 0 : 1);
    uint32_t b = d_unrank(e, nf, k - 1);
    int lo = p < q ? p : q, hi = p < q ? q : p;
    uint32_t s = 0;
    int kk = 0;
    int neg = 0;
    for (int i = 0; i < n; i++) {
        if (i == lo || i == hi) continue;
        uint32_t bit = b >> kk & 1u;
        kk++;
        if (bit) {
            s |= 1u << i;
            if (i > lo && i < hi) neg ^= 1;
        }
    }
    uint32_t Is = (s & ~(1u << p)) | (1u << q);
    uint32_t Js = (s & ~(1u << q)) | (1u << p);
    sign[e] = neg ? -1 : 1;
    I[e] = d_rank(Is, n);
    J[e] = d_rank(Js, n);
}

// OO (forte/fci/fci_string_oo_list.cc:69-115): a+_p a+_q a_q a_p, p > q, sign +1
__global__ void k_oo_list(int n, int k, int p, int q, int len, int8_t* sign, uint32_t* I, uint32_t* J) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= len) return;
    uint32_t b = d_unrank(e, n - 2, k - 2);
    uint32_t s = 0;
    int kk = 0;
    for (int i = 0; i < n; i++) {
        if (i == p || i == q) continue;
        if (b >> kk & 1u) s |= 1u << i;
        kk++;
    }
    s |= (1u << p) | (1u << q);
    uint32_t a = d_rank(s, n);
    sign[e] = 1;
    I[e] = a;
    J[e] = a;
}

// VVOO (forte/fci/fci_string_vvoo_list.cc:88-187): J = sign a+_p a+_q a_s a_r I.  Patterns
// for which p or q is already occupied after the annihilations are skipped, so entries are
// written compactly through an atomic counter and put back in pattern order by the host.
__global__ void k_vvoo_list(int n, int k, int p, int q, int r, int s, int npat, int* count,
                            int* pat, int8_t* sign, uint32_t* I, uint32_t* J) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= npat) return;
    int a0 = s, a1 = r, a2 = q, a3 = p;
    int a[4] = {a0, a1, a2, a3};
    // sort network identical to the reference's
#define CSW(x, y) if (a[x] > a[y]) { int t_ = a[x]; a[x] = a[y]; a[y] = t_; }
    CSW(1, 2);
    CSW(0, 1); CSW(1, 2); CSW(2, 3);
    CSW(0, 1); CSW(1, 2); CSW(2, 3);
#undef CSW
    bool overlap = (a[0] == a[1]) || (a[1] == a[2]) || (a[2] == a[3]);
    int nf = n - 4 + (overlap ? 1 : 0);
    uint32_t b = d_unrank(e, nf, k - 2);
    uint32_t Is = 0;
    Is |= (1u << s) | (1u << r);
    Is &= ~(1u << p);
    Is &= ~(1u << q);
    Is |= (1u << s) | (1u << r);
    int kk = 0;
    for (int i = 0; i < n; i++) {
        if (i == a[0] || i == a[1] || i == a[2] || i == a[3]) continue;
        if (b >> kk & 1u) Is |= 1u << i;
        else Is &= ~(1u << i);
        kk++;
    }
    // the reference sets I[p]=I[q]=0 then I[s]=I[r]=1 before filling the free positions
    Is &= ~(1u << p);
    Is &= ~(1u << q);
    Is |= (1u << s) | (1u << r);
    uint32_t Js = Is;
    int neg = 0;
    for (int i = s; i < r; i++)
        if (Js >> i & 1u) neg ^= 1;
    Js &= ~(1u << r);
    Js &= ~(1u << s);
    if (Js >> q & 1u) return;
    Js |= 1u << q;
    neg ^= __popc(Js & ((1u << q) - 1u)) & 1u;
    if (Js >> p & 1u) return;
    Js |= 1u << p;
    neg ^= __popc(Js & ((1u << p) - 1u)) & 1u;
    int slot = atomicAdd(count, 1);
    pat[slot] = e;
    sign[slot] = neg ? -1 : 1;
    I[slot] = d_rank(Is, n);
    J[slot] = d_rank(Js, n);
}

}  // namespace fcib

// ------------------------------------------------------------------------------------------
// list export (called from the C ABI)
// ------------------------------------------------------------------------------------------
namespace fcib {
void export_list(int n, int k, int kind, int p, int q, int r, int s, std::vector<int8_t>& sign,
                 std::vector<uint32_t>& I, std::vector<uint32_t>& J, cudaStream_t st) {
    upload_binom();
    const Binom& B = host_binom();
    sign.clear(); I.clear(); J.clear();
    auto run = [&](int len, auto launch) {
        if (len <= 0) return;
        DBuf<int8_t> ds; DBuf<uint32_t> dI, dJ;
        ds.alloc(len); dI.alloc(len); dJ.alloc(len);
        launch(ds.p, dI.p, dJ.p);
        FCIB_KCHECK();
        sign.resize(len); I.resize(len); J.resize(len);
        FCIB_CUDA(cudaMemcpyAsync(sign.data(), ds.p, len, cudaMemcpyDeviceToHost, st));
        FCIB_CUDA(cudaMemcpyAsync(I.data(), dI.p, 4 * len, cudaMemcpyDeviceToHost, st));
        FCIB_CUDA(cudaMemcpyAsync(J.data(), dJ.p, 4 * len, cudaMemcpyDeviceToHost, st));
        FCIB_CUDA(cudaStreamSynchronize(st));
    };
    if (kind == 0) {
        int nf = n - 1 - (p == q ? 0 : 1), kf = k - 1;
        if (kf < 0 || kf > nf) return;
        int len = (int)B.c[nf][kf];
        run(len, [&](int8_t* a, uint32_t* b, uint32_t* c) {
            k_vo_list<<<(len + 127) / 128, 128, 0, st>>>(n, k, p, q, len, a, b, c);
        });
    } else if (kind == 1) {
        // p is the pair index of (pp > qq) in make_pair_list order
        int pp = 1, t = p;
        while (t >= pp) { t -= pp; pp++; }
        int qq = t;
        if (k - 2 < 0) return;
        int len = (int)B.c[n - 2][k - 2];
        run(len, [&](int8_t* a, uint32_t* b, uint32_t* c) {
            k_oo_list<<<(len + 127) / 128, 128, 0, st>>>(n, k, pp, qq, len, a, b, c);
        });
    } else {
        int a[4] = {s, r, q, p};
        std::sort(a, a + 4);
        bool overlap = (a[0] == a[1]) || (a[1] == a[2]) || (a[2] == a[3]);
        int nf = n - 4 + (overlap ? 1 : 0), kf = k - 2;
        if (!(kf >= 0 && nf >= 0 && nf >= kf)) return;
        int npat = (int)B.c[nf][kf];
        DBuf<int> cnt, pat;
        cnt.alloc(1);
        pat.alloc(npat);
        FCIB_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int), st));
        DBuf<int8_t> ds; DBuf<uint32_t> dI, dJ;
        ds.alloc(npat); dI.alloc(npat); dJ.alloc(npat);
        k_vvoo_list<<<(npat + 127) / 128, 128, 0, st>>>(n, k, p, q, r, s, npat, cnt.p, pat.p, ds.p, dI.p, dJ.p);
        FCIB_KCHECK();
        int len = 0;
        FCIB_CUDA(cudaMemcpyAsync(&len, cnt.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        FCIB_CUDA(cudaStreamSynchronize(st));
        std::vector<int> hp(len);
        std::vector<int8_t> hs(len);
        std::vector<uint32_t> hI(len), hJ(len);
        if (len) {
            FCIB_CUDA(cudaMemcpy(hp.data(), pat.p, 4 * len, cudaMemcpyDeviceToHost));
            FCIB_CUDA(cudaMemcpy(hs.data(), ds.p, len, cudaMemcpyDeviceToHost));
            FCIB_CUDA(cudaMemcpy(hI.data(), dI.p, 4 * len, cudaMemcpyDeviceToHost));
            FCIB_CUDA(cudaMemcpy(hJ.data(), dJ.p, 4 * len, cudaMemcpyDeviceToHost));
        }
        std::vector<int> order(len);
        for (int i = 0; i < len; i++) order[i] = i;
        std::sort(order.begin(), order.end(), [&](int x, int y) { return hp[x] < hp[y]; });
        sign.resize(len); I.resize(len); J.resize(len);
        for (int i = 0; i < len; i++) {
            sign[i] = hs[order[i]];
            I[i] = hI[order[i]];
            J[i] = hJ[order[i]];
        }
    }
}
}  // namespace fcib
