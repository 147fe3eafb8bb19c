// Host-side pieces of the solver that work on small dense problems: the symmetric
// eigensolver used for the Davidson subspace and the initial guess, Slater rules over
// determinants, and the spin-projected initial guess.
//
// Initial guess (forte/fci/fci_solver_initial_guess.cc:44-103 and
// forte/sparse_ci/sparse_initial_guess.cc:72-264): take the determinants with the lowest
// diagonal energies, complete them to closed spin sets, diagonalize S^2 in that space,
// diagonalize H inside each S^2 eigenspace of integer multiplicity, keep the lowest states
// of the requested multiplicity as guesses and return lower states of other
// multiplicities as vectors to project out.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <stdexcept>

#include "guess.h"

namespace fcib {

// Symmetric eigensolver: Householder reduction to tridiagonal form followed by the implicit
// QL algorithm with Wilkinson-type shifts (the classical tred2/tql2 scheme, O(n^3)).  Eigenvalues
// ascending, eigenvectors in the columns of V; each eigenvector's largest component positive.
void sym_eigen(int n, const double* Ain, double* evals, double* V) {
    if (n <= 0) return;
    std::vector<double> a(Ain, Ain + (size_t)n * n);  // row-major, becomes the transform
    std::vector<double> d(n), e(n);
    auto A = [&](int i, int j) -> double& { return a[(size_t)i * n + j]; };
    // --- tridiagonalisation (Householder), accumulating the orthogonal transform in a ---
    for (int i = n - 1; i > 0; i--) {
        int l = i - 1;
        double h = 0.0, scale = 0.0;
        if (l > 0) {
            for (int k = 0; k <= l; k++) scale += std::fabs(A(i, k));
            if (scale == 0.0) {
                e[i] = A(i, l);
            } else {
                for (int k = 0; k <= l; k++) {
                    A(i, k) /= scale;
                    h += A(i, k) * A(i, k);
                }
                double f = A(i, l);
                double g = (f >= 0.0) ? -std::sqrt(h) : std::sqrt(h);
                e[i] = scale * g;
                h -= f * g;
                A(i, l) = f - g;
                f = 0.0;
                for (int j = 0; j <= l; j++) {
                    A(j, i) = A(i, j) / h;
                    g = 0.0;
                    for (int k = 0; k <= j; k++) g += A(j, k) * A(i, k);
                    for (int k = j + 1; k <= l; k++) g += A(k, j) * A(i, k);
                    e[j] = g / h;
                    f += e[j] * A(i, j);
                }
                double hh = f / (h + h);
                for (int j = 0; j <= l; j++) {
                    f = A(i, j);
                    e[j] = g = e[j] - hh * f;
                    for (int k = 0; k <= j; k++) A(j, k) -= (f * e[k] + g * A(i, k));
                }
            }
        } else {
            e[i] = A(i, l);
        }
        d[i] = h;
    }
    d[0] = 0.0;
    e[0] = 0.0;
    for (int i = 0; i < n; i++) {
        int l = i - 1;
        if (d[i] != 0.0) {
            for (int j = 0; j <= l; j++) {
                double g = 0.0;
                for (int k = 0; k <= l; k++) g += A(i, k) * A(k, j);
                for (int k = 0; k <= l; k++) A(k, j) -= g * A(k, i);
            }
        }
        d[i] = A(i, i);
        A(i, i) = 1.0;
        for (int j = 0; j <= l; j++) A(j, i) = A(i, j) = 0.0;
    }
    // --- implicit QL on the tridiagonal matrix (d, e), rotating the columns of a ---
    for (int i = 1; i < n; i++) e[i - 1] = e[i];
    e[n - 1] = 0.0;
    for (int l = 0; l < n; l++) {
        int iter = 0, m;
        do {
            for (m = l; m < n - 1; m++) {
                double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
                if (std::fabs(e[m]) <= 1e-15 * dd) break;
            }
            if (m != l) {
                if (iter++ == 200) break;
                double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
                double r = std::hypot(g, 1.0);
                g = d[m] - d[l] + e[l] / (g + (g >= 0.0 ? std::fabs(r) : -std::fabs(r)));
                double s = 1.0, c = 1.0, p = 0.0;
                int i;
                for (i = m - 1; i >= l; i--) {
                    double f = s * e[i], b = c * e[i];
                    e[i + 1] = (r = std::hypot(f, g));
                    if (r == 0.0) {
                        d[i + 1] -= p;
                        e[m] = 0.0;
                        break;
                    }
                    s = f / r;
                    c = g / r;
                    g = d[i + 1] - p;
                    r = (d[i] - g) * s + 2.0 * c * b;
                    d[i + 1] = g + (p = s * r);
                    g = c * r - b;
                    for (int k = 0; k < n; k++) {
                        f = A(k, i + 1);
                        A(k, i + 1) = s * A(k, i) + c * f;
                        A(k, i) = c * A(k, i) - s * f;
                    }
                }
                if (r == 0.0 && i >= l) continue;
                d[l] -= p;
                e[l] = g;
                e[m] = 0.0;
            }
        } while (m != l);
    }
    // sort ascending, copy out, normalise the sign convention
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return d[x] < d[y]; });
    for (int j = 0; j < n; j++) {
        evals[j] = d[order[j]];
        for (int i = 0; i < n; i++) V[(size_t)i * n + j] = A(i, order[j]);
    }
    for (int j = 0; j < n; j++) {
        int im = 0;
        for (int i = 1; i < n; i++)
            if (std::fabs(V[(size_t)i * n + j]) > std::fabs(V[(size_t)im * n + j]) + 1e-14) im = i;
        if (V[(size_t)im * n + j] < 0)
            for (int i = 0; i < n; i++) V[(size_t)i * n + j] = -V[(size_t)i * n + j];
    }
}

static inline int popc(uint64_t x) { return __builtin_popcountll(x); }
static inline double below(uint64_t s, int n) { return (popc(s & ((1ull << n) - 1ull)) & 1) ? -1.0 : 1.0; }
static inline double between(uint64_t s, int m, int n) {
    if (m > n) std::swap(m, n);
    if (n - m < 2) return 1.0;
    uint64_t mask = ((1ull << n) - 1ull) & ~((1ull << (m + 1)) - 1ull);
    return (popc(s & mask) & 1) ? -1.0 : 1.0;
}

// DeterminantImpl::slater_sign_aaaa (forte/sparse_ci/determinant.hpp:391-406)
static double sign_aaaa(uint64_t s, int i, int j, int a, int b) {
    if (((i < a) && (j < a) && (i < b) && (j < b)) || !((i < a) || (j < a) || (i < b) || (j < b))) {
        double v = between(s, i, j) * between(s, a, b);
        return ((i < j) ^ (a < b)) ? -v : v;
    }
    if ((i < j) ^ (a < b)) return -1.0 * between(s, i, b) * between(s, j, a);
    return between(s, i, a) * between(s, j, b);
}

double HostInts::slater(uint64_t la, uint64_t lb, uint64_t ra, uint64_t rb) const {
    // ActiveSpaceIntegrals::slater_rules (forte/integrals/active_space_integrals.cc:247-411)
    const size_t n2 = (size_t)n * n, n3 = n2 * n;
    auto T = [&](const std::vector<double>& t, int p, int q, int r, int s) {
        return t[p * n3 + q * n2 + r * n + s];
    };
    if (popc(la) != popc(ra) || popc(lb) != popc(rb)) return 0.0;
    int nad = popc(la ^ ra), nbd = popc(lb ^ rb);
    if (nad + nbd > 4) return 0.0;
    nad /= 2;
    nbd /= 2;
    double me = 0.0;
    if (nad == 0 && nbd == 0) {
        for (int p = 0; p < n; p++) {
            int ap = la >> p & 1, bp = lb >> p & 1;
            if (ap) me += (*oa)[p * n + p];
            if (bp) me += (*ob)[p * n + p];
            for (int q = 0; q < n; q++) {
                int aq = la >> q & 1, bq = lb >> q & 1;
                if (ap && aq) me += 0.5 * T(*taa, p, q, p, q);
                if (bp && bq) me += 0.5 * T(*tbb, p, q, p, q);
                if (ap && bq) me += T(*tab, p, q, p, q);
            }
        }
    } else if (nad == 1 && nbd == 0) {
        int i = 0, j = 0;
        for (int p = 0; p < n; p++) {
            if (((la ^ ra) >> p & 1) && (la >> p & 1)) i = p;
            if (((la ^ ra) >> p & 1) && (ra >> p & 1)) j = p;
        }
        double sg = between(la, i, j);
        me = sg * (*oa)[i * n + j];
        for (int p = 0; p < n; p++) {
            if ((la >> p & 1) && (ra >> p & 1)) me += sg * T(*taa, i, p, j, p);
            if ((lb >> p & 1) && (rb >> p & 1)) me += sg * T(*tab, i, p, j, p);
        }
    } else if (nad == 0 && nbd == 1) {
        int i = 0, j = 0;
        for (int p = 0; p < n; p++) {
            if (((lb ^ rb) >> p & 1) && (lb >> p & 1)) i = p;
            if (((lb ^ rb) >> p & 1) && (rb >> p & 1)) j = p;
        }
        double sg = between(lb, i, j);
        me = sg * (*ob)[i * n + j];
        for (int p = 0; p < n; p++) {
            if ((la >> p & 1) && (ra >> p & 1)) me += sg * T(*tab, p, i, p, j);
            if ((lb >> p & 1) && (rb >> p & 1)) me += sg * T(*tbb, i, p, j, p);
        }
    } else if (nad == 2 && nbd == 0) {
        int i = -1, j = 0, k = -1, l = 0;
        for (int p = 0; p < n; p++) {
            if (((la ^ ra) >> p & 1) && (la >> p & 1)) { if (i == -1) i = p; else j = p; }
            if (((la ^ ra) >> p & 1) && (ra >> p & 1)) { if (k == -1) k = p; else l = p; }
        }
        me = sign_aaaa(la, i, j, k, l) * T(*taa, i, j, k, l);
    } else if (nad == 0 && nbd == 2) {
        int i = -1, j = -1, k = -1, l = -1;
        for (int p = 0; p < n; p++) {
            if (((lb ^ rb) >> p & 1) && (lb >> p & 1)) { if (i == -1) i = p; else j = p; }
            if (((lb ^ rb) >> p & 1) && (rb >> p & 1)) { if (k == -1) k = p; else l = p; }
        }
        me = sign_aaaa(lb, i, j, k, l) * T(*tbb, i, j, k, l);
    } else if (nad == 1 && nbd == 1) {
        int i = -1, j = -1, k = -1, l = -1;
        for (int p = 0; p < n; p++) {
            if (((la ^ ra) >> p & 1) && (la >> p & 1)) i = p;
            if (((lb ^ rb) >> p & 1) && (lb >> p & 1)) j = p;
            if (((la ^ ra) >> p & 1) && (ra >> p & 1)) k = p;
            if (((lb ^ rb) >> p & 1) && (rb >> p & 1)) l = p;
        }
        me = between(la, i, k) * between(lb, j, l) * T(*tab, i, j, k, l);
    }
    return me;
}

// spin2(lhs, rhs) (forte/sparse_ci/determinant.hpp:910-958)
double det_spin2(uint64_t Ia, uint64_t Ib, uint64_t Ja, uint64_t Jb, int nmo) {
    if (popc(Ia) != popc(Ja) || popc(Ib) != popc(Jb)) return 0.0;
    int nad = popc(Ia ^ Ja) / 2, nbd = popc(Ib ^ Jb) / 2;
    int na = popc(Ia), nb = popc(Ib), npair = popc(Ia & Ib);
    double Ms = 0.5 * (double)(na - nb);
    double me = 0.0;
    if (nad == 0 && nbd == 0) me += Ms * (Ms + 1.0) + (double)nb - (double)npair;
    if (nad == 1 && nbd == 1) {
        int i = -1, j = -1;
        for (int p = 0; p < nmo; p++) {
            if ((Ja >> p & 1) && (Ib >> p & 1) && !(Jb >> p & 1) && !(Ia >> p & 1)) i = p;
            if ((Jb >> p & 1) && (Ia >> p & 1) && !(Ja >> p & 1) && !(Ib >> p & 1)) j = p;
        }
        if (i != j && i >= 0 && j >= 0) {
            double sg = below(Ja, i) * ((popc(Ja) & 1) ? -1.0 : 1.0) * below(Jb, j) * below(Ia, j) *
                        ((popc(Ia) & 1) ? -1.0 : 1.0) * below(Ib, i);
            me -= sg;
        }
    }
    return me;
}

static bool next_perm01(std::vector<int8_t>& a) {
    int n = (int)a.size();
    if (n < 2) return false;
    int i = n - 2;
    while (i >= 0 && !(a[i] < a[i + 1])) i--;
    if (i < 0) return false;
    int j = n - 1;
    while (!(a[i] < a[j])) j--;
    std::swap(a[i], a[j]);
    std::reverse(a.begin() + i + 1, a.end());
    return true;
}

// enforce_spin_completeness (forte/sparse_ci/determinant_functions.cc:133-190)
static void spin_complete(std::vector<Det>& dets, int nmo) {
    size_t n0 = dets.size();
    for (size_t I = 0; I < n0; I++) {
        uint64_t a = dets[I].a, b = dets[I].b;
        uint64_t closed = a & b, oa = a & ~b, ob = b & ~a;
        int nao = popc(oa), nbo = popc(ob);
        if (nao + nbo == 0) continue;
        std::vector<int> open;
        for (int i = 0; i < nmo; i++)
            if (((oa | ob) >> i) & 1) open.push_back(i);
        std::vector<int8_t> bits(open.size());
        for (size_t i = 0; i < open.size(); i++) bits[i] = ((int)i >= nbo) ? 1 : 0;
        do {
            uint64_t na_ = closed, nb_ = closed;
            for (size_t o = 0; o < open.size(); o++) {
                if (bits[o]) na_ |= 1ull << open[o];
                else nb_ |= 1ull << open[o];
            }
            bool found = false;
            for (const auto& d : dets)
                if (d.a == na_ && d.b == nb_) { found = true; break; }
            if (!found) dets.push_back({na_, nb_});
        } while (next_perm01(bits));
    }
}

static bool near_int(double v, double t) { return std::fabs(v - std::round(v)) <= t; }

GuessResult make_guess(const HostInts& ints, const std::vector<std::pair<double, int64_t>>& lowest,
                       const std::function<Det(int64_t)>& det_of, const std::function<int64_t(const Det&)>& addr_of,
                       int num_guess_states, int multiplicity) {
    std::vector<Det> dets;
    for (auto& eI : lowest) dets.push_back(det_of(eI.second));
    spin_complete(dets, ints.n);
    const int nd = (int)dets.size();
    std::vector<int64_t> pos(nd);
    for (int i = 0; i < nd; i++) pos[i] = addr_of(dets[i]);
    std::vector<double> S2((size_t)nd * nd), S2v((size_t)nd * nd), S2e(nd);
    for (int i = 0; i < nd; i++)
        for (int j = i; j < nd; j++) S2[i * nd + j] = S2[j * nd + i] = det_spin2(dets[i].a, dets[i].b, dets[j].a, dets[j].b, ints.n);
    sym_eigen(nd, S2.data(), S2e.data(), S2v.data());
    std::vector<double> H((size_t)nd * nd), T1((size_t)nd * nd, 0.0), HS((size_t)nd * nd, 0.0);
    for (int i = 0; i < nd; i++)
        for (int j = i; j < nd; j++) H[i * nd + j] = H[j * nd + i] = ints.slater(dets[i].a, dets[i].b, dets[j].a, dets[j].b);
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
    std::vector<double> mult(nd);
    for (int i = 0; i < nd; i++) mult[i] = std::sqrt(1.0 + 4.0 * S2e[i]);
    // find_integer_groups (forte/helpers/helpers.cc:237-263)
    struct Group { int m, start, end; };
    std::vector<Group> groups;
    {
        int it = 0;
        const double tol = 1.0e-6;
        while (it < nd) {
            while (it < nd && !near_int(mult[it], tol)) it++;
            if (it < nd) {
                int start = it, end = -1;
                for (int k = it; k + 1 < nd; k++)
                    if (near_int(mult[k], tol) && std::fabs(mult[k] - mult[k + 1]) > 2 * tol) { end = k; break; }
                if (end < 0) end = nd - 1;
                groups.push_back({(int)std::llround(mult[start]), start, end + 1});
                it = end + 1;
            }
        }
    }
    struct Info { std::vector<double> e; std::vector<double> C; int bs; };
    std::map<int, Info> info;
    for (auto& g : groups) {
        int bs = g.end - g.start;
        std::vector<double> Hb((size_t)bs * bs), ev(bs), evv((size_t)bs * bs);
        for (int i = 0; i < bs; i++)
            for (int j = 0; j < bs; j++) Hb[i * bs + j] = HS[(g.start + i) * nd + g.start + j];
        sym_eigen(bs, Hb.data(), ev.data(), evv.data());
        Info f;
        f.e = ev;
        f.bs = bs;
        f.C.assign((size_t)nd * bs, 0.0);
        for (int i = 0; i < nd; i++)
            for (int r = 0; r < bs; r++) {
                double s = 0.0;
                for (int k = 0; k < bs; k++) s += S2v[i * nd + g.start + k] * evv[k * bs + r];
                f.C[i * bs + r] = s;
            }
        info[g.m] = f;  // a later group with the same multiplicity replaces an earlier one
    }
    if (multiplicity == 0) {
        // no spin selection: lowest states of the guess Hamiltonian of any multiplicity
        std::vector<double> ev(nd), evv((size_t)nd * nd);
        sym_eigen(nd, H.data(), ev.data(), evv.data());
        if (nd < num_guess_states) throw std::runtime_error("guess space smaller than the number of guess states");
        GuessResult res;
        for (int r = 0; r < num_guess_states; r++) {
            SparseVec v;
            for (int i = 0; i < nd; i++) v.push_back({pos[i], evv[i * nd + r]});
            res.guesses.push_back(v);
        }
        res.perturb = true;  // the solver adds a small seeded random component (all spin sectors)
        return res;
    }
    auto it = info.find(multiplicity);
    if (it == info.end()) throw std::runtime_error("No guess with the requested multiplicity was found.");
    const Info& tg = it->second;
    if ((int)tg.e.size() < num_guess_states)
        throw std::runtime_error("Found " + std::to_string(tg.e.size()) + " guess(es) with the requested multiplicity but " +
                                 std::to_string(num_guess_states) + " were requested. Increase the value of DL_DETS_PER_GUESS");
    GuessResult res;
    double gmax = -1.7976931348623157e308;
    for (int r = 0; r < num_guess_states; r++) {
        SparseVec v;
        for (int i = 0; i < nd; i++) v.push_back({pos[i], tg.C[i * tg.bs + r]});
        res.guesses.push_back(v);
        gmax = std::max(gmax, tg.e[r]);
    }
    for (auto& kv : info) {
        if (kv.first == multiplicity) continue;
        const Info& f = kv.second;
        for (int r = 0; r < f.bs; r++)
            if (f.e[r] < gmax) {
                SparseVec v;
                for (int i = 0; i < nd; i++) v.push_back({pos[i], f.C[i * f.bs + r]});
                res.bad_roots.push_back(v);
            }
    }
    return res;
}

}  // namespace fcib
