/*
 * fcib_solver.hpp -- header-only C++ wrapper over the C ABI (fcib.h) with the calling pattern of
 * Forte's FCISolver (forte/fci/fci_solver.h:87-122, forte/base_classes/active_space_method.h:95-388):
 * set integrals, state and options, compute_energy, rdms over (left, right) root pairs, and
 * transition_rdms against a second solver.  Errors become std::runtime_error with the engine's
 * message, non-convergence with die_if_not_converged gives the reference's message
 * (fci_solver.cc:269-276).  A Forte-side ActiveSpaceMethod adapter only has to map ambit tensors and
 * option objects onto this class.  Plain C++17, no CUDA headers.
 */
#ifndef FCIB_SOLVER_HPP
#define FCIB_SOLVER_HPP

#include <cstddef>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "fcib.h"

namespace fcib_cpp {

/* One (left, right) root pair's reduced density matrices, dense row-major like ambit::Tensor:
 * spin-dependent g1a, g1b [n^2], g2aa, g2ab, g2bb [n^4], g3aaa, g3aab, g3abb, g3bbb [n^6];
 * spin-free g1 (in g1a), g2 (in g2aa), g3 (in g3aaa).  Empty vectors for levels not asked for. */
struct RdmSet {
    bool spin_free = false;
    int level = 0;
    std::vector<double> g1a, g1b, g2aa, g2ab, g2bb, g3aaa, g3aab, g3abb, g3bbb;
};

class Solver {
  public:
    explicit Solver(int device = 0) {
        check(fcib_create(&ctx_, device));
        fcib_default_options(&opt_);
    }
    ~Solver() {
        if (ctx_) fcib_destroy(ctx_);
    }
    Solver(const Solver&) = delete;
    Solver& operator=(const Solver&) = delete;

    /* Forte's ActiveSpaceIntegrals layouts: oei [n*n], tei_aa/bb = <pq||rs>, tei_ab = <pq|rs> [n^4];
     * scalar = nuclear repulsion + scalar + frozen-core energy; orbsym[n] (empty = C1). */
    void set_integrals(int n, int nirrep, const std::vector<int>& orbsym, double scalar,
                       const double* oei_a, const double* oei_b, const double* tei_aa, const double* tei_ab,
                       const double* tei_bb) {
        n_ = n;
        check(fcib_set_integrals(ctx_, n, nirrep, orbsym.empty() ? nullptr : orbsym.data(), scalar, oei_a, oei_b,
                                 tei_aa, tei_ab, tei_bb));
    }
    void set_state(int na, int nb, int irrep, int multiplicity, int nroot, int root = 0) {
        nroot_ = nroot;
        root_ = root;
        check(fcib_set_state(ctx_, na, nb, irrep, multiplicity, nroot, root));
    }
    /* GenCISolver's GAS space: space[p] = GAS space of active orbital p, electron bounds per space;
     * an empty space vector restores the full determinant space */
    void set_gas(const std::vector<int>& space, const std::vector<int>& gas_min, const std::vector<int>& gas_max) {
        int ngas = 0;
        for (int k : space) ngas = k + 1 > ngas ? k + 1 : ngas;
        if ((int)gas_min.size() < ngas || (int)gas_max.size() < ngas)
            throw std::runtime_error("GAS bounds are needed for every space");
        check(fcib_set_gas(ctx_, ngas, space.empty() ? nullptr : space.data(), gas_min.data(), gas_max.data()));
    }
    fcib_options& options() { return opt_; }
    void set_die_if_not_converged(bool v) { opt_.die_if_not_converged = v ? 1 : 0; }

    /* FCISolver::compute_energy: energy of the selected root; energies() and spin2() for all */
    double compute_energy() {
        check(fcib_set_options(ctx_, &opt_));
        energies_.assign(nroot_, 0.0);
        spin2_.assign(nroot_, 0.0);
        iterations_ = 0;
        const int rc = fcib_solve(ctx_, energies_.data(), spin2_.data(), &iterations_);
        if (rc == FCIB_ERR_NOT_CONVERGED)
            throw std::runtime_error(fcib_last_error());  // the reference's message (fci_solver.cc:269-276)
        check(rc);
        return energies_.at(root_);
    }
    const std::vector<double>& energies() const { return energies_; }
    const std::vector<double>& spin2() const { return spin2_; }
    int iterations() const { return iterations_; }
    int nroot() const { return nroot_; }

    /* determinant-space size in flat order (FCIVector, or GenCIVector with GAS spaces) */
    int64_t size() {
        int64_t nd = 0;
        check(fcib_size(ctx_, &nd));
        return nd;
    }

    /* eigenvector of a root in FCIVector flat order */
    std::vector<double> evec(int root) {
        int64_t nd = 0;
        check(fcib_size(ctx_, &nd));
        std::vector<double> v((size_t)nd);
        check(fcib_get_vector(ctx_, root, v.data()));
        return v;
    }

    /* FCISolver::rdms (fci_solver_rdms.cc:40-104); level 1..3, level <= 0 gives empty sets */
    std::vector<RdmSet> rdms(const std::vector<std::pair<size_t, size_t>>& roots, int level, bool spin_free) {
        if (level > 3) throw std::runtime_error("Invalid max_rdm_level, required max_rdm_level <= 3.");
        std::vector<RdmSet> out;
        for (const auto& pr : roots) {
            RdmSet r = alloc(level, spin_free);
            if (level >= 1) {
                check(fcib_rdms(ctx_, (int)pr.first, (int)pr.second, level, spin_free ? 1 : 0, r.g1a.data(),
                                spin_free ? nullptr : r.g1b.data(), level >= 2 ? r.g2aa.data() : nullptr,
                                (level >= 2 && !spin_free) ? r.g2ab.data() : nullptr,
                                (level >= 2 && !spin_free) ? r.g2bb.data() : nullptr));
            }
            if (level >= 3)
                check(fcib_rdms3(ctx_, (int)pr.first, (int)pr.second, spin_free ? 1 : 0, r.g3aaa.data(),
                                 spin_free ? nullptr : r.g3aab.data(), spin_free ? nullptr : r.g3abb.data(),
                                 spin_free ? nullptr : r.g3bbb.data()));
            out.push_back(std::move(r));
        }
        return out;
    }

    /* FCISolver::transition_rdms (fci_solver_transition_rdms.cc:37-109): <this root| ... |other root> */
    std::vector<RdmSet> transition_rdms(const std::vector<std::pair<size_t, size_t>>& roots, Solver& method2,
                                        int level, bool spin_free) {
        std::vector<RdmSet> out;
        for (const auto& pr : roots) {
            RdmSet r = alloc(level >= 1 ? 1 : 0, spin_free);
            if (level >= 1)
                check(fcib_transition_rdms(ctx_, (int)pr.first, method2.ctx_, (int)pr.second, level,
                                           spin_free ? 1 : 0, r.g1a.data(), spin_free ? nullptr : r.g1b.data()));
            out.push_back(std::move(r));
        }
        return out;
    }

    fcib_ctx* handle() { return ctx_; }

  private:
    static void check(int rc) {
        if (rc != FCIB_OK) throw std::runtime_error(fcib_last_error());
    }
    RdmSet alloc(int level, bool spin_free) const {
        RdmSet r;
        r.spin_free = spin_free;
        r.level = level;
        const size_t n1 = (size_t)n_ * n_, n2 = n1 * n1, n3 = n2 * n1;
        if (level >= 1) {
            r.g1a.assign(n1, 0.0);
            if (!spin_free) r.g1b.assign(n1, 0.0);
        }
        if (level >= 2) {
            r.g2aa.assign(n2, 0.0);
            if (!spin_free) {
                r.g2ab.assign(n2, 0.0);
                r.g2bb.assign(n2, 0.0);
            }
        }
        if (level >= 3) {
            r.g3aaa.assign(n3, 0.0);
            if (!spin_free) {
                r.g3aab.assign(n3, 0.0);
                r.g3abb.assign(n3, 0.0);
                r.g3bbb.assign(n3, 0.0);
            }
        }
        return r;
    }
    fcib_ctx* ctx_ = nullptr;
    fcib_options opt_{};
    int n_ = 0, nroot_ = 1, root_ = 0, iterations_ = 0;
    std::vector<double> energies_, spin2_;
};

}  // namespace fcib_cpp

#endif /* FCIB_SOLVER_HPP */
