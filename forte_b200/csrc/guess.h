// Host-side dense helpers of the solver (see guess.cpp).
#pragma once

#include <stdint.h>

#include <functional>
#include <utility>
#include <vector>

namespace fcib {

// symmetric eigensolver: ascending eigenvalues, eigenvectors in columns V[i*n+k]
void sym_eigen(int n, const double* A, double* evals, double* V);

struct Det {
    uint64_t a, b;
};

struct HostInts {
    int n = 0;
    const std::vector<double>*oa = nullptr, *ob = nullptr, *taa = nullptr, *tab = nullptr, *tbb = nullptr;
    double slater(uint64_t la, uint64_t lb, uint64_t ra, uint64_t rb) const;
};

double det_spin2(uint64_t Ia, uint64_t Ib, uint64_t Ja, uint64_t Jb, int nmo);

using SparseVec = std::vector<std::pair<int64_t, double>>;
struct GuessResult {
    std::vector<SparseVec> guesses;
    std::vector<SparseVec> bad_roots;
    bool perturb = false;  // guesses are not spin-selected: add a small random component
};

// lowest: (diagonal energy, determinant address) sorted ascending
GuessResult make_guess(const HostInts& ints, const std::vector<std::pair<double, int64_t>>& lowest,
                       const std::function<Det(int64_t)>& det_of,
                       const std::function<int64_t(const Det&)>& addr_of, int num_guess_states,
                       int multiplicity);

}  // namespace fcib
