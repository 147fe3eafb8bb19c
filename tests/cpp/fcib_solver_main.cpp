// C++ driver of the engine through include/fcib_solver.hpp, the way a Forte-side ActiveSpaceMethod
// adapter calls it: integrals and state in, compute_energy, spin-free and spin-dependent RDMs of the
// roots, transition 1-RDMs against a second solver whose state belongs to another irrep, and a
// GenCISolver-style solve on a GAS space (at most two electrons in the upper half of the orbitals).
//
//   fcib_solver_main <input.bin> <output.bin>
//
// input.bin (little endian): int32 n, nirrep, na, nb, multiplicity, nroot, irrep2, device;
//   int32 orbsym[n]; float64 scalar, oei[n*n], tei_aa[n^4], tei_ab[n^4] (oei_b = oei_a, tei_bb = tei_aa)
// output.bin: float64 energies[nroot], spin2[nroot], iterations, then for root 0 the spin-dependent
//   g1a, g1b [n^2], g2aa, g2ab, g2bb [n^4], the spin-free g1 [n^2] and g2 [n^4], then the second
//   solver's energy and the transition g1a, g1b [n^2] of <root 0, irrep| ... |root 0, irrep2>, the
//   refusal flag of a level-2 transition RDM, and the GAS solve's energy and determinant count.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <vector>

#include "fcib_solver.hpp"

template <typename T>
static void rd(std::ifstream& f, T* p, size_t count) {
    f.read(reinterpret_cast<char*>(p), sizeof(T) * count);
    if (!f) throw std::runtime_error("short input file");
}
template <typename T>
static void wr(std::ofstream& f, const std::vector<T>& v) {
    f.write(reinterpret_cast<const char*>(v.data()), sizeof(T) * v.size());
}

int main(int argc, char** argv) {
    if (argc != 3) {
        std::cerr << "usage: fcib_solver_main <input.bin> <output.bin>\n";
        return 2;
    }
    try {
        std::ifstream in(argv[1], std::ios::binary);
        int hdr[8];
        rd(in, hdr, 8);
        const int n = hdr[0], nirrep = hdr[1], na = hdr[2], nb = hdr[3], mult = hdr[4], nroot = hdr[5];
        const int irrep2 = hdr[6], device = hdr[7];
        std::vector<int> orbsym(n);
        rd(in, orbsym.data(), n);
        double scalar = 0.0;
        rd(in, &scalar, 1);
        const size_t n2 = (size_t)n * n, n4 = n2 * n2;
        std::vector<double> oei(n2), taa(n4), tab(n4);
        rd(in, oei.data(), n2);
        rd(in, taa.data(), n4);
        rd(in, tab.data(), n4);

        fcib_cpp::Solver s(device);
        s.set_integrals(n, nirrep, orbsym, scalar, oei.data(), oei.data(), taa.data(), tab.data(), taa.data());
        s.set_state(na, nb, /*irrep=*/0, mult, nroot);
        s.options().e_convergence = 1e-12;
        s.options().r_convergence = 1e-8;
        s.set_die_if_not_converged(true);
        s.compute_energy();
        auto sd = s.rdms({{0, 0}}, 2, false);
        auto sf = s.rdms({{0, 0}}, 2, true);

        fcib_cpp::Solver t(device);
        t.set_integrals(n, nirrep, orbsym, scalar, oei.data(), oei.data(), taa.data(), tab.data(), taa.data());
        t.set_state(na, nb, irrep2, mult, 1);
        t.options().e_convergence = 1e-12;
        t.options().r_convergence = 1e-8;
        t.compute_energy();
        auto tr = s.transition_rdms({{0, 0}}, t, 1, false);
        // the reference's limit: transition RDMs beyond the one-body level are not implemented
        bool level2_refused = false;
        try {
            s.transition_rdms({{0, 0}}, t, 2, false);
        } catch (const std::runtime_error&) {
            level2_refused = true;
        }

        // GenCISolver: at most two electrons in the upper half of the orbitals
        fcib_cpp::Solver g(device);
        g.set_integrals(n, nirrep, orbsym, scalar, oei.data(), oei.data(), taa.data(), tab.data(), taa.data());
        g.set_state(na, nb, /*irrep=*/0, mult, 1);
        std::vector<int> space(n);
        for (int p = 0; p < n; p++) space[p] = p < n / 2 ? 0 : 1;
        g.set_gas(space, {na + nb - 2, 0}, {2 * (n / 2), 2});
        g.options().e_convergence = 1e-12;
        g.options().r_convergence = 1e-8;
        g.compute_energy();

        std::ofstream out(argv[2], std::ios::binary);
        wr(out, s.energies());
        wr(out, s.spin2());
        wr(out, std::vector<double>{(double)s.iterations()});
        for (auto* v : {&sd[0].g1a, &sd[0].g1b, &sd[0].g2aa, &sd[0].g2ab, &sd[0].g2bb, &sf[0].g1a, &sf[0].g2aa})
            wr(out, *v);
        wr(out, t.energies());
        wr(out, tr[0].g1a);
        wr(out, tr[0].g1b);
        wr(out, std::vector<double>{level2_refused ? 1.0 : 0.0});
        wr(out, std::vector<double>{g.energies()[0], (double)g.size()});
        std::printf("fcib_solver_main: E = %.12f (%d iterations), second state E = %.12f\n", s.energies()[0],
                    s.iterations(), t.energies()[0]);
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "fcib_solver_main: " << e.what() << "\n";
        return 1;
    }
}
