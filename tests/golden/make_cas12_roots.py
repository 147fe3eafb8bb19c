"""Generates cas12_roots.json: the oracle's Davidson-Liu (the CPU restatement of Forte's
DavidsonLiuSolver and FCISolver guess) on the three-root CAS(12,12) workload, converged.

Workload: synthetic integrals n = 12, L = 36, seed 1 (forte_b200.integrals.synthetic), 6 alpha and
6 beta electrons, C1, 3 roots, no spin selection (multiplicity 0: the lowest roots of the Ms = 0
space), E_CONVERGENCE 1e-10, R_CONVERGENCE 1e-6, DL_SUBSPACE_PER_ROOT 8, DL_COLLAPSE_PER_ROOT 2.
With the default DL_MAXITER of 100 the solver stops unconverged (root 0 is still 9e-5 Eh above its
limit at iteration 100); the fixture uses DL_MAXITER 400 and records where it converged.  About
15 minutes on one core.

  python tests/golden/make_cas12_roots.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from forte_b200 import synthetic  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402


def main():
    cfg = {"n": 12, "L": 36, "seed": 1, "na": 6, "nb": 6, "nroot": 3}
    opts = {"E_CONVERGENCE": 1e-10, "R_CONVERGENCE": 1e-6, "DL_SUBSPACE_PER_ROOT": 8, "DL_COLLAPSE_PER_ROOT": 2,
            "DL_MAXITER": 400}
    o = Oracle(cfg["n"], cfg["na"], cfg["nb"])
    o.set_integrals(synthetic(cfg["n"], cfg["L"], cfg["seed"]))
    r = o.solve(nroot=cfg["nroot"], maxiter=opts["DL_MAXITER"], subspace_per_root=opts["DL_SUBSPACE_PER_ROOT"],
                collapse_per_root=opts["DL_COLLAPSE_PER_ROOT"], multiplicity=0, e_conv=opts["E_CONVERGENCE"],
                r_conv=opts["R_CONVERGENCE"])
    assert r["converged"]
    out = dict(cfg, options=opts, energies=[float(x) for x in r["energies"]], iterations=r["iterations"],
               converged=r["converged"], source="oracle Davidson-Liu (CPU restatement of the reference), FP64")
    with open(os.path.join(HERE, "cas12_roots.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
