"""FCISolver: the B200 engine behind Forte's ActiveSpaceMethod interface.

Mirrors forte::FCISolver (forte/fci/fci_solver.h:51-246) and the ActiveSpaceMethod contract
(forte/base_classes/active_space_method.h:95-388): same option names and defaults
(forte/options.yaml), ``compute_energy()`` returning the energy of ``root``, ``energies()``,
``spin2()``, ``evals()``, ``evecs()`` in FCIVector flat order, ``rdms(root_list,
max_rdm_level, rdm_type)`` and the set_* convergence knobs.  Errors surface as RuntimeError
subclasses like the reference's std::runtime_error.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import capi
from .integrals import ActiveSpaceIntegrals


@dataclass(frozen=True)
class StateInfo:
    """Active-space state: electron counts, 2S+1, 2*Ms, irrep and the GAS electron bounds per space
    (forte StateInfo, base_classes/state_info.h; gas_min/gas_max are read by GenCISolver only)."""
    na: int
    nb: int
    multiplicity: int = 1
    twice_ms: int = 0
    irrep: int = 0
    gas_min: tuple = ()
    gas_max: tuple = ()


#: Forte option names understood by FCISolver.set_options with their defaults
DEFAULT_OPTIONS = {
    "DL_MAXITER": 100,
    "E_CONVERGENCE": 1.0e-9,
    "R_CONVERGENCE": 1.0e-6,
    "DL_GUESS_PER_ROOT": 1,
    "DL_DETS_PER_GUESS": 50,
    "DL_COLLAPSE_PER_ROOT": 2,
    "DL_SUBSPACE_PER_ROOT": 10,
    "ROOT": 0,
    "PRINT": 0,
    # engine-specific knobs
    "FCI_PRECISION": "FP64",        # FP64 | MIXED | MIXED_TF32
    "FCI_PRECONDITIONER": "DIAG",   # DIAG | MLP
    "FCI_MIXED_SWITCH": 1.0e-4,
    "FCI_SAME_SPIN": "TC",          # TC | CUDA_CORES (mixed modes)
    "CI_SPIN_ADAPT": False,         # solve in the spin sector of the state's multiplicity
    "FCI_SYM_BLOCKED": True,        # with symmetry: vectors over the target irrep's blocks only
    "CI_SPIN_ADAPT_FULL_PRECONDITIONER": False,  # CSF diagonal with the spin-exchange elements
}


class RDMs:
    """Spin-dependent (g1a, g1b, g2aa, g2ab, g2bb) or spin-free (g1, g2) RDMs."""

    def __init__(self, spin_free, **t):
        self.spin_free = spin_free
        self.__dict__.update(t)


class FCISolver:
    def __init__(self, state: StateInfo, nroot: int, ints: ActiveSpaceIntegrals, options=None, device=0):
        L = capi.lib()
        h = C.c_void_p()
        capi.check(L.fcib_create(C.byref(h), device))
        self._h = h
        self.state = state
        self.nroot = nroot
        self.ints = ints
        self._opts = dict(DEFAULT_OPTIONS)
        self._die = False
        self._energies = None
        self._spin2 = None
        self._iterations = 0
        self.set_integrals(ints)
        self._root = 0
        if options:
            self.set_options(options)
        self._push_state()

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                capi.lib().fcib_destroy(self._h)
                self._h = None
        except Exception:
            pass

    # ---- configuration -------------------------------------------------------------------
    def set_integrals(self, ints: ActiveSpaceIntegrals):
        self.ints = ints
        n = ints.n
        self._keep = [np.ascontiguousarray(x, dtype=np.float64) for x in
                      (ints.oei_a, ints.oei_b, ints.tei_aa, ints.tei_ab, ints.tei_bb)]
        nirrep = max(ints.orbsym) + 1 if ints.orbsym else 1
        nirrep = 1 << (nirrep - 1).bit_length() if nirrep > 1 else 1
        osym = (C.c_int * n)(*ints.orbsym)
        capi.check(capi.lib().fcib_set_integrals(self._h, n, nirrep, osym, float(ints.scalar),
                                                 *[capi.dptr(x) for x in self._keep]))
        self._nirrep = nirrep

    def _push_state(self):
        s = self.state
        capi.check(capi.lib().fcib_set_state(self._h, s.na, s.nb, s.irrep, s.multiplicity, self.nroot,
                                             self._root))
        self._push_options()

    def _push_options(self):
        o = capi.default_options()
        d = self._opts
        o.maxiter = int(d["DL_MAXITER"])
        o.e_convergence = float(d["E_CONVERGENCE"])
        o.r_convergence = float(d["R_CONVERGENCE"])
        o.guess_per_root = int(d["DL_GUESS_PER_ROOT"])
        o.dets_per_guess = int(d["DL_DETS_PER_GUESS"])
        o.collapse_per_root = int(d["DL_COLLAPSE_PER_ROOT"])
        o.subspace_per_root = int(d["DL_SUBSPACE_PER_ROOT"])
        o.die_if_not_converged = 1 if self._die else 0
        o.print_ = int(d["PRINT"])
        o.precision = {"FP64": capi.PREC_FP64, "MIXED": capi.PREC_MIXED,
                       "MIXED_TF32": capi.PREC_MIXED_TF32}[str(d["FCI_PRECISION"]).upper()]
        o.preconditioner = {"DIAG": capi.PRECOND_DIAG, "MLP": capi.PRECOND_MLP}[str(d["FCI_PRECONDITIONER"]).upper()]
        o.mixed_switch = float(d["FCI_MIXED_SWITCH"])
        o.same_spin_kernel = {"TC": capi.SAME_TC, "CUDA_CORES": capi.SAME_CUDA_CORES}[str(d["FCI_SAME_SPIN"]).upper()]
        o.spin_adapt = 1 if d["CI_SPIN_ADAPT"] else 0
        o.sym_blocked = 1 if d["FCI_SYM_BLOCKED"] else 0
        o.spin_adapt_full_preconditioner = 1 if d["CI_SPIN_ADAPT_FULL_PRECONDITIONER"] else 0
        if o.preconditioner == capi.PRECOND_MLP and getattr(self, "_mlp", None) is None:
            from .learned_precond import load_weights
            self.set_mlp_weights(load_weights())
        capi.check(capi.lib().fcib_set_options(self._h, C.byref(o)))

    def set_options(self, options: dict):
        """FCISolver::set_options (forte/fci/fci_solver.cc:156-172)."""
        for k, v in options.items():
            K = k.upper()
            if K not in DEFAULT_OPTIONS:
                raise KeyError(f"unknown FCI option {k}")
            self._opts[K] = v
        self._root = int(self._opts["ROOT"])
        if self._root >= self.nroot:
            raise RuntimeError(f"ROOT ({self._root}) must be smaller than nroot ({self.nroot})")
        self._push_state()

    def set_e_convergence(self, v):
        self.set_options({"E_CONVERGENCE": v})

    def set_r_convergence(self, v):
        self.set_options({"R_CONVERGENCE": v})

    def set_maxiter(self, v):
        self.set_options({"DL_MAXITER": v})

    def set_root(self, v):
        self.set_options({"ROOT": v})

    def set_print(self, v):
        self.set_options({"PRINT": v})

    def set_mlp_weights(self, weights):
        """Weights of the learned preconditioner (FCIB_MLP_NWEIGHTS floats); None unloads.  With
        FCI_PRECONDITIONER = MLP and no weights set, the committed default weights are used."""
        if weights is None:
            self._mlp = None
            capi.check(capi.lib().fcib_set_mlp(self._h, None, 0))
            return
        self._mlp = np.ascontiguousarray(weights, dtype=np.float32)
        capi.check(capi.lib().fcib_set_mlp(self._h, capi.fptr(self._mlp), len(self._mlp)))

    def set_die_if_not_converged(self, v: bool):
        self._die = bool(v)
        self._push_options()

    # ---- results ---------------------------------------------------------------------------
    def size(self) -> int:
        n = C.c_int64()
        capi.check(capi.lib().fcib_size(self._h, C.byref(n)))
        return n.value

    def layout_size(self) -> int:
        """Length of device vectors in the engine's layout (the *_device entry points)."""
        n = C.c_int64()
        capi.check(capi.lib().fcib_layout_size(self._h, C.byref(n)))
        return n.value

    def csf_to_det(self, z: np.ndarray) -> np.ndarray:
        """SpinAdapter::csf_C_to_det_C: CSF coefficients -> determinant vector (flat order)."""
        z = np.ascontiguousarray(z, dtype=np.float64)
        out = np.zeros(self.size())
        capi.check(capi.lib().fcib_csf_to_det(self._h, capi.dptr(z), capi.dptr(out)))
        return out

    def det_to_csf(self, c: np.ndarray) -> np.ndarray:
        """SpinAdapter::det_C_to_csf_C: determinant vector (flat order) -> CSF coefficients."""
        c = np.ascontiguousarray(c, dtype=np.float64)
        out = np.zeros(self.ncsf())
        capi.check(capi.lib().fcib_det_to_csf(self._h, capi.dptr(c), capi.dptr(out)))
        return out

    def csf_hdiag(self, full=False) -> np.ndarray:
        """FCISolver::form_Hdiag_csf: the CSF diagonal, plain (full=False) or full preconditioner."""
        out = np.zeros(self.ncsf())
        capi.check(capi.lib().fcib_csf_hdiag(self._h, 1 if full else 0, capi.dptr(out)))
        return out

    def ncsf(self) -> int:
        """Size of the CSF basis of the state's multiplicity (the Davidson space with CI_SPIN_ADAPT)."""
        n = C.c_int64()
        capi.check(capi.lib().fcib_ncsf(self._h, C.byref(n)))
        return n.value

    def compute_energy(self) -> float:
        """FCISolver::compute_energy (forte/fci/fci_solver.cc:177-314)."""
        e = np.zeros(self.nroot)
        s2 = np.zeros(self.nroot)
        it = C.c_int()
        rc = capi.lib().fcib_solve(self._h, capi.dptr(e), capi.dptr(s2), C.byref(it))
        if rc == capi.FCIB_ERR_NOT_CONVERGED:
            # the reference's message (forte/fci/fci_solver.cc:269-276)
            raise RuntimeError("Davidson-Liu solver did not converge.\nPlease try to increase the number of "
                               "Davidson-Liu iterations (DL_MAXITER). You can also try to increase:\n - the "
                               "maximum size of the subspace (DL_SUBSPACE_PER_ROOT)"
                               "\n - the number of guess states (DL_GUESS_PER_ROOT)")
        capi.check(rc)
        self._energies, self._spin2, self._iterations = e, s2, it.value
        return float(e[self._root])

    def reset_guess(self):
        """Forget the previous solution: the next compute_energy starts from a fresh guess, as a
        newly constructed FCISolver would, instead of restarting from the previous eigenvectors."""
        capi.check(capi.lib().fcib_reset_guess(self._h))

    def energies(self):
        return list(self._energies)

    def evals(self):
        return np.array(self._energies)

    def spin2(self):
        return list(self._spin2)

    def iterations(self):
        return self._iterations

    def evecs(self) -> np.ndarray:
        N = self.size()
        out = np.zeros((self.nroot, N))
        for r in range(self.nroot):
            capi.check(capi.lib().fcib_get_vector(self._h, r, capi.dptr(out[r])))
        return out

    def sigma(self, b: np.ndarray) -> np.ndarray:
        b = np.ascontiguousarray(b, dtype=np.float64)
        s = np.zeros_like(b)
        capi.check(capi.lib().fcib_sigma(self._h, capi.dptr(b), capi.dptr(s)))
        return s

    def hdiag(self) -> np.ndarray:
        out = np.zeros(self.size())
        capi.check(capi.lib().fcib_hdiag(self._h, capi.dptr(out)))
        return out

    def compute_spin2(self, c) -> float:
        c = np.ascontiguousarray(c, dtype=np.float64)
        s = C.c_double()
        capi.check(capi.lib().fcib_spin2(self._h, capi.dptr(c), C.byref(s)))
        return s.value

    def profile(self) -> dict:
        p = capi.FcibProfile()
        capi.check(capi.lib().fcib_get_profile(self._h, C.byref(p)))
        return {k: getattr(p, k) for k, _ in capi.FcibProfile._fields_}

    def stream(self) -> int:
        s = C.c_void_p()
        capi.check(capi.lib().fcib_stream(self._h, C.byref(s)))
        return s.value or 0

    def timing(self):
        sm = C.c_double()
        ns = C.c_int()
        tt = C.c_double()
        capi.check(capi.lib().fcib_last_timing(self._h, C.byref(sm), C.byref(ns), C.byref(tt)))
        return {"sigma_ms": sm.value, "n_sigma": ns.value, "total_ms": tt.value}

    def rdms(self, root_list, max_rdm_level=2, rdm_type="spin_dependent"):
        """FCISolver::rdms (forte/fci/fci_solver_rdms.cc:40-104): one RDMs object per (left, right)
        root pair of the last solve; max_rdm_level <= 0 gives empty objects, 3 adds the 3-RDMs."""
        if max_rdm_level > 3:
            raise RuntimeError("RDMs of order higher than 3 are not available")
        out = []
        for (rl, rr) in root_list:
            if max(rl, rr) >= self.nroot:
                raise RuntimeError(f"Cannot compute RDMs <{rl}| ... |{rr}> (0-based) because nroot = {self.nroot}")
            out.append(self._rdm_call(lambda *a, rl=rl, rr=rr: capi.lib().fcib_rdms(self._h, rl, rr, *a),
                                      max_rdm_level, rdm_type,
                                      lambda *a, rl=rl, rr=rr: capi.lib().fcib_rdms3(self._h, rl, rr, *a)))
        return out

    def max_abs_elements(self, num_dets, root=0):
        """FCIVector::max_abs_elements (forte/fci/fci_vector_h_diag.cc:37-68) of a root: a list of
        (|C|, C, alpha irrep, alpha address, beta address) tuples, largest |C| first."""
        a = np.zeros(max(num_dets, 1))
        v = np.zeros(max(num_dets, 1))
        h = np.zeros(max(num_dets, 1), dtype=np.int32)
        ia = np.zeros(max(num_dets, 1), dtype=np.int64)
        ib = np.zeros(max(num_dets, 1), dtype=np.int64)
        cnt = C.c_int()
        capi.check(capi.lib().fcib_max_abs_elements(
            self._h, root, num_dets, capi.dptr(a), capi.dptr(v), h.ctypes.data_as(C.POINTER(C.c_int)),
            ia.ctypes.data_as(C.POINTER(C.c_int64)), ib.ctypes.data_as(C.POINTER(C.c_int64)), C.byref(cnt)))
        return [(float(a[i]), float(v[i]), int(h[i]), int(ia[i]), int(ib[i])) for i in range(cnt.value)]

    def transition_rdms(self, root_list, method2, max_rdm_level=1, rdm_type="spin_dependent"):
        """FCISolver::transition_rdms (forte/fci/fci_solver_transition_rdms.cc:37-109): one RDMs object
        per (left root of this solver, right root of method2) pair; method2 is another FCISolver on the
        same orbitals and electrons, possibly for a state of another irrep.  As in the reference only
        the one-body level exists (max_rdm_level >= 2 raises)."""
        sf = rdm_type in ("spin_free", 1)
        if max_rdm_level <= 0:
            return [RDMs(sf) for _ in root_list]
        n = self.ints.n
        out = []
        for (rl, rr) in root_list:
            g1a = np.zeros((n, n))
            g1b = np.zeros((n, n))
            capi.check(capi.lib().fcib_transition_rdms(self._h, rl, method2._h, rr, max_rdm_level, 1 if sf else 0,
                                                       capi.dptr(g1a), capi.dptr(g1b)))
            out.append(RDMs(True, g1=g1a) if sf else RDMs(False, g1a=g1a, g1b=g1b))
        return out

    def compute_rdms(self, left, right=None, max_rdm_level=2, rdm_type="spin_dependent"):
        """FCIVector::compute_rdms (forte/fci/fci_vector_rdm.cc:43-145) between two vectors in
        FCIVector flat order (right defaults to left)."""
        left = np.ascontiguousarray(left, dtype=np.float64)
        right = left if right is None else np.ascontiguousarray(right, dtype=np.float64)
        return self._rdm_call(lambda *a: capi.lib().fcib_compute_rdms(self._h, capi.dptr(left), capi.dptr(right), *a),
                              max_rdm_level, rdm_type,
                              lambda *a: capi.lib().fcib_compute_rdms3(self._h, capi.dptr(left), capi.dptr(right), *a))

    def _rdm_call(self, fn, level, rdm_type, fn3=None):
        """One- and two-body blocks through fn; with max_rdm_level 3 the three-body blocks through
        fn3 (RDMsSpinDependent g3aaa, g3aab, g3abb, g3bbb or RDMsSpinFree g3)."""
        n = self.ints.n
        sf = rdm_type in ("spin_free", 1)
        if level <= 0:
            return RDMs(sf)
        g1a = np.zeros((n, n))
        g1b = np.zeros((n, n))
        g2 = [np.zeros((n,) * 4) for _ in range(3)] if level > 1 else [None] * 3
        ptr = [capi.dptr(x) if x is not None else None for x in (g1a, g1b, *g2)]
        capi.check(fn(level, 1 if sf else 0, *ptr))
        g3 = {}
        if level >= 3:
            blocks = [np.zeros((n,) * 6) for _ in range(1 if sf else 4)]
            ptr3 = [capi.dptr(x) for x in blocks] + [None] * (4 - len(blocks))
            capi.check(fn3(1 if sf else 0, *ptr3))
            g3 = {"g3": blocks[0]} if sf else dict(zip(("g3aaa", "g3aab", "g3abb", "g3bbb"), blocks))
        if sf:
            return RDMs(True, g1=g1a, g2=g2[0], **g3)
        return RDMs(False, g1a=g1a, g1b=g1b, g2aa=g2[0], g2ab=g2[1], g2bb=g2[2], **g3)

    def determinants(self):
        """Alpha and beta strings (bit p = orbital p) of every flat position
        (FCIStringLists / GenCIStringLists::make_determinants)."""
        N = self.size()
        a = np.zeros(max(N, 1), dtype=np.uint32)
        b = np.zeros(max(N, 1), dtype=np.uint32)
        capi.check(capi.lib().fcib_determinants(self._h, a.ctypes.data_as(C.POINTER(C.c_uint32)),
                                                b.ctypes.data_as(C.POINTER(C.c_uint32))))
        return a[:N], b[:N]

    # ---- string tables (parity checks) ----------------------------------------------------
    def strings(self, spin):
        cnt = C.c_int64()
        capi.check(capi.lib().fcib_num_strings(self._h, spin, C.byref(cnt)))
        out = np.zeros(cnt.value, dtype=np.uint32)
        capi.check(capi.lib().fcib_strings(self._h, spin, out.ctypes.data_as(C.POINTER(C.c_uint32))))
        return out

    def string_list(self, spin, kind, p=0, q=0, r=0, s=0):
        ln = C.c_int64()
        L = capi.lib()
        capi.check(L.fcib_string_list(self._h, spin, kind, p, q, r, s, C.byref(ln), None, None, None))
        n = ln.value
        sg = np.zeros(max(n, 1), dtype=np.int8)
        I = np.zeros(max(n, 1), dtype=np.uint32)
        J = np.zeros(max(n, 1), dtype=np.uint32)
        capi.check(L.fcib_string_list(self._h, spin, kind, p, q, r, s, C.byref(ln),
                                      sg.ctypes.data_as(C.POINTER(C.c_int8)),
                                      I.ctypes.data_as(C.POINTER(C.c_uint32)),
                                      J.ctypes.data_as(C.POINTER(C.c_uint32))))
        return sg[:n], I[:n], J[:n]


class GenCISolver(FCISolver):
    """GenCISolver (forte/genci/genci_solver.h): the FCISolver interface over a generalized active
    space -- the determinants whose number of electrons in each orbital space k lies in
    [state.gas_min[k], state.gas_max[k]].

    gas_spaces: the active orbitals of GAS1, GAS2, ... (what MOSpaceInfo.pos_in_space("GASn",
    "ACTIVE") returns); every active orbital belongs to one space, and empty spaces may only trail.
    Missing bounds default to 0 and 2 * size, as make_state_weights_map sets them
    (base_classes/active_space_solver.cc:706-740).  Vectors are in GenCIVector flat order.
    """

    def __init__(self, state: StateInfo, nroot: int, ints: ActiveSpaceIntegrals, gas_spaces, options=None,
                 device=0):
        super().__init__(state, nroot, ints, options, device)
        self.set_gas(gas_spaces, state.gas_min, state.gas_max)

    def set_gas(self, gas_spaces, gas_min=(), gas_max=()):
        """Set the GAS spaces and bounds; no spaces restores the full determinant space."""
        n = self.ints.n
        spaces, owner, mn, mx = gas_layout(gas_spaces, n, gas_min, gas_max)
        ng = len(spaces)
        self.gas_spaces, self.gas_min, self.gas_max = spaces, mn, mx
        capi.check(capi.lib().fcib_set_gas(self._h, ng, (C.c_int * max(n, 1))(*owner),
                                           (C.c_int * max(ng, 1))(*mn), (C.c_int * max(ng, 1))(*mx)))


def gas_layout(gas_spaces, n, gas_min=(), gas_max=()):
    """The GAS spaces as the engine takes them: (spaces without trailing empty ones, the space of
    each of the n orbitals, lower and upper electron bounds per space).  Missing bounds default to
    0 and 2 * size (make_state_weights_map, base_classes/active_space_solver.cc:706-740).  Raises
    ValueError for more than six spaces, an empty space before a non-empty one, an orbital outside
    0..n-1 or in two spaces, or (with any space given) an orbital in none."""
    spaces = [sorted(int(p) for p in sp) for sp in gas_spaces]
    while spaces and not spaces[-1]:
        spaces.pop()
    if len(spaces) > 6:
        raise ValueError("at most six GAS spaces")
    if any(not sp for sp in spaces):
        raise ValueError("an empty GAS space is followed by a non-empty one")
    owner = [-1] * n
    for k, sp in enumerate(spaces):
        for p in sp:
            if not 0 <= p < n or owner[p] >= 0:
                raise ValueError(f"orbital {p} is outside the active space or in two GAS spaces")
            owner[p] = k
    if spaces and n and min(owner) < 0:
        raise ValueError("every active orbital must belong to a GAS space")
    mn = [int(gas_min[k]) if k < len(gas_min) else 0 for k in range(len(spaces))]
    mx = [int(gas_max[k]) if k < len(gas_max) else 2 * len(sp) for k, sp in enumerate(spaces)]
    return spaces, owner, mn, mx


def make_active_space_method(method: str, state: StateInfo, nroot: int, ints: ActiveSpaceIntegrals,
                             options=None, device=0, gas_spaces=None):
    """make_active_space_method (forte/base_classes/active_space_method.cc:126-184): "FCI", or
    "GENCI" with the GAS orbital spaces."""
    m = method.upper()
    if m == "FCI":
        return FCISolver(state, nroot, ints, options, device)
    if m == "GENCI":
        if gas_spaces is None:
            raise ValueError("GENCI needs the GAS orbital spaces (gas_spaces)")
        return GenCISolver(state, nroot, ints, gas_spaces, options, device)
    raise ValueError(f"active space method {method} is not provided by the B200 engine")
