#!/usr/bin/env python
"""Benchmark of the B200 FCI engine on its headline workload.

Metric: Davidson time to |dE| < 1e-8 Eh at CAS(16,16) (165,636,900 determinants, Ms = 0, one root,
subspace <= 8) with the mixed-precision sigma, against the plain FP64 GPU path.  Synthetic integrals:
h symmetric with diagonal ~ U[-2, 1] (sorted, +0.3 Eh on orbitals 8..15) and off-diagonal ~ N(0, 0.1),
(pq|rs) = sum_L B^L_pq B^L_rs with L = 48 symmetric B^L ~ N(0, 0.15), numpy PCG64(seed 1).

One step = one complete Davidson-Liu solve from the initial guess to convergence
(E_CONVERGENCE 1e-9, R_CONVERGENCE 1e-5 certified by the FP64 sigma), timed with CUDA events on the
engine's stream.  The CI vectors (1.3 GB each) are far larger than L2, so no flush is needed.
One FP64 solve of the same problem gives the reference energy (|dE| check) and the FP64 time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --mode sigma --n 15 [--precision MIXED|MIXED_TF32|FP64]   (sigma builds/s)
  python bench.py --mode gas                       (GAS spaces: kept-string blocks vs the masked C1 layout)

N > 1 runs independent replicas (the solve does not shard across GPUs), one per rank.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Davidson time-to-|ΔE|<1e-8 Eh @CAS(16,16): mixed+learned vs plain FP64, 1 B200"
N_ORB, L_AUX, GAP, SEED = 16, 48, 0.3, 1
SUBSPACE_PER_ROOT = 8
OPTS = {"DL_SUBSPACE_PER_ROOT": SUBSPACE_PER_ROOT, "DL_COLLAPSE_PER_ROOT": 2, "DL_MAXITER": 300,
        "E_CONVERGENCE": 1e-9, "R_CONVERGENCE": 1e-5}
# DRAM traffic of one tensor-core opposite-spin launch, from the ncu capture of CAS(15,15)
# (41,409,225 determinants, 63 connections per string: 5.153 GB read + 0.328 GB written), scaled
# by the gathered elements N_det * s1 to CAS(16,16) (165,636,900 determinants, 72 connections).
NCU_TRAFFIC_CAS15 = 5.481e9
NCU_UNITS_CAS15 = 41409225 * 63


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d["hbm_gbs"], d["bf16_tflops"], d.get("bf16_tflops_sustained", d["bf16_tflops"]), "measured"
    except Exception:
        return 6650.0, 1590.0, 1400.0, "fallback"


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        # the reference arm is CPU work: gloo, no device; the GPU arms: NCCL, one GPU per rank
        backend = "gloo" if args.impl == "reference" else "nccl"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allmax(world, v):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class Clocks:
    """nvidia-smi clock / throttle sampling during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.p = None
        self.path = os.path.join("/tmp", f"fcib_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(self.gpu)], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if not self.p:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in open(self.path):
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def solve_once(solver, torch, stream):
    """One Davidson solve from a fresh guess (no restart from the previous solve's vectors), timed
    with CUDA events on the engine stream; returns seconds."""
    solver.reset_guess()
    st = torch.cuda.Event(enable_timing=True)
    en = torch.cuda.Event(enable_timing=True)
    st.record(stream)
    solver.compute_energy()
    en.record(stream)
    en.synchronize()
    return st.elapsed_time(en) / 1e3


def cpu_sigma_sample(nsig=1, n=14):
    """Bounded CPU sample: the oracle (single-threaded restatement of Forte's FCI sigma) on
    CAS(n,n) with synthetic integrals L = 3n; returns seconds per sigma (string lists excluded)."""
    from oracle.oracle import Oracle
    from forte_b200 import synthetic
    ints = synthetic(n, 3 * n, SEED)
    o = Oracle(n, n // 2, n // 2)
    o.set_integrals(ints)
    c = np.random.default_rng(0).normal(size=o.ndet)
    c /= np.linalg.norm(c)
    t = time.perf_counter()
    for _ in range(nsig):
        o.sigma(c)
    return (time.perf_counter() - t) / nsig


def host_cpu():
    """Model name and logical core count of this host."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return model, os.cpu_count()


def cpu_extrapolation(sig14, iters):
    """CAS(16,16) solve time of the single-threaded CPU path: measured CAS(14,14) sigma x the
    reference sigma's FMA-count ratio CAS(16,16)/CAS(14,14) x the FP64 iteration count, plus 5% for
    the Davidson-Liu vector work."""
    ratio = ref_fma(16, 8) / ref_fma(14, 7)
    return iters * sig14 * ratio * 1.05, ratio


def ref_fma(n, k):
    """FMA count of one reference sigma (H1 + same-spin + opposite-spin list loops)."""
    from math import comb
    N = comb(n, k) ** 2
    s1 = k * (n - k) + k
    d2 = comb(k, 2) * comb(n - k + 2, 2)
    return N * (s1 * s1 + 2 * d2 + 2 * s1)


def run_reference(args, world, rank):
    """The reference arm: the CPU path (the oracle's restatement of Forte's single-threaded FCI sigma)
    on this host.  Each step is one measured CAS(14,14) sigma (11,778,624 determinants), extrapolated
    to a CAS(16,16) solve; at most two steps are run, since one step is about a minute of CPU work, and
    no warm-up (CPU code has nothing to warm)."""
    if rank != 0:
        return
    steps = max(1, min(args.steps, 2))
    times = [cpu_sigma_sample(1, 14) for _ in range(steps)]
    sig14 = statistics.mean(times)
    iters = args.ref_iterations
    value, ratio = cpu_extrapolation(sig14, iters)
    model, ncpu = host_cpu()
    line = {
        "metric": METRIC, "value": value, "unit": "s", "impl": "reference", "n_gpus": args.gpus, "steps": steps,
        "warmup": 0, "ms_per_step": sig14 * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "CAS(16,16) synthetic L=48 gap=0.3 Ms=0 1 root subspace 8", "n_det": 165636900},
        "cpu_baseline": {"value": value, "unit": "s", "cores": 1, "kind": "port",
                         "host_cpu": model, "host_cores": ncpu,
                         "sample": f"{steps} sigma build(s) of CAS(14,14) (11,778,624 dets) by the CPU oracle on 1 "
                                   f"core ({sig14:.2f} s each), extrapolated to a CAS(16,16) solve of {iters} "
                                   f"iterations by the reference FMA-count ratio {ratio:.2f} plus 5% Davidson "
                                   f"overhead; the reference FCI path is single-threaded"},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_sigma(args, world, rank, local):
    """Sigma builds per second at CAS(n,n) (Ms = 0, C1) on device vectors, through fcib_sigma_device."""
    import ctypes as C
    import torch
    from forte_b200 import FCISolver, StateInfo, build, capi, synthetic
    build.build()
    torch.cuda.set_device(local)
    n, k = args.n, args.n // 2
    ints = synthetic(n, 3 * n, SEED, gap=GAP)
    s = FCISolver(StateInfo(k, k, 0), 1, ints, {"FCI_SAME_SPIN": args.same_spin}, device=local)
    N = s.size()
    g = torch.Generator(device="cuda").manual_seed(0)
    b = torch.randn(N, dtype=torch.float64, device="cuda", generator=g)
    b /= b.norm()
    out = torch.empty_like(b)
    torch.cuda.synchronize()
    prec = {"FP64": capi.PREC_FP64, "MIXED": capi.PREC_MIXED, "MIXED_TF32": capi.PREC_MIXED_TF32}[args.precision]
    L = capi.lib()
    stream = torch.cuda.ExternalStream(s.stream())

    def one():
        capi.check(L.fcib_sigma_device(s._h, C.c_void_p(b.data_ptr()), C.c_void_p(out.data_ptr()), prec, None))

    for _ in range(args.warmup):
        one()
    barrier(world)
    torch.cuda.synchronize()
    p0 = s.profile()
    st = torch.cuda.Event(enable_timing=True)
    en = torch.cuda.Event(enable_timing=True)
    st.record(stream)
    for _ in range(args.steps):
        one()
    en.record(stream)
    en.synchronize()
    p1 = s.profile()
    sec = allmax(world, st.elapsed_time(en) / 1e3)
    launches = p1["launches"] - p0["launches"]
    npair = n * (n + 1) // 2
    s1 = k * (n - k) + k
    flops = 2.0 * N * s1 * npair
    hbm, bf16, bf16s, peak_kind = peaks()
    roofline = None
    if prec != capi.PREC_FP64:
        tc_ms = (p1["tc_kernel_ms"] - p0["tc_kernel_ms"]) / args.steps
        ach = flops / (tc_ms * 1e-3) / 1e12
        roofline = {"bound": "tensor", "kernel": "k_ab_tc<3xTF32>" if prec == capi.PREC_MIXED else "k_ab_tc<TF32>",
                    "achieved": ach, "peak": bf16, "unit": "TFLOP/s", "frac": ach / bf16,
                    "peak_kind": f"bf16 burst ({peak_kind}); the TF32 tensor rate is half of bf16",
                    "frac_vs_tf32": 2 * ach / bf16, "flops_per_launch": flops, "launch_ms": tc_ms,
                    "traffic": None}
    if rank == 0:
        print(json.dumps({
            "metric": f"sigma builds/s @CAS({n},{n})", "value": world * args.steps / sec, "unit": "sigma/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"FP64": "f64", "MIXED": "tf32x3/f32", "MIXED_TF32": "tf32/f32"}[args.precision],
            "data": "synthetic",
            "config": {"workload": f"sigma of a random unit vector, CAS({n},{n}) synthetic L={3 * n} Ms=0",
                       "n_det": N, "precision": args.precision, "same_spin": args.same_spin,
                       "l2": f"vectors of {N * 8 / 1e9:.2f} GB" + (" (> L2)" if N * 8 > 126e6 else " (fit in L2)")},
            "roofline": roofline, "gpu_launches": int(launches / args.steps),
            "sigma_profile_ms": {"opposite_spin": ((p1["ab_ms"] - p0["ab_ms"]) + (p1["ab64_ms"] - p0["ab64_ms"])) / args.steps,
                                 "same_spin": ((p1["same_ms"] - p0["same_ms"]) + (p1["same64_ms"] - p0["same64_ms"])) / args.steps},
        }), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_sym(args, world, rank, local):
    """Point-group symmetry: sigma time and time to solution of the irrep-blocked layout (vectors over the
    target irrep's determinants) against the masked C1 layout, for a D2h CAS(n,n) (two orbitals per
    irrep, totally symmetric singlet, Ms = 0)."""
    import ctypes as C
    import torch
    from forte_b200 import FCISolver, StateInfo, build, capi, synthetic
    build.build()
    torch.cuda.set_device(local)
    n, k = args.n, args.n // 2
    osym = [(i // 2) % 8 for i in range(n)]
    ints = synthetic(n, 3 * n, SEED, gap=GAP, orbsym=osym)
    L = capi.lib()
    out = {"sigma_ms": {}, "n_vec": {}, "solve": {}}
    for blocked in (True, False):
        lay = "blocked" if blocked else "masked"
        s = FCISolver(StateInfo(k, k, 1, 0, 0), 1, ints, {"FCI_SYM_BLOCKED": blocked, "E_CONVERGENCE": 1e-9,
                                                          "R_CONVERGENCE": 1e-5, "DL_SUBSPACE_PER_ROOT": 8}, device=local)
        # device vectors in the engine layout: the target irrep's blocks, or the whole C1 space (the
        # masked layout's sigma costs the same whatever the input holds outside the irrep)
        nv = s.size() if blocked else len(s.strings(0)) * len(s.strings(1))
        out["n_vec"][lay] = nv
        g = torch.Generator(device="cuda").manual_seed(0)
        x = torch.randn(nv, dtype=torch.float64, device="cuda", generator=g)
        x /= x.norm()
        y = torch.empty_like(x)
        stream = torch.cuda.ExternalStream(s.stream())
        for prec_name, prec in (("FP64", capi.PREC_FP64), ("MIXED", capi.PREC_MIXED)):
            def one():
                capi.check(L.fcib_sigma_device(s._h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), prec, None))
            for _ in range(args.warmup):
                one()
            torch.cuda.synchronize()
            p0 = s.profile()
            st = torch.cuda.Event(enable_timing=True)
            en = torch.cuda.Event(enable_timing=True)
            st.record(stream)
            for _ in range(args.steps):
                one()
            en.record(stream)
            en.synchronize()
            p1 = s.profile()
            out["sigma_ms"][f"{lay}_{prec_name}"] = st.elapsed_time(en) / args.steps
            ab, same = ("ab64_ms", "same64_ms") if prec == capi.PREC_FP64 else ("ab_ms", "same_ms")
            out.setdefault("sigma_parts_ms", {})[f"{lay}_{prec_name}"] = {
                "opposite_spin": (p1[ab] - p0[ab]) / args.steps, "same_spin": (p1[same] - p0[same]) / args.steps}
        del x, y
        torch.cuda.empty_cache()
        for prec_name in ("MIXED", "FP64"):
            if prec_name == "FP64" and not blocked and args.no_fp64:
                continue
            s.set_options({"FCI_PRECISION": prec_name})
            s.reset_guess()  # a fresh guess, not a restart from the previous solve
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e = s.compute_energy()
            out["solve"][f"{lay}_{prec_name}"] = {"seconds": time.perf_counter() - t0, "energy": e,
                                                  "iterations": s.iterations()}
        del s
        torch.cuda.empty_cache()
    sp = {p: out["sigma_ms"][f"masked_{p}"] / out["sigma_ms"][f"blocked_{p}"] for p in ("FP64", "MIXED")}
    if rank == 0:
        print(json.dumps({
            "metric": f"sigma ms @D2h CAS({n},{n}): irrep-blocked layout", "value": out["sigma_ms"]["blocked_MIXED"],
            "unit": "ms", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
            "dtype": "tf32x3/f64", "data": "synthetic",
            "config": {"workload": f"D2h CAS({n},{n}) synthetic L={3 * n}, orbital irreps {osym}, Ag singlet",
                       "n_vec": out["n_vec"]},
            "sigma_ms": out["sigma_ms"], "sigma_parts_ms": out["sigma_parts_ms"],
            "sigma_speedup_blocked_vs_masked": sp, "solve": out["solve"],
        }), flush=True)


def run_gas(args, world, rank, local):
    """GAS spaces (GenCISolver): C1 CAS(n,n), GAS1 = the lower half of the orbitals, GAS2 = the upper
    half holding at most m electrons (m = 2, 4).  Sigma time and time to solution of the kept-string
    blocked layout (blocks of the strings some GAS determinant uses) against the masked C1 layout."""
    import ctypes as C
    import torch
    from forte_b200 import GenCISolver, StateInfo, build, capi, synthetic
    build.build()
    torch.cuda.set_device(local)
    n, k = args.n, args.n // 2
    osym = [(i // 2) % 8 for i in range(n)] if args.gas_sym == "d2h" else None
    ints = synthetic(n, 3 * n, SEED, gap=GAP, orbsym=osym)
    spaces = [list(range(k)), list(range(k, n))]
    L = capi.lib()
    res = {}
    for m in [int(x) for x in args.gas_m.split(",")]:
        st = StateInfo(k, k, 1, 0, 0, (2 * k - m, 0), (2 * k, m))
        for lay in args.gas_layouts.split(","):
            blocked = lay == "blocked"
            s = GenCISolver(st, 1, ints, spaces, {"FCI_SYM_BLOCKED": blocked, "E_CONVERGENCE": 1e-9,
                                                   "R_CONVERGENCE": 1e-5, "DL_SUBSPACE_PER_ROOT": 8,
                                                   "DL_MAXITER": 400}, device=local)
            ndet = s.size()
            nv = s.layout_size()
            r = {"gas_determinants": ndet, "layout_elements": nv, "sigma_ms": {}, "solve": {}}
            g = torch.Generator(device="cuda").manual_seed(0)
            x = torch.randn(nv, dtype=torch.float64, device="cuda", generator=g)
            x /= x.norm()
            y = torch.empty_like(x)
            stream = torch.cuda.ExternalStream(s.stream())
            for prec_name, prec in (("FP64", capi.PREC_FP64), ("MIXED", capi.PREC_MIXED)):
                def one():
                    capi.check(L.fcib_sigma_device(s._h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), prec,
                                                   None))
                for _ in range(args.warmup):
                    one()
                torch.cuda.synchronize()
                l0 = s.profile()["launches"]
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(args.steps):
                    one()
                e1.record(stream)
                e1.synchronize()
                r["sigma_ms"][prec_name] = e0.elapsed_time(e1) / args.steps
                r.setdefault("launches_per_sigma", {})[prec_name] = (s.profile()["launches"] - l0) / args.steps
            del x, y
            torch.cuda.empty_cache()
            for prec_name in ("MIXED", "FP64"):
                s.set_options({"FCI_PRECISION": prec_name})
                s.reset_guess()
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                e = s.compute_energy()
                r["solve"][prec_name] = {"seconds": time.perf_counter() - t0, "energy": e,
                                         "iterations": s.iterations()}
            res[f"m{m}_{lay}"] = r
            del s
            torch.cuda.empty_cache()
    if rank == 0:
        print(json.dumps({
            "metric": f"GAS CAS({n},{n}) time to solution (mixed), upper half <= 4 electrons, kept-string blocks",
            "value": res.get("m4_blocked", next(iter(res.values())))["solve"]["MIXED"]["seconds"], "unit": "s",
            "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": False, "dtype": "tf32x3/f64",
            "data": "synthetic",
            "config": {"workload": f"{'D2h' if osym else 'C1'} CAS({n},{n}) synthetic L={3 * n}, GAS1 = orbitals "
                                   f"0..{k - 1}, GAS2 = {k}..{n - 1} with at most m electrons, Ag singlet",
                       "orbital_irreps": osym},
            "results": res,
        }), flush=True)


def run_configs(args, world, rank, local):
    """Time to solution of the two small workloads: CAS(8,8) (4,900 determinants, 1 root, FP64,
    synthetic L = 24; also solved by the CPU oracle on one core) and CAS(12,12) (853,776
    determinants, 3 roots, L = 36, FP64 vs mixed, plus the 1-/2-RDMs of the three roots).  Every
    step is a fresh solve (no restart), timed with CUDA events on the engine stream."""
    import torch
    from forte_b200 import FCISolver, StateInfo, build, synthetic
    build.build()
    torch.cuda.set_device(local)
    out = {}
    # CAS(8,8)
    ints8 = synthetic(8, 24, SEED)
    opts = {"E_CONVERGENCE": 1e-9, "R_CONVERGENCE": 1e-6}
    s8 = FCISolver(StateInfo(4, 4, 0), 1, ints8, opts, device=local)
    st8 = torch.cuda.ExternalStream(s8.stream())
    for _ in range(args.warmup):
        solve_once(s8, torch, st8)
    t8 = [solve_once(s8, torch, st8) for _ in range(args.steps)]
    cpu8 = None
    if rank == 0 and not args.no_cpu:
        from oracle.oracle import Oracle
        o = Oracle(8, 4, 4)
        o.set_integrals(ints8)
        t0 = time.perf_counter()
        r = o.solve(nroot=1, multiplicity=0, e_conv=1e-9, r_conv=1e-6)
        cpu8 = {"seconds": time.perf_counter() - t0, "iterations": r["iterations"],
                "energy_difference": abs(r["energies"][0] - s8.energies()[0]), "cores": 1, "kind": "port"}
    out["cas8_fp64"] = {"seconds": allmax(world, statistics.mean(t8)), "iterations": s8.iterations(),
                        "energy": s8.energies()[0], "cpu_oracle": cpu8}
    # CAS(12,12), 3 roots
    ints12 = synthetic(12, 36, SEED)
    # DL_MAXITER 400: the reference's solver needs 125 iterations here (its restatement in the oracle
    # stops unconverged at the default 100), so the default would time iterations, not a solution
    opts12 = {"E_CONVERGENCE": 1e-10, "R_CONVERGENCE": 1e-6, "DL_SUBSPACE_PER_ROOT": 8, "DL_MAXITER": 400}
    res = {}
    for prec in ("FP64", "MIXED"):
        s = FCISolver(StateInfo(6, 6, 0), 3, ints12, dict(opts12, FCI_PRECISION=prec), device=local)
        st = torch.cuda.ExternalStream(s.stream())
        for _ in range(args.warmup):
            solve_once(s, torch, st)
        ts = [solve_once(s, torch, st) for _ in range(args.steps)]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.rdms([(0, 0), (1, 1), (2, 2)], 2)
        rdm_s = time.perf_counter() - t0
        res[prec] = {"seconds": allmax(world, statistics.mean(ts)), "iterations": s.iterations(),
                     "energies": s.energies(), "rdms_3_roots_seconds": rdm_s}
        del s
        torch.cuda.empty_cache()
    de = max(abs(a - b) for a, b in zip(res["MIXED"]["energies"], res["FP64"]["energies"]))
    with open(os.path.join(ROOT, "tests", "golden", "cas12_roots.json")) as f:
        oracle12 = json.load(f)
    for prec in res:
        res[prec]["max_difference_vs_oracle_davidson"] = max(
            abs(a - b) for a, b in zip(res[prec]["energies"], oracle12["energies"]))
    res["oracle_davidson"] = {"energies": oracle12["energies"], "iterations": oracle12["iterations"],
                              "source": "tests/golden/cas12_roots.json"}
    out["cas12_3roots"] = dict(res, max_energy_difference=de,
                               speedup_mixed_vs_fp64=res["FP64"]["seconds"] / res["MIXED"]["seconds"])
    if rank == 0:
        print(json.dumps({
            "metric": "time to solution of the CAS(8,8) and CAS(12,12) workloads", "value": res["MIXED"]["seconds"],
            "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64 / tf32x3", "data": "synthetic",
            "config": {"workload": "CAS(8,8) L=24 1 root FP64; CAS(12,12) L=36 3 roots FP64 vs mixed",
                       "parallelism": f"replicas x{world}"},
            **out}), flush=True)


def run_precond(args, world, rank, local):
    """Learned vs diagonal preconditioner: Davidson at CAS(14,14) (11,778,624 determinants, Ms = 0,
    2 roots, synthetic L = 42) over several integral seeds, same precision for both, every energy
    certified by FP64 sigma.  The mixed sigma accumulates in integers, so a repeated solve of one
    seed reproduces its iteration count exactly; the line records that check."""
    import torch
    from forte_b200 import FCISolver, StateInfo, build, synthetic
    build.build()
    torch.cuda.set_device(local)
    n = args.n if args.n != 16 else 14
    opts = {"DL_SUBSPACE_PER_ROOT": 8, "DL_COLLAPSE_PER_ROOT": 2, "DL_MAXITER": 300, "E_CONVERGENCE": 1e-9,
            "R_CONVERGENCE": 1e-5, "FCI_PRECISION": args.precision, "FCI_SAME_SPIN": args.same_spin}
    seeds = list(range(1, args.seeds + 1))
    per_seed = []
    repeat_ok = True
    for seed in seeds:
        ints = synthetic(n, 3 * n, seed)
        row = {"seed": seed}
        for pre in ("DIAG", "MLP"):
            s = FCISolver(StateInfo(n // 2, n // 2, 0), 2, ints, dict(opts, FCI_PRECONDITIONER=pre), device=local)
            stream = torch.cuda.ExternalStream(s.stream())
            for _ in range(args.warmup):
                solve_once(s, torch, stream)
            it_w = s.iterations()
            times = [solve_once(s, torch, stream) for _ in range(args.steps)]
            if args.warmup > 0 and s.iterations() != it_w:
                repeat_ok = False
            row[pre] = {"seconds": statistics.mean(times), "iterations": s.iterations(), "energies": s.energies()}
            del s
            torch.cuda.empty_cache()
        row["max_energy_difference"] = max(abs(a - b) for a, b in zip(row["MLP"]["energies"], row["DIAG"]["energies"]))
        per_seed.append(row)
    if rank == 0:
        tot = {pre: {"seconds": sum(r[pre]["seconds"] for r in per_seed),
                     "iterations": sum(r[pre]["iterations"] for r in per_seed)} for pre in ("DIAG", "MLP")}
        print(json.dumps({
            "metric": f"Davidson time-to-solution @CAS({n},{n}) 2 roots over {len(seeds)} seeds: learned vs diagonal "
                      f"preconditioner", "value": tot["MLP"]["seconds"], "unit": "s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": args.precision.lower(), "data": "synthetic",
            "config": {"workload": f"CAS({n},{n}) synthetic L={3 * n} Ms=0 2 roots subspace 8, seeds {seeds}"},
            "totals": tot, "per_seed": per_seed,
            "seeds_with_fewer_iterations_learned": sum(r["MLP"]["iterations"] < r["DIAG"]["iterations"] for r in per_seed),
            "repeat_solves_same_iterations": repeat_ok,
            "speedup_learned_vs_diagonal": tot["DIAG"]["seconds"] / tot["MLP"]["seconds"],
        }), flush=True)


# the batched workload asks for FP32/FP64 mixed precision: FP32 sigma, FP64 subspace and residuals,
# FP64 sigma after the restart that certifies convergence
BATCH_OPTS = {"E_CONVERGENCE": 1e-9, "R_CONVERGENCE": 1e-5, "DL_SUBSPACE_PER_ROOT": 8, "DL_COLLAPSE_PER_ROOT": 2,
              "DL_MAXITER": 200, "FCI_PRECISION": "MIXED"}


def batch_instances(count, sizes, seed):
    """Seeded CAS instances: n drawn uniformly from `sizes`, integrals synthetic(n, 3n, seed_i)."""
    from forte_b200 import synthetic
    rng = np.random.default_rng(seed)
    ns = rng.choice(sizes, size=count)
    return [(synthetic(int(n), 3 * int(n), seed * 100003 + i), (int(n) + 1) // 2, int(n) // 2) for i, n in enumerate(ns)]


def cpu_batch_sample(instances, nroot, iterations):
    """The oracle's CPU Davidson (single-threaded C), scaled to the batch: instances of up to 8 orbitals
    are solved in full (one per size); for larger ones one oracle sigma is timed and multiplied by
    the sigma builds the batch needed for that size (about nroot per iteration plus the guess).
    Returns (instances/s on one core for the whole size distribution, description).  Instances are
    independent, so a host with P free cores would reach at most P times this."""
    from oracle.oracle import Oracle
    sizes = sorted({x[0].n for x in instances})
    per = {}
    how = []
    for n in sizes:
        ints, na, nb = next(x for x in instances if x[0].n == n)
        o = Oracle(n, na, nb)
        o.set_integrals(ints)
        if n <= 8:
            t0 = time.perf_counter()
            o.solve(nroot=nroot, multiplicity=0, e_conv=BATCH_OPTS["E_CONVERGENCE"], r_conv=BATCH_OPTS["R_CONVERGENCE"],
                    maxiter=BATCH_OPTS["DL_MAXITER"], subspace_per_root=BATCH_OPTS["DL_SUBSPACE_PER_ROOT"],
                    collapse_per_root=BATCH_OPTS["DL_COLLAPSE_PER_ROOT"])
            per[n] = time.perf_counter() - t0
            how.append(f"CAS({n},{n}) solved")
        else:
            c = np.random.default_rng(0).normal(size=o.ndet)
            t0 = time.perf_counter()
            o.sigma(c)
            ts = time.perf_counter() - t0
            its = [it for x, it in zip(instances, iterations) if x[0].n == n]
            nsig = nroot * float(np.mean(its)) + 2 * nroot
            per[n] = ts * nsig
            how.append(f"CAS({n},{n}) one sigma x {nsig:.0f}")
    total = sum(per[x[0].n] for x in instances)
    return len(instances) / total, "oracle Davidson on 1 core: " + ", ".join(how) + \
        f"; summed over the {len(instances)}-instance size distribution"


def run_batch(args, world, rank, local):
    """Batched CASCI: instances/s of one persistent launch over seeded CAS instances."""
    import ctypes as C
    import torch
    from forte_b200 import build, capi
    from forte_b200.batch import BatchSolver
    if args.phases:
        # the profiling build: the same kernels with per-phase clock counters
        capi.LIB_PATH = build.build(phases=True)
    else:
        build.build()
    torch.cuda.set_device(local)
    sizes = [int(x) for x in args.batch_sizes.split(",")]
    inst = batch_instances(args.batch_count, sizes, SEED + rank)
    opts = dict(BATCH_OPTS)
    if args.maxiter:
        opts["DL_MAXITER"] = args.maxiter
    t0 = time.perf_counter()
    b = BatchSolver(inst, nroot=4, options=opts, device=local)
    setup_s = time.perf_counter() - t0
    tuned = b.tune() if args.warmup > 0 else None
    for _ in range(max(0, args.warmup - 1)):
        b.solve()
    barrier(world)
    cycles = (C.c_ulonglong * 8)()
    if args.phases:
        capi.check(capi.lib().fcib_batch_phase_cycles(cycles))  # reset
    ms = []
    for _ in range(args.steps):
        e, it, cv, d = b.solve()
        ms.append(d)
    step_s = allmax(world, statistics.mean(ms) / 1e3)
    phases = None
    if args.phases:
        capi.check(capi.lib().fcib_batch_phase_cycles(cycles))
        names = ["sigma_opposite_spin", "sigma_same_spin", "g_update", "subspace", "residuals", "preconditioner",
                 "collapse", "gram_schmidt"]
        tot = float(sum(cycles)) or 1.0
        phases = {nm: cycles[i] / tot for i, nm in enumerate(names)}
    # end to end: integrals from host memory to energies back, through the public API
    t1 = time.perf_counter()
    b2 = BatchSolver(inst, nroot=4, options=opts, device=local)
    if tuned:
        b2.set_shape(tuned["threads"], tuned["pair_tile"], tuned["cluster"])
    e2, it2, cv2, _ = b2.solve()
    e2e_s = allmax(world, time.perf_counter() - t1)
    h2d = sum(sum(getattr(x[0], k).nbytes for k in ("oei_a", "oei_b", "tei_aa", "tei_ab", "tei_bb")) for x in inst)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, sample = cpu_batch_sample(inst, 4, it)
        cpu = {"value": v, "unit": "instances/s", "cores": 1, "kind": "port", "sample": sample}
    if rank == 0:
        ndets = [x[0].n for x in inst]
        print(json.dumps({
            "metric": f"batched CASCI instances/s ({args.batch_count} instances CAS({min(sizes)},{min(sizes)})-"
                      f"CAS({max(sizes)},{max(sizes)}), 4 roots, one persistent launch)",
            "value": world * args.batch_count / step_s, "unit": "instances/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
            "config": {"workload": f"{args.batch_count} seeded instances, n uniform in {sizes}, L=3n, 4 roots, "
                                   "subspace 8/root", "e_convergence": opts["E_CONVERGENCE"],
                       "r_convergence": opts["R_CONVERGENCE"], "parallelism": f"replicas x{world}"},
            "iterations_mean": float(np.mean(it)), "iterations_max": int(np.max(it)),
            "converged_fraction": float(np.mean(cv)), "autotune": tuned, "setup_seconds": setup_s,
            "phase_fractions": phases, "build": "profiling (phase clocks)" if args.phases else "default",
            "e2e": {"value": world * args.batch_count / e2e_s, "unit": "instances/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(e2.nbytes + it2.nbytes + cv2.nbytes)},
            "cpu_baseline": cpu, "gpu_launches": 1,
            "instances_by_orbitals": {str(n): int(ndets.count(n)) for n in sorted(set(ndets))},
        }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="MIXED", choices=["MIXED", "MIXED_TF32", "FP64"])
    ap.add_argument("--preconditioner", default="DIAG", choices=["DIAG", "MLP"])
    ap.add_argument("--same-spin", default="TC", choices=["TC", "CUDA_CORES"],
                    help="mixed same-spin kernel: tensor cores (3xTF32) or FP32 CUDA cores")
    ap.add_argument("--ref-iterations", type=int, default=63,
                    help="FP64 iteration count used by the CPU arm (the FP64 GPU solve of this workload takes 63)")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparator solve")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mlp", action="store_true", help="skip the mixed + learned-preconditioner solve")
    ap.add_argument("--batch-count", type=int, default=256)
    ap.add_argument("--batch-sizes", default="6,7,8,9,10")
    ap.add_argument("--maxiter", type=int, default=0, help="batch mode: Davidson iteration cap (0 = 200)")
    ap.add_argument("--phases", action="store_true",
                    help="batch mode: run the profiling build and report the share of clock cycles per phase")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--mode", default="solve", choices=["solve", "sigma", "precond", "batch", "configs", "sym", "gas"],
                    help="solve: the Davidson time-to-solution metric; sigma: sigma builds/s at CAS(n,n); "
                         "precond: learned vs diagonal preconditioner at CAS(14,14), 2 roots; "
                         "batch: batched CASCI instances/s; configs: time to solution at CAS(8,8) and "
                         "CAS(12,12) (3 roots, FP64 vs mixed); sym: blocked vs masked layout of a D2h CAS(n,n)")
    ap.add_argument("--n", type=int, default=16, help="active orbitals of the sigma mode")
    ap.add_argument("--seeds", type=int, default=5, help="precond mode: integral seeds of the A/B comparison")
    ap.add_argument("--gas-m", default="2,4", help="gas mode: upper-half electron limits to run")
    ap.add_argument("--gas-layouts", default="blocked,masked", help="gas mode: layouts to run")
    ap.add_argument("--gas-sym", default="c1", choices=["c1", "d2h"],
                    help="gas mode: no symmetry, or D2h with two orbitals per irrep")
    args = ap.parse_args()
    world, rank, local = dist_init(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.mode == "sigma":
        run_sigma(args, world, rank, local)
        return
    if args.mode == "precond":
        run_precond(args, world, rank, local)
        return
    if args.mode == "batch":
        run_batch(args, world, rank, local)
        return
    if args.mode == "configs":
        run_configs(args, world, rank, local)
        return
    if args.mode == "gas":
        run_gas(args, world, rank, local)
        return
    if args.mode == "sym":
        run_sym(args, world, rank, local)
        return

    import torch
    from forte_b200 import FCISolver, StateInfo, build, synthetic
    build.build()
    torch.cuda.set_device(local)
    ints = synthetic(N_ORB, L_AUX, SEED, gap=GAP)
    state = StateInfo(N_ORB // 2, N_ORB // 2, 0)  # multiplicity 0: lowest root of the Ms=0 space
    hbm, bf16, bf16s, peak_kind = peaks()

    # FP64 comparator (reference energy and time)
    fp64_s = None
    e_ref = None
    prof64 = None
    w64 = max(1, min(args.warmup, 2))
    k64 = max(1, min(args.steps, 2))
    if not args.no_fp64:
        # warm-up solves like the mixed arm's (tables, buffers and kernels ready), then timed solves
        f = FCISolver(state, 1, ints, dict(OPTS, FCI_PRECISION="FP64"), device=local)
        fstream = torch.cuda.ExternalStream(f.stream())
        for _ in range(w64):
            solve_once(f, torch, fstream)
        t64 = [solve_once(f, torch, fstream) for _ in range(k64)]
        fp64_s = allmax(world, statistics.mean(t64))
        e_ref = f.energies()[0]
        prof64 = f.profile()
        iters64 = f.iterations()
        del f
        torch.cuda.empty_cache()
    # FP64 peak of this GPU (CUDA-core FMA and FP64 tensor-core MMA), for the FP64 sigma's fraction
    from forte_b200 import capi as _capi
    import ctypes as _C
    pk_fma, pk_dmma = _C.c_double(), _C.c_double()
    _capi.check(_capi.lib().fcib_fp64_peak(local, _C.byref(pk_fma), _C.byref(pk_dmma)))
    fp64_peak = max(pk_fma.value, pk_dmma.value)

    opts = dict(OPTS, FCI_PRECISION=args.precision, FCI_PRECONDITIONER=args.preconditioner,
                FCI_SAME_SPIN=args.same_spin)
    s = FCISolver(state, 1, ints, opts, device=local)
    stream = torch.cuda.ExternalStream(s.stream())
    for _ in range(args.warmup):
        solve_once(s, torch, stream)
    barrier(world)
    torch.cuda.synchronize()
    gpu_index = local
    cvd = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    if cvd and cvd.split(",")[local].strip().isdigit():
        gpu_index = int(cvd.split(",")[local])
    clocks = Clocks(gpu_index)
    launches0 = s.profile()["launches"]
    clocks.start()
    times, profs = [], []
    t_wall = time.perf_counter()
    for _ in range(args.steps):
        times.append(solve_once(s, torch, stream))
        profs.append(s.profile())
    torch.cuda.synchronize()
    wall = time.perf_counter() - t_wall
    clk = clocks.stop()
    barrier(world)
    launches = s.profile()["launches"] - launches0
    step_s = allmax(world, statistics.mean(times))
    energy = s.energies()[0]
    iters = s.iterations()

    # roofline of the dominant kernel: tensor-core opposite-spin contraction
    n, k = N_ORB, N_ORB // 2
    npair = n * (n + 1) // 2
    s1 = k * (n - k) + k
    ndet = (len(s.strings(0))) * (len(s.strings(1)))
    flops_per_launch = 2.0 * ndet * s1 * npair  # one TF32 pass of the connected-pair contraction
    ab_ms = sum(p["tc_kernel_ms"] for p in profs) / max(1, sum(p["n_ab"] for p in profs))
    achieved = flops_per_launch / (ab_ms * 1e-3) / 1e12 if ab_ms > 0 else None
    traffic = NCU_TRAFFIC_CAS15 * (ndet * s1) / NCU_UNITS_CAS15
    roofline = {"bound": "tensor", "kernel": "k_ab_tc<3xTF32>", "achieved": achieved, "peak": bf16s,
                "unit": "TFLOP/s", "frac": (achieved / bf16s) if achieved else None, "traffic": traffic,
                "peak_kind": f"bf16 sustained ({peak_kind}); the TF32 tensor rate is half of bf16",
                "frac_vs_tf32": (2 * achieved / bf16s) if achieved else None,
                "flops_per_launch": flops_per_launch, "launch_ms": ab_ms}

    # FP64 sigma: algorithmic flops (opposite-spin 2 N s1 npair + same-spin 2 x 2 N d2) over its time
    from math import comb
    d2 = comb(k, 2) * comb(n - k + 2, 2)
    flops64 = 2.0 * ndet * s1 * npair + 2 * 2.0 * ndet * d2
    sigma64_ms = fp64_sigma_tf = fp64_ab_tf = None
    if prof64 and prof64["n_ab64"] > 0:
        sigma64_ms = (prof64["ab64_ms"] + prof64["same64_ms"]) / prof64["n_ab64"]
        fp64_sigma_tf = flops64 / (sigma64_ms * 1e-3) / 1e12
        fp64_ab_tf = flops_per_launch / (prof64["ab64_ms"] / prof64["n_ab64"] * 1e-3) / 1e12

    # end to end through the C ABI with host buffers: integrals in, energies + CI vector out
    e2e = None
    if not args.no_e2e:
        nsteps = min(args.steps, 2)
        host_vec = np.empty(ndet)
        from forte_b200 import capi
        import ctypes as C
        et = []
        h2d = sum(x.nbytes for x in (ints.oei_a, ints.oei_b, ints.tei_aa, ints.tei_ab, ints.tei_bb))
        for _ in range(nsteps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s.set_integrals(ints)
            s.reset_guess()  # a fresh solve, not a restart from the previous step's vectors
            s.compute_energy()
            capi.check(capi.lib().fcib_get_vector(s._h, 0, capi.dptr(host_vec)))
            torch.cuda.synchronize()
            et.append(time.perf_counter() - t0)
        e2e = {"value": allmax(world, statistics.mean(et)), "unit": "s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(host_vec.nbytes + 16)}

    # the metric's learned configuration: mixed sigma + the learned preconditioner, one warm-up solve
    # (network tables built) and one timed solve, its energy certified by the FP64 sigma like the rest
    mlp = None
    if not args.no_mlp and args.preconditioner == "DIAG":
        sm = FCISolver(state, 1, ints, dict(opts, FCI_PRECONDITIONER="MLP"), device=local)
        mstream = torch.cuda.ExternalStream(sm.stream())
        solve_once(sm, torch, mstream)
        t_mlp = solve_once(sm, torch, mstream)
        mlp = {"seconds": allmax(world, t_mlp), "iterations": sm.iterations(), "energy": sm.energies()[0],
               "energy_error_vs_fp64": (abs(sm.energies()[0] - e_ref) if e_ref is not None else None),
               "speedup_vs_fp64": (fp64_s / t_mlp) if fp64_s else None}
        del sm
        torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        sig14 = cpu_sigma_sample(1, 14)
        it_ref = iters64 if fp64_s is not None else args.ref_iterations
        cpu_s, ratio = cpu_extrapolation(sig14, it_ref)
        model, ncpu = host_cpu()
        cpu = {"value": cpu_s, "unit": "s", "cores": 1, "kind": "port", "host_cpu": model, "host_cores": ncpu,
               "sample": f"1 sigma build of CAS(14,14) (11,778,624 dets) by the CPU oracle on 1 core "
                         f"({sig14:.2f} s), extrapolated to a {it_ref}-iteration CAS(16,16) solve by the reference "
                         f"FMA-count ratio {ratio:.2f} plus 5% Davidson overhead"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": step_s, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "tf32x3/f64" if args.precision == "MIXED" else args.precision.lower(),
            "data": "synthetic",
            "config": {"workload": "CAS(16,16) synthetic L=48 gap=0.3 Ms=0 1 root subspace 8", "n_orb": N_ORB,
                       "n_det": ndet, "precision": args.precision, "preconditioner": args.preconditioner,
                       "same_spin": args.same_spin,
                       "e_convergence": OPTS["E_CONVERGENCE"], "r_convergence": OPTS["R_CONVERGENCE"],
                       "l2": "inputs larger than L2 (1.3 GB CI vectors)", "parallelism": f"replicas x{world}"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches / max(1, args.steps)),
            "clocks": clk,
            "iterations": iters, "energy": energy,
            "fp64_seconds": fp64_s, "fp64_energy": e_ref,
            "energy_error_vs_fp64": (abs(energy - e_ref) if e_ref is not None else None),
            "speedup_vs_fp64": (fp64_s / step_s) if fp64_s else None,
            "fp64_iterations": (iters64 if fp64_s is not None else None),
            "sigma_ms_mixed": profs[-1]["ab_ms"] / max(1, profs[-1]["n_ab"]) + profs[-1]["same_ms"] / max(1, profs[-1]["n_ab"]),
            "sigma_ms_fp64": sigma64_ms,
            "fp64_warmup": w64 if fp64_s is not None else None, "fp64_steps": k64 if fp64_s is not None else None,
            "fp64_peak_tflops": {"dfma": pk_fma.value, "dmma": pk_dmma.value,
                                 "how": "fcib_fp64_peak: FMA chains / m8n8k4 f64 MMA chains, CUDA events"},
            "fp64_sigma_tflops": fp64_sigma_tf, "fp64_sigma_frac": (fp64_sigma_tf / fp64_peak) if fp64_sigma_tf else None,
            "fp64_ab_tflops": fp64_ab_tf, "fp64_ab_frac": (fp64_ab_tf / fp64_peak) if fp64_ab_tf else None,
            "davidson_ms_per_iter": (profs[-1]["total_ms"] - profs[-1]["sigma_ms"]) / max(1, iters),
            "wall_s_timed_region": wall,
            "learned": mlp,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
