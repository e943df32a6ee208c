#!/usr/bin/env python
"""Benchmark of the self-gravity FMG Poisson solve on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload jeans6|nested5|uniform64|uniform256|deep8]

A step is one complete solve (zero initial guess) to relative residual
<= 1e-10 on the 6-level Jeans-refined hierarchy (128^3 periodic base of 8^3
blocks, 133,856 blocks, 60.2M leaf cells).  `value` is the mixed-precision
solves/s with inputs resident in HBM (device-timed with CUDA events on the
solve's stream); `fp64` repeats it for the plain FP64 path; `e2e` is the same
metric through the host-buffer C ABI call (sfm_solve) with pinned buffers,
the host<->device copies inside the timed region.  Inputs (>= 1 GB per field)
exceed the 126 MB L2, so no flush is needed between steps.

Multi-GPU: the path runs as independent replicas (one hierarchy per GPU, no
collective in the data path); value = all ranks' solves / max-over-ranks time.

--impl reference times the CPU restatement of the reference algorithm
(oracle/, the reference itself cannot be built here) on the host cores:
every step, warm-up included, is one complete FP64 solve to 1e-10.  The GPU
line's cpu_baseline is one such solve, whose potential and g also give the
GPU results' error against the oracle (phi_rel_err_vs_oracle).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "AMR Poisson solves/s & Gcell-updates/s at rel. resid ≤1e-10, mixed vs plain FP64"
REL_TOL = 1e-10
MAX_OUTER = 30


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="jeans6")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the adjoint leg (one adjoint solve of W = 1/2 sum rho phi dV, mixed precision)")
    ap.add_argument("--tune-table", default=None,
                    help="with --single: load this tuning table if the file exists, else tune and write it "
                         "(a profiler run then launches only the solve)")
    ap.add_argument("--single", choices=["mixed", "fp64"], default=None,
                    help="autotune, then run exactly one solve of that precision and exit (for profiler launch lists)")
    return ap.parse_args()


def load_workload(name):
    """(hierarchy, rho array [nb,G,G,G] with 2 ghost layers, bc), cached on local disk."""
    import numpy as np
    from code_only_b200 import workloads as w
    cache = os.path.join("/tmp", f"sfmg_{name}_v1.npz")
    h, fn, bc = None, None, None
    if os.path.exists(cache):
        try:
            z = np.load(cache)
            h = w.Hierarchy(ni=int(z["ni"]), ngb=tuple(z["ngb"].tolist()), nlev=int(z["nlev"]),
                            periodic=bool(z["periodic"]), box_lo=z["box_lo"], box_size=float(z["box_size"]),
                            level=z["level"], ijk=z["ijk"], parent=z["parent"], child=z["child"],
                            nbr=z["nbr"], touch=z["touch"], cellwidth=z["cellwidth"], x0=z["x0"])
            return h.contiguous(), z["rho"], int(z["bc"])
        except Exception:
            pass
    h, fn, bc = w.config_hierarchy(name)
    rho = w.block_field(h, 2, fn)
    try:
        np.savez(cache, ni=h.ni, ngb=np.array(h.ngb), nlev=h.nlev, periodic=h.periodic, box_lo=h.box_lo,
                 box_size=h.box_size, level=h.level, ijk=h.ijk, parent=h.parent, child=h.child, nbr=h.nbr,
                 touch=h.touch, cellwidth=h.cellwidth, x0=h.x0, rho=rho, bc=bc)
    except Exception:
        pass
    return h, rho, bc


def workload_config(name, h, bc):
    """The `config` object of both arms (same keys and values for one workload)."""
    return {
        "workload": name,
        "hierarchy": f"{h.nlev} AMR levels, {h.nblocks} blocks of {h.ni}^3, {h.leaf_cells()} leaf cells",
        "level_blocks": [int(v) for v in h.level_counts()],
        "bc": "periodic" if bc == 0 else "isolated sphere (multipole l<=4)",
        "rel_tol": REL_TOL,
        "l2": _l2_note(h),
    }


def _l2_note(h):
    """How the timed steps stand to the 126 MB L2: the FP64 level-0 field
    (one of the solve's arrays) against it."""
    field = h.nblocks * (h.ni + 2) ** 3 * 8
    if field > 126 * 2 ** 20:
        return f"inputs larger than L2 ({field / 2 ** 30:.2f} GiB per FP64 field), no flush"
    return f"inputs fit in L2 ({field / 2 ** 20:.1f} MiB per FP64 field), no flush: warm-cache figures"


def params_for(bc, precision, profile=0):
    from code_only_b200 import abi
    kw = dict(rel_tol=REL_TOL, max_outer=MAX_OUTER, precision=precision, profile=profile)
    if bc == abi.SFM_BC_SPHERE:
        kw["zero_mean"] = 0
        kw["lmax"] = 4
    return abi.default_params(bc, **kw)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n):
    from code_only_b200 import replicas
    info = replicas.setup()
    return info


def max_over_ranks(x, info):
    from code_only_b200 import replicas
    return replicas.max_over_ranks(info, x)


def barrier(info):
    from code_only_b200 import replicas
    replicas.barrier(info)


def time_device(solver, rho_d, psi_d, g_d, steps, warmup, info):
    """Device-timed solves (CUDA events on the solve's stream).  Returns
    (ms per solve over all ranks' max, last stats, launches, smoother stats)."""
    import torch
    stream = torch.cuda.Stream()            # the solve and the events share this stream
    torch.cuda.set_stream(stream)
    sptr = stream.cuda_stream
    st = None
    for _ in range(warmup):
        psi_d.zero_()
        st = solver.solve_device(rho_d.data_ptr(), psi_d.data_ptr(), g_d.data_ptr(), sptr)
    barrier(info)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches, sm_ms, sm_n, sm_cells, iters = 0, 0.0, 0, 0, []
    e0.record(stream)
    for _ in range(steps):
        psi_d.zero_()
        st = solver.solve_device(rho_d.data_ptr(), psi_d.data_ptr(), g_d.data_ptr(), sptr)
        launches += st.kernel_launches
        sm_ms += st.smoother_ms
        sm_n += st.smoother_launches
        sm_cells += st.smoother_cells
        iters.append(st.outer_iters)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(info)
    ms = e0.elapsed_time(e1) / steps
    return max_over_ranks(ms, info), st, launches, (sm_ms, sm_n, sm_cells), iters


def run_single(args):
    """One solve (no warm-up) of the chosen precision: the launch list of a
    profiler run then covers exactly one solve."""
    import torch
    from code_only_b200 import abi
    from code_only_b200.solver import FMGPoisson
    h, rho, bc = load_workload(args.workload)
    rho_d = torch.from_numpy(rho).cuda()
    psi_d = torch.zeros_like(rho_d)
    G = rho.shape[1]
    g_d = torch.zeros((h.nblocks, 3, G, G, G), dtype=torch.float64, device="cuda")
    prec = abi.SFM_PREC_MIXED if args.single == "mixed" else abi.SFM_PREC_FP64
    with FMGPoisson(h, params=params_for(bc, prec)) as s:
        if args.tune_table and os.path.exists(args.tune_table):
            s.load_tune_table(open(args.tune_table).read())
        else:
            s.autotune(3, rho_d.data_ptr())   # the launch shapes and schedule the timed bench uses
            if args.tune_table:
                with open(args.tune_table, "w") as fh:
                    fh.write(s.tune_table())
        torch.cuda.synchronize()
        st = s.solve_device(rho_d.data_ptr(), psi_d.data_ptr(), g_d.data_ptr())
        torch.cuda.synchronize()
    print(json.dumps({"single": args.single, "workload": args.workload, "outer_iters": st.outer_iters,
                      "true_rel_residual": st.true_rel_residual, "kernel_launches": st.kernel_launches,
                      "device_ms": st.device_ms}), flush=True)


def run_ours(args):
    import numpy as np
    import torch
    from code_only_b200 import abi, build as b
    from code_only_b200.solver import FMGPoisson

    info = dist_setup(args.gpus)
    rank, world, local = info.rank, info.world, info.local
    if rank == 0:
        b.build(verbose=False)
    barrier(info)
    h, rho, bc = load_workload(args.workload)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    rho_d = torch.from_numpy(rho).to(dev)
    psi_d = torch.zeros_like(rho_d)
    G = rho.shape[1]
    g_d = torch.zeros((h.nblocks, 3, G, G, G), dtype=torch.float64, device=dev)
    leaf_cells = h.leaf_cells()

    sampler = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    results = {}
    tables = {}
    for prec, key in ((abi.SFM_PREC_MIXED, "mixed"), (abi.SFM_PREC_FP64, "fp64")):
        t0 = time.perf_counter()
        ctx = FMGPoisson(h, params=params_for(bc, prec, profile=1))   # sfm_create: tables, device arrays
        create_s = time.perf_counter() - t0
        with ctx as s:
            # the built-in launch shapes, then the autotuned ones (sfm_autotune;
            # the results are bit-identical, only the launch shapes differ)
            ms_default = time_device(s, rho_d, psi_d, g_d, max(2, args.steps // 4), 1, info)[0]
            t0 = time.perf_counter()
            s.autotune(3, rho_d.data_ptr())
            tune_s = time.perf_counter() - t0
            tables[key] = s.tune_table()
            if key == "mixed" and sampler:
                sampler.start()
            ms, st, launches, smo, iters = time_device(s, rho_d, psi_d, g_d, args.steps, args.warmup, info)
            if key == "mixed" and sampler:
                clocks = sampler.stop()
            results[key] = dict(ms=ms, st=st, launches=launches, smo=smo, iters=iters,
                                resid=st.true_rel_residual, info=s.info(), ms_default=ms_default, tune_s=tune_s,
                                create_s=create_s)
            if rank == 0 and not args.no_cpu:   # kept on the host for the oracle comparison
                ng = (G - h.ni) // 2
                sl = slice(ng, ng + h.ni)
                results[key]["psi_h"] = psi_d[:, sl, sl, sl].cpu().numpy()
                results[key]["g_h"] = g_d[:, :, sl, sl, sl].cpu().numpy()
            if key == "mixed":
                psi_mixed = psi_d.clone()
    # phi of the mixed path against the plain FP64 path (block interiors;
    # each potential's mean removed first: a periodic box fixes phi up to a constant)
    ng = (G - h.ni) // 2
    a = psi_mixed[:, ng:ng + h.ni, ng:ng + h.ni, ng:ng + h.ni]
    bfp = psi_d[:, ng:ng + h.ni, ng:ng + h.ni, ng:ng + h.ni]
    if bc == abi.SFM_BC_PERIODIC:
        a = a - a.mean()
        bfp = bfp - bfp.mean()
    phi_err = float((a - bfp).abs().max() / bfp.abs().max())
    del psi_mixed, a, bfp
    # end to end through the host-buffer ABI (pinned host memory)
    e2e = None
    if not args.no_e2e:
        with FMGPoisson(h, params=params_for(bc, abi.SFM_PREC_MIXED)) as s:
            s.load_tune_table(tables["mixed"])
            rho_h = torch.from_numpy(rho).pin_memory().numpy()
            psi_h = torch.zeros(rho.shape, dtype=torch.float64).pin_memory().numpy()
            g_h = torch.zeros((h.nblocks, 3, G, G, G), dtype=torch.float64).pin_memory().numpy()
            for _ in range(max(1, args.warmup // 2)):
                psi_h[...] = 0.0
                s.solve(rho_h, psi_h)
            barrier(info)
            t_sum = 0.0
            st_e = abi.SfmStats()
            for _ in range(args.steps):
                psi_h[...] = 0.0   # the caller's cold start, outside the call
                t0 = time.perf_counter()
                out = s.lib.sfm_solve(s.ctx, rho_h.ctypes.data, psi_h.ctypes.data, g_h.ctypes.data,
                                      ctypes.byref(st_e))
                t_sum += time.perf_counter() - t0
                if out not in (abi.SFM_OK, abi.SFM_ENOTCONVERGED):
                    raise RuntimeError(f"sfm_solve failed {out}")
            barrier(info)
            ms_e2e = max_over_ranks(t_sum * 1e3 / args.steps, info)
            # bytes the call moved, as it reports them: the (-1:ni)^3 region of
            # rho and psi in, of psi out, and g's block interiors out
            e2e = {"value": world * 1e3 / ms_e2e, "unit": "solves/s",
                   "h2d_bytes_per_step": int(st_e.h2d_bytes),
                   "d2h_bytes_per_step": int(st_e.d2h_bytes),
                   "timing": "host wall clock around each blocking sfm_solve call (pinned host arrays)"}
    if rank != 0:
        from code_only_b200 import replicas
        replicas.teardown(info)
        return
    mx, fp = results["mixed"], results["fp64"]
    value = world * 1e3 / mx["ms"]
    # roofline of the dominant kernel: level-0 red-black colour launch
    sm_ms, sm_n, sm_cells = mx["smo"]
    elem = mx["st"].elem_bytes or 4
    colours = mx["st"].smoother_colours or 1
    # algorithmic bytes of one launch: one colour reads u, half of rhs and
    # writes half of u (2 values per leaf cell, the floor of the reference's
    # schedule, which refreshes ghosts between the colours); a fused launch
    # does colours / 2 full sweeps, each 3 values per leaf cell (u and rhs
    # read, u written) -- the per-sweep unit counted once per sweep done
    cells_per_launch = sm_cells / max(sm_n, 1)
    alg_bytes_per_launch = cells_per_launch * (2 if colours == 1 else 3 * (colours // 2)) * elem
    launch_s = (sm_ms / max(sm_n, 1)) * 1e-3
    achieved = alg_bytes_per_launch / launch_s / 1e9 if launch_s > 0 else None
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    traffic = None
    try:
        prof = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        traffic = prof.get(args.workload, {}).get("one_colour" if colours == 1 else "fused")
    except Exception:
        pass
    cells_updates = leaf_cells * 1.0
    sweeps = mx["smo"][1] * colours / max(args.steps, 1) / 2   # full red+black sweeps at level 0 per solve
    line = {
        "metric": METRIC,
        "value": round(value, 4),
        "unit": "solves/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(mx["ms"], 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 inner / f64 outer",
        "data": "synthetic",
        "config": workload_config(args.workload, h, bc),
        "parallelism": f"replicas x{world}",
        "gcell_updates_per_s": round(value * sweeps * cells_updates / 1e9, 3),
        "outer_iterations": {"mixed": mx["iters"][-1], "fp64": fp["iters"][-1]},
        "true_rel_residual": {"mixed": mx["resid"], "fp64": fp["resid"]},
        "fp64": {"value": round(world * 1e3 / fp["ms"], 4), "unit": "solves/s", "ms_per_step": round(fp["ms"], 4)},
        "mixed_over_fp64": round(fp["ms"] / mx["ms"], 3),
        "autotune": {
            "mixed_default_ms_per_step": round(mx["ms_default"], 3), "mixed_tuned_ms_per_step": round(mx["ms"], 3),
            "fp64_default_ms_per_step": round(fp["ms_default"], 3), "fp64_tuned_ms_per_step": round(fp["ms"], 3),
            "tuning_s": {"mixed": round(mx["tune_s"], 2), "fp64": round(fp["tune_s"], 2)},
            "choices_mixed": tune_summary(tables["mixed"]),
        },
        # sfm_create wall time (host tables, device arrays), paid once per hierarchy
        "context_create_s": {"mixed": round(mx["create_s"], 3), "fp64": round(fp["create_s"], 3)},
        "phi_rel_err_mixed_vs_fp64": phi_err,
        "roofline": {
            "kernel": f"k_relax_bulk<float, {h.ni}>: " + (f"{colours // 2} fused red-black sweep(s)" if colours >= 2
                                                          else "one red-black colour") + " over the leaf cells, fmg level 0",
            "bound": "hbm", "achieved": round(achieved, 1) if achieved else None, "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4) if achieved else None,
            "traffic": traffic,
            "alg_bytes_per_launch": alg_bytes_per_launch,
            "alg_bytes_rule": ("2 values per leaf cell (one colour)" if colours == 1 else
                               f"3 values per leaf cell per full sweep x {colours // 2} sweep(s) per launch"),
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if "hbm_gbs" in peaks else "fallback 6650 GB/s",
        },
        "gpu_launches": int(mx["launches"]),
        "clocks": clocks,
        "device_bytes": mx["info"]["device_bytes"],
    }
    if e2e:
        line["e2e"] = e2e
    if not args.no_adjoint:
        line["adjoint"] = time_adjoint(h, rho, bc)
    if not args.no_cpu:
        cpu, psi_o, g_o = cpu_baseline(h, rho, bc)
        line["cpu_baseline"] = cpu
        line["phi_rel_err_vs_oracle"] = oracle_errors(h, bc, psi_o, g_o, results)
    print(json.dumps(line), flush=True)
    from code_only_b200 import replicas
    replicas.teardown(info)


def tune_summary(text):
    """Counts of the tuned choices per knob, e.g. {"ghost_fill": {"0": 9, "1": 6}, ...}."""
    out = {}
    for ln in text.splitlines():
        f = ln.split()
        if len(f) == 6 and not ln.startswith("#"):
            out.setdefault(f[0], {}).setdefault(f[5], 0)
            out[f[0]][f[5]] += 1
    return out


def time_adjoint(h, rho, bc):
    """One adjoint solve (sfm_adjoint, host arrays, mixed precision) of
    W = 1/2 sum rho phi dV over leaf cells, to a Krylov residual of 1e-10;
    wall time around the call (host<->device copies of two fields included)."""
    import numpy as np
    from code_only_b200 import abi
    from code_only_b200.solver import FMGPoisson
    kw = dict(rel_tol=1e-10, max_outer=60, precision=abi.SFM_PREC_MIXED)
    if bc == abi.SFM_BC_SPHERE:
        kw.update(zero_mean=0, lmax=4)
    G = rho.shape[1]
    ng = (G - h.ni) // 2
    leaf = (h.level == h.nlev - 1) | (h.child[:, 0] < 0)
    dv = np.asarray(h.cellwidth)[np.asarray(h.level)] ** 3
    dJ = np.zeros_like(rho)
    sl = slice(ng, ng + h.ni)
    dJ[leaf, sl, sl, sl] = 0.5 * rho[leaf, sl, sl, sl] * dv[leaf, None, None, None]
    with FMGPoisson(h, params=abi.default_params(bc, **kw)) as s:
        s.adjoint(dJ, allow_unconverged=True)          # first call allocates the Krylov vectors
        t0 = time.perf_counter()
        _, st = s.adjoint(dJ, allow_unconverged=True)
        ms = (time.perf_counter() - t0) * 1e3
    return {"ms": round(ms, 2), "krylov_iterations": st.outer_iters, "true_rel_residual": st.true_rel_residual,
            "device_ms": round(st.device_ms, 2), "functional": "W = 1/2 sum(rho phi dV), leaf cells"}


def oracle_solve_timed(h, rho, bc):
    """One complete FP64 oracle solve to 1e-10 (g included).  Returns
    (seconds, outer iterations, psi interiors, g interiors)."""
    from tests.oracle_lib import oracle_solve
    t = time.perf_counter()
    rc, psi, g, st, _ = oracle_solve(h, rho, params_for(bc, 0), want_g=True)
    dt = time.perf_counter() - t
    if rc not in (0, -5):
        raise RuntimeError(f"oracle solve failed: {rc}")
    ng = (rho.shape[1] - h.ni) // 2
    sl = slice(ng, ng + h.ni)
    return dt, st.outer_iters, psi[:, sl, sl, sl].copy(), g[:, :, sl, sl, sl].copy()


def oracle_solve_profiled(h, rho, bc):
    """One complete FP64 oracle solve to 1e-10 with the exclusive time of each
    routine class.  Returns (seconds, outer iterations, {class: share of the solve})."""
    from tests.oracle_lib import oracle_profile
    t = time.perf_counter()
    rc, secs, total, st = oracle_profile(h, rho, params_for(bc, 0))
    dt = time.perf_counter() - t
    if rc not in (0, -5):
        raise RuntimeError(f"oracle solve failed: {rc}")
    return dt, st.outer_iters, {k: round(v / total, 4) for k, v in sorted(secs.items(), key=lambda kv: -kv[1])}


def cpu_baseline(h, rho, bc):
    """One complete solve of the oracle (CPU restatement of the reference
    algorithm, FP64, OpenMP over blocks) to 1e-10, measured."""
    from tests.oracle_lib import load_oracle
    threads = load_oracle().oracle_threads()
    dt, iters, psi, g = oracle_solve_timed(h, rho, bc)
    cpu = {"value": round(1.0 / dt, 6), "unit": "solves/s", "cores": threads, "kind": "port",
           "sample": f"one complete FP64 oracle solve of the same workload to 1e-10 ({iters} outer "
                     f"iterations, g included): {dt:.2f} s on {threads} OpenMP threads"}
    return cpu, psi, g


def oracle_errors(h, bc, psi_o, g_o, results):
    """Max-norm relative error of the GPU potentials and g against the oracle
    (block interiors; phi's mean removed on periodic boxes, whose constant is free)."""
    import numpy as np
    leaf = ((h.level == h.nlev - 1) | (h.child[:, 0] < 0))
    out = {}
    for key in ("fp64", "mixed"):
        r = results[key]
        if "psi_h" not in r:
            continue
        a, b = r["psi_h"], psi_o
        if bc == 0:
            a, b = a - a[leaf].mean(), b - b[leaf].mean()
        out[key] = {"phi": float(np.abs(a - b).max() / np.abs(b).max()),
                    "g": float(np.abs(r["g_h"] - g_o).max() / np.abs(g_o).max())}
    out["bitwise_fp64"] = bool(np.array_equal(results["fp64"].get("psi_h"), psi_o)) if "psi_h" in results["fp64"] \
        else None
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    h, rho, bc = load_workload(args.workload)
    from tests.oracle_lib import load_oracle
    threads = load_oracle().oracle_threads()
    samples, iters, shares = [], [], None
    for i in range(args.warmup + args.steps):   # every step one complete FP64 solve
        if i == args.warmup + args.steps - 1:   # the last one with the time of each routine class
            dt, n_outer, shares = oracle_solve_profiled(h, rho, bc)
        else:
            dt, n_outer, _, _ = oracle_solve_timed(h, rho, bc)
        iters.append(n_outer)
        if i >= args.warmup:
            samples.append(dt)
    t_solve = statistics.median(samples)
    value = 1.0 / t_solve
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 6), "unit": "solves/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_solve * 1e3, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": workload_config(args.workload, h, bc),
        "cpu_baseline": {"value": round(value, 6), "unit": "solves/s", "cores": threads, "kind": "port",
                         "sample": f"each step one complete FP64 oracle solve to 1e-10 ({iters[-1]} outer "
                                   f"iterations, g included), median of {len(samples)} after {args.warmup} "
                                   f"warm-up solves; min {min(samples):.2f} s, max {max(samples):.2f} s"},
        "e2e": {"value": round(value, 6), "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_note": "the Fortran/MPI reference cannot be built in this image; the CPU restatement of "
                          "its algorithm (oracle/) is timed",
        "cpu_profile": {"shares": shares, "note": "exclusive wall time of each routine class in the last "
                                                  "step's solve (nested routines counted once)"},
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.single:
        run_single(a)
    else:
        run_ours(a)
