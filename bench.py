#!/usr/bin/env python
"""Benchmark: PBE solve ms and matvec GB/s on B200 (mixed FP32/FP64 vs FP64).

Workload (default): the synthetic protein-like blob — level-6 icosphere
(81 920 flat panels) of radius 22 A displaced radially by seeded real spherical
harmonics of degree <= 8 (15 % amplitude), 2 500 seeded charges uniform inside
(>= 1.5 A from every panel centroid, U[-0.6, 0.6] e shifted to zero net),
eps_in 4, eps_out 80, kappa 0.125 1/A, leaf <= 32 panels, grid 4, FFTSVD
tolerance 1e-4, GMRES tolerance 1e-6.

One step = one complete GMRES solve of A x = b with b resident in HBM
(mixed: FP32 operator inside GMRES, FP64 residual refinement).  L2 is flushed
(256 MiB write on the solve stream) before every timed step.  Prints one JSON
line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config blob|born|large] [--no-cpu-baseline]
"""
from __future__ import annotations

import argparse
import collections
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    # the headline single-solve configuration
    "blob": dict(name="blob L6 (81920 panels, R 22 A, 2500 charges, eps 4/80, kappa 0.125)", kind="blob",
                 level=6, radius=22.0, nq=2500, eps_in=4.0, eps_out=80.0, kappa=0.125, seed=1),
    "born": dict(name="Born ion L5 (20480 panels, R 10 A, +1 e, eps 1/80)", kind="born", level=5, radius=10.0,
                 nq=1, eps_in=1.0, eps_out=80.0, kappa=0.0, seed=0),
    "blob5": dict(name="blob L5 (20480 panels, R 22 A, 2500 charges, eps 4/80, kappa 0.125)", kind="blob",
                  level=5, radius=22.0, nq=2500, eps_in=4.0, eps_out=80.0, kappa=0.125, seed=1),
    "large": dict(name="large blob L7 (327680 panels, R 60 A, 30000 charges, eps 4/80, kappa 0.125)", kind="blob",
                  level=7, radius=60.0, nq=30000, eps_in=4.0, eps_out=80.0, kappa=0.125, seed=3),
    # adjoint forces on the blob system, checked by central differences on seeded atoms
    "adjoint": dict(name="blob L6 (81920 panels, 2500 charges): adjoint dG/dx and dG/dq", kind="blob",
                    level=6, radius=22.0, nq=2500, eps_in=4.0, eps_out=80.0, kappa=0.125, seed=1, fd_atoms=50),
    # adjoint forces on the large blob, central differences on fewer seeded atoms
    "adjoint_large": dict(name="large blob L7 (327680 panels, 30000 charges): adjoint dG/dx and dG/dq", kind="blob",
                          level=7, radius=60.0, nq=30000, eps_in=4.0, eps_out=80.0, kappa=0.125, seed=3,
                          fd_atoms=10),
    # many surfaces: 64 seeded blobs of level 3 to 6 solved concurrently
    "many": dict(name="64 seeded blobs, level 3-6 icospheres (1280-81920 panels), 50-2500 charges", kind="many",
                 surfaces=64, seed=5, eps_in=4.0, eps_out=80.0, kappa=0.125),
    # many right-hand sides: the blob surface with its charges in 256 seeded disjoint groups
    "batch": dict(name="blob L6 (81920 panels), 256 right-hand sides of ~10 charges each", kind="blob",
                  level=6, radius=22.0, nq=2500, eps_in=4.0, eps_out=80.0, kappa=0.125, seed=1, groups=256),
}
SVD_TOL = 1e-4
GMRES_TOL = 1e-6
METRIC = "PBE solve ms & matvec GB/s, 40k-400k panels: mixed vs FP64 GPU at 1e-6 dG err"


def make_workload(cfg, rank=0):
    """The seeded system of a configuration.  Under torchrun every rank solves its own
    system of the same size: rank 0 the configuration's, rank r > 0 the blob of seed
    seed + 100 r (independent work, no replicas of one solve)."""
    from fftsvd_b200 import meshes
    if cfg["kind"] == "born":
        tri, qpos, q = meshes.born_ion(cfg["level"], cfg["radius"])
    else:
        seed = cfg["seed"] + 100 * rank
        tri = meshes.blob(cfg["level"], cfg["radius"], seed=seed)
        qpos, q = meshes.blob_charges(tri, cfg["radius"], cfg["nq"], seed=seed + 1, surface_seed=seed)
    return tri, qpos, q


def golden_ref64(name, tri, qpos, q):
    """The reference FP64 build's results on this system (tests/golden/<name>_ref64.npz,
    written by tests/golden/make_golden_large.py), or None when the fixture is absent or
    was made from other inputs."""
    import hashlib
    path = os.path.join(ROOT, "tests", "golden", name + "_ref64.npz")
    if not os.path.exists(path):
        return None
    g = np.load(path)
    h = hashlib.sha256()
    for a in (tri, qpos, q):
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return g if h.hexdigest() == str(g["inputs_sha256"]) else None


def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.rows = []
        self.gpu = str(gpu_index)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.gpu, f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) > 8:
                for i, nm in enumerate(names):
                    if r[5 + i].lower().startswith("active"):
                        reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def barrier_max(value: float, ws: int) -> float:
    """Max of a per-rank value over all ranks (timings are reported as the slowest rank)."""
    if ws == 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_shares(num_units: int, ws: int):
    """Contiguous, disjoint shares of independent units (surfaces or right-hand sides) per rank."""
    base, extra = divmod(num_units, ws)
    out, start = [], 0
    for r in range(ws):
        cnt = base + (1 if r < extra else 0)
        out.append(range(start, start + cnt))
        start += cnt
    return out


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_reference_solve(tri, qpos, q, cfg, threads):
    """The reference CPU solve (compiled reference, OpenMP) of the same system: ms, iterations, dG."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref
    if not ref.available(False):
        return None
    ref.set_threads(threads)
    t0 = time.time()
    with ref.stdout_to_stderr():
        rs = ref.RefSystem(tri, qpos, q, cfg["eps_in"], cfg["eps_out"], cfg["kappa"], svd_tol=SVD_TOL)
    setup_s = time.time() - t0
    rhs = rs.rhs()
    t1 = time.perf_counter()
    sol, it = rs.solve(rhs, GMRES_TOL)
    solve_ms = (time.perf_counter() - t1) * 1e3
    e = rs.energy(rs.reaction(sol))
    rs.close()
    return dict(solve_ms=solve_ms, iterations=it, dG=e, setup_s=setup_s)


def run_reference(args, cfg, ws, rank):
    if rank != 0:
        return
    tri, qpos, q = make_workload(cfg)
    threads = os.cpu_count() or 1
    steps = max(1, min(args.steps, 2))  # each step is a full CPU solve of tens of seconds
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref
    if not ref.available(False):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libfftsvd_ref.so is not built"}))
        return
    ref.set_threads(threads)
    with ref.stdout_to_stderr():
        rs = ref.RefSystem(tri, qpos, q, cfg["eps_in"], cfg["eps_out"], cfg["kappa"], svd_tol=SVD_TOL)
    rhs = rs.rhs()
    times = []
    it = 0
    for _ in range(steps):
        t0 = time.perf_counter()
        sol, it = rs.solve(rhs, GMRES_TOL)
        times.append((time.perf_counter() - t0) * 1e3)
    ms = float(np.mean(times))
    e = rs.energy(rs.reaction(sol))
    sample = f"full GMRES solve to {GMRES_TOL} of the same system per step ({it} iterations), operator setup excluded"
    line = {"metric": METRIC, "value": ms, "unit": "ms", "n_gpus": args.gpus, "steps": steps, "warmup": 0,
            "ms_per_step": ms, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": cfg["name"], "svd_tol": SVD_TOL, "gmres_tol": GMRES_TOL,
                       "panels": len(tri), "charges": len(q)},
            "cpu_baseline": {"value": ms, "unit": "ms", "cores": threads, "kind": "reference", "sample": sample},
            "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "iterations": it, "dG_kcal": e}
    print(json.dumps(line), flush=True)


def _time_solves(s, stream, flush, rhs, sol, precision, k, warm):
    """k timed solves (CUDA events on the library stream, L2 flushed before each) after
    warm untimed ones: total ms and the last solve's info."""
    import torch
    for _ in range(warm):
        s.solve_device(rhs.data_ptr(), sol.data_ptr(), precision, GMRES_TOL)
    total, info = 0.0, None
    for _ in range(k):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        info = s.solve_device(rhs.data_ptr(), sol.data_ptr(), precision, GMRES_TOL)
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    return total, info


def _setup_stats(s):
    from fftsvd_b200 import _abi
    from fftsvd_b200.lib import load
    st = _abi.SurfaceStats()
    load().fftsvd_b200_surface_stats(s._h, C.byref(st))
    return st


def smem_roofline(smem_bytes, ms, sm_count, sm_mhz):
    """The translation stage against the shared-memory bandwidth of the SMs."""
    mhz = sm_mhz or 1965.0
    peak = sm_count * 128.0 * mhz * 1e6 / 1e9  # GB/s
    ach = smem_bytes / (ms * 1e6) if ms > 0 else None
    return {"kernel": "translate", "bytes_per_launch": smem_bytes, "achieved": ach, "peak": peak, "unit": "GB/s",
            "frac": ach / peak if ach else None,
            "peak_kind": f"nominal: 128 bytes per clock per SM x {sm_count} SMs at {mhz:.0f} MHz"}


def _ref64_errors(g, e_mixed, e64):
    if g is None:
        return None
    r = float(g["dG"])
    return {"dG_ref_fp64": r, "dG_ref_fp64_converged": float(g["dG_tight"]),
            "mixed": abs(e_mixed - r) / abs(r), "fp64": abs(e64 - r) / abs(r),
            "mixed_vs_converged": abs(e_mixed - float(g["dG_tight"])) / abs(float(g["dG_tight"]))}


def run_large(flush, steps, warmup):
    """The 327 680-panel blob (30 000 charges): mixed and FP64 solve times, their ratio and
    their energies against the reference FP64 build (committed fixture)."""
    import torch
    from fftsvd_b200.lib import load
    from fftsvd_b200.surface import Surface
    cfg = CONFIGS["large"]
    tri, qpos, q = make_workload(cfg)
    t0 = time.time()
    s = Surface.from_problem(tri, qpos, q, cfg["eps_in"], cfg["eps_out"], cfg["kappa"], svd_tol=SVD_TOL)
    setup_s = time.time() - t0
    st = _setup_stats(s)
    stream = torch.cuda.ExternalStream(load().fftsvd_b200_surface_stream(s._h))
    rhs = torch.empty(s.n, dtype=torch.float64, device="cuda")
    s.rhs_device(rhs.data_ptr())
    sol = torch.empty_like(rhs)
    torch.cuda.synchronize()
    tm, im = _time_solves(s, stream, flush, rhs, sol, "mixed", steps, warmup)
    em = s.energy(s.reaction_potentials(sol.cpu().numpy()))
    k64 = max(1, steps // 2)
    t64, i64 = _time_solves(s, stream, flush, rhs, sol, "fp64", k64, 1)
    e64 = s.energy(s.reaction_potentials(sol.cpu().numpy()))
    out = {"workload": cfg["name"], "panels": len(tri), "charges": len(q), "steps": steps,
           "mixed_ms": tm / steps, "fp64_ms": t64 / k64, "speedup_mixed_vs_fp64": (t64 / k64) / (tm / steps),
           "iterations_mixed": im.iterations, "refinements_mixed": im.refinements, "iterations_fp64": i64.iterations,
           "dG_kcal_mixed": em, "dG_kcal_fp64": e64, "dG_rel_err_mixed_vs_fp64": abs(em - e64) / abs(e64),
           "dG_rel_err_vs_ref_fp64": _ref64_errors(golden_ref64("blob7", tri, qpos, q), em, e64),
           "setup_s": setup_s, "setup_stage_ms": list(st.setup_ms)}
    # the batched solve at this end of the panel range: 256 charge groups as one block GMRES
    del rhs, sol
    out["batched_256_rhs"] = run_block256(s, qpos, q, cfg, flush, t64 / k64)
    s.close()
    return out


def group_single_solve_ms(s, stream, R, precision, groups=(0, 64, 128, 192), reps=2):
    """Mean time of one plain single solve of a charge group's right-hand side, over a few
    groups (a group's system converges in fewer iterations than the whole charge set's)."""
    import torch
    one = torch.empty_like(R[0])
    sol = torch.empty_like(one)
    total = 0.0
    for gi in groups:
        one.copy_(R[gi % R.shape[0]])
        s.solve_device(one.data_ptr(), sol.data_ptr(), precision, GMRES_TOL)  # warm-up
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            s.solve_device(one.data_ptr(), sol.data_ptr(), precision, GMRES_TOL)
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1) / reps
    return total / len(groups)


def run_block256(s, qpos, q, cfg, flush, fp64_single_ms):
    """The blob's charges in 256 seeded disjoint groups, one right-hand side per group,
    solved as one block GMRES (mixed precision) on the same surface; against 256 plain
    FP64 single solves of group right-hand sides (mean over four groups)."""
    import torch
    from fftsvd_b200.lib import load
    groups = 256
    perm, gptr = charge_groups(len(q), groups, cfg["seed"])
    s.set_charges(qpos[perm], q[perm])
    stream = torch.cuda.ExternalStream(load().fftsvd_b200_surface_stream(s._h))
    R = torch.empty((groups, s.n), dtype=torch.float64, device="cuda")
    S = torch.empty_like(R)
    s.rhs_groups_device(gptr, R.data_ptr())
    s.solve_block_device(R.data_ptr(), S.data_ptr(), groups, "mixed", GMRES_TOL, 150)  # warm-up
    with torch.cuda.stream(stream):
        flush.fill_(1.0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    info = s.solve_block_device(R.data_ptr(), S.data_ptr(), groups, "mixed", GMRES_TOL, 150)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    group_fp64_ms = group_single_solve_ms(s, stream, R, "fp64")
    s.set_charges(qpos, q)
    return {"workload": f"{cfg['name']}, charges in {groups} seeded groups", "right_hand_sides": groups,
            "block_mixed_ms": ms, "ms_per_rhs": ms / groups, "fp64_single_group_solve_ms": group_fp64_ms,
            "speedup_vs_fp64_single_solves": group_fp64_ms * groups / ms,
            "fp64_single_solve_ms_all_charges": fp64_single_ms,
            "block_steps_max": max(info[c].iterations for c in range(groups))}


def run_ours(args, cfg, ws, rank, local):
    import torch
    from fftsvd_b200 import _abi
    from fftsvd_b200.lib import load
    from fftsvd_b200.surface import Surface

    torch.cuda.set_device(local)
    torch.zeros(1, device="cuda")  # the CUDA context exists before the setup is timed
    lib = load()
    tri, qpos, q = make_workload(cfg, rank)
    t0 = time.time()
    s = Surface.from_problem(tri, qpos, q, cfg["eps_in"], cfg["eps_out"], cfg["kappa"], svd_tol=SVD_TOL)
    setup_s = time.time() - t0
    st = _setup_stats(s)
    n = s.n
    stream = torch.cuda.ExternalStream(lib.fftsvd_b200_surface_stream(s._h))
    rhs = torch.empty(n, dtype=torch.float64, device="cuda")
    s.rhs_device(rhs.data_ptr())
    torch.cuda.synchronize()
    sol = torch.empty_like(rhs)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > L2

    barrier(ws)
    torch.cuda.synchronize()
    launches0 = lib.fftsvd_b200_launch_count()
    with ClockSampler(local) as clk:
        t_mixed, info_mixed = _time_solves(s, stream, flush, rhs, sol, "mixed", args.steps, args.warmup)
    launches = lib.fftsvd_b200_launch_count() - launches0
    torch.cuda.synchronize()
    barrier(ws)
    t_max = barrier_max(t_mixed, ws)
    ms_per_step = t_max / args.steps
    value = t_max / (args.steps * ws)  # ws independent systems solved per step
    x_mixed = sol.cpu().numpy()

    # plain FP64 GPU solve of the same system (the comparison the target is stated against)
    k64 = max(1, args.steps // 2)
    t64, info64 = _time_solves(s, stream, flush, rhs, sol, "fp64", k64, 1)
    x64 = sol.cpu().numpy()
    fp64_ms = t64 / k64
    e_mixed = s.energy(s.reaction_potentials(x_mixed))
    e64 = s.energy(s.reaction_potentials(x64))
    ref64 = _ref64_errors(golden_ref64("blob6", tri, qpos, q) if cfg is CONFIGS["blob"] and rank == 0 else None,
                          e_mixed, e64)

    # matvec: per-kernel CUDA-event times on the library stream, algorithmic bytes per kernel
    xv = torch.randn(n, dtype=torch.float64, device="cuda")
    yv = torch.empty_like(xv)
    kernels = ["join", "far_forward", "translate", "far_backward", "near"]
    prof = {}
    for prec, pid in (("fp32", _abi.PREC_FP32), ("fp64", _abi.PREC_FP64)):
        ms5 = (C.c_double * 5)()
        b5 = (C.c_double * 5)()
        lib.fftsvd_b200_profile_matvec(s._h, pid, C.c_void_p(xv.data_ptr()), C.c_void_p(yv.data_ptr()), 3, ms5)
        lib.fftsvd_b200_profile_matvec(s._h, pid, C.c_void_p(xv.data_ptr()), C.c_void_p(yv.data_ptr()), 20, ms5)
        lib.fftsvd_b200_matvec_kernel_bytes(s._h, pid, b5)
        prof[prec] = {k: {"ms": ms5[i], "bytes": b5[i], "gbs": b5[i] / (ms5[i] * 1e6) if ms5[i] > 0 else None}
                      for i, k in enumerate(kernels)}
        prof[prec]["total_ms"] = sum(ms5[i] for i in range(5))
    mv_bytes32 = st.matvec_bytes_fp32
    mv_bytes64 = st.matvec_bytes_fp64
    # matvec as the solver issues it (grid-size chains and the near field on concurrent streams)
    mv_streams = {}
    for prec in ("fp32", "fp64"):
        for _ in range(3):
            s.matvec_device(xv.data_ptr(), yv.data_ptr(), prec)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(20):
            s.matvec_device(xv.data_ptr(), yv.data_ptr(), prec)
        e1.record(stream)
        e1.synchronize()
        mv_streams[prec] = e0.elapsed_time(e1) / 20

    # e2e through the host-pointer C-ABI (pinned host buffers, copies inside the timed region)
    rhs_h = torch.empty(n, dtype=torch.float64, pin_memory=True)
    sol_h = torch.empty(n, dtype=torch.float64, pin_memory=True)
    rhs_h.copy_(rhs.cpu())
    infoC = _abi.SolveInfo()
    e2e_total = 0.0
    for i in range(args.warmup + args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = lib.fftsvd_b200_solve(s._h, _abi.PREC_MIXED, C.c_void_p(rhs_h.data_ptr()), C.c_void_p(sol_h.data_ptr()),
                                   GMRES_TOL, 1000, C.byref(infoC))
        e1.record(stream)
        e1.synchronize()
        if rc != 0:
            raise RuntimeError(f"solve failed: {rc}")
        if i >= args.warmup:
            e2e_total += e0.elapsed_time(e1)
    e2e_ms = barrier_max(e2e_total, ws) / (args.steps * ws)

    # roofline of the dominant kernel of the mixed solve's matvec (FP32 operator)
    peak, peak_kind = hbm_peak()
    dom = max(kernels, key=lambda k: prof["fp32"][k]["ms"])
    ach = prof["fp32"][dom]["gbs"]
    # the translation's own bound: shared-memory bytes it moves over the SMs' shared-memory
    # bandwidth (128 bytes per clock per SM, at the SM clock sampled during the timed region)
    smem_b = C.c_double()
    lib.fftsvd_b200_translate_smem_bytes(s._h, _abi.PREC_FP32, C.byref(smem_b))
    sm_count = torch.cuda.get_device_properties(local).multi_processor_count
    # DRAM traffic of that stage per matvec, from the ncu capture summarised in profiles/
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "translate_dram_blob_l6.md")
    key = cfg["kind"] + str(cfg.get("level", ""))
    if os.path.exists(tpath):
        for line in open(tpath):
            cells = [c.strip() for c in line.strip().strip("|").split("|")]
            if len(cells) == 3 and cells[0] == key and cells[1] == dom and cells[2].isdigit():
                traffic = float(cells[2])

    # the other end of the metric's panel range and the batched solve: one GPU only
    extras = ws == 1 and cfg is CONFIGS["blob"] and not args.no_extras
    large = run_large(flush, max(3, args.steps // 4), 2) if extras else None
    block = run_block256(s, qpos, q, cfg, flush, fp64_ms) if extras else None

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        r = cpu_reference_solve(tri, qpos, q, cfg, threads)
        if r is not None:
            cpu = {"value": r["solve_ms"], "unit": "ms", "cores": threads, "kind": "reference",
                   "sample": f"the reference's full GMRES solve of the same system ({r['iterations']} iterations, "
                             f"setup {r['setup_s']:.0f} s excluded), OpenMP build, dG {r['dG']:.6f} kcal/mol"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "ms", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": cfg["name"], "panels": len(tri), "charges": len(q), "svd_tol": SVD_TOL,
                       "gmres_tol": GMRES_TOL, "precision": "FP32 operator, FP64 Krylov + FP64 refinement",
                       "l2": "flushed before every timed step (256 MiB write)",
                       "parallelism": "one system per GPU" if ws == 1 else
                                      f"{ws} independent seeded systems of this size, one per GPU",
                       "depth": list(st.depth), "leaves": list(st.num_leaves), "far_cubes": list(st.num_cubes)},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak if ach else None, "traffic": traffic, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": prof["fp32"][dom]["bytes"],
                         "smem": smem_roofline(smem_b.value, prof["fp32"]["translate"]["ms"], sm_count,
                                               clk.summary().get("sm_mhz"))},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "fp64_solve_ms": fp64_ms, "speedup_mixed_vs_fp64": fp64_ms / (t_mixed / args.steps),
            "iterations_mixed": info_mixed.iterations, "refinements_mixed": info_mixed.refinements,
            "iterations_fp64": info64.iterations,
            "dG_kcal_mixed": e_mixed, "dG_kcal_fp64": e64, "dG_rel_err_mixed_vs_fp64": abs(e_mixed - e64) / abs(e64),
            "dG_rel_err_vs_ref_fp64": ref64,
            "matvec_ms_fp32": prof["fp32"]["total_ms"], "matvec_ms_fp64": prof["fp64"]["total_ms"],
            "matvec_ms_fp32_streams": mv_streams["fp32"], "matvec_ms_fp64_streams": mv_streams["fp64"],
            "matvec_gbs_fp32": mv_bytes32 / (prof["fp32"]["total_ms"] * 1e6),
            "matvec_gbs_fp64": mv_bytes64 / (prof["fp64"]["total_ms"] * 1e6),
            "matvec_kernels": prof, "setup_s": setup_s, "setup_stage_ms": list(st.setup_ms),
            "large": large, "batched_256_rhs": block,
        }
        print(json.dumps(line), flush=True)
    s.close()


def charge_groups(num_charges, groups, seed):
    """Seeded disjoint charge groups of nearly equal size: a permutation of the charges
    (group members contiguous after it) and the group offsets."""
    rng = np.random.default_rng(seed + 1000)
    perm = rng.permutation(num_charges)
    base, extra = divmod(num_charges, groups)
    sizes = [base + (1 if g < extra else 0) for g in range(groups)]
    gptr = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    return perm, gptr


def run_batch(args, cfg, ws, rank, local):
    """Batched solve: every charge group's right-hand side in one block GMRES (one Krylov
    space shared by the groups, mixed precision), groups sharded over ranks; beside it the
    block FP64 solve, the lockstep batch (each column its own Krylov basis) in both
    precisions and one FP64 solve alone."""
    import torch
    from fftsvd_b200.lib import load
    from fftsvd_b200.surface import Surface

    torch.cuda.set_device(local)
    lib = load()
    tri, qpos, q = make_workload(cfg)
    perm, gptr = charge_groups(len(q), cfg["groups"], cfg["seed"])
    qpos, q = qpos[perm], q[perm]
    s = Surface.from_problem(tri, qpos, q, cfg["eps_in"], cfg["eps_out"], cfg["kappa"], svd_tol=SVD_TOL)
    n = s.n
    mine = replica_shares(cfg["groups"], ws)[rank]
    sub = gptr[mine.start:mine.stop + 1].astype(np.int32)
    k = len(sub) - 1
    stream = torch.cuda.ExternalStream(lib.fftsvd_b200_surface_stream(s._h))
    R = torch.empty((k, n), dtype=torch.float64, device="cuda")
    S = torch.empty_like(R)
    s.rhs_groups_device(sub, R.data_ptr())
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > L2
    maxit = 150

    def timed(solve, precision, steps, warm, tol=GMRES_TOL):
        for _ in range(warm):
            solve(R.data_ptr(), S.data_ptr(), k, precision, tol, maxit)
        total, info = 0.0, None
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            info = solve(R.data_ptr(), S.data_ptr(), k, precision, tol, maxit)
            e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
        return total / steps, info

    torch.cuda.synchronize()
    barrier(ws)
    warm = max(1, args.warmup - 2)
    launches0 = lib.fftsvd_b200_launch_count()
    with ClockSampler(local) as clk:
        t_block, info_b = timed(s.solve_block_device, "mixed", args.steps, warm)
    launches = (lib.fftsvd_b200_launch_count() - launches0) // (args.steps + warm)
    torch.cuda.synchronize()
    barrier(ws)
    t_max = barrier_max(t_block, ws)
    e_block = s.group_energies_device(sub, S.data_ptr())
    t_block64, info_b64 = timed(s.solve_block_device, "fp64", 1, 0)
    e_block64 = s.group_energies_device(sub, S.data_ptr())
    t_lock, info_m = timed(s.solve_batch_device, "mixed", 1, 0)
    e_lock = s.group_energies_device(sub, S.data_ptr())
    t_lock64, _ = timed(s.solve_batch_device, "fp64", 1, 0)
    e64 = s.group_energies_device(sub, S.data_ptr())
    # converged FP64 energies (block FP64 GMRES to 1e-10) as the reference of the errors
    timed(s.solve_block_device, "fp64", 1, 0, tol=1e-10)
    e_conv = s.group_energies_device(sub, S.data_ptr())

    def errs(e):
        v = [abs(a - b) / abs(b) for a, b in zip(e, e_conv) if b != 0.0]
        return max(v) if v else None

    # right-hand sides solved alone (same surface, same kernels), both precisions: mean over
    # four groups
    single = {prec: group_single_solve_ms(s, stream, R, prec) for prec in ("mixed", "fp64")}
    if rank == 0:
        its = [info_m[c].iterations for c in range(k)]
        bits = [info_b[c].iterations for c in range(k)]
        line = {
            "metric": f"batched mixed-precision PBE solve ms ({cfg['groups']} charge-group right-hand sides)",
            "value": t_max, "unit": "ms", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_max, "higher_is_better": False, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32 operator, f64 Krylov vectors and refinement", "data": "synthetic",
            "config": {"workload": cfg["name"], "groups": cfg["groups"], "rhs_per_rank": k, "gmres_tol": GMRES_TOL,
                       "svd_tol": SVD_TOL, "solver": "block GMRES, one Krylov space for the block of groups",
                       "l2": "256 MiB buffer written between timed solves"},
            "ms_per_rhs": t_max / k, "block_fp64_ms": t_block64, "lockstep_mixed_ms": t_lock,
            "lockstep_fp64_ms": t_lock64, "single_solve_mixed_ms": single["mixed"],
            "single_solve_fp64_ms": single["fp64"],
            "speedup_vs_fp64_single_solves": single["fp64"] * k / t_max,
            "speedup_vs_lockstep_fp64": t_lock64 / t_max, "speedup_vs_lockstep_mixed": t_lock / t_max,
            "dG_rel_err_vs_converged_fp64_max": {"block_mixed": errs(e_block), "block_fp64": errs(e_block64),
                                                 "lockstep_mixed": errs(e_lock), "lockstep_fp64": errs(e64)},
            "block_steps_mixed_max": max(bits), "block_steps_fp64_max": max(info_b64[c].iterations for c in range(k)),
            "lockstep_iterations_mixed_max": max(its), "lockstep_iterations_mixed_mean": sum(its) / len(its),
            "gpu_launches": launches, "clocks": clk.summary(),
        }
        print(json.dumps(line))
    s.close()


def run_adjoint(args, cfg, ws, rank, local):
    """Energy derivatives by one forward and one transposed solve (mixed precision), timed
    on the device; central differences (FP64 solves, h = 1e-4 A / 1e-4 e) on seeded atoms."""
    import torch
    from fftsvd_b200.lib import load
    from fftsvd_b200.surface import Surface

    torch.cuda.set_device(local)
    lib = load()
    tri, qpos, q = make_workload(cfg)
    s = Surface.from_problem(tri, qpos, q, cfg["eps_in"], cfg["eps_out"], cfg["kappa"], svd_tol=SVD_TOL)
    stream = torch.cuda.ExternalStream(lib.fftsvd_b200_surface_stream(s._h))
    for _ in range(max(1, args.warmup - 2)):
        s.adjoint(precision="mixed", tol=GMRES_TOL)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        total = 0.0
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            e, dq, dx, info = s.adjoint(precision="mixed", tol=GMRES_TOL)
            e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
    ms = barrier_max(total / args.steps, ws)
    # FP64 adjoint to the finite differences' tolerance, and the differences themselves
    tol_fd = 1e-12  # energy noise ~1e-12 |dG|: far below the differences over 2h = 2e-4 A
    e64, dq64, dx64, _ = s.adjoint(precision="fp64", tol=tol_fd)

    def energy(pos, chg):
        s.set_charges(pos, chg)
        sol = s.solve(s.rhs(), precision="fp64", tol=tol_fd).solution
        return s.energy(s.reaction_potentials(sol))

    rng = np.random.default_rng(cfg["seed"] + 2000)
    atoms = rng.choice(len(q), size=min(cfg["fd_atoms"], len(q)), replace=False)
    h = 1e-4
    fscale = np.abs(dx64).max()
    errx, errq = [], []
    for j in atoms:
        for a in range(3):
            p, m = qpos.copy(), qpos.copy()
            p[j, a] += h
            m[j, a] -= h
            fd = (energy(p, q) - energy(m, q)) / (2 * h)
            errx.append(abs(dx64[j, a] - fd) / max(abs(fd), 1e-2 * fscale))
        qp, qm = q.copy(), q.copy()
        qp[j] += h
        qm[j] -= h
        fdq = (energy(qpos, qp) - energy(qpos, qm)) / (2 * h)
        errq.append(abs(dq64[j] - fdq) / abs(fdq))
    # the worst component again at half and twice the step: an error growing like 1/h is a
    # jump of the discrete energy (a collection integral changing formula between x-h and x+h)
    worst = int(np.argmax(errx))
    wj, wa = atoms[worst // 3], worst % 3
    step_err = {}
    for hh in (h / 2, h, 2 * h):
        p, m = qpos.copy(), qpos.copy()
        p[wj, wa] += hh
        m[wj, wa] -= hh
        fd = (energy(p, q) - energy(m, q)) / (2 * hh)
        step_err[f"{hh:g}"] = abs(dx64[wj, wa] - fd)
    s.set_charges(qpos, q)
    if rank == 0:
        line = {
            "metric": "adjoint dG/dx and dG/dq ms (forward and transposed mixed-precision solves + derivative kernels)",
            "value": ms, "unit": "ms", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 operator, f64 Krylov vectors, refinement and derivative kernels", "data": "synthetic",
            "config": {"workload": cfg["name"], "charges": len(q), "gmres_tol": GMRES_TOL, "svd_tol": SVD_TOL,
                       "fd_atoms": len(atoms), "fd_step": h, "fd_solver_tol": tol_fd},
            "iterations_forward": info[0].iterations, "iterations_adjoint": info[1].iterations,
            "dG_kcal": e, "dG_rel_err_mixed_vs_fp64": abs(e - e64) / abs(e64),
            "force_rel_err_mixed_vs_fp64": float(np.abs(dx - dx64).max() / fscale),
            "fd_max_rel_err_dG_dx": max(errx), "fd_median_rel_err_dG_dx": float(np.median(errx)),
            "fd_max_rel_err_dG_dq": max(errq),
            "fd_worst_component": {"atom": int(wj), "axis": int(wa), "force": float(dx64[wj, wa]),
                                   "abs_err_by_step": step_err},
            "max_force_kcal_per_A": float(fscale), "clocks": clk.summary(),
        }
        print(json.dumps(line))
    s.close()


MANY_LEVELS = {3: (8.0, 50), 4: (12.0, 200), 5: (16.0, 800), 6: (22.0, 2500)}  # level -> (radius A, charges)


def run_many(args, cfg, ws, rank, local):
    """Independent surfaces: the same set solved one after another and through one
    fftsvd_b200_solve_many call (host threads, per-surface streams); surfaces sharded
    over ranks."""
    import torch
    from fftsvd_b200.lib import load
    from fftsvd_b200.surface import Surface, solve_many

    torch.cuda.set_device(local)
    lib = load()
    rng = np.random.default_rng(cfg["seed"])
    levels = rng.choice([3, 4, 5, 6], size=cfg["surfaces"], p=[0.4, 0.3, 0.2, 0.1])
    mine = replica_shares(cfg["surfaces"], ws)[rank]
    surfs, rhs, sols, panels = [], [], [], 0
    t0 = time.time()
    for i in mine:
        lv = int(levels[i])
        radius, nq = MANY_LEVELS[lv]
        sub = dict(kind="blob", level=lv, radius=radius, nq=nq, seed=cfg["seed"] * 1000 + i)
        tri, qpos, q = make_workload(sub)
        s = Surface.from_problem(tri, qpos, q, cfg["eps_in"], cfg["eps_out"], cfg["kappa"], svd_tol=SVD_TOL)
        surfs.append(s)
        r = torch.empty(s.n, dtype=torch.float64, device="cuda")
        s.rhs_device(r.data_ptr())
        rhs.append(r)
        sols.append(torch.empty_like(r))
        panels += len(tri)
    setup_s = time.time() - t0
    # translation tile shapes per surface from the autotuner (launch shapes only: same results)
    t1 = time.time()
    tuned = [s.autotune() for s in surfs]
    tune_s = time.time() - t1
    torch.cuda.synchronize()

    def sequential(precision):
        total = 0.0
        for s, r, x in zip(surfs, rhs, sols):
            st = torch.cuda.ExternalStream(lib.fftsvd_b200_surface_stream(s._h))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            s.solve_device(r.data_ptr(), x.data_ptr(), precision, GMRES_TOL)
            e1.record(st)
            e1.synchronize()
            total += e0.elapsed_time(e1)
        return total

    def concurrent(precision):
        torch.cuda.synchronize()
        t = time.perf_counter()
        info = solve_many(surfs, [r.data_ptr() for r in rhs], [x.data_ptr() for x in sols], precision, GMRES_TOL)
        torch.cuda.synchronize()
        return (time.perf_counter() - t) * 1e3, info

    for _ in range(max(1, args.warmup - 2)):
        concurrent("mixed")
    seq_ms = sequential("mixed")
    barrier(ws)
    with ClockSampler(local) as clk:
        runs = [concurrent("mixed")[0] for _ in range(args.steps)]
    conc_ms = barrier_max(sum(runs) / len(runs), ws)
    e_mixed = [s.energy(s.reaction_potentials(x.cpu().numpy())) for s, x in zip(surfs, sols)]
    conc64, _ = concurrent("fp64")
    e64 = [s.energy(s.reaction_potentials(x.cpu().numpy())) for s, x in zip(surfs, sols)]
    errs = [abs(a - b) / abs(b) for a, b in zip(e_mixed, e64) if b != 0.0]
    if rank == 0:
        line = {
            "metric": f"many-surface PBE solve ms ({cfg['surfaces']} surfaces, mixed precision)",
            "value": conc_ms, "unit": "ms", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": conc_ms, "higher_is_better": False, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32 operator, f64 Krylov vectors and refinement", "data": "synthetic",
            "config": {"workload": cfg["name"], "surfaces_per_rank": len(surfs), "panels_per_rank": panels,
                       "levels": [int(levels[i]) for i in mine], "gmres_tol": GMRES_TOL, "svd_tol": SVD_TOL,
                       "timing": "host clock around one fftsvd_b200_solve_many call (it returns after every solve)"},
            "sequential_ms": seq_ms, "concurrency_speedup": seq_ms / conc_ms, "fp64_ms": conc64,
            "speedup_mixed_vs_fp64": conc64 / conc_ms, "dG_rel_err_mixed_vs_fp64_max": max(errs) if errs else None,
            "setup_s": setup_s, "autotune_s": tune_s,
            "autotune_chosen_fp32": collections.Counter(str(t["candidates"][t["chosen_fp32"]]) for t in tuned),
            "clocks": clk.summary(),
        }
        print(json.dumps(line))
    for s in surfs:
        s.close()


def run_matvec_only(args, cfg, local):
    """Build the surface and run `--reps` FP32 and FP64 matvecs (for profiler captures)."""
    import torch
    from fftsvd_b200.surface import Surface

    torch.cuda.set_device(local)
    tri, qpos, q = make_workload(cfg)
    s = Surface.from_problem(tri, qpos, q, cfg["eps_in"], cfg["eps_out"], cfg["kappa"], svd_tol=SVD_TOL)
    k = 64 if "groups" in cfg else 1  # batched configuration: a 64-column multi-vector matvec
    x = torch.randn((k, s.n), dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    for prec in ("fp32", "fp64"):
        for _ in range(args.reps):
            if k > 1:
                s.matvec_batch_device(x.data_ptr(), y.data_ptr(), k, prec)
            else:
                s.matvec_device(x.data_ptr(), y.data_ptr(), prec)
    torch.cuda.synchronize()
    print(json.dumps({"matvec_only": cfg["name"], "reps": args.reps, "norm": float(y.norm())}))
    s.close()


def run_capture(args, cfg, local):
    """Build the surface and run one part of the workload for a profiler capture:
    `gmres` = right-hand side, 12 steps of an FP64 GMRES solve and the reaction potentials;
    `transpose` = one FP32 transposed matvec (the adjoint's operator);
    `block` = one mixed-precision block GMRES solve of the charge groups' right-hand sides
    (configurations with groups);
    `near_tc` = two 128-column FP32 multi-vector matvecs with the tensor-core near field."""
    import ctypes as C

    import torch
    from fftsvd_b200 import _abi
    from fftsvd_b200.lib import load
    from fftsvd_b200.surface import Surface

    torch.cuda.set_device(local)
    tri, qpos, q = make_workload(cfg)
    if args.capture == "block":
        perm, gptr = charge_groups(len(q), cfg["groups"], cfg["seed"])
        qpos, q = qpos[perm], q[perm]
    s = Surface.from_problem(tri, qpos, q, cfg["eps_in"], cfg["eps_out"], cfg["kappa"], svd_tol=SVD_TOL)
    x = torch.randn(s.n, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    if args.capture == "block":
        k = cfg["groups"]
        R = torch.empty((k, s.n), dtype=torch.float64, device="cuda")
        S = torch.empty_like(R)
        s.rhs_groups_device(gptr.astype(np.int32), R.data_ptr())
        info = s.solve_block_device(R.data_ptr(), S.data_ptr(), k, "mixed", GMRES_TOL, 150)
        torch.cuda.synchronize()
        passes = collections.Counter(info[c].refinements for c in range(k))
        steps = collections.Counter(info[c].iterations for c in range(k))
        print(json.dumps({"capture": "block", "workload": cfg["name"], "solve_ms": info[0].solve_ms,
                          "passes": dict(passes), "block_steps": dict(steps),
                          "residual_max": max(info[c].residual for c in range(k))}))
        s.close()
        return
    if args.capture == "near_tc":
        k = 128
        X = torch.randn((k, s.n), dtype=torch.float64, device="cuda")
        Y = torch.empty_like(X)
        lib = load()
        for _ in range(2):
            rc = lib.fftsvd_b200_matvec_batch_tensor_device(s._h, k, C.c_void_p(X.data_ptr()),
                                                            C.c_void_p(Y.data_ptr()))
            if rc != 0:
                raise RuntimeError(lib.fftsvd_b200_last_error().decode())
        torch.cuda.synchronize()
        print(json.dumps({"capture": "near_tc", "workload": cfg["name"], "nrhs": k, "norm": float(Y.norm())}))
        s.close()
        return
    if args.capture == "gmres":
        s.rhs_device(x.data_ptr())
        info = _abi.SolveInfo()
        load().fftsvd_b200_solve_device(s._h, _abi.PREC_FP64, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                        GMRES_TOL, 12, C.byref(info))  # stops at the cap: a capture, not a solve
        phi = torch.empty(len(q), dtype=torch.float64, device="cuda")
        s.reaction_potentials_device(y.data_ptr(), phi.data_ptr())
    else:
        load().fftsvd_b200_matvec_transpose_device(s._h, _abi.PREC_FP32, C.c_void_p(x.data_ptr()),
                                                   C.c_void_p(y.data_ptr()))
    torch.cuda.synchronize()
    print(json.dumps({"capture": args.capture, "workload": cfg["name"], "norm": float(y.norm())}))
    s.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--matvec-only", action="store_true", help="only run --reps matvecs (profiling)")
    ap.add_argument("--capture", choices=["gmres", "transpose", "block", "near_tc"], default=None,
                    help="only run one part of the workload (profiling)")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=list(CONFIGS), default="blob")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the large-blob and 256-right-hand-side sections of the default line")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    cfg = CONFIGS[args.config]
    ws, rank, local = dist_init()
    try:
        if args.matvec_only:
            run_matvec_only(args, cfg, local)
        elif args.capture:
            run_capture(args, cfg, local)
        elif args.impl == "reference":
            run_reference(args, cfg, ws, rank)
        elif cfg.get("kind") == "many":
            run_many(args, cfg, ws, rank, local)
        elif "groups" in cfg:
            run_batch(args, cfg, ws, rank, local)
        elif "fd_atoms" in cfg:
            run_adjoint(args, cfg, ws, rank, local)
        else:
            run_ours(args, cfg, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
