#!/usr/bin/env python
"""HMC trajectories/hour at L=48, Ltau=480 (mixed precision) on B200.

One step = one HMC trajectory (Metropolis update) of every chain: 20 leapfrog
steps of size 0.05, dtau = 0.1, J = K = 1, PCG on M^dag M to relative residual
1e-10 (float iterations, double reliable updates every <= 50 iterations), the
reference's physical start (staggered pi-flux +-pi/4 plus Gaussian noise).
The line also reports, measured in the same run: the plain FP64 path's
trajectories/hour, Delta H of one shared trajectory in both precisions, the
M^dag M matvec bandwidth, and the roofline of the dominant kernel (the
persistent PCG).  ``--impl reference`` times the CPU restatement of the
reference's path (the oracle) on the host cores instead.

Multi-GPU (torchrun): replicas only -- every rank runs its own chains, no
data-path collective; the timed region is bracketed by barriers and the
maximum over ranks is reported.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "HMC trajectories/hour at L=48, Ltau=480 (mixed precision, Delta H checked against FP64)"
UNIT = "trajectories/hour"
# DRAM bytes (read + write) per site and PCG iteration of k_pcg on this
# workload, mixed precision, 2 right-hand sides: ncu --metrics
# dram__bytes_read.sum,dram__bytes_write.sum of `bench.py --solve-only 482`
PCG_DRAM_BYTES_PER_SITE_ITER = 72.7
# PCG iterations per solve of this workload (mixed, rtol 1e-10) as the GPU run
# measures them: the CPU arms' fallback when they run neither a GPU solve nor
# their own trajectory
CG_ITERS_PER_SOLVE = 482


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--prewarm-seconds", type=float, default=10.0,
                    help="untimed solver runs on a scratch right-hand side before the warm-up "
                         "trajectories (brings an idle GPU to steady state; the sampler's random "
                         "state is untouched, so the timed trajectories stay the same)")
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--L", type=int, default=48)
    ap.add_argument("--Ltau", type=int, default=480)
    ap.add_argument("--bs", type=int, default=2, help="chains per GPU")
    ap.add_argument("--n-leapfrog", type=int, default=20)
    ap.add_argument("--delta-t", type=float, default=0.05)
    ap.add_argument("--rtol", type=float, default=1e-10)
    ap.add_argument("--fp64-steps", type=int, default=5, help="trajectories timed on the plain FP64 path")
    ap.add_argument("--bf16-steps", type=int, default=5,
                    help="trajectories timed with the PCG's vectors stored as bf16 (mixed arithmetic)")
    ap.add_argument("--f16-steps", type=int, default=5,
                    help="trajectories timed with the PCG's vectors stored as scaled fp16 (mixed arithmetic)")
    ap.add_argument("--options-steps", type=int, default=5,
                    help="trajectories timed with fp16 storage, chronological guesses and graph replay together")
    ap.add_argument("--graph-steps", type=int, default=10,
                    help="trajectories timed with each trajectory replayed from a CUDA graph (mixed)")
    ap.add_argument("--chrono-steps", type=int, default=10,
                    help="trajectories timed with the leapfrog's solves started from extrapolated solutions")
    ap.add_argument("--dropin-steps", type=int, default=1,
                    help="trajectories of the reference's per-iteration loop on the _C kernels (complex128)")
    ap.add_argument("--accept-steps", type=int, default=20,
                    help="Metropolis steps of the acceptance comparison, mixed against FP64")
    ap.add_argument("--accept-delta-t", type=float, default=0.002,
                    help="leapfrog step of the acceptance comparison: at the headline step 0.05 Delta H is "
                         "about 500 on this lattice and nothing is accepted")
    ap.add_argument("--mhm-rhs", type=int, default=8)
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--cg-iters-per-solve", type=float, default=None,
                    help="reference arm with --no-cpu-trajectory: PCG iterations per solve to extrapolate with")
    ap.add_argument("--cpu-sample-iters", type=int, default=30,
                    help="reference arm: PCG iterations in each timed sample step")
    ap.add_argument("--no-cpu-trajectory", dest="cpu_trajectory", action="store_false",
                    help="reference arm: skip the full CPU trajectory that sets the iteration count and checks "
                         "the extrapolation")
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--solve-only", type=int, default=0,
                    help="profiling mode: one PCG solve of the workload with exactly this many iterations")
    ap.add_argument("--kernels", action="store_true",
                    help="time every library kernel once on the bench lattice, one JSON line each")
    ap.add_argument("--configs", action="store_true",
                    help="time the other benchmark configurations (C2, C4a, C4b, C5), one JSON line each")
    ap.add_argument("--matvec-only", type=int, default=0,
                    help="only time M^dag M on this many right-hand sides (c64; c128 with --mode fp64)")
    ap.add_argument("--mode", default="mixed", choices=["mixed", "mixed_bf16", "mixed_f16", "fp32", "fp64"],
                    help="precision of the --solve-only solve or --matvec-only launch")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="the library's static launch shapes instead of the autotuner's timed choice")
    ap.add_argument("--quick", action="store_true",
                    help="timed trajectories only (no e2e, FP64, Delta H, matvec or CPU legs): for profiling")
    return ap.parse_args(argv)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id):
        self.bus_id = bus_id
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
            if self.bus_id:
                cmd += ["-i", self.bus_id]
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self):
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
            for k, nm in enumerate(names):
                if f[5 + k].lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# reference arm / CPU baseline: the oracle (CPU restatement of the reference)
# ---------------------------------------------------------------------------
class CpuPort:
    """The CPU restatement of the path (the C/OpenMP port of the oracle,
    oracle/qedf_cpu.c, complex128, all host threads) on one chain of the
    bench workload: the same lattice, start and solver tolerance."""

    def __init__(self, L, Ltau, seed):
        import numpy as np
        from oracle import cpu_port as C
        from oracle import qedf_oracle as O
        C.build()
        self.C, self.O = C, O
        self.L, self.Ltau = L, Ltau
        rng = np.random.default_rng(seed)
        Vs = L * L
        self.boson = pi_flux_np(rng, L, Ltau, 1)
        self.p0 = rng.standard_normal(self.boson.shape)
        self.R = (rng.standard_normal(Ltau * Vs) + 1j * rng.standard_normal(Ltau * Vs)) / math.sqrt(2)
        self.phi = O.ref_to_kernel_layout(self.boson)[0]
        self.psi = O.mh_vec(self.phi[None], self.R.reshape(1, Ltau, Vs), L, 0.1)[0]
        self.csr = C.csr_of(O.precon_tau_matrix(Ltau).real.astype(np.float64)) \
            if Ltau >= O.precon_min_ltau() else None
        self.cp = O.Couplings()
        self.nth = C.threads()

    def sample(self, n_it):
        """One bounded sample: n_it PCG iterations, one fermion force and one
        boson substep of the leapfrog.  Returns seconds per unit and in all."""
        C, O = self.C, self.O
        s = C.Pcg(self.phi, self.psi, self.L, 0.1, self.csr)
        t0 = time.perf_counter()
        for _ in range(n_it):
            s.step()
        t1 = time.perf_counter()
        C.force(self.phi, s.x, self.L, 0.1)
        t2 = time.perf_counter()
        fb = O.force_b_plaq(self.boson, self.cp) + O.force_b_tau(self.boson, self.cp)
        C.inner_boson_step(self.boson, self.p0, 0.05, fb, self.cp)
        t3 = time.perf_counter()
        return {"cg_iteration": (t1 - t0) / n_it, "force": t2 - t1, "boson_substep": t3 - t2,
                "sample_s": t3 - t0}

    def trajectory(self, n_leapfrog, delta_t, rtol):
        """One full trajectory of this chain, timed: (seconds, iterations per solve, Delta H, seconds by part)."""
        t0 = time.perf_counter()
        H0, H1, iters, secs = self.C.trajectory(self.boson, self.p0, self.R, self.L, self.cp, delta_t, n_leapfrog,
                                                rtol, 100000, self.csr)
        return time.perf_counter() - t0, iters, H1 - H0, secs


def cpu_traj_seconds(u, iters_per_solve, n_leapfrog, M=5):
    """Seconds of one chain's trajectory from per-unit costs: n_leapfrog + 1
    solves and forces, n_leapfrog * M boson substeps."""
    return (n_leapfrog + 1) * (iters_per_solve * u["cg_iteration"] + u["force"]) + n_leapfrog * M * u["boson_substep"]


def cpu_sample(L, Ltau, seed, seconds):
    """Per-unit seconds of the CPU port on this workload, the medians of as
    many bounded samples as fit in about ``seconds``.  Returns (units,
    description, threads)."""
    port = CpuPort(L, Ltau, seed)
    port.sample(2)  # warm the caches and the thread pool
    t0 = time.perf_counter()
    runs = []
    while not runs or time.perf_counter() - t0 < seconds:
        runs.append(port.sample(24))
    u = {k: statistics.median(r[k] for r in runs) for k in runs[0]}
    return u, (f"{len(runs)} samples of 24 PCG iterations + 1 fermion force + 1 boson substep of the C/OpenMP port "
               f"of the oracle (complex128) at L={L}, Ltau={Ltau} on {port.nth} threads"), port.nth


def run_reference(args):
    """The reference arm: the CPU restatement of the reference's path on the
    host cores.  Each step is a bounded sample (PCG iterations, a fermion
    force, a boson substep of one chain); the value is the trajectories/hour
    those per-unit costs imply with the iteration count of a full trajectory
    that this arm runs and times first, whose measured time checks the
    extrapolation."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    port = CpuPort(args.L, args.Ltau, args.seed)
    port.sample(2)
    check = None
    iters = args.cg_iters_per_solve
    if args.cpu_trajectory:
        t_traj, its, dH, secs = port.trajectory(args.n_leapfrog, args.delta_t, args.rtol)
        iters = statistics.mean(its)
        check = {"measured_s": t_traj, "iters_per_solve": iters, "delta_H": dH, "seconds_by_part": secs}
    elif iters is None:
        iters = CG_ITERS_PER_SOLVE
    runs, step_s = [], []
    for k in range(args.warmup + args.steps):
        r = port.sample(args.cpu_sample_iters)
        if k >= args.warmup:
            runs.append(r)
            step_s.append(r["sample_s"])
    u = {k: statistics.median(r[k] for r in runs) for k in runs[0]}
    t_extrap = cpu_traj_seconds(u, iters, args.n_leapfrog)
    value = 3600.0 / t_extrap
    sample = (f"each step: {args.cpu_sample_iters} PCG iterations + 1 fermion force + 1 boson substep of one chain, "
              f"C/OpenMP port of the oracle (complex128) at L={args.L}, Ltau={args.Ltau} on {port.nth} threads; "
              f"value extrapolated to a trajectory with {iters:.1f} PCG iterations per solve, "
              f"{args.n_leapfrog + 1} solves and forces, {5 * args.n_leapfrog} boson substeps")
    if check:
        check["extrapolated_s"] = cpu_traj_seconds(u, check["iters_per_solve"], args.n_leapfrog)
        check["extrapolation_error"] = check["extrapolated_s"] / check["measured_s"] - 1.0
        sample += (f"; one full trajectory of this chain measured first: {check['measured_s']:.1f} s against "
                   f"{check['extrapolated_s']:.1f} s extrapolated ({100 * check['extrapolation_error']:+.1f} %)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(step_s),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128/f64 (C/OpenMP)",
        "data": "synthetic", "config": workload_config(args),
        "value_kind": "extrapolated from the timed samples (ms_per_step is one sample, not a trajectory)",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": port.nth, "kind": "port", "sample": sample,
                         "s_per_unit": u},
        "trajectory_check": check,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(args):
    return {"workload": f"HMC trajectory L={args.L} Ltau={args.Ltau} dtau=0.1 J=1 K=1, {args.n_leapfrog} leapfrog "
                        f"steps of {args.delta_t}, PCG rtol {args.rtol}, {args.bs} chains per GPU",
            "lattice": [args.L, args.L, args.Ltau], "chains_per_gpu": args.bs, "n_leapfrog": args.n_leapfrog,
            "delta_t": args.delta_t, "cg_rtol": args.rtol, "precision": "mixed (float CG, double reliable "
            "updates / H / Metropolis)", "l2": "inputs larger than L2 (per-GPU working set > 126 MB)",
            "init": "staggered pi-flux +-pi/4 plus Gaussian noise (reference's physical start)"}


def pi_flux_np(rng, L, Ltau, bs):
    import numpy as np
    x = np.arange(L)[:, None]
    y = np.arange(L)[None, :]
    sg = 1 - 2 * ((x + y) % 2)
    b = np.zeros((bs, 2, L, L, Ltau))
    b[:, 0] = (sg * math.pi / 4)[None, :, :, None]
    b[:, 1] = (-sg * math.pi / 4)[None, :, :, None]
    return b + 0.05 * rng.standard_normal(b.shape)


# ---------------------------------------------------------------------------
# replicas: whole-job aggregation over ranks
# ---------------------------------------------------------------------------
def replica_seed(base_seed, rank):
    """Independent chains per rank: a distinct seed per replica."""
    return base_seed + 1000 * rank


def aggregate_over_ranks(elapsed_s, trajectories_per_rank, world, dist=None, device=None):
    """Max of the per-rank timed region over ranks (the job ends with the
    slowest replica) and the whole-job throughput: all ranks' trajectories
    divided by that time.  Returns (max_elapsed_s, trajectories_per_hour)."""
    if world > 1:
        import torch
        t = torch.tensor([float(elapsed_s)], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_s = float(t)
    return elapsed_s, 3600.0 * trajectories_per_rank * world / elapsed_s


# ---------------------------------------------------------------------------
# native arm
# ---------------------------------------------------------------------------
def run_native(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    from qed_fermion_b200 import _lib, build, ops
    from qed_fermion_b200.hmc import HmcSampler, ref_to_kernel
    build.build()
    L, Lt, bs = args.L, args.Ltau, args.bs
    seed = replica_seed(args.seed, rank)
    rng = np.random.default_rng(seed)

    def make(precision, solver_impl="persistent", graph=False, chrono_guess=None):
        h = HmcSampler(Lx=L, Ltau=Lt, J=1.0, K=1.0, dtau=0.1, bs=bs, delta_t=args.delta_t,
                       N_leapfrog=args.n_leapfrog, precision=precision, cg_rtol=args.rtol, max_iter=20000,
                       device=dev, seed=seed, solver_impl=solver_impl, autotune=args.autotune, graph=graph,
                       chrono_guess=chrono_guess)
        return h

    hmc = make("mixed")
    boson0 = torch.tensor(pi_flux_np(rng, L, Lt, bs), device=dev)
    hmc.boson = boson0.to(torch.float32)
    stream = torch.cuda.current_stream()

    # --- pre-warm: the persistent solver on a scratch right-hand side for a few
    # seconds (torch's default generator, not the sampler's)
    if args.prewarm_seconds > 0:
        ang = ref_to_kernel(hmc.boson).reshape(-1).to(hmc.solver.angle_dtype)
        bw = torch.randn(hmc.solver.nrhs * L * L * Lt, dtype=torch.complex128, device=dev).to(hmc.solver.vec_dtype)
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < args.prewarm_seconds:
            hmc.solver.solve(ang, bw)
            torch.cuda.synchronize()
        del ang, bw

    # --- instrumentation of the persistent PCG launches (events on the stream)
    solve_events = []
    orig_solve = hmc.solver.solve

    def timed_solve(*a, **k):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = orig_solve(*a, **k)
        e1.record(stream)
        solve_events.append((e0, e1, res.iters))
        return res

    hmc.solver.solve = timed_solve

    # --- warm-up
    for _ in range(args.warmup):
        hmc.metropolis_update()
    torch.cuda.synchronize()
    solve_events.clear()

    # --- timed region (device residency: inputs already in HBM)
    bus = None
    try:
        pci = torch.cuda.get_device_properties(dev)
        bus = f"{pci.pci_domain_id:08X}:{pci.pci_bus_id:02X}:{pci.pci_device_id:02X}.0"
    except Exception:
        bus = None
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = _lib.LAUNCHES["count"]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    accepted = []
    with ClockSampler(bus) as clk:
        t_start.record(stream)
        for _ in range(args.steps):
            _, accp, it, err, H0, H1 = hmc.metropolis_update()
            accepted.append(accp)
        t_end.record(stream)
        torch.cuda.synchronize()
    launches = _lib.LAUNCHES["count"] - launches0
    elapsed = t_start.elapsed_time(t_end) / 1e3
    elapsed, value = aggregate_over_ranks(elapsed, args.steps * bs, world, dist, dev)
    if world > 1:
        dist.barrier()
    clocks = clk.summary()
    acc_rate = float(torch.stack(accepted).double().mean())

    # --- dominant kernel: the persistent PCG (algorithmic bytes per launch)
    N = L * L * Lt
    pcg_ms, pcg_bytes, iters_all = [], [], []
    for e0, e1, its in solve_events:
        ms = e0.elapsed_time(e1)
        it_sum = int(its.sum())
        iters_all.extend(its.cpu().tolist())
        pcg_ms.append(ms)
        pcg_bytes.append(it_sum * N * (7 * 8 + 2 * 4))  # float vectors and angles per iteration
    pcg_time = sum(pcg_ms) / 1e3
    achieved = sum(pcg_bytes) / pcg_time / 1e9 if pcg_time > 0 else None
    # DRAM traffic per launch: bytes per site and iteration from one ncu capture
    # of a full-length solve of this workload, scaled by the site-iterations of
    # the average launch here
    site_iters = statistics.mean(b / (7 * 8 + 2 * 4) for b in pcg_bytes) if pcg_bytes else 0
    traffic = PCG_DRAM_BYTES_PER_SITE_ITER * site_iters if site_iters else None
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_kind = "measured" if "hbm_gbs" in peaks else "fallback"

    result = {}
    if rank == 0:
        result["pcg_share_of_step"] = pcg_time / elapsed
        result["cg_iters_per_solve"] = statistics.mean(iters_all) if iters_all else None

    # --- end to end through the public API with host buffers (every rank, the
    # whole job's trajectories over the slowest rank's time)
    e2e = None
    if not args.quick:
        hb = torch.empty((bs, 2, L, L, Lt), dtype=torch.float32, pin_memory=True)
        hb.copy_(hmc.boson.cpu())
        hout = torch.empty_like(hb).pin_memory()
        hH = torch.empty((3, bs), dtype=torch.float64, pin_memory=True)
        k_e2e = args.steps
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k_e2e):
            hmc.boson = hb.to(dev, non_blocking=True)
            _, accp, it, err, H0, H1 = hmc.metropolis_update()
            hout.copy_(hmc.boson, non_blocking=True)
            hH[0].copy_(H0, non_blocking=True)
            hH[1].copy_(H1, non_blocking=True)
            hH[2].copy_(accp.double(), non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        t_e2e = e0.elapsed_time(e1) / 1e3
        if world > 1:
            dist.barrier()
        t_e2e, v_e2e = aggregate_over_ranks(t_e2e, k_e2e * bs, world, dist, dev)
        e2e = {"value": v_e2e, "unit": UNIT, "h2d_bytes_per_step": hb.numel() * 4,
               "d2h_bytes_per_step": hout.numel() * 4 + hH.numel() * 8, "steps": k_e2e}

    def time_trajectories(h, n):
        h.metropolis_update()  # warm-up
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        its = []
        e0.record(stream)
        for _ in range(n):
            _, _, it, _, _, _ = h.metropolis_update()
            its.append(it)
        e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        shape = ({k: h.solver.tuned[k] for k in ("by", "slab", "stage", "chunk")} if h.solver.tuned else None)
        return {"value": 3600.0 * n * bs / t, "unit": UNIT, "steps": n, "s_per_trajectory": t / n,
                "cg_iters_per_solve": float(torch.stack(its).double().mean()), "pcg_launch_shape": shape}

    # --- plain FP64 path, same workload
    fp64 = None
    if rank == 0 and world == 1 and args.fp64_steps > 0 and not args.quick:
        h64 = make("fp64")
        h64.boson = hmc.boson.to(torch.float64)
        fp64 = time_trajectories(h64, args.fp64_steps)
        fp64["path"] = "same engine in double (persistent PCG, double force)"
        del h64
        if args.dropin_steps > 0:
            # the drop-in path: the reference's per-iteration PCG loop on this library's
            # _C kernels in complex128, same workload
            hd = make("fp64", solver_impl="reference_loop")
            hd.boson = hmc.boson.to(torch.float64)
            fp64["dropin"] = time_trajectories(hd, args.dropin_steps)
            fp64["dropin"]["path"] = ("reference loop structure (preconditioned_cg_fast_test) on _C kernels, "
                                      "complex128")
            del hd

    # --- every option at once: fp16 storage, linear chronological guesses and
    # trajectories replayed from a CUDA graph
    fastest = None
    if rank == 0 and world == 1 and args.options_steps > 0 and not args.quick:
        ho = make("mixed_f16", graph=True, chrono_guess="linear")
        ho.boson = hmc.boson.clone()
        fastest = time_trajectories(ho, args.options_steps)
        fastest["path"] = ("mixed precision with p and z stored as scaled fp16, linear chronological initial "
                           "guesses and trajectories replayed from a CUDA graph")
        del ho

    # --- the same trajectories replayed from a CUDA graph (one graph launch per
    # trajectory; the first proposal, in the warm-up, captures it)
    graph = None
    if rank == 0 and world == 1 and args.graph_steps > 0 and not args.quick:
        hg = make("mixed", graph=True)
        hg.boson = hmc.boson.clone()
        graph = time_trajectories(hg, args.graph_steps)
        graph["path"] = "mixed precision, each trajectory replayed from a CUDA graph"
        del hg

    # --- the leapfrog's solves started from the linear extrapolation of the
    # previous two solutions instead of zero
    chrono = None
    if rank == 0 and world == 1 and args.chrono_steps > 0 and not args.quick:
        hc = make("mixed", chrono_guess="linear")
        hc.boson = hmc.boson.clone()
        chrono = time_trajectories(hc, args.chrono_steps)
        chrono["path"] = ("mixed precision; each leapfrog solve after the first starts from the linear "
                          "extrapolation of the previous two solutions (the reference starts from zero)")
        del hc

    # --- bf16 vector storage, same workload
    bf16 = None
    if rank == 0 and world == 1 and args.bf16_steps > 0 and not args.quick:
        hb16 = make("mixed_bf16")
        hb16.boson = hmc.boson.clone()
        bf16 = time_trajectories(hb16, args.bf16_steps)
        bf16["path"] = "mixed precision with the PCG's p and z stored as bf16 pairs"
        # read p (bf16), x, r, angles; write x, r, p (bf16)
        bf16["pcg_bytes_per_site_iteration"] = 2 * 4 + 4 * 8 + 2 * 4
        del hb16

    # --- scaled fp16 vector storage, same workload
    f16 = None
    if rank == 0 and world == 1 and args.f16_steps > 0 and not args.quick:
        hf16 = make("mixed_f16")
        hf16.boson = hmc.boson.clone()
        f16 = time_trajectories(hf16, args.f16_steps)
        f16["path"] = ("mixed precision with the PCG's p and z stored as fp16 pairs scaled by a power of two "
                       "per vector")
        f16["pcg_bytes_per_site_iteration"] = 2 * 4 + 4 * 8 + 2 * 4
        del hf16

    # --- Delta H of one shared trajectory: mixed and bf16 storage against FP64
    dH = None
    if rank == 0 and world == 1 and not args.quick:
        gen = torch.Generator(device=dev)
        gen.manual_seed(seed + 7)
        x0 = hmc.boson.to(torch.float64)
        p0 = torch.randn(x0.shape, device=dev, dtype=torch.float64, generator=gen)
        R = torch.randn((bs, N), device=dev, dtype=torch.complex128, generator=gen) / math.sqrt(2)
        h64 = make("fp64")
        _, H0d, H1d, _, _ = h64.leapfrog_proposer5(x0.to(torch.float32).to(torch.float64),
                                                    p0=p0.to(torch.float32).to(torch.float64), R=R)
        del h64
        dHd = (H1d - H0d).cpu()
        dH = {"dH_fp64": dHd.tolist(), "H0": H0d.cpu().tolist()}
        for name, h in (("mixed", hmc), ("mixed_bf16", make("mixed_bf16")), ("mixed_f16", make("mixed_f16")),
                        ("mixed_chrono_linear", make("mixed", chrono_guess="linear"))):
            _, H0m, H1m, _, _ = h.leapfrog_proposer5(x0.to(torch.float32), p0=p0.to(torch.float32), R=R)
            dHm = (H1m - H0m).cpu()
            dH[name] = {"dH": dHm.tolist(), "abs_err": (dHm - dHd).abs().tolist(),
                        "rel_err_vs_H0": ((dHm - dHd).abs() / H0d.abs().cpu()).tolist(),
                        "rel_err_vs_dH": ((dHm - dHd).abs() / dHd.abs()).tolist()}

    # --- acceptance, mixed (float and scaled fp16 storage) against FP64, at a
    # step where proposals are accepted: all chains take the same momenta,
    # pseudofermions and uniforms each step
    acc = None
    if rank == 0 and world == 1 and args.accept_steps > 0 and not args.quick:
        from qed_fermion_b200.hmc import metropolis_accept
        gen = torch.Generator(device=dev)
        gen.manual_seed(seed + 11)
        chains = {"fp64": make("fp64"), "mixed": make("mixed"), "mixed_f16": make("mixed_f16")}
        xs = {}
        for k, h in chains.items():
            h.delta_t_tensor.fill_(args.accept_delta_t)
            xs[k] = hmc.boson.to(torch.float32).clone().to(h.dtype)
        rec = {k: [] for k in chains}
        nmis = {k: 0 for k in chains if k != "fp64"}
        dd = {k: [] for k in nmis}
        for _ in range(args.accept_steps):
            p0 = torch.randn(xs["fp64"].shape, device=dev, dtype=torch.float64, generator=gen).to(torch.float32)
            R = torch.randn((bs, N), device=dev, dtype=torch.complex128, generator=gen) / math.sqrt(2)
            u = torch.rand(bs, device=dev, dtype=torch.float64, generator=gen)
            step = {}
            for k, h in chains.items():
                nx, H0, H1, _, _ = h.leapfrog_proposer5(xs[k], p0=p0.to(h.dtype), R=R)
                a, _ = metropolis_accept(H0, H1, u)
                xs[k] = torch.where(a.view(-1, 1, 1, 1, 1), nx.to(h.dtype), xs[k])
                step[k] = (H1 - H0, a)
                rec[k].append(((H1 - H0).cpu(), a.cpu()))
            for k in nmis:
                nmis[k] += int((step[k][1] != step["fp64"][1]).sum())
                dd[k].append((step[k][0] - step["fp64"][0]).abs().cpu())
        acc = {"delta_t": args.accept_delta_t, "n_leapfrog": args.n_leapfrog, "steps": args.accept_steps,
               "chains": bs, "decisions_differing": nmis["mixed"],
               "max_abs_dH_difference": float(torch.stack(dd["mixed"]).max()),
               "mixed_f16_vs_fp64": {"decisions_differing": nmis["mixed_f16"],
                                     "max_abs_dH_difference": float(torch.stack(dd["mixed_f16"]).max())}}
        for k, v in rec.items():
            d = torch.stack([a for a, _ in v]).double()
            acc[k] = {"acceptance": float(torch.stack([b for _, b in v]).double().mean()),
                      "mean_exp_minus_dH": float(torch.exp(-d).mean()), "mean_dH": float(d.mean())}
        del chains

    # --- M^dag M matvec bandwidth (several right-hand sides, working set > L2)
    mhm = None
    if rank == 0 and world == 1 and args.mhm_rhs > 0 and not args.quick:
        nr = args.mhm_rhs
        mhm = {}
        for prec, cdt, rdt, bps in (("c64", torch.complex64, torch.float32, 24), ("c128", torch.complex128,
                                                                                 torch.float64, 48)):
            phi = torch.rand((nr, 2 * N), device=dev, dtype=rdt) * 6.28 - 3.14
            xv = torch.randn((nr, N), device=dev, dtype=cdt)
            out = torch.empty_like(xv)
            for _ in range(3):
                ops.apply_operator("mhm", phi, xv, L, 0.1, out=out)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            reps = 10
            e0.record(stream)
            for _ in range(reps):
                ops.apply_operator("mhm", phi, xv, L, 0.1, out=out)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            gbs = bps * N * nr / (ms / 1e3) / 1e9
            mhm[prec] = {"GBps": gbs, "frac_of_measured_hbm": gbs / hbm_peak, "ms_per_launch": ms,
                         "rhs": nr, "bytes_per_site": bps}
            del phi, xv, out

    # --- CPU baseline (oracle restatement) on a bounded sample
    cpu = None
    if rank == 0 and world == 1 and args.cpu_seconds > 0 and not args.quick:
        u, sample, nth = cpu_sample(L, Lt, seed, args.cpu_seconds)
        ips = result.get("cg_iters_per_solve") or CG_ITERS_PER_SOLVE
        cpu = {"value": 3600.0 / cpu_traj_seconds(u, ips, args.n_leapfrog), "unit": UNIT, "cores": nth,
               "kind": "port", "sample": sample + f"; extrapolated to a trajectory with the {ips:.0f} PCG iterations "
                                                  f"per solve this run needed, {args.n_leapfrog + 1} solves and "
                                                  f"forces, {5 * args.n_leapfrog} boson substeps",
               "s_per_unit": u}

    if rank == 0:
        for leg in (f16, bf16, graph, chrono, fastest):
            if leg and fp64:
                leg["speedup_vs_fp64"] = leg["value"] / fp64["value"]
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (c64) iterations, f64 reliable updates/H",
            "data": "synthetic", "config": workload_config(args),
            "roofline": {"bound": "hbm", "kernel": "k_pcg (persistent batched PCG)",
                         "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": (achieved / hbm_peak) if achieved else None, "peak_kind": peak_kind,
                         "traffic": traffic,
                         "algorithmic_bytes_per_launch": statistics.mean(pcg_bytes) if pcg_bytes else None,
                         "traffic_source": f"dram__bytes_read+write of k_pcg, {PCG_DRAM_BYTES_PER_SITE_ITER} B per "
                                           "site-iteration from an ncu capture of a 482-iteration solve of this "
                                           "workload, times the average launch's site-iterations",
                         "bytes_model": "per PCG iteration per rhs: N*(7*8 + 2*4) B (read p,x,r,angles; write x,r,p)"},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
            "fp64_plain": fp64, "speedup_vs_fp64": (value / world) / fp64["value"] if fp64 else None,
            "speedup_vs_fp64_dropin": ((value / world) / fp64["dropin"]["value"]
                                       if fp64 and "dropin" in fp64 else None),
            "pcg_launch_shape": ({k: hmc.solver.tuned[k] for k in ("by", "slab", "stage", "chunk")}
                                 if hmc.solver.tuned else None),
            "bf16": bf16, "f16": f16, "all_options": fastest, "graph": graph, "chrono": chrono, "delta_H": dH, "mhm_matvec": mhm, "acceptance": acc_rate,
            "acceptance_vs_fp64": acc, **result,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_solve_only(args):
    """One PCG solve on the bench workload with a fixed iteration count (rtol 0):
    the small, self-contained launch that ncu captures of the solver use."""
    import numpy as np
    import torch
    from qed_fermion_b200 import build
    from qed_fermion_b200.hmc import ref_to_kernel
    from qed_fermion_b200.solver import PcgSolver, System
    build.build()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(args.seed)
    L, Lt, bs = args.L, args.Ltau, args.bs
    phi = ref_to_kernel(torch.tensor(pi_flux_np(rng, L, Lt, bs), device=dev))
    b = torch.randn((bs, L * L * Lt), dtype=torch.complex128, device=dev,
                    generator=torch.Generator(device=dev).manual_seed(args.seed)) / math.sqrt(2)
    s = PcgSolver([System(L, Lt, bs)], mode=args.mode, rtol=0.0, max_iter=args.solve_only, device=dev)
    args_ = (phi.to(s.angle_dtype), b.to(s.vec_dtype))
    s.solve(*args_)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    res = s.solve(*args_)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    it = int(res.iters.max())
    n = L * L * Lt * bs
    # bytes per site and iteration: 7 vector accesses and the two angles
    bps = {"mixed": 64, "fp32": 64, "fp64": 128, "mixed_bf16": 48, "mixed_f16": 48}[args.mode]
    print(json.dumps({"solve_only": True, "mode": args.mode, "lattice": [L, L, Lt], "rhs": bs, "iters": it,
                      "ms": ms, "us_per_iter": ms * 1e3 / max(it, 1), "bytes_per_site_iter": bps,
                      "algorithmic_GBps": n * bps * it / (ms / 1e3) / 1e9}), flush=True)
    return 0


def run_kernels(args):
    """Every kernel of the library on L=48, Ltau=480 (--mhm-rhs right-hand
    sides, 8 by default, each with its own field: inputs and outputs larger
    than L2), after warm-up: the algorithmic bytes of one launch and the
    bandwidth they imply.  The launches are replayed from a CUDA graph of 10
    calls and timed with CUDA events, so the device time is measured rather
    than the host's dispatch; the persistent solver (milliseconds a launch,
    two right-hand sides as in the trajectory benchmark) is timed directly."""
    import numpy as np
    import torch
    from qed_fermion_b200 import build, ops, precon
    from qed_fermion_b200.hmc import ref_to_kernel
    from qed_fermion_b200.solver import PcgSolver, System
    build.build()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(args.seed)
    L, Lt, bs = args.L, args.Ltau, args.mhm_rhs
    N = L * L * Lt
    boson = torch.tensor(pi_flux_np(rng, L, Lt, bs), device=dev)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)

    def timed(fn, reps=10, graph=True):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        if graph:
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                for _ in range(reps):
                    fn()
            g.replay()
            run = g.replay
        else:
            def run():
                for _ in range(reps):
                    fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        run()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def emit(kernel, what, ms, nbytes):
        gbs = nbytes / (ms / 1e3) / 1e9
        print(json.dumps({"kernel_run": True, "kernel": kernel, "what": what, "ms": ms, "algorithmic_bytes": nbytes,
                          "GBps": gbs, "frac_of_measured_hbm": gbs / hbm}), flush=True)

    for prec, rdt, cdt, sv, sp in (("c64", torch.float32, torch.complex64, 8, 4),
                                   ("c128", torch.float64, torch.complex128, 16, 8)):
        phi = ref_to_kernel(boson).reshape(bs, -1).to(rdt)
        x = torch.randn((bs, N), dtype=cdt, device=dev)
        out = torch.empty_like(x)
        for op in ("m", "mh", "mhm"):
            ms = timed(lambda: ops.apply_operator(op, phi, x, L, 0.1, out=out))
            emit(f"k_operator ({op}, {prec})", f"{bs} rhs", ms, bs * N * (2 * sv + 2 * sp))
        vt = x[:, :L * L].contiguous()
        ms = timed(lambda: ops.b_vec_per_tau(phi[0, :2 * L * L].contiguous(), vt, L, 0.1, True))
        emit(f"k_bvec ({prec})", f"{bs} vectors of one slice, six partial products", ms,
             bs * L * L * (sv + 6 * sv) + 2 * L * L * sp)
        F = None
        ms = timed(lambda: ops.fermion_force(phi, x, L, 0.1))
        emit(f"k_force ({prec})", f"{bs} rhs", ms, bs * N * (sv + 4 * sp))
        csr = precon.to_device(precon.builtin_tau_csr(Lt), dev)
        ms = timed(lambda: ops.precon_apply(x, csr, L))
        emit(f"k_precon ({prec})", f"{bs} rhs", ms, bs * N * 2 * sv)
        ms = timed(lambda: ops.cdot(x, out))
        emit(f"k_cdot ({prec})", f"{bs} rows", ms, bs * N * 2 * sv)
        ang = phi.clone()
        ms = timed(lambda: ops.boson_force(ang, L, 0.1, 10.0))
        emit(f"k_boson_force ({prec})", f"{bs} fields", ms, bs * N * 2 * sp * 2)
        ms = timed(lambda: ops.boson_action(ang, L, 0.1, 10.0, momenta=ang))
        emit(f"k_boson_action ({prec})", f"{bs} fields with momenta", ms, bs * N * 2 * sp * 2)
        # bond-bond correlator passes: 8 noise vectors, their 28 pairs
        nrv = 8
        eta_b = torch.randn((nrv, N), dtype=cdt, device=dev)
        g_b = torch.randn((nrv, N), dtype=cdt, device=dev)
        ep_b = torch.exp(1j * torch.rand(N, dtype=rdt, device=dev)).to(cdt)
        prs = torch.combinations(torch.arange(nrv, device=dev), r=2).to(torch.int32)
        ps_b, pt_b = prs[:, 0].contiguous(), prs[:, 1].contiguous()
        fa_b = torch.empty((len(prs), Lt, L, L), dtype=cdt, device=dev)
        fb_b = torch.empty_like(fa_b)
        ms = timed(lambda: ops.bb_pair_fields("T21", eta_b, g_b, ep_b, ps_b, pt_b, L, fa_b, fb_b))
        emit(f"k_bb_pair_fields (T21, {prec})", f"{len(prs)} pairs of {nrv} vectors", ms,
             len(prs) * N * 2 * sv + (2 * nrv + 1) * N * sv)
        S_b = torch.zeros(L * L, dtype=torch.complex128, device=dev)
        ms = timed(lambda: ops.bb_kspace_acc(fa_b, fb_b, S_b))
        emit(f"k_bb_kspace_acc ({prec})", f"{len(prs)} pairs x {Lt} slices", ms, len(prs) * N * 2 * sv)
        v_b = torch.empty_like(eta_b)
        tv_b = torch.zeros(L * L, dtype=torch.complex128, device=dev)
        ms = timed(lambda: ops.bb_vfield(eta_b, g_b, ep_b, L, v_b, tv_b))
        emit(f"k_bb_vfield ({prec})", f"{nrv} vectors", ms, (3 * nrv + 1) * N * sv)
        ms = timed(lambda: ops.bb_diag(eta_b, g_b, ep_b, L))
        emit(f"k_bb_diag ({prec})", f"{nrv} vectors", ms, (2 * nrv + 1) * N * sv)
        del eta_b, g_b, fa_b, fb_b, v_b
        pm = torch.zeros_like(ang)
        fm = torch.ones_like(ang)
        dt = torch.full((bs,), 0.01, dtype=torch.float64, device=dev)
        ms = timed(lambda: ops.kick_drift(pm, fm, ang, dt, None, 0.5, 1.0, L))
        emit(f"k_kick_drift ({prec})", f"{bs} fields, kick and drift", ms, bs * N * 2 * sp * 5)
    nb = 2
    for mode in ("mixed", "mixed_f16", "fp64"):
        s = PcgSolver([System(L, Lt, nb)], mode=mode, rtol=0.0, max_iter=100, device=dev)
        a_ = ref_to_kernel(boson[:nb]).reshape(-1).to(s.angle_dtype)
        b_ = torch.randn(nb * N, dtype=torch.complex128, device=dev).to(s.vec_dtype)
        ms = timed(lambda: s.solve(a_, b_), reps=2, graph=False)
        bps = {"mixed": 64, "mixed_f16": 48, "fp64": 128}[mode]  # the algorithmic model per site-iteration
        emit(f"k_pcg ({mode})", f"100 iterations, {nb} rhs", ms, 100 * nb * N * bps)
    return 0


def run_configs(args):
    """The benchmark's other configurations on one GPU, each after a warm-up
    run and timed with CUDA events: C2 (L=24 matvec and PCG to 1e-8 in both
    precisions), C4a (64 Z2 noise vectors on one L=36 field), C4b (16 lattices
    of uneven size in one launch), C5 (one 30-step trajectory at L=66)."""
    import numpy as np
    import torch
    from qed_fermion_b200 import build, ops
    from qed_fermion_b200.estimator import StochaticEstimator
    from qed_fermion_b200.hmc import HmcSampler, ref_to_kernel
    from qed_fermion_b200.solver import PcgSolver, System
    build.build()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(args.seed)

    def timed(fn, reps=1):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            out = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps, out

    def emit(d):
        print(json.dumps({"config_run": True, **d}), flush=True)

    def tuned(solver):
        t = solver.tuned
        return None if t is None else {k: t[k] for k in ("by", "slab", "stage", "chunk", "us_per_iter")}

    # C2: uniform angles, b = M^dag eta
    L, Lt = 24, 240
    N = L * L * Lt
    boson = torch.tensor(rng.uniform(-np.pi, np.pi, size=(1, 2, L, L, Lt)), device=dev)
    phi = ref_to_kernel(boson).reshape(1, -1)
    eta = torch.randn((1, N), dtype=torch.complex128, device=dev) / math.sqrt(2)
    b = ops.apply_operator("mh", phi, eta, L, 0.1)
    for prec, rdt, cdt, bps in (("c64", torch.float32, torch.complex64, 24), ("c128", torch.float64,
                                                                             torch.complex128, 48)):
        phi_p, b_p = phi.to(rdt), b.to(cdt)
        out = torch.empty_like(b_p)
        ms, _ = timed(lambda: ops.apply_operator("mhm", phi_p, b_p, L, 0.1, out=out), reps=20)
        emit({"config": "C2", "what": f"M^dag M {prec}, 1 rhs (a single launch of 138,240 sites)", "ms": ms,
              "GBps": bps * N / (ms / 1e3) / 1e9})
    for mode in ("mixed", "fp64"):
        s = PcgSolver([System(L, Lt, 1)], mode=mode, rtol=1e-8, max_iter=100000, device=dev, tune=True)
        args_ = (phi.reshape(-1).to(s.angle_dtype), b.reshape(-1).to(s.vec_dtype))
        ms, res = timed(lambda: s.solve(*args_))
        emit({"config": "C2", "what": f"PCG to 1e-8, {mode}", "ms": ms, "iters": int(res.iters.max()),
              "relres": float(res.relres.max()), "status": int(res.status.max()), "tuned": tuned(s)})

    # C4a: 64 Z2 noise vectors sharing one L=36 field
    L, Lt, nrv = 36, 360, 64
    bos = torch.tensor(pi_flux_np(rng, L, Lt, 1), device=dev)
    se = StochaticEstimator(L, Lt, Nrv=nrv, precision="mixed", cg_rtol=1e-10, device=dev, seed=5, noise="z2")
    eta = se.random_vec_bin()
    ms, _ = timed(lambda: se.set_eta_G_eta(bos, eta))
    emit({"config": "C4a", "what": "G_eta = (M^dag M)^-1 M^dag eta, 64 rhs, mixed, rtol 1e-10", "ms": ms,
          "iters": int(se.iters.max()), "relres": float(se.relres.max()), "tuned": tuned(se.solver)})
    se16 = StochaticEstimator(L, Lt, Nrv=nrv, precision="mixed_f16", cg_rtol=1e-10, device=dev, seed=5, noise="z2")
    ms16, _ = timed(lambda: se16.set_eta_G_eta(bos, eta))
    emit({"config": "C4a", "what": "the same solve with p and z stored as scaled fp16 (mixed_f16)", "ms": ms16,
          "iters": int(se16.iters.max()), "relres": float(se16.relres.max()), "tuned": tuned(se16.solver)})
    del se16
    ms, _ = timed(lambda: se.get_bond_bond_per_b2(bos))
    emit({"config": "C4a", "what": "bond-bond correlators T1+T21+T2+T4+Tvv over the 2016 noise pairs "
                                   "(complex128, pair-field and k-space kernels around cuFFT)", "ms": ms})
    se.corr_dtype = torch.complex64
    ms, _ = timed(lambda: se.get_bond_bond_per_b2(bos))
    emit({"config": "C4a", "what": "the same correlators in complex64 (the reference estimator's precision)",
          "ms": ms})
    se.corr_dtype = None
    # where one correlator's time goes: the passes of one chunk of pairs (the
    # default 1 GiB chunk: 34 pairs), each timed over 10 launches
    e128 = se.eta.to(torch.complex128).resolve_conj().contiguous()
    g128 = se.G_eta.to(torch.complex128).resolve_conj().contiguous()
    ep = torch.exp(1j * bos.permute(0, 1, 4, 3, 2)[0, 0].to(torch.float64)).contiguous()
    prs = torch.combinations(torch.arange(nrv, device=dev), r=2).to(torch.int32)
    nch = (1 << 30) // (4 * L * L * Lt * 16)
    ps, pt = prs[:nch, 0].contiguous(), prs[:nch, 1].contiguous()
    fa = torch.empty((nch, Lt, L, L), dtype=torch.complex128, device=dev)
    fb = torch.empty_like(fa)
    Sk = torch.zeros(L * L, dtype=torch.complex128, device=dev)
    chunks = len(prs) / nch
    parts = {}
    parts["pair_fields"], _ = timed(lambda: ops.bb_pair_fields("T21", e128, g128, ep, ps, pt, L, fa, fb), reps=10)
    parts["ifft2"], A = timed(lambda: torch.fft.ifft2(fa, norm="forward"), reps=10)
    parts["fft2"], B = timed(lambda: torch.fft.fft2(fb, norm="backward"), reps=10)
    parts["kspace_acc"], _ = timed(lambda: ops.bb_kspace_acc(A, B, Sk), reps=10)
    field_gb = nch * L * L * Lt * 16 / 1e9
    emit({"config": "C4a", "what": f"one correlator (T21) per chunk of {nch} pairs, {chunks:.1f} chunks",
          "ms_per_chunk": parts, "ms_per_correlator": {k: v * chunks for k, v in parts.items()},
          "GBps": {"pair_fields": 2 * field_gb / (parts["pair_fields"] / 1e3),
                   "ifft2": 2 * field_gb / (parts["ifft2"] / 1e3), "fft2": 2 * field_gb / (parts["fft2"] / 1e3),
                   "kspace_acc": 2 * field_gb / (parts["kspace_acc"] / 1e3)}})
    del fa, fb, A, B

    # C4b: 16 lattices L in {12, 18, 24, 30} x 4, Ltau = 10 L, one launch
    Ls = [12, 18, 24, 30] * 4
    systems = [System(L, 10 * L, 1) for L in Ls]
    phis = [ref_to_kernel(torch.tensor(pi_flux_np(rng, L, 10 * L, 1), device=dev)).reshape(-1) for L in Ls]
    rhs = [torch.randn(10 * L ** 3, dtype=torch.complex128, device=dev) / math.sqrt(2) for L in Ls]
    args_ = (torch.cat(phis).float(), torch.cat(rhs))
    for mode in ("mixed", "mixed_f16"):
        s = PcgSolver(systems, mode=mode, rtol=1e-10, max_iter=20000, device=dev, tune=True)
        ms, res = timed(lambda: s.solve(*args_))
        emit({"config": "C4b", "what": f"16 uneven lattices, one launch, {mode}, rtol 1e-10", "ms": ms,
              "iters_min": int(res.iters.min()), "iters_max": int(res.iters.max()),
              "relres_max": float(res.relres.max()), "tuned": tuned(s)})

    # C5: one 30-step trajectory at L=66, Ltau=660 (mixed)
    L, Lt = 66, 660
    hmc = HmcSampler(Lx=L, Ltau=Lt, bs=1, precision="mixed", cg_rtol=1e-10, max_iter=50000, delta_t=0.02,
                     N_leapfrog=30, device=dev, seed=6)
    b0 = torch.tensor(pi_flux_np(rng, L, Lt, 1), dtype=torch.float32, device=dev)
    hmc.leapfrog_proposer5(b0)  # warm-up
    torch.cuda.synchronize()
    ev = []
    orig = hmc.solver.solve

    def timed_solve(*a, **k):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        r = orig(*a, **k)
        e1.record()
        ev.append((e0, e1, r.iters))
        return r

    hmc.solver.solve = timed_solve
    ms, out = timed(lambda: hmc.leapfrog_proposer5(b0))
    hmc.solver.solve = orig
    N5 = L * L * Lt
    solves = ev[-31:]
    t_pcg = sum(a.elapsed_time(b) for a, b, _ in solves) / 1e3
    site_it = sum(int(i.sum()) for _, _, i in solves) * N5
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    pcg_gbs = site_it * 64 / t_pcg / 1e9
    emit({"config": "C5", "what": "one trajectory, 30 leapfrog steps of 0.02, mixed, rtol 1e-10", "ms": ms,
          "cg_iters_per_solve": float(out[3].float().mean()), "delta_H": float(out[2] - out[1]),
          "tuned": tuned(hmc.solver), "pcg_share": t_pcg / (ms / 1e3),
          "pcg_roofline": {"achieved_GBps": pcg_gbs, "frac_of_measured_hbm": pcg_gbs / hbm,
                           "bytes_model": "64 B per site-iteration (mixed)"}})
    return 0


def run_matvec_only(args):
    """Three warm-up and ten timed launches of M^dag M on the bench lattice: the
    small, self-contained case that ncu captures of the operator kernel use."""
    import torch
    from qed_fermion_b200 import build, ops
    build.build()
    dev = torch.device("cuda", 0)
    L, Lt, nr = args.L, args.Ltau, args.matvec_only
    N = L * L * Lt
    c128 = args.mode == "fp64"
    rdt, cdt, bps = (torch.float64, torch.complex128, 48) if c128 else (torch.float32, torch.complex64, 24)
    g = torch.Generator(device=dev).manual_seed(args.seed)
    phi = torch.rand((nr, 2 * N), device=dev, dtype=rdt, generator=g) * 6.28 - 3.14
    xv = torch.randn((nr, N), device=dev, dtype=cdt, generator=g)
    out = torch.empty_like(xv)
    for _ in range(3):
        ops.apply_operator("mhm", phi, xv, L, 0.1, out=out)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    reps = 10
    e0.record()
    for _ in range(reps):
        ops.apply_operator("mhm", phi, xv, L, 0.1, out=out)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    print(json.dumps({"matvec_only": True, "dtype": "c128" if c128 else "c64", "lattice": [L, L, Lt], "rhs": nr,
                      "ms_per_launch": ms, "GBps": bps * N * nr / (ms / 1e3) / 1e9}), flush=True)
    return 0


def main(argv=None):
    args = parse_args(argv)
    if args.impl == "reference":
        return run_reference(args)
    if args.solve_only > 0:
        return run_solve_only(args)
    if args.matvec_only > 0:
        return run_matvec_only(args)
    if args.configs:
        return run_configs(args)
    if args.kernels:
        return run_kernels(args)
    return run_native(args)


if __name__ == "__main__":
    sys.exit(main())
