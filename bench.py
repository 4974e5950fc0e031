#!/usr/bin/env python
"""Benchmark of the B200 fermion path: sigma-HMC trajectories per second at L = 64.

Workload (one "step" = one trajectory): L = 64 (V = 262,144 sites), beta_s =
0.85, sigma i.i.d. N(0, 2/(N_f beta_s)) on the dual sites, the reference's
default integrator LFMN2VF with 10 steps of eps = 0.05, two pseudofermion
flavours, every CG solve stopped at a true relative residual of 1e-10.
Synthetic data: momenta and chi drawn N(0, 1) (seeded), as the reference
draws them.

  value      mixed-precision solver, draws already resident in HBM, CUDA events
             on the library's stream; L2 flushed (512 MB write) before every
             trajectory, inside the timed region.
  e2e        the same trajectories through the host-buffer C-ABI: per step the
             draws are copied from pinned host memory (gn_write_state), the
             trajectory runs (gn_trajectory) and sigma / sigma-mass are read
             back (gn_store_sigma); host wall clock.
  roofline   the dominant kernel: the persistent CG kernel (mixed precision,
             two flavours) of one solve; algorithmic bytes from its iteration
             counts, duration from CUDA events.
  cpu_baseline one full trajectory of the reference's own C code (compiled
             from its sources into oracle/_ref/, every CG to 1e-10 |phi|) on
             one host core, run in a spawned process beside the GPU work.
  --impl reference: the reference arm, K trajectories of the same code spread
             over the host cores (one serial process per core); value = K over
             the wall clock from a common start to the last finish.

The line ends with short summaries of the side measurements (batched chains,
serving, L = 128, U(1)), the Dirac apply's roofline, the FP64 arm and the
mixed / FP64 ratio; --detail PATH writes all of them in full.

Multi-GPU: one process per GPU, each an independent chain (the path does not
shard; replicas only), max over ranks of the timed region.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG = ROOT / "3d-gross-neveu-model_b200"
for _p in (str(ROOT), str(PKG)):
    if _p not in sys.path:
        sys.path.insert(0, _p)

L_DEFAULT = 64
BETA_S = 0.85
NFLAV = 4
# DRAM bytes per launch measured with ncu (one capture each; summaries under
# profiles/): the dominant solver kernel at L = 64 and the Dirac apply at L = 256.
CG_MIXED_DRAM_BYTES = 6_790_400      # 6.449 MB read + 0.342 MB written (cg_mixed_duo_kernel)
DIRAC256_DRAM_BYTES = 379_232_256    # 269.540 MB read + 109.692 MB written
METRIC = "HMC trajectories/s at L=64 (LFMN2VF, 10 x eps 0.05, CG to 1e-10 true relative residual)"
UNIT = "traj/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--L", type=int, default=L_DEFAULT)
    ap.add_argument("--md-steps", type=int, default=10)
    ap.add_argument("--eps", type=float, default=0.05)
    ap.add_argument("--tol", type=float, default=1e-10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-l128", action="store_true", help="skip the L = 128 mixed-precision case")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving sweep")
    ap.add_argument("--detail", default=None, help="write every side measurement to this JSON file")
    ap.add_argument("--case", choices=["cg64", "dirac128", "dirac256", "traj64", "batched", "serve", "serve_sharded",
                                       "l128", "u1", "ens", "kernels"],
                    default=None, help="run one small case for a profiler instead of the benchmark")
    return ap.parse_args()


# ---------------------------------------------------------------- distributed
def dist_setup(backend):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def dist_max(x, world, device=None):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------- clocks
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None
        self.offset = 0

    def mark(self):
        """Only samples written after this call are reported (the timed region's)."""
        if self.proc is not None:
            self.fh.flush()
            self.offset = os.path.getsize(self.path)

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.device), "-lms", "50"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
            # wait for the first sample: the sampler's start-up (NVML initialisation)
            # must not fall inside a timed region
            t0 = time.perf_counter()
            while time.perf_counter() - t0 < 5.0 and os.path.getsize(self.path) == 0:
                time.sleep(0.05)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            fh.seek(self.offset)
            lines = fh.read().splitlines()
        for ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power)}


# ---------------------------------------------------------------- reference (CPU)
REF_REL_TAG = "_rel"  # the reference built with GN_REF_RELATIVE_TOL=1e-10 (oracle/build_ref.py REL_TAG)


def ref_rel_path(L):
    from oracle import build_ref
    return build_ref.lib_path(L, 0, REF_REL_TAG)


def _ref_traj_worker(L, eps, md_steps, seed, ntraj, warm, barrier, q):
    """`ntraj` trajectories of the reference's own integrator
    LeapFrog2MinimumNormSigmaVelocityFirst (moleculardynamics.c:1234) at L, in
    this process, drawing from the reference's dSFMT stream seeded with `seed`.
    The build (oracle/_ref/libgnref_L{L}_i0_rel.so) stops every CG at
    |r| < 1e-10 |phi|, the benchmark's rule.  `warm` Dirac applies (dirac.c:46)
    come first; the clock starts when every worker has reached the barrier.
    Puts (t_start, t_end, ntraj, cg_iterations, accepted, error)."""
    try:
        sys.path.insert(0, str(ROOT))
        from oracle.oracle import Ref
        ref = Ref(L, build=False, tag=REF_REL_TAG)
        ref.init(seed, BETA_S, eps, md_steps)
        rng = np.random.default_rng(seed)
        V = L ** 3
        ref.set_sigma(rng.normal(0.0, np.sqrt(2.0 / (NFLAV * BETA_S)), V))
        psi = rng.normal(size=V).astype(complex)
        for _ in range(warm):
            ref.dirac(psi, 0)
        acc = 0
        with tempfile.TemporaryDirectory() as d:
            barrier.wait()
            t0 = time.monotonic()
            for _ in range(ntraj):
                ok, a, _ = ref.trajectory(os.path.join(d, "acc.txt"))
                acc += int(a)
            t1 = time.monotonic()
        q.put((t0, t1, ntraj, ref.counters()[0], acc, None))
    except Exception as e:  # reported by the parent
        barrier.abort()
        q.put((0.0, 0.0, 0, 0.0, 0, repr(e)))


def _port_traj_worker(L, eps, md_steps, seed, ntraj, warm, barrier, q):
    """The same as _ref_traj_worker with the CPU restatement (oracle/gn_oracle.c)
    when the reference's build is absent: its own Gaussian draws, every CG to
    |r| < 1e-10 |b|."""
    try:
        sys.path.insert(0, str(ROOT))
        from oracle.oracle import Port
        port = Port()
        V = L ** 3
        rng = np.random.default_rng(seed)
        sigma = rng.normal(0.0, np.sqrt(2.0 / (NFLAV * BETA_S)), V)
        st = dict(sigma=sigma, sm=port.sigma_mass(L, sigma), P=np.zeros(V), F=np.zeros(V), chi=np.zeros((2, V)),
                  phi=np.zeros((2, V)), X=np.zeros((2, V)), Y=np.zeros((2, V)))
        gp, up = port.replay(rng.normal(size=3 * V * ntraj), rng.uniform(size=ntraj))
        for _ in range(warm):
            port.dirac(L, st["sm"], sigma, 0)
        acc = 0
        barrier.wait()
        t0 = time.monotonic()
        for _ in range(ntraj):
            ok, dH, a, _, _ = port.trajectory(L, BETA_S, eps, md_steps, st, gp, up, tol_med=-1e-10, tol_high=-1e-10)
            acc += int(a)
        t1 = time.monotonic()
        q.put((t0, t1, ntraj, st["iterations"], acc, None))
    except Exception as e:
        barrier.abort()
        q.put((0.0, 0.0, 0, 0.0, 0, repr(e)))


class CpuTrajectories:
    """`ntraj` CPU trajectories spread over `procs` spawned processes (the
    reference is serial: one chain per core, as its own scripts run it).
    start() returns at once; result() waits and gives trajectories per second
    from the common start to the last finish."""

    def __init__(self, L, eps, md_steps, ntraj, procs, warm, seed0=1231):
        import multiprocessing as mp
        self.kind = "reference" if ref_rel_path(L).exists() else "port"
        worker = _ref_traj_worker if self.kind == "reference" else _port_traj_worker
        ctx = mp.get_context("spawn")
        self.procs = max(1, min(procs, ntraj))
        self.barrier = ctx.Barrier(self.procs)
        self.q = ctx.Queue()
        self.ntraj, self.L = ntraj, L
        self.ps = [ctx.Process(target=worker, daemon=True,
                               args=(L, eps, md_steps, seed0 + i, ntraj // self.procs + (i < ntraj % self.procs),
                                     warm, self.barrier, self.q)) for i in range(self.procs)]

    def start(self):
        for p in self.ps:
            p.start()
        return self

    def result(self, timeout=3600.0):
        out = [self.q.get(timeout=timeout) for _ in self.ps]
        for p in self.ps:
            p.join(timeout=60)
        errs = [o[5] for o in out if o[5]]
        if errs:
            raise RuntimeError(f"CPU trajectories failed: {errs[0]}")
        wall = max(o[1] for o in out) - min(o[0] for o in out)
        return {"value": self.ntraj / wall, "wall_s": wall, "kind": self.kind, "cores": self.procs,
                "cg_iterations_per_traj": sum(o[3] for o in out) / self.ntraj,
                "acceptance": sum(o[4] for o in out) / self.ntraj}


def _u1_ref_solve(L, tol, seed=0):
    """One complex CG solve of the reference built with PI_INTERACTION
    (ConjugateGradient..., conjugategradient.c:115, from x = 0) at L on
    b = M chi, to the absolute tolerance tol * |b|: (seconds, iterations)."""
    sys.path.insert(0, str(ROOT))
    from oracle import build_ref
    from oracle.oracle import Ref
    ref = Ref(L, 0, build=False, tag=build_ref.PI_TAG)
    ref.init(1231, BETA_S, 0.05, 10)
    rng = np.random.default_rng(seed)
    V = L ** 3
    ref.set_sigma(rng.normal(0.0, np.sqrt(2.0 / (NFLAV * BETA_S)), V))
    ref.set_pi(rng.normal(0.0, np.sqrt(2.0 / (NFLAV * BETA_S)), V))
    b = ref.dirac(rng.normal(size=V).astype(complex), 0)
    t0 = time.perf_counter()
    _, ok = ref.cg(b, None, tol * float(np.linalg.norm(b)), 1)
    dt = time.perf_counter() - t0
    return dt, ref.counters()[0]


def solves_per_trajectory(md_steps):
    # 2 flavours x (1 initial solve + (2 md_steps + 1) forces), minus the first
    # force, whose start vector is already the solution (conjugategradient.c:16-27)
    return 2 * (1 + 2 * md_steps + 1) - 2


def cpu_line_fields(r, a):
    sample = (f"{r['cores']} process(es) of the {'reference' if r['kind'] == 'reference' else 'CPU restatement'}'s "
              f"serial code, {round(r['value'] * r['wall_s'])} full trajectories (LFMN2VF {a.md_steps} x {a.eps}, "
              f"L={a.L}, every CG to 1e-10 |phi|, {r['cg_iterations_per_traj']:.0f} CG iterations per trajectory), "
              f"wall clock from a common start to the last finish")
    return {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": r["kind"], "sample": sample}


def run_reference(a, world, rank):
    """The reference arm: a.steps trajectories of the reference's own serial
    code on the host cores, one process per core; a.warmup Dirac applies per
    process before the clock starts."""
    if rank != 0:
        return
    ncores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    r = CpuTrajectories(a.L, a.eps, a.md_steps, a.steps, min(ncores, 64), a.warmup).start().result()
    value = r["value"]
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": 1000.0 * r["wall_s"] / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded sigma; the reference's own dSFMT draws)",
            "config": {"workload": f"sigma-HMC LFMN2VF L={a.L} beta_s={BETA_S} steps={a.md_steps} eps={a.eps}, "
                                   f"every CG to |r| < {a.tol:g}|phi|", "l2": "n/a (CPU)",
                       "warmup": f"{a.warmup} Dirac applies per process"},
            "impl": "reference",
            "cpu_baseline": cpu_line_fields(r, a),
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- ours (GPU)
def cuda_events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def run_ours(a, world, rank, local):
    import torch

    import gn_b200 as G
    L, V = a.L, a.L ** 3
    # CPU jobs beside the GPU work (spawned processes, started before the first
    # CUDA call): one reference trajectory on one core (cpu_baseline), and the
    # CPU restatement's force at L = 128 for the mixed-precision case
    cpu_job = l128_job = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu_job = CpuTrajectories(L, a.eps, a.md_steps, 1, 1, a.warmup).start()
    if world == 1 and not a.no_l128:
        l128_job = L128Oracle().start()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    lat = G.Lattice(L, local)
    stream = torch.cuda.ExternalStream(lat.stream, device=dev)
    rng = np.random.default_rng(1231 + rank)
    sigma0 = rng.normal(0.0, np.sqrt(2.0 / (NFLAV * BETA_S)), V)
    nsteps = a.warmup + a.steps
    # draws for every trajectory, resident on the device (value) and pinned on the host (e2e)
    draws_h = torch.empty((nsteps, 3 * V), dtype=torch.float64, pin_memory=True)
    draws_h.numpy()[:] = rng.normal(size=(nsteps, 3 * V))
    draws_d = draws_h.to(dev)
    torch.cuda.synchronize(dev)
    unif = rng.uniform(size=4 * nsteps + 16)
    upos = [0]

    def uniform():
        upos[0] += 1
        return float(unif[(upos[0] - 1) % len(unif)])

    ucb = G.DRAW_FN(uniform)
    params = dict(tol_medium=a.tol, tol_high=a.tol, relative=True)

    def traj_dev(s, prec):
        base = draws_d[s].data_ptr()
        return lat.trajectory_device(base, base + 8 * V, BETA_S, a.eps, a.md_steps, ucb, precision=prec, **params)

    results = {}
    for prec, name in ((G.GN_PREC_MIXED, "mixed"), (G.GN_PREC_FP64, "fp64")):
        clocks = Clocks(local)
        clocks.start()  # sampling from before the warm-up to the end of the timed steps
        lat.load_sigma(sigma0)
        for s in range(a.warmup):  # the same steps as the timed ones (the first flush allocates its buffer)
            lat.flush_l2()
            traj_dev(s, prec)
        l0 = lat.launch_count()
        dist_barrier(world)
        torch.cuda.synchronize(dev)
        clocks.mark()
        e0, e1 = cuda_events()
        e0.record(stream)
        out = []
        for s in range(a.warmup, nsteps):
            lat.flush_l2()
            out.append(traj_dev(s, prec))
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ck = clocks.stop()
        dist_barrier(world)
        ms = e0.elapsed_time(e1)
        ms = dist_max(ms, world, dev)
        results[name] = dict(ms=ms, out=out, clocks=ck, launches=(lat.launch_count() - l0) / a.steps)

    # e2e: host buffers through the C-ABI
    lat.load_sigma(sigma0)
    hv = draws_h.numpy()
    sig_out = np.empty(V)
    sm_out = np.empty(V)
    for s in range(a.warmup):
        lat.write_state(G.GN_F_P, hv[s, :V])
        lat.write_state(G.GN_F_CHI, hv[s, V:])
        lat.trajectory(BETA_S, a.eps, a.md_steps, None, ucb, precision=G.GN_PREC_MIXED, **params)
    dist_barrier(world)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for s in range(a.warmup, nsteps):
        lat.write_state(G.GN_F_P, hv[s, :V])
        lat.write_state(G.GN_F_CHI, hv[s, V:])
        lat.trajectory(BETA_S, a.eps, a.md_steps, None, ucb, precision=G.GN_PREC_MIXED, **params)
        lat.lib.gn_store_sigma(lat.ctx, sig_out.ctypes.data_as(G._dp), sm_out.ctypes.data_as(G._dp))
    torch.cuda.synchronize(dev)
    e2e_s = dist_max(time.perf_counter() - t0, world, dev)

    # dominant kernel: one two-flavour mixed CG solve, events around the kernel
    roof = kernel_roofline(lat, stream, a, G)
    dirac = dirac_roofline(G, stream, dev)
    peaks = load_peaks()
    detail = {}
    detail["batched"] = batched_bench(G, dev, world=world)
    if world == 1:
        lay = (detail["batched"]["layout"]["group_blocks"], detail["batched"]["layout"]["big_min_volume"])
        detail["batched_fp64"] = batched_bench(G, dev, precision=G.GN_PREC_FP64, layout=lay)
        if l128_job is not None:
            detail["l128"] = l128_case(G, dev, oracle=l128_job)
        detail["u1"] = u1_case(G, dev)
        if not a.no_serve:
            detail["serving"] = serve_sweep(G)
    elif not a.no_serve:
        detail["serving_sharded"] = serve_sharded_bench(G, world, dev)
    cpu = None
    if cpu_job is not None:
        cpu = cpu_line_fields(cpu_job.result(), a)

    line = bench_line(a, world, L, V, results, e2e_s, roof, dirac, peaks, cpu, detail)
    if rank == 0:
        if a.detail:
            Path(a.detail).parent.mkdir(parents=True, exist_ok=True)
            Path(a.detail).write_text(json.dumps({"line": line, "detail": detail}, indent=1, default=str))
        print(json.dumps(line), flush=True)
    lat.close()


def bench_line(a, world, L, V, results, e2e_s, roof, dirac, peaks, cpu, detail):
    """The bench's JSON line from the measurements: the contract's keys first,
    then short summaries of the side measurements, the claims (Dirac roofline,
    the FP64 arm, mixed over FP64) last, so that a log tail keeps them.
    results: {"mixed"|"fp64": {"ms", "out", "clocks", "launches"}}; adds the
    per-arm figures to detail."""
    mixed, fp64 = results["mixed"], results["fp64"]
    value = world * a.steps / (mixed["ms"] / 1000.0)
    fp64_rate = world * a.steps / (fp64["ms"] / 1000.0)
    iters = [o["inner_iterations"] for o in mixed["out"]]
    detail["mixed"] = {"inner_iterations_per_traj": statistics.mean(iters),
                       "reliable_updates_per_traj": statistics.mean(o["reliable_updates"] for o in mixed["out"]),
                       "acceptance": statistics.mean(o["accepted"] for o in mixed["out"]),
                       "dH": [round(o["dH"], 6) for o in mixed["out"]]}
    detail["fp64"] = {"cg_iterations_per_traj": statistics.mean(o["cg_iterations"] for o in fp64["out"]),
                      "clocks": fp64["clocks"]}
    detail["roofline"], detail["dirac_roofline"] = roof, dirac
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": mixed["ms"] / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 inner CG, f64 reliable updates and dH", "data": "synthetic (seeded N(0,1) P and chi)",
            "config": {"workload": f"sigma-HMC LFMN2VF L={L} beta_s={BETA_S} {a.md_steps} x eps {a.eps}, "
                                   f"every CG to |r| < {a.tol:g}|phi| (true residual)",
                       "parallelism": f"replicas x{world}", "l2": "flushed (512 MB write) before every trajectory"},
            "clocks": mixed["clocks"],
            "gpu_launches": int(round(mixed["launches"] * a.steps)),
            "e2e": {"value": world * a.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 3 * V * 8,
                    "d2h_bytes_per_step": 2 * V * 8},
            "cpu_baseline": cpu,
            "roofline": roof_json(roof, peaks)}
    line.update(summaries(detail, peaks))
    line["dirac_roofline"] = {"kernel": "dirac_item_kernel M, L=256", "achieved_gbs": round(dirac["gbs"], 1),
                              "frac": round(dirac["gbs"] / peaks["hbm_gbs"], 3)}
    line["fp64"] = {"value": round(fp64_rate, 3), "ms_per_step": round(fp64["ms"] / a.steps, 2)}
    line["mixed_over_fp64"] = round(value / fp64_rate, 3)
    return line


def summaries(d, peaks):
    """Short forms of the side measurements for the bench line."""
    out = {}
    if "batched" in d:
        b, b64 = d["batched"], d.get("batched_fp64")
        out["batched"] = {"mixed_traj_s": round(b["value"], 1),
                          "fp64_traj_s": None if b64 is None else round(b64["value"], 1),
                          "solver_frac": round(b["solver_gbs"] / peaks["hbm_gbs"], 3)}
    if "serving" in d:
        s = d["serving"]
        out["serving"] = {"max_sustained_req_s": s["max_sustained_req_s"],
                          "alone_L64_traj_ms": s.get("standalone_mixed", {}).get("trajectory_L64_ms"),
                          "mixed": [[r["offered_req_per_s"], round(r["throughput_req_per_s"], 1), round(r["p50_ms"]),
                                     round(r["p99_ms"])] for r in s["mixed"]],
                          "cols": "offered/s, done/s, p50 ms, p99 ms"}
    if "serving_sharded" in d:
        s = d["serving_sharded"]
        out["serving"] = {"n_gpus": s["n_gpus"], "offered_req_per_s": s["offered_req_per_s"],
                          "done_req_per_s": round(s["throughput_req_per_s"], 1), "p50_ms": round(s["p50_ms"]),
                          "p99_ms": round(s["p99_ms"])}
    if "l128" in d:
        out["l128"] = [{k: (round(v, 3) if k in ("beta_s", "solve_speedup", "trajectory_speedup") else
                            float(f"{v:.2e}")) for k, v in r.items()
                        if k in ("beta_s", "x_err_vs_oracle", "force_err_vs_oracle", "dH_err_vs_oracle",
                                 "solve_speedup", "trajectory_speedup") and v is not None} for r in d["l128"]["rows"]]
    if "u1" in d:
        out["u1_mixed_speedup"] = [d["u1"]["u1_sigma_mixed_speedup"], d["u1"]["u1_pi_mixed_speedup"]]
    return out


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "src": "measured"}
    return {"hbm_gbs": 6650.0, "src": "fallback"}


def roof_json(r, peaks):
    if r is None:
        return None
    peak = peaks["hbm_gbs"]
    return {"bound": "hbm", "achieved": r["gbs"], "peak": peak, "unit": "GB/s", "frac": r["gbs"] / peak,
            "traffic": r.get("traffic"), "kernel": r["kernel"], "note": r["note"] + f"; peak {peaks['src']}"}


def kernel_roofline(lat, stream, a, G):
    """Persistent CG kernel, mixed precision, 2 flavours, b = the resident phi,
    x = 0, tol 1e-10 relative.  Algorithmic bytes per site (each vector read or
    written once per phase; FP32 words of 4 B, FP64 of 8 B):
      inner iteration  8 + 44 nrhs  (sm twice; A: r, t, p in, p, t out;
                                     B: t, p, x^, r in, x^, r out)
      reliable update  72 per system (C: x, x^ in, t out; D: x, x^, t, b in,
                                      x, x^, r^ out; sm shared)
      start            12 + 28 nrhs (b in; x, x^, r^, p^ out; sm in, sm32 out)
    DRAM traffic per launch from ncu (--case cg64, dram__bytes_read.sum +
    dram__bytes_write.sum of cg_mixed_duo_kernel): the working set stays in L2."""
    V = lat.V
    sm = lat.field_ptr(G.GN_F_SM)
    phi = lat.field_ptr(G.GN_F_PHI)
    x = lat.field_ptr(G.GN_F_X)
    times = []
    for rep in range(4):
        lat.flush_l2()
        e0, e1 = cuda_events()
        e0.record(stream)
        infos, st = lat.cg_device(sm, phi, x, 2, 1, a.tol, 1, True, 0, G.GN_PREC_MIXED)
        e1.record(stream)
        e1.synchronize()
        if rep:
            times.append(e0.elapsed_time(e1))
    ms = statistics.median(times)
    inner = max(i["inner_iterations"] for i in infos)
    ru = sum(i["reliable_updates"] for i in infos)
    nbytes = V * ((8 + 44 * 2) * inner + 72 * ru + 12 + 28 * 2)
    return {"gbs": nbytes / (ms * 1e-3) / 1e9,
            "kernel": "cg_mixed_duo_kernel<1, 1024, 4> (2 flavours as two teams, L=%d)" % lat.L,
            "ms": ms, "bytes": nbytes, "traffic": CG_MIXED_DRAM_BYTES if lat.L == 64 else None,
            "note": f"{inner} inner iterations, {ru} reliable updates, {ms:.3f} ms per launch; working set "
                    f"{(2 * 5 * 4 + 8 * 3) * V / 1e6:.0f} MB is L2-resident within the solve"}


def batched_bench(G, dev, nchains=256, ntraj=2, warmup=1, tune=True, precision=None, layout=None, world=1):
    """The batched ensemble: nchains chains per GPU with L uniform in {8, 12, 16,
    24, 32, 48} (seeded), beta_s on a uniform grid over [0.5, 1.2], LFMN2VF 8 x
    eps 0.08, every solve mixed precision to 1e-10 (true relative residual),
    device Philox draws, one persistent kernel per MD step replayed as a CUDA
    graph.  On N GPUs the N x nchains chains are spread over the ranks by
    gn_shard (each rank its own ensemble; no exchange), so the work per GPU
    stays fixed.  Timed with CUDA events on each rank's ensemble stream over
    `ntraj` trajectories of every chain after `warmup`, the slowest rank's
    time.  Algorithmic bytes: 96 per site per pair of solver iterations (the
    two flavours' FP32 sweeps, 8 + 2 x 44 B)."""
    import torch

    import gn_shard
    prec = G.GN_PREC_MIXED if precision is None else precision
    ntot = nchains * world
    rng = np.random.default_rng(4242)
    Ls = [int(x) for x in rng.choice([8, 12, 16, 24, 32, 48], size=ntot)]
    betas = list(np.linspace(0.5, 1.2, ntot))
    p = G.Ensemble.params(0.08, 8, precision=prec)
    with gn_shard.ShardedEnsemble(Ls, betas, seed=1231, device=dev.index) as e:
        for c in e.mine:
            e.load_sigma(c, np.random.default_rng([4242, c]).normal(0.0, np.sqrt(2.0 / (NFLAV * betas[c])),
                                                                    Ls[c] ** 3))
        if layout is not None:
            e.set_layout(*layout)
        else:
            layout = e.tune(p) if tune else (1, 0)
        e.run(p, warmup)
        e.stats(reset=True)
        st = torch.cuda.ExternalStream(e.ens.stream, device=dev)
        e0, e1 = cuda_events()
        torch.cuda.synchronize(dev)
        dist_barrier(world)
        e0.record(st)
        e.run(p, ntraj)
        e1.record(st)
        e1.synchronize()
        ms = dist_max(e0.elapsed_time(e1), world, dev)
        stats = e.stats()
        info = e.ens.info()
    sites = sum(L ** 3 for L in Ls)
    iters = sum(s["cg_iterations"] for s in stats)
    acc = sum(s["accepted"] for s in stats) / (ntot * ntraj)
    nbytes = sum(L ** 3 * s["cg_iterations"] / 2 * 96 for L, s in zip(Ls, stats))
    return {"metric": f"chain trajectories/s, {nchains} chains per GPU L in {{8..48}}, LFMN2VF 8 x eps 0.08, "
                      "CG to 1e-10",
            "precision": "mixed" if prec == G.GN_PREC_MIXED else "fp64", "n_gpus": world,
            "value": ntot * ntraj / (ms / 1e3), "unit": "traj/s",
            "site_trajectories_per_s": sites * ntraj / (ms / 1e3), "ms_per_ensemble_trajectory": ms / ntraj,
            "chains": ntot, "sites": sites, "acceptance": acc,
            "cg_iterations_per_chain_trajectory": iters / (ntot * ntraj),
            "solver_gbs": nbytes / (ms / 1e3) / 1e9 / world,
            "layout": {"group_blocks": layout[0], "big_min_volume": layout[1]},
            "graph": info["graph"], "launches_per_trajectory": info["launches_per_trajectory"] + 2}


def serve_bench(G, nreq=600, rate=200.0, warm=24, seed=5, precision=None, tiers=None):
    """The serving loop: Poisson arrivals at `rate`/s of requests -- one HMC
    trajectory (70 %), one solve with an N(0, 1) right-hand side (20 %), a
    condensate estimate from 16 Z2 vectors (10 %) -- on 256 resident chains,
    32 for each L in 8, 16, ..., 64 with beta_s uniform in [0.6, 1.1];
    trajectories LFMN2VF 8 x eps 0.08, every solve mixed precision to 1e-10.
    Latency = completion - scheduled arrival (host clock), so queueing counts.
    A warm-up of `warm` requests runs and drains first."""
    prec = G.GN_PREC_MIXED if precision is None else precision
    rng = np.random.default_rng(seed)
    Ls = [L for L in range(8, 65, 8) for _ in range(32)]
    betas = rng.uniform(0.6, 1.1, len(Ls))
    types = (G.GN_REQ_TRAJECTORY, G.GN_REQ_SOLVE, G.GN_REQ_CONDENSATE)
    kw = {} if tiers is None else {"tiers": tiers}
    with G.Server(G.Ensemble.params(0.08, 8, precision=prec), mem_budget_bytes=32e9, seed=seed, **kw) as srv:
        for c, (L, b) in enumerate(zip(Ls, betas)):
            srv.add_chain(L, b, rng.normal(0.0, np.sqrt(2.0 / (NFLAV * b)), L ** 3), stream_id=c)
        for k in range(warm):
            t = types[k % 3]
            srv.submit(int(rng.integers(len(Ls))), t, 16 if t == G.GN_REQ_CONDENSATE else 0)
        srv.drain()
        gaps = rng.exponential(1.0 / rate, nreq)
        kinds = rng.choice(3, size=nreq, p=[0.7, 0.2, 0.1])
        chains = rng.integers(len(Ls), size=nreq)
        t0 = srv.clock() + 0.01
        arrive = t0 + np.cumsum(gaps)
        ids, nxt, steps = [], 0, 0
        while True:
            now = srv.clock()
            while nxt < nreq and arrive[nxt] <= now:
                t = types[kinds[nxt]]
                ids.append(srv.submit(int(chains[nxt]), t, 16 if t == G.GN_REQ_CONDENSATE else 0, arrive[nxt]))
                nxt += 1
            ld = srv.load()
            if ld["running"] == 0 and ld["queued"] == 0:
                if nxt == nreq:
                    break
                time.sleep(max(0.0, arrive[nxt] - srv.clock()))
                continue
            srv.step()
            steps += 1
        info = [srv.request(i) for i in ids]
    lat = np.array([r["t_done"] - r["t_arrival"] for r in info])
    span = max(r["t_done"] for r in info) - arrive[0]  # first arrival to last completion
    out = {"metric": f"serving: p50 / p99 request latency and throughput at Poisson {rate:g}/s (70 % trajectory, "
                     "20 % solve, 10 % condensate x 16 Z2), L in {8..64}, CG to 1e-10",
           "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
           "throughput_req_per_s": nreq / span, "offered_req_per_s": rate, "requests": nreq, "steps": steps,
           "failed": int(sum(r["failed"] for r in info)),
           "precision": "mixed" if prec == G.GN_PREC_MIXED else "fp64"}
    for name, t in (("trajectory", 0), ("solve", 1), ("condensate", 2)):
        lt = np.array([r["t_done"] - r["t_arrival"] for r in info if r["type"] == t])
        if len(lt):
            out[name] = {"n": int(len(lt)), "p50_ms": float(np.percentile(lt, 50) * 1e3),
                         "p99_ms": float(np.percentile(lt, 99) * 1e3)}
    # trajectories by lattice size: median and worst latency
    by_L = {}
    for r in info:
        if r["type"] == 0:
            by_L.setdefault(Ls[r["chain"]], []).append(r["t_done"] - r["t_arrival"])
    out["trajectory_by_L_ms"] = {str(L): [round(float(np.median(v)) * 1e3, 1), round(float(max(v)) * 1e3, 1)]
                                 for L, v in sorted(by_L.items())}
    # the slowest requests: L, type, queueing (arrival to admission), run (admission to completion), ms
    slow = sorted(info, key=lambda r: r["t_done"] - r["t_arrival"])[-5:]
    out["slowest"] = [[Ls[r["chain"]], int(r["type"]), round((r["t_admit"] - r["t_arrival"]) * 1e3, 1),
                       round((r["t_done"] - r["t_admit"]) * 1e3, 1)] for r in slow]
    return out


def serve_sharded_bench(G, world, dev=None, rate_per_gpu=100.0, nreq_per_gpu=300, seed=5):
    """Serving on N GPUs (gn_shard.ShardedServer): 256 chains per GPU (32 per
    L in 8, 16, ..., 64, beta_s uniform in [0.6, 1.1]) spread over the ranks by
    the online balancer, and one Poisson stream at N x rate_per_gpu requests/s
    of serve_bench's mix, replicated on every rank; each rank serves the
    requests on its own chains.  Latency as in serve_bench, on each rank's own
    clock; throughput = all requests over the longest rank's span from the
    first arrival to its last completion.  The records are gathered after the
    run (host objects); nothing crosses between GPUs while it runs."""
    import gn_shard
    rng = np.random.default_rng(seed)
    Ls = [L for L in range(8, 65, 8) for _ in range(32 * world)]
    betas = rng.uniform(0.6, 1.1, len(Ls))
    types = (G.GN_REQ_TRAJECTORY, G.GN_REQ_SOLVE, G.GN_REQ_CONDENSATE)
    nreq, rate = nreq_per_gpu * world, rate_per_gpu * world
    with gn_shard.ShardedServer(G.Ensemble.params(0.08, 8), mem_budget_bytes=32e9, seed=seed,
                                device=int(os.environ.get("LOCAL_RANK", "0")), server_factory=G.Server) as srv:
        for c, (L, b) in enumerate(zip(Ls, betas)):
            srv.add_chain(L, b, lambda L=L, b=b, c=c: np.random.default_rng([seed, c]).normal(
                0.0, np.sqrt(2.0 / (NFLAV * b)), L ** 3))
        gaps = rng.exponential(1.0 / rate, nreq)
        kinds = rng.choice(3, size=nreq, p=[0.7, 0.2, 0.1])
        chains = rng.integers(len(Ls), size=nreq)
        dist_barrier(world)
        t0 = srv.clock() + 0.01
        arrive = t0 + np.cumsum(gaps)
        ids, nxt = [], 0
        while True:
            now = srv.clock()
            while nxt < nreq and arrive[nxt] <= now:
                t = types[kinds[nxt]]
                ids.append(srv.submit(int(chains[nxt]), t, 16 if t == G.GN_REQ_CONDENSATE else 0, arrive[nxt]))
                nxt += 1
            ld = srv.load()
            if ld["running"] == 0 and ld["queued"] == 0:
                if nxt == nreq:
                    break
                time.sleep(max(0.0, arrive[nxt] - srv.clock()))
                continue
            srv.step()
        mine = [srv.request(i) for i in ids if i in srv.req_local]
        span = (max(r["t_done"] for r in mine) - arrive[0]) if mine else 0.0
        recs = srv.gather_requests(ids)
        per_rank = [0] * world
        for r in recs.values():
            per_rank[srv.owner[r["chain"]]] += 1
    span = dist_max(span, world, dev)
    lat = np.array([r["t_done"] - r["t_arrival"] for r in recs.values()])
    return {"metric": f"serving on {world} GPU(s): Poisson {rate:g}/s, {len(Ls)} chains, serve_bench's mix",
            "n_gpus": world, "offered_req_per_s": rate, "requests": nreq,
            "throughput_req_per_s": nreq / span, "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3), "failed": int(sum(r["failed"] for r in recs.values())),
            "requests_per_rank": per_rank}


def serve_standalone(G, precision=None, seed=5):
    """Latency of one request alone on the server (nothing else queued or
    running): a trajectory on a chain of each L in 8..64, a solve and a
    16-vector condensate at L = 64."""
    prec = G.GN_PREC_MIXED if precision is None else precision
    rng = np.random.default_rng(seed)
    Ls = list(range(8, 65, 8))
    out = {}
    with G.Server(G.Ensemble.params(0.08, 8, precision=prec), mem_budget_bytes=32e9, seed=seed) as srv:
        for c, L in enumerate(Ls):
            srv.add_chain(L, 0.85, rng.normal(0.0, np.sqrt(2.0 / (NFLAV * 0.85)), L ** 3), stream_id=c)
        for c in range(len(Ls)):  # warm-up
            srv.submit(c, G.GN_REQ_TRAJECTORY, 0)
        srv.drain()
        for name, t, chains in (("trajectory", G.GN_REQ_TRAJECTORY, range(len(Ls))),
                                ("solve", G.GN_REQ_SOLVE, [len(Ls) - 1]),
                                ("condensate", G.GN_REQ_CONDENSATE, [len(Ls) - 1])):
            for c in chains:
                rid = srv.submit(c, t, 16 if t == G.GN_REQ_CONDENSATE else 0)
                srv.drain()
                r = srv.request(rid)
                out[f"{name}_L{Ls[c]}_ms"] = round((r["t_done"] - r["t_arrival"]) * 1e3, 2)
    return out


def serve_sweep(G, rates=(25.0, 50.0, 75.0, 100.0, 150.0, 200.0), nreq=600):
    """serve_bench at a ladder of offered rates in mixed precision, and at 50/s
    and 200/s in FP64.  max_sustained_req_s: the highest offered rate whose
    completion rate (requests over first arrival to last completion) stays
    within 5 % of it, i.e. where the queue does not grow."""
    mixed = [serve_bench(G, nreq=nreq, rate=r) for r in rates]
    fp64 = [serve_bench(G, nreq=nreq, rate=r, precision=G.GN_PREC_FP64) for r in (50.0, 200.0)]
    sus = [r["offered_req_per_s"] for r in mixed if r["throughput_req_per_s"] >= 0.95 * r["offered_req_per_s"]]
    return {"mixed": mixed, "fp64": fp64, "max_sustained_req_s": max(sus) if sus else None,
            "standalone_mixed": serve_standalone(G)}


def u1_case(G, dev, L=64, md_steps=10, eps=0.05, pi_steps=10, tol=1e-10, reps=2):
    """The U(1) model (PI_INTERACTION) at L = 64: ms per sigma trajectory
    (LFMN2VF md_steps x eps with the complex M, every solve to a true relative
    residual of tol) and per LeapFrog2Pi (pi_steps x eps), in FP64 and in
    mixed precision (FP32 inner iterations, FP64 reliable updates, dH in
    FP64), against the Z2 model's FP64 trajectory on the same sigma and draws.
    Draws resident on the device (gn_trajectory_device; P_pi and chi written
    before the pi trajectory), CUDA events around each trajectory, `reps`
    after one warm-up."""
    import torch
    V = L ** 3
    rng = np.random.default_rng(64)
    sigma = rng.normal(0.0, np.sqrt(2.0 / (NFLAV * BETA_S)), V)
    pi = rng.normal(0.0, np.sqrt(2.0 / (NFLAV * BETA_S)), V)
    draws = torch.tensor(rng.normal(size=3 * V), dtype=torch.float64, device=dev)
    chi_c = np.zeros(4 * V)
    chi_c[0:V], chi_c[2 * V:3 * V] = rng.normal(size=V), rng.normal(size=V)
    ppi = rng.normal(size=V)
    out = {"L": L}
    lat = G.Lattice(L, dev.index)
    stream = torch.cuda.ExternalStream(lat.stream, device=dev)

    def timed(run):
        ts, res = [], None
        for rep in range(reps + 1):
            e0, e1 = cuda_events()
            e0.record(stream)
            res = run()
            e1.record(stream)
            e1.synchronize()
            if rep > 0:
                ts.append(e0.elapsed_time(e1))
        return min(ts), res

    params = dict(tol_medium=tol, tol_high=tol, relative=True)
    cases = (("z2_sigma_trajectory", False, G.GN_PREC_FP64), ("u1_sigma_trajectory", True, G.GN_PREC_FP64),
             ("u1_sigma_trajectory_mixed", True, G.GN_PREC_MIXED))
    for name, u1, prec in cases:
        def run():
            lat.load_sigma(sigma)
            if u1:
                lat.load_pi(pi)
            else:
                lat.set_u1(False)
            base = draws.data_ptr()
            return lat.trajectory_device(base, base + 8 * V, BETA_S, eps, md_steps, None, precision=prec, **params)
        ms, r = timed(run)
        out[name] = {"ms": round(ms, 2), "cg_iterations": r["cg_iterations"], "dH": r["dH"]}

    for name, prec in (("u1_pi_trajectory", G.GN_PREC_FP64), ("u1_pi_trajectory_mixed", G.GN_PREC_MIXED)):
        def run_pi():
            lat.load_sigma(sigma)
            lat.load_pi(pi)
            lat.write_state(G.GN_F_PI_P, ppi)
            lat.write_state(G.GN_F_CHI_C, chi_c)
            return lat.trajectory_pi(BETA_S, eps, pi_steps, None, None, None, tol_high=tol, relative=True,
                                     precision=prec)
        ms, r = timed(run_pi)
        out[name] = {"ms": round(ms, 2), "cg_iterations": r["cg_iterations"], "dH": r["dH"]}
    lat.close()
    for kind in ("sigma", "pi"):
        a, b = out[f"u1_{kind}_trajectory"], out[f"u1_{kind}_trajectory_mixed"]
        out[f"u1_{kind}_mixed_speedup"] = round(a["ms"] / b["ms"], 3)
        out[f"u1_{kind}_mixed_abs_ddH"] = abs(a["dH"] - b["dH"])
    # the reference's own complex solve on one host core, beside ours
    nsol = solves_per_trajectory(md_steps)
    out["gpu_ms_per_solve"] = round(out["u1_sigma_trajectory"]["ms"] / nsol, 3)
    from oracle import build_ref
    if build_ref.lib_path(L, 0, build_ref.PI_TAG).exists():
        t, it = _u1_ref_solve(L, tol)
        out["cpu_reference_one_solve"] = {"s": round(t, 3), "iterations": it, "cores": 1,
                                          "kind": "reference (PI_INTERACTION build)",
                                          "sample": f"one two-plane CG solve from x=0 at L={L} to |r| < {tol:g}|b|"}
    return out


def _l128_fields(beta, L):
    """sigma, the trajectory's draws and chi_0, chi_1 of the L = 128 case, in
    the order they are drawn (also the order tests/golden/make_l128_dH.py uses)."""
    V = L ** 3
    rng = np.random.default_rng(int(beta * 100))
    sigma = rng.normal(0.0, np.sqrt(2.0 / (NFLAV * beta)), V)
    draws = rng.normal(size=3 * V)
    chi = np.stack([rng.normal(size=V) for _ in range(2)])
    return sigma, draws, chi


def _l128_oracle_worker(beta, L, tol, path, q):
    """The CPU restatement's sigma force (ComputeSigmaForce, moleculardynamics.c:631)
    on the L = 128 case's fields: X = (M M^T)^-1 phi from x = 0 and F, at the
    absolute tolerance tol * min_f |phi_f|, the one the GPU's force is given."""
    try:
        sys.path.insert(0, str(ROOT))
        from oracle.oracle import Port
        port = Port()
        sigma, _, chi = _l128_fields(beta, L)
        sm = port.sigma_mass(L, sigma)
        phi = np.stack([port.dirac(L, sm, chi[f], 0) for f in range(2)])
        tol_abs = tol * float(min(np.linalg.norm(phi[0]), np.linalg.norm(phi[1])))
        t0 = time.monotonic()
        F, X, Y, ok, it, calls = port.force(L, beta, sigma, sm, phi, np.zeros((2, L ** 3)), tol_abs)
        np.savez(path, F=F, X=X)
        q.put((beta, path, ok, it, time.monotonic() - t0, None))
    except Exception as e:
        q.put((beta, None, False, 0, 0.0, repr(e)))


class L128Oracle:
    """The oracle side of the L = 128 case: the force and X from the CPU
    restatement (a spawned process per beta_s, about a minute each), and dH of
    one trajectory from the fixture tests/golden/oracle_L128_dH.json (about 15
    CPU minutes per beta_s, made by tests/golden/make_l128_dH.py)."""

    def __init__(self, betas=(0.85,), L=128, tol=1e-10):
        import multiprocessing as mp
        ctx = mp.get_context("spawn")
        self.dir = tempfile.mkdtemp(prefix="gn_l128_")
        self.q = ctx.Queue()
        self.ps = [ctx.Process(target=_l128_oracle_worker, daemon=True,
                               args=(b, L, tol, os.path.join(self.dir, f"b{b}.npz"), self.q)) for b in betas]
        self.res = None
        fx = ROOT / "tests" / "golden" / "oracle_L128_dH.json"
        self.dH = {}
        if fx.exists():
            self.dH = {round(r["beta_s"], 6): r["dH"] for r in json.loads(fx.read_text())["rows"] if r["ok"]}

    def start(self):
        for p in self.ps:
            p.start()
        return self

    def force(self, beta):
        """(X, F, seconds) of the oracle at beta_s, or None if it was not asked for."""
        if self.res is None:
            self.res = {}
            for _ in self.ps:
                b, path, ok, it, dt, err = self.q.get(timeout=1800)
                if err is None and ok:
                    d = np.load(path)
                    self.res[round(b, 6)] = (d["X"], d["F"], dt)
                    os.unlink(path)
            for p in self.ps:
                p.join(timeout=60)
        return self.res.get(round(beta, 6))


def l128_case(G, dev, betas=(0.7, 0.85, 1.0), L=128, md_steps=10, eps=0.05, tol=1e-10, reliable=50, oracle=None):
    """Mixed precision at L = 128 (V = 2,097,152): FP32 fields and inner CG,
    FP64 reliable updates at least every `reliable` iterations, FP64 dH and
    Metropolis.  Per beta_s (sigma ~ N(0, 2/(N_f beta_s)), chi ~ N(0, 1),
    phi = M chi), FP64 and mixed on the same fields:
      - against the FP64 oracle (`oracle`, an L128Oracle): the relative error
        of X = (M M^T)^-1 phi and of the sigma force, both solved to the same
        tolerance, and |dH - dH_oracle| of one trajectory from the same state
        and draws (LFMN2VF md_steps x eps, every solve to 1e-10 |b|);
      - against the GPU's own FP64 path: the relative error of x, of the force
        and of dH;
      - the iteration counts and the solve and trajectory times (CUDA events)."""
    import torch
    rows = []
    V = L ** 3
    for beta in betas:
        sigma, draws_h, chi = _l128_fields(beta, L)
        draws = torch.tensor(draws_h, dtype=torch.float64, device=dev)
        with G.Lattice(L, dev.index) as lat:
            lat.set_reliable_interval(reliable)
            st = torch.cuda.ExternalStream(lat.stream, device=dev)
            lat.load_sigma(sigma)
            sm = lat.store_sigma()[1]
            phi = np.stack([lat.dirac(sm, chi[f], G.GN_OP_M) for f in range(2)])
            row = {"beta_s": beta}
            out = {}
            for prec, name in ((G.GN_PREC_FP64, "fp64"), (G.GN_PREC_MIXED, "mixed")):
                lat.load_sigma(sigma)  # the previous pass's trajectory moved sigma
                lat.write_state(G.GN_F_PHI, phi.reshape(-1))
                e0, e1 = cuda_events()
                e0.record(st)
                infos, stt = lat.cg_device(lat.field_ptr(G.GN_F_SM), lat.field_ptr(G.GN_F_PHI),
                                           lat.field_ptr(G.GN_F_X), 2, 1, tol, 1, True, 0, prec)
                e1.record(st)
                e1.synchronize()
                x = lat.read_state(G.GN_F_X).copy()
                # gn_sigma_force takes the reference's absolute tolerance: the
                # relative 1e-10 of this case, for the smaller of the two |phi_f|
                tol_abs = tol * float(min(np.linalg.norm(phi[0]), np.linalg.norm(phi[1])))
                F, X, Y, finfo, _ = lat.sigma_force(beta, sigma, sm, phi, np.zeros((2, V)), tol_abs,
                                                    precision=prec)
                lat.load_sigma(sigma)
                t0, t1 = cuda_events()
                t0.record(st)
                r = lat.trajectory_device(draws.data_ptr(), draws.data_ptr() + 8 * V, beta, eps, md_steps, None,
                                          tol_medium=tol, tol_high=tol, relative=True, precision=prec)
                t1.record(st)
                t1.synchronize()
                out[name] = dict(x=x, X=X, F=F, dH=r["dH"])
                row[name] = {"iterations": int(max(i["inner_iterations"] for i in infos)),
                             "reliable_updates": int(sum(i["reliable_updates"] for i in infos)),
                             "solve_ms": e0.elapsed_time(e1), "trajectory_ms": t0.elapsed_time(t1),
                             "trajectory_cg_iterations": r["cg_iterations"], "dH": r["dH"]}

            def rerr(u, v):
                return float(np.linalg.norm(u - v) / np.linalg.norm(v))
            row["x_rel_err"] = rerr(out["mixed"]["x"], out["fp64"]["x"])
            row["force_rel_err"] = rerr(out["mixed"]["F"], out["fp64"]["F"])
            row["dH_abs_diff"] = abs(out["mixed"]["dH"] - out["fp64"]["dH"])
            orc = oracle.force(beta) if oracle is not None else None
            if orc is not None:
                Xo, Fo, secs = orc
                for name in ("fp64", "mixed"):
                    row[name]["X_err_vs_oracle"] = rerr(out[name]["X"], Xo)
                    row[name]["force_err_vs_oracle"] = rerr(out[name]["F"], Fo)
                row["x_err_vs_oracle"] = row["mixed"]["X_err_vs_oracle"]
                row["force_err_vs_oracle"] = row["mixed"]["force_err_vs_oracle"]
                row["oracle_force_cpu_s"] = round(secs, 1)
            dHo = oracle.dH.get(round(beta, 6)) if oracle is not None else None
            if dHo is not None:
                row["dH_oracle"] = dHo
                for name in ("fp64", "mixed"):
                    row[name]["dH_err_vs_oracle"] = abs(out[name]["dH"] - dHo)
                row["dH_err_vs_oracle"] = row["mixed"]["dH_err_vs_oracle"]
            row["iteration_overhead"] = row["mixed"]["iterations"] / row["fp64"]["iterations"] - 1.0
            row["solve_speedup"] = row["fp64"]["solve_ms"] / row["mixed"]["solve_ms"]
            row["trajectory_speedup"] = row["fp64"]["trajectory_ms"] / row["mixed"]["trajectory_ms"]
        rows.append(row)
    return {"case": f"mixed precision at L={L}, reliable updates every {reliable} iterations, tol {tol:g}",
            "rows": rows}


def dirac_roofline(G, stream, dev, reps=20, L=256):
    """Dirac M on one FP64 plane at L = 256 (V = 16,777,216): psi, sm and the
    output are 384 MB, three times the L2, so back-to-back launches run from
    HBM (no flush needed); `reps` launches between two CUDA events.
    Algorithmic bytes 3 * 8 * V per launch (psi, sm in; out).  DRAM traffic per
    launch from ncu (--case dirac256, dram__bytes_read.sum + dram__bytes_write.sum)."""
    import torch
    lat = G.Lattice(L, dev.index)
    V = L ** 3
    sm = lat.field_ptr(G.GN_F_SM)
    X = lat.field_ptr(G.GN_F_X)
    Y = lat.field_ptr(G.GN_F_Y)
    torch_stream = torch.cuda.ExternalStream(lat.stream, device=dev)
    for _ in range(3):
        lat.dirac_device(sm, X, Y, 1, G.GN_OP_M)
    times = []
    for rep in range(3):
        e0, e1 = cuda_events()
        e0.record(torch_stream)
        for _ in range(reps):
            lat.dirac_device(sm, X, Y, 1, G.GN_OP_M)
        e1.record(torch_stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) / reps)
    ms = min(times)
    nbytes = 3 * 8 * V
    lat.close()
    return {"gbs": nbytes / (ms * 1e-3) / 1e9, "kernel": f"dirac_item_kernel<2, M> L={L} (inputs 3x L2)", "ms": ms,
            "bytes": nbytes, "traffic": DIRAC256_DRAM_BYTES if L == 256 else None,
            "note": f"{ms * 1e3:.1f} us per launch, {reps} back-to-back launches on 384 MB (> L2)"}


def ens_case(G, dev, nchains=48, ntraj=2):
    """A small batched ensemble for a profiler: nchains chains with L drawn
    from the benchmark's mix {8, 12, 16, 24, 32, 48}, the benchmark's layout
    (teams of 4 blocks for L >= 16), LFMN2VF 8 x 0.08, mixed precision to
    1e-10, launched without the graph: per trajectory the refresh launch, one
    launch per MD step and the final one."""
    rng = np.random.default_rng(4242)
    Ls = [int(x) for x in rng.choice([8, 12, 16, 24, 32, 48], size=nchains)]
    betas = list(np.linspace(0.5, 1.2, nchains))
    p = G.Ensemble.params(0.08, 8)
    with G.Ensemble(Ls, betas, seed=1231) as e:
        for c, (L, b) in enumerate(zip(Ls, betas)):
            e.load_sigma(c, rng.normal(0.0, np.sqrt(2.0 / (NFLAV * b)), L ** 3))
        e.set_layout(4, 16 ** 3)
        e.run(p, ntraj, graph=False)
        st = e.stats()
    return {"chains": nchains, "sites": sum(L ** 3 for L in Ls), "trajectories": ntraj,
            "cg_iterations": sum(s["cg_iterations"] for s in st)}


def kernels_case(G, dev, L=128):
    """One launch of each small kernel of the path at L = 128 (V = 2,097,152;
    an FP64 plane is 16.8 MB; a profiler run with its cache flush between
    passes sees every kernel start cold): sigma
    mass, M, M^T, the sigma force's gather (its CG exits at the start: X is
    given with a tolerance of 1e300), the energy, the condensate's source and
    dot kernels (solves exit at once the same way), and the U(1) model's
    complex-mass M, force and energy."""
    V = L ** 3
    rng = np.random.default_rng(160)
    sigma = rng.normal(0.0, np.sqrt(2.0 / (NFLAV * BETA_S)), V)
    pi = rng.normal(0.0, np.sqrt(2.0 / (NFLAV * BETA_S)), V)
    with G.Lattice(L, dev.index) as lat:
        sm = lat.sigma_mass(sigma)
        psi = rng.normal(size=V)
        lat.dirac(sm, psi, G.GN_OP_M)
        lat.dirac(sm, psi, G.GN_OP_MT)
        phi = rng.normal(size=(2, V))
        X = rng.normal(size=(2, V))
        lat.sigma_force(BETA_S, sigma, sm, phi, X, 1e300)
        lat.energy(BETA_S, sigma, rng.normal(size=V), phi, X)
        lat.condensate(sm, 1e300, np.zeros(V, complex), lambda: float(rng.uniform()))
        lat.load_pi(pi)
        pm = lat.store_pi()[1]
        z = psi + 1j * rng.normal(size=V)
        lat.dirac_u1(sm, pm, z, G.GN_OP_M)
        phic = phi + 1j * rng.normal(size=(2, V))
        Xc = X + 1j * rng.normal(size=(2, V))
        lat.sigma_force_u1(BETA_S, sigma, sm, pm, phic, Xc, 1e300)
        lat.energy_u1(0, BETA_S, sigma, rng.normal(size=V), phic, Xc)
    return {"L": L, "V": V}


def run_case(a):
    """Small cases for ncu: cg64 = one two-flavour CG solve at L=64 in FP64 and in
    mixed precision; dirac128 / dirac256 = 3 Dirac applies at L=128 / 256; traj64 = one
    mixed-precision trajectory at L=64."""
    import torch

    import gn_b200 as G
    dev = torch.device("cuda", 0)
    if a.case in ("dirac128", "dirac256"):
        r = dirac_roofline(G, None, dev, reps=3, L=128 if a.case == "dirac128" else 256)
        print(json.dumps(r))
        return
    if a.case == "l128":
        print(json.dumps(l128_case(G, dev, oracle=L128Oracle().start())))
        return
    if a.case == "u1":
        print(json.dumps(u1_case(G, dev)))
        return
    if a.case == "ens":
        print(json.dumps(ens_case(G, dev)))
        return
    if a.case == "kernels":
        print(json.dumps(kernels_case(G, dev)))
        return
    if a.case == "batched":
        r = batched_bench(G, dev)
        print(json.dumps(r), flush=True)
        lay = (r["layout"]["group_blocks"], r["layout"]["big_min_volume"])
        print(json.dumps(batched_bench(G, dev, precision=G.GN_PREC_FP64, layout=lay)), flush=True)
        return
    if a.case == "serve":
        print(json.dumps(serve_sweep(G)), flush=True)
        return
    if a.case == "serve_sharded":
        print(json.dumps(serve_sharded_bench(G, 1)), flush=True)
        return
    L, V = 64, 64 ** 3
    lat = G.Lattice(L, 0)
    rng = np.random.default_rng(1231)
    lat.load_sigma(rng.normal(0.0, np.sqrt(2.0 / (NFLAV * BETA_S)), V))
    draws = torch.tensor(rng.normal(size=3 * V), dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    if a.case == "traj64":
        r = lat.trajectory_device(draws.data_ptr(), draws.data_ptr() + 8 * V, BETA_S, a.eps, a.md_steps, None,
                                  tol_medium=a.tol, tol_high=a.tol, relative=True, precision=G.GN_PREC_MIXED)
        print(json.dumps(r))
        return
    lat.write_state(G.GN_F_CHI, draws[V:].cpu().numpy())
    lat.dirac_device(lat.field_ptr(G.GN_F_SM), lat.field_ptr(G.GN_F_CHI), lat.field_ptr(G.GN_F_PHI), 2, G.GN_OP_M)
    for prec in (G.GN_PREC_FP64, G.GN_PREC_MIXED):
        infos, st = lat.cg_device(lat.field_ptr(G.GN_F_SM), lat.field_ptr(G.GN_F_PHI), lat.field_ptr(G.GN_F_X), 2, 1,
                                  a.tol, 1, True, 0, prec)
        print(json.dumps({"precision": prec, "status": st, "info": infos}))
    lat.close()


def main():
    a = parse()
    if a.case:
        run_case(a)
        return
    if a.impl == "reference":
        world, rank, local = dist_setup("gloo")
        run_reference(a, world, rank)
    else:
        world, rank, local = dist_setup("nccl")
        run_ours(a, world, rank, local)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
