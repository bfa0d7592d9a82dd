"""Benchmark: registrations/s (+ p50/p99 latency) of the CLAIRE GN-Krylov path.

Workload (default): 128^3 periodic grid, FP32, H2 regularisation beta=1e-3,
nt=8, tricubic SL, GN + PCG (inverse-regularisation preconditioner) +
Armijo, gradient tolerance 1e-2, at most `--maxit` GN iterations.  Inputs
are the seeded synthetic ellipsoid template and random smooth velocity
(claire_b200.synthetic), mR = transport(mT, v).  A step solves one batch of
`--batch` registrations to the stopping test.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1): every rank solves its own batch
(independent problems, no collective on the data path: weak scaling); the
timed region is bracketed by a barrier + synchronize, timed with CUDA events,
and the max over ranks is reported.  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "registrations/s at 128^3 (H2 beta=1e-3, nt=8, gradient reduced 1e-2 or maxit)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--nt", type=int, default=8)
    ap.add_argument("--norm", default="h2")
    ap.add_argument("--beta", type=float, default=1e-3)
    ap.add_argument("--maxit", type=int, default=10)
    ap.add_argument("--opttol", type=float, default=1e-2)
    ap.add_argument("--batch", type=int, default=8, help="registrations per GPU per step")
    ap.add_argument("--no-plain", action="store_true", help="skip the single-problem comparison leg")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--serve", action="store_true",
                    help="serving run instead: Poisson arrivals of mixed grids / norms / weights / nt")
    ap.add_argument("--requests", type=int, default=40, help="--serve: number of requests")
    ap.add_argument("--rate", type=float, default=20.0, help="--serve: arrivals per second")
    ap.add_argument("--slots", type=int, default=4, help="--serve: slots per pool")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default FFT variants (no measurement)")
    ap.add_argument("--fft-variant", type=int, default=-1,
                    help="use this FFT variant for the workload's grid instead of measuring (profiling runs)")
    ap.add_argument("--mixed", action="store_true",
                    help="mixed batch instead: 12 x 64^3 + 12 x 96^3 + 8 x 128^3 (H1 beta=1e-2, nt=4) served "
                         "together against plain one-at-a-time runs")
    ap.add_argument("--mixed-slots", type=int, default=12, help="--mixed: slots per pool")
    ap.add_argument("--conv-norm", default="h1s",
                    help="norm of the converging leg (the reference's synthetic problem; its Newton system carries hd)")
    ap.add_argument("--conv-beta", type=float, default=1e-4, help="beta of the converging leg")
    ap.add_argument("--conv-maxit", type=int, default=50, help="GN iteration cap of the converging leg")
    ap.add_argument("--conv-nt", type=int, default=8, help="time steps of the converging leg")
    ap.add_argument("--no-converge", action="store_true", help="skip the converging leg")
    ap.add_argument("--profile-case", action="store_true",
                    help="small fixed workload for ncu captures: one 128^3 recipe problem, objective, gradient, "
                         "Hessian matvec and preconditioner with FP32 and bf16 images, and a Stokes-model gradient")
    ap.add_argument("--precision", action="store_true",
                    help="bf16-image study instead: 256^3 H2 beta=1e-4 nt=8 with bf16 and FP32 image storage")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
# One process per GPU, independent problems per rank (replicas: no collective
# on the data path); the process group carries only the start / stop barriers,
# the max-over-ranks time and the gathered latencies.  The backend is NCCL on
# GPUs; CLAIRE_B200_DIST_BACKEND=gloo runs the same plumbing on host tensors.
def dist_backend():
    return os.environ.get("CLAIRE_B200_DIST_BACKEND", "nccl")


def dist_init(args=None):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        if dist_backend() == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(dist_backend(), timeout=datetime.timedelta(seconds=600))
    return rank, world, local


def problem_indices(rank, batch):
    """Seeded problem indices of a rank: disjoint across ranks (weak scaling)."""
    return [rank * batch + b for b in range(batch)]


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_list(vals, world):
    if world == 1:
        return list(vals)
    import torch.distributed as dist
    out = [None] * world
    dist.all_gather_object(out, list(vals))
    return [v for part in out for v in part]


# ---------------------------------------------------------------------------
# clocks sampler (nvidia-smi during the timed region)
# ---------------------------------------------------------------------------
class Clocks:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([s.strip() for s in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for i, nm in enumerate(names):
                if len(s) > 5 + i and s[5 + i].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def make_opt(cb, a):
    return cb.RegOpt(["-nx", str(a.n), "-nt", str(a.nt), "-regnorm", a.norm, "-beta", repr(a.beta),
                      "-maxit", str(a.maxit), "-opttol", repr(a.opttol)])


def run_ours(a, rank, world, local):
    import torch
    import claire_b200 as cb
    from claire_b200 import synthetic

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    B = a.batch
    if a.fft_variant >= 0:
        cb.set_fft_variant(a.n, a.fft_variant)
        tuned = {str(a.n): {"variant": a.fft_variant, "set_by": "--fft-variant"}}
    else:
        tuned = None if a.no_autotune else tune(cb, [a.n], B)
    # seeded inputs: problem index = rank*B + b
    probs = [synthetic.ellipsoid_problem(a.n, a.nt, 1, i, dev) for i in problem_indices(rank, B)]
    host = [(p[0].cpu().pin_memory(), p[1].cpu().pin_memory()) for p in probs]
    n = a.n ** 3
    stream = torch.cuda.Stream(device=dev)
    opt = make_opt(cb, a)
    ci = cb.CLAIREInterface(opt, nbatch=B)
    ci.set_stream(stream)
    zero_v = torch.zeros((3, a.n, a.n, a.n), device=dev)

    def load_device():
        for b, (mR, mT, _) in enumerate(probs):
            ci.set_images(mR, mT, b)
            ci.SetInitialGuess(zero_v, b)

    # --- device-resident throughput ---------------------------------------------
    for _ in range(a.warmup):
        load_device()
        ci.Run()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    launches0 = cb.kernel_launches()
    step_ms = []
    with Clocks(local) as clk:
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(a.steps):
            load_device()
            es = torch.cuda.Event(enable_timing=True)
            ee = torch.cuda.Event(enable_timing=True)
            es.record(stream)
            ci.Run()
            ee.record(stream)
            step_ms.append((es, ee))
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = cb.kernel_launches() - launches0
    barrier(world)
    total_ms = ev0.elapsed_time(ev1)
    total_ms = max_over_ranks(total_ms, world)
    lat = [s.elapsed_time(e) for s, e in step_ms]   # every problem of a batch completes with its batch
    lat_all = gather_list([x for x in lat for _ in range(B)], world)
    stats = [ci.stats(b) for b in range(B)]

    # --- e2e through the registration server: host images in, host velocity out ---
    # claire_b200_server_*: one pool of B slots; every step submits the B
    # problems from host buffers, the server copies them in, admits them at a
    # GN-iteration boundary, solves and copies each velocity back when its
    # stopping test fires.  Latency = submit to result, per request.
    host_np = [(h[0].numpy(), h[1].numpy()) for h in host]
    h2d = 2 * n * 4 * B
    d2h = 3 * n * 4 * B
    srv = cb.Server(slots_per_pool=B, idle_ms=600000, device=local)

    def serve_round():
        ids = [srv.submit(opt, mRh, mTh) for mRh, mTh in host_np]
        out = []
        for rid in ids:
            if srv.wait(rid, -1) != cb.REQ_DONE:
                raise RuntimeError("registration request failed")
            out.append(srv.result(rid, (a.n, a.n, a.n)))
        return out

    serve_round()  # creates the pool (allocation outside the timed region)
    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    lat_srv = []
    for _ in range(a.steps):
        lat_srv += [r[2] for r in serve_round()]
    torch.cuda.synchronize()   # the server's pool streams are done: e1 follows all their work
    e1.record(stream)
    torch.cuda.synchronize()
    rounds_ms = max_over_ranks(e0.elapsed_time(e1), world)
    lat_srv = gather_list(lat_srv, world)

    # --- e2e as a stream: all steps x B requests submitted at once ------------
    # the server keeps its B slots full (continuous batching: a slot freed by
    # a finished request takes the next queued one at the following GN-iteration
    # boundary), with every request's host-to-device and device-to-host copies
    # inside the timed region
    barrier(world)
    torch.cuda.synchronize()
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    ids = [srv.submit(opt, mRh, mTh) for _ in range(a.steps) for mRh, mTh in host_np]
    for rid in ids:
        if srv.wait(rid, -1) != cb.REQ_DONE:
            raise RuntimeError("registration request failed")
        srv.result(rid, (a.n, a.n, a.n))
    torch.cuda.synchronize()
    s1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(s0.elapsed_time(s1), world)
    srv.close()

    # --- plain single-problem path (B = 1, same problems one at a time) ----------
    plain = None
    if not a.no_plain:
        ci1 = cb.CLAIREInterface(opt, nbatch=1)
        ci1.set_stream(stream)
        ci1.set_images(probs[0][0], probs[0][1])
        ci1.SetInitialGuess(zero_v)
        ci1.Run()
        torch.cuda.synchronize()
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for b in range(B):
            ci1.set_images(probs[b][0], probs[b][1])
            ci1.SetInitialGuess(zero_v)
            ci1.Run()
        p1.record(stream)
        torch.cuda.synchronize()
        plain_ms = max_over_ranks(p0.elapsed_time(p1), world)
        plain = world * B / (plain_ms / 1e3)
        ci1.close()

    roof = roofline(cb, a, ci, load_device, B) if rank == 0 else None
    ci.close()
    fixed = fixed_work(cb, a, probs, stream, zero_v) if rank == 0 else None
    conv = converging_leg(cb, a, stream, B) if (rank == 0 and not a.no_converge) else None
    return dict(total_ms=total_ms, lat=lat_all, lat_srv=lat_srv, stats=stats, e2e_ms=e2e_ms, rounds_ms=rounds_ms,
                h2d=h2d, d2h=d2h,
                launches=launches, clocks=clk.summary(), plain=plain, roof=roof, tuned=tuned, fixed=fixed,
                conv=conv)


def converging_leg(cb, a, stream, B):
    """Registrations/s to the metric's target: the headline H2 solves never
    reach a relative mismatch of 1e-2 (the H2 gradient lacks the hd of its
    objective), so this leg registers the reference's own synthetic problem
    (-synthetic 0: sin^2 template transported by the trig velocity,
    src/CLAIREBase.cpp:1026-1250) at the same grid with the H1 seminorm, whose
    Newton system carries hd: a batch of B copies solved to the gradient
    tolerance 1e-2, timed with CUDA events; the line states whether every
    problem reached relative mismatch <= 1e-2 and |g| <= 1e-2 |g0|."""
    import torch
    from claire_b200 import synthetic
    dev = torch.device("cuda", torch.cuda.current_device())
    mR, mT, _ = synthetic.sin2_problem(a.n, a.conv_nt, reference_case=True, device=dev)
    zero = torch.zeros((3, a.n, a.n, a.n), device=dev)
    opt = cb.RegOpt(["-nx", str(a.n), "-nt", str(a.conv_nt), "-regnorm", a.conv_norm, "-beta", repr(a.conv_beta),
                     "-maxit", str(a.conv_maxit), "-opttol", "1e-2"])
    ci = cb.CLAIREInterface(opt, nbatch=B)
    ci.set_stream(stream)
    out = None
    for rep in range(2):  # warm-up, then timed
        for b in range(B):
            ci.set_images(mR, mT, b)
            ci.SetInitialGuess(zero, b)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ci.Run()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        st = [ci.stats(b) for b in range(B)]
        out = {"workload": f"{B} registrations of the reference's synthetic problem (-synthetic 0) at {a.n}^3, "
                           f"{a.conv_norm} beta={a.conv_beta} nt={a.conv_nt} maxit={a.conv_maxit} opttol=0.01",
               "value": B / (ms / 1e3), "unit": "registrations/s", "ms": ms,
               "rel_mismatch": max(s["rel_mismatch"] for s in st),
               "grad_reduction": max(s["gnorm"] / s["gnorm0"] for s in st),
               "gn_iterations": st[0]["gn_iterations"], "pcg_iterations": st[0]["pcg_iterations"]}
    out["reaches_target"] = bool(out["rel_mismatch"] <= 1e-2 and out["grad_reduction"] <= 1e-2)
    ci.close()
    return out


def fixed_work(cb, a, probs, stream, zero_v, matvecs=10):
    """Time of one GN iteration with a fixed amount of work: PCG forced to
    `matvecs` iterations (no forcing sequence, relative tolerance 1e-30), no
    early stop; the difference of 2- and 1-iteration solves on the same
    problems.  Unlike registrations/s on this workload it does not move with
    the GN path, so kernel changes compare."""
    import torch
    out = {}
    for B in (len(probs), 1):
        ms, st = {}, {}
        for maxit in (1, 2):
            opt = cb.RegOpt(["-nx", str(a.n), "-nt", str(a.nt), "-regnorm", a.norm, "-beta", repr(a.beta),
                             "-krylovfseq", "none", "-krylovtol", "1e-30", "-krylovmaxit", str(matvecs + 1),
                             "-opttol", "0", "-gabs", "0", "-maxit", str(maxit)])
            ci = cb.CLAIREInterface(opt, nbatch=B)
            ci.set_stream(stream)
            for rep in range(2):  # warm-up, then timed
                for b in range(B):
                    ci.set_images(probs[b][0], probs[b][1], b)
                    ci.SetInitialGuess(zero_v, b)
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                ci.Run()
                e1.record(stream)
                torch.cuda.synchronize()
                ms[maxit] = e0.elapsed_time(e1)
            st[maxit] = ci.stats(0)
            ci.close()
        out["batch_%d" % B] = {
            "gn_iteration_ms": ms[2] - ms[1],
            "hess_matvecs_in_iteration": st[2]["hess_matvecs"] - st[1]["hess_matvecs"],
            "obj_evals_in_iteration": st[2]["obj_evals"] - st[1]["obj_evals"]}
    return out


def tune(cb, sizes, nbatch):
    """FFT variant per grid size by measurement (claire_b200_autotune), before any timing."""
    out = {}
    for n in sizes:
        v, times = cb.autotune(n, nbatch)
        out[str(n)] = {"variant": v, "ms_per_candidate": {str(k): round(t, 4) for k, t in times.items()}}
    return out


# dram__bytes_read.sum + dram__bytes_write.sum of one k_gather_scale launch over
# one 128^3 problem of the workload (42,417,664 bytes; ncu --set full, the
# command in profiles/k_gather_scale_128.md), per point
GATHER_SCALE_DRAM_BYTES_PER_POINT = 42417664 / 128 ** 3
# l1tex__data_pipe_lsu_wavefronts_mem_shared.sum of the same capture (4.29 M
# shared-memory wavefronts for 128^3 points: the 64 taps per point; the box
# arrives by bulk copies, which this counter does not see), per point; a B200
# SM serves one 128-byte wavefront per clock
GATHER_SCALE_SMEM_WAVEFRONTS_PER_POINT = 4.286e6 / 128 ** 3


def roofline(cb, a, ci, load_device, B):
    """Dominant kernel of the registration: the adjoint time step
    k_gather_scale (lambda^{l-1} = c * lambda^l(X), tricubic tile gather).

    One more registration of the timed workload runs with the library's device
    timers on; every adjoint-step launch is bracketed by CUDA events on the
    solve's stream.  Algorithmic bytes per launch (B problems of n points):
    field 4n + displacement 12n + factor c 4n + output 4n = 24n per problem.
    `traffic` is DRAM bytes per launch: GATHER_SCALE_DRAM_BYTES_PER_POINT (an
    ncu capture of the same kernel in the same workload) times the points of
    the launch.
    """
    import torch
    n = a.n ** 3
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    load_device()
    ci.profile(True)
    ci.Run()
    ms, cnt = ci.profile_read(cb.PROF_ADJOINT_STEP)
    pc_ms, pc_cnt = ci.profile_read(cb.PROF_PRECOND)
    # the operations apps/benchmark.cpp of the reference times one by one
    # (src/apps/benchmark.cpp:116-295), here in situ over the batch
    per_op = {}
    for name, cat in (("objective", cb.PROF_OBJECTIVE), ("gradient", cb.PROF_GRADIENT),
                      ("hessian_matvec", cb.PROF_HESSIAN)):
        op_ms, op_cnt = ci.profile_read(cat)
        per_op[name] = {"ms_per_call": round(op_ms / max(op_cnt, 1), 3), "calls": op_cnt}
    ci.profile(False)
    torch.cuda.synchronize()
    avg_ms = ms / max(cnt, 1)
    bytes_ = 24 * n * B
    achieved = bytes_ / (avg_ms / 1e3) / 1e9
    traffic = GATHER_SCALE_DRAM_BYTES_PER_POINT * n * B
    # the bound that binds: shared-memory wavefronts against one per SM per clock
    sm_mhz = float(peaks.get("sm_max_mhz", 1965.0))
    wf = GATHER_SCALE_SMEM_WAVEFRONTS_PER_POINT * n * B
    wf_peak = 148 * sm_mhz * 1e6
    smem = {"what": "shared-memory wavefronts per second against one 128-byte wavefront per SM per clock "
                    f"(148 SMs at {sm_mhz:.0f} MHz)", "wavefronts_per_launch": wf,
            "achieved_per_s": wf / (avg_ms / 1e3), "peak_per_s": wf_peak,
            "frac": round(wf / (avg_ms / 1e3) / wf_peak, 4)}
    # the PCG preconditioner z = P r: one 3-field r2c -> inverse symbol -> c2r
    # over the B problems (5 passes: rows, x2 columns, x1 pencil with the
    # symbol, x2 columns, rows with the r.z epilogue); algorithmic bytes 24n
    # per problem (3 fields in, 3 out)
    pc_avg = pc_ms / max(pc_cnt, 1)
    pc_bytes = 24 * n * B
    spectral = {"what": "z = P r (3-field forward + inverse FFT with the inverse regularisation symbol), "
                        "B problems per launch sequence",
                "avg_us": round(pc_avg * 1e3, 2), "us_per_problem": round(pc_avg * 1e3 / B, 2),
                "algorithmic_bytes": pc_bytes,
                "achieved": round(pc_bytes / (pc_avg / 1e3) / 1e9, 1) if pc_cnt else None,
                "frac": round(pc_bytes / (pc_avg / 1e3) / 1e9 / peak, 4) if pc_cnt else None,
                "applications_timed": pc_cnt}
    return {"kernel": "k_gather_scale (adjoint time step: tricubic tile gather x per-point factor)",
            "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": traffic, "algorithmic_bytes": bytes_,
            "avg_launch_us": round(avg_ms * 1e3, 2), "launches_timed": cnt, "peak_source": peak_src,
            "shared_memory_roofline": smem, "spectral_operator": spectral, "per_op": per_op}


# ---------------------------------------------------------------------------
# CPU legs: the C++/OpenMP restatement of the reference (oracle/cpu_ref.cpp)
# ---------------------------------------------------------------------------
def cpu_cores():
    """Host threads the CPU legs use: every core this process may run on."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_per_op(a, reps=3):
    """Per-operation times of the C++ restatement (FP32, all host cores) on
    the workload's first problem, as apps/benchmark.cpp of the reference
    times them: objective (state solve + distance + regularisation),
    gradient, GN Hessian matvec, at half the problem's true velocity."""
    from oracle import claire_ref as R
    from oracle.cpu_ref import CpuRef
    shape = (a.n,) * 3
    rng = np.random.Generator(np.random.PCG64(R.problem_seed(1, 0)))
    mT = R.template_ellipsoids(shape, rng)
    v = R.velocity_random(shape, rng)
    c = CpuRef(shape, a.nt, a.norm, a.beta, fp64=False, threads=cpu_cores())
    mR = c.forward(v, mT)
    c.set_images(mR, mT)
    vh = 0.5 * v
    vt = 0.1 * v
    out = {}
    # the matvec reuses the state and adjoint of the gradient at vh, as the
    # reference's HessianMatVec does after EvaluateGradient
    for name, fn in (("objective", lambda: c.objective(vh)), ("gradient", lambda: c.gradient(vh)),
                     ("hessian_matvec", lambda: c.hessian_matvec_current(vt))):
        fn()
        t = time.perf_counter()
        for _ in range(reps):
            fn()
        out[name] = round((time.perf_counter() - t) / reps * 1e3, 1)
    c.close()
    return out


def cpu_problem(a, problem_index=0):
    """Inputs of one benchmark problem built on the host (no GPU library):
    the oracle's ellipsoid template and random velocity of the recipe (same
    seeds and draws as claire_b200.synthetic), mR = transport of mT by that
    velocity with the C++ restatement's own semi-Lagrangian solver (FP64)."""
    from oracle import claire_ref as R
    from oracle.cpu_ref import CpuRef
    shape = (a.n,) * 3
    rng = np.random.Generator(np.random.PCG64(R.problem_seed(1, problem_index)))
    mT = R.template_ellipsoids(shape, rng)
    v = R.velocity_random(shape, rng)
    c = CpuRef(shape, a.nt, a.norm, a.beta, fp64=True, threads=cpu_cores())
    mR = c.forward(v, mT)
    c.close()
    return mR, mT


class CpuRegistrations:
    """Registrations of the workload on the C++ restatement in FP32 (the
    reference's single-precision build; its loop structure: 5 nt + 4 scalar
    gathers and 12 nt + 14 3D real transforms per Hessian matvec), on all host
    cores.  A step is one GN iteration; a registration's first step also runs
    its initialisation (J0, ||g0|| at v = 0); the next registration starts
    when the stopping test of the current one fires."""

    def __init__(self, a, mR, mT):
        from oracle.cpu_ref import CpuRef
        self.a = a
        self.cores = cpu_cores()
        self.c = CpuRef((a.n,) * 3, a.nt, a.norm, a.beta, fp64=False, threads=self.cores)
        self.c.set_gn(maxit=a.maxit, gttol=a.opttol)
        self.c.set_images(mR, mT)
        self.fresh = True
        self.done = []       # (seconds, stats) of completed registrations
        self.cur_s = 0.0

    def step(self):
        t = time.perf_counter()
        if self.fresh:
            self.c.reset_counters()
            self.c.begin()
            self.fresh = False
        finished = self.c.step()
        if finished:
            self.c.finish()
        dt = time.perf_counter() - t
        self.cur_s += dt
        if finished:
            self.done.append((self.cur_s, self.c.stats()))
            self.cur_s = 0.0
            self.fresh = True
        return dt

    def summary(self, elapsed, gn_done):
        """registrations/s: completed registrations over their own seconds; with
        none completed, GN iterations per second over maxit (flagged)."""
        if self.done:
            secs = [d[0] for d in self.done]
            value = len(secs) / sum(secs)
            partial = False
        else:
            value = gn_done / elapsed / self.a.maxit
            partial = True
        st = [d[1] for d in self.done]
        work = {k: float(np.mean([s[k] for s in st])) for k in
                ("iters", "pcg_iters", "hess_matvecs", "pc_matvecs", "obj_evals", "grad_evals", "gathers",
                 "ffts")} if st else None
        return value, partial, {"registrations_completed": len(self.done),
                                "seconds_per_registration": [round(d[0], 3) for d in self.done],
                                "work_per_registration": work,
                                "rel_mismatch": [round(s["rel_mismatch"], 6) for s in st],
                                "extrapolated_from_gn_iterations": partial}

    def close(self):
        self.c.close()


def cpu_baseline_sample(a, budget_s=20.0):
    """cpu_baseline of our line: one registration of the workload on the C++
    restatement (FP32, all host cores), GN iterations until it finishes or
    `budget_s` has passed.  An unfinished run is extrapolated as GN iterations
    per second over maxit: the first GN iterations carry the fewest Krylov
    iterations (forcing sequence), so that figure overstates the CPU's speed."""
    mR, mT = cpu_problem(a)
    reg = CpuRegistrations(a, mR, mT)
    t0 = time.perf_counter()
    gn = 0
    while time.perf_counter() - t0 < budget_s:
        reg.step()
        gn += 1
        if reg.done:
            break
    elapsed = time.perf_counter() - t0
    value, partial, info = reg.summary(elapsed, gn)
    reg.close()
    what = ("one complete registration" if not partial else
            f"the first {gn} GN iterations of one registration ({elapsed:.1f} s), extrapolated to maxit={a.maxit}")
    return {"value": value, "unit": "registrations/s", "cores": reg.cores, "kind": "port",
            "sample": f"C++/OpenMP FP32 restatement of the reference (oracle/cpu_ref.cpp, reference loop "
                      f"structure) on {reg.cores} host threads ({cpu_model()}), {a.n}^3 {a.norm} nt={a.nt}: "
                      + what, **info}


def run_reference(a, rank, world):
    """Reference arm: the reference's CPU path as restated in C++ (the
    reference itself needs MPI, PETSc 3.9.1, AccFFT and FFTW, none of which is
    here), timed on the host cores.  Rank 0 only; W warm-up GN iterations of
    one registration, then K timed GN iterations of fresh registrations."""
    if rank != 0:
        return
    mR, mT = cpu_problem(a)
    warm = CpuRegistrations(a, mR, mT)
    for _ in range(a.warmup):
        warm.step()
    warm.close()
    reg = CpuRegistrations(a, mR, mT)
    times = [reg.step() for _ in range(a.steps)]
    elapsed = sum(times)
    value, partial, info = reg.summary(elapsed, len(times))
    cores = reg.cores
    reg.close()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "registrations/s", "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": elapsed * 1e3 / max(1, a.steps),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"single registrations {a.n}^3 {a.norm} beta={a.beta} nt={a.nt} maxit={a.maxit} "
                               f"opttol={a.opttol}, one after another; a step is one GN iteration",
                   "n": a.n, "nt": a.nt, "regnorm": a.norm, "beta": a.beta, **info},
        "cpu_baseline": {"value": value, "unit": "registrations/s", "cores": cores, "kind": "port",
                         "sample": f"C++/OpenMP FP32 restatement of the reference's CPU path (oracle/cpu_ref.cpp) "
                                   f"on {cores} host threads ({cpu_model()}): {a.steps} GN iterations of "
                                   "real registrations of the workload"},
        "e2e": {"value": value, "unit": "registrations/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# serving run (--serve): Poisson stream of mixed registration requests
# ---------------------------------------------------------------------------
EDGES = (64, 96, 128, 192, 256)


def serve_requests(a, rank):
    """Request mix: exponential inter-arrival at `rate`; grid edge u ~ U[ln 64,
    ln 256] snapped to the nearest of EDGES in log space; norm H1 or H2; beta
    log-uniform in [1e-4, 1e-2]; nt 4 or 8; per-request seeded ellipsoid /
    random-velocity images (config index 5)."""
    rng = np.random.Generator(np.random.PCG64(20261203 + 5000 + rank))
    t = 0.0
    out = []
    logs = np.log(np.array(EDGES, dtype=np.float64))
    for i in range(a.requests):
        t += rng.exponential(1.0 / a.rate)
        u = rng.uniform(np.log(64.0), np.log(256.0))
        edge = int(EDGES[int(np.argmin(np.abs(logs - u)))])
        norm = "h1" if rng.uniform() < 0.5 else "h2"
        beta = float(np.exp(rng.uniform(np.log(1e-4), np.log(1e-2))))
        nt = 4 if rng.uniform() < 0.5 else 8
        out.append({"t": t, "n": edge, "norm": norm, "beta": beta, "nt": nt, "idx": rank * a.requests + i})
    return out


def run_serve(a, rank, world, local):
    import threading as th
    import torch
    import claire_b200 as cb
    from claire_b200 import synthetic

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    tuned = None if a.no_autotune else tune(cb, list(EDGES), a.slots)
    reqs = serve_requests(a, rank)
    for r in reqs:  # inputs are built before the timed run (setup, not served work)
        mR, mT, _ = synthetic.ellipsoid_problem(r["n"], r["nt"], 5, r["idx"], dev)
        r["mR"], r["mT"] = mR.cpu().numpy(), mT.cpu().numpy()
        r["opt"] = cb.RegOpt(["-nx", str(r["n"]), "-nt", str(r["nt"]), "-regnorm", r["norm"], "-beta",
                              repr(r["beta"]), "-maxit", str(a.maxit), "-opttol", repr(a.opttol)])
    torch.cuda.synchronize()
    srv = cb.Server(slots_per_pool=a.slots, idle_ms=5000, device=local)
    ids = [None] * len(reqs)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()

    def submitter():
        for i, r in enumerate(reqs):
            d = r["t"] - (time.perf_counter() - t0)
            if d > 0:
                time.sleep(d)
            ids[i] = srv.submit(r["opt"], r["mR"], r["mT"])

    sub = th.Thread(target=submitter)
    sub.start()
    sub.join()
    lats, stats = [], []
    for i, r in enumerate(reqs):
        if srv.wait(ids[i], -1) != cb.REQ_DONE:
            raise RuntimeError("registration request failed")
        _, st, lat = srv.result(ids[i], (r["n"],) * 3)
        lats.append(lat)
        stats.append(st)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    srv.close()
    wall = max_over_ranks(wall, world)
    lats = gather_list(lats, world)
    if rank != 0:
        return
    ls = sorted(lats)
    total = len(ls)
    line = {
        "metric": "served registrations/s and p50/p99 latency (mixed Poisson stream)",
        "value": total / wall, "unit": "registrations/s", "n_gpus": world, "steps": 1, "warmup": 0,
        "ms_per_step": wall * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{a.requests} requests per GPU, Poisson {a.rate}/s, edges {list(EDGES)} "
                               f"log-uniform, H1/H2, beta log-U[1e-4,1e-2], nt 4|8, maxit {a.maxit}",
                   "slots_per_pool": a.slots,
                   "edge_counts": {str(e): sum(1 for r in reqs if r["n"] == e) for e in EDGES}},
        "latency_ms": {"p50": float(np.percentile(ls, 50)), "p99": float(np.percentile(ls, 99)),
                       "max": float(ls[-1])},
        "timing": "wall clock from the first arrival to the last result (host-to-host, includes queueing)",
        "mean_gn_iterations": float(np.mean([s["gn_iterations"] for s in stats])),
        "fft_variants": tuned or "defaults (--no-autotune)",
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# mixed batch (--mixed): 32 registrations of uneven sizes
# ---------------------------------------------------------------------------
MIXED = [64] * 12 + [96] * 12 + [128] * 8


def run_mixed(a, rank, world, local):
    """12 x 64^3 + 12 x 96^3 + 8 x 128^3, H1 beta=1e-2 (beta1=1e-4), nt=4,
    seeded ellipsoid / random-velocity recipe (config index 2), all submitted
    at once to the registration server (one pool per size, concurrent streams)
    and, for comparison, solved one at a time by plain single-problem contexts
    (one per size, created before timing).  Both legs are timed on the device
    (events around the whole batch, synchronised)."""
    import torch
    import claire_b200 as cb
    from claire_b200 import synthetic

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    nt, norm, beta = 4, "h1", 1e-2
    tuned = None if a.no_autotune else tune(cb, sorted(set(MIXED)), a.mixed_slots)
    probs = []
    for i, n in enumerate(MIXED):
        mR, mT, _ = synthetic.ellipsoid_problem(n, nt, 2, rank * len(MIXED) + i, dev)
        probs.append((n, mR, mT, mR.cpu().numpy(), mT.cpu().numpy()))
    opts = {n: cb.RegOpt(["-nx", str(n), "-nt", str(nt), "-regnorm", norm, "-beta", repr(beta),
                          "-maxit", str(a.maxit), "-opttol", repr(a.opttol)]) for n in sorted(set(MIXED))}
    stream = torch.cuda.Stream(device=dev)
    srv = cb.Server(slots_per_pool=a.mixed_slots, idle_ms=600000, device=local)

    def serve_all():
        ids = [srv.submit(opts[n], mRh, mTh) for n, _, _, mRh, mTh in probs]
        out = []
        for (n, *_), rid in zip(probs, ids):
            if srv.wait(rid, -1) != cb.REQ_DONE:
                raise RuntimeError("registration request failed")
            out.append(srv.result(rid, (n, n, n)))
        return out

    serve_all()  # pools are created (and their memory allocated) before timing
    with Clocks(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = serve_all()
        torch.cuda.synchronize()
        e1.record(stream)
        torch.cuda.synchronize()
    served_ms = max_over_ranks(e0.elapsed_time(e1), world)
    lats = gather_list([r[2] for r in res], world)
    srv.close()

    ctx = {n: cb.CLAIREInterface(opts[n], nbatch=1) for n in opts}
    zero = {n: torch.zeros((3, n, n, n), device=dev) for n in opts}
    for c in ctx.values():
        c.set_stream(stream)

    def plain_all():
        for n, mR, mT, _, _ in probs:
            ctx[n].set_images(mR, mT)
            ctx[n].SetInitialGuess(zero[n])
            ctx[n].Run()

    for n, mR, mT, _, _ in probs[::12]:  # one warm run per size
        ctx[n].set_images(mR, mT)
        ctx[n].SetInitialGuess(zero[n])
        ctx[n].Run()
    barrier(world)
    torch.cuda.synchronize()
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    plain_all()
    p1.record(stream)
    torch.cuda.synchronize()
    plain_ms = max_over_ranks(p0.elapsed_time(p1), world)
    for c in ctx.values():
        c.close()
    if rank != 0:
        return
    total = world * len(MIXED)
    ls = sorted(lats)
    line = {
        "metric": "registrations/s, mixed batch (12 x 64^3 + 12 x 96^3 + 8 x 128^3, H1 beta=1e-2, nt=4)",
        "value": total / (served_ms / 1e3), "unit": "registrations/s", "n_gpus": world, "steps": 1,
        "warmup": 1, "ms_per_step": served_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "32 registrations per GPU of uneven sizes through the registration server "
                               f"(one pool per size, {a.mixed_slots} slots), maxit {a.maxit}, opttol {a.opttol}",
                   "plain_single_problem_value": total / (plain_ms / 1e3),
                   "served_over_plain": plain_ms / served_ms,
                   "latency_ms": {"p50": float(np.percentile(ls, 50)), "p99": float(np.percentile(ls, 99)),
                                  "what": "per request, submit of host images to host velocity, all 32 "
                                          "submitted at once"},
                   "mean_gn_iterations": float(np.mean([r[1]["gn_iterations"] for r in res])),
                   "mean_pcg_iterations": float(np.mean([r[1]["pcg_iterations"] for r in res])),
                   "fft_variants": tuned or "defaults (--no-autotune)"},
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# bf16 image storage study (--precision): 256^3 H2 beta=1e-4 nt=8
# ---------------------------------------------------------------------------
def run_precision(a, rank, world, local):
    """One 256^3 problem (ellipsoid recipe, config index 3) with bf16 and with
    FP32 image storage.  Errors of the bf16 storage are measured per operation
    at one fixed velocity (half the recipe's velocity; random direction for the
    Hessian): distance, relative mismatch, body force (the data part of the
    gradient), gradient, GN Hessian matvec and transported image, each against
    the FP32-image result on the same GPU (the device has no FP64 path; the
    FP64 oracle's agreement with both formats is tested at 32^3).  Both
    formats then solve the registration; with H2's gradient lacking the hd
    factor of its objective the GN path of this problem is sensitive to any
    perturbation, so the two solves are reported side by side, not differenced."""
    import torch
    import claire_b200 as cb
    from claire_b200 import synthetic

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n, nt, norm, beta = 256, 8, "h2", 1e-4
    tuned = None if a.no_autotune else tune(cb, [n], 1)
    mR, mT, vrec = synthetic.ellipsoid_problem(n, nt, 3, rank, dev)
    v = (0.5 * vrec).cpu().numpy()
    vt = np.random.default_rng(3).standard_normal(v.shape).astype(np.float32) * float(np.std(v))
    torch.cuda.synchronize()
    out = {}
    for tag, extra in (("fp32", []), ("bf16", ["-bf16images"])):
        opt = cb.RegOpt(["-nx", str(n), "-nt", str(nt), "-regnorm", norm, "-beta", repr(beta), "-maxit",
                         str(a.maxit), "-opttol", repr(a.opttol)] + extra)
        with cb.CLAIREInterface(opt) as ci:
            stream = torch.cuda.Stream(device=dev)
            ci.set_stream(stream)
            ci.set_images(mR, mT)
            r = {"bytes": ci.footprint_bytes()}
            r["J"], r["D"], _ = ci.EvaluateObjective(v)
            r["g"] = ci.EvaluateGradient(v)
            r["bf"] = ci.GetAdjoint()[1]
            r["H"] = ci.HessianMatVec(v, vt)
            ci.SetInitialGuess(v)
            r["m1"] = ci.GetFinalState()
            ci.SetInitialGuess(np.zeros_like(v))
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ci.Run()
            e1.record(stream)
            torch.cuda.synchronize()
            r["ms"] = e0.elapsed_time(e1)
            r["stats"] = ci.stats()
            out[tag] = r
        torch.cuda.synchronize()
    if rank != 0:
        return

    def rel(x, y):
        x = np.asarray(x, np.float64)
        y = np.asarray(y, np.float64)
        return float(np.linalg.norm((x - y).ravel()) / max(np.linalg.norm(y.ravel()), 1e-300))

    f, h = out["fp32"], out["bf16"]
    mRn, mTn = mR.cpu().numpy().astype(np.float64), mT.cpu().numpy().astype(np.float64)
    den = np.linalg.norm((mRn - mTn).ravel())
    mis = {k: float(np.linalg.norm((mRn - out[k]["m1"]).ravel()) / den) for k in out}

    def solve(r):
        st = r["stats"]
        return {"ms": r["ms"], "gn_iterations": st["gn_iterations"], "pcg_iterations": st["pcg_iterations"],
                "rel_mismatch": st["rel_mismatch"], "grad_reduction": st["gnorm"] / st["gnorm0"],
                "reason": st["converged_reason"]}

    line = {
        "metric": "256^3 registration with bf16 image storage: per-operation error against FP32 images, and time",
        "value": h["ms"], "unit": "ms", "n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": h["ms"],
        "higher_is_better": False, "scaling": "none", "vs_baseline": None, "dtype": "bf16 images / f32 / f64 dots",
        "data": "synthetic",
        "config": {"workload": f"256^3 h2 beta=1e-4 nt=8 maxit={a.maxit} opttol={a.opttol}, ellipsoid recipe",
                   "footprint_bytes": {"fp32": f["bytes"], "bf16": h["bytes"]},
                   "errors_vs_fp32_images_at_fixed_velocity": {
                       "objective": abs(h["J"] - f["J"]) / abs(f["J"]),
                       "distance": abs(h["D"] - f["D"]) / abs(f["D"]),
                       "rel_mismatch": abs(mis["bf16"] - mis["fp32"]) / mis["fp32"],
                       "transported_image_rel_l2": rel(h["m1"], f["m1"]),
                       "body_force_rel_l2": rel(h["bf"], f["bf"]),
                       "gradient_rel_l2": rel(h["g"], f["g"]),
                       "hessian_matvec_rel_l2": rel(h["H"], f["H"])},
                   "solve": {"fp32": solve(f), "bf16": solve(h)},
                   "fft_variants": tuned or "defaults (--no-autotune)",
                   "reference_for_errors": "the FP32-image result on the same GPU (no FP64 device path)"},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def run_profile_case(a, local):
    """Every kernel of the path once or twice on one 128^3 problem (a few GB on
    the device): the workload the committed ncu summaries capture."""
    import torch
    import claire_b200 as cb
    from claire_b200 import synthetic
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if a.fft_variant >= 0:
        cb.set_fft_variant(a.n, a.fft_variant)
    mR, mT, v = synthetic.ellipsoid_problem(a.n, a.nt, 1, 0, dev)
    vh = (0.5 * v).cpu().numpy()
    vt = (0.1 * v).cpu().numpy()
    for extra in ([], ["-bf16images"]):
        opt = cb.RegOpt(["-nx", str(a.n), "-nt", str(a.nt), "-regnorm", a.norm, "-beta", repr(a.beta)] + extra)
        with cb.CLAIREInterface(opt) as ci:
            ci.set_images(mR, mT)
            for _ in range(2):
                ci.EvaluateObjective(vh)
                ci.EvaluateGradient(vh)
                ci.HessianMatVec(vh, vt)
                ci.ApplyInvRegularizationOperator(vt)
    opt = cb.RegOpt(["-nx", str(a.n), "-nt", str(a.nt), "-regnorm", "h1s", "-beta", "1e-2"]).set("model", "stokes")
    with cb.CLAIREInterface(opt) as ci:
        ci.set_images(mR, mT)
        ci.EvaluateObjective(vh)
        ci.EvaluateGradient(vh)
    torch.cuda.synchronize()
    print(json.dumps({"profile_case": "done", "n": a.n, "nt": a.nt}), flush=True)


def main():
    a = parse()
    rank, world, local = dist_init(a)
    if a.impl == "reference":
        run_reference(a, rank, world)
        return
    if a.serve:
        run_serve(a, rank, world, local)
        return
    if a.mixed:
        run_mixed(a, rank, world, local)
        return
    if a.precision:
        run_precision(a, rank, world, local)
        return
    if a.profile_case:
        run_profile_case(a, local)
        return
    r = run_ours(a, rank, world, local)
    if rank != 0:
        return
    B = a.batch
    regs = world * B * a.steps
    value = regs / (r["total_ms"] / 1e3)
    lat = sorted(r["lat"])
    p50 = float(np.percentile(lat, 50))
    p99 = float(np.percentile(lat, 99))
    ls = sorted(r["lat_srv"])
    s50 = float(np.percentile(ls, 50))
    s99 = float(np.percentile(ls, 99))
    st0 = r["stats"][0]
    cpu = None if a.no_cpu else cpu_baseline_sample(a)
    # per-operation table (the reference's apps/benchmark.cpp operations): the
    # device's in-situ calls over the batch beside the CPU restatement's
    per_op = None
    if r["roof"] is not None:
        dev = r["roof"].pop("per_op", None)
        per_op = {"device_ms_per_call": dev, "problems_per_device_call": B,
                  "what": "device: mean CUDA-event time per call in the timed registration of the roofline leg "
                          "(line-search objectives cover the problems still searching); cpu: the C++ FP32 "
                          "restatement on one problem"}
        if not a.no_cpu:
            cpu_ops = cpu_per_op(a)
            per_op["cpu_ms_per_problem"] = cpu_ops
            if dev:
                per_op["cpu_over_device_per_problem"] = {
                    k: round(cpu_ops[k] / (dev[k]["ms_per_call"] / B), 1) for k in cpu_ops
                    if dev.get(k) and dev[k]["ms_per_call"] > 0}
    line = {
        "metric": METRIC, "value": value, "unit": "registrations/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": r["total_ms"] / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"batched registrations {a.n}^3 {a.norm} beta={a.beta} nt={a.nt} "
                               f"maxit={a.maxit} opttol={a.opttol}, {B} per GPU per step",
                   "n": a.n, "nt": a.nt, "regnorm": a.norm, "beta": a.beta, "batch_per_gpu": B,
                   "parallelism": f"independent problems, {world} GPU(s)",
                   "l2": "inputs larger than L2 (per-problem working set ~1 GB), no flush between steps",
                   "latency_ms": {"p50": p50, "p99": p99, "what": "batched step, device-resident inputs"},
                   "served_latency_ms": {"p50": s50, "p99": s99,
                                         "what": "per request through the registration server, submitted in "
                                                 f"rounds of {B} (each round waits for its results): submit of "
                                                 "host images to host velocity"},
                   "served_rounds_value": regs / (r["rounds_ms"] / 1e3),
                   "plain_single_problem_value": r["plain"],
                   "gn_iterations": st0["gn_iterations"], "pcg_iterations": st0["pcg_iterations"],
                   "rel_mismatch": st0["rel_mismatch"], "grad_reduction": st0["gnorm"] / st0["gnorm0"],
                   # the H2 gradient's missing hd makes the GN path of this workload sensitive to
                   # roundoff; work per registration is reported so runs compare on equal terms
                   "work_per_registration": {k: float(np.mean([s[k] for s in r["stats"]])) for k in
                                             ("gn_iterations", "pcg_iterations", "hess_matvecs", "pc_matvecs",
                                              "obj_evals", "grad_evals")},
                   "hess_matvecs_per_s": float(sum(s["hess_matvecs"] for s in r["stats"]) * world * a.steps
                                               / (r["total_ms"] / 1e3)),
                   "fft_variants": r["tuned"] or "defaults (--no-autotune)",
                   "fixed_work": r["fixed"],
                   "per_op": per_op,
                   "converging": r["conv"]},
        "e2e": {"value": regs / (r["e2e_ms"] / 1e3), "unit": "registrations/s",
                "h2d_bytes_per_step": r["h2d"], "d2h_bytes_per_step": r["d2h"],
                "path": f"claire_b200_server_submit / _wait / _result (host buffers): {a.steps} x {B} requests "
                        "submitted at once, served by continuous batching in one pool of "
                        f"{B} slots"},
        "roofline": r["roof"],
        "cpu_baseline": cpu,
        "clocks": r["clocks"],
        "gpu_launches": r["launches"],
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
