"""Benchmark: force evaluations per second on the 400k-cylinder network.

A step is one force evaluation in the reference's updateMechanics sense
(src/Controller/MController.h:214-230): the total energy and the forces of all
force fields (filament stretching and bending, linker, motor, branching,
cylinder excluded volume, boundary) at one set of coordinates. The workload
is 20,000 filaments x 20 cylinders in a 10 um cube with 100k linkers, 10k
motors and 5k branch points; excluded-volume and boundary interactions come
from the device neighbor list (54 nm cutoff).

value: steps/s with coordinates resident in HBM, L2 flushed (256 MiB write)
before every timed step, device time from CUDA events on the library's stream.
e2e: the same step through the C ABI from page-locked host buffers:
coordinates in, energies and forces out, every step's copies inside the timed
region. The steps go through medyan_mech_evaluate_async, which overlaps one
step's inbound copy with the previous step's pass and outbound copy (two
staging slots); e2e.sync is the synchronous medyan_mech_evaluate, one step at
a time.

--impl reference times the reference's own compiled CPU kernels
(oracle/_ref/libmedyan_ref.so, one thread: the reference is single-threaded)
on the same workload.

Multi-GPU: replicas only (each rank evaluates its own copy; no collective on
the path), value = all ranks' steps / max rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "CG minimizations/s & force-evals/s, mixed vs FP64 GPU at rel force err ≤1e-6"
WORKLOAD = "cfg4_400k_cylinders_20000x20_10um"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-minimize", action="store_true", help="skip the minimization extras")
    ap.add_argument("--cpu-sample-s", type=float, default=15.0)
    ap.add_argument("--cpu-ensemble", action="store_true",
                    help="only the host baseline of the batched ensemble (one JSON line; used by the bench itself)")
    return ap.parse_args()


# ----------------------------------------------------------------- workload
def build_network():
    from medyan_b200.network import make_workload
    return make_workload(4)


def algorithmic_bytes(ff_counts: dict, n_beads: int) -> dict:
    """Compulsory traffic of one energy pass and one force pass: each bead's
    coordinates read once (24 B), forces written once (24 B), each
    interaction's int32 bead offsets and FP64 parameters read once."""
    per = {"stretch": 2 * 4 + 2 * 8, "bend": 3 * 4 + 2 * 8, "linker": 4 * 4 + 4 * 8, "motor": 4 * 4 + 4 * 8,
           "branch": (3 * 4 + 3 * 8) + (4 * 4 + 2 * 8) + (4 * 4 + 2 * 8), "excl": 4 * 4 + 3 * 8,
           "boundary": 1 * 4 + 2 * 8}
    inter = sum(per[k] * ff_counts.get(k, 0) for k in per)
    coords = 24 * n_beads
    return {"energy": inter + coords, "forces": inter + coords + 24 * n_beads,
            "step": 2 * inter + 2 * coords + 24 * n_beads}


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[4 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------ multi-rank
def max_over_ranks(t: float, world: int, device: str) -> float:
    """The largest of every rank's t (each rank runs its own replica; the
    job's time is the slowest rank's). Every rank calls this the same number
    of times, in the same order."""
    if world <= 1:
        return t
    import torch
    import torch.distributed as dist
    tt = torch.tensor([t], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


# ---------------------------------------------------------------- our arm
def run_ours(args, rank: int, world: int) -> dict:
    import ctypes as C

    import numpy as np
    import torch

    from medyan_b200.forcefield import ForceFieldManager, conjugate_gradient_params

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    net = build_network()
    x = net.flat_coords()
    bp, planes = net.boundary_params()

    def make_for(nw, prec):
        bpn, _ = nw.boundary_params()
        ff = ForceFieldManager(prec)
        ff.vectorize_all_force_fields(nw.system_view())
        ff.set_coords(nw.flat_coords())
        ff.set_cylinders(nw.cylinders_view(), nw.nl_params(), bpn)
        ff.rebuild_neighbor_lists()
        ff.lib.medyan_mech_synchronize(ff.handle)
        # block and tile shapes per potential for this network (autotuner,
        # at setup, outside every timed region)
        ff.tuned_shapes = ff.autotune(reps=10)
        return ff

    def make(prec):
        return make_for(net, prec)

    ff = make(args.precision)
    L, h = ff.lib, ff.handle
    ne, nb = ff.rebuild_neighbor_lists()
    counts = {"stretch": net.ff["stretch_beads"].shape[0], "bend": net.ff["bend_beads"].shape[0],
              "linker": net.ff["linker_beads"].shape[0], "motor": net.ff["motor_beads"].shape[0],
              "branch": net.ff["branch_beads"].shape[0], "excl": ne, "boundary": nb}
    abytes = algorithmic_bytes(counts, net.n_beads)

    stream = torch.cuda.ExternalStream(L.medyan_mech_stream(h))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step():
        # one evaluation: energy and forces at x (ForceFieldManager::computeEnergy
        # + computeForces), both sets of kernels in one pass graph
        L.medyan_mech_enqueue_evaluate(h)

    # warm-up (with the NVTX calls of the timed steps: the first one
    # initializes NVTX, which must not happen inside a timed step)
    for _ in range(max(args.warmup, 3)):
        torch.cuda.nvtx.range_push("evaluate_step")
        step()
        torch.cuda.nvtx.range_pop()
    if L.medyan_mech_synchronize(h) != 0:
        raise RuntimeError("force evaluation reported an error")

    K = args.steps
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    # the clock sampler's process starts before the timed region: its
    # start-up (fork, exec, NVML init) must not stall the launch of a timed step
    with ClockSampler(dev) as clocks:
        time.sleep(0.3)
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with torch.cuda.stream(stream):
            # two more untimed steps enqueued right before the timed ones,
            # so the first timed step does not start on a GPU that has just
            # been idle (its clocks ramping up after the host-side waits)
            for i in range(-2, K):
                flush.zero_()
                if i >= 0:
                    ev[i][0].record(stream)
                torch.cuda.nvtx.range_push("evaluate_step")
                step()
                torch.cuda.nvtx.range_pop()
                if i >= 0:
                    ev[i][1].record(stream)
        L.medyan_mech_synchronize(h)
        torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    t_steps = [ev[i][0].elapsed_time(ev[i][1]) / 1e3 for i in range(K)]
    # the two passes alone, for the breakdown (same flush before each)
    for _ in range(3):
        L.medyan_mech_enqueue_forces(h)
        L.medyan_mech_enqueue_energy(h)
    L.medyan_mech_synchronize(h)
    evp = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(K)]
    # NVTX ranges name the passes for a profiler (ncu --nvtx --nvtx-include "force_pass/")
    nvtx = torch.cuda.nvtx
    with torch.cuda.stream(stream):
        for i in range(K):
            flush.zero_()
            evp[i][0].record(stream)
            nvtx.range_push("force_pass")
            L.medyan_mech_enqueue_forces(h)
            nvtx.range_pop()
            evp[i][1].record(stream)
            flush.zero_()
            evp[i][2].record(stream)
            nvtx.range_push("energy_pass")
            L.medyan_mech_enqueue_energy(h)
            nvtx.range_pop()
            evp[i][3].record(stream)
    L.medyan_mech_synchronize(h)
    torch.cuda.synchronize()
    t_force = [evp[i][0].elapsed_time(evp[i][1]) / 1e3 for i in range(K)]
    t_energy = [evp[i][2].elapsed_time(evp[i][3]) / 1e3 for i in range(K)]
    # the same steps back to back without the L2 flush (working set L2-resident)
    with torch.cuda.stream(stream):
        w0, w1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0.record(stream)
        for i in range(K):
            step()
        w1.record(stream)
    L.medyan_mech_synchronize(h)
    t_warm = w0.elapsed_time(w1) / 1e3 / K
    # force passes back to back without the flush: the L2-warm side of the
    # roofline (coordinates and records stay in the 126 MB L2)
    with torch.cuda.stream(stream):
        w0.record(stream)
        for i in range(K):
            L.medyan_mech_enqueue_forces(h)
        w1.record(stream)
    L.medyan_mech_synchronize(h)
    t_force_warm = w0.elapsed_time(w1) / 1e3 / K
    t_step = max_over_ranks(sum(t_steps), world, "cuda")

    # e2e through the C ABI from page-locked host buffers: each step's own
    # coordinates in, its energies and forces out (the asynchronous entry,
    # two steps in flight), and the synchronous entry for comparison
    pd = C.POINTER(C.c_double)
    xh = [torch.from_numpy(x.copy()).pin_memory() for _ in range(2)]
    fh = [torch.empty_like(xh[0]).pin_memory() for _ in range(2)]
    eh = [torch.empty(11, dtype=torch.float64).pin_memory() for _ in range(2)]

    def e2e_async(n):
        for i in range(n):
            st = L.medyan_mech_evaluate_async(h, C.cast(xh[i % 2].data_ptr(), pd), C.cast(fh[i % 2].data_ptr(), pd),
                                              C.cast(eh[i % 2].data_ptr(), pd))
            if st != 0:
                raise RuntimeError(f"medyan_mech_evaluate_async status {st}")
        st = L.medyan_mech_wait(h)
        if st not in (0, 3):
            raise RuntimeError(f"medyan_mech_wait status {st}")

    e2e_async(4)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_async(K)
    e2e_t = max_over_ranks(time.perf_counter() - t0, world, "cuda")
    etot = C.c_double()
    per = (C.c_double * 10)()
    xptr = C.cast(xh[0].data_ptr(), pd)
    fptr = C.cast(fh[0].data_ptr(), pd)
    for _ in range(2):
        L.medyan_mech_evaluate(h, xptr, C.byref(etot), per, fptr)
    t0 = time.perf_counter()
    for _ in range(K):
        st = L.medyan_mech_evaluate(h, xptr, C.byref(etot), per, fptr)
        if st not in (0, 3):
            raise RuntimeError(f"medyan_mech_evaluate status {st}")
    e2e_sync_t = max_over_ranks(time.perf_counter() - t0, world, "cuda")

    # accuracy of this precision against the FP64 path on the same inputs
    ff64 = make("fp64") if args.precision != "fp64" else ff
    e64, per64, f64 = ff64.evaluate(x)
    e_, per_, f_ = ff.evaluate(x)
    rel_force_err = float(np.abs(f_ - f64).max() / np.abs(f64).max())
    rel_energy_err = float(abs(e_ - e64) / abs(e64))
    # the FP64 arm: the same steps, same protocol, on the FP64 handle
    fp64_arm = None
    if ff64 is not ff:
        L64, h64 = ff64.lib, ff64.handle
        s64 = torch.cuda.ExternalStream(L64.medyan_mech_stream(h64))
        t64 = timed_passes(L64.medyan_mech_enqueue_evaluate, h64, L64, s64, flush, K, max(args.warmup, 3))
        f64t = timed_passes(L64.medyan_mech_enqueue_forces, h64, L64, s64, flush, K, 3)
        t64_step = max_over_ranks(sum(t64), world, "cuda")
        fp64_arm = {"value": world * K / t64_step, "unit": "force-evals/s", "ms_per_step": 1e3 * t64_step / K,
                    "force_pass_alone_ms": 1e3 * sum(f64t) / K, "launch_shapes": ff64.tuned_shapes,
                    "l2": "flushed (256 MiB write) before each timed step"}

    result = {
        "metric": METRIC,
        "value": world * K / t_step,
        "unit": "force-evals/s",
        "n_gpus": world,
        "steps": K,
        "warmup": max(args.warmup, 3) + 2,
        "ms_per_step": 1e3 * t_step / K,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32+f64" if args.precision == "mixed" else "f64",
        "data": "synthetic (seeded network generator, reference initializer rules)",
        "config": {"workload": WORKLOAD, "precision": args.precision, "n_beads": net.n_beads,
                   "launch_shapes": ff.tuned_shapes,
                   "interactions": counts, "l2": "flushed (256 MiB write) before each timed step",
                   "step": "total energy + forces of all force fields", "parallelism": f"replicas x{world}"},
        "e2e": {"value": world * K / e2e_t, "unit": "force-evals/s", "h2d_bytes_per_step": 8 * x.size,
                "d2h_bytes_per_step": 8 * x.size + 8 * 11,
                "api": "medyan_mech_evaluate_async + medyan_mech_wait (two steps in flight)",
                "sync": {"value": world * K / e2e_sync_t, "unit": "force-evals/s",
                         "api": "medyan_mech_evaluate, one step at a time"}},
        # kernel nodes of the evaluate pass graph each timed step launches
        "gpu_launches": K * L.medyan_mech_pass_kernel_count(h, 2),
        "clocks": clocks.summary(),
        "wall_s_timed_region": wall,
        "accuracy_vs_fp64": {"rel_force_err": rel_force_err, "rel_energy_err": rel_energy_err},
        "fp64": fp64_arm,
        "breakdown_ms": {"force_pass_alone": 1e3 * sum(t_force) / K, "energy_pass_alone": 1e3 * sum(t_energy) / K,
                         "step_l2_warm": 1e3 * t_warm, "force_pass_l2_warm": 1e3 * t_force_warm,
                         "step_spread": {"min": 1e3 * min(t_steps), "median": 1e3 * statistics.median(t_steps),
                                         "max": 1e3 * max(t_steps)}},
    }
    fb = abytes["forces"]
    t_f = sum(t_force) / K
    result["roofline"] = roofline(fb / t_f / 1e9, fb)
    # the same bytes over the L2-warm pass time: what the pass would reach if
    # DRAM were free, so the gap to the peak is not DRAM time
    result["roofline"]["l2_warm"] = {"achieved": fb / t_force_warm / 1e9,
                                     "frac": fb / t_force_warm / 1e9 / result["roofline"]["peak"]}
    result["algorithmic_bytes"] = abytes

    # neighbor-list rebuild on the device (host call, coordinates resident)
    ff.rebuild_neighbor_lists()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(5):
        ff.rebuild_neighbor_lists()
    torch.cuda.synchronize()
    result["nl_rebuild"] = {"rebuilds_per_s": 5 / (time.perf_counter() - t0),
                            "timed": "medyan_mech_rebuild_neighbors (binning, pair search, re-vectorization of the "
                                     "excluded-volume and boundary records), host call to return"}
    if not args.no_minimize and rank == 0:
        result["minimization"] = minimize_extras(net, make)
        result["batched_ensemble"] = batch_extras()
        result["medium_network"] = medium_network_extras(make_for)
    if rank == 0:
        result["cpu_extras"] = cpu_extras(net, result.get("minimization"))
    for f in {id(ff): ff, id(ff64): ff64}.values():
        f.close()
    return result


def timed_passes(fn, h, L, stream, flush, K: int, warmup: int) -> list:
    """K passes of fn(h), each after a 256 MiB L2 flush, timed with CUDA
    events on the handle's stream; seconds per pass."""
    import torch
    for _ in range(warmup):
        fn(h)
    if L.medyan_mech_synchronize(h) != 0:
        raise RuntimeError("pass reported an error")
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    with torch.cuda.stream(stream):
        for i in range(K):
            flush.zero_()
            ev[i][0].record(stream)
            fn(h)
            ev[i][1].record(stream)
    L.medyan_mech_synchronize(h)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) / 1e3 for a, b in ev]


def roofline(achieved_gbs: float, nbytes: int) -> dict:
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        with open(peaks_path) as fh:
            peak, src = float(json.load(fh)["hbm_gbs"]), "measured"
    traffic = None
    prof = os.path.join(ROOT, "profiles", "force_pass_traffic.json")
    if os.path.exists(prof):
        with open(prof) as fh:
            traffic = json.load(fh).get("bytes_per_launch")
    return {"bound": "hbm", "achieved": achieved_gbs, "peak": peak, "unit": "GB/s", "frac": achieved_gbs / peak,
            "traffic": traffic, "peak_source": src, "kernel": "force pass (chain, bonded groups, excluded volume), timed alone",
            "algorithmic_bytes_per_launch": nbytes}


def minimize_extras(net, make) -> dict:
    """Minimization of the benchmark network per precision with the
    reference's criteria (gradTol 1 pN, or |dE|/|E| < 1e-9: whichever comes
    first, CGMethod.hpp:1431) and the reference example's MAXDISTANCE and
    LAMBDAMAX. Each timed run rebuilds the neighbor list at the start
    coordinates first (the workload rebuilds it per minimization). With
    deterministic force sums a run is bitwise reproducible, so one run per
    precision is the number (a second is checked identical); three runs with
    floating-point atomic sums show the spread that summation order alone
    gives a trajectory."""
    import numpy as np
    import torch

    from medyan_b200.forcefield import conjugate_gradient_params
    out = {"criteria": "gradTol 1 pN or energyRelTol 1e-9 (first met), maxDist 1 nm, lambdaMax 0.01",
           "timed": "neighbor-list rebuild at the start coordinates + minimization"}
    p = conjugate_gradient_params(grad_tol=1.0, max_dist=1.0, lambda_max=0.01, energy_rel_tol=1e-9)
    x = net.flat_coords()
    warm = conjugate_gradient_params(grad_tol=1.0, energy_call_limit=3)

    def run(ff):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ff.set_coords(x)
        ff.rebuild_neighbor_lists()
        st, xm, fm, r = ff.minimize(x, p)
        return time.perf_counter() - t0, st, xm, r

    for prec in ("fp64", "mixed"):
        ff = make(prec)
        ff.set_deterministic(True)
        ff.minimize(x, warm)  # builds the minimizer's graph outside the timed runs
        (dt, st, xm, r), (dt2, st2, xm2, r2) = run(ff), run(ff)
        rec = {"status": st, "seconds": dt, "minimizations_per_s": 1.0 / dt, "iterations": r.num_iter,
               "us_per_iteration": 1e6 * dt / max(r.num_iter, 1), "energy_calls": r.num_energy_call,
               "force_calls": r.num_force_call, "energy_before": r.energy_before_total,
               "energy_after": r.energy_after_total, "grad_inf_norm": r.grad_inf_norm,
               "energy_rel_change": r.energy_rel_change,
               "second_run_identical": bool(np.array_equal(xm, xm2) and r.num_iter == r2.num_iter),
               "second_run_seconds": dt2}
        ff.set_deterministic(False)
        ff.minimize(x, warm)
        atomic = [run(ff) for _ in range(3)]
        ts = [a[0] for a in atomic]
        rec["atomic_sums"] = {"seconds_median": statistics.median(ts), "seconds_min": min(ts), "seconds_max": max(ts),
                              "iterations": [a[3].num_iter for a in atomic],
                              "energy_after": [a[3].energy_after_total for a in atomic],
                              "grad_inf_norm": [a[3].grad_inf_norm for a in atomic]}
        out[prec] = rec
        ff.close()
    e64, em = out["fp64"]["energy_after"], out["mixed"]["energy_after"]
    out["final_energy_rel_diff_mixed_vs_fp64"] = abs(em - e64) / abs(e64)
    ea = out["fp64"]["atomic_sums"]["energy_after"]
    out["final_energy_rel_spread_fp64_atomic_runs"] = (max(ea) - min(ea)) / abs(e64)
    return out


_CPU_WORKER = {}


def _cpu_replica_init() -> None:
    from oracle.oracle import Oracle, Reference
    _CPU_WORKER["orc"] = Oracle()
    _CPU_WORKER["ref"] = Reference() if Reference.available() else None


def _cpu_replica_minimize(net):
    """One replica minimized by the reference's CGMethod (oracle/_ref), in a
    worker process: (start, end, force calls)."""
    from medyan_b200.forcefield import conjugate_gradient_params
    orc, ref = _CPU_WORKER["orc"], _CPU_WORKER["ref"]
    st, extra = orc.complete(net)
    sv = net.system_view(**extra)
    p = conjugate_gradient_params(grad_tol=1.0, max_dist=1.0, lambda_max=0.01, energy_rel_tol=1e-9)
    t0 = time.perf_counter()
    s, xm, fm, r = (ref or orc).minimize(sv, net.flat_coords(), p)
    return t0, time.perf_counter(), int(r.num_force_call)


def cpu_ensemble(n_replicas: int = 256, budget_s: float = 60.0) -> dict:
    """The batched ensemble on the host: every replica minimized by the
    reference's CGMethod, one replica per host core at a time (a spawn pool
    of one process per core), the same networks and criteria as the device
    batch. Bounded: replicas not finished within budget_s are not counted."""
    import multiprocessing as mp

    from oracle.oracle import Reference
    nets = ensemble(n_replicas)
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    ctx = mp.get_context("spawn")
    done = []
    t_wall = time.perf_counter()
    with ctx.Pool(cores, initializer=_cpu_replica_init) as pool:
        # largest replicas first, so the pool's tail is short
        order = sorted(range(len(nets)), key=lambda r: -nets[r].n_beads)
        it = pool.imap_unordered(_cpu_replica_minimize, [nets[r] for r in order])
        for _ in order:
            left = budget_s - (time.perf_counter() - t_wall)
            if left <= 0:
                break
            try:
                done.append(it.next(timeout=left))
            except mp.TimeoutError:
                break
        pool.terminate()
    if not done:
        return {"unavailable": f"no replica finished within {budget_s:.0f} s"}
    t0 = min(d[0] for d in done)
    t1 = max(d[1] for d in done)
    # process start-up is excluded: the span runs from the first replica's
    # start to the last one's end
    return {"kind": "reference" if Reference.available() else "port", "cores": cores,
            "minimizations_per_s": len(done) / (t1 - t0), "replicas_done": len(done), "replicas": len(nets),
            "sample": f"{len(done)} of {len(nets)} replicas minimized in {t1 - t0:.1f} s on {cores} processes",
            "force_calls_mean": float(sum(d[2] for d in done) / len(done))}


def cpu_extras(net, gpu_min: dict | None) -> dict:
    """CPU baselines beside the device numbers, each a bounded sample on one
    host thread: the reference's own CGMethod (oracle/_ref) on the benchmark
    network for a fixed number of energy calls (seconds per CG iteration; the
    minimizations/s estimate scales it by the device FP64 run's iteration
    count, the same algorithm and criteria), and the neighbor-list rebuild
    (the oracle's restatement of HybridCylinderCylinderNL, whose reference
    code is entangled with the simulator's globals and not compiled)."""
    from medyan_b200.forcefield import conjugate_gradient_params
    from oracle.oracle import Oracle, Reference
    out = {}
    orc = Oracle()
    st, extra = orc.complete(net)
    sv = net.system_view(**extra)
    x = net.flat_coords()
    if Reference.available():
        ref, kind = Reference(), "reference"
    else:
        ref, kind = orc, "port"
    p = conjugate_gradient_params(grad_tol=1.0, max_dist=1.0, lambda_max=0.01, energy_rel_tol=1e-9,
                                  energy_call_limit=120)
    t0 = time.perf_counter()
    s, xm, fm, r = ref.minimize(sv, x, p)
    dt = time.perf_counter() - t0
    # a run stopped by its call limit reports numIter -1; every iteration
    # after the first force call makes one more
    iters = r.num_iter if r.num_iter > 0 else r.num_force_call - 1
    s_iter = dt / max(iters, 1)
    rec = {"kind": kind, "cores": 1, "sample": f"{iters} CG iterations ({r.num_energy_call} energy, "
                                                f"{r.num_force_call} force calls) in {dt:.1f} s",
           "seconds_per_iteration": s_iter}
    if gpu_min and "fp64" in gpu_min:
        n_it = gpu_min["fp64"]["iterations"]
        rec["minimizations_per_s_estimate"] = 1.0 / (s_iter * n_it)
        rec["estimate"] = f"1 / (seconds per iteration x {n_it} iterations of the device FP64 run)"
    out["minimization"] = rec
    cv = net.cylinders_view()
    nl = net.nl_params()
    orc.neighbor_pairs(cv, x, net.n_beads, nl)
    n, t0 = 0, time.perf_counter()
    while n < 3:
        orc.neighbor_pairs(cv, x, net.n_beads, nl)
        n += 1
    dt = time.perf_counter() - t0
    out["nl_rebuild"] = {"kind": "port", "cores": 1, "rebuilds_per_s": n / dt,
                         "sample": f"{n} rebuilds of the 400k-cylinder list in {dt:.1f} s"}
    out["batched_ensemble"] = cpu_ensemble_in_child()
    return out


def cpu_ensemble_in_child(budget_s: float = 60.0) -> dict:
    """cpu_ensemble in a child process (bench.py --cpu-ensemble), so its
    process pool never shares a process with the device work, and a hard
    timeout ends the child's whole process group."""
    import signal
    cmd = [sys.executable, os.path.abspath(__file__), "--cpu-ensemble", "--cpu-sample-s", str(budget_s)]
    proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, start_new_session=True,
                            text=True)
    try:
        out, _ = proc.communicate(timeout=budget_s + 120)
    except subprocess.TimeoutExpired:
        os.killpg(proc.pid, signal.SIGKILL)
        proc.communicate()
        return {"unavailable": "the host ensemble run did not end in time"}
    try:
        return json.loads(out.strip().splitlines()[-1])
    except (ValueError, IndexError):
        return {"unavailable": f"the host ensemble run exited with {proc.returncode}"}


def medium_network_extras(make_for) -> dict:
    """The medium network (2,000 filaments x 20 cylinders, 42k beads, 4k
    linkers, 500 motors, 400 branch points): force-evals/s on the device in
    both precisions (same protocol as the headline) and on one host thread
    with the reference's kernels."""
    import torch

    from medyan_b200.network import make_workload
    net = make_workload(1)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    out = {"workload": "cfg1_2000x20_5um", "n_beads": net.n_beads}
    for prec in ("fp64", "mixed"):
        ff = make_for(net, prec)
        L, h = ff.lib, ff.handle
        s = torch.cuda.ExternalStream(L.medyan_mech_stream(h))
        t = timed_passes(L.medyan_mech_enqueue_evaluate, h, L, s, flush, 20, 5)
        out[prec] = {"force_evals_per_s": len(t) / sum(t), "us_per_step": 1e6 * sum(t) / len(t),
                     "launch_shapes": ff.tuned_shapes}
        ff.close()
    rate, n, dt, kind = cpu_reference_rate(net, 3.0)
    out["cpu"] = {"force_evals_per_s": rate, "kind": kind, "cores": 1,
                  "sample": f"{n} energy+force evaluations in {dt:.1f} s"}
    return out


_ENSEMBLE = {}


def ensemble(n_replicas: int = 256) -> list:
    """The batched-ensemble networks (config-1 composition, 200-4,000
    cylinders each, seed 2), built once per process."""
    if n_replicas not in _ENSEMBLE:
        from medyan_b200.network import make_batch
        _ENSEMBLE[n_replicas] = make_batch(n_replicas, 2)
    return _ENSEMBLE[n_replicas]


def batch_extras(n_replicas: int = 256) -> dict:
    """The batched ensemble (256 networks of the medium network's composition,
    200-4,000 cylinders each): one batched minimization per precision, gradTol
    1 pN, and the same replicas minimized one at a time for comparison (first
    16 replicas). Neighbor lists are built on the device per replica."""
    import numpy as np
    import torch

    from medyan_b200.forcefield import BatchMinimizer, ForceFieldManager, conjugate_gradient_params
    nets = ensemble(n_replicas)
    p = conjugate_gradient_params(grad_tol=1.0, max_dist=1.0, lambda_max=0.01, energy_rel_tol=1e-9)
    warm = conjugate_gradient_params(grad_tol=1.0, energy_call_limit=3)
    xs = [net.flat_coords() for net in nets]
    out = {"replicas": n_replicas, "beads": int(sum(n.n_beads for n in nets))}
    for prec in ("fp64", "mixed"):
        svs = [net.system_view() for net in nets]
        with BatchMinimizer(svs, prec) as b:
            for r, net in enumerate(nets):
                bp, _ = net.boundary_params()
                b.rebuild_neighbor_lists(r, xs[r], net.cylinders_view(), net.nl_params(), bp)
            shapes = b.autotune(reps=3)
            # deterministic sums: the batch ends with its slowest replica,
            # whose iteration count with atomic sums varies from run to run;
            # fixed-point sums make the figure reproducible (checked by a
            # second run). One atomic-sum run is reported beside it.
            b.set_deterministic(True)
            b.minimize(xs, warm)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            st, xo, fo, rs = b.minimize(xs, p)
            dt = time.perf_counter() - t0
            st2, xo2, fo2, rs2 = b.minimize(xs, p)
            identical = all(np.array_equal(a, c) for a, c in zip(xo, xo2))
            b.set_deterministic(False)
            b.minimize(xs, warm)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            sta, xa, fa, rsa = b.minimize(xs, p)
            dta = time.perf_counter() - t0
        m = 16
        seq = 0.0
        for r in range(m):
            with ForceFieldManager(prec) as ff:
                ff.vectorize_all_force_fields(svs[r])
                bp, _ = nets[r].boundary_params()
                ff.set_coords(xs[r])
                ff.set_cylinders(nets[r].cylinders_view(), nets[r].nl_params(), bp)
                ff.rebuild_neighbor_lists()
                ff.minimize(xs[r], warm)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                ff.minimize(xs[r], p)
                seq += time.perf_counter() - t0
        its = [r.num_iter for r in rs]
        itsa = [r.num_iter for r in rsa]
        out[prec] = {"seconds": dt, "minimizations_per_s": n_replicas / dt, "sums": "deterministic",
                     "second_run_identical": identical,
                     "one_at_a_time_minimizations_per_s": m / seq, "iterations_mean": float(np.mean(its)),
                     "iterations_max": int(max(its)), "statuses": sorted(set(int(v) for v in st)),
                     "launch_shapes": shapes,
                     "atomic_sums": {"seconds": dta, "minimizations_per_s": n_replicas / dta,
                                     "iterations_mean": float(np.mean(itsa)), "iterations_max": int(max(itsa))}}
    return out


# -------------------------------------------------------- CPU (reference)
def cpu_reference_fns(net):
    """energy() and forces() of the reference's compiled kernels
    (oracle/_ref/libmedyan_ref.so, -O2 -ffast-math as the reference builds)
    on the network, or of the oracle port when that build is absent."""
    import ctypes as C

    import numpy as np

    from oracle.oracle import Oracle, Reference
    orc = Oracle()
    st, extra = orc.complete(net)
    sv = net.system_view(**extra)
    x = net.flat_coords()
    f = np.zeros_like(x)
    pd = C.POINTER(C.c_double)
    if Reference.available():
        ref = Reference()
        hnd = ref.lib.medyan_ref_prepare(sv.ref())
        keep = (sv, x, f, ref)

        def energy():
            return ref.lib.medyan_ref_prepared_energy(hnd, keep[1].ctypes.data_as(pd), None)

        def forces():
            ref.lib.medyan_ref_prepared_forces(hnd, keep[1].ctypes.data_as(pd), keep[2].ctypes.data_as(pd))
        return energy, forces, "reference"
    return (lambda: orc.energy(sv, x)), (lambda: orc.forces(sv, x)), "port"


def cpu_reference_rate(net, sample_s: float):
    """Energy + forces per second on one host thread over a bounded sample."""
    energy, forces, kind = cpu_reference_fns(net)
    energy()
    forces()
    n = 0
    t0 = time.perf_counter()
    while True:
        energy()
        forces()
        n += 1
        dt = time.perf_counter() - t0
        if dt >= sample_s or n >= 10000:
            break
    return n / dt, n, dt, kind


def main():
    args = parse()
    if args.cpu_ensemble:
        print(json.dumps(cpu_ensemble(budget_s=args.cpu_sample_s)), flush=True)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        if args.impl == "ours":
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist.init_process_group("nccl" if args.impl == "ours" else "gloo", timeout=timedelta(seconds=600))

    if args.impl == "reference":
        if rank == 0:
            net = build_network()
            energy, forces, kind = cpu_reference_fns(net)
            for _ in range(args.warmup):
                energy()
                forces()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                energy()
                forces()
            dt = time.perf_counter() - t0
            rate = args.steps / dt
            line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": "force-evals/s", "n_gpus": 0,
                    "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
                    "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                    "data": "synthetic (seeded network generator, reference initializer rules)",
                    "config": {"workload": WORKLOAD, "step": "total energy + forces of all force fields"},
                    "cpu_baseline": {"value": rate, "unit": "force-evals/s", "cores": 1, "kind": kind,
                                     "sample": f"{args.steps} energy+force evaluations of the full network "
                                               f"in {dt:.1f} s (single-threaded, as the reference)"},
                    "e2e": {"value": rate, "unit": "force-evals/s", "h2d_bytes_per_step": 0,
                            "d2h_bytes_per_step": 0}}
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    result = run_ours(args, rank, world)
    if rank == 0:
        net = build_network()
        rate, n, dt, kind = cpu_reference_rate(net, args.cpu_sample_s)
        result["cpu_baseline"] = {"value": rate, "unit": "force-evals/s", "cores": 1, "kind": kind,
                                  "sample": f"{n} energy+force evaluations of the full network in {dt:.1f} s"}
        print(json.dumps(result), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
