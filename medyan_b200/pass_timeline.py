"""Per-block timeline of the fused passes inside their CUDA graphs.

ncu replays each kernel alone, so it cannot show how the kernels of one pass
share the GPU. This tool runs passes through the profiling build of the
library (libmedyan_b200_trace.so, `python -m medyan_b200.build --trace`), in
which thread 0 of every block of the pass kernels records its SM and its
start and end on the global timer, and prints per kernel: blocks, first
start and last end relative to the pass's first block, the last block start
and the block durations (median, 90th percentile, max). The blocks that
complete a group of energy rows (group.*) and the block that finishes the
pass (finish.*) are listed as stages of their own.

    python -m medyan_b200.pass_timeline [--workload 4] [--layout 0]
        [--precision mixed] [--passes evaluate,forces,energy] [--no-flush]

Each pass is recorded once after three unrecorded ones, after a 256 MiB
write that evicts the L2 (unless --no-flush). The records cost a global
atomic per block, so the timeline is for reading the schedule, not timing.
"""
from __future__ import annotations

import argparse
import ctypes as C
import sys

import numpy as np

from . import build as _build
from . import lib as _lib

KINDS = {0: "main.forces", 1: "branch.forces", 2: "excl.forces", 3: "zero", 4: "chain.forces",
         10: "main.energy", 11: "branch.energy", 12: "excl.energy", 14: "chain.energy",
         100: "group.main", 101: "group.branch", 102: "group.excl", 200: "finish.main", 201: "finish.branch",
         202: "finish.excl"}
REC = np.dtype([("kind", "u4"), ("smid", "u4"), ("block", "u4"), ("pad", "u4"), ("t0", "u8"), ("t1", "u8")])


def summarize(r: np.ndarray) -> list[str]:
    base = int(r["t0"].min())
    out = [f"{len(r)} records, span {(int(r['t1'].max()) - base) / 1e3:.1f} us"]
    for kind in sorted(set(r["kind"].tolist())):
        q = r[r["kind"] == kind]
        d = (q["t1"].astype(np.int64) - q["t0"].astype(np.int64)) / 1e3
        out.append(f"  {KINDS.get(kind, str(kind)):14s} blocks {len(q):5d}  start {(int(q['t0'].min()) - base) / 1e3:6.1f}"
                   f"  end {(int(q['t1'].max()) - base) / 1e3:6.1f}  last start {(int(q['t0'].max()) - base) / 1e3:6.1f}"
                   f"  block us: median {np.median(d):5.2f} p90 {np.percentile(d, 90):5.2f} max {d.max():6.2f}")
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--workload", type=int, default=4, help="seeded workload network (0-4)")
    ap.add_argument("--layout", type=int, default=0, help="pass layout (0 or 2: the fused layouts)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--passes", default="evaluate,forces,energy")
    ap.add_argument("--no-flush", action="store_true")
    args = ap.parse_args(argv)

    import torch

    from .forcefield import ForceFieldManager
    from .network import make_workload

    _build.build(trace=True)  # recompiles only what is stale
    _lib.LIB_PATH = _build.LIB_TRACE
    raw = C.CDLL(_build.LIB_TRACE)
    raw.medyan_pass_trace_dump.restype = C.c_int
    raw.medyan_pass_trace_reset.restype = C.c_int

    net = make_workload(args.workload)
    x = net.flat_coords()
    bp, _ = net.boundary_params()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    with ForceFieldManager(args.precision) as ff:
        ff.vectorize_all_force_fields(net.system_view())
        ff.set_coords(x)
        ff.set_cylinders(net.cylinders_view(), net.nl_params(), bp)
        ff.rebuild_neighbor_lists()
        ff.set_shapes(pass_layout=args.layout)
        L, h = ff.lib, ff.handle
        fns = {"evaluate": L.medyan_mech_enqueue_evaluate, "forces": L.medyan_mech_enqueue_forces,
               "energy": L.medyan_mech_enqueue_energy}
        for name in args.passes.split(","):
            fn = fns[name]
            for _ in range(3):
                fn(h)
            if L.medyan_mech_synchronize(h) != 0:
                raise RuntimeError(f"{name} pass reported an error")
            if not args.no_flush:
                flush.zero_()
            torch.cuda.synchronize()
            raw.medyan_pass_trace_reset()
            fn(h)
            L.medyan_mech_synchronize(h)
            torch.cuda.synchronize()
            buf = np.zeros(1 << 16, dtype=REC)
            n = raw.medyan_pass_trace_dump(buf.ctypes.data_as(C.c_void_p), len(buf))
            if n <= 0:
                raise RuntimeError("no trace records")
            print(f"{name} pass (workload {args.workload}, layout {args.layout}, {args.precision}):")
            print("\n".join(summarize(buf[:n])))
    return 0


if __name__ == "__main__":
    sys.exit(main())
