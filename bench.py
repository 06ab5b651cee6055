"""Benchmark: batched canonical labeling of 10,000 small graphs on B200.

Workload (one "step"): the batched small-graph workload -- 10,000 uncoloured
graphs, n ~ U[10, 64], each a random labelled tree (Pruefer sequence, max
degree 4) plus 0-6 extra edges that keep the max degree <= 4, 20% of them
random relabelings of earlier graphs, packed into one int32 ragged CSR
arena and canonized in one batched call (max_aut = 10000).

Reported JSON line (rank 0):
  value  graphs/s with the arena resident in HBM, device time (CUDA events on
         the library's stream) summed over K steps, L2 flushed between steps
  e2e    graphs/s through the C ABI with pinned host buffers: H2D of the arena,
         the kernels, D2H of every canonical matrix, stats and status
  roofline  algorithmic bytes of the batch (CSR read + n^2 canonical matrix
         write + per search node one CSR pass and one read+write of the
         partition) / kernel time, against the measured HBM copy bandwidth
  cpu_baseline  the reference's own sequential path (oracle/_ref), on all
         host cores, over the same graphs
  plain_per_launch  the same library launched once per graph (the plain form)
  serving  an open-loop Poisson request stream through the serving loop
         (gcl_serve_replay): p50 / p99 latency from the scheduled arrival,
         throughput, per-size and per-lane-class figures, and the plain form
         (one gcl_canon_one per graph, FIFO) under the same arrivals
  single_graph  search-heavy single graphs (random 3-regular n = 1024, 4096;
         tori 32x32, 64x64) through gcl_canon_one (the wide search), each also
         relabeled, with the reference's CPU path beside the ones it finishes
         in seconds

--impl reference: the reference's CPU implementation of the path (its own
sequential sources compiled into oracle/_ref, else the C restatement) on all
host cores, on the same workload, metric and unit.
"""
from __future__ import annotations

import argparse
import ctypes
import importlib
import json
import os
import subprocess
import sys
import time

import numpy as np

# The serving loop runs a dozen streams at once; with the default of 8
# hardware work queues, streams share queues and a short batch can wait
# behind a long search queued on another stream.  Must be set before CUDA
# starts in this process.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
PKG = "gpu-canonical-labeling_b200"

METRIC = "graphs canonized/sec"
UNIT = "graphs/s"
WORKLOAD = ("batched small graphs: 10,000 uncoloured graphs, n ~ U[10,64], Pruefer tree "
            "(max deg 4) + U{0..6} extra edges, 20% relabelings, one ragged CSR arena, "
            "max_aut 10000")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--graphs", type=int, default=10000)
    p.add_argument("--seed", type=int, default=3000)
    p.add_argument("--max-aut", type=int, default=10000)
    p.add_argument("--cpu-seconds", type=float, default=12.0,
                   help="wall-clock budget of the CPU-baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-sustained", action="store_true",
                   help="skip the one-second repeat of the step that samples clocks")
    p.add_argument("--e2e-contexts", type=int, default=4,
                   help="e2e with this many contexts on host threads, so one call's copies "
                        "and search tail run under another call's kernels (1 = one call "
                        "at a time)")
    p.add_argument("--e2e-mapped", action="store_true",
                   help="also time e2e through gcl_canon_batch_mapped (arena and results in "
                        "mapped host memory, no staging copies; key e2e_mapped)")
    p.add_argument("--no-serving", action="store_true")
    p.add_argument("--serve-requests", type=int, default=4000)
    p.add_argument("--serve-rate", type=float, default=350.0,
                   help="Poisson arrival rate of the serving run, requests/s")
    p.add_argument("--serve-nmax", type=int, default=4096,
                   help="largest request size (the 1%% tail is log-uniform on (2048, nmax])")
    p.add_argument("--serve-large-n", type=int, default=0,
                   help="server large_n (0 = the library default)")
    p.add_argument("--serve-large-sizes", type=int, nargs="*", default=[8192, 20000],
                   help="sizes of single requests timed alone on a server (the 1%% tail)")
    p.add_argument("--serve-large-budget-s", type=float, default=60.0)
    p.add_argument("--serve-big-wide", action="store_true",
                   help="server big_wide: big requests through the wide search")
    p.add_argument("--single-gate", type=int, default=1, choices=(0, 1, 2),
                   help="level gate of the single-graph block's wide searches")
    p.add_argument("--single-share", action="store_true",
                   help="work sharing in the single-graph block's wide searches")
    p.add_argument("--single-extra", action="store_true",
                   help="add a tree of 2,048 vertices and a union of five cubic graphs "
                        "to the single-graph block")
    p.add_argument("--serve-plain", type=int, default=800,
                   help="requests replayed through the plain one-graph-per-launch form")
    p.add_argument("--no-single", action="store_true")
    p.add_argument("--mixed", action="store_true",
                   help="also time the mixed-size batch (n log-uniform [64,4096]); off by default: "
                        "its union graphs take the reference's search minutes each")
    p.add_argument("--mixed-graphs", type=int, default=2000)
    p.add_argument("--union-budget-s", type=float, default=30.0,
                   help="time budget of the 16-copy union in the single-graph block")
    p.add_argument("--mixed-budget-s", type=float, default=10.0,
                   help="per-graph time budget of the mixed-size batch")
    p.add_argument("--mixed-handoff-ms", type=int, default=1000,
                   help="hand-off budget of the third mixed-batch run (GCL_OPT_BATCH_HANDOFF_MS)")
    p.add_argument("--mixed-plain", type=int, default=200,
                   help="graphs of the mixed batch timed one launch each")
    return p.parse_args()


def workload(args):
    G = importlib.import_module(PKG + ".graphs")
    return G.pack(G.small_batch(args.graphs, seed=args.seed))


def bench_config(args, count: int, world: int) -> dict:
    """The workload both arms run (the GPU arm and --impl reference print the
    same dict)."""
    return {"workload": WORKLOAD, "graphs_per_step_per_gpu": count, "max_aut": args.max_aut,
            "seed": args.seed, "parallelism": f"graph-sharded x{world} (no collective)",
            "l2": "GPU arm: flushed between steps (256 MiB write outside the timed events)",
            "output": "canonical forms (bit-packed rows on the GPU arm), stats and status "
                      "per graph"}


def algorithmic_bytes(arena, nodes: np.ndarray, packed: bool = False) -> int:
    """B(g) = (4(n+1) + 8m) + n^2 + nodes(g) * (4(n+1) + 8m + 32n), summed.
    With packed, the n^2 byte matrix is charged as the bit-packed rows the
    timed call writes instead: n * ceil(n/64) 8-byte words."""
    n = arena.sizes().astype(np.int64)
    m = (np.diff(arena.eoff) // 2).astype(np.int64)
    csr = 4 * (n + 1) + 8 * m
    out = n * ((n + 63) // 64) * 8 if packed else n * n
    return int((csr + out + nodes.astype(np.int64) * (csr + 32 * n)).sum())


# --------------------------------------------------------------------------
# CPU side: the reference's sequential path on all host cores
# --------------------------------------------------------------------------
_W = {}


def _cpu_init(kind, arrays):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # the oracle: the timed CPU baseline (test infrastructure)
    G = importlib.import_module(PKG + ".graphs")
    _W["oracle"] = oracle
    _W["kind"] = kind
    _W["arena"] = G.Arena(*arrays)


def _cpu_run(lo_hi):
    lo, hi = lo_hi
    O, A, kind = _W["oracle"], _W["arena"], _W["kind"]
    G = importlib.import_module(PKG + ".graphs")
    sub = G.Arena(hi - lo, A.voff[lo:hi + 1] - A.voff[lo], A.eoff[lo:hi + 1] - A.eoff[lo],
                  A.rowptr[A.voff[lo] + lo: A.voff[hi] + hi], A.col[A.eoff[lo]:A.eoff[hi]],
                  A.color[A.voff[lo]:A.voff[hi]])
    t = time.perf_counter()
    O.canon_batch(sub, max_aut=10000, kind=kind, want_matrix=True)
    return hi - lo, time.perf_counter() - t


def cpu_kind():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if oracle.available("reference"):
        return "reference"
    if not oracle.available("port"):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    return "port"


class CpuPool:
    def __init__(self, arena, kind):
        import multiprocessing as mp
        self.cores = os.cpu_count() or 1
        self.kind = kind
        arrays = (arena.count, arena.voff, arena.eoff, arena.rowptr, arena.col, arena.color)
        self.pool = mp.get_context("spawn").Pool(self.cores, initializer=_cpu_init,
                                                  initargs=(kind, arrays))
        self.count = arena.count
        chunks = max(self.cores * 4, 1)
        b = np.linspace(0, arena.count, chunks + 1).astype(int)
        self.tasks = [(int(b[i]), int(b[i + 1])) for i in range(chunks) if b[i + 1] > b[i]]

    def step(self):
        t = time.perf_counter()
        done = sum(x[0] for x in self.pool.map(self._run, self.tasks))
        return done, time.perf_counter() - t

    _run = staticmethod(_cpu_run)

    def close(self):
        self.pool.close()
        self.pool.join()


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    kind = cpu_kind()
    arena = workload(args)
    pool = CpuPool(arena, kind)
    for _ in range(max(args.warmup, 1)):
        pool.step()
    tot_g, tot_t, per = 0, 0.0, []
    for _ in range(args.steps):
        g, t = pool.step()
        tot_g += g
        tot_t += t
        per.append(t)
    pool.close()
    v = tot_g / tot_t
    # one core: the same reference code in this process on the first 2,000 graphs
    _cpu_init(kind, (arena.count, arena.voff, arena.eoff, arena.rowptr, arena.col, arena.color))
    g1, t1 = _cpu_run((0, min(2000, arena.count)))
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded generator, same graphs as the GPU arm)",
        "config": bench_config(args, arena.count, int(os.environ.get("WORLD_SIZE", "1"))),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": pool.cores, "kind": kind,
                         "sample": f"the full {arena.count}-graph batch per step, split over "
                                   f"{pool.cores} processes",
                         "value_1core": g1 / t1,
                         "sample_1core": f"the first {g1} graphs in one process"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "latency_ms": {"p50": float(np.percentile(per, 50)) * 1e3,
                       "p99": float(np.percentile(per, 99)) * 1e3},
    }
    print(json.dumps(line))


# --------------------------------------------------------------------------
# Multi-rank timing: every rank canonizes its own batch (graphs are
# independent: no data-path collective); the job's time is the slowest rank's
# --------------------------------------------------------------------------
def max_over_ranks(seconds_or_ms: float, world: int, device=None) -> float:
    """The largest value over all ranks (an all-reduce MAX; the value itself
    when there is one rank).  Every rank must call it at the same point."""
    if world <= 1:
        return seconds_or_ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([seconds_or_ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(graphs_per_rank: int, world: int, steps: int, seconds: float) -> float:
    """Whole-job graphs/s: the graphs all ranks processed over the slowest
    rank's time (weak scaling: the per-rank batch is fixed)."""
    return world * graphs_per_rank * steps / seconds


# --------------------------------------------------------------------------
# GPU side
# --------------------------------------------------------------------------
class Clocks:
    """SM clock and throttle reasons sampled through NVML every ~0.2 ms on a
    background thread (read-only queries; no setting is changed)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, device):
        import threading
        self.device = device
        self.samples = []
        self.stop_ev = threading.Event()
        self.thread = None
        self.window = None

    def _loop(self):
        import pynvml as N
        h = N.nvmlDeviceGetHandleByIndex(self.device)
        while not self.stop_ev.is_set():
            try:
                sm = N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)
                rs = N.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((time.perf_counter(), sm, rs))
            except Exception:
                pass
            time.sleep(0.0002)

    def start(self):
        import threading
        try:
            import pynvml as N
            N.nvmlInit()
            h = N.nvmlDeviceGetHandleByIndex(self.device)
            self.max_mhz = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
        except Exception:
            return
        self.thread = threading.Thread(target=self._loop, daemon=True)
        self.thread.start()

    def mark(self, t0, t1):
        self.window = (t0, t1)

    def stop(self):
        if not self.thread:
            return None
        self.stop_ev.set()
        self.thread.join()
        rows = self.samples
        if self.window:
            t0, t1 = self.window
            inside = [r for r in rows if t0 <= r[0] <= t1]
            rows = inside or [min(rows, key=lambda r: abs(r[0] - t1))] if rows else []
        if not rows:
            return None
        reasons = sorted({k for _, _, rs in rows for k, bit in self.REASONS.items() if rs & bit})
        return {"sm_mhz": float(np.median([r[1] for r in rows])), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(rows), "source": "nvml, 0.2 ms period"}


def read_traffic():
    """DRAM bytes of one step's pipelined warp-kernel launch from the
    committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "w64_pipe_kernel_small10k.txt")
    if not os.path.exists(p):
        return None
    for ln in open(p):
        if ln.strip().startswith("dram_bytes_per_step:"):
            return float(ln.split(":")[1].split()[0])
    return None


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def gpu_arm(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    pkg = importlib.import_module(PKG)
    api = pkg.api
    arena = workload(args)
    count = arena.count
    dev = torch.device("cuda", local)
    ctx = api.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    ooff = arena.out_offsets()
    roff = api.rows_offsets(arena)
    max_n = int(arena.sizes().max())
    max_m2 = int(np.diff(arena.eoff).max())

    # device-resident inputs and outputs
    def d(a, dtype):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev, dtype=dtype)

    t_voff, t_eoff = d(arena.voff, torch.int64), d(arena.eoff, torch.int64)
    t_rp, t_col = d(arena.rowptr, torch.int32), d(arena.col, torch.int32)
    t_ooff = d(ooff, torch.int64)
    t_roff = d(roff, torch.int64)
    t_dense = torch.empty(int(ooff[-1]), dtype=torch.uint8, device=dev)
    t_rows = torch.empty(int(roff[-1]), dtype=torch.int64, device=dev)
    t_stats = torch.empty((count, 2), dtype=torch.int64, device=dev)
    t_status = torch.empty(count, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    lib = ctx.lib
    P = ctypes.c_void_p

    def launch():
        rc = lib.gcl_canon_batch_device_async(
            ctx.handle, count, P(t_voff.data_ptr()), P(t_eoff.data_ptr()), P(t_rp.data_ptr()),
            P(t_col.data_ptr()), None, args.max_aut, max_n, max_m2, None, None,
            P(t_rows.data_ptr()), P(t_roff.data_ptr()), None, P(t_stats.data_ptr()),
            P(t_status.data_ptr()))
        if rc != 0:
            raise RuntimeError(f"gcl_canon_batch_device_async failed: {rc}")

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        flush.zero_()
        with torch.cuda.stream(stream):
            launch()
    torch.cuda.synchronize()
    assert int((t_status != 0).sum()) == 0, "a graph failed"
    nodes = t_stats[:, 1].cpu().numpy()

    clocks = Clocks(local)
    clocks.start()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    barrier()
    tw0 = time.perf_counter()
    for i in range(args.steps):
        flush.zero_()  # L2 flush outside the timed events
        stream.wait_stream(torch.cuda.current_stream())
        evs[i][0].record(stream)
        launch()
        evs[i][1].record(stream)
        torch.cuda.current_stream().wait_stream(stream)
    barrier()
    clocks.mark(tw0, time.perf_counter())
    clk = clocks.stop()
    per = np.array([a.elapsed_time(b) for a, b in evs])  # ms
    dev_ms = max_over_ranks(float(per.sum()), world, dev)
    value = job_rate(count, world, args.steps, dev_ms / 1e3)

    # The same steps repeated for about a second after the timed region, so
    # the clocks are sampled over a window long enough to mean something
    # (K steps of this batch last only milliseconds).  Reported beside the
    # headline, not in it.
    sus_steps = 0 if args.no_sustained else int(
        min(20000, max(args.steps, np.ceil(1.0 / max(float(per.mean()) / 1e3, 1e-6)))))
    sustained = None
    if sus_steps:
        sclocks = Clocks(local)
        sclocks.start()
        sev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(sus_steps)]
        barrier()
        ts0 = time.perf_counter()
        for i in range(sus_steps):
            flush.zero_()
            stream.wait_stream(torch.cuda.current_stream())
            sev[i][0].record(stream)
            launch()
            sev[i][1].record(stream)
            torch.cuda.current_stream().wait_stream(stream)
        barrier()
        sclocks.mark(ts0, time.perf_counter())
        sclk = sclocks.stop()
        sper = np.array([a.elapsed_time(b) for a, b in sev])
        sus_ms = max_over_ranks(float(sper.sum()), world, dev)
        sustained = {"value": job_rate(count, world, sus_steps, sus_ms / 1e3), "unit": UNIT,
                     "steps": sus_steps, "device_seconds": sus_ms / 1e3,
                     "wall_seconds": time.perf_counter() - ts0, "clocks": sclk,
                     "note": "the timed step repeated after the timed region (L2 flushed "
                             "between steps) to sample clocks over about a second"}

    # end to end through the C ABI: pinned host buffers, copies inside
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    h_voff, h_eoff, h_rp, h_col = pin(arena.voff), pin(arena.eoff), pin(arena.rowptr), pin(arena.col)
    h_ooff, h_roff = pin(ooff), pin(roff)
    h_dense = torch.empty(int(ooff[-1]), dtype=torch.uint8).pin_memory().numpy()
    h_rows = torch.empty(int(roff[-1]), dtype=torch.int64).pin_memory().numpy()
    h_stats = torch.empty((count, 2), dtype=torch.int64).pin_memory().numpy()
    h_status = torch.empty(count, dtype=torch.int32).pin_memory().numpy()
    pp = lambda a: a.ctypes.data_as(P)  # noqa: E731

    def e2e_call(dense):
        if dense:  # the reference's n*n byte matrices
            outs = (pp(h_dense), pp(h_ooff), None, None)
        else:  # the same canonical forms bit-packed
            outs = (None, None, pp(h_rows), pp(h_roff))
        rc = lib.gcl_canon_batch(ctx.handle, count, pp(h_voff), pp(h_eoff), pp(h_rp), pp(h_col),
                                 None, args.max_aut, *outs, None, pp(h_stats), pp(h_status))
        if rc != 0:
            raise RuntimeError(f"gcl_canon_batch failed: {rc}")

    def e2e_run(dense):
        for _ in range(max(2, args.warmup // 2) if not args.no_e2e else 0):
            e2e_call(dense)
        barrier()
        ts = []
        for _ in range(args.steps if not args.no_e2e else 0):
            t0 = time.perf_counter()
            e2e_call(dense)
            ts.append(time.perf_counter() - t0)
        barrier()
        return max_over_ranks(float(np.sum(ts)) if ts else float("nan"), world, dev)

    e2e_s = e2e_run(False)
    e2e_dense_s = e2e_run(True)
    # the same call with the batch in two halves on two streams
    ctx.set_option(api.GCL_OPT_BATCH_SPLIT, 1)
    e2e_split_s = e2e_run(False)
    ctx.set_option(api.GCL_OPT_BATCH_SPLIT, 0)

    def e2e_overlap(k):
        # k contexts (k streams) on k host threads, each with its own output
        # buffers; the inputs are shared read-only.  The steps are split over
        # the threads and timed together by the wall clock.
        import threading
        ctxs = [ctx] + [api.Context(local) for _ in range(k - 1)]
        outs = [(h_rows, h_stats, h_status)] + [
            (torch.empty(int(roff[-1]), dtype=torch.int64).pin_memory().numpy(),
             torch.empty((count, 2), dtype=torch.int64).pin_memory().numpy(),
             torch.empty(count, dtype=torch.int32).pin_memory().numpy()) for _ in range(k - 1)]
        errors = []

        def call(j):
            rows, stats, status = outs[j]
            rc = lib.gcl_canon_batch(ctxs[j].handle, count, pp(h_voff), pp(h_eoff), pp(h_rp),
                                     pp(h_col), None, args.max_aut, None, None, pp(rows),
                                     pp(h_roff), None, pp(stats), pp(status))
            if rc != 0:
                errors.append(rc)

        def worker(j, steps):
            for _ in range(steps):
                call(j)

        for j in range(k):
            call(j)  # warm-up: each context sizes its buffers
        share = [args.steps // k + (1 if j < args.steps % k else 0) for j in range(k)]
        barrier()
        t0 = time.perf_counter()
        ths = [threading.Thread(target=worker, args=(j, share[j])) for j in range(k)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        wall = time.perf_counter() - t0
        barrier()
        for c in ctxs[1:]:
            c.close()
        if errors:
            raise RuntimeError(f"gcl_canon_batch failed: {errors[0]}")
        return max_over_ranks(wall, world, dev)

    e2e_ov_s = e2e_overlap(args.e2e_contexts) if args.e2e_contexts > 1 and not args.no_e2e else None

    def e2e_mapped():
        # the arena and the outputs in mapped host memory of the context: the
        # warp kernel reads the graphs and writes the rows over the bus, with
        # no staging copies (set up once, outside the timed steps)
        held = []

        def mapped(a, dtype=None):
            m = ctx.host_array(a.shape, dtype or a.dtype)
            m[...] = a
            held.append(m)
            return m
        m_voff, m_eoff, m_rp, m_col, m_roff = (mapped(a) for a in (
            arena.voff, arena.eoff, arena.rowptr, arena.col, roff))
        m_rows = mapped(np.zeros(h_rows.shape, np.uint64))
        m_stats = mapped(np.zeros((count, 2), np.int64))
        m_status = mapped(np.zeros(count, np.int32))

        def call():
            rc = lib.gcl_canon_batch_mapped(ctx.handle, count, pp(m_voff), pp(m_eoff), pp(m_rp),
                                            pp(m_col), None, args.max_aut, None, None,
                                            pp(m_rows), pp(m_roff), None, pp(m_stats),
                                            pp(m_status))
            if rc != 0:
                raise RuntimeError(f"gcl_canon_batch_mapped failed: {rc}")
        for _ in range(max(2, args.warmup // 2)):
            call()
        barrier()
        ts = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            call()
            ts.append(time.perf_counter() - t0)
        barrier()
        # the same canonical forms as the staged-copy path (h_rows: its last step)
        same = bool(np.array_equal(m_rows.view(np.int64), h_rows))
        for m in held:
            ctx.host_free(m)
        if not same:
            raise RuntimeError("gcl_canon_batch_mapped: rows differ from gcl_canon_batch")
        return max_over_ranks(float(np.sum(ts)), world, dev)

    e2e_map_s = e2e_mapped() if args.e2e_mapped and not args.no_e2e else None
    h2d = sum(a.nbytes for a in (h_voff, h_eoff, h_rp, h_col, h_roff))
    d2h = h_rows.nbytes + h_stats.nbytes + h_status.nbytes
    if e2e_ov_s is not None:
        # the library driven the way a throughput user drives it (the
        # reference arm runs one process per host core): k contexts on k host
        # threads, every step its own upload, kernels and download
        e2e_line = {"value": job_rate(count, world, args.steps, e2e_ov_s), "unit": UNIT,
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "contexts": args.e2e_contexts,
                    "output": "bit-packed canonical rows (n x ceil(n/64) words per graph)",
                    "call": f"gcl_canon_batch from {args.e2e_contexts} host threads, one "
                            "context each, the steps split over them; wall clock"}
    else:
        e2e_line = {"value": job_rate(count, world, args.steps, e2e_s), "unit": UNIT,
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "output": "bit-packed canonical rows (n x ceil(n/64) words per graph)",
                    "call": "gcl_canon_batch, one call at a time, timed per call"}
    h2d_dense = sum(a.nbytes for a in (h_voff, h_eoff, h_rp, h_col, h_ooff))
    d2h_dense = h_dense.nbytes + h_stats.nbytes + h_status.nbytes

    line = None
    if rank == 0:
        peak, peak_kind = measured_peak()
        alg = algorithmic_bytes(arena, nodes)
        alg_packed = algorithmic_bytes(arena, nodes, packed=True)
        kern_ms = float(per.mean())
        achieved = alg / (kern_ms / 1e3) / 1e9
        achieved_packed = alg_packed / (kern_ms / 1e3) / 1e9
        traffic = read_traffic()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded generator)",
            "config": bench_config(args, count, world),
            "e2e": e2e_line,
            "e2e_single_call": {"value": job_rate(count, world, args.steps, e2e_s), "unit": UNIT,
                                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                                "output": "bit-packed canonical rows (n x ceil(n/64) words "
                                          "per graph)",
                                "call": "gcl_canon_batch, one call at a time, timed per call"},
            "e2e_split": {"value": job_rate(count, world, args.steps, e2e_split_s),
                          "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                          "d2h_bytes_per_step": int(d2h),
                          "call": "gcl_canon_batch with GCL_OPT_BATCH_SPLIT 1 (two halves on two "
                                  "streams)"},
            "e2e_dense": {"value": job_rate(count, world, args.steps, e2e_dense_s), "unit": UNIT,
                          "h2d_bytes_per_step": int(h2d_dense),
                          "d2h_bytes_per_step": int(d2h_dense),
                          "output": "n*n byte matrices (the reference's Nauty_Parallel form)"},
            # per step: order_by_size, the pipelined root-and-search kernel
            # and the full-ring rerun pass (which exits at once when no graph
            # outgrew the first ring)
            "gpu_launches": 3 * args.steps,
            **({"e2e_mapped": {"value": job_rate(count, world, args.steps, e2e_map_s),
                               "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                               "d2h_bytes_per_step": int(d2h),
                               "output": "bit-packed canonical rows; arena and results in "
                                         "mapped host memory, read and written by the "
                                         "kernels over the bus"}}
               if e2e_map_s is not None else {}),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": alg,
                         "algorithmic_bytes_packed_output": alg_packed,
                         "achieved_packed_output": achieved_packed,
                         "frac_packed_output": achieved_packed / peak},
            "latency_ms": {"p50": float(np.percentile(per, 50)),
                           "p99": float(np.percentile(per, 99))},
            "clocks": clk,
            **({"sustained": sustained} if sustained else {}),
        }

    # the plain form: one graph per launch (device-resident, same kernels)
    if rank == 0 and not args.no_plain:
        k = min(1000, count)
        one_v = torch.zeros(2, dtype=torch.int64, device=dev)
        one_o = torch.zeros(2, dtype=torch.int64, device=dev)
        hv, hee = arena.voff, arena.eoff
        starts = []
        for g in range(k):
            n, m = int(hv[g + 1] - hv[g]), int(hee[g + 1] - hee[g])
            starts.append((g, n, m))
        vo_all = torch.tensor([[0, n] for _, n, _ in starts], dtype=torch.int64, device=dev)
        eo_all = torch.tensor([[0, m] for _, _, m in starts], dtype=torch.int64, device=dev)
        oo_all = torch.tensor([[0, n * n] for _, n, _ in starts], dtype=torch.int64, device=dev)

        def one(i):
            g, n, m = starts[i]
            rc = lib.gcl_canon_batch_device_async(
                ctx.handle, 1, P(vo_all[i].data_ptr()), P(eo_all[i].data_ptr()),
                P(t_rp.data_ptr() + 4 * int(hv[g] + g)), P(t_col.data_ptr() + 4 * int(hee[g])),
                None, args.max_aut, n, m, P(t_dense.data_ptr() + int(ooff[g])),
                P(oo_all[i].data_ptr()), None, None, None, P(t_stats.data_ptr() + 16 * g),
                P(t_status.data_ptr() + 4 * g))
            if rc != 0:
                raise RuntimeError("plain launch failed")

        for i in range(min(50, k)):
            one(i)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(k):
            one(i)
        e1.record(stream)
        torch.cuda.synchronize()
        pl = k / (e0.elapsed_time(e1) / 1e3)
        line["plain_per_launch"] = {"value": pl, "unit": UNIT, "graphs": k,
                                    "batched_over_plain": value / world / pl}
        del one_v, one_o

    if rank == 0 and not args.no_cpu_baseline:
        kind = cpu_kind()
        pool = CpuPool(arena, kind)
        pool.step()  # warm-up (imports, page-in)
        g_done, t_done = 0, 0.0
        while t_done < args.cpu_seconds:
            g, t = pool.step()
            g_done += g
            t_done += t
        pool.close()
        line["cpu_baseline"] = {"value": g_done / t_done, "unit": UNIT, "cores": pool.cores,
                                "kind": kind,
                                "sample": f"{g_done} graphs (the {count}-graph batch repeated) "
                                          f"in {t_done:.1f} s on {pool.cores} processes"}
    if rank == 0 and not args.no_serving:
        line["serving"] = serving_block(args, pkg, local)
    if rank == 0 and not args.no_single:
        line["single_graph"] = single_graph_block(args, pkg, local, not args.no_cpu_baseline)
    if rank == 0 and args.mixed:
        line["mixed_batch"] = mixed_block(args, pkg, local)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    ctx.close()


# --------------------------------------------------------------------------
# Secondary workloads, reported beside the headline
# --------------------------------------------------------------------------
def _tail_timeline(res, lat, ns):
    """Where the slowest 1% of each size class spent its time: medians over
    those requests of the time queued (arrival -> taken into a batch), the
    host's enqueueing, the batch on the GPU and the hand-out after it."""
    out = {}
    adm = np.array([r.admit_s for r in res]) * 1e3
    lau = np.array([r.launch_s for r in res]) * 1e3
    gpu = np.array([r.gpu_done_s for r in res]) * 1e3
    launched = np.array([r.batch > 0 for r in res])
    for name, m in (("n<=64", ns <= 64), ("65-256", (ns > 64) & (ns <= 256)),
                    ("257-2048", (ns > 256) & (ns <= 2048)), (">2048", ns > 2048)):
        m = m & launched
        if not m.any():
            continue
        cut = np.percentile(lat[m], 99)
        t = m & (lat >= cut)
        out[name] = {"requests": int(t.sum()), "latency": float(np.median(lat[t])),
                     "queued": float(np.median(adm[t])),
                     "enqueue": float(np.median(lau[t] - adm[t])),
                     "gpu": float(np.median(gpu[t] - lau[t])),
                     "hand_out": float(np.median(lat[t] - gpu[t]))}
    return out


def serving_block(args, pkg, local):
    """Open-loop Poisson stream through the serving loop (gcl_serve_replay),
    then the plain form: the same requests one at a time, one launch each."""
    G = pkg.graphs
    W = G.serving_workload(args.serve_requests, args.serve_rate, seed=5000,
                           n_max=args.serve_nmax)
    arena = G.pack(W.graphs)
    scfg = {"large_n": args.serve_large_n} if args.serve_large_n else {}
    if args.serve_big_wide:
        scfg["big_wide"] = 1
    srv = pkg.Server(local, **scfg)
    # warm-up on the same server (its lanes size their workspaces): a short
    # replay of another stream with the same size range
    Ww = G.serving_workload(600, args.serve_rate, seed=5001, n_max=args.serve_nmax)
    srv.replay(G.pack(Ww.graphs), Ww.kind, Ww.g1, Ww.g2, Ww.arrival, timeout_s=600)
    st0 = srv.stats()
    t0 = time.perf_counter()
    res = srv.replay(arena, W.kind, W.g1, W.g2, W.arrival, timeout_s=1800)
    wall = time.perf_counter() - t0
    st1 = srv.stats()
    # counters over the timed replay; maxima ("max" in the name) are the
    # server's, warm-up included
    st = {k: (v if "max" in k else
              [a - b for a, b in zip(v, st0[k])] if isinstance(v, list) else v - st0[k])
          for k, v in st1.items()}
    srv.close()
    lat = np.array([r.latency_s for r in res]) * 1e3
    ok = all(r.status == 0 for r in res)
    ns = np.array([max(W.graphs[W.g1[i]].n, W.graphs[W.g2[i]].n) for i in range(len(res))])
    big = ns > 2048
    iso = W.kind == 1
    block = {
        "workload": (f"open-loop Poisson stream, {len(res)} requests at {args.serve_rate:.0f}/s; "
                     f"sizes 90% n<=128, 9% 128<n<=2048, 1% 2048<n<={args.serve_nmax}; tree "
                     f"(max deg 4) + 0-6 edges; 30% iso pairs (half relabelings), 20% of "
                     f"canonizations relabeled repeats"),
        "requests": len(res), "all_ok": ok, "wall_s": wall,
        "throughput_req_s": len(res) / wall,
        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
        "p999_ms": float(np.percentile(lat, 99.9)), "max_ms": float(lat.max()),
        "p50_ms_n_le_2048": float(np.percentile(lat[~big], 50)),
        "p99_ms_n_le_2048": float(np.percentile(lat[~big], 99)),
        "p50_ms_iso": float(np.percentile(lat[iso], 50)) if iso.any() else None,
        "large_requests": int(big.sum()),
        "p50_p99_ms_by_size": {
            name: [float(np.percentile(lat[m], 50)), float(np.percentile(lat[m], 99)), int(m.sum())]
            for name, m in (("n<=64", ns <= 64), ("65-256", (ns > 64) & (ns <= 256)),
                            ("257-2048", (ns > 256) & (ns <= 2048)), (">2048", ns > 2048))
            if m.any()},
        "batches": st["batches"], "graphs": st["graphs"], "memo_hits": st["memo_hits"],
        "per_class": {name: {"batches": st["class_batches"][c],
                             "mean_batch_ms": st["class_batch_ns"][c] / 1e6 / max(st["class_batches"][c], 1),
                             "mean_queue_ms": st["class_queue_ns"][c] / 1e6 / max(st["class_batches"][c], 1)}
                      for c, name in enumerate(("small", "mid", "big", "large"))},
        "class_repeats": st["class_repeats"],
        "dispatcher_max_ms": {name: {"launch": st["class_max_launch_ns"][c] / 1e6,
                                     "complete": st["class_max_complete_ns"][c] / 1e6}
                              for c, name in enumerate(("small", "mid", "big", "large"))},
        "tail_timeline_ms": _tail_timeline(res, lat, ns),
        "enqueue_part_max_ms": dict(zip(("pinned_buffers", "device_buffers", "pack",
                                         "copies_in", "search_launch", "table_and_copies_out"),
                                        (x / 1e6 for x in st["enqueue_part_max_ns"]))),
    }
    # the size tail beyond the stream's n_max (config: 1% up to 20,000):
    # single requests of the stream's family, each alone on the server, with
    # a time budget; what bounds them is the reference's search on trees
    # (its node count grows about quadratically with n), each node a
    # refinement of the whole graph
    big = {}
    old = os.environ.get("GCL_GRAPH_BUDGET_S")
    os.environ["GCL_GRAPH_BUDGET_S"] = str(args.serve_large_budget_s)
    try:
        rng = np.random.default_rng(5002)
        for n in args.serve_large_sizes:
            g = G.tree_plus_edges(n, rng)
            srv = pkg.Server(local)
            t = time.perf_counter()
            r = srv.replay(G.pack([g]), np.zeros(1, np.int32), np.zeros(1, np.int32),
                           np.zeros(1, np.int32), np.zeros(1), timeout_s=args.serve_large_budget_s + 60)
            dt = time.perf_counter() - t
            srv.close()
            big[str(n)] = {"status": int(r[0].status), "latency_ms": r[0].latency_s * 1e3,
                           "gpu_ms": (r[0].gpu_done_s - r[0].launch_s) * 1e3, "wall_ms": dt * 1e3}
    finally:
        if old is None:
            os.environ.pop("GCL_GRAPH_BUDGET_S", None)
        else:
            os.environ["GCL_GRAPH_BUDGET_S"] = old
    block["size_tail_alone"] = {"budget_s": args.serve_large_budget_s,
                                "family": "tree (max deg 4) + 0-6 edges", "requests": big}
    # the plain form under the same arrivals: the first requests served one
    # at a time in arrival order, each graph through its own gcl_canon_one
    # call; service times are measured, queueing (FIFO, one server) follows
    # from the arrival times
    ctx = pkg.Context(local)
    k = min(len(res), args.serve_plain)
    for i in range(min(20, k)):
        pkg.canon(W.graphs[W.g1[i]], ctx=ctx)
    svc = np.zeros(k)
    for i in range(k):
        t = time.perf_counter()
        pkg.canon(W.graphs[W.g1[i]], ctx=ctx)
        if W.kind[i] == 1:
            pkg.canon(W.graphs[W.g2[i]], ctx=ctx)
        svc[i] = time.perf_counter() - t
    ctx.close()
    done, plat = 0.0, np.zeros(k)
    for i in range(k):
        start = max(W.arrival[i], done)
        done = start + svc[i]
        plat[i] = done - W.arrival[i]
    plat *= 1e3
    block["plain_one_per_launch"] = {
        "sample": f"the first {k} requests in arrival order, one gcl_canon_one per graph, "
                  f"FIFO single server at the same arrival times",
        "p50_ms": float(np.percentile(plat, 50)), "p99_ms": float(np.percentile(plat, 99)),
        "service_p50_ms": float(np.percentile(svc, 50) * 1e3),
        "capacity_req_s": k / float(svc.sum()),
        "served_p50_ms_same_requests": float(np.percentile(lat[:k], 50)),
        "served_p99_ms_same_requests": float(np.percentile(lat[:k], 99))}
    return block


def single_graph_block(args, pkg, local, with_cpu):
    """Search-heavy single graphs through gcl_canon_one (the wide search),
    each also under a random relabeling; the reference CPU path beside the
    ones it finishes in seconds."""
    G = pkg.graphs
    rng = np.random.default_rng(2000)
    cases = [("reg3_n1024", G.random_regular(1024, 3, rng), True),
             ("reg3_n4096", G.random_regular(4096, 3, rng), False),
             ("torus_32x32", G.torus(32), True), ("torus_64x64", G.torus(64), True)]
    if args.single_extra:
        cases += [("tree_n2048", G.from_edges(2048, G.recursive_tree(2048, rng)), True),
                  ("union_5x_reg3_32", G.disjoint_union(G.random_regular(32, 3, rng), 5), True)]
    ctx = pkg.Context(local)
    if args.single_gate != 1:
        ctx.set_option(pkg.api.GCL_OPT_WIDE_GATE, args.single_gate)
    if args.single_share:
        ctx.set_option(pkg.api.GCL_OPT_WIDE_SHARE, 1)
    pkg.canon(G.from_edges(3, [(0, 1)]), ctx=ctx)
    out = {}
    O = None
    if with_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O  # the reference's CPU path (the oracle / baseline)
    for name, g, cpu in cases:
        rel = G.random_relabel(g, rng)
        pkg.canon(g, ctx=ctx)  # warm-up (workspace)
        t = time.perf_counter()
        a = pkg.canon(g, ctx=ctx)
        t1 = time.perf_counter()
        b = pkg.canon(rel, ctx=ctx)
        t2 = time.perf_counter()
        row = {"n": g.n, "gpu_ms": (t1 - t) * 1e3, "gpu_ms_relabeled": (t2 - t1) * 1e3,
               "nodes": a.nodes, "relabel_invariant": bool(np.array_equal(a.matrix, b.matrix))}
        if cpu and O is not None and O.available("reference"):
            t = time.perf_counter()
            m = O.canon(g, kind="reference")[0]
            row["cpu_ref_ms"] = (time.perf_counter() - t) * 1e3
            row["equal_to_cpu_ref"] = bool(np.array_equal(m, a.matrix))
        out[name] = row
    ctx.close()
    out["union_reg4_64"] = union_block(args, pkg, local)
    return out


def union_block(args, pkg, local):
    """Disjoint unions of k copies of one random 4-regular graph on 64
    vertices (seed 66, the fixture's union family) through the wide search
    with work sharing: k = 2..6 against the reference's canonical forms in
    the fixture, and k = 16 (beyond the reference: 8 copies take it minutes)
    under a time budget, relabeling-checked when it finishes."""
    G = pkg.graphs
    gold = _golden_large()
    comp = G.random_regular(64, 4, np.random.default_rng(66))
    ctx = pkg.Context(local)
    ctx.set_option(pkg.api.GCL_OPT_WIDE_SHARE, 1)
    out = {"copies_vs_reference": {}}
    old = os.environ.get("GCL_GRAPH_BUDGET_S")
    try:
        for k in (2, 3, 4, 5, 6):
            g = G.disjoint_union(comp, k)
            t = time.perf_counter()
            rows, nodes, _ = pkg.api.canon_rows(g, ctx=ctx)
            rec = gold.get(f"union_reg4_64_x{k}")
            out["copies_vs_reference"][k] = {
                "gpu_ms": (time.perf_counter() - t) * 1e3, "nodes": nodes,
                "reference_nodes": rec["nodes"] if rec else None,
                "reference_single_core_s": rec["ref_seconds"] if rec else None,
                "equal_to_reference": bool(rec and _rows_sha256(rows) == rec["rows_sha256"])}
        os.environ["GCL_GRAPH_BUDGET_S"] = str(args.union_budget_s)
        g = G.disjoint_union(comp, 16)
        row = {"n": g.n, "budget_s": args.union_budget_s}
        t = time.perf_counter()
        try:
            a, nodes, _ = pkg.api.canon_rows(g, ctx=ctx)
            row.update(gpu_ms=(time.perf_counter() - t) * 1e3, nodes=nodes, finished=True)
            b, _, _ = pkg.api.canon_rows(G.random_relabel(g, np.random.default_rng(16)), ctx=ctx)
            row["relabel_invariant"] = bool(np.array_equal(a, b))
        except pkg.GclError as e:
            row.update(gpu_ms=(time.perf_counter() - t) * 1e3, finished=False, status=int(e.rc))
        out["copies_16"] = row
    finally:
        if old is None:
            os.environ.pop("GCL_GRAPH_BUDGET_S", None)
        else:
            os.environ["GCL_GRAPH_BUDGET_S"] = old
        ctx.close()
    return out


def _golden_large():
    """The reference's outputs at the configurations' sizes (the committed
    fixture tests/golden/golden_large.json: recipes and hashes), by name."""
    p = os.path.join(ROOT, "tests", "golden", "golden_large.json")
    if not os.path.exists(p):
        return {}
    with open(p) as f:
        return {r["name"]: r for r in json.load(f)["records"]}


def _rows_sha256(rows) -> str:
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(rows, dtype=np.uint64).tobytes()).hexdigest()


def mixed_block(args, pkg, local):
    """Mixed-size batch (n log-uniform in [64, 4096], four families), one
    batched call with a per-graph time budget: some unions of identical
    components take the reference's sequential search minutes, so a graph
    past the budget reports a timeout instead of holding the batch.  The
    graphs that finish are checked against the reference's canonical forms
    where the fixture has them.  The autotuner picks the launch shapes on a
    sample of quick graphs first; the default shapes are timed too."""
    G = pkg.graphs
    gs = G.mixed_batch(args.mixed_graphs, seed=4000)
    arena = G.pack(gs)
    gold = _golden_large()
    quick = [i for i in range(len(gs)) if gold.get(f"mixed_{i}", {}).get("ref_seconds", 1e9) < 0.02]
    old = os.environ.get("GCL_GRAPH_BUDGET_S")
    os.environ["GCL_GRAPH_BUDGET_S"] = str(args.mixed_budget_s)
    try:
        out = {"workload": f"{arena.count} graphs, n log-uniform [64,4096], ER(deg 8) / "
                           f"d-regular d in {{3,4,6}} / tori / 2-4 copies of a regular component "
                           f"(seed 4000)",
               "graph_budget_s": args.mixed_budget_s}
        tuning = None
        for label, tune, handoff in (("default_shapes", False, 0), ("autotuned", True, 0),
                                     ("autotuned_handoff", True, args.mixed_handoff_ms)):
            ctx = pkg.Context(local)
            if tune and quick:
                if tuning is None:
                    tuning = ctx.autotune([gs[i] for i in quick[:200]], repeats=1)
                    out["tuning"] = tuning
                else:
                    ctx.set_tuning(tuning)
            if handoff:
                ctx.set_option(pkg.api.GCL_OPT_BATCH_HANDOFF_MS, handoff)
            warm = [gs[i] for i in quick[:64]] or gs[:1]
            pkg.canon_batch(warm, ctx=ctx, dense=False, rows=True)  # workspace warm-up
            t = time.perf_counter()
            r = pkg.canon_batch(arena, ctx=ctx, dense=False, rows=True, per_graph_errors=True)
            dt = time.perf_counter() - t
            ctx.close()
            ok = r.status == 0
            checked = same = 0
            for i in np.flatnonzero(ok):
                rec = gold.get(f"mixed_{i}")
                if rec is not None:
                    checked += 1
                    same += _rows_sha256(r.packed(int(i))) == rec["rows_sha256"]
            out[label] = {"seconds": dt, "graphs_finished": int(ok.sum()),
                          "handoff_ms": handoff,
                          "graphs_timed_out": int((r.status == 5).sum()),
                          "other_status": int(((~ok) & (r.status != 5)).sum()),
                          "graphs_per_s": float(ok.sum()) / dt,
                          "checked_against_reference": checked,
                          "equal_to_reference": same,
                          "max_nodes_finished": int(r.stats[ok, 1].max()) if ok.any() else 0}
        # the plain form: the finished graphs one launch each, on a sample
        ctx = pkg.Context(local)
        sample = [i for i in quick[: args.mixed_plain]]
        if sample:
            for i in sample[:5]:
                pkg.canon_batch([gs[i]], ctx=ctx, dense=False, rows=True)
            t = time.perf_counter()
            for i in sample:
                pkg.canon_batch([gs[i]], ctx=ctx, dense=False, rows=True)
            dt = time.perf_counter() - t
            out["plain_per_launch_quick_sample"] = {
                "graphs": len(sample), "graphs_per_s": len(sample) / dt,
                "sample": "graphs the reference finishes in under 20 ms, one gcl_canon_batch "
                          "call each"}
        ctx.close()
        ref = [gold[f"mixed_{i}"]["ref_seconds"] for i in range(len(gs)) if f"mixed_{i}" in gold]
        out["reference_single_core_seconds_of_fixture_graphs"] = {
            "graphs": len(ref), "seconds": float(np.sum(ref)),
            "note": "the reference's sequential path on one core of the build container, from "
                    "the fixture (graphs it finishes within 5 s); not timed on this box"}
        return out
    finally:
        if old is None:
            os.environ.pop("GCL_GRAPH_BUDGET_S", None)
        else:
            os.environ["GCL_GRAPH_BUDGET_S"] = old


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
