"""Benchmark of the Q1 hot path on B200 (one JSON line on rank 0).

Workload (N=1): 600,000,000 rows of the seeded lineitem generator, compressed (uint16 day offset,
uint8 quantity/discount/tax, uint32 cents, 2-bit (returnflag, linestatus) pair codes: 9.25 B/row),
HBM-resident, default placement in_registers_per_thread, cutoff 1998-09-02. A step is one pass of
the scan kernel over the whole table (inputs 5.55 GB > 126 MB L2, so no L2 flush is needed).

  value     rows/s of the scan kernel with inputs resident in HBM (CUDA events, launch stream)
  e2e       rows/s through the public C ABI q1_run with the table in pinned HOST memory, so every
            step copies the columns host->device (4 streams) and reads the result back
  roofline  algorithmic bytes per launch (9.25 B/row x rows) / average launch duration vs the
            measured HBM copy bandwidth (MEASURED_PEAKS.json)
  cpu_baseline  the reference's own CPU kernel (KernelX100<kMagic,true,kNoAvx512>, oracle/_ref)
            on the host cores, on a bounded sample of the same generator

--impl reference: the reference's CPU implementation of the path (oracle/_ref) on all host
threads, timed on a bounded sample per step. N>1 (torchrun): every rank scans its own 600M-row
shard (weak scaling) and the per-group partials are exchanged once per step (all_gather of
36 x 128-bit, summed exactly on the host).
"""
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

METRIC = "rows/s & HBM GB/s (% peak), bit-exact; batched/served vs plain, p50/p99 ms"
UNIT = "rows/s"
ROWS = 600_000_000
DEFAULT_ROWS = ROWS
SEED = 20260102
BYTES_PER_ROW = 9.25          # 2 + 1 + 1 + 1 + 4 + 2/8
CUTOFF = 729999
WORKLOAD = "q1_600M_compressed_hbm"


def config_dict(n_gpus, placement):
    return {"workload": WORKLOAD, "rows_per_gpu": ROWS, "layout": "compressed 9.25 B/row (u16 ship, u8 qty/disc/tax, "
            "u32 price, 2-bit pair codes)", "placement": placement, "cutoff_day": CUTOFF,
            "residency": "hbm", "l2": "inputs 5.55 GB per pass > 126 MB L2 (no flush needed)",
            "parallelism": f"shard{n_gpus}" if n_gpus > 1 else "single"}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per launch of the scan kernel from the committed ncu summary, scaled to 600M rows."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            t = json.load(f)
        return float(t["bytes_per_row"]) * ROWS
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.reader = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.reader:
            self.reader.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_info():
    model = ""
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                model = ln.split(":", 1)[1].strip()
                break
    except Exception:
        pass
    return model, os.cpu_count()


REF_CHUNK_ROWS = 1 << 25      # 33.5 M rows per chunk of the reference's table


def reference_chunks(rows, seed, threads=None, first_row=0):
    """The reference's KernelX100 (oracle/_ref, built from the reference sources) over `rows` rows
    of the generator, the inputs generated by the oracle itself (oracle/gen_rows.h) and held as
    chunks of the reference's compact copy (12 B/row); no product code is loaded."""
    from oracle import py_oracle as O
    return O.RefChunks(seed, first_row, rows, chunk_rows=REF_CHUNK_ROWS, cutoff_day=CUTOFF, threads=threads)


def time_reference(chunks, seconds=None, steps=None, warmup=0):
    """Times full passes of KernelX100 over every chunk: (rows/s, threads, pass times, last table)."""
    for _ in range(warmup):
        chunks.run()
    times, table = [], None
    t0 = time.perf_counter()
    while True:
        s = time.perf_counter()
        table, rc = chunks.run()
        times.append(time.perf_counter() - s)
        if rc != 0:
            raise RuntimeError(f"reference KernelX100 run failed: {rc}")
        if steps is not None and len(times) >= steps:
            break
        if seconds is not None and time.perf_counter() - t0 >= seconds and len(times) >= 3:
            break
    return chunks.rows * len(times) / sum(times), chunks.threads(), times, table


def reference_comparators(rows=20_000_000, reps=3):
    """The reference's single-thread tuple-at-a-time kernels as extra CPU comparators (rows/s,
    best of `reps`): KernelHyPer<true> on the int64 columns and KernelHyPerCompact<true> on the
    compact int8/int16/int32 copy. The reference's AVX-512 kernel (cpu/kernel_avx512.hpp) is
    disabled in the reference (cpu/q1.cpp:14-15) and gathers/scatters through the addresses of
    its table pointers ((int64_t*)&aggr_avx0_count, :178-184) instead of the tables, so it is not
    run."""
    from oracle import py_oracle as O
    out = {}
    for name, shift, fn in [("hyper_1_thread", 0, "hyper"), ("hyper_compact_1_thread", O.HYPER_COMPACT_SHIFT,
                                                             "hyper_compact")]:
        t = O.RefTable.generated(SEED, 0, rows, CUTOFF - shift)
        try:
            best = None
            for _ in range(reps):
                s = time.perf_counter()
                _, flag = getattr(t, fn)()
                el = time.perf_counter() - s
                best = el if best is None else min(best, el)
            out[name] = {"rows_per_s": rows / best, "rows": rows, "overflow": bool(flag)}
        finally:
            t.close()
    return out


def reference_gpu_arm(args):
    """The reference's own compressed GPU kernels (src/kernels/*, built unmodified for sm_100a
    into oracle/_ref/libq1refgpu.so) on the same B200, HBM-resident separate-flags layout
    (9.375 B/row), one launch over the whole table with the reference's launch formula; for each
    placement the best of a tuples-per-thread sweep is reported."""
    import ctypes
    import torch
    import tpchq01_gpu_b200 as q
    from tpchq01_gpu_b200 import _lib
    path = os.path.join(ROOT, "oracle", "_ref", "libq1refgpu.so")
    if not os.path.exists(path):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libq1refgpu.so not built"}), flush=True)
        return 0
    R = ctypes.CDLL(path)
    R.refgpu_launch_compressed.restype = ctypes.c_int
    R.refgpu_launch_compressed.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 9 + [
        ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    torch.cuda.set_device(0)
    ctx = q.Q1Context()
    ctx.generate(SEED, ROWS, layout="compressed", packing="separate")
    comp, _, rows, _, _ = ctx.table_columns()
    filt = torch.empty((rows + 31) // 32 + 8, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    q.precompute_filter(comp.shipdate, rows, CUTOFF, filt.data_ptr(), stream.cuda_stream)
    sums = torch.zeros(32, dtype=torch.int64, device="cuda")
    counts = torch.zeros(8, dtype=torch.int32, device="cuda")
    peak, _ = measured_peaks()
    results = []
    for pushdown in [0, 1]:
        bpr = 7.5 if pushdown else 9.375
        for pid, pname in enumerate(["in_registers", "in_registers_per_thread", "local_mem", "shared_mem_per_thread",
                                     "global"]):
            best = None
            for tpt in [1, 4, 16, 64, 256, 1024]:
                def launch():
                    sums.zero_()
                    counts.zero_()
                    rc = R.refgpu_launch_compressed(pid, pushdown, sums.data_ptr(), counts.data_ptr(),
                                                    filt.data_ptr() if pushdown else comp.shipdate, comp.discount,
                                                    comp.extendedprice, comp.tax, comp.quantity, comp.returnflag,
                                                    comp.linestatus, rows, 256, tpt, stream.cuda_stream)
                    if rc:
                        raise RuntimeError(f"reference kernel launch failed: {rc}")
                for _ in range(2):
                    launch()
                torch.cuda.synchronize()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                reps = max(1, min(args.steps, 5))
                a.record(stream)
                for _ in range(reps):
                    launch()
                b.record(stream)
                torch.cuda.synchronize()
                ms = a.elapsed_time(b) / reps
                if best is None or ms < best["ms"]:
                    best = {"placement": pname, "pushdown": bool(pushdown), "tuples_per_thread": tpt, "ms": ms,
                            "rows_per_s": rows / (ms / 1e3), "gbs": bpr * rows / (ms / 1e3) / 1e9}
            best["frac_hbm"] = best["gbs"] / peak
            results.append(best)
            print(json.dumps(best), file=sys.stderr, flush=True)
    ctx.close()
    top = max(results, key=lambda r: r["rows_per_s"])
    line = {"impl": "reference", "kind": "reference_gpu_same_box", "metric": METRIC, "value": top["rows_per_s"],
            "unit": UNIT, "n_gpus": 1, "higher_is_better": True, "dtype": "int64", "data": "synthetic",
            "config": {"workload": WORKLOAD + "_separate_flags", "rows": rows, "cutoff_day": CUTOFF,
                       "layout": "compressed, separate rf (2-bit) and ls (1-bit) containers, 9.375 B/row "
                                 "(7.5 B/row with the filter bitmap)", "residency": "hbm"},
            "best": top, "placements": results}
    print(json.dumps(line), flush=True)
    return 0


def reference_arm(args, rank):
    """The reference's own CPU implementation of the path (KernelX100 on all host threads) on
    this arm's workload: every step is one pass over all 600 M rows (chunks of 33.5 M rows of the
    reference's compact copy, resident in host memory)."""
    if rank != 0:
        return 0
    if args.ref_gpu:
        return reference_gpu_arm(args)
    model, ncpu = cpu_info()
    t0 = time.perf_counter()
    chunks = reference_chunks(ROWS, SEED)
    build_s = time.perf_counter() - t0
    try:
        value, used, times, _ = time_reference(chunks, steps=args.steps, warmup=args.warmup)
        nchunks = chunks.chunks()
    finally:
        chunks.close()
    desc = (f"reference KernelX100<kMagic,true,kNoAvx512> (cpu/kernel_x100.hpp) on {used} host threads, all "
            f"{ROWS:,} rows per step in {nchunks} chunks of its compact copy ({model})")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic", "config": dict(config_dict(args.gpus, args.placement), residency="host"),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": used, "kind": "reference", "sample": desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "setup_s": build_s}
    try:
        line["comparators"] = reference_comparators()
    except Exception as e:   # informative only
        line["comparators"] = {"unavailable": str(e)}
    print(json.dumps(line), flush=True)
    return 0


def main():
    global ROWS
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--placement", default="in_registers_per_thread")
    ap.add_argument("--rows", type=int, default=ROWS)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--pushdown", action="store_true", help="scan: read the predicate bitmap (filter pushdown)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="scan mode: leave out the batched-vs-plain (C3) object")
    ap.add_argument("--no-serve", action="store_true", help="scan mode: leave out the served-vs-plain (C4) object")
    ap.add_argument("--mode", default="scan", choices=["scan", "c1sweep", "groupkey", "batch", "serve", "tbl"],
                    help="scan: the 600M-row aggregation (default); batch: 256 instances in one persistent "
                         "launch vs one plain launch each; serve: Poisson request stream, served vs plain")
    ap.add_argument("--instances", type=int, default=256)
    ap.add_argument("--groups", default="4,64,1024,65536", help="groupkey: group counts to sweep")
    ap.add_argument("--pass-fracs", default="0.01,0.10,0.50,0.98,1.0", help="groupkey: pass fractions to sweep")
    ap.add_argument("--key-dists", default="uniform,zipf", help="groupkey: key distributions to sweep")
    ap.add_argument("--placements", default="", help="groupkey: placements to time (default: every one that applies)")
    ap.add_argument("--batch-groups", default="4,64,1024", help="batch: group counts instances draw from")
    ap.add_argument("--tune", type=int, default=1, help="batch: 0 heuristic placements, 1 autotuner")
    ap.add_argument("--ref-gpu", action="store_true",
                    help="with --impl reference: the reference's own GPU kernels on this GPU instead of its CPU kernels")
    ap.add_argument("--packing", default="pair", choices=["pair", "separate"],
                    help="scan: flag packing of the table (pair 9.25 B/row, separate 9.375 B/row)")
    ap.add_argument("--duration", type=float, default=60.0, help="serve: seconds of Poisson arrivals per arm")
    ap.add_argument("--rate", type=float, default=2000.0, help="serve: mean requests per second")
    args = ap.parse_args()
    ROWS = args.rows
    if args.mode == "groupkey" and args.impl == "ours":
        return bench_groupkey(args)
    if args.mode == "c1sweep" and args.impl == "ours":
        return bench_c1sweep(args)
    if args.mode == "batch" and args.impl == "ours":
        return bench_batch(args)
    if args.mode == "serve" and args.impl == "ours":
        return bench_serve(args)
    if args.mode == "tbl" and args.impl == "ours":
        return bench_tbl(args)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return reference_arm(args, rank)

    import torch
    import tpchq01_gpu_b200 as q
    from tpchq01_gpu_b200 import _lib

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))

    from tpchq01_gpu_b200 import shard

    # Table: this rank's shard of the generator, compressed, HBM-resident.
    ctx = q.Q1Context(device=local_rank)
    first_row, shard_rows = shard.shard_rows(ROWS, rank)
    ctx.generate(SEED, shard_rows, first_row=first_row, layout="compressed", packing=args.packing)
    comp, _, rows, _, _ = ctx.table_columns()
    aggs = torch.zeros(36 * 2, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    launches = [0]
    if args.pushdown:
        # filter pushdown: the kernels read the predicate bitmap (1 bit/row) instead of ship dates
        filt = torch.empty((rows + 31) // 32 + 8, dtype=torch.int32, device="cuda")
        q.precompute_filter(comp.shipdate, rows, CUTOFF, filt.data_ptr(), sh)
        comp.filter = filt.data_ptr()

    def step():
        aggs.zero_()
        q.launch_compressed(args.placement, comp, rows, CUTOFF, args.pushdown, aggs.data_ptr(), sh)
        launches[0] += 1

    def exchange():
        if world > 1:
            return shard.gather_partials(aggs, dist)
        return [aggs]

    for _ in range(max(args.warmup, 3)):
        step()
        exchange()
    q.sync_check(sh)
    torch.cuda.synchronize()

    sampler = ClockSampler(local_rank)
    sampler.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches[0] = 0
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for i in range(args.steps):
        aggs.zero_()
        ev[i][0].record(stream)
        q.launch_compressed(args.placement, comp, rows, CUTOFF, args.pushdown, aggs.data_ptr(), sh)
        launches[0] += 1
        ev[i][1].record(stream)
        exchange()
    t_end.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    q.sync_check(sh)
    total_ms = t_start.elapsed_time(t_end)
    kern_ms = [a.elapsed_time(b) for a, b in ev]
    if dist:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    # exact merged result of the last step (per-group int128 partials summed on the host)
    merged = shard.merge_partials(exchange())

    value = world * ROWS * args.steps / (total_ms / 1000.0)
    avg_kernel_s = sum(kern_ms) / len(kern_ms) / 1000.0
    bytes_per_row = (BYTES_PER_ROW if args.packing == "pair" else 9.375) - (1.875 if args.pushdown else 0.0)
    achieved = bytes_per_row * ROWS / avg_kernel_s / 1e9
    peak, peak_kind = measured_peaks()
    traffic = profiled_traffic() if args.packing == "pair" and not args.pushdown else None

    result = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
              "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
              "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
              "config": dict(config_dict(world, args.placement), **(
                  {} if args.packing == "pair" else {"layout": "compressed 9.375 B/row (separate rf/ls containers)"}),
                  **({"filter_pushdown": True, "bytes_per_row": bytes_per_row} if args.pushdown else {})),
              "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                           "frac": achieved / peak, "traffic": traffic, "peak_kind": f"{peak_kind} (hbm_gbs)",
                           "kernel_ms": sum(kern_ms) / len(kern_ms)},
              "gpu_launches": launches[0], "clocks": clocks,
              "check": {"groups_count_sum": int(sum(int(merged[g, 0]) for g in range(6)))}}

    if not args.no_e2e:
        if world == 1:
            result["e2e"] = e2e_pinned(q, args)
        else:   # every rank takes part (a collective); rank 0 reports
            result["e2e"] = e2e_sharded(q, args, rank, world, local_rank, dist)
    if rank == 0 and world == 1 and not args.no_cpu:
        # The reference's KernelX100 over the same 600 M rows: the timed CPU baseline, and its
        # table is the parity check of the GPU table of the timed steps (tolerance 0).
        model, ncpu = cpu_info()
        chunks = reference_chunks(ROWS, SEED)
        try:
            v, used, times, ref_table = time_reference(chunks, seconds=8.0, warmup=1)
            nchunks = chunks.chunks()
        finally:
            chunks.close()
        result["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": used, "kind": "reference",
                                  "sample": f"reference KernelX100<kMagic,true,kNoAvx512> on {used} threads, all "
                                            f"{ROWS:,} rows of the same generator per pass ({nchunks} chunks), "
                                            f"{len(times)} passes ({model})"}
        identical = all(int(merged[g][a]) == int(ref_table[g][a]) for g in range(6) for a in range(6))
        result["parity"] = {"rows": ROWS, "identical": bool(identical), "tolerance": 0,
                            "against": "reference KernelX100 (cpu/kernel_x100.hpp) on the same generated rows, "
                                       "every group x {count, sum_qty, sum_base_price, sum_disc, "
                                       "sum_disc_price, sum_charge} as exact integers",
                            "table": [[str(int(merged[g][a])) for a in range(6)] for g in range(6)]}
    ctx.close()
    # No number of a run under a profiler is a bench value, and the batched and served forms are
    # thousands of launches, two of them persistent kernels meant to run side by side: profile the
    # scan with --no-batch --no-serve (the committed profile commands do). An injection variable in
    # the environment, where a tool sets one, also leaves them out; not every ncu sets it.
    profiled = any(os.environ.get(k) for k in ("CUDA_INJECTION64_PATH", "NV_COMPUTE_PROFILER_PERFWORKS_DIR"))
    if world == 1 and profiled:
        result["batch"] = result["serve"] = {"skipped": "running under a profiler"}
    if world == 1 and not profiled:
        # the metric's second half: batched and served forms against plain launches on this GPU
        torch.cuda.empty_cache()
        if not args.no_batch:
            b = run_batch(args)
            result["batch"] = {k: b[k] for k in ["config", "batched", "plain_launches", "plain_synchronised",
                                                 "speedup_vs_plain", "speedup_vs_plain_synchronised", "identical",
                                                 "clocks"]}
            result["gpu_launches_batch"] = b["gpu_launches"]
        if not args.no_serve:
            result["serve"] = run_serve(args)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)
    if result.get("parity", {}).get("identical") is False:
        print("parity failure: the GPU table differs from the reference's", file=sys.stderr, flush=True)
        return 1
    if result.get("batch", {}).get("identical") is False or result.get("serve", {}).get("identical") is False:
        print("parity failure: a batched or served result differs from the plain launch", file=sys.stderr, flush=True)
        return 1
    return 0


def event_timed(call):
    """Seconds one synchronous public-API call takes, from CUDA events recorded on the current
    stream right before and right after it (the call returns once its copies, kernels and host
    work are done, so the events bracket all of it)."""
    import torch
    stream = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    call()
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b) / 1e3


def e2e_sharded(q, args, rank, world, local_rank, dist):
    """e2e at N > 1 GPUs (weak scaling): every rank streams its own 600 M-row shard from pinned host
    memory through q1_run over its own PCIe link (GPU only: filter pushdown and coprocessing would
    have every rank's host threads contend for the same cores); the job's rows over the slowest
    rank's time."""
    import torch
    ctx = q.Q1Context(device=local_rank, cpu_threads=1)
    try:
        from tpchq01_gpu_b200 import shard
        first_row, rows = shard.shard_rows(ROWS, rank)
        ctx.generate(SEED, rows, first_row=first_row, layout="compressed", packing="pair", residency="pinned")
        p = q.Q1Params(hash_table_placement=args.placement, apply_compression=True, num_gpu_streams=4,
                       num_tuples_per_kernel_launch=1 << 24, num_query_execution_runs=1, cutoff_day=CUTOFF)
        ctx.run(p)
        steps = max(3, min(args.steps, 10))
        dist.barrier()
        el = torch.tensor([sum(event_timed(lambda: ctx.run(p)) for _ in range(steps))], device="cuda")
        dist.all_reduce(el, op=dist.ReduceOp.MAX)
        t = float(el.item())
        h2d = int(rows * 9 + 4 * ((rows + 15) // 16)) * world
        return {"value": world * rows * steps / t, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": 576 * world, "steps": steps, "ms_per_step": 1000 * t / steps,
                "path": f"q1_run on each of {world} ranks, PINNED_HOST residency (its own shard), GPU only, "
                        "4 streams x 16M-row chunks; the slowest rank's wall time"}
    finally:
        ctx.close()


def e2e_pinned(q, args):
    """Same workload through the public API with host buffers: q1_run on a pinned-host table with
    the reference's own options --use-filter-pushdown --use-coprocessing: host threads build the
    predicate bitmap for the GPU's share (7.375 B/row cross PCIe instead of 9.25) and aggregate
    the CPU's share, merged exactly. The CPU fraction is picked from a short sweep during warm-up."""
    threads = max(1, (os.cpu_count() or 2) - 2)
    ctx = q.Q1Context(cpu_threads=threads)
    try:
        ctx.generate(SEED, ROWS, layout="compressed", packing="pair", residency="pinned")

        def params(frac):
            return q.Q1Params(hash_table_placement=args.placement, apply_compression=True, use_filter_pushdown=True,
                              use_coprocessing=True, cpu_processing_fraction=frac, num_gpu_streams=4,
                              num_tuples_per_kernel_launch=1 << 24, num_query_execution_runs=1, cutoff_day=CUTOFF)

        def timed(p, n):
            return [event_timed(lambda: ctx.run(p)) for _ in range(n)]

        sweep = {}
        frac, worse = 0.25, 0
        while frac < 0.86 and worse < 2:   # climb until two steps in a row are slower
            timed(params(frac), 1)
            sweep[frac] = min(timed(params(frac), 2))
            worse = worse + 1 if sweep[frac] > min(sweep.values()) else 0
            frac = round(frac + 0.05, 2)
        best = min(sweep, key=sweep.get)
        steps = max(3, min(args.steps, 10))
        t = timed(params(best), steps)
        gpu_rows = int(ROWS * (1 - best))
        cpu_rows = ROWS - gpu_rows
        bitmap = 4 * ((gpu_rows + 31) // 32)
        h2d = int(gpu_rows * 3 + gpu_rows * 4 + bitmap + 4 * ((gpu_rows + 15) // 16))
        step_s = sum(t) / steps
        # Host-memory bytes of one step: the CPU share reads its rows (9.25 B/row), the bitmap
        # producer reads the GPU rows' ship dates (2 B/row) and writes the bitmap, and the copy
        # engines read everything that crosses PCIe.
        host_bytes = int(cpu_rows * BYTES_PER_ROW + gpu_rows * 2 + bitmap + h2d)
        peaks = host_stream_peaks(q)
        roof = {"pcie_h2d_gbs": peaks["pcie_h2d_gbs"], "host_read_gbs": peaks["host_read_gbs"],
                "host_read_threads": peaks["threads"], "h2d_bytes_per_step": h2d,
                "host_bytes_per_step": host_bytes, "h2d_achieved_gbs": h2d / step_s / 1e9,
                "host_achieved_gbs": host_bytes / step_s / 1e9,
                "how": "pcie_h2d_gbs: best of 5 cudaMemcpyAsync of 2 GiB from pinned host memory (CUDA events); "
                       "host_read_gbs: best of 3 reads of a 4 GiB host buffer on all host threads "
                       "(q1_measure_host_read); both in this run"}
        roof["frac_pcie"] = roof["h2d_achieved_gbs"] / roof["pcie_h2d_gbs"] if roof["pcie_h2d_gbs"] else None
        roof["frac_host"] = roof["host_achieved_gbs"] / roof["host_read_gbs"] if roof["host_read_gbs"] else None
        t_pcie = h2d / (roof["pcie_h2d_gbs"] * 1e9) if roof["pcie_h2d_gbs"] else 0.0
        t_host = host_bytes / (roof["host_read_gbs"] * 1e9) if roof["host_read_gbs"] else 0.0
        roof["bound"] = "host_memory" if t_host >= t_pcie else "pcie"
        roof["frac"] = max(t_pcie, t_host) / step_s
        return {"value": ROWS * steps / sum(t), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 576,
                "steps": steps, "ms_per_step": 1000 * step_s,
                "path": "q1_run, PINNED_HOST residency, use_filter_pushdown + use_coprocessing, 4 streams x 16M-row "
                        "chunks (H2D + scan per chunk), host predicate bitmap and CPU share on "
                        f"{threads} threads",
                "cpu_fraction": best, "cpu_fraction_sweep_ms": {str(k): 1000 * v for k, v in sweep.items()},
                "roofline": roof}
    finally:
        ctx.close()


def host_stream_peaks(q):
    """Measured ceilings of the host-streamed mode on this box: pinned host->device copy rate over
    PCIe and the host's memory read rate on all its threads."""
    import ctypes
    import torch
    from tpchq01_gpu_b200 import _lib
    n = 2 << 30
    src = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    src.fill_(1)
    dst = torch.empty(n, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    best = None
    for _ in range(5):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        dst.copy_(src, non_blocking=True)
        b.record(stream)
        b.synchronize()
        ms = a.elapsed_time(b)
        best = ms if best is None else min(best, ms)
    del dst, src
    torch.cuda.empty_cache()
    import numpy as np
    buf = np.ones(4 << 30, dtype=np.uint8)
    threads = os.cpu_count() or 1
    g = ctypes.c_double()
    rates = []
    for _ in range(3):
        _lib.check(q.lib().q1_measure_host_read(buf.ctypes.data_as(ctypes.c_void_p), buf.nbytes, threads,
                                                ctypes.byref(g)))
        rates.append(g.value)
    del buf
    return {"pcie_h2d_gbs": n / (best / 1e3) / 1e9, "host_read_gbs": max(rates), "threads": threads}


# ------------------------------------------------------------------------------------------
# --mode c1sweep: the 600M-row table in every HBM layout (pair / separate flags, filter pushdown
# off / on, uncompressed) under every placement, then the host-streamed mode (pinned table) with
# CPU fractions 0, 0.1, 0.25, 0.5, pushdown off / on. Every result is checked against the first.
# ------------------------------------------------------------------------------------------

# ------------------------------------------------------------------------------------------
# --mode tbl: lineitem text ingestion (the reference's lineitem::FromFile path, run when no
# column cache exists). An SF-1-sized table (6,001,215 rows) written as .tbl text by
# q1_tbl_format; timed: the GPU parse of device-resident text (q1_tbl_parse_device, text bytes
# and 38 B/row of columns per pass against HBM), the file path through q1_tbl_read_file (host
# read, H2D, parse, D2H), and the reference's value types over a 1 M-row sample on one thread.
# ------------------------------------------------------------------------------------------

def bench_tbl(args):
    import ctypes
    import tempfile
    import numpy as np
    import torch
    import tpchq01_gpu_b200 as q
    from tpchq01_gpu_b200 import _lib

    L = q.lib()
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    sh = ctypes.c_void_p(stream.cuda_stream)
    rows = args.rows if args.rows != DEFAULT_ROWS else 6_001_215
    text = q.tbl_format(q.generate_host(SEED, 0, rows))
    nbytes = len(text)
    dev = torch.frombuffer(bytearray(text), dtype=torch.uint8).cuda()
    out = {"shipdate": torch.empty(rows + 1, dtype=torch.int32, device="cuda")}
    for k in ["returnflag", "linestatus"]:
        out[k] = torch.empty(rows + 1, dtype=torch.uint8, device="cuda")
    for k in ["discount", "tax", "extendedprice", "quantity"]:
        out[k] = torch.empty(rows + 1, dtype=torch.int64, device="cuda")
    o = _lib.ColumnsOut(*[out[k].data_ptr() for k in ["shipdate", "returnflag", "linestatus", "discount", "tax",
                                                       "extendedprice", "quantity"]])
    got = ctypes.c_uint64(0)

    def parse():
        _lib.check(L.q1_tbl_parse_device(ctypes.c_void_p(dev.data_ptr()), nbytes, ctypes.byref(o), rows,
                                         ctypes.byref(got), sh))

    for _ in range(max(args.warmup, 3)):
        parse()
    steps = max(1, min(args.steps, 20))
    sampler = ClockSampler(0)
    sampler.start()
    times, walls = [], []
    for _ in range(steps):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        ev0.record(stream)
        parse()                      # synchronous: count, scan, parse, read back the row count
        ev1.record(stream)
        ev1.synchronize()
        walls.append((time.perf_counter() - t0) * 1e3)
        times.append(ev0.elapsed_time(ev1))
    clocks = sampler.stop()
    ms = sorted(times)[len(times) // 2]
    wall_ms = sorted(walls)[len(walls) // 2]
    peak, kind = measured_peaks()
    moved = nbytes * 2 + rows * 38   # the text is read twice (count, parse), the columns written once
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "lineitem.tbl")
        with open(path, "wb") as f:
            f.write(text)
        q.tbl_read_file(path)        # warm the page cache
        t0 = time.perf_counter()
        cols = q.tbl_read_file(path)
        file_ms = (time.perf_counter() - t0) * 1e3
    assert len(cols["shipdate"]) == rows
    ref = None
    try:
        sys.path.insert(0, ROOT)
        from oracle import py_oracle as O
        if O.ref_available():
            sample = text[: nbytes * min(rows, 1_000_000) // max(rows, 1)]
            sample = sample[: sample.rfind(b"\n") + 1]
            t0 = time.perf_counter()
            _, srows = O.ref_parse_tbl(sample)
            ref_s = time.perf_counter() - t0
            ref = {"rows_per_s": srows / ref_s, "rows": srows, "cores": 1,
                   "kind": "reference value types (Decimal<15,2>, Char, Date) with the tokenizer restated"}
    except Exception as e:   # the reference build is optional for this mode
        ref = {"unavailable": str(e)}
    line = {"metric": "lineitem .tbl rows parsed per second", "mode": "tbl", "value": rows / (ms / 1e3),
            "unit": "rows/s", "n_gpus": 1, "steps": steps, "warmup": max(args.warmup, 3), "ms_per_step": ms,
            "higher_is_better": True, "dtype": "u8", "data": "synthetic",
            "config": {"workload": f"lineitem_tbl_{rows}_rows", "rows": rows, "text_bytes": nbytes,
                       "bytes_per_row": nbytes / rows},
            "gpu_parse": {"ms": ms, "text_gbs": nbytes / (ms / 1e3) / 1e9, "moved_gbs": moved / (ms / 1e3) / 1e9,
                          "frac_hbm": moved / (ms / 1e3) / 1e9 / peak, "peak_kind": kind,
                          "wall_ms": wall_ms,
                          "note": "CUDA events around the synchronous call on its stream (three kernels, two "
                                  "memsets, two small reads); wall_ms adds the host side"},
            "file": {"ms": file_ms, "rows_per_s": rows / (file_ms / 1e3),
                     "note": "q1_tbl_read_file from the page cache: read, H2D, parse, D2H of the columns"},
            "reference_cpu": ref, "clocks": clocks, "gpu_launches": 3}
    print(json.dumps(line), flush=True)
    return 0


def bench_c1sweep(args):
    import ctypes
    import torch
    import tpchq01_gpu_b200 as q
    from tpchq01_gpu_b200 import _lib

    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    peak, _ = measured_peaks()
    placements = ["in_registers_per_thread", "in_registers", "shared_mem_per_thread", "local_mem", "global"]
    out = torch.zeros(72, dtype=torch.int64, device="cuda")
    points, ref = [], None
    reps = max(3, min(args.steps, 10))

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        q.sync_check(sh)
        return a.elapsed_time(b) / reps

    def record(layout, pushdown, placement, bpr, ms):
        nonlocal ref
        got = out.clone()
        same = True if ref is None else bool(torch.equal(got, ref))
        ref = got if ref is None else ref
        gbs = bpr * ROWS / (ms / 1e3) / 1e9
        points.append({"layout": layout, "pushdown": pushdown, "placement": placement, "ms": ms,
                       "rows_per_s": ROWS / (ms / 1e3), "gbs": gbs, "frac_hbm": gbs / peak, "identical": same})
        print(json.dumps(points[-1]), file=sys.stderr, flush=True)

    for packing, bpr0 in [("pair", 9.25), ("separate", 9.375)]:
        ctx = q.Q1Context()
        ctx.generate(SEED, ROWS, layout="compressed", packing=packing)
        comp, _, rows, _, _ = ctx.table_columns()
        filt = torch.empty((rows + 31) // 32 + 8, dtype=torch.int32, device="cuda")
        q.precompute_filter(comp.shipdate, rows, CUTOFF, filt.data_ptr(), sh)
        comp.filter = filt.data_ptr()
        for pushdown in [False, True]:
            for pl in placements:
                def fn():
                    out.zero_()
                    q.launch_compressed(pl, comp, rows, CUTOFF, pushdown, out.data_ptr(), sh)
                ms = timed(fn)
                record(packing, pushdown, pl, bpr0 - (1.875 if pushdown else 0.0), ms)
        ctx.close()
    # uncompressed: 100M rows (3.8 GB; the host generator stages the table in host memory)
    ctx = q.Q1Context()
    urows = min(ROWS, 100_000_000)
    ctx.generate(SEED, urows, layout="uncompressed")
    _, unc, rows, _, _ = ctx.table_columns()
    uref = None
    for pl in placements:
        def fn():
            out.zero_()
            q.launch_uncompressed(pl, unc, rows, CUTOFF, out.data_ptr(), sh)
        ms = timed(fn)
        got = out.clone()
        same = True if uref is None else bool(torch.equal(got, uref))
        uref = got if uref is None else uref
        gbs = 38.0 * rows / (ms / 1e3) / 1e9
        points.append({"layout": "uncompressed", "rows": rows, "pushdown": False, "placement": pl, "ms": ms,
                       "rows_per_s": rows / (ms / 1e3), "gbs": gbs, "frac_hbm": gbs / peak, "identical": same})
        print(json.dumps(points[-1]), file=sys.stderr, flush=True)
    ctx.close()

    # host-streamed (pinned table, H2D inside every run)
    streamed = []
    ctx = q.Q1Context(cpu_threads=max(1, (os.cpu_count() or 2) - 2))
    ctx.generate(SEED, ROWS, layout="compressed", packing="pair", residency="pinned")
    for pushdown in [False, True]:
        for frac in [0.0, 0.1, 0.25, 0.5]:
            p = q.Q1Params(apply_compression=True, use_filter_pushdown=pushdown, use_coprocessing=frac > 0,
                           cpu_processing_fraction=frac, num_gpu_streams=4, num_tuples_per_kernel_launch=1 << 24,
                           num_query_execution_runs=1, cutoff_day=CUTOFF)
            ctx.run(p)
            ms = 1000 * min(event_timed(lambda: ctx.run(p)) for _ in range(3))
            gpu_b = ROWS * (1 - frac) * (7.375 if pushdown else 9.25)
            streamed.append({"pushdown": pushdown, "cpu_fraction": frac, "ms": ms, "rows_per_s": ROWS / (ms / 1e3),
                             "pcie_gbs": gpu_b / (ms / 1e3) / 1e9})
            print(json.dumps(streamed[-1]), file=sys.stderr, flush=True)
    ctx.close()
    line = {"metric": METRIC, "mode": "c1sweep", "unit": UNIT, "n_gpus": 1, "dtype": "int64", "data": "synthetic",
            "config": {"workload": WORKLOAD + "_sweep", "rows": ROWS, "cutoff_day": CUTOFF},
            "value": max(p_["rows_per_s"] for p_ in points), "higher_is_better": True,
            "identical": all(p_["identical"] for p_ in points), "hbm": points, "host_streamed": streamed}
    print(json.dumps(line), flush=True)
    return 0 if line["identical"] else 1


# ------------------------------------------------------------------------------------------
# --mode groupkey: the 600M-row table plus a uint32 group key (uniform or Zipf(1.1) over G in
# {4, 64, 1024, 65536}), cutoffs chosen so that 1/10/50/98/100% of rows pass, every placement
# timed at every point and checked bit-exact against the first placement's table.
# ------------------------------------------------------------------------------------------

def pass_cutoffs(fracs, seed, sample=1_000_000):
    """Cutoff days at which about `fracs` of the generator's rows pass (from a host sample)."""
    import numpy as np
    import tpchq01_gpu_b200 as q
    ship = np.sort(q.generate_host(seed, 0, sample)["shipdate"])
    out = []
    for f in fracs:
        out.append(int(ship[min(len(ship) - 1, int(f * len(ship)))]) if f < 1.0 else 740000)
    return out


def bench_groupkey(args):
    import ctypes
    import numpy as np
    import torch
    import tpchq01_gpu_b200 as q
    from tpchq01_gpu_b200 import _lib

    L = q.lib()
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    sh = ctypes.c_void_p(stream.cuda_stream)
    ctx = q.Q1Context()
    ctx.generate(SEED, ROWS, layout="compressed", packing="pair")
    comp, _, rows, _, _ = ctx.table_columns()
    fracs = [float(f) for f in args.pass_fracs.split(",")]
    cutoffs = pass_cutoffs(fracs, SEED)
    keys = torch.empty(rows + 16, dtype=torch.int32, device="cuda")
    points = []
    peak, _ = measured_peaks()
    groups_list = [int(g) for g in args.groups.split(",")]
    for G in groups_list:
        for dist in args.key_dists.split(","):
            cdf = None
            if dist == "zipf":
                h = np.zeros(G, dtype=np.uint32)
                _lib.check(L.q1_zipf_cdf(G, 1.1, h.ctypes.data_as(ctypes.c_void_p)))
                cdf = torch.from_numpy(h.view(np.int32)).cuda()
            _lib.check(L.q1_generate_group_keys_device(SEED + 7, 0, rows, G,
                                                       None if cdf is None else ctypes.c_void_p(cdf.data_ptr()),
                                                       ctypes.c_void_p(keys.data_ptr()), sh))
            scratch = torch.empty(int(L.q1_groupkey_scratch_bytes(G)) // 8 + 1, dtype=torch.int64, device="cuda")
            out = torch.zeros(G * 12, dtype=torch.int64, device="cuda")
            placements = ([("in_registers_per_thread", 1)] if G <= 8 else []) + [("shared_mem_per_thread", 3),
                                                                                 ("global", 4)]
            if args.placements:
                placements = [p_ for p_ in placements if p_[0] in args.placements.split(",")]
            # placements outer: a point of the global placement can take seconds of L2 atomics
            # (Zipf keys at a high pass rate), after which the GPU rests before the next point
            refs = {}
            for pname, pid in placements:
                for frac, cutoff in zip(fracs, cutoffs):
                    def launch():
                        out.zero_()
                        _lib.check(L.q1_launch_groupkey(pid, ctypes.byref(comp), ctypes.c_void_p(keys.data_ptr()), G,
                                                        rows, cutoff, None, ctypes.c_void_p(scratch.data_ptr()),
                                                        ctypes.c_void_p(out.data_ptr()), sh))
                    launch()
                    _lib.check(L.q1_sync_check(sh))
                    reps = 3
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                    for _ in range(reps):
                        launch()
                    b.record(stream)
                    torch.cuda.synchronize()
                    _lib.check(L.q1_sync_check(sh))
                    ms = a.elapsed_time(b) / reps
                    got = out.clone()
                    ref = refs.setdefault(frac, got)
                    same = bool(torch.equal(got, ref))
                    if ms > 50:
                        time.sleep(2.0)
                    gbs = 13 * rows / (ms / 1e3) / 1e9
                    points.append({"groups": G, "keys": dist, "pass_frac": frac, "cutoff_day": cutoff,
                                   "placement": pname, "ms": ms, "rows_per_s": rows / (ms / 1e3), "gbs": gbs,
                                   "frac_hbm": gbs / peak, "identical": same})
                    print(json.dumps(points[-1]), file=sys.stderr, flush=True)
    ctx.close()
    best = {}
    for p_ in points:
        k = (p_["groups"], p_["keys"], p_["pass_frac"])
        if k not in best or p_["ms"] < best[k]["ms"]:
            best[k] = p_
    line = {"metric": METRIC, "mode": "groupkey", "unit": UNIT, "n_gpus": 1, "dtype": "int64", "data": "synthetic",
            "config": {"workload": "q1_600M_groupkey", "rows": rows, "bytes_per_row": 13, "groups": groups_list,
                       "keys": ["uniform", "zipf(1.1)"], "pass_fracs": fracs, "cutoffs": cutoffs},
            "value": min(p_["rows_per_s"] for p_ in best.values()), "higher_is_better": True,
            "identical": all(p_["identical"] for p_ in points), "points": points}
    print(json.dumps(line), flush=True)
    return 0 if line["identical"] else 1


# ------------------------------------------------------------------------------------------
# --mode batch: 256 independent group-key instances (rows log-uniform in [1e4, 5e7], cutoff
# uniform in [1998-06-01, 1998-12-01], groups in {4, 64, 1024}) in one persistent launch over a
# device tile queue (CUDA graph, autotuned placements), against one plain q1_launch_groupkey per
# instance; every instance's table must be identical.
# ------------------------------------------------------------------------------------------

BATCH_BYTES_PER_ROW = 13      # ship 2 + qty 1 + disc 1 + tax 1 + price 4 + key 4


def batch_instances(n, seed, group_choices=(4, 64, 1024)):
    import numpy as np
    rng = np.random.default_rng(seed)
    rows = np.exp(rng.uniform(np.log(1e4), np.log(5e7), n)).astype(np.int64)
    cutoffs = rng.integers(729906, 730090, n)
    groups = rng.choice(list(group_choices), n)
    return [(int(r), int(c), int(g)) for r, c, g in zip(rows, cutoffs, groups)]


def bench_batch(args):
    line = run_batch(args)
    print(json.dumps(line), flush=True)
    return 0 if line["identical"] else 1


def run_batch(args):
    """C3: the 256 instances in one CUDA-graph launch of the persistent batch kernels against one
    plain q1_launch_groupkey per instance; returns the JSON object (results compared bit for bit)."""
    import ctypes
    import tempfile
    import torch
    import tpchq01_gpu_b200 as q
    from tpchq01_gpu_b200 import _lib

    L = q.lib()
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    sh = ctypes.c_void_p(stream.cuda_stream)
    choices = tuple(int(g) for g in args.batch_groups.split(","))
    spec = batch_instances(args.instances, SEED + 3, choices)
    keep, descs, outs_b, outs_p, scratch = [], [], [], [], []
    for i, (rows, cutoff, g) in enumerate(spec):
        cols = {k: torch.empty(rows * w + 64, dtype=torch.uint8, device="cuda")
                for k, w in [("shipdate", 2), ("discount", 1), ("extendedprice", 4), ("tax", 1), ("quantity", 1)]}
        keys = torch.empty(rows * 4 + 64, dtype=torch.uint8, device="cuda")
        flags = torch.empty(4 * ((rows + 15) // 16) + 64, dtype=torch.uint8, device="cuda")
        out = _lib.CompressedHostOut()
        for k, t in cols.items():
            setattr(out, k, t.data_ptr())
        out.flags = flags.data_ptr()
        _lib.check(L.q1_generate_compressed_device(SEED + 1000 + i, 0, rows, 0, ctypes.byref(out), sh))
        _lib.check(L.q1_generate_group_keys_device(SEED + 1000 + i, 0, rows, g, None,
                                                   ctypes.c_void_p(keys.data_ptr()), sh))
        bi = _lib.BatchInstance()
        for k, t in cols.items():
            setattr(bi.cols, k, t.data_ptr())
        bi.keys, bi.rows, bi.cutoff_day, bi.num_groups = keys.data_ptr(), rows, cutoff, g
        ob = torch.zeros(g * 12, dtype=torch.int64, device="cuda")
        bi.aggregates = ob.data_ptr()
        keep.append((cols, keys, flags))
        descs.append(bi)
        outs_b.append(ob)
        outs_p.append(torch.zeros(g * 12, dtype=torch.int64, device="cuda"))
        scratch.append(torch.empty(int(L.q1_groupkey_scratch_bytes(g)) // 8 + 1, dtype=torch.int64, device="cuda"))
    _lib.check(L.q1_sync_check(sh))
    total_rows = sum(r for r, _, _ in spec)
    arr = (_lib.BatchInstance * len(descs))(*descs)

    def plain_pass(sync_each):
        for i, (rows, cutoff, g) in enumerate(spec):
            outs_p[i].zero_()
            _lib.check(L.q1_launch_groupkey(1 if g <= 8 else 3, ctypes.byref(arr[i].cols), ctypes.c_void_p(arr[i].keys),
                                            g, rows, cutoff, None, ctypes.c_void_p(scratch[i].data_ptr()),
                                            ctypes.c_void_p(outs_p[i].data_ptr()), sh))
            if sync_each:
                _lib.check(L.q1_sync_check(sh))

    def timed(fn, steps):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(steps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / steps

    with tempfile.TemporaryDirectory() as td:
        cache = os.path.join(td, "tune.txt").encode()
        b = ctypes.c_void_p()
        t0 = time.perf_counter()
        _lib.check(L.q1_batch_create(arr, len(descs), ctypes.byref(_lib.BatchOpts(1, 0, 0, args.tune, cache)), sh,
                                     ctypes.byref(b)))
        tune_s = time.perf_counter() - t0
        try:
            desc = _lib.BatchDesc()
            _lib.check(L.q1_batch_describe(b, ctypes.byref(desc)))
            run = lambda: _lib.check(L.q1_batch_run(b, sh))   # noqa: E731
            for _ in range(max(args.warmup, 3)):
                run()
                plain_pass(False)
            _lib.check(L.q1_sync_check(sh))
            sampler = ClockSampler(0)
            sampler.start()
            ms_batch = timed(run, args.steps)
            ms_plain = timed(lambda: plain_pass(False), args.steps)
            clocks = sampler.stop()
            # client-style plain: each instance's result checked (synchronised) before the next
            t1 = time.perf_counter()
            plain_pass(True)
            ms_plain_sync = 1000 * (time.perf_counter() - t1)
            _lib.check(L.q1_sync_check(sh))
            same = all(torch.equal(x, y) for x, y in zip(outs_b, outs_p))
        finally:
            L.q1_batch_destroy(b)
    peak, peak_kind = measured_peaks()
    gbs = BATCH_BYTES_PER_ROW * total_rows / (ms_batch / 1e3) / 1e9
    line = {"metric": METRIC, "mode": "batch", "value": total_rows / (ms_batch / 1e3), "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_batch, "higher_is_better": True,
            "dtype": "int64", "data": "synthetic",
            "config": {"workload": f"q1_batch_{len(spec)}_instances", "instances": len(spec), "total_rows": total_rows,
                       "rows": "log-uniform [1e4, 5e7]", "cutoff": "uniform [729906, 730089]",
                       "groups": "{" + args.batch_groups.replace(",", ", ") + "} uniform keys", "seed": SEED + 3,
                       "l2": f"inputs {BATCH_BYTES_PER_ROW * total_rows / 1e9:.1f} GB per pass > 126 MB L2"},
            "batched": {"ms": ms_batch, "rows_per_s": total_rows / (ms_batch / 1e3), "gbs": gbs,
                        "frac_hbm": gbs / peak, "peak_kind": peak_kind, "items": desc.items, "grid": desc.grid,
                        "chunk_tiles": desc.chunk_tiles, "modes": list(desc.mode_count), "uses_graph": desc.uses_graph,
                        "tune_s": tune_s},
            "plain_launches": {"ms": ms_plain, "rows_per_s": total_rows / (ms_plain / 1e3),
                               "note": "one q1_launch_groupkey per instance, queued back to back on one stream"},
            "plain_synchronised": {"ms": ms_plain_sync, "rows_per_s": total_rows / (ms_plain_sync / 1e3),
                                   "note": "one launch per instance, each result checked before the next launch"},
            "speedup_vs_plain": ms_plain / ms_batch, "speedup_vs_plain_synchronised": ms_plain_sync / ms_batch,
            "identical": bool(same), "clocks": clocks, "gpu_launches": args.steps}
    del keep, outs_b, outs_p, scratch
    torch.cuda.empty_cache()
    return line


# ------------------------------------------------------------------------------------------
# --mode serve: a Poisson request stream against the resident 600M-row table and a pool of
# ad-hoc tables (rows log-uniform in [1e6, 1e8]), half of each kind, grouping (returnflag,
# linestatus) or 64 keys, cutoff uniform in [1998-06-01, 1998-12-01]. The same arrival trace
# runs through the batched server and through the plain one-launch-per-request server; both
# report p50/p99 and rows/s, and a sample of responses is checked against the plain arbiter path.
# ------------------------------------------------------------------------------------------

def serve_trace(rate, duration, pool, seed):
    import numpy as np
    rng = np.random.default_rng(seed)
    n = int(rate * duration)
    gaps = rng.exponential(1.0 / rate, n)
    arrivals = np.cumsum(gaps)
    pool_rows = np.exp(rng.uniform(np.log(1e6), np.log(1e8), pool)).astype(np.int64)
    pool_grouping = rng.integers(0, 2, pool)
    reqs = []
    for i in range(n):
        cutoff = int(rng.integers(729906, 730090))
        if rng.random() < 0.5:
            grouping = int(rng.integers(0, 2))
            reqs.append((0, grouping, 64 if grouping else 0, cutoff, 0, 0))
        else:
            t = int(rng.integers(0, pool))
            grouping = int(pool_grouping[t])
            reqs.append((1, grouping, 64 if grouping else 0, cutoff, int(pool_rows[t]), 50_000 + t))
    return arrivals, reqs


def percentile(values, pct):
    if not values:
        return None
    v = sorted(values)
    return v[min(len(v) - 1, int(round(pct / 100.0 * (len(v) - 1))))]


def closed_loop(L, _lib, h, reqs):
    """Capacity: every request submitted at once, then all waited for."""
    import ctypes
    if not reqs:
        return {"requests": 0}
    _lib.check(L.q1_server_reset_stats(h))
    t0 = time.perf_counter()
    tks = []
    for r in reqs:
        t = ctypes.c_uint64()
        _lib.check(L.q1_server_submit(h, ctypes.byref(_lib.Request(*r)), ctypes.byref(t)))
        tks.append(t.value)
    for t in tks:
        _lib.check(L.q1_server_wait(h, t, 600_000, ctypes.byref(_lib.Response())))
    cap_s = time.perf_counter() - t0
    cst = _lib.ServerStats()
    _lib.check(L.q1_server_stats_get(h, ctypes.byref(cst)))
    return {"requests": len(reqs), "wall_s": cap_s, "requests_per_s": len(reqs) / cap_s,
            "logical_rows_per_s": cst.logical_rows / cap_s, "scanned_rows_per_s": cst.scanned_rows / cap_s,
            "rounds": cst.rounds, "mean_round_size": cst.mean_round_size, "p50_ms": cst.p50_ms, "p99_ms": cst.p99_ms,
            "overlapped_rounds": cst.overlapped_rounds}


def run_trace(q, _lib, h, arrivals, reqs, limit_s):
    """Submits at the trace's times (open loop) from this thread, waits from another."""
    import ctypes
    import queue as _queue
    L = q.lib()
    tickets = _queue.Queue()
    results = {}

    def waiter():
        while True:
            item = tickets.get()
            if item is None:
                return
            i, t = item
            resp = _lib.Response()
            st = L.q1_server_wait(h, t, 600_000, ctypes.byref(resp))
            results[i] = (st, resp)

    th = threading.Thread(target=waiter, daemon=True)
    th.start()
    t0 = time.perf_counter()
    submitted = 0
    for i, (at, r) in enumerate(zip(arrivals, reqs)):
        now = time.perf_counter() - t0
        if at > limit_s:
            break
        if at > now:
            time.sleep(at - now)
        req = _lib.Request(*r)
        t = ctypes.c_uint64()
        _lib.check(L.q1_server_submit(h, ctypes.byref(req), ctypes.byref(t)))
        tickets.put((i, t.value))
        submitted += 1
    tickets.put(None)
    th.join()
    return submitted, results


def bench_serve(args):
    out = run_serve(args)
    print(json.dumps(out), flush=True)
    return 0 if out["identical"] else 1


def run_serve(args):
    """C4: the Poisson trace through the batched server and through the plain one-launch-per-request
    server (Q1_SERVE_PLAIN); returns the JSON object."""
    import ctypes
    import torch
    import tpchq01_gpu_b200 as q
    from tpchq01_gpu_b200 import _lib

    L = q.lib()
    torch.cuda.set_device(0)
    pool = 128
    arrivals, reqs = serve_trace(args.rate, args.duration, pool, SEED + 4)
    out = {"metric": METRIC, "mode": "serve", "unit": UNIT, "n_gpus": 1, "higher_is_better": True,
           "dtype": "int64", "data": "synthetic",
           "config": {"workload": "q1_serving", "resident_rows": ROWS, "rate_per_s": args.rate,
                      "duration_s": args.duration, "requests": len(reqs), "adhoc_pool_tables": pool,
                      "adhoc_rows": "log-uniform [1e6, 1e8]", "mix": "50% resident / 50% ad-hoc",
                      "grouping": "(returnflag, linestatus) or 64 uniform keys", "cutoff": "uniform [729906, 730089]",
                      "hbm_budget_gib": 120}}
    for mode_name, mode in [("served", _lib.SERVE_BATCHED), ("plain", _lib.SERVE_PLAIN)]:
        o = _lib.ServerOpts()
        L.q1_server_opts_default(ctypes.byref(o))
        o.resident_rows = ROWS
        o.mode = mode
        h = ctypes.c_void_p()
        t0 = time.perf_counter()
        _lib.check(L.q1_server_open(ctypes.byref(o), ctypes.byref(h)))
        open_s = time.perf_counter() - t0
        try:
            # warm the ad-hoc table cache: every pool table named once
            warm = {}
            for r in reqs:
                if r[0] == 1 and r[5] not in warm:
                    warm[r[5]] = r
            tk = []
            for r in warm.values():
                t = ctypes.c_uint64()
                _lib.check(L.q1_server_submit(h, ctypes.byref(_lib.Request(*r)), ctypes.byref(t)))
                tk.append(t.value)
            for t in tk:
                _lib.check(L.q1_server_wait(h, t, 600_000, ctypes.byref(_lib.Response())))
            _lib.check(L.q1_server_reset_stats(h))
            sampler = ClockSampler(0)
            sampler.start()
            submitted, results = run_trace(q, _lib, h, arrivals, reqs, args.duration)
            clocks = sampler.stop()
            st = _lib.ServerStats()
            _lib.check(L.q1_server_stats_get(h, ctypes.byref(st)))
            ok = sum(1 for s_, r in results.values() if s_ == 0)
            # arbiter check: a sample of responses against the plain one-request path, bit for bit
            sample = sorted(results)[:: max(1, len(results) // 64)]
            same = True
            for i in sample:
                resp_j = _lib.Response()
                _lib.check(L.q1_server_plain(h, ctypes.byref(_lib.Request(*reqs[i])), ctypes.byref(resp_j)))
                g = resp_j.num_groups
                a = bytes(results[i][1].aggregates)[: g * 96]
                b_ = bytes(resp_j.aggregates)[: g * 96]
                same = same and a == b_ and results[i][0] == 0
            wall = st.wall_ms / 1e3
            # latency and rows/s at the offered rate, per request kind
            per_kind = {}
            for kind, kname in [(0, "resident"), (1, "adhoc")]:
                lat = [results[i][1].latency_ms for i in results if reqs[i][0] == kind and results[i][0] == 0]
                rows_k = sum(ROWS if kind == 0 else reqs[i][4] for i in results
                             if reqs[i][0] == kind and results[i][0] == 0)
                per_kind[kname] = {"completed": len(lat), "p50_ms": percentile(lat, 50), "p99_ms": percentile(lat, 99),
                                   "logical_rows_per_s": rows_k / wall if wall else None}
            # capacity: the first requests of the trace submitted at once (closed loop), the mix and
            # each kind alone
            capacity = closed_loop(L, _lib, h, reqs[: min(len(reqs), 5000)])
            capacity_kind = {kname: closed_loop(L, _lib, h, [r for r in reqs if r[0] == kind][:2000])
                             for kind, kname in [(0, "resident"), (1, "adhoc")]}
            out[mode_name] = {"capacity": capacity, "capacity_by_kind": capacity_kind, "by_kind": per_kind,
                              "overlapped_rounds": st.overlapped_rounds, "max_rounds_in_flight": st.max_rounds_in_flight,
                              "submitted": submitted, "completed": st.completed, "ok": ok, "failed": st.failed,
                              "rounds": st.rounds, "mean_round_size": st.mean_round_size,
                              "p50_ms": st.p50_ms, "p90_ms": st.p90_ms, "p99_ms": st.p99_ms, "max_ms": st.max_ms,
                              "mean_ms": st.mean_ms, "wall_s": wall,
                              "logical_rows_per_s": st.logical_rows / wall if wall else None,
                              "scanned_rows_per_s": st.scanned_rows / wall if wall else None,
                              "cache_hits": st.cache_hits, "cache_misses": st.cache_misses,
                              "evictions": st.evictions, "cached_gb": st.cached_bytes / 1e9,
                              "open_s": open_s, "arbiter_sample": len(sample), "arbiter_identical": bool(same),
                              "clocks": clocks}
        finally:
            L.q1_server_close(h)
    s_, p_ = out["served"], out["plain"]
    out["speedup_capacity_by_kind"] = {
        k: s_["capacity_by_kind"][k]["logical_rows_per_s"] / p_["capacity_by_kind"][k]["logical_rows_per_s"]
        for k in ["resident", "adhoc"] if p_["capacity_by_kind"][k]["logical_rows_per_s"]}
    out["value"] = s_["capacity"]["logical_rows_per_s"]
    out["speedup_capacity_rows_per_s"] = s_["capacity"]["logical_rows_per_s"] / p_["capacity"]["logical_rows_per_s"]
    out["speedup_at_offered_rate_rows_per_s"] = (s_["logical_rows_per_s"] or 0) / max(p_["logical_rows_per_s"] or 1e-9,
                                                                                     1e-9)
    out["identical"] = s_["arbiter_identical"] and p_["arbiter_identical"]
    return out


if __name__ == "__main__":
    sys.exit(main())
