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
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

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
                                          "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE,
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


def reference_table(rows, seed):
    """The reference's lineitem filled from the generator (oracle/_ref; test/bench infrastructure)."""
    from oracle import py_oracle as O
    import tpchq01_gpu_b200 as q
    cols = q.generate_host(seed, 0, rows)
    return O.RefTable(cols, CUTOFF)


def run_reference_cpu(rows, seconds=None, steps=None, warmup=0, threads=None):
    """Times KernelX100 of the reference on `threads` host threads over `rows` rows."""
    threads = threads or os.cpu_count() or 1
    t = reference_table(rows, SEED)
    try:
        for _ in range(warmup):
            t.x100_parallel(threads)
        times = []
        t0 = time.perf_counter()
        while True:
            s = time.perf_counter()
            _, rc = t.x100_parallel(threads)
            times.append(time.perf_counter() - s)
            if steps is not None and len(times) >= steps:
                break
            if seconds is not None and time.perf_counter() - t0 >= seconds and len(times) >= 3:
                break
        used = t.threads()
    finally:
        t.close()
    return rows * len(times) / sum(times), used, times


def reference_arm(args, rank):
    if rank != 0:
        return 0
    model, ncpu = cpu_info()
    sample = 50_000_000
    value, used, times = run_reference_cpu(sample, steps=args.steps, warmup=args.warmup)
    desc = (f"reference KernelX100<kMagic,true,kNoAvx512> (cpu/kernel_x100.hpp) on {used} host threads, "
            f"{sample:,} rows of the same generator per step ({model})")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic", "config": config_dict(args.gpus, args.placement),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": used, "kind": "reference", "sample": desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    global ROWS
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--placement", default="in_registers_per_thread")
    ap.add_argument("--rows", type=int, default=ROWS)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    ROWS = args.rows

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

    # Table: this rank's shard of the generator, compressed, HBM-resident.
    ctx = q.Q1Context(device=local_rank)
    ctx.generate(SEED, ROWS, first_row=rank * ROWS, layout="compressed", packing="pair")
    comp, _, rows, _, _ = ctx.table_columns()
    aggs = torch.zeros(36 * 2, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    launches = [0]

    def step():
        aggs.zero_()
        q.launch_compressed(args.placement, comp, rows, CUTOFF, False, aggs.data_ptr(), sh)
        launches[0] += 1

    def exchange():
        if world > 1:
            parts = [torch.zeros_like(aggs) for _ in range(world)]
            dist.all_gather(parts, aggs)
            return parts
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
        q.launch_compressed(args.placement, comp, rows, CUTOFF, False, aggs.data_ptr(), sh)
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
    parts = [p.cpu().numpy().view("uint64") for p in exchange()]
    merged = sum(q.decode_aggregates(p) for p in parts)

    value = world * ROWS * args.steps / (total_ms / 1000.0)
    avg_kernel_s = sum(kern_ms) / len(kern_ms) / 1000.0
    achieved = BYTES_PER_ROW * ROWS / avg_kernel_s / 1e9
    peak, peak_kind = measured_peaks()
    traffic = profiled_traffic()

    result = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
              "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
              "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
              "config": config_dict(world, args.placement),
              "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                           "frac": achieved / peak, "traffic": traffic, "peak_kind": f"{peak_kind} (hbm_gbs)",
                           "kernel_ms": sum(kern_ms) / len(kern_ms)},
              "gpu_launches": launches[0], "clocks": clocks,
              "check": {"groups_count_sum": int(sum(int(merged[g, 0]) for g in range(6)))}}

    if rank == 0 and world == 1 and not args.no_e2e:
        result["e2e"] = e2e_pinned(q, args)
    if rank == 0 and world == 1 and not args.no_cpu:
        model, ncpu = cpu_info()
        sample = 50_000_000
        v, used, times = run_reference_cpu(sample, seconds=10.0, warmup=1)
        result["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": used, "kind": "reference",
                                  "sample": f"reference KernelX100<kMagic,true,kNoAvx512> on {used} threads, "
                                            f"{sample:,} rows of the same generator, {len(times)} passes ({model})"}
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)
    return 0


def e2e_pinned(q, args):
    """Same workload through the public API with host buffers: q1_run on a pinned-host table."""
    ctx = q.Q1Context()
    try:
        ctx.generate(SEED, ROWS, layout="compressed", packing="pair", residency="pinned")
        p = q.Q1Params(hash_table_placement=args.placement, apply_compression=True, num_gpu_streams=4,
                       num_tuples_per_kernel_launch=1 << 24, num_query_execution_runs=1, cutoff_day=CUTOFF)
        for _ in range(max(1, min(args.warmup, 2))):
            ctx.run(p)
        steps = max(3, min(args.steps, 10))
        t = []
        for _ in range(steps):
            s = time.perf_counter()
            ctx.run(p)
            t.append(time.perf_counter() - s)
        h2d = int(ROWS * 2 + ROWS * 3 + ROWS * 4 + 4 * ((ROWS + 15) // 16))
        return {"value": ROWS * steps / sum(t), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 576,
                "steps": steps, "ms_per_step": 1000 * sum(t) / steps,
                "path": "q1_run, PINNED_HOST residency, 4 streams x 16M-row chunks (H2D + scan per chunk)"}
    finally:
        ctx.close()


if __name__ == "__main__":
    sys.exit(main())
