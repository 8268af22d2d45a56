"""Benchmark of the off-target search hot path on B200.

Default workload: the full-genome scan -- a 3.1 Gbp synthetic genome (24
records of 50-250 Mbp, ~5% N), resident in HBM, x 100 guides of 20 nt + NRG,
<= 6 mismatches, both strands.  One step = one complete search through the C
ABI (cof_search): PAM prefilter + popcount scan, exact verification, row
formatting, rows copied to host memory.

  value : Gbp*guides/s over the device pipeline (scan + verify + format,
          CUDA events on the library's stream), genome resident.
  e2e   : same metric over the whole cof_search call (request tables
          host->device, row text device->host into a host buffer).
  roofline : the scan kernel against the measured peak of its own inner loop
          (window x pattern comparisons per second, microbenchmarked live).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
Multi-GPU (torchrun): each rank searches its own 100-guide set over its own
resident copy of the genome (weak scaling, no data-path collective).
"""
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
PKG = os.path.join(ROOT, "cas-offinder-rust-old_b200")
ORACLE = os.path.join(ROOT, "oracle")
sys.path.insert(0, PKG)

# dram__bytes_read.sum + dram__bytes_write.sum of one scan_kernel launch,
# from the ncu capture summarised in profiles/ (620 Mbp case, scaled x5 by
# genome size to the 3.1 Gbp workload: the scan reads each plane word once)
TRAFFIC = (350.28e6 + 16.16e6) * 5

METRIC = "Gbp*guides/s scanned (3.1 Gbp x 100 guides, 20 nt + NRG, mm<=6, both strands)"
UNIT = "Gbp*guides/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cof", choices=["cof", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="genome size factor (1.0 = 3.1 Gbp)")
    ap.add_argument("--guides", type=int, default=100)
    ap.add_argument("--cpu-sample-s", type=float, default=15.0,
                    help="target seconds of CPU work for the CPU baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            c = [x.strip() for x in l.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1]))
                mx = float(c[2])
            except ValueError:
                continue
            for n, v in zip(names, c[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "samples": len(sm), "reasons": sorted(reasons)}


def measure_peaks(device):
    lib = ctypes.CDLL(os.path.join(PKG, "libcof_peak.so"))
    out = (ctypes.c_double * 4)()
    rc = lib.cof_peak_measure(device, out)
    if rc != 0:
        raise RuntimeError(f"peak microbenchmark failed: {rc}")
    return dict(popc_per_s=out[0], lop3_per_s=out[1], pairs_per_s=out[2], clock_khz=out[3])


def hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def make_workload(args, rank):
    import synth
    cfg = synth.config_full_genome(seed=2, scale=args.scale, n_guides=args.guides)
    if rank:
        # weak scaling: every rank brings its own guide set
        import numpy as np
        rng = np.random.default_rng(1000 + rank)
        cfg["patterns"] = [synth.random_guide(rng, 20) + "NNN" for _ in range(args.guides)]
    return cfg


def cpu_baseline(cfg, target_s, n_threads=0):
    """The reference CPU path (C restatement, oracle/) over a leading slice of
    the same genome, all host threads, CPU batch size (64 chunks)."""
    sys.path.insert(0, ORACLE)
    import oracle
    oracle.build()
    cores = n_threads or os.cpu_count()
    chunks = list(cfg["genome"].chunks())

    def run(n_chunks):
        o = oracle.OracleGenome()
        nt = 0
        for name, data, s, e in chunks[:n_chunks]:
            o.add_chunk(name, data, s, e)
            nt += e - s
        t0 = time.perf_counter()
        o.search(cfg["filter"], cfg["patterns"], cfg["max_mismatches"], chunks_per_search=64,
                 n_threads=n_threads)
        return time.perf_counter() - t0, nt

    t, nt = run(min(len(chunks), 64))  # calibration: one 4 Mnt batch
    per_nt = t / max(nt, 1)
    want = int(target_s / max(per_nt, 1e-12))
    n_chunks = max(64, min(len(chunks), want // 65520 // 64 * 64))
    t, nt = run(n_chunks)
    rate = nt * 1e-9 * len(cfg["patterns"]) / t
    return dict(value=rate, unit=UNIT, cores=cores, kind="port",
                sample=f"first {nt / 1e6:.1f} Mbp of the genome x {len(cfg['patterns'])} "
                       f"guides, oracle/ C restatement of search_compute_cpu + writer, "
                       f"{cores} threads, {t:.1f} s"), t


def run_reference(args, rank, world):
    if rank != 0:
        return
    cfg = make_workload(args, 0)
    gbp_guides = None
    vals = []
    for i in range(args.warmup + args.steps):
        base, t = cpu_baseline(cfg, args.cpu_sample_s / 2)
        if i >= args.warmup:
            vals.append(base["value"])
    v = statistics.median(vals)
    base["value"] = v
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": cfg["name"], "genome_nt": cfg["genome"].n_nucl,
                       "guides": len(cfg["patterns"])},
            "cpu_baseline": base,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    import build as cof_build
    if rank == 0:
        cof_build.build()
    if dist:
        dist.barrier()
    import cof

    t0 = time.perf_counter()
    cfg = make_workload(args, rank)
    t_gen = time.perf_counter() - t0
    gen = cfg["genome"]
    n_nt = gen.n_nucl
    g = cof.Genome(device=local)
    t0 = time.perf_counter()
    gen.load_into(g)
    g.upload()
    torch.cuda.synchronize()
    t_upload = time.perf_counter() - t0

    peaks = measure_peaks(local)
    req = dict(search_filter=cfg["filter"], patterns=cfg["patterns"],
               max_mismatches=cfg["max_mismatches"])
    prepared = g.prepare([req])
    for _ in range(args.warmup):
        (text_bytes, n_rows), = g.run_prepared(prepared, as_text=None)
    rows_per_step = n_rows

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    stats = []
    wall = []
    for _ in range(args.steps):
        # one C-ABI call: request tables in, row text out in a host buffer
        t1 = time.perf_counter()
        g.run_prepared(prepared, as_text=None)
        wall.append(time.perf_counter() - t1)
        stats.append(g.last_stats())
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()

    dev_ms = sum(s["scan_ms"] + s["verify_ms"] + s["format_ms"] for s in stats)
    scan_ms = sum(s["scan_ms"] for s in stats) / len(stats)
    e2e_s = sum(wall)
    if dist:
        t = torch.tensor([dev_ms, e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_ms, e2e_s = t.tolist()
    gbp_guides = n_nt * 1e-9 * len(cfg["patterns"])
    value = world * gbp_guides * args.steps / (dev_ms * 1e-3)
    e2e = world * gbp_guides * args.steps / e2e_s
    pairs = stats[-1]["pairs"]
    achieved = pairs / (scan_ms * 1e-3)
    hbm, hbm_kind = hbm_peak()
    plane_bytes = n_nt * 0.375 * 2  # both strand groups read the planes
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": cfg["name"], "genome_nt": n_nt, "guides": len(cfg["patterns"]),
                   "max_mismatches": cfg["max_mismatches"], "pam": "NRG",
                   "parallelism": f"guide-set replicas x{world}",
                   "l2": "inputs larger than L2 (1.16 GB planes + 1.55 GB bit4 per pass)"},
        "gpu_launches": stats[-1]["kernel_launches"] * args.steps,
        "e2e": {"value": e2e, "unit": UNIT, "ms_per_step": e2e_s * 1e3 / args.steps,
                "h2d_bytes_per_step": 100 * 23 * 2 + 4096,
                "d2h_bytes_per_step": text_bytes},
        "roofline": {"bound": "alu", "kernel": "scan_kernel",
                     "achieved": achieved, "peak": peaks["popc_per_s"], "unit": "pairs/s",
                     "frac": achieved / peaks["popc_per_s"], "traffic": TRAFFIC,
                     "peak_kind": "measured live: POPC results/s of this GPU (XU pipe); "
                                  "the scan needs one POPC per window x pattern pair",
                     "inner_loop_peak_pairs_per_s": peaks["pairs_per_s"],
                     "frac_of_inner_loop": achieved / peaks["pairs_per_s"],
                     "lop3_per_s": peaks["lop3_per_s"],
                     "hbm_gbs_achieved": plane_bytes / (scan_ms * 1e-3) / 1e9,
                     "hbm_peak_gbs": hbm, "hbm_peak_kind": hbm_kind},
        "stages_ms": {k: statistics.median(s[k] for s in stats)
                      for k in ("scan_ms", "verify_ms", "format_ms", "d2h_ms", "total_ms")},
        "rows_per_step": rows_per_step, "candidates_per_step": stats[-1]["candidates"],
        "pairs_per_step": pairs,
        "genome_upload_s": t_upload, "genome_generate_s": t_gen,
        "clocks": clk,
    }
    if not args.no_cpu_baseline and world == 1:
        base, _ = cpu_baseline(cfg, args.cpu_sample_s)
        line["cpu_baseline"] = base
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
