"""Benchmark of the off-target search hot path on B200.

Default workload: the full-genome scan -- a 3.1 Gbp synthetic genome (24
records of 50-250 Mbp, ~5% N), resident in HBM, x 100 guides of 20 nt + NRG,
<= 6 mismatches, both strands.  One step = one complete search through the C
ABI (cof_search): PAM prefilter + popcount scan, exact verification, row
formatting, rows copied to host memory.

  value : Gbp*guides/s over the device pipeline (scan + verify + format,
          CUDA events on the library's stream), genome resident.  The
          library scans one request on a genome this large in 4 slices and
          sums their stage times.
  e2e   : same metric over the whole cof_search call (request tables
          host->device, row text device->host into a host buffer; each
          slice's text crosses while the next slice scans).
  roofline : the scan kernel against the measured POPC peak of this GPU (one
          POPC per window x pattern comparison, microbenchmarked live).

Extra measurements on one GPU (--no-extras skips them): two PAMs batched in
one pass, the serving loop (spec mix and small requests, batched vs one
request per pass, p50/p99 latency), the bulge path (--only-bulge), and the
command line tool as a whole process on .2bit and FASTA genome files
(--only-cli).  cpu_baseline times the oracle port of the reference CPU path
on a slice of the genome.

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

# dram__bytes_read.sum + dram__bytes_write.sum of one scan_warp_kernel
# launch, from the ncu capture summarised in profiles/ (620 Mbp case, scaled
# x5 by genome size to the 3.1 Gbp workload: each strand group reads every
# plane word once, so traffic grows in proportion to the genome)
TRAFFIC = (465.17e6 + 22.00e6) * 5

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
    ap.add_argument("--cpu-rounds", type=int, default=4,
                    help="CPU baseline and --impl reference: the genome slice is this many "
                         "4.19 Mnt batches per host thread (about 1 s each at 100 guides)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-few-guide", action="store_true",
                    help="skip the 1-guide scan measurement (few_guide)")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="--impl reference: skip timing the reference's own GPU kernel")
    ap.add_argument("--serving-requests", type=int, default=1000)
    ap.add_argument("--serving-c5", action="store_true",
                    help="only the serving stream at its stated sizes (10,000 requests at "
                         "500/s, 1,000 at 50/s and 200/s) over the resident genome")
    ap.add_argument("--serving-rate", type=float, default=200.0, help="arrivals per second")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched mixed-PAM, serving, bulge and whole-process CLI "
                         "measurements")
    ap.add_argument("--only-bulge", action="store_true",
                    help="run only the bulge-path measurement (10 Mbp x 20 guides, mm<=4, "
                         "DNA/RNA bulges<=2) and print it")
    ap.add_argument("--only-cli", action="store_true",
                    help="run only the whole-process CLI measurement and print it")
    ap.add_argument("--bulge-scale", type=float, default=0.02,
                    help="bulge genome factor (1.0 = 500 Mbp; ~720 k rows per Mbp)")
    ap.add_argument("--bulge-full-scale", type=float, default=1.0,
                    help="--only-bulge: genome factor of the streamed bulge measurement "
                         "(0 skips it)")
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


def rank_patterns(patterns, rank):
    """Weak scaling: rank 0 searches the workload's own guides; every other
    rank brings its own seeded guide set of the same size and shape
    (20 nt + NNN)."""
    if rank == 0:
        return list(patterns)
    import numpy as np
    import synth
    rng = np.random.default_rng(1000 + rank)
    return [synth.random_guide(rng, 20) + "NNN" for _ in range(len(patterns))]


def max_over_ranks(dist, values, device):
    """Per-rank measurements reduced to the slowest rank's (MAX all-reduce):
    the job is done when the last rank is."""
    if dist is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def make_workload(args, rank):
    import synth
    cfg = synth.config_full_genome(seed=2, scale=args.scale, n_guides=args.guides)
    cfg["patterns"] = rank_patterns(cfg["patterns"], rank)
    return cfg


def mixed_pam_requests(seed=3, n_each=50):
    """Batched workload: 50 x (25 nt + NNGRRT) and 50 x (TTTN + 25 nt), mm <= 6."""
    import numpy as np
    import synth
    rng = np.random.default_rng(seed)
    a = [synth.random_guide(rng, 25) + "NNNNNN" for _ in range(n_each)]
    b = ["NNNN" + synth.random_guide(rng, 25) for _ in range(n_each)]
    return [dict(search_filter="N" * 25 + "NNGRRT", patterns=a, max_mismatches=6),
            dict(search_filter="TTTN" + "N" * 25, patterns=b, max_mismatches=6)]


def bench_mixed_pam(g, n_nt, steps):
    """Both guide sets in one pass (cof_search_batch) vs one pass each."""
    reqs = mixed_pam_requests()
    both = g.prepare(reqs)
    single = [g.prepare([r]) for r in reqs]
    g.run_prepared(both, as_text=None)
    for p in single:
        g.run_prepared(p, as_text=None)
    bat, plain = [], []
    for _ in range(steps):
        g.run_prepared(both, as_text=None)
        st = g.last_stats()
        bat.append(st["total_ms"])
        t = 0.0
        for p in single:
            g.run_prepared(p, as_text=None)
            t += g.last_stats()["total_ms"]
        plain.append(t)
    work = n_nt * 1e-9 * 100
    b, p = statistics.median(bat), statistics.median(plain)
    return {"workload": "50 x (25 nt + NNGRRT) + 50 x (TTTN + 25 nt), mm<=6, same genome",
            "batched_value": work / (b * 1e-3), "plain_value": work / (p * 1e-3),
            "unit": UNIT, "batched_ms": b, "plain_ms": p, "speedup": p / b}


def bench_few_guide(g, cfg, steps, guides=1, max_mm=3):
    """The few-guide end of the scan on the resident genome: `guides` of the
    workload's guides (20 nt + NRG) at mm <= max_mm, the reference's
    1-guide NRG row (README.md:73).  Here the comparisons are few and the
    scan's bound is the plane reads: 0.375 B per nucleotide (H, L and S
    bits) of algorithmic traffic, so the line reports the scan's achieved
    GB/s against the measured HBM copy bandwidth.  value = Gbp*guides /
    device time of the search; e2e = the same over the C-ABI call."""
    req = dict(search_filter=cfg["filter"], patterns=cfg["patterns"][:guides],
               max_mismatches=max_mm)
    prep = g.prepare([req])
    for _ in range(3):
        g.run_prepared(prep, as_text=None)
    stats, wall = [], []
    for _ in range(steps):
        t0 = time.perf_counter()
        (nbytes, rows), = g.run_prepared(prep, as_text=None)
        wall.append(time.perf_counter() - t0)
        stats.append(g.last_stats())
    n_nt = cfg["genome"].n_nucl
    scan = statistics.median(s["scan_ms"] for s in stats)
    dev = statistics.median(s["scan_ms"] + s["verify_ms"] + s["format_ms"] for s in stats)
    w = statistics.median(wall)
    hbm, kind = hbm_peak()
    plane_bytes = n_nt * 0.375
    achieved = plane_bytes / (scan * 1e-3) / 1e9
    units = n_nt * 1e-9 * guides
    return {"workload": f"{n_nt / 1e9:.1f} Gbp x {guides} guide (20 nt + NRG), mm<={max_mm}",
            "value": units / (dev * 1e-3), "unit": UNIT, "device_ms": dev,
            "e2e": {"value": units / w, "unit": UNIT, "ms_per_step": w * 1e3,
                    "d2h_bytes_per_step": nbytes},
            "scan_ms": scan, "scan_tile_shape": g.tuning()["last"],
            "kernel": scan_kernel_name(g.tuning()["last"]),
            "hbm_gbs_achieved": achieved, "hbm_peak_gbs": hbm, "hbm_peak_kind": kind,
            "hbm_frac": achieved / hbm,
            "algorithmic_bytes": plane_bytes,
            "note": "algorithmic bytes = 0.375 B/nt of H/L/S planes, read once for both "
                    "strands; hbm_frac = achieved / the measured copy bandwidth",
            "rows_per_step": rows, "steps": steps}


def serving_requests(n, seed=5, max_guides=500, max_mm=4):
    """Request mix of the serving stream: guides log-uniform in 1..max_guides,
    guide length U{17..25}, PAM in {NRG, NNGRRT, TTTN, NNNRRT}, mm U{0..4},
    no bulges.  Over a 3.1 Gbp genome one bulge request with 20-nt guides
    yields 1e8-1e9 rows and mm 5-6 with 17-nt guides 1e8+, so those are
    measured apart (bench_serving_bulge, on a 10 Mbp genome)."""
    import numpy as np
    import synth
    rng = np.random.default_rng(seed)
    pams = [("NRG", False), ("NNGRRT", False), ("TTTN", True), ("NNNRRT", False)]
    out = []
    for _ in range(n):
        ng = int(round(np.exp(rng.uniform(0, np.log(max_guides)))))
        gl = int(rng.integers(17, 26))
        pam, five = pams[int(rng.integers(0, 4))]
        mm = int(rng.integers(0, max_mm + 1))
        guides = [synth.random_guide(rng, gl) for _ in range(ng)]
        if five:
            filt = pam + "N" * gl
            pats = ["N" * len(pam) + x for x in guides]
        else:
            filt = "N" * gl + pam
            pats = [x + "N" * len(pam) for x in guides]
        out.append(dict(search_filter=filt, patterns=pats, max_mismatches=mm))
    return out


SERVING_MODES = (
    # (name, max_requests_per_pass, ring_slices)
    ("plain", 1, 1),            # one request per whole-genome pass
    ("batched_passes", 0, 1),   # arrivals wait for the running pass, then share the next
    ("batched", 0, 0),          # the ring: arrivals join at the next slice boundary
)


def bench_serving(cof, g, n_nt, n_req, rate, seed=7, max_guides=500, max_mm=4, reqs=None,
                  modes=SERVING_MODES):
    """A Poisson stream of requests through the server (cof_server_*), once
    per mode: the plain loop (one request per whole-genome pass), batching
    by whole passes, and the ring (continuous batching: the genome walked in
    slices, arrivals admitted at every slice boundary).  value = the
    stream's Gbp*guides / makespan; latency from submit to completion."""
    import numpy as np
    given = reqs is not None
    if not given:
        reqs = serving_requests(n_req, max_guides=max_guides, max_mm=max_mm)
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n_req))
    work = sum(n_nt * 1e-9 * len(r["patterns"]) for r in reqs)
    res = {}
    # every mode runs the default scan tile shape: first-time autotuning of
    # a new request shape would otherwise be charged to whichever mode meets it
    prev = os.environ.get("COF_AUTOTUNE")
    os.environ["COF_AUTOTUNE"] = "0"
    rows = {}
    for mode, per_pass, ring in modes:
        srv = cof.Server(g, max_requests_per_pass=per_pass, ring_slices=ring)
        t0 = time.perf_counter()
        tickets = []
        for a, r in zip(arrivals, reqs):
            dt = t0 + a - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            tickets.append(srv.submit(**r))
        out = [srv.wait(t, as_text=None) for t in tickets]
        span = time.perf_counter() - t0
        st = srv.stats()
        srv.close()
        rows[mode] = [o[1] for o in out]
        lats = sorted(o[2] for o in out)
        res[mode] = {"value": work / span, "unit": UNIT, "makespan_s": span,
                     "p50_ms": lats[len(lats) // 2],
                     "p99_ms": lats[min(len(lats) - 1, int(0.99 * len(lats)))],
                     "steps": st["passes"], "most_active": st["largest_pass"]}
    if prev is None:
        os.environ.pop("COF_AUTOTUNE", None)
    else:
        os.environ["COF_AUTOTUNE"] = prev
    names = [m[0] for m in modes]
    if len({tuple(v) for v in rows.values()}) != 1:
        raise RuntimeError("serving modes returned different row counts")
    if "plain" in names:
        for m in names:
            if m != "plain":
                res[f"speedup_{m}"] = res[m]["value"] / res["plain"]["value"]
        if "batched" in names:
            res["speedup"] = res["batched"]["value"] / res["plain"]["value"]
    res["requests"] = n_req
    res["rate_per_s"] = rate
    if not given:
        res["workload"] = (f"{n_req} requests, Poisson arrivals at {rate:g}/s, guides log-uniform "
                           f"1..{max_guides} (17-25 nt), PAM NRG/NNGRRT/TTTN/NNNRRT, "
                           f"mm 0..{max_mm}, no bulges")
    return res


def bench_serving_c5(cof, g, n_nt):
    """The serving stream at its stated sizes: 10,000 requests at 500/s,
    and 1,000 each at 50/s and 200/s, of the serving mix (guides 1..500
    log-uniform, 17-25 nt, four PAMs, mm 0..4, no bulges)."""
    out = {}
    for n_req, rate, seed in ((1000, 50.0, 11), (1000, 200.0, 12), (10000, 500.0, 13)):
        reqs = serving_requests(n_req, seed=seed)
        r = bench_serving(cof, g, n_nt, n_req, rate, seed=seed + 100, reqs=reqs)
        r["workload"] = (f"{n_req} requests, Poisson arrivals at {rate:g}/s, guides log-uniform "
                         f"1..500 (17-25 nt), PAM NRG/NNGRRT/TTTN/NNNRRT, mm 0..4, no bulges")
        out[f"{n_req}_at_{rate:g}"] = r
        print(json.dumps({f"serving_c5_{n_req}_at_{rate:g}": r}), flush=True)
    return out


def bench_serving_bulge(cof, device, n_req=96, rate=4000.0, seed=9, scale=0.02):
    """The serving loop with bulge requests: the 10 Mbp bulge-workload genome,
    requests of 1-20 guides (17-25 nt, the four PAMs), mm U{0..4}; half of
    them with DNA and RNA bulges U{1..2} (the Myers path, mm <= 3), the rest
    popcount.  Batched passes against one request per pass, as in
    bench_serving.  The stream runs once, untimed, through the new genome
    first: the first use of each kernel (loaded on first launch) and the
    growth of the genome's work buffers would otherwise be charged to
    whichever mode runs first, about 80 ms on this stream."""
    import numpy as np
    import synth
    cfg = synth.config_bulge(seed=4, scale=scale)
    g = cof.Genome(device=device)
    cfg["genome"].load_into(g)
    g.upload()
    rng = np.random.default_rng(seed)
    reqs = []
    for r in serving_requests(n_req, seed=seed, max_guides=20, max_mm=4):
        if rng.random() < 0.5:
            r = dict(r, max_mismatches=min(r["max_mismatches"], 3),
                     max_dna_bulges=int(rng.integers(1, 3)), max_rna_bulges=int(rng.integers(1, 3)))
        reqs.append(r)
    for r in reqs:
        g.run_prepared(g.prepare([r]), as_text=None)
    res = bench_serving(cof, g, cfg["genome"].n_nucl, n_req, rate, seed=seed, reqs=reqs)
    g.close()
    res["workload"] = (f"{n_req} requests over {cfg['genome'].n_nucl / 1e6:.0f} Mbp, Poisson "
                       f"arrivals at {rate:g}/s, guides log-uniform 1..20 (17-25 nt), four PAMs, "
                       f"mm 0..4; half with DNA/RNA bulges 1..2 (mm <= 3)")
    return res


def bench_bulge(cof, device, steps, scale):
    """The bulge (Myers + DP traceback) path: a 500 Mbp-generator genome
    scaled to `scale`, 20 guides of 20 nt + NRG, mm<=4, DNA and RNA bulges
    <= 2.  value = Gbp*guides / device time (Myers filter + budget pre-test +
    traceback + format); e2e = the same over the C-ABI call with the rows
    copied into a host buffer."""
    import synth
    cfg = synth.config_bulge(seed=4, scale=scale)
    g = cof.Genome(device=device)
    cfg["genome"].load_into(g)
    g.upload()
    prep = g.prepare([dict(search_filter=cfg["filter"], patterns=cfg["patterns"],
                           max_mismatches=cfg["max_mismatches"],
                           max_dna_bulges=cfg["max_dna_bulges"],
                           max_rna_bulges=cfg["max_rna_bulges"])])
    g.run_prepared(prep, as_text=None)  # warm-up: buffers, pinned memory
    dev, wall, stats = [], [], []
    for _ in range(steps):
        t0 = time.perf_counter()
        (nbytes, rows), = g.run_prepared(prep, as_text=None)
        wall.append(time.perf_counter() - t0)
        st = g.last_stats()
        stats.append(st)
        dev.append(st["scan_ms"] + st["verify_ms"] + st["format_ms"])
    g.close()
    units = cfg["genome"].n_nucl * 1e-9 * len(cfg["patterns"])
    d, w = statistics.median(dev), statistics.median(wall)
    return {"workload": f"{cfg['genome'].n_nucl / 1e6:.0f} Mbp x 20 guides (20 nt + NRG), "
                        f"mm<=4, DNA/RNA bulges<=2",
            "value": units / (d * 1e-3), "unit": UNIT, "device_ms": d,
            "e2e": {"value": units / w, "unit": UNIT, "ms_per_step": w * 1e3,
                    "d2h_bytes_per_step": nbytes},
            "stages_ms": {k: statistics.median(s[k] for s in stats)
                          for k in ("scan_ms", "verify_ms", "format_ms", "d2h_ms", "total_ms")},
            "rows_per_step": rows, "candidates_per_step": stats[-1]["candidates"],
            "gpu_launches_per_step": stats[-1]["kernel_launches"], "steps": steps,
            "stage_rates": bulge_rates(cfg, stats, rows)}


def bench_bulge_full(cof, device, steps, scale=1.0, cpu_nt=2_000_000):
    """The bulge workload at its stated size: 500 Mbp in 5 records x 20
    guides of 20 nt + NRG, mm<=4, DNA and RNA bulges <= 2 (about 3.6e8
    alignment rows, ~27 GB of row text per search).  The rows are streamed
    through cof_search_stream to a sink that counts them (the dest channel
    of search.rs:1490-1500): each candidate chunk's text crosses to a
    page-locked staging buffer while the next chunk's traceback runs, so
    host memory holds a few chunks, not the result.  value = Gbp*guides /
    device time (Myers filter + budget pre-test + traceback + format); e2e =
    the same over the whole streamed call, every row delivered to the sink.
    cpu_baseline: the oracle's restatement of the reference's Myers CPU
    path (search.rs:951-1031, traceback.rs:181-381) on the genome's first
    cpu_nt nucleotides, all host threads."""
    import synth
    t0 = time.perf_counter()
    cfg = synth.config_bulge(seed=4, scale=scale)
    t_gen = time.perf_counter() - t0
    g = cof.Genome(device=device)
    cfg["genome"].load_into(g)
    g.upload()
    req = dict(search_filter=cfg["filter"], patterns=cfg["patterns"],
               max_mismatches=cfg["max_mismatches"], max_dna_bulges=cfg["max_dna_bulges"],
               max_rna_bulges=cfg["max_rna_bulges"])
    prep = g.prepare([req])
    g.stream_count(prep)  # warm-up: buffers, page-locked staging
    dev, wall, stats, res = [], [], [], []
    for _ in range(steps):
        t1 = time.perf_counter()
        res.append(g.stream_count(prep))
        wall.append(time.perf_counter() - t1)
        st = g.last_stats()
        stats.append(st)
        dev.append(st["scan_ms"] + st["verify_ms"] + st["format_ms"])
    g.close()
    rows, nbytes, pieces = res[-1]
    assert all(r == res[0] for r in res), "streamed row counts differ between steps"
    n_nt = cfg["genome"].n_nucl
    units = n_nt * 1e-9 * len(cfg["patterns"])
    d, w = statistics.median(dev), statistics.median(wall)
    out = {"workload": f"{n_nt / 1e6:.0f} Mbp x 20 guides (20 nt + NRG), mm<=4, "
                       f"DNA/RNA bulges<=2, rows streamed to a counting sink",
           "value": units / (d * 1e-3), "unit": UNIT, "device_ms": d,
           "e2e": {"value": units / w, "unit": UNIT, "ms_per_step": w * 1e3,
                   "h2d_bytes_per_step": 20 * 23 * 2 + 4096, "d2h_bytes_per_step": nbytes},
           "rows_per_step": rows, "rows_per_s_e2e": rows / w, "text_gb_per_step": nbytes / 1e9,
           "pieces_per_step": pieces,
           "stages_ms": {k: statistics.median(s[k] for s in stats)
                         for k in ("scan_ms", "verify_ms", "format_ms", "d2h_ms", "total_ms")},
           "candidates_per_step": stats[-1]["candidates"],
           "gpu_launches_per_step": stats[-1]["kernel_launches"], "steps": steps,
           "genome_generate_s": t_gen, "stage_rates": bulge_rates(cfg, stats, rows)}
    # the reference's Myers CPU path (oracle port) on a leading slice
    sys.path.insert(0, ORACLE)
    import oracle
    oracle.build()
    o = oracle.OracleGenome()
    nt = 0
    for name, data, s0, e0 in cfg["genome"].chunks():
        if nt >= cpu_nt:
            break
        o.add_chunk(name, data, s0, e0)
        nt += e0 - s0
    t1 = time.perf_counter()
    _text, crow = o.search(cfg["filter"], cfg["patterns"], cfg["max_mismatches"],
                           cfg["max_dna_bulges"], cfg["max_rna_bulges"])
    tc = time.perf_counter() - t1
    o.close()
    out["cpu_baseline"] = {
        "value": nt * 1e-9 * len(cfg["patterns"]) / tc, "unit": UNIT, "cores": os.cpu_count(),
        "kind": "port",
        "sample": f"first {nt / 1e6:.1f} Mbp x 20 guides, oracle/ C restatement of the Myers "
                  f"CPU path (check_pam_quick, Myers sweep, traceback_all, classify, writer), "
                  f"{os.cpu_count()} threads, {tc:.1f} s, {crow} rows"}
    return out


def scan_kernel_name(shape):
    """The scan kernel a tile shape name (cof_genome_tuning "last") runs."""
    if shape.startswith("pair-"):
        return "scan_direct_kernel"
    return "scan_warp_kernel" if shape.startswith("warp-") else "scan_kernel"


def bulge_rates(cfg, stats, rows):
    """Per-stage work rates of the bulge path (its kernels are integer DP, so
    rates of their own units stand in for a roofline): Myers steps (one text
    position x one pattern, both strands), budget-DP cells of the Myers
    candidates (L x (L + max_db + 1) per candidate, an upper bound: the test
    stops early), and rows enumerated by the traceback."""
    L = len(cfg["patterns"][0])
    n_pat = 2 * len(cfg["patterns"])
    scan = statistics.median(s["scan_ms"] for s in stats) * 1e-3
    verify = statistics.median(s["verify_ms"] for s in stats) * 1e-3
    fmt = statistics.median(s["format_ms"] for s in stats) * 1e-3
    cand = stats[-1]["candidates"]
    return {"myers_steps_per_s": cfg["genome"].n_nucl * n_pat / scan,
            "budget_dp_cells_per_s": cand * L * (L + cfg["max_dna_bulges"] + 1) / verify,
            "candidates_per_s": cand / verify, "rows_per_s_traceback": rows / verify,
            "rows_per_s_format": rows / fmt,
            "note": "budget pre-test and traceback share one timed stage (verify_ms)"}


class CpuSample:
    """The reference CPU path (C restatement, oracle/) over a leading slice of
    the workload's genome, with the CPU batch size (64 chunks of 65,520 nt,
    4.19 Mnt) and all host threads.  The oracle, like search_compute_cpu
    (search.rs:549-569), gives each worker thread whole batches, so the slice
    is `rounds` batches per thread: every thread has the same work, no thread
    idles for want of a batch, and the slice follows from the thread count
    alone.  Both the product's cpu_baseline and the reference arm
    (--impl reference) use this rule, so on one machine they time the same
    slice."""

    BATCH_CHUNKS = 64

    def __init__(self, cfg, rounds=4, n_threads=0):
        sys.path.insert(0, ORACLE)
        import oracle
        oracle.build()
        self.oracle = oracle
        self.cfg = cfg
        self.n_threads = n_threads
        self.cores = n_threads or os.cpu_count()
        self.rounds = rounds
        self.chunks = list(cfg["genome"].chunks())
        # batches after the first start with the previous batch's last chunk
        # (the head overlap of search.rs:1531-1572): B batches hold
        # 64 + 63 (B - 1) chunks
        n_batches = rounds * self.cores
        self.n_chunks = min(len(self.chunks),
                            self.BATCH_CHUNKS + (self.BATCH_CHUNKS - 1) * (n_batches - 1))
        self.genome = self._genome(self.n_chunks)
        self.nt = self.genome.n_nucl
        self.batches = self.genome.n_batches(self.BATCH_CHUNKS)

    def _genome(self, n_chunks):
        o = self.oracle.OracleGenome()
        for name, data, s, e in self.chunks[:n_chunks]:
            o.add_chunk(name, data, s, e)
        return o

    def _time(self, o):
        c = self.cfg
        t0 = time.perf_counter()
        o.search(c["filter"], c["patterns"], c["max_mismatches"],
                 chunks_per_search=self.BATCH_CHUNKS, n_threads=self.n_threads)
        return time.perf_counter() - t0, o.n_nucl

    def run(self):
        """One timed pass over the slice; returns (Gbp*guides/s, seconds)."""
        t, nt = self._time(self.genome)
        return nt * 1e-9 * len(self.cfg["patterns"]) / t, t

    def describe(self, value, t):
        return dict(value=value, unit=UNIT, cores=self.cores, kind="port",
                    sample_nt=self.nt, sample_batches=self.batches,
                    sample=f"first {self.nt / 1e6:.1f} Mbp of the genome ({self.batches} "
                           f"batches of 64 chunks: {self.rounds} per thread) x "
                           f"{len(self.cfg['patterns'])} guides, oracle/ C restatement of "
                           f"search_compute_cpu + writer, {self.cores} threads, {t:.1f} s")


def bench_cli(cfg, n_rows, runs=2, fmt="2bit"):
    """The command line tool as a fresh process, the way main.rs is run:
    `cof-offinder input.txt G out.txt` reads the genome file (`fmt`: "2bit"
    or "fasta", 60-column lines), uploads it, searches, and writes the rows
    and the .log summary.  The genome file is written once beforehand (page
    cache warm for every run)."""
    import shutil
    import tempfile
    import build as cof_build
    d = tempfile.mkdtemp(prefix="cof_cli_")
    try:
        t0 = time.perf_counter()
        path = os.path.join(d, "genome." + ("2bit" if fmt == "2bit" else "fa"))
        if fmt == "2bit":
            cfg["genome"].write_2bit(path)
        else:
            cfg["genome"].write_fasta(path)
        os.sync()  # a genome file at rest: no writeback during the timed runs
        t_write = time.perf_counter() - t0
        # one plain read of the file first: the page cache then holds it where
        # host memory allows, and its rate shows what the runs read from
        t0 = time.perf_counter()
        buf = bytearray(64 << 20)
        with open(path, "rb", buffering=0) as f:
            while f.readinto(buf):
                pass
        t_read = time.perf_counter() - t0
        inp = os.path.join(d, "input.txt")
        with open(inp, "w") as f:
            f.write(path + "\n" + cfg["filter"] + "\n")
            for p in cfg["patterns"]:
                f.write(f"{p} {cfg['max_mismatches']}\n")
        out = os.path.join(d, "out.txt")
        secs, stages = [], []
        env = dict(os.environ, COF_CLI_TIMES="1")
        for _ in range(runs):
            t1 = time.perf_counter()
            r = subprocess.run([cof_build.CLI, inp, "G", out], capture_output=True, text=True,
                               timeout=600, env=env)
            secs.append(time.perf_counter() - t1)
            if r.returncode:
                raise RuntimeError("cof-offinder failed: " + r.stderr.strip())
            for ln in r.stderr.splitlines():
                if ln.startswith("stage seconds:"):
                    f = ln.split(":", 1)[1].split()
                    stages.append({f[i]: float(f[i + 1]) for i in range(0, len(f), 2)})
        rows = 0
        with open(out, "rb") as f:
            for line in f:
                rows += not line.startswith(b"#")
        return {"workload": "cof-offinder input.txt G out.txt, " + cfg["name"],
                "genome_file": fmt, "seconds": min(secs), "runs_s": secs, "rows": rows,
                "stage_s": stages[secs.index(min(secs))] if len(stages) == len(secs) else None,
                "rows_match_c_abi": None if n_rows is None else rows == n_rows,
                "genome_file_bytes": os.path.getsize(path),
                "output_bytes": os.path.getsize(out),
                "includes": "process start, CUDA context, genome file read + convert, upload, "
                            "search, output + .log written",
                "genome_file_write_s": t_write,
                "genome_file_read_s": t_read,
                "genome_file_read_gbs": os.path.getsize(path) / t_read / 1e9}
    finally:
        shutil.rmtree(d, ignore_errors=True)


def cpu_baseline(cfg, rounds, n_threads=0):
    smp = CpuSample(cfg, rounds, n_threads)
    v, t = smp.run()
    return smp.describe(v, t), t


def reference_gpu_kernel(cfg):
    """The reference's own find_matches kernel (oracle/_ref, built from the
    reference sources for sm_100a) launched as search.rs launches it, on this
    workload: device time of its launches and of its whole device loop."""
    sys.path.insert(0, ORACLE)
    try:
        import ref_gpu
    except ImportError as e:
        return {"unavailable": f"oracle/ref_gpu.py: {e}"}
    if not ref_gpu.available():
        return {"unavailable": "oracle/_ref not built (the reference tree was absent)"}
    import synth
    chunks = list(cfg["genome"].chunks())
    pats = cfg["patterns"] + [synth.revcomp(p) for p in cfg["patterns"]]
    ref = ref_gpu.RefGpu(chunks, 0)
    try:
        counts = ref.popcount_counts(pats, cfg["max_mismatches"])
        runs = [ref.popcount(pats, cfg["max_mismatches"], counts, keep=False)[1]
                for _ in range(3)]
    finally:
        ref.close()
    best = min(runs[1:], key=lambda t: t["kernel_ms"])
    units = cfg["genome"].n_nucl * 1e-9 * len(cfg["patterns"])
    return {"kernel": "find_matches (kernel.cu), 1 Gnt batches, grid (n/128, patterns)",
            "kernel_ms": best["kernel_ms"], "launches": best["launches"],
            "kernel_value": units / (best["kernel_ms"] * 1e-3),
            "device_loop_ms": best["wall_ms"],
            "device_loop_value": units / (best["wall_ms"] * 1e-3), "unit": UNIT,
            "kernel_records": sum(counts),
            "note": "device loop = pack + N mask + H2D + kernel + D2H per batch, "
                    "before the reference's CPU writer; best of 2 after 1 warm-up"}


def run_reference(args, rank, world):
    """The reference arm: the reference's CPU search path on the host cores
    (oracle/ C restatement; Rust cannot be built here), each step one pass
    over the slice CpuSample picks (--cpu-rounds batches per host thread, the
    same slice as the product's cpu_baseline).  Under torchrun only rank 0
    runs."""
    if rank != 0:
        return
    cfg = make_workload(args, 0)
    smp = CpuSample(cfg, args.cpu_rounds)
    vals, times = [], []
    for i in range(args.warmup + args.steps):
        v, t = smp.run()
        if i >= args.warmup:
            vals.append(v)
            times.append(t)
    v = statistics.median(vals)
    base = smp.describe(v, statistics.median(times))
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": statistics.median(times) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": cfg["name"], "genome_nt": cfg["genome"].n_nucl,
                       "guides": len(cfg["patterns"]),
                       "sample_nt": smp.nt, "chunks_per_search": 64},
            "cpu_baseline": base,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_ref_gpu:
        try:
            line["reference_gpu_kernel"] = reference_gpu_kernel(cfg)
        except Exception as e:  # the CPU line above stands on its own
            line["reference_gpu_kernel"] = {"unavailable": f"{type(e).__name__}: {e}"}
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
    if args.only_bulge:
        if rank == 0:
            res = {"bulge": bench_bulge(cof, local, max(1, args.steps), args.bulge_scale)}
            if args.bulge_full_scale > 0:
                res["bulge_full"] = bench_bulge_full(cof, local, max(1, args.steps),
                                                     args.bulge_full_scale)
            print(json.dumps(res), flush=True)
        if dist:
            dist.destroy_process_group()
        return

    t0 = time.perf_counter()
    cfg = make_workload(args, rank)
    t_gen = time.perf_counter() - t0
    if args.only_cli:
        if rank == 0:
            print(json.dumps({"cli_whole_process": bench_cli(cfg, None, max(1, args.steps)),
                              "cli_whole_process_fasta": bench_cli(cfg, None, max(1, args.steps),
                                                                   "fasta")}),
                  flush=True)
        if dist:
            dist.destroy_process_group()
        return
    gen = cfg["genome"]
    n_nt = gen.n_nucl
    g = cof.Genome(device=local)
    t0 = time.perf_counter()
    gen.load_into(g)
    g.upload()
    torch.cuda.synchronize()
    t_upload = time.perf_counter() - t0

    if args.serving_c5:
        if rank == 0:
            bench_serving_c5(cof, g, n_nt)
        g.close()
        if dist:
            dist.destroy_process_group()
        return

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
    dev_ms, e2e_s = max_over_ranks(dist, [dev_ms, e2e_s], "cuda")
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
        "roofline": {"bound": "alu",
                     "kernel": scan_kernel_name(g.tuning()["last"]),
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
        "scan_tile_shape": g.tuning()["last"],
        "genome_upload_s": t_upload, "genome_generate_s": t_gen,
        "clocks": clk,
    }
    if world == 1 and not args.no_few_guide:
        line["few_guide"] = bench_few_guide(g, cfg, max(5, args.steps))
    if not args.no_extras and world == 1:
        line["batched_mixed_pam"] = bench_mixed_pam(g, n_nt, max(3, args.steps // 2))
        line["serving"] = bench_serving(cof, g, n_nt, args.serving_requests, args.serving_rate)
        line["serving_small_requests"] = bench_serving(cof, g, n_nt, 256, 2000.0, seed=8,
                                                       max_guides=4, max_mm=3)
        line["bulge"] = bench_bulge(cof, local, 3, args.bulge_scale)
        line["bulge_full"] = bench_bulge_full(cof, local, 2)
        line["serving_bulge_mix"] = bench_serving_bulge(cof, local)
        g.close()  # the CLI runs as its own process: free this one's device genome first
        line["cli_whole_process"] = bench_cli(cfg, rows_per_step)
        line["cli_whole_process_fasta"] = bench_cli(cfg, rows_per_step, fmt="fasta")
    if not args.no_cpu_baseline and world == 1:
        base, _ = cpu_baseline(cfg, args.cpu_rounds)
        line["cpu_baseline"] = base
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
