"""Speed of the reference's own GPU path on this B200: kernel.cu and
kernel_myers.cu built unmodified for sm_100a (oracle/_ref/) and launched the
way search.rs launches them (ref_gpu.cu), on the benchmark workloads:

  popcount : 3.1 Gbp synthetic genome x 100 guides (20 nt + NRG), mm <= 6,
             1 Gnt batches (chunks_per_search 16384, the reference GPU batch)
  myers    : 500 Mbp x 20 guides (20 nt + NRG), mm <= 4, DNA/RNA bulges <= 2,
             scaled down (every hit enumerates many alignments)

MEASUREMENT INFRASTRUCTURE ONLY.  The product's own device time on the same
genome and request is taken in the same process for the side-by-side.

Usage: python oracle/ref_gpu_bar.py [--workload popcount|myers|both] [--scale S]
                                    [--myers-scale S] [--reps R] [--json OUT]
"""
import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "cas-offinder-rust-old_b200"))
sys.path.insert(0, HERE)

import ref_gpu  # noqa: E402
import synth  # noqa: E402


def product_ms(chunks, cfg, reps):
    import cof
    g = cof.Genome()
    for name, data, s, e in chunks:
        g.add_chunk(name, data, s, e)
    g.upload()
    prep = g.prepare([dict(search_filter=cfg["filter"], patterns=cfg["patterns"],
                           max_mismatches=cfg["max_mismatches"],
                           max_dna_bulges=cfg.get("max_dna_bulges", 0),
                           max_rna_bulges=cfg.get("max_rna_bulges", 0))])
    g.run_prepared(prep, as_text=None)  # warm-up (and tile autotuning)
    best = None
    for _ in range(reps):
        g.run_prepared(prep, as_text=None)
        st = g.last_stats()
        dev = st["scan_ms"] + st["verify_ms"] + st["format_ms"]
        if best is None or dev < best["device_ms"]:
            best = dict(device_ms=dev, total_ms=st["total_ms"], rows=st["rows"],
                        launches=st["kernel_launches"])
    g.close()
    return best


def _side_by_side(out, units, chunks, cfg, reps, best):
    out["reference"] = dict(best, kernel_gbp_guides_per_s=units / (best["kernel_ms"] / 1e3),
                            loop_gbp_guides_per_s=units / (best["wall_ms"] / 1e3))
    p = product_ms(chunks, cfg, reps)
    p["device_gbp_guides_per_s"] = units / (p["device_ms"] / 1e3)
    p["total_gbp_guides_per_s"] = units / (p["total_ms"] / 1e3)
    out["product"] = p
    out["kernel_speedup"] = best["kernel_ms"] / p["device_ms"]
    return out


def bar_popcount(scale, reps):
    cfg = synth.config_full_genome(seed=2, scale=scale, n_guides=100)
    chunks = list(cfg["genome"].chunks())
    n_nt = cfg["genome"].n_nucl
    pats = cfg["patterns"] + [synth.revcomp(p) for p in cfg["patterns"]]
    mm = cfg["max_mismatches"]
    ref = ref_gpu.RefGpu(chunks, 0)
    t0 = time.perf_counter()
    counts = ref.popcount_counts(pats, mm)
    t_count = time.perf_counter() - t0
    runs = []
    for _ in range(reps + 1):  # the first run is a warm-up
        _per, t = ref.popcount(pats, mm, counts, keep=False)
        runs.append(t)
    ref.close()
    best = min(runs[1:], key=lambda t: t["kernel_ms"])
    out = dict(workload=cfg["name"], genome_nt=n_nt, guides=len(cfg["patterns"]),
               batches=best["n_batches"], kernel_matches=sum(counts),
               max_batch_matches=max(counts), count_pass_s=round(t_count, 2))
    return _side_by_side(out, n_nt * 1e-9 * len(cfg["patterns"]), chunks, cfg, reps, best)


def bar_myers(scale, reps):
    cfg = synth.config_bulge(seed=4, scale=scale)
    chunks = list(cfg["genome"].chunks())
    n_nt = cfg["genome"].n_nucl
    pats = cfg["patterns"] + [synth.revcomp(p) for p in cfg["patterns"]]
    ref = ref_gpu.RefGpu(chunks, 0)
    runs = []
    for _ in range(reps + 1):
        _per, t = ref.myers(cfg["filter"], pats, len(cfg["patterns"]), cfg["max_mismatches"],
                            cfg["max_dna_bulges"], cfg["max_rna_bulges"], keep=False)
        runs.append(t)
    ref.close()
    best = min(runs[1:], key=lambda t: t["kernel_ms"])
    out = dict(workload=cfg["name"], genome_nt=n_nt, guides=len(cfg["patterns"]))
    return _side_by_side(out, n_nt * 1e-9 * len(cfg["patterns"]), chunks, cfg, reps, best)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="both", choices=["popcount", "myers", "both"])
    ap.add_argument("--scale", type=float, default=1.0, help="popcount genome factor (3.1 Gbp)")
    ap.add_argument("--myers-scale", type=float, default=0.02,
                    help="Myers genome factor (1.0 = 500 Mbp; ~720 k alignments per Mbp, "
                         "so the full size emits ~3.6e8 records)")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--json", default=None)
    a = ap.parse_args()
    res = {}
    if a.workload in ("popcount", "both"):
        res["popcount"] = bar_popcount(a.scale, a.reps)
        print(json.dumps(res["popcount"]), flush=True)
    if a.workload in ("myers", "both"):
        res["myers"] = bar_myers(a.myers_scale, a.reps)
        print(json.dumps(res["myers"]), flush=True)
    if a.json:
        with open(a.json, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
