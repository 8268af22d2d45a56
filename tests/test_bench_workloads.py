"""The workloads bench.py times, checked on CPU (no GPU):

* the serving request mix has its stated distribution (guides log-uniform
  in 1..500, guide length 17-25, the four PAMs, mm 0-4, no bulges) and is
  the same for the same seed, so every serving mode meets the same stream;
* the CPU-baseline slice is `rounds` whole batches per host thread (64
  chunks for the first batch, 63 more for each further one: the head
  overlap of search.rs:1531-1572), so the product's cpu_baseline and the
  reference arm time the same slice on one machine;
* the synthetic configurations have the shapes they are named for."""
import os
import statistics
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "cas-offinder-rust-old_b200"))

import bench  # noqa: E402
import synth  # noqa: E402

# the PAM of a filter, from what is left once its leading N cells go
_PAM_OF_TAIL = {"RG": "NRG", "GRRT": "NNGRRT", "RRT": "NNNRRT"}


def _pam(search_filter):
    if search_filter.startswith("TTTN"):
        return "TTTN"
    return _PAM_OF_TAIL[search_filter.lstrip("N")]


def test_serving_request_mix():
    reqs = bench.serving_requests(3000, seed=21)
    assert reqs == bench.serving_requests(3000, seed=21)
    assert reqs != bench.serving_requests(3000, seed=22)
    counts = {"NRG": 0, "NNGRRT": 0, "TTTN": 0, "NNNRRT": 0}
    n_guides, mms = [], []
    for r in reqs:
        f, pats, mm = r["search_filter"], r["patterns"], r["max_mismatches"]
        assert set(r) == {"search_filter", "patterns", "max_mismatches"}  # no bulges
        pam = _pam(f)
        counts[pam] += 1
        guide_len = len(f) - len(pam)
        assert 17 <= guide_len <= 25
        assert 1 <= len(pats) <= 500
        for p in pats:
            assert len(p) == len(f)
            guide = p[len(pam):] if pam == "TTTN" else p[:guide_len]
            pad = p[:len(pam)] if pam == "TTTN" else p[guide_len:]
            assert set(guide) <= set("ACGT") and set(pad) == {"N"}
        n_guides.append(len(pats))
        mms.append(mm)
    # log-uniform in 1..500: median sqrt(500) = 22.4, and a request has one
    # guide with probability ln 1.5 / ln 500 = 0.065
    assert 15 <= statistics.median(n_guides) <= 33
    assert 0.04 <= n_guides.count(1) / len(reqs) <= 0.09
    assert max(n_guides) > 300
    for pam, c in counts.items():
        assert 0.21 <= c / len(reqs) <= 0.29, (pam, c)
    assert set(mms) == {0, 1, 2, 3, 4}


def test_serving_request_mix_limits():
    for r in bench.serving_requests(400, seed=9, max_guides=20, max_mm=2):
        assert 1 <= len(r["patterns"]) <= 20 and 0 <= r["max_mismatches"] <= 2


def test_cpu_sample_slice_is_whole_batches_per_thread():
    # 20 Mbp: enough chunks of 65,520 nt for 2 rounds x 2 threads
    cfg = synth.config_bulge(seed=4, scale=0.04, n_guides=2, planted=1)
    s = bench.CpuSample(cfg, rounds=2, n_threads=2)
    assert s.cores == 2
    assert s.n_chunks == 64 + 63 * 3
    assert s.batches == 4
    # a genome with fewer chunks is taken whole
    small = synth.config_bulge(seed=4, scale=0.002, n_guides=2, planted=1)
    s2 = bench.CpuSample(small, rounds=4, n_threads=4)
    assert s2.n_chunks == len(list(small["genome"].chunks()))
    assert s2.nt == small["genome"].n_nucl


def test_config_shapes():
    full = synth.config_full_genome(seed=2, scale=0.002, n_guides=100, planted=2)
    g = full["genome"]
    assert len(g.records) == 24
    n_frac = sum(int(np.count_nonzero(r == 15)) for r in g.records) / g.n_nucl
    assert 0.03 <= n_frac <= 0.06  # about 5% N in runs
    assert full["filter"] == "N" * 21 + "RG" and full["max_mismatches"] == 6
    assert len(full["patterns"]) == 100
    assert all(len(p) == 23 and p.endswith("NNN") for p in full["patterns"])

    bulge = synth.config_bulge(seed=4, scale=0.0002, n_guides=20, planted=2)
    assert len(bulge["genome"].records) == 5
    assert (bulge["max_mismatches"], bulge["max_dna_bulges"], bulge["max_rna_bulges"]) == (4, 2, 2)
    assert len(bulge["patterns"]) == 20

    mixed = synth.config_mixed_pam(seed=3, scale=0.0005, n_each=50, planted=2)
    a, b = mixed["requests"]
    assert a["search_filter"] == "N" * 25 + "NNGRRT" and len(a["patterns"]) == 50
    assert b["search_filter"] == "TTTN" + "N" * 25 and len(b["patterns"]) == 50
