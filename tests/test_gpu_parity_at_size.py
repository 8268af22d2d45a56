"""Parity at the benchmark's own sizes, row for row.

* The full-genome workload that bench.py times: 3.1 Gbp in 24 records with
  N runs, 100 guides of 20 nt + NRG, mm <= 6, both strands
  (synth.config_full_genome(seed=2)).  Every row equals the oracle's, the
  CPU restatement of search_compute_cpu + convert_matches + the writer
  (search.rs:378-569, main.rs:159-242), run on all host threads.
* The mixed-PAM workload (50 NNGRRT + 50 TTTN guides of 25 nt, mm <= 6,
  batched into one pass) on 310 Mbp of its generator, against one oracle run
  per request.
* The bulge workload of bench.py (10 Mbp x 20 guides of 20 nt + NRG, mm <= 4,
  DNA and RNA bulges <= 2): the raw Match stream equals the reference's own
  find_matches_myers (kernel_myers.cu, built unmodified for sm_100a) decoded
  the way search.rs:152-206 and :1316-1374 decode it, and the 8-column rows
  equal the oracle's Myers path (search.rs:951-1031, traceback.rs:181-381).

Rows are compared as sorted lists (the reference's row order is
unspecified), with their SHA-256 reported on failure."""
import hashlib
import os
import sys

import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def _sorted(text):
    rows = text.split("\n")
    if rows and rows[-1] == "":
        rows.pop()
    rows.sort()
    return rows


def _assert_same_rows(mine, ref, what):
    a, b = _sorted(mine), _sorted(ref)
    if a != b:
        ha = hashlib.sha256("\n".join(a).encode("latin-1")).hexdigest()
        hb = hashlib.sha256("\n".join(b).encode("latin-1")).hexdigest()
        sa, sb = set(a), set(b)
        extra, missing = sorted(sa - sb)[:5], sorted(sb - sa)[:5]
        pytest.fail(f"{what}: {len(a)} rows (sha256 {ha[:16]}) vs {len(b)} reference rows "
                    f"(sha256 {hb[:16]}); extra {extra}; missing {missing}")
    return len(a)


def _both(cof_mod, oracle_mod, gen):
    g = cof_mod.Genome()
    o = oracle_mod.OracleGenome()
    for name, data, s, e in gen.chunks():
        g.add_chunk(name, data, s, e)
        o.add_chunk(name, data, s, e)
    return g, o


def test_full_genome_workload_vs_oracle(cof_mod, oracle_mod):
    import synth
    cfg = synth.config_full_genome(seed=2, scale=1.0, n_guides=100)
    g, o = _both(cof_mod, oracle_mod, cfg["genome"])
    del cfg["genome"]
    args = (cfg["filter"], cfg["patterns"], cfg["max_mismatches"])
    text, n = g.search(*args)
    g.close()
    ref, nref = o.search(*args)
    o.close()
    assert n == nref > 1_000_000
    assert _assert_same_rows(text, ref, "3.1 Gbp x 100 guides") == n


def test_mixed_pam_workload_vs_oracle_at_310Mbp(cof_mod, oracle_mod):
    import synth
    cfg = synth.config_mixed_pam(seed=3, scale=0.1, n_each=50)
    g, o = _both(cof_mod, oracle_mod, cfg["genome"])
    res = g.search_batch(cfg["requests"])
    g.close()
    for req, (text, n) in zip(cfg["requests"], res):
        ref, nref = o.search(req["search_filter"], req["patterns"], req["max_mismatches"])
        assert n == nref > 0
        _assert_same_rows(text, ref, req["search_filter"])
    o.close()


def test_bulge_workload_vs_reference_kernel_and_oracle(cof_mod, oracle_mod):
    import synth
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "oracle"))
    import bruteforce
    import ref_gpu
    cfg = synth.config_bulge(seed=4, scale=0.02)
    chunks = list(cfg["genome"].chunks())
    g = cof_mod.Genome()
    for c in chunks:
        g.add_chunk(*c)
    filt, pats = cfg["filter"], cfg["patterns"]
    mm, db, rb = cfg["max_mismatches"], cfg["max_dna_bulges"], cfg["max_rna_bulges"]
    raw, n_raw = g.search(filt, pats, mm, db, rb, raw=True)
    rows, n_rows = g.search(filt, pats, mm, db, rb)
    g.close()
    assert n_rows > 5_000_000
    if ref_gpu.available():
        full = list(pats) + [bruteforce.revcomp(p) for p in pats]
        ref = ref_gpu.RefGpu(chunks, 0)
        rtext, n_ref, _t = ref.myers_text(filt, full, len(pats), mm, db, rb,
                                          out_cap=n_raw + (1 << 20))
        ref.close()
        assert n_raw == n_ref
        _assert_same_rows(raw, rtext, "bulge raw Match stream vs find_matches_myers")
    del raw
    o = oracle_mod.OracleGenome()
    for c in chunks:
        o.add_chunk(*c)
    orows, n_o = o.search(filt, pats, mm, db, rb)
    o.close()
    assert n_rows == n_o
    _assert_same_rows(rows, orows, "bulge rows vs the oracle")
