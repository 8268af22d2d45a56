"""The reference's own CUDA kernels (kernel.cu, kernel_myers.cu), built
unmodified for sm_100a into oracle/_ref/ and launched as search.rs launches
them, against the product's raw Match stream (COF_F_RAW_MATCHES).  A second
pin of the scan and bulge paths that does not go through the C restatement.

The reference GPU popcount loop never scans the last < 32 window starts of a
batch (search.rs:280-284, a documented CPU/GPU divergence); the product
follows the CPU path, so those windows are the only allowed difference."""
import collections
import os
import random
import sys

import pytest

import bruteforce
import randgen

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                "oracle"))
import ref_gpu  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_gpu.available(),
                                 reason="oracle/_ref not built (needs the reference tree)")]

KAT_PATS = ["CCGTGGTTCAACATTTGCTTAGCA", "GATGTTGGTAAGTGGGATATGGCA"]


def _engine(cof_mod, chunks):
    g = cof_mod.Genome()
    for name, data, s, e in chunks:
        g.add_chunk(name, data, s, e)
    return g


def _lines(text):
    return text.split("\n")[:-1]


def _check_popcount(cof_mod, chunks, filt, user_pats, mm, cps):
    pats = list(user_pats) + [bruteforce.revcomp(p) for p in user_pats]
    ref = ref_gpu.RefGpu(chunks, cps)
    per, _t = ref.popcount(pats, mm)
    ref_lines = ref_gpu.popcount_raw_lines(ref, per, pats)
    text, n = _engine(cof_mod, chunks).search(filt, user_pats, mm, chunks_per_search=cps,
                                              raw=True)
    mine = _lines(text)
    assert n == len(mine)
    a, b = collections.Counter(ref_lines), collections.Counter(mine)
    assert not (a - b), "reference kernel match missing from the raw stream"
    skipped = ref_gpu.skipped_starts(ref)
    for line in (b - a):
        f = line.split("\t")
        assert (f[0], int(f[1])) in skipped, line
    return len(ref_lines)


@pytest.mark.parametrize("seed", range(10))
def test_reference_popcount_kernel(cof_mod, seed):
    case = randgen.random_case(seed)
    chunks = [(n, d, s, e) for n, d, _nibs, s, e in case["chunks"]]
    assert _check_popcount(cof_mod, chunks, case["filter"], case["patterns"], case["mm"],
                           case["cps"]) > 0


def test_reference_popcount_kernel_kat(cof_mod, oracle_mod, golden):
    # no PAM cells and no N in the genome windows: raw stream == the 117 rows
    chunks = oracle_mod.OracleGenome(os.path.join(golden, "upstream1000.fa")).chunks()
    assert _check_popcount(cof_mod, chunks, "N" * 24, KAT_PATS, 11, 0) == 117


@pytest.mark.parametrize("mm,db,rb", [(3, 1, 1), (2, 2, 0), (2, 0, 2), (4, 2, 2)])
def test_reference_myers_kernel(cof_mod, mm, db, rb):
    rng = random.Random(100 + 10 * mm + 3 * db + rb)
    guides = ["".join(rng.choice("ACGT") for _ in range(20)) for _ in range(2)]
    pats = [g + "NNN" for g in guides]
    filt = "N" * 21 + "RG"
    _, records = randgen.random_genome(rng, 3, 1500, 4000)
    for p in pats:
        randgen.plant_sites(rng, records, p, filt, 8, 2)
    chunks = [(n, d, s, e) for n, d, _nibs, s, e in randgen.chunk_records(rng, records, 900)]
    cps = 4
    full = pats + [bruteforce.revcomp(p) for p in pats]
    ref = ref_gpu.RefGpu(chunks, cps)
    per, _t = ref.myers(filt, full, len(pats), mm, db, rb)
    ref_lines = ref_gpu.myers_raw_lines(ref, per, full)
    text, n = _engine(cof_mod, chunks).search(filt, pats, mm, db, rb, chunks_per_search=cps,
                                              raw=True)
    assert sorted(ref_lines) == sorted(_lines(text))
    assert n == len(ref_lines) > 0
    # the C decode used at the benchmark's size gives the same lines
    ctext, nc, _t = ref.myers_text(filt, full, len(pats), mm, db, rb, out_cap=1 << 20)
    assert sorted(_lines(ctext)) == sorted(ref_lines) and nc == n
