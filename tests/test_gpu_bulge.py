"""GPU parity tests of the bulge (Myers + DP traceback) path against the oracle
and the committed golden rows.  Bit-exact: sorted row sets must be equal."""
import os
import random

import pytest

import randgen

pytestmark = pytest.mark.gpu


def _rows(text):
    return sorted(text.splitlines())


def _both(cof_mod, oracle_mod, chunks):
    g = cof_mod.Genome()
    o = oracle_mod.OracleGenome()
    for name, data, _nibs, s, e in chunks:
        g.add_chunk(name, data, s, e)
        o.add_chunk(name, data, s, e)
    return g, o


@pytest.mark.parametrize("cps", [0, 64, 3])
def test_kat_bulge_rows(cof_mod, golden, cps):
    # integration_bulge.rs:208-259 input; rows pinned by the oracle
    g = cof_mod.Genome(os.path.join(golden, "upstream1000.fa"))
    text, n = g.search("N" * 25 + "GG", ["CCGTGGTTCAACATTTGCTTAGCANNN"], 5, 1, 1,
                       chunks_per_search=cps)
    with open(os.path.join(golden, "kat_bulge_rows.txt")) as f:
        want = f.read().splitlines()
    assert _rows(text) == want and n == len(want)
    for r in want:
        c = r.split("\t")
        assert len(c) == 8 and c[0] in ("X", "DNA", "RNA")


@pytest.mark.parametrize("seed", range(20))
def test_random_bulge_parity(cof_mod, oracle_mod, seed):
    case = randgen.random_case(100 + seed, bulge=True)
    g, o = _both(cof_mod, oracle_mod, case["chunks"])
    text, n = g.search(case["filter"], case["patterns"], case["mm"], case["db"], case["rb"],
                       chunks_per_search=case["cps"])
    ref, nref = o.search(case["filter"], case["patterns"], case["mm"], case["db"], case["rb"],
                         chunks_per_search=case["cps"])
    assert _rows(text) == _rows(ref)
    assert n == nref


def test_bulge_shape_small(cof_mod, oracle_mod):
    # the bulge benchmark shape (20 nt + NRG, mm <= 4, DNA/RNA bulges <= 2) on
    # a 200 kb genome with planted bulged sites
    import synth
    cfg = synth.config_bulge(seed=9, scale=0.0004, n_guides=4, planted=3)
    gen = cfg["genome"]
    g = cof_mod.Genome()
    o = oracle_mod.OracleGenome()
    for name, data, s, e in gen.chunks():
        g.add_chunk(name, data, s, e)
        o.add_chunk(name, data, s, e)
    args = (cfg["filter"], cfg["patterns"], 4, 2, 2)
    text, n = g.search(*args)
    ref, nref = o.search(*args)
    assert n == nref > 1000
    assert _rows(text) == _rows(ref)
    st = g.last_stats()
    assert st["candidates"] > 0 and st["rows"] == n


def test_mixed_popcount_and_bulge_batch(cof_mod, oracle_mod):
    rng = random.Random(77)
    _, records = randgen.random_genome(rng, 3, 2000, 6000)
    reqs = []
    for k, (filt, mk, mm) in enumerate([randgen.REQUEST_SHAPES[i] for i in (0, 1, 2)]):
        guides = ["".join(rng.choice("ACGT") for _ in range(25)) for _ in range(2)]
        pats = [mk(x) for x in guides]
        for p in pats:
            randgen.plant_sites(rng, records, p, filt, 4, 2)
        db, rb = [(0, 0), (1, 1), (2, 0)][k]
        reqs.append(dict(search_filter=filt, patterns=pats, max_mismatches=min(mm, 3),
                         max_dna_bulges=db, max_rna_bulges=rb))
    chunks = randgen.chunk_records(rng, records, 700)
    g, o = _both(cof_mod, oracle_mod, chunks)
    batched = g.search_batch(reqs)
    for r, (text, n) in zip(reqs, batched):
        single, ns = g.search(**r)
        ref, nref = o.search(r["search_filter"], r["patterns"], r["max_mismatches"],
                             r["max_dna_bulges"], r["max_rna_bulges"])
        assert _rows(text) == _rows(single) == _rows(ref)
        assert n == ns == nref


@pytest.mark.parametrize("n_guides,planted", [(4, 5), (20, 30)])
def test_warp_traceback_equals_thread_traceback(cof_mod, oracle_mod, monkeypatch, n_guides,
                                                planted):
    # planted sites with up to 4 mismatches and 2 bulges: candidates with
    # hundreds of alignments next to ones with none.  The warp-per-candidate
    # traceback must give the rows of the thread-per-candidate kernel (and of
    # the oracle, on the smaller case).
    import synth
    cfg = synth.config_bulge(seed=4, scale=0.0004, n_guides=n_guides, planted=planted)
    g = cof_mod.Genome()
    cfg["genome"].load_into(g)
    args = (cfg["filter"], cfg["patterns"], cfg["max_mismatches"], cfg["max_dna_bulges"],
            cfg["max_rna_bulges"])
    monkeypatch.delenv("COF_BULGE_WARP", raising=False)
    text, n = g.search(*args)
    monkeypatch.setenv("COF_BULGE_WARP", "0")
    text0, n0 = g.search(*args)
    assert n == n0 > 0
    assert sorted(text.splitlines()) == sorted(text0.splitlines())
    if n_guides == 4:
        o = oracle_mod.OracleGenome()
        for name, data, s, e in cfg["genome"].chunks():
            o.add_chunk(name, data, s, e)
        ref, nref = o.search(*args)
        assert nref == n and sorted(ref.splitlines()) == sorted(text.splitlines())


@pytest.mark.parametrize("per_chunk", [1, 7, 64])
def test_many_traceback_chunks(cof_mod, oracle_mod, monkeypatch, per_chunk):
    # the surviving candidates are walked in chunks whose row texts follow
    # each other in one device arena, which grows as they come (a large
    # genome makes many chunks; COF_BULGE_CHUNK forces them here); the rows
    # equal the one-chunk search and the oracle
    import synth
    cfg = synth.config_bulge(seed=6, scale=0.0002, n_guides=6, planted=8)
    g = cof_mod.Genome()
    cfg["genome"].load_into(g)
    args = (cfg["filter"], cfg["patterns"], cfg["max_mismatches"], cfg["max_dna_bulges"],
            cfg["max_rna_bulges"])
    # many chunks first: the fresh text arena grows chunk by chunk
    monkeypatch.setenv("COF_BULGE_CHUNK", str(per_chunk))
    many, nm = g.search(*args)
    monkeypatch.delenv("COF_BULGE_CHUNK", raising=False)
    one, n1 = g.search(*args)
    assert nm == n1 > 0 and sorted(many.splitlines()) == sorted(one.splitlines())
    o = oracle_mod.OracleGenome()
    for name, data, s, e in cfg["genome"].chunks():
        o.add_chunk(name, data, s, e)
    ref, nref = o.search(*args)
    assert nref == n1 and sorted(ref.splitlines()) == sorted(one.splitlines())


def test_myers_candidate_list_overflow(cof_mod, oracle_mod, monkeypatch):
    # the Myers candidate list starts at 64 entries (COF_CAND_CAP) on a fresh
    # genome: it overflows, grows and the filter runs again
    import synth
    monkeypatch.setenv("COF_CAND_CAP", "1")
    cfg = synth.config_bulge(seed=7, scale=0.0002, n_guides=4, planted=6)
    g = cof_mod.Genome()
    cfg["genome"].load_into(g)
    args = (cfg["filter"], cfg["patterns"], cfg["max_mismatches"], cfg["max_dna_bulges"],
            cfg["max_rna_bulges"])
    text, n = g.search(*args)
    assert g.last_stats()["candidates"] > 64  # it did overflow
    o = oracle_mod.OracleGenome()
    for name, data, s, e in cfg["genome"].chunks():
        o.add_chunk(name, data, s, e)
    ref, nref = o.search(*args)
    assert n == nref > 0 and sorted(ref.splitlines()) == sorted(text.splitlines())


def test_row_buffer_overflow_halves_chunks(cof_mod, oracle_mod, monkeypatch):
    # a chunk whose alignments pass the row buffer is halved and walked
    # again (COF_BULGE_ROW_CAP lowers the buffer from 16 M rows); the rows
    # equal the oracle's and take more launches than one chunk does
    import synth
    cfg = synth.config_bulge(seed=8, scale=0.0002, n_guides=6, planted=8)
    g = cof_mod.Genome()
    cfg["genome"].load_into(g)
    args = (cfg["filter"], cfg["patterns"], cfg["max_mismatches"], cfg["max_dna_bulges"],
            cfg["max_rna_bulges"])
    monkeypatch.delenv("COF_BULGE_ROW_CAP", raising=False)
    _, n1 = g.search(*args)
    one = g.last_stats()["kernel_launches"]
    monkeypatch.setenv("COF_BULGE_ROW_CAP", str(max(64, n1 // 5)))
    text, n = g.search(*args)
    assert g.last_stats()["kernel_launches"] > one
    o = oracle_mod.OracleGenome()
    for name, data, s, e in cfg["genome"].chunks():
        o.add_chunk(name, data, s, e)
    ref, nref = o.search(*args)
    assert n == n1 == nref > 0 and sorted(ref.splitlines()) == sorted(text.splitlines())
