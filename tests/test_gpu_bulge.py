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


def test_bulge_eq_tables_and_pam_forms_beyond_staging(cof_mod, oracle_mod):
    # myers_tile_kernel stages the Eq tables of at most 512 patterns in
    # shared memory (more are read from the patterns in global memory) and
    # tests at most 8 PAM forms per launch (more go to myers_filter_kernel,
    # which tests the PAM per lane): one request of 300 guides (600
    # patterns), and one pass of five PAM shapes on both strands (10 forms),
    # each request's rows equal to the oracle's
    rng = random.Random(515)
    _, records = randgen.random_genome(rng, 2, 8000, 12000)
    filt0, mk0, _ = randgen.REQUEST_SHAPES[0]
    big_pats = [mk0("".join(rng.choice("ACGT") for _ in range(25))) for _ in range(300)]
    for p in big_pats[:6]:
        randgen.plant_sites(rng, records, p, filt0, 3, 2)
    big = dict(search_filter=filt0, patterns=big_pats, max_mismatches=2, max_dna_bulges=1,
               max_rna_bulges=1)
    mixed = []
    for filt, mk, mm in [randgen.REQUEST_SHAPES[i] for i in (0, 1, 2, 4, 5)]:
        pats = [mk("".join(rng.choice("ACGT") for _ in range(25))) for _ in range(2)]
        for p in pats:
            randgen.plant_sites(rng, records, p, filt, 3, 2)
        mixed.append(dict(search_filter=filt, patterns=pats, max_mismatches=min(mm, 3),
                          max_dna_bulges=1, max_rna_bulges=1))
    g, o = _both(cof_mod, oracle_mod, randgen.chunk_records(rng, records, 700))
    total = 0
    for batch in ([big], mixed):
        for r, (text, n) in zip(batch, g.search_batch(batch)):
            ref, nref = o.search(r["search_filter"], r["patterns"], r["max_mismatches"],
                                 r["max_dna_bulges"], r["max_rna_bulges"])
            assert n == nref and _rows(text) == _rows(ref)
            total += n
    g.close()
    o.close()
    assert total > 100


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


@pytest.mark.parametrize("mm,db,rb", [(4, 2, 2), (3, 1, 1), (2, 3, 0), (2, 0, 3), (3, 3, 3)])
def test_band_dp_equals_whole_table(cof_mod, oracle_mod, monkeypatch, mm, db, rb):
    # the budget pre-test and the traceback read only the band of the DP
    # that alignments within the caps can touch (db + rb + 1 cells per row);
    # their rows must equal those of the whole-table kernels
    # (COF_BULGE_BAND=0) and of the oracle, also near record and batch
    # starts, where the window is shorter than L + db
    import synth
    cfg = synth.config_bulge(seed=7, scale=0.0004, n_guides=4, planted=6)
    g = cof_mod.Genome()
    cfg["genome"].load_into(g)
    args = (cfg["filter"], cfg["patterns"], mm, db, rb)
    monkeypatch.delenv("COF_BULGE_BAND", raising=False)
    text, n = g.search(*args, chunks_per_search=3)
    monkeypatch.setenv("COF_BULGE_BAND", "0")
    text0, n0 = g.search(*args, chunks_per_search=3)
    assert n == n0 > 0
    assert sorted(text.splitlines()) == sorted(text0.splitlines())
    o = oracle_mod.OracleGenome()
    for name, data, s, e in cfg["genome"].chunks():
        o.add_chunk(name, data, s, e)
    ref, nref = o.search(*args, chunks_per_search=3)
    assert nref == n and sorted(ref.splitlines()) == sorted(text.splitlines())


@pytest.mark.parametrize("slots,budget,chunk,tables", [
    (6, 0, 0, "global"), (8, 1, 0, "global"), (1, 2, 0, "global"), (6, 3, 5, "global"),
    (4, 0, 0, "shared"), (2, 0, 0, "shared"), (1, 0, 0, "shared"), (4, 1, 0, "shared"),
    (3, 2, 0, "shared"), (4, 3, 5, "shared")])
def test_slot_traceback_equals_one_tree_per_warp(cof_mod, oracle_mod, monkeypatch, slots, budget,
                                                 chunk, tables):
    # traceback_slots_kernel keeps several candidates' trees in one warp's
    # stack, reading their band tables from global memory or from copies in
    # the slots (COF_TB_GLOBAL=0); its rows must equal those of one tree
    # per warp (COF_TB_SLOTS=0) and of the oracle.  Budgets of 1-3 steps
    # make slots hand their nodes on after almost every step (hand-on
    # passes up to the last, which finishes every tree); small candidate
    # chunks make many launches with few candidates
    import synth
    cfg = synth.config_bulge(seed=5, scale=0.0004, n_guides=6, planted=8)
    g = cof_mod.Genome()
    cfg["genome"].load_into(g)
    args = (cfg["filter"], cfg["patterns"], 4, 2, 2)
    monkeypatch.setenv("COF_TB_SLOTS", "0")
    text0, n0 = g.search(*args)
    monkeypatch.setenv("COF_TB_SLOTS", str(slots))
    monkeypatch.setenv("COF_TB_GLOBAL", "1" if tables == "global" else "0")
    if budget:
        monkeypatch.setenv("COF_TB_BUDGET", str(budget))
    if chunk:
        monkeypatch.setenv("COF_BULGE_CHUNK", str(chunk))
    text, n = g.search(*args)
    g.close()
    assert n == n0 > 1000
    assert sorted(text.splitlines()) == sorted(text0.splitlines())
    o = oracle_mod.OracleGenome()
    for name, data, s, e in cfg["genome"].chunks():
        o.add_chunk(name, data, s, e)
    ref, nref = o.search(*args)
    o.close()
    assert nref == n and sorted(ref.splitlines()) == sorted(text.splitlines())


@pytest.mark.parametrize("stage", [0, 7, 100])
def test_myers_stage_overflow(cof_mod, oracle_mod, monkeypatch, stage):
    # myers_tile_kernel stages a round's candidates in shared memory and
    # appends them with one atomic; candidates past the stage go straight
    # to the list.  A stage of 0 / 7 / 100 candidates (COF_MYERS_STAGE; the
    # default holds 3072) sends most of them that way: the rows must not
    # change
    import synth
    cfg = synth.config_bulge(seed=8, scale=0.0004, n_guides=6, planted=8)
    g = cof_mod.Genome()
    cfg["genome"].load_into(g)
    args = (cfg["filter"], cfg["patterns"], 4, 2, 2)
    monkeypatch.delenv("COF_MYERS_STAGE", raising=False)
    text0, n0 = g.search(*args)
    cand0 = g.last_stats()["candidates"]
    monkeypatch.setenv("COF_MYERS_STAGE", str(stage))
    text, n = g.search(*args)
    assert g.last_stats()["candidates"] == cand0 > 10000
    g.close()
    assert n == n0 > 1000
    assert sorted(text.splitlines()) == sorted(text0.splitlines())
    o = oracle_mod.OracleGenome()
    for name, data, s, e in cfg["genome"].chunks():
        o.add_chunk(name, data, s, e)
    ref, nref = o.search(*args)
    o.close()
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


def _plant_bulged(rng, records, pattern, filt, count, subs):
    """Near-copies of pattern with subs substitutions and one inserted or
    deleted cell outside the PAM, on either strand."""
    comp = {"A": "T", "C": "G", "G": "C", "T": "A"}
    free = [i for i, c in enumerate(pattern) if c in "ACGT" and filt[i] == "N"]
    for _ in range(count):
        r = rng.randrange(len(records))
        seq = records[r]
        site = []
        for i, c in enumerate(pattern):
            f = filt[i]
            if c not in "ACGT":
                site.append(rng.choice([b for b in "ACGT" if randgen.B4[b] & randgen.B4[f]]))
            else:
                site.append(c)
        for i in rng.sample(free, subs):
            site[i] = rng.choice([b for b in "ACGT" if b != site[i]])
        k = rng.choice(free[2:-2])
        if rng.random() < 0.5:
            site.insert(k, rng.choice("ACGT"))  # a DNA bulge
        else:
            del site[k]  # an RNA bulge
        s = "".join(site)
        if rng.random() < 0.5:
            s = "".join(comp[c] for c in reversed(s))
        p = rng.randrange(0, len(seq) - len(s))
        records[r] = seq[:p] + s + seq[p + len(s):]


# (L, PAM side, mm, db, rb): 64-bit Myers words for every L > 32; windows
# W = L + db of <= 48 cells (one op word per traceback node) and above
# (two, with ops past 64 in the row's third word); (db + 1)(rb + 1)(mm + 1)
# budget bits of one word and of two
LONG_BULGE_CASES = [
    (33, "3", 3, 1, 1),
    (40, "5", 3, 2, 1),
    (48, "3", 2, 1, 2),
    (57, "5", 8, 1, 3),
    (64, "3", 3, 8, 0),
    (64, "-", 2, 2, 2),
]


@pytest.mark.parametrize("L,pam,mm,db,rb", LONG_BULGE_CASES)
def test_bulge_patterns_longer_than_32_cells(cof_mod, oracle_mod, monkeypatch, L, pam, mm, db,
                                             rb):
    rng = random.Random(900 + L + db)
    _, records = randgen.random_genome(rng, 3, 20000, 30000)
    guide = lambda n: "".join(rng.choice("ACGT") for _ in range(n))
    if pam == "3":
        filt, pats = "N" * (L - 2) + "RG", [guide(L - 3) + "NNN" for _ in range(2)]
    elif pam == "5":
        filt, pats = "TTTN" + "N" * (L - 4), ["NNNN" + guide(L - 4) for _ in range(2)]
    else:
        filt, pats = "N" * L, [guide(L) for _ in range(2)]
    for p in pats:
        _plant_bulged(rng, records, p, filt, 4, min(mm, 2))
        randgen.plant_sites(rng, records, p, filt, 2, mm)
    g, o = _both(cof_mod, oracle_mod, randgen.chunk_records(rng, records, 5000))
    args = (filt, pats, mm, db, rb)
    monkeypatch.delenv("COF_BULGE_WARP", raising=False)
    text, n = g.search(*args)
    ref, nref = o.search(*args)
    assert n == nref > 0
    assert _rows(text) == _rows(ref)
    assert any(r.split("\t")[0] in ("DNA", "RNA") for r in ref.splitlines())
    if L + db > 64 and db > 0:  # alignments of more than 64 ops
        assert any(len(r.split("\t")[1]) > 64 for r in ref.splitlines())
    raw, nraw = g.search(*args, raw=True)
    rref, nrref = o.search(*args, raw=True)
    assert nraw == nrref and sorted(raw.split("\n")[:-1]) == sorted(rref.split("\n")[:-1])
    monkeypatch.setenv("COF_BULGE_WARP", "0")  # the thread-per-candidate traceback
    text0, n0 = g.search(*args)
    assert n0 == n and _rows(text0) == _rows(text)


def test_long_and_short_bulge_requests_in_one_batch(cof_mod, oracle_mod):
    # a 23-cell and a 60-cell request share one launch: 64-bit Myers words,
    # two-word nodes and the five-word budget filter serve both
    rng = random.Random(31)
    _, records = randgen.random_genome(rng, 3, 15000, 25000)
    guide = lambda n: "".join(rng.choice("ACGT") for _ in range(n))
    short = ("N" * 21 + "RG", [guide(20) + "NNN" for _ in range(2)], 3, 1, 1)
    long_ = ("N" * 58 + "RG", [guide(57) + "NNN" for _ in range(2)], 3, 2, 1)
    for filt, pats, mm, _db, _rb in (short, long_):
        for p in pats:
            _plant_bulged(rng, records, p, filt, 4, 2)
    g, o = _both(cof_mod, oracle_mod, randgen.chunk_records(rng, records, 4000))
    reqs = [dict(search_filter=f, patterns=p, max_mismatches=m, max_dna_bulges=d,
                 max_rna_bulges=r) for f, p, m, d, r in (short, long_)]
    for (f, p, m, d, r), (text, n) in zip((short, long_), g.search_batch(reqs)):
        ref, nref = o.search(f, p, m, d, r)
        assert n == nref > 0 and _rows(text) == _rows(ref)
