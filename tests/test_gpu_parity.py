"""GPU parity tests: libcof.so (through the C ABI) against the oracle and the
committed golden rows.  Bit-exact: sorted row sets must be identical."""
import os
import random
import subprocess

import pytest

import randgen

pytestmark = pytest.mark.gpu

KAT_PATS = ["CCGTGGTTCAACATTTGCTTAGCA", "GATGTTGGTAAGTGGGATATGGCA"]


def _rows(text):
    return sorted(text.splitlines())


def _golden_rows(golden, name):
    with open(os.path.join(golden, name)) as f:
        return f.read().splitlines()


@pytest.mark.parametrize("cps", [0, 64, 2])
def test_kat_popcount_117(cof_mod, golden, cps):
    g = cof_mod.Genome(os.path.join(golden, "upstream1000.fa"))
    text, n = g.search("N" * 24, KAT_PATS, 11, chunks_per_search=cps)
    assert n == 117
    assert _rows(text) == _golden_rows(golden, "kat_popcount_rows.txt")


def test_kat_popcount_2bit(cof_mod, oracle_mod, golden):
    path = os.path.join(golden, "upstream1000.2bit")
    g = cof_mod.Genome(path)
    text, n = g.search("N" * 24, KAT_PATS, 11)
    o, _ = oracle_mod.OracleGenome(path).search("N" * 24, KAT_PATS, 11)
    assert n == 117 and _rows(text) == _rows(o)


def _both(cof_mod, oracle_mod, chunks):
    g = cof_mod.Genome()
    o = oracle_mod.OracleGenome()
    for name, data, _nibs, s, e in chunks:
        g.add_chunk(name, data, s, e)
        o.add_chunk(name, data, s, e)
    return g, o


@pytest.mark.parametrize("seed", range(24))
def test_random_popcount_parity(cof_mod, oracle_mod, seed):
    case = randgen.random_case(seed)
    g, o = _both(cof_mod, oracle_mod, case["chunks"])
    text, n = g.search(case["filter"], case["patterns"], case["mm"],
                       chunks_per_search=case["cps"])
    ref, nref = o.search(case["filter"], case["patterns"], case["mm"],
                         chunks_per_search=case["cps"])
    assert _rows(text) == _rows(ref)
    assert n == nref > 0


def test_full_pattern_list_matches_add_revcomp(cof_mod, golden):
    # search() takes fwd+rc as main.rs builds them; COF_F_ADD_REVCOMP builds them
    import bruteforce
    g = cof_mod.Genome(os.path.join(golden, "upstream1000.fa"))
    a, _ = g.search("N" * 24, KAT_PATS, 11)
    full = KAT_PATS + [bruteforce.revcomp(p) for p in KAT_PATS]
    b, _ = g.search("N" * 24, full, 11, add_revcomp=False)
    assert a == b


def test_batched_equals_single(cof_mod, oracle_mod):
    rng = random.Random(5)
    _, records = randgen.random_genome(rng, 4, 3000, 9000)
    cases = [randgen.REQUEST_SHAPES[i] for i in (0, 1, 2, 4)]
    reqs = []
    for filt, mk, mm in cases:
        guides = ["".join(rng.choice("ACGT") for _ in range(25)) for _ in range(3)]
        pats = [mk(x) for x in guides]
        for p in pats:
            randgen.plant_sites(rng, records, p, filt, 5, 2)
        reqs.append(dict(search_filter=filt, patterns=pats, max_mismatches=mm))
    chunks = randgen.chunk_records(rng, records, 500)
    g, o = _both(cof_mod, oracle_mod, chunks)
    batched = g.search_batch(reqs)
    for r, (text, n) in zip(reqs, batched):
        single, ns = g.search(**r)
        ref, _ = o.search(r["search_filter"], r["patterns"], r["max_mismatches"])
        assert text == single and n == ns
        assert _rows(text) == _rows(ref)


def test_many_small_requests_in_one_pass(cof_mod):
    # 300 one-guide requests in one pass: their result texts are blocks cut
    # from shared page-locked slabs and their text boundaries are read in one
    # wait; every request equals its own search, twice over (blocks reused)
    rng = random.Random(15)
    _, records = randgen.random_genome(rng, 3, 20000, 30000)
    reqs = []
    for i in range(300):
        filt, mk, mm = randgen.REQUEST_SHAPES[i % 3]
        pat = mk("".join(rng.choice("ACGT") for _ in range(25)))
        if i % 2:
            randgen.plant_sites(rng, records, pat, filt, 2, 1)
        reqs.append(dict(search_filter=filt, patterns=[pat], max_mismatches=mm))
    g = cof_mod.Genome()
    for name, data, _nibs, s, e in randgen.chunk_records(rng, records, 3000):
        g.add_chunk(name, data, s, e)
    singles = [g.search(**r) for r in reqs]
    assert sum(n for _, n in singles) > 100
    for _ in range(2):
        assert g.search_batch(reqs) == singles


@pytest.mark.parametrize("scale", [0.05, 1.0])
def test_planted_sites_found(cof_mod, oracle_mod, tmp_path, scale):
    # the plain small workload (10 Mbp x 1 guide at scale 1.0) through a
    # FASTA file: every planted site, and exactly the oracle's rows
    import synth
    cfg = synth.config_plain_small(seed=11, scale=scale)
    gen = cfg["genome"]
    g = cof_mod.Genome()
    gen.load_into(g)
    text, n = g.search(cfg["filter"], cfg["patterns"], cfg["max_mismatches"])
    rows = text.splitlines()
    found = {(r.split("\t")[3], int(r.split("\t")[4]), r.split("\t")[5]) for r in rows}
    for rec, pos, strand, _gi, _k, ln in cfg["truth"]:
        # − strand rows report the position shifted by pam_len - 1 (main.rs:229-236)
        want = pos + (2 if strand == "-" else 0)
        assert (gen.names[rec], want, strand) in found
    fa = tmp_path / "g.fa"
    gen.write_fasta(str(fa))
    ref, nref = oracle_mod.OracleGenome(str(fa)).search(cfg["filter"], cfg["patterns"],
                                                         cfg["max_mismatches"])
    assert _rows(text) == _rows(ref) and n == nref
    text2, n2 = cof_mod.Genome(str(fa)).search(cfg["filter"], cfg["patterns"],
                                               cfg["max_mismatches"])
    assert _rows(text2) == _rows(ref) and n2 == nref  # the file converted on the device


def test_cli_matches_oracle_cli(cof_mod, oracle_mod, golden, tmp_path):
    cli = os.path.join(os.path.dirname(cof_mod.LIB_PATH), "cof-offinder")
    ocli = os.path.join(os.path.dirname(oracle_mod.LIB_PATH), "cof_oracle")
    inp = tmp_path / "in.txt"
    inp.write_text(os.path.join(golden, "upstream1000.fa") + "\n" + "N" * 24 + "\n" +
                   "".join(f"{p} 11\n" for p in KAT_PATS))
    for dev in ("C", "G"):
        out, oout = tmp_path / f"o{dev}.txt", tmp_path / f"r{dev}.txt"
        subprocess.run([cli, str(inp), dev, str(out)], check=True, capture_output=True)
        subprocess.run([ocli, str(inp), dev, str(oout)], check=True, capture_output=True)
        a, b = out.read_text().splitlines(), oout.read_text().splitlines()
        assert a[0] == b[0] and a[0].startswith("#Bulge type")
        assert sorted(a[1:]) == sorted(b[1:]) and len(a) == 118
        log = (tmp_path / f"o{dev}.txt.log").read_text()
        assert "=== Cas-OFFinder Rust ===" in log and "Matches found: 117" in log


# per-warp work items: 0-4 and 8; CTA work items: 5-7; strand pairs compared
# directly, holding 1 or 2 patterns per group: 9-12 (a request whose groups
# are larger runs the default shape instead)
N_SCAN_VARIANTS = 13
PAIR_VARIANTS = {9: 1, 10: 2, 11: 1, 12: 2}


def _expected_variant(variant, patterns_per_group):
    if variant in PAIR_VARIANTS and patterns_per_group > PAIR_VARIANTS[variant]:
        return 0
    return variant


@pytest.mark.parametrize("variant", range(N_SCAN_VARIANTS))
def test_every_scan_tile_shape(cof_mod, oracle_mod, golden, variant, monkeypatch):
    # the autotuner may pick any tile shape; all must give the same rows
    monkeypatch.setenv("COF_SCAN_VARIANT", str(variant))
    g = cof_mod.Genome(os.path.join(golden, "upstream1000.fa"))
    text, n = g.search("N" * 24, KAT_PATS, 11)
    assert n == 117 and _rows(text) == _golden_rows(golden, "kat_popcount_rows.txt")
    case = randgen.random_case(variant + 40)
    g2, o = _both(cof_mod, oracle_mod, case["chunks"])
    text, _ = g2.search(case["filter"], case["patterns"], case["mm"], chunks_per_search=case["cps"])
    ref, _ = o.search(case["filter"], case["patterns"], case["mm"], chunks_per_search=case["cps"])
    assert _rows(text) == _rows(ref)
    assert g2.tuning()["variant"] == _expected_variant(variant, len(case["patterns"]))


@pytest.mark.parametrize("variant", [0, 3, 5])
def test_patterns_beyond_the_shared_memory_table(cof_mod, oracle_mod, variant, monkeypatch):
    # 1500 guides: 3000 patterns in two strand groups; the per-warp scan
    # stages the first 1024 or 2048 patterns, so later groups read their
    # patterns from global memory
    monkeypatch.setenv("COF_SCAN_VARIANT", str(variant))
    rng = random.Random(77)
    _, records = randgen.random_genome(rng, 2, 20000, 30000)
    pats = ["".join(rng.choice("ACGT") for _ in range(20)) + "NNN" for _ in range(1500)]
    for p in pats[::100]:
        randgen.plant_sites(rng, records, p, "N" * 21 + "RG", 2, 3)
    chunks = randgen.chunk_records(rng, records, 4000)
    g, o = _both(cof_mod, oracle_mod, chunks)
    text, n = g.search("N" * 21 + "RG", pats, 4)
    ref, nref = o.search("N" * 21 + "RG", pats, 4)
    assert n == nref > 0 and _rows(text) == _rows(ref)
    assert g.tuning()["variant"] == variant


@pytest.mark.parametrize("variant", sorted(PAIR_VARIANTS))
@pytest.mark.parametrize("cps", [0, 3])
def test_strand_pairs_in_a_mixed_batch(cof_mod, oracle_mod, variant, cps, monkeypatch):
    # the direct strand-pair scan takes both strand groups of a filter as
    # one work item (and a group without a partner alone), with the groups'
    # patterns in registers: a batch of requests with 3' and 5' PAMs, no
    # PAM, a 40-cell pattern, IUPAC guides and different lengths and
    # thresholds gives every request's rows, equal to its own oracle run
    monkeypatch.setenv("COF_SCAN_VARIANT", str(variant))
    rng = random.Random(900 + variant + cps)
    _, records = randgen.random_genome(rng, 3, 20000, 40000)
    n_pat = PAIR_VARIANTS[variant]
    reqs = []
    for filt, mk, mm in randgen.REQUEST_SHAPES:
        pats = [mk("".join(rng.choice("ACGT") for _ in range(25))) for _ in range(n_pat)]
        for p in pats:
            randgen.plant_sites(rng, records, p.upper(), filt, 8, 2)
        reqs.append(dict(search_filter=filt, patterns=pats, max_mismatches=mm,
                         chunks_per_search=cps))
    g40 = "".join(rng.choice("ACGT") for _ in range(37))
    reqs.append(dict(search_filter="N" * 38 + "AG", patterns=[g40 + "NNN"], max_mismatches=5,
                     chunks_per_search=cps))
    randgen.plant_sites(rng, records, g40 + "NNN", "N" * 38 + "AG", 8, 3)
    g, o = _both(cof_mod, oracle_mod, randgen.chunk_records(rng, records, 2500))
    res = g.search_batch(reqs)
    assert g.tuning()["variant"] == variant and g.tuning()["last"].startswith("pair-")
    for r, (text, n) in zip(reqs, res):
        ref, nref = o.search(r["search_filter"], r["patterns"], r["max_mismatches"],
                             chunks_per_search=cps)
        assert n == nref and _rows(text) == _rows(ref)
    for r, (text, n) in zip(reqs, res):  # alone, each gives the same text
        assert g.search(r["search_filter"], r["patterns"], r["max_mismatches"],
                        chunks_per_search=cps) == (text, n)


def test_candidate_list_overflow(cof_mod, golden, monkeypatch):
    # a fresh genome whose scan hit list starts at 64 entries (COF_CAND_CAP):
    # the KAT's hits overflow it, the list grows and the scan runs again
    monkeypatch.setenv("COF_CAND_CAP", "1")
    g = cof_mod.Genome(os.path.join(golden, "upstream1000.fa"))
    text, n = g.search("N" * 24, KAT_PATS, 11)
    assert n == 117 and _rows(text) == _golden_rows(golden, "kat_popcount_rows.txt")
    assert g.last_stats()["raw_hits"] > 64  # it did overflow


@pytest.mark.parametrize("L", [33, 40, 51, 64])
def test_patterns_longer_than_the_scan_window(cof_mod, oracle_mod, L):
    # patterns of 33-64 cells: the 32-cell scan window holds the PAM end
    # (3' PAM) or start (5' PAM) of the pattern, and verify recounts all of
    # it; rows equal the oracle's for a 3' PAM, a 5' PAM and no PAM, and in a
    # batch that mixes 23- and L-cell NRG requests (one scan group)
    rng = random.Random(700 + L)
    _, records = randgen.random_genome(rng, 3, 30000, 50000)
    guide = lambda n: "".join(rng.choice("ACGT") for _ in range(n))
    shapes = [
        ("N" * (L - 2) + "RG", [guide(L - 3) + "NNN" for _ in range(3)], 6),
        ("TTTN" + "N" * (L - 4), ["NNNN" + guide(L - 4) for _ in range(3)], 6),
        ("N" * L, [guide(L) for _ in range(2)], 5),
    ]
    for filt, pats, mm in shapes:
        for p in pats:
            randgen.plant_sites(rng, records, p, filt, 6, mm)
    short = ("N" * 21 + "RG", [guide(20) + "NNN" for _ in range(2)], 4)
    for p in short[1]:
        randgen.plant_sites(rng, records, p, short[0], 4, 3)
    g, o = _both(cof_mod, oracle_mod, randgen.chunk_records(rng, records, 5000))
    for filt, pats, mm in shapes:
        text, n = g.search(filt, pats, mm)
        ref, nref = o.search(filt, pats, mm)
        assert n == nref and _rows(text) == _rows(ref), filt
    assert sum(o.search(f, p, m)[1] for f, p, m in shapes) > 10
    reqs = [dict(search_filter=short[0], patterns=short[1], max_mismatches=short[2]),
            dict(search_filter=shapes[0][0], patterns=shapes[0][1], max_mismatches=shapes[0][2])]
    for r, (text, n) in zip(reqs, g.search_batch(reqs)):
        ref, nref = o.search(r["search_filter"], r["patterns"], r["max_mismatches"])
        assert n == nref and _rows(text) == _rows(ref)
    for filt, pats, mm in shapes:  # the raw Match stream compares all L cells
        raw, nraw = g.search(filt, pats, mm, raw=True)
        rref, nrref = o.search(filt, pats, mm, raw=True)
        assert nraw == nrref and sorted(raw.split("\n")[:-1]) == sorted(rref.split("\n")[:-1])


def test_autotuner_records_choice(cof_mod, golden, monkeypatch):
    monkeypatch.delenv("COF_SCAN_VARIANT", raising=False)
    g = cof_mod.Genome(os.path.join(golden, "upstream1000.fa"))
    g.search("N" * 24, KAT_PATS, 11)
    t = g.tuning()
    assert ("cpt" in t["last"] or "direct" in t["last"]) and 0 <= t["variant"] < N_SCAN_VARIANTS


@pytest.mark.parametrize("seed", range(8))
def test_raw_matches_parity(cof_mod, oracle_mod, seed):
    # COF_F_RAW_MATCHES: search()'s Match stream before the writer
    case = randgen.random_case(seed)
    g, o = _both(cof_mod, oracle_mod, case["chunks"])
    text, n = g.search(case["filter"], case["patterns"], case["mm"],
                       chunks_per_search=case["cps"], raw=True)
    ref, nref = o.search(case["filter"], case["patterns"], case["mm"],
                         chunks_per_search=case["cps"], raw=True)
    assert sorted(text.split("\n")[:-1]) == sorted(ref.split("\n")[:-1])
    assert n == nref > 0


def test_raw_matches_bulge_parity(cof_mod, oracle_mod):
    case = randgen.random_case(105, bulge=True)
    g, o = _both(cof_mod, oracle_mod, case["chunks"])
    args = (case["filter"], case["patterns"], case["mm"], case["db"], case["rb"])
    text, n = g.search(*args, chunks_per_search=case["cps"], raw=True)
    ref, nref = o.search(*args, chunks_per_search=case["cps"], raw=True)
    assert sorted(text.split("\n")[:-1]) == sorted(ref.split("\n")[:-1]) and n == nref


def test_raw_kat_has_unfiltered_windows(cof_mod, golden):
    # with a PAM in the filter the raw stream holds windows the writer drops
    g = cof_mod.Genome(os.path.join(golden, "upstream1000.fa"))
    raw, nraw = g.search("N" * 21 + "GG", ["CCGTGGTTCAACATTTGCTTNNN"], 6, raw=True)
    rows, nrows = g.search("N" * 21 + "GG", ["CCGTGGTTCAACATTTGCTTNNN"], 6)
    assert nraw > nrows


@pytest.mark.parametrize("cps", [0, 3])
def test_shared_pam_groups_of_mixed_lengths(cof_mod, oracle_mod, cps):
    # requests with one PAM but different guide lengths and mismatch limits
    # share a scan group (windows anchored at the PAM); each result must
    # equal the request alone and the oracle, also across batch boundaries
    rng = random.Random(77)
    _, records = randgen.random_genome(rng, 3, 4000, 9000)
    reqs = []
    for gl, mm in ((17, 2), (20, 4), (25, 3), (29, 5)):  # 3' NRG
        guides = ["".join(rng.choice("ACGT") for _ in range(gl)) for _ in range(2)]
        pats = [x + "NNN" for x in guides]
        for p in pats:
            randgen.plant_sites(rng, records, p, "N" * gl + "NRG", 4, 2)
        reqs.append(dict(search_filter="N" * gl + "NRG", patterns=pats, max_mismatches=mm))
    for gl, mm in ((18, 3), (23, 4)):  # 5' TTTN
        guides = ["".join(rng.choice("ACGT") for _ in range(gl)) for _ in range(2)]
        pats = ["NNNN" + x for x in guides]
        for p in pats:
            randgen.plant_sites(rng, records, p, "TTTN" + "N" * gl, 4, 2)
        reqs.append(dict(search_filter="TTTN" + "N" * gl, patterns=pats, max_mismatches=mm))
    chunks = randgen.chunk_records(rng, records, 700)
    g, o = _both(cof_mod, oracle_mod, chunks)
    for r in reqs:
        r["chunks_per_search"] = cps
    batched = g.search_batch(reqs)
    for r, (text, n) in zip(reqs, batched):
        single, ns = g.search(**r)
        ref, nref = o.search(r["search_filter"], r["patterns"], r["max_mismatches"],
                             chunks_per_search=cps)
        assert text == single and n == ns
        assert _rows(text) == _rows(ref) and n == nref > 0


def test_fasta_loader_matches_chunks(cof_mod, tmp_path):
    # the parallel FASTA reader yields the chunks read_fasta.rs would: same
    # chunk table and the same rows as the genome added chunk by chunk
    import synth
    cfg = synth.config_plain_small(seed=13, scale=0.05)
    gen = cfg["genome"]
    fa = tmp_path / "g.fa"
    gen.write_fasta(str(fa))
    a = cof_mod.Genome(str(fa))
    b = cof_mod.Genome()
    gen.load_into(b)
    assert a.n_nucl == b.n_nucl == gen.n_nucl
    args = (cfg["filter"], cfg["patterns"], cfg["max_mismatches"])
    ta, na = a.search(*args, chunks_per_search=3)
    tb, nb = b.search(*args, chunks_per_search=3)
    assert ta == tb and na == nb > 0


def test_2bit_loader_matches_fasta(cof_mod, oracle_mod, tmp_path):
    # records of odd lengths, N runs crossing 64 Knt chunk boundaries and
    # several runs per chunk; an all-N pattern in raw mode lists every window
    # with its cells, so equal raw streams mean equal genomes
    import twobit
    rng = random.Random(21)
    recs = []
    for r, n in enumerate((70001, 140003, 3)):
        seq = [rng.choice("ACGTacgt") for _ in range(n)]
        for a, b in ((65530, 65541), (100, 130), (131060, 131090)):
            for i in range(a, min(b, n)):
                seq[i] = "N"
        recs.append((f"chr{r}", "".join(seq)))
    fa, tb = tmp_path / "g.fa", tmp_path / "g.2bit"
    with open(fa, "w") as f:
        for name, seq in recs:
            f.write(">" + name + "\n")
            for i in range(0, len(seq), 61):
                f.write(seq[i:i + 61].upper() + "\n")
    twobit.write_2bit(str(tb), recs)
    a, b = cof_mod.Genome(str(tb)), cof_mod.Genome(str(fa))
    assert a.n_nucl == b.n_nucl == sum(len(s) for _, s in recs)
    ra, na = a.search("N" * 8, ["N" * 8], 7, raw=True)
    rb, nb = b.search("N" * 8, ["N" * 8], 7, raw=True)
    ref, nref = oracle_mod.OracleGenome(str(tb)).search("N" * 8, ["N" * 8], 7, raw=True)
    assert na == nb == nref > 0
    assert sorted(ra.split("\n")) == sorted(ref.split("\n"))


def _nrun_records(rng, lengths, n_runs):
    recs = []
    for r, n in enumerate(lengths):
        seq = [rng.choice("ACGTacgt") for _ in range(n)]
        for _ in range(n_runs):
            a = rng.randrange(n)
            for i in range(a, min(n, a + rng.randint(1, 60))):
                seq[i] = "N"
        recs.append((f"chr{r}", "".join(seq)))
    return recs


def test_2bit_device_decode_many_n_blocks(cof_mod, oracle_mod, tmp_path):
    # .2bit bases are decoded on the device at upload; hundreds of short N
    # blocks per 64 Knt chunk, blocks touching chunk ends, odd record
    # lengths: every window of the raw stream equals the oracle's
    import twobit
    rng = random.Random(23)
    recs = _nrun_records(rng, (200003, 65536, 65537, 1, 7), 400)
    tb = tmp_path / "g.2bit"
    twobit.write_2bit(str(tb), recs)
    g = cof_mod.Genome(str(tb))
    o = oracle_mod.OracleGenome(str(tb))
    assert g.n_nucl == o.n_nucl == sum(len(x) for _, x in recs)
    ra, na = g.search("N" * 6, ["N" * 6], 5, raw=True)
    ref, nref = o.search("N" * 6, ["N" * 6], 5, raw=True)
    assert na == nref > 0 and sorted(ra.split("\n")) == sorted(ref.split("\n"))
    pats = ["".join(rng.choice("ACGT") for _ in range(20)) + "NNN" for _ in range(4)]
    text, n = g.search("N" * 21 + "RG", pats, 5)
    rtext, rn = o.search("N" * 21 + "RG", pats, 5)
    assert n == rn and _rows(text) == _rows(rtext)


def test_chunk_added_after_2bit_load(cof_mod, oracle_mod, tmp_path):
    # adding a chunk to a genome loaded from .2bit decodes the file's bases
    # on the host first (the device decode only covers a genome that is one
    # .2bit file); the result equals the oracle's genome built the same way
    import twobit
    rng = random.Random(29)
    recs = _nrun_records(rng, (70001, 3001), 30)
    tb = tmp_path / "g.2bit"
    twobit.write_2bit(str(tb), recs)
    extra = randgen.chunk_records(rng, ["".join(rng.choice("ACGT") for _ in range(5000))], 5000)
    g = cof_mod.Genome(str(tb))
    o = oracle_mod.OracleGenome(str(tb))
    for name, data, _nibs, s, e in extra:
        g.add_chunk("extra", data, s, e)
        o.add_chunk("extra", data, s, e)
    ra, na = g.search("N" * 6, ["N" * 6], 5, raw=True)
    ref, nref = o.search("N" * 6, ["N" * 6], 5, raw=True)
    assert na == nref > 0 and sorted(ra.split("\n")) == sorted(ref.split("\n"))


@pytest.mark.parametrize("final_newline", [True, False])
def test_fasta_device_conversion(cof_mod, oracle_mod, tmp_path, final_newline):
    # a FASTA file is converted on the device at upload; every window of the
    # raw stream equals the oracle's own FASTA reader
    rng = random.Random(41 + final_newline)
    fa = tmp_path / "g.fa"
    randgen.write_messy_fasta(rng, fa, final_newline)
    g = cof_mod.Genome(str(fa))
    o = oracle_mod.OracleGenome(str(fa))
    assert g.n_nucl == o.n_nucl and g.n_chunks == o.n_chunks
    ra, na = g.search("N" * 5, ["N" * 5], 4, raw=True)
    ref, nref = o.search("N" * 5, ["N" * 5], 4, raw=True)
    assert na == nref > 0 and sorted(ra.split("\n")) == sorted(ref.split("\n"))


@pytest.mark.parametrize("seed", range(6))
def test_random_genome_files_device_decode(cof_mod, oracle_mod, tmp_path, seed):
    # seeded random FASTA and .2bit files of a few records: the device
    # conversion of each equals the oracle's reader, window by window
    import twobit
    rng = random.Random(100 + seed)
    fa = tmp_path / "r.fa"
    parts = []
    recs = []
    for r in range(rng.randint(1, 4)):
        n = rng.randint(1, 90000)
        seq = "".join(rng.choice("ACGTNacgtnRY") for _ in range(n))
        recs.append((f"s{r}", seq.replace("R", "N").replace("Y", "N")))
        parts.append(f">s{r} x\n")
        i = 0
        while i < n:
            ln = rng.choice([1, 7, 50, 60, 61, 80, 4000])
            parts.append(seq[i:i + ln] + rng.choice(["\n", "\r\n"]))
            i += ln
    fa.write_text("".join(parts), newline="")
    tb = tmp_path / "r.2bit"
    twobit.write_2bit(str(tb), recs)
    for path in (fa, tb):
        g = cof_mod.Genome(str(path))
        o = oracle_mod.OracleGenome(str(path))
        assert g.n_nucl == o.n_nucl and g.n_chunks == o.n_chunks
        ra, na = g.search("N" * 4, ["N" * 4], 3, raw=True)
        ref, nref = o.search("N" * 4, ["N" * 4], 3, raw=True)
        assert na == nref and sorted(ra.split("\n")) == sorted(ref.split("\n"))


def test_chunk_added_after_fasta_load(cof_mod, oracle_mod, tmp_path):
    # adding a chunk after a FASTA load converts the file on the host first
    rng = random.Random(43)
    fa = tmp_path / "g.fa"
    randgen.write_messy_fasta(rng, fa, True)
    extra = randgen.chunk_records(rng, ["".join(rng.choice("ACGT") for _ in range(3000))], 3000)
    g = cof_mod.Genome(str(fa))
    o = oracle_mod.OracleGenome(str(fa))
    for name, data, _nibs, s, e in extra:
        g.add_chunk("extra", data, s, e)
        o.add_chunk("extra", data, s, e)
    ra, na = g.search("N" * 5, ["N" * 5], 4, raw=True)
    ref, nref = o.search("N" * 5, ["N" * 5], 4, raw=True)
    assert na == nref > 0 and sorted(ra.split("\n")) == sorted(ref.split("\n"))


@pytest.mark.parametrize("variant", [0, 5, 10])
def test_more_batches_than_one_scan_group_holds(cof_mod, oracle_mod, variant, monkeypatch):
    # ~300 batches (2 chunks each): more batch segments than a scan group
    # stages, as with chunks_per_search 64 (the CLI's C) on a large genome
    monkeypatch.setenv("COF_SCAN_VARIANT", str(variant))
    rng = random.Random(31)
    _, records = randgen.random_genome(rng, 3, 12000, 16000)
    n_pat = PAIR_VARIANTS.get(variant, 3)
    pats = ["".join(rng.choice("ACGT") for _ in range(20)) + "NNN" for _ in range(n_pat)]
    for p in pats:
        randgen.plant_sites(rng, records, p, "N" * 21 + "RG", 10, 2)
    chunks = randgen.chunk_records(rng, records, 160)
    assert len(chunks) > 250
    g, o = _both(cof_mod, oracle_mod, chunks)
    text, n = g.search("N" * 21 + "RG", pats, 4, chunks_per_search=2)
    ref, nref = o.search("N" * 21 + "RG", pats, 4, chunks_per_search=2)
    assert _rows(text) == _rows(ref) and n == nref > 0
    assert g.tuning()["variant"] == variant


@pytest.mark.parametrize("shape", ["nrg", "tttn", "nrg40"])
@pytest.mark.parametrize("cps", [16384, 3])
def test_sliced_scan_equals_one_pass(cof_mod, oracle_mod, monkeypatch, shape, cps):
    # one request on a genome scanned in slices of pattern starts (forced on a
    # small genome by COF_SLICE_NT), each slice's text copied out while the
    # next one scans: rows sort by position first, so the text equals the
    # one-pass text byte for byte, and a two-request batch (one pass) gives
    # the same text; the rows equal the oracle's.  cps = 3 puts many batch
    # heads (overlapping starts) across the slice cuts; the 40-cell pattern
    # has a window shift above 32 on one strand.
    rng = random.Random(1234 + cps + len(shape))
    _, records = randgen.random_genome(rng, 3, 30000, 60000)
    guide = lambda n: "".join(rng.choice("ACGT") for _ in range(n))
    if shape == "nrg":
        filt, pats, mm = "N" * 21 + "RG", [guide(20) + "NNN" for _ in range(3)], 5
    elif shape == "tttn":
        filt, pats, mm = "TTTN" + "N" * 25, ["NNNN" + guide(25) for _ in range(3)], 6
    else:
        filt, pats, mm = "N" * 38 + "RG", [guide(37) + "NNN" for _ in range(2)], 6
    for p in pats:
        randgen.plant_sites(rng, records, p, filt, 12, min(mm, 4))
    g, o = _both(cof_mod, oracle_mod, randgen.chunk_records(rng, records, 3000))
    monkeypatch.delenv("COF_SLICE_NT", raising=False)
    one, n1 = g.search(filt, pats, mm, chunks_per_search=cps)
    assert g.tuning()["slices"] == 0
    monkeypatch.setenv("COF_SLICE_NT", "5000")
    sliced, n2 = g.search(filt, pats, mm, chunks_per_search=cps)
    assert g.tuning()["slices"] > 10
    assert sliced == one and n2 == n1
    req = dict(search_filter=filt, patterns=pats, max_mismatches=mm, chunks_per_search=cps)
    other = dict(req, patterns=pats[:1], max_mismatches=2)
    (bt, bn), _ = g.search_batch([req, other])
    assert bt == one and bn == n1
    ref, nref = o.search(filt, pats, mm, chunks_per_search=cps)
    assert n1 == nref > 0 and _rows(one) == _rows(ref)


def test_sliced_result_buffer_grows(cof_mod, oracle_mod, monkeypatch):
    # one row in the first slices and thousands in the last: the page-locked
    # result buffer, sized from the first slices' rate, has to grow while
    # copies are in flight and keep the text already copied; a second call
    # starts from the last result's size
    rng = random.Random(5)
    site = "".join(rng.choice("ACGT") for _ in range(20)) + "AGG"
    pattern = site[:20] + "NNN"
    head = randgen.random_seq(rng, 60000, n_rate=0, iupac_rate=0)
    head = head[:1000] + site + head[1000 + len(site):]
    tail = "".join(site + "".join(rng.choice("ACGT") for _ in range(7)) for _ in range(20000))
    records = [head, randgen.random_seq(rng, 40000, n_rate=0, iupac_rate=0), tail]
    g, o = _both(cof_mod, oracle_mod, randgen.chunk_records(rng, records, 60000))
    monkeypatch.setenv("COF_SLICE_NT", "20000")
    text, n = g.search("N" * 21 + "RG", [pattern], 2)
    assert g.tuning()["slices"] > 20
    assert len(text) > (1 << 20) + 2 * 35 * 75  # beyond the first estimate
    again, n2 = g.search("N" * 21 + "RG", [pattern], 2)
    assert again == text and n2 == n
    monkeypatch.delenv("COF_SLICE_NT")
    one, n1 = g.search("N" * 21 + "RG", [pattern], 2)
    assert one == text and n1 == n
    ref, nref = o.search("N" * 21 + "RG", [pattern], 2)
    assert nref == n > 19000 and _rows(ref) == _rows(text)
