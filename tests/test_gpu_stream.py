"""GPU tests of the streamed results (cof_search_stream), the dest channel of
search() (search.rs:1490-1500): the pieces a request receives, in order, are
its cof_search text -- byte for byte on the popcount path (one pass or genome
slices), the same rows on the bulge path (candidate chunks) -- and equal the
oracle's rows; the optional match records describe exactly the lines they
point at; a sink that stops the search gets COF_E_CANCELLED and leaves the
genome usable."""
import collections
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


def _collect(g, reqs, matches=False):
    """{request: [(text, n_rows, records)]} in arrival order, and the counts."""
    got = collections.defaultdict(list)

    def on_piece(r, text, n, recs):
        got[r].append((text.decode("latin-1"), n, recs))
        return 0

    counts = g.search_stream(reqs, on_piece, matches=matches)
    return got, counts


def _pam_len(pattern):
    return len(pattern) - len(pattern.rstrip("Nn"))


def _check_records(g, pieces, req):
    """Every record names its line: record name, position (the writer's
    '-' strand shift), strand, mismatches, bulge sizes and rna string."""
    user = [p.upper() for p in req["patterns"]]
    pam_len = _pam_len(req["patterns"][0])
    raw = req.get("raw", False)
    n = 0
    for text, n_rows, recs in pieces:
        assert recs is not None and len(recs) == n_rows
        starts = [0] + [i + 1 for i, ch in enumerate(text) if ch == "\n"][:-1]
        assert [r[1] for r in recs] == starts  # text order, one record per line
        for (pos, off, rec, pidx, mm, db, rb, fwd), start in zip(recs, starts):
            c = text[start:text.index("\n", start)].split("\t")
            if raw:
                assert c[0] == g.record_name(rec) and int(c[1]) == pos
                assert (int(c[2]), c[3], int(c[4]), int(c[5]), int(c[6])) == (
                    pidx, "+" if fwd else "-", mm, db, rb)
                continue
            assert c[3] == g.record_name(rec)
            a = max(pam_len - 1, 0)
            shift = 0 if fwd else (a - db if a > db else 0)
            assert int(c[4]) == pos + shift
            assert c[5] == ("+" if fwd else "-") and int(c[6]) == mm
            assert int(c[7]) == db + rb
            # the crRNA column prints the user's pattern on both strands
            assert c[1].replace("-", "").upper() == user[pidx if fwd else pidx - len(user)]
        n += n_rows
    return n


def test_stream_equals_search_batch(cof_mod, oracle_mod):
    rng = random.Random(31)
    _, records = randgen.random_genome(rng, 3, 4000, 9000)
    reqs = []
    for shape in (0, 1, 2, 0):
        filt, mk, mm = randgen.REQUEST_SHAPES[shape]
        pats = [mk("".join(rng.choice("ACGT") for _ in range(25))) for _ in range(2)]
        for p in pats:
            randgen.plant_sites(rng, records, p, filt, 6, 2)
        reqs.append(dict(search_filter=filt, patterns=pats, max_mismatches=mm))
    reqs.append(dict(reqs[0], max_dna_bulges=1, max_rna_bulges=1, max_mismatches=3))
    g, o = _both(cof_mod, oracle_mod, randgen.chunk_records(rng, records, 900))
    whole = g.search_batch(reqs)
    got, counts = _collect(g, reqs)
    for i, (text, n) in enumerate(whole):
        pieces = got.get(i, [])
        assert counts[i] == n == sum(p[1] for p in pieces)
        joined = "".join(p[0] for p in pieces)
        if i < 4:
            assert joined == text  # popcount: byte for byte
        else:
            assert _rows(joined) == _rows(text)
        r = reqs[i]
        ref, nref = o.search(r["search_filter"], r["patterns"], r["max_mismatches"],
                             r.get("max_dna_bulges", 0), r.get("max_rna_bulges", 0))
        assert nref == n and _rows(ref) == _rows(joined)


def test_stream_sliced_popcount(cof_mod, oracle_mod, monkeypatch):
    rng = random.Random(77)
    _, records = randgen.random_genome(rng, 3, 30000, 60000)
    pats = ["".join(rng.choice("ACGT") for _ in range(20)) + "NNN" for _ in range(3)]
    filt = "N" * 21 + "RG"
    for p in pats:
        randgen.plant_sites(rng, records, p, filt, 12, 4)
    g, o = _both(cof_mod, oracle_mod, randgen.chunk_records(rng, records, 3000))
    req = dict(search_filter=filt, patterns=pats, max_mismatches=5)
    monkeypatch.setenv("COF_SLICE_NT", "5000")
    text, n = g.search(filt, pats, 5)
    got, counts = _collect(g, [req], matches=True)
    assert g.tuning()["slices"] > 10
    pieces = got[0]
    assert len(pieces) > 3  # one per slice with rows
    assert "".join(p[0] for p in pieces) == text and counts[0] == n
    assert _check_records(g, pieces, req) == n
    ref, nref = o.search(filt, pats, 5)
    assert nref == n and _rows(ref) == _rows(text)


@pytest.mark.parametrize("raw", [False, True])
def test_stream_bulge_chunks_with_records(cof_mod, oracle_mod, monkeypatch, raw):
    import synth
    cfg = synth.config_bulge(seed=6, scale=0.0002, n_guides=6, planted=8)
    g = cof_mod.Genome()
    cfg["genome"].load_into(g)
    req = dict(search_filter=cfg["filter"], patterns=cfg["patterns"],
               max_mismatches=cfg["max_mismatches"], max_dna_bulges=cfg["max_dna_bulges"],
               max_rna_bulges=cfg["max_rna_bulges"], raw=raw)
    text, n = g.search_batch([req])[0]
    monkeypatch.setenv("COF_BULGE_CHUNK", "7")
    got, counts = _collect(g, [req], matches=True)
    pieces = got[0]
    assert len(pieces) > 3 and counts[0] == n
    assert _rows("".join(p[0] for p in pieces)) == _rows(text)
    assert _check_records(g, pieces, req) == n
    if not raw:
        o = oracle_mod.OracleGenome()
        for c in cfg["genome"].chunks():
            o.add_chunk(*c)
        ref, nref = o.search(req["search_filter"], req["patterns"], req["max_mismatches"],
                             req["max_dna_bulges"], req["max_rna_bulges"])
        assert nref == n and _rows(ref) == _rows(text)


def test_stream_raw_popcount_is_one_piece(cof_mod, oracle_mod, golden):
    import os
    g = cof_mod.Genome(os.path.join(golden, "upstream1000.fa"))
    pats = ["CCGTGGTTCAACATTTGCTTAGCA", "GATGTTGGTAAGTGGGATATGGCA"]
    req = dict(search_filter="N" * 24, patterns=pats, max_mismatches=11, raw=True)
    text, n = g.search_batch([req])[0]
    got, counts = _collect(g, [req], matches=True)
    assert len(got[0]) == 1 and got[0][0][0] == text and counts[0] == n == 117
    assert got[0][0][2] is None  # the popcount raw stream carries no records


def test_stream_cancel(cof_mod, golden):
    import os
    g = cof_mod.Genome(os.path.join(golden, "upstream1000.fa"))
    pats = ["CCGTGGTTCAACATTTGCTTAGCA", "GATGTTGGTAAGTGGGATATGGCA"]
    req = dict(search_filter="N" * 24, patterns=pats, max_mismatches=11)
    seen = []
    with pytest.raises(cof_mod.CofError) as e:
        g.search_stream([req], lambda *a: seen.append(a) or 1)
    assert e.value.code == cof_mod.COF_E_CANCELLED and len(seen) == 1
    text, n = g.search("N" * 24, pats, 11)
    assert n == 117  # the genome is still usable
