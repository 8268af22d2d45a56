"""Parity at the benchmark's sizes through properties that do not need the
oracle to run over the whole input:

* every planted site (synth truth list) is reported, at the position rule of
  main.rs:229-236;
* a sample of rows, re-derived from the genome by an independent check
  (window bytes, lowercase marking, mismatch count, PAM cells, reverse
  strand orientation), is exactly what the writer (main.rs:159-242) prints;
* the row text does not depend on the scan tile shape.

The mixed-PAM batch (NNGRRT + TTTN in one pass) is also compared with the
oracle outright on a scaled-down genome of the same generator."""
import os
import random

import pytest

pytestmark = pytest.mark.gpu

_SET = {"A": "A", "C": "C", "G": "G", "T": "T", "R": "AG", "Y": "CT", "S": "CG", "W": "AT",
        "K": "GT", "M": "AC", "B": "CGT", "D": "AGT", "H": "ACT", "V": "ACG", "N": "ACGT"}
_COMP = {"A": "T", "C": "G", "G": "C", "T": "A", "N": "N"}


def _revcomp(s):
    return "".join(_COMP[c] for c in reversed(s))


def _pam_len(pattern):
    n = 0
    for c in reversed(pattern):
        if c not in "Nn":
            break
        n += 1
    return n


def _check_row(row, gen, rec_of, filt, patterns, pam_len, max_mm):
    import synth
    typ, rna, dna, name, pos, strand, mm, size = row.split("\t")
    pos, mm = int(pos), int(mm)
    assert typ == "X" and size == "0" and mm <= max_mm
    L = len(rna)
    fwd_pats = {p.upper() for p in patterns}
    assert rna in fwd_pats  # reverse-strand rows print the guide orientation
    start = pos if strand == "+" else pos - max(pam_len - 1, 0)
    window = bytes(synth._CHARS[gen.records[rec_of[name]][start:start + L]]).decode()
    if strand == "-":
        window = _revcomp(window)
    assert dna.upper() == window, row
    lower = 0
    for i in range(L):
        if rna[i] == "N":
            assert not dna[i].islower(), row
            continue
        mismatch = window[i] not in _SET[rna[i]]  # genome N never matches a base
        assert dna[i].islower() == mismatch, row
        lower += mismatch
    assert lower == mm, row
    for i, f in enumerate(filt):  # PAM cells: a single base of the filter set
        if f != "N":
            assert window[i] in "ACGT" and window[i] in _SET[f], row


def _found(text):
    out = set()
    for r in text.splitlines():
        f = r.split("\t")
        out.add((f[3], int(f[4]), f[5]))
    return out


def test_full_genome_properties(cof_mod, monkeypatch):
    import synth
    cfg = synth.config_full_genome(seed=2, scale=1.0, n_guides=100)
    gen = cfg["genome"]
    g = cof_mod.Genome()
    gen.load_into(g)
    args = (cfg["filter"], cfg["patterns"], cfg["max_mismatches"])
    monkeypatch.setenv("COF_SCAN_VARIANT", "0")
    text, n = g.search(*args)
    monkeypatch.setenv("COF_SCAN_VARIANT", "5")
    text6, n6 = g.search(*args)
    assert n == n6 > 1_000_000 and text == text6
    rows = text.splitlines()
    assert len(rows) == n
    pam_len = _pam_len(cfg["patterns"][0])
    found = _found(text)
    for rec, pos, strand, _gi, _k, _ln in cfg["truth"]:
        want = pos + (max(pam_len - 1, 0) if strand == "-" else 0)
        assert (gen.names[rec], want, strand) in found
    rec_of = {nm: i for i, nm in enumerate(gen.names)}
    for r in random.Random(0).sample(rows, 3000):
        _check_row(r, gen, rec_of, cfg["filter"], cfg["patterns"], pam_len,
                   cfg["max_mismatches"])
    g.close()


def test_mixed_pam_batch_vs_oracle(cof_mod, oracle_mod):
    import synth
    cfg = synth.config_mixed_pam(seed=3, scale=0.002, n_each=50, planted=3)
    gen = cfg["genome"]
    g = cof_mod.Genome()
    o = oracle_mod.OracleGenome()
    for name, data, s, e in gen.chunks():
        g.add_chunk(name, data, s, e)
        o.add_chunk(name, data, s, e)
    res = g.search_batch(cfg["requests"])
    rec_of = {nm: i for i, nm in enumerate(gen.names)}
    for req, (text, n) in zip(cfg["requests"], res):
        ref, nref = o.search(req["search_filter"], req["patterns"], req["max_mismatches"])
        assert sorted(text.splitlines()) == sorted(ref.splitlines()) and n == nref > 0
        pam_len = _pam_len(req["patterns"][0])
        for r in text.splitlines():
            _check_row(r, gen, rec_of, req["search_filter"], req["patterns"], pam_len,
                       req["max_mismatches"])
    found = _found(res[0][0]) | _found(res[1][0])
    for rec, pos, strand, gi, _k, _ln in cfg["truth"]:
        pats = cfg["requests"][0 if gi < 50 else 1]["patterns"]
        want = pos + (max(_pam_len(pats[0]) - 1, 0) if strand == "-" else 0)
        assert (gen.names[rec], want, strand) in found


def test_full_genome_workload_vs_oracle_at_310Mbp(cof_mod, oracle_mod):
    # the 100-guide workload's generator at a tenth of its size (310 Mbp,
    # 24 records, N runs, 50 planted sites per guide): every row equals the
    # oracle's (the oracle takes seconds here on all host threads)
    import synth
    cfg = synth.config_full_genome(seed=2, scale=0.1, n_guides=100)
    gen = cfg["genome"]
    g = cof_mod.Genome()
    o = oracle_mod.OracleGenome()
    for name, data, s, e in gen.chunks():
        g.add_chunk(name, data, s, e)
        o.add_chunk(name, data, s, e)
    args = (cfg["filter"], cfg["patterns"], cfg["max_mismatches"])
    text, n = g.search(*args)
    ref, nref = o.search(*args)
    assert n == nref > 100_000
    assert sorted(text.splitlines()) == sorted(ref.splitlines())
