"""CPU tests of the C ABI: the library loads, exports every symbol that
include/cof.h declares, validates requests, loads genomes on the host exactly
like the oracle, and fails loudly (an error status, no fallback) when no GPU
is usable."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    with open(os.path.join(ROOT, "include", "cof.h")) as f:
        src = f.read()
    return sorted(set(re.findall(r"COF_API\s+[\w\s\*]+?\b(cof_\w+)\s*\(", src)))


def test_exports_every_declared_symbol(cof_mod):
    lib = cof_mod.load_library()
    names = _declared()
    assert len(names) >= 13
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(cof_mod.EXPORTS)
    assert lib.cof_abi_version() == 2


def test_nm_dynamic_symbols(cof_mod):
    out = subprocess.run(["nm", "-D", "--defined-only", cof_mod.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    assert set(_declared()) <= exported
    # no C++ internals leak through the boundary
    assert not [s for s in exported if s.startswith("_Z")]


def test_host_loader_matches_oracle(cof_mod, oracle_mod, golden):
    for name in ("upstream1000.fa", "upstream1000.2bit"):
        path = os.path.join(golden, name)
        g = cof_mod.Genome(path)
        o = oracle_mod.OracleGenome(path)
        assert g.n_chunks == o.n_chunks == 13
        assert g.n_nucl == o.n_nucl == 12507


def test_record_names(cof_mod, oracle_mod, golden):
    # cof_match.record indexes the genome's record names (Match.chr_name)
    for name in ("upstream1000.fa", "upstream1000.2bit"):
        path = os.path.join(golden, name)
        g = cof_mod.Genome(path)
        want = []
        for nm, _d, s, _e in oracle_mod.OracleGenome(path).chunks():
            if s == 0:
                want.append(nm)
        assert g.n_records == len(want) > 1
        assert [g.record_name(i) for i in range(g.n_records)] == want
        assert g.record_name(g.n_records) is None


def test_fasta_index_matches_oracle(cof_mod, oracle_mod, tmp_path):
    # a FASTA file loaded into an empty genome is only indexed on the host
    # (all threads measure lines, one pass decides the chunks); the chunk
    # table must be the oracle reader's
    import random
    import randgen
    for final_newline in (True, False):
        fa = tmp_path / f"g{final_newline}.fa"
        randgen.write_messy_fasta(random.Random(7), fa, final_newline)
        g = cof_mod.Genome(str(fa))
        o = oracle_mod.OracleGenome(str(fa))
        assert g.n_chunks == o.n_chunks > 8
        assert g.n_nucl == o.n_nucl


def test_fasta_index_errors(cof_mod, tmp_path):
    for text in (">\nACGT\n", ">a\n" + "A" * 65537 + "\n"):
        p = tmp_path / "bad.fa"
        p.write_text(text)
        with pytest.raises(cof_mod.CofError) as e:
            cof_mod.Genome(str(p))
        assert e.value.code == cof_mod.COF_E_BADINPUT


def test_genome_freed_in_forked_child(cof_mod):
    # a genome starts a thread that creates the CUDA context; a child forked
    # while the genome exists holds a copy of it but not the thread, and
    # freeing it there must neither wait on that thread nor fail
    g = cof_mod.Genome()
    pid = os.fork()
    if pid == 0:  # child
        code = 1
        try:
            g.close()
            code = 0
        finally:
            os._exit(code)
    _, status = os.waitpid(pid, 0)
    assert os.WIFEXITED(status) and os.WEXITSTATUS(status) == 0
    g.close()


def test_bad_requests_rejected(cof_mod, golden):
    g = cof_mod.Genome(os.path.join(golden, "upstream1000.fa"))
    with pytest.raises(cof_mod.CofError) as e:
        g.search("NNNN", ["ACGTA"], 1)  # length mismatch
    assert e.value.code == cof_mod.COF_E_BADINPUT
    with pytest.raises(cof_mod.CofError) as e:
        g.search("NNXN", ["ACGT"], 1)  # not a mixed-base filter
    assert e.value.code == cof_mod.COF_E_BADINPUT
    with pytest.raises(cof_mod.CofError) as e:
        g.search("NNNN", ["ACGT"], 4)  # mm >= pattern length
    assert e.value.code == cof_mod.COF_E_BADINPUT
    with pytest.raises(cof_mod.CofError) as e:
        g.search("N" * 65, ["A" * 65], 3)  # above 64 cells
    assert e.value.code == cof_mod.COF_E_UNSUPPORTED
    with pytest.raises(cof_mod.CofError) as e:
        g.search("N" * 65, ["A" * 65], 3, 1, 1)  # bulges: at most 64 cells
    assert e.value.code == cof_mod.COF_E_UNSUPPORTED
    with pytest.raises(cof_mod.CofError) as e:
        g.search("N" * 65, ["A" * 65], 3, raw=True)  # raw matches: at most 64 cells
    assert e.value.code == cof_mod.COF_E_UNSUPPORTED
    with pytest.raises(cof_mod.CofError) as e:
        g.search("N" * 40, ["A" * 40], 3, 9, 1)  # more than 8 DNA bulges
    assert e.value.code == cof_mod.COF_E_UNSUPPORTED


def test_stream_argument_errors(cof_mod, golden):
    # cof_search_stream rejects a null genome or sink, an unknown stream
    # flag and a bad request before any device work (no GPU needed); the
    # sink is never called
    import ctypes
    lib = cof_mod.load_library()
    g = cof_mod.Genome(os.path.join(golden, "upstream1000.fa"))
    good = dict(search_filter="N" * 24, patterns=["CCGTGGTTCAACATTTGCTTAGCA"], max_mismatches=3)
    calls = []
    sink = cof_mod._SINK(lambda _u, _p: calls.append(1) or 0)
    reqs, _keep = g.prepare([good])
    n = (ctypes.c_uint64 * 1)()
    assert lib.cof_search_stream(None, reqs, 1, 0, sink, None, n) == cof_mod.COF_E_BADINPUT
    assert lib.cof_search_stream(g._h, reqs, 1, 0, cof_mod._SINK(), None, n) == cof_mod.COF_E_BADINPUT
    assert lib.cof_search_stream(g._h, None, 1, 0, sink, None, n) == cof_mod.COF_E_BADINPUT
    assert lib.cof_search_stream(g._h, reqs, 1, 0x80, sink, None, n) == cof_mod.COF_E_BADINPUT
    assert b"stream flag" in lib.cof_last_error()
    with pytest.raises(cof_mod.CofError) as e:
        g.search_stream([dict(good, search_filter="NNNN")], lambda *a: 0)
    assert e.value.code == cof_mod.COF_E_BADINPUT
    assert calls == []
    # the record-name calls answer for a null genome too
    assert lib.cof_genome_n_records(None) == 0
    assert lib.cof_genome_record_name(None, 0) is None
    assert lib.cof_genome_record_name(g._h, g.n_records) is None
    g.close()


def test_bad_genome_files(cof_mod, tmp_path):
    p = tmp_path / "bad.fa"
    p.write_text("ACGT\n>x\nACGT\n")  # sequence before the first header
    g = cof_mod.Genome()
    with pytest.raises(cof_mod.CofError) as e:
        g.load(str(p))
    assert e.value.code == cof_mod.COF_E_BADINPUT
    p2 = tmp_path / "bad.2bit"
    p2.write_bytes(b"\x00\x01\x02\x03junk")
    with pytest.raises(cof_mod.CofError):
        cof_mod.Genome(str(p2))
    with pytest.raises(cof_mod.CofError) as e:
        cof_mod.Genome(str(tmp_path / "missing.fa"))
    assert e.value.code == cof_mod.COF_E_IO


def test_chunk_order_enforced(cof_mod):
    g = cof_mod.Genome()
    g.add_chunk("a", b"\x44", 0, 2)
    with pytest.raises(cof_mod.CofError):
        g.add_chunk("a", b"\x44", 5, 7)  # search.rs:1396-1399


def _gpu_usable():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_gpu_usable(), reason="checks the no-GPU failure path")
def test_no_gpu_fails_loudly(cof_mod, golden):
    g = cof_mod.Genome(os.path.join(golden, "upstream1000.fa"))
    with pytest.raises(cof_mod.CofError) as e:
        g.search("N" * 24, ["CCGTGGTTCAACATTTGCTTAGCA"], 3)
    assert e.value.code in (cof_mod.COF_E_CUDA, cof_mod.COF_E_OOM)


def test_server_argument_errors(cof_mod, golden):
    # with a memory budget given, a server is created without touching the
    # device; a bad request is refused at submit, an unknown ticket at wait
    import ctypes
    lib = cof_mod.load_library()
    g = cof_mod.Genome(os.path.join(golden, "upstream1000.fa"))
    h = ctypes.c_void_p()
    assert lib.cof_server_create(None, None, ctypes.byref(h)) == cof_mod.COF_E_BADINPUT
    srv = cof_mod.Server(g, memory_budget_bytes=1 << 30, ring_slices=3)
    with pytest.raises(cof_mod.CofError) as e:
        srv.submit("NNNN", ["ACGTA"], 1)
    assert e.value.code == cof_mod.COF_E_BADINPUT
    with pytest.raises(cof_mod.CofError) as e:
        srv.wait(12345)
    assert e.value.code == cof_mod.COF_E_BADINPUT
    assert srv.stats()["queued"] == 0
    if not _gpu_usable():
        # no GPU: the request completes with the CUDA error, it does not hang
        t = srv.submit("N" * 24, ["CCGTGGTTCAACATTTGCTTAGCA"], 3)
        with pytest.raises(cof_mod.CofError) as e:
            srv.wait(t, timeout_ms=120000)
        assert e.value.code in (cof_mod.COF_E_CUDA, cof_mod.COF_E_OOM)
    srv.close()
    g.close()


@pytest.mark.skipif(_gpu_usable(), reason="passes a placeholder device address; never run with a GPU")
def test_noalloc_argument_checks(cof_mod):
    # cof_search_seq_noalloc checks its arguments before any CUDA call.  The
    # device buffers here are a placeholder address, which every case below
    # rejects before it could be used (and no GPU is present)
    import ctypes
    lib = cof_mod.load_library()
    fake = 1 << 20  # 16-byte aligned
    n_rows = ctypes.c_uint32(0)
    pats2 = [b"ACGTACGTACGTNNN", b"NNNACGTACGTACGT"]

    def call(seq=fake, n_nucl=8000, filt=b"N" * 15, pats=pats2, npat=None, mm=2, rows=fake,
             cap=10):
        arr = (ctypes.c_char_p * len(pats))(*pats)
        rc = lib.cof_search_seq_noalloc(seq, n_nucl, filt, arr, len(pats) if npat is None else npat,
                                        mm, rows, cap, ctypes.byref(n_rows), None)
        return rc, lib.cof_last_error()

    bad, uns = cof_mod.COF_E_BADINPUT, cof_mod.COF_E_UNSUPPORTED
    assert call(seq=None)[0] == bad
    assert call(rows=None)[0] == bad  # rows_cap > 0 needs a row buffer
    assert call(seq=fake + 4) == (bad, b"d_bit4 must be 16-byte aligned")
    assert call(filt=b"")[0] == uns
    assert call(filt=b"N" * 33, pats=[b"A" * 33, b"T" * 33])[0] == uns
    assert call(pats=pats2 * 257)[0] == uns and b"n_patterns" in call(pats=pats2 * 257)[1]
    assert call(npat=0)[0] == uns
    rc, msg = call(pats=pats2 + [pats2[0]])
    assert rc == bad and b"even" in msg
    assert call(n_nucl=1 << 31)[0] == uns
    assert call(mm=15)[0] == bad
    assert call(filt=b"N" * 14 + b"X")[0] == bad
    assert call(pats=[b"ACGT", b"ACGT"])[0] == bad  # length differs from the filter
    assert call(pats=[b"ACGTACGTACGTNN!", pats2[1]])[0] == bad


def test_cli_input_errors(cof_mod, tmp_path):
    cli = os.path.join(os.path.dirname(cof_mod.LIB_PATH), "cof-offinder")
    cases = {
        "x.fa\nNNNN\nACGT\n": "Pattern line must have",
        "x.fa\nNNNN\nACGT 1\nACG 1\n": "same length",
        "x.fa\nNNNN\nACGT 1\nACGT 2\n": "all mismatches",
        "x.fa\nNNNN 1\nACGT 1\n": "2nd line must be",
        "x.fa\nNNNN\n": "at least 1 pattern",
        "x.fa\nNNNN\nAXGT 1\n": "mixed base",
    }
    for text, msg in cases.items():
        p = tmp_path / "in.txt"
        p.write_text(text)
        r = subprocess.run([cli, str(p), "G", "-"], capture_output=True, text=True)
        assert r.returncode != 0 and msg in r.stderr, (text, r.stderr)
    r = subprocess.run([cli, str(p), "X", "-"], capture_output=True, text=True)
    assert r.returncode != 0 and "C|G|A" in r.stderr
