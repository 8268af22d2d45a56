"""GPU tests of cof_search_seq_noalloc, the entry point for callers that
cannot allocate device memory: an application whose own pool allocator owns
the GPU's memory (an allocation from this library would bypass it), or a
serving loop whose request path must not allocate because an allocation can
synchronise the whole device.

Its rows must be exactly the rows of the oracle (the CPU restatement of the
reference's search and writer) and of cof_search for the same single-record
genome, on two calls in a row: the fixed scratch array keeps the previous
call's contents and each call must reset what it needs.  A call must leave
the device's free memory unchanged.

The buffers below are allocated by the test (the caller) before anything is
measured; the entry point itself allocates nothing.  This file sorts last so
that a run stopping at its first failure has run every other test first."""
import ctypes
import gc
import random

import pytest

import bruteforce
import randgen

pytestmark = pytest.mark.gpu


def _pack(seq):
    b4 = [randgen.B4[c] for c in seq]
    if len(b4) % 2:
        b4.append(0)
    return bytes(b4[i] | (b4[i + 1] << 4) for i in range(0, len(b4), 2))


def _chunks(seq, name="seq1"):
    data = _pack(seq)
    for s in range(0, len(seq), 65536):
        e = min(s + 65536, len(seq))
        yield name, data[s // 2:(e + 1) // 2], s, e


def _genome(cof_mod, seq):
    g = cof_mod.Genome()
    for c in _chunks(seq):
        g.add_chunk(*c)
    return g


def _as_triples(text, user, pam_len):
    """Writer rows -> the entry point's (scan start, pattern index, mismatches)."""
    n_user = len(user)
    up = [u.upper() for u in user]
    out = set()
    for row in text.splitlines():
        c = row.split("\t")
        p = up.index(c[1])
        pos = int(c[4])
        if c[5] == "+":
            out.add((pos, p, int(c[6])))
        else:
            out.add((pos - max(pam_len - 1, 0), n_user + p, int(c[6])))
    return out


def _call(cof_mod, rows, seq_dev, n_nucl, filt, full, mm, cap):
    """One call into caller-owned buffers (rows holds 3 * cap int32)."""
    lib = cof_mod.load_library()
    arr = (ctypes.c_char_p * len(full))(*[p.encode() for p in full])
    n_rows = ctypes.c_uint32(0)
    rc = lib.cof_search_seq_noalloc(seq_dev.data_ptr(), n_nucl, filt.encode(), arr, len(full),
                                    mm, rows.data_ptr(), cap, ctypes.byref(n_rows), None)
    return rc, n_rows.value


def _workload(shape):
    rng = random.Random(4242)
    if shape == "nrg":
        seq = randgen.random_seq(rng, 300_001)
        filt, mm = "N" * 21 + "RG", 4
        user = ["".join(rng.choice("ACGT") for _ in range(20)) + "NNN" for _ in range(5)]
        recs = [seq]
        for u in user:
            randgen.plant_sites(rng, recs, u, filt, 30, 2)
        seq = recs[0]
    else:
        # permissive: ~1.5 M scan candidates, more than the fixed candidate
        # list holds, so the entry point has to split the range
        seq = randgen.random_seq(rng, 2_000_000, n_rate=0.001, iupac_rate=0.001)
        filt, mm = "N" * 12, 8
        user = ["".join(rng.choice("ACGT") for _ in range(12))]
    return seq, filt, mm, user


@pytest.mark.parametrize("shape", ["nrg", "dense"])
def test_noalloc_matches_oracle_and_cof_search(cof_mod, oracle_mod, shape):
    torch = pytest.importorskip("torch")
    seq, filt, mm, user = _workload(shape)
    pam_len = len(user[0]) - len(user[0].rstrip("N"))
    o = oracle_mod.OracleGenome()
    for c in _chunks(seq):
        o.add_chunk(*c)
    ref, nref = o.search(filt, user, mm)
    o.close()
    want = _as_triples(ref, user, pam_len)
    assert len(want) == nref > 0
    g = _genome(cof_mod, seq)
    text, n = g.search(filt, user, mm)
    g.close()
    assert _as_triples(text, user, pam_len) == want and n == nref

    full = user + [bruteforce.revcomp(u) for u in user]
    cap = nref + 16
    seq_dev = torch.frombuffer(bytearray(_pack(seq)), dtype=torch.uint8).cuda()
    bufs = [torch.full((3 * cap,), -1, dtype=torch.int32, device="cuda") for _ in range(3)]
    # genomes of earlier tests that the garbage collector frees in the middle
    # of the measurement would raise the free memory: collect them first and
    # keep the collector off while the calls are measured
    gc.collect()
    torch.cuda.synchronize()
    free, results = [], []
    gc.disable()
    try:
        for rows in bufs:
            rc, n_rows = _call(cof_mod, rows, seq_dev, len(seq), filt, full, mm, cap)
            torch.cuda.synchronize()
            free.append(torch.cuda.mem_get_info()[0])
            results.append((rc, n_rows, rows))
    finally:
        gc.enable()
    for rc, n_rows, rows in results:
        assert rc == 0, cof_mod.load_library().cof_last_error().decode()
        assert n_rows == nref
        got = {tuple(x) for x in rows[:3 * n_rows].view(-1, 3).cpu().tolist()}
        assert got == want
    # measured after each call: the first call may load the module (the
    # scratch array comes with it); no call after it changes free memory
    assert free[0] == free[1] == free[2], free


def test_noalloc_rows_cap_overflow(cof_mod, oracle_mod):
    torch = pytest.importorskip("torch")
    seq, filt, mm, user = _workload("nrg")
    pam_len = len(user[0]) - len(user[0].rstrip("N"))
    o = oracle_mod.OracleGenome()
    for c in _chunks(seq):
        o.add_chunk(*c)
    ref, nref = o.search(filt, user, mm)
    o.close()
    want = _as_triples(ref, user, pam_len)
    full = user + [bruteforce.revcomp(u) for u in user]
    cap = nref // 3
    seq_dev = torch.frombuffer(bytearray(_pack(seq)), dtype=torch.uint8).cuda()
    # one guard row past rows_cap must stay untouched
    rows = torch.full((3 * (cap + 1),), -1, dtype=torch.int32, device="cuda")
    for _ in range(2):
        rc, n_rows = _call(cof_mod, rows, seq_dev, len(seq), filt, full, mm, cap)
        assert rc == cof_mod.COF_E_UNSUPPORTED
        assert b"rows_cap" in cof_mod.load_library().cof_last_error()
        assert n_rows == nref  # the true count comes back
        got = [tuple(x) for x in rows[:3 * cap].view(-1, 3).cpu().tolist()]
        assert len(set(got)) == cap and set(got) <= want
        assert rows[3 * cap:].cpu().tolist() == [-1, -1, -1]


def test_noalloc_limits(cof_mod):
    torch = pytest.importorskip("torch")
    lib = cof_mod.load_library()
    seq_dev = torch.zeros(4096, dtype=torch.uint8, device="cuda")
    rows = torch.zeros(30, dtype=torch.int32, device="cuda")
    n_rows = ctypes.c_uint32(0)
    pats = ["ACGTACGTACGTNNN"] * 514
    arr = (ctypes.c_char_p * len(pats))(*[p.encode() for p in pats])
    rc = lib.cof_search_seq_noalloc(seq_dev.data_ptr(), 8000, b"N" * 15, arr, len(pats), 2,
                                    rows.data_ptr(), 10, ctypes.byref(n_rows), None)
    assert rc == cof_mod.COF_E_UNSUPPORTED and b"n_patterns" in lib.cof_last_error()
    # an odd count cannot be split into forward patterns and their reverse
    # complements
    rc = lib.cof_search_seq_noalloc(seq_dev.data_ptr(), 8000, b"N" * 15, arr, 3, 2,
                                    rows.data_ptr(), 10, ctypes.byref(n_rows), None)
    assert rc == cof_mod.COF_E_BADINPUT and b"even" in lib.cof_last_error()
    rc = lib.cof_search_seq_noalloc(seq_dev.data_ptr() + 1, 8000, b"N" * 15, arr, 2, 2,
                                    rows.data_ptr(), 10, ctypes.byref(n_rows), None)
    assert rc == cof_mod.COF_E_BADINPUT and b"aligned" in lib.cof_last_error()
    long_pats = (ctypes.c_char_p * 2)(b"A" * 40, b"T" * 40)
    rc = lib.cof_search_seq_noalloc(seq_dev.data_ptr(), 8000, b"N" * 40, long_pats, 2, 2,
                                    rows.data_ptr(), 10, ctypes.byref(n_rows), None)
    assert rc == cof_mod.COF_E_UNSUPPORTED
