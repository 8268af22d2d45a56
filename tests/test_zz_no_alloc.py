"""GPU test of cof_search_seq_noalloc, the entry point for callers that cannot
allocate device memory (their own pool owns it, or their request path must
not allocate): it must give exactly the rows cof_search gives for the same
single-record genome, on two calls in a row (the fixed scratch array keeps
the previous call's contents and must be reset by each call).

The buffers below are allocated by the test (the caller); the entry point
itself allocates nothing."""
import ctypes
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


def _genome(cof_mod, seq, name="seq1"):
    g = cof_mod.Genome()
    data = _pack(seq)
    for s in range(0, len(seq), 65536):
        e = min(s + 65536, len(seq))
        g.add_chunk(name, data[s // 2:(e + 1) // 2], s, e)
    return g


def _expected(text, user, pam_len):
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


def _call(cof_mod, torch, seq_dev, n_nucl, filt, full, mm, cap):
    lib = cof_mod.load_library()
    rows = torch.full((3 * cap,), -1, dtype=torch.int32, device="cuda")
    arr = (ctypes.c_char_p * len(full))(*[p.encode() for p in full])
    n_rows = ctypes.c_uint32(0)
    torch.cuda.synchronize()
    rc = lib.cof_search_seq_noalloc(seq_dev.data_ptr(), n_nucl, filt.encode(), arr, len(full),
                                    mm, rows.data_ptr(), cap, ctypes.byref(n_rows), None)
    assert rc == 0, lib.cof_last_error().decode()
    r = rows[:3 * n_rows.value].view(-1, 3).cpu().tolist()
    return {tuple(x) for x in r}, n_rows.value


@pytest.mark.parametrize("shape", ["nrg", "dense"])
def test_noalloc_matches_cof_search(cof_mod, shape):
    torch = pytest.importorskip("torch")
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
    pam_len = len(user[0]) - len(user[0].rstrip("N"))
    g = _genome(cof_mod, seq)
    text, n = g.search(filt, user, mm)
    want = _expected(text, user, pam_len)
    assert len(want) == n > 0
    full = user + [bruteforce.revcomp(u) for u in user]
    seq_dev = torch.frombuffer(bytearray(_pack(seq)), dtype=torch.uint8).cuda()
    for _ in range(2):
        got, n_rows = _call(cof_mod, torch, seq_dev, len(seq), filt, full, mm, n + 16)
        assert n_rows == n
        assert got == want


def test_noalloc_limits(cof_mod):
    torch = pytest.importorskip("torch")
    lib = cof_mod.load_library()
    seq_dev = torch.zeros(4096, dtype=torch.uint8, device="cuda")
    rows = torch.zeros(30, dtype=torch.int32, device="cuda")
    n_rows = ctypes.c_uint32(0)
    pats = ["ACGTACGTACGTNNN"] * 513
    arr = (ctypes.c_char_p * len(pats))(*[p.encode() for p in pats])
    rc = lib.cof_search_seq_noalloc(seq_dev.data_ptr(), 8000, b"N" * 15, arr, len(pats), 2,
                                    rows.data_ptr(), 10, ctypes.byref(n_rows), None)
    assert rc == cof_mod.COF_E_UNSUPPORTED and b"n_patterns" in lib.cof_last_error()
    rc = lib.cof_search_seq_noalloc(seq_dev.data_ptr() + 1, 8000, b"N" * 15, arr, 2, 2,
                                    rows.data_ptr(), 10, ctypes.byref(n_rows), None)
    assert rc == cof_mod.COF_E_BADINPUT and b"aligned" in lib.cof_last_error()
    long_pats = (ctypes.c_char_p * 2)(b"A" * 40, b"T" * 40)
    rc = lib.cof_search_seq_noalloc(seq_dev.data_ptr(), 8000, b"N" * 40, long_pats, 2, 2,
                                    rows.data_ptr(), 10, ctypes.byref(n_rows), None)
    assert rc == cof_mod.COF_E_UNSUPPORTED
