"""ctypes binding of _ref/libref_gpu.so, the launcher of the reference's own
CUDA kernels (kernel.cu `find_matches`, kernel_myers.cu `find_matches_myers`)
built unmodified for sm_100a by `make -C oracle ref`.

TEST AND MEASUREMENT INFRASTRUCTURE ONLY: used by tests/ as a second,
independent check of the product's raw match stream and by the reference GPU
timing script (ref_gpu_bar.py).  The product never imports it.

Besides the launches, this module restates the host-side decode of the
kernels' records into search()'s raw Match lines: chunk ownership and the
record-end rule of convert_matches (search.rs:1428-1488) for the popcount
kernel, decode_gpu_enum_match (search.rs:152-206) and convert_matches_myers
(search.rs:1316-1374) for the Myers kernel.
"""
import bisect
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
LIB_PATH = os.path.join(REF_DIR, "libref_gpu.so")
OUT_BUF_SIZE = 4 * 1024 * 1024  # kernel_myers cubins are built with this


def popcount_cubin(L):
    return os.path.join(REF_DIR, f"kernel_popcount_L{L}.cubin")


def myers_cubin(L, pam_len, mm, db, rb):
    return os.path.join(REF_DIR, f"kernel_myers_{L}_P{pam_len}_M{mm}_D{db}_R{rb}.cubin")


def available():
    return os.path.exists(LIB_PATH)


class PMatch(ctypes.Structure):
    _fields_ = [("loc", ctypes.c_uint32), ("pattern_idx", ctypes.c_uint32),
                ("mismatches", ctypes.c_uint32), ("dna_bulge_size", ctypes.c_uint16),
                ("rna_bulge_size", ctypes.c_uint16)]


class MMatch(ctypes.Structure):
    _fields_ = [("chunk_idx", ctypes.c_uint32), ("pattern_idx", ctypes.c_uint32),
                ("ops_packed", ctypes.c_uint64), ("mismatches", ctypes.c_uint32),
                ("dna_bulge_size", ctypes.c_uint16), ("rna_bulge_size", ctypes.c_uint16),
                ("ops_count", ctypes.c_uint32), ("pad", ctypes.c_uint32)]


class Times(ctypes.Structure):
    _fields_ = [("kernel_ms", ctypes.c_double), ("h2d_ms", ctypes.c_double),
                ("d2h_ms", ctypes.c_double), ("host_ms", ctypes.c_double),
                ("wall_ms", ctypes.c_double), ("launches", ctypes.c_uint64),
                ("n_batches", ctypes.c_uint64), ("matches", ctypes.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH)
        vp, sz, u32, u64 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint64
        cp = ctypes.c_char_p
        pp = ctypes.POINTER(ctypes.c_char_p)
        L.refgpu_open.restype = vp
        L.refgpu_open.argtypes = [vp, vp, vp, sz, u32, ctypes.c_int, cp, sz]
        L.refgpu_n_batches.restype = sz
        L.refgpu_n_batches.argtypes = [vp]
        L.refgpu_batch.argtypes = [vp, sz, ctypes.POINTER(sz), ctypes.POINTER(sz),
                                   ctypes.POINTER(ctypes.c_int)]
        L.refgpu_close.argtypes = [vp]
        L.refgpu_popcount_count.restype = ctypes.c_int
        L.refgpu_popcount_count.argtypes = [vp, cp, pp, sz, u32, u64, vp, cp, sz]
        L.refgpu_popcount_run.restype = ctypes.c_int
        L.refgpu_popcount_run.argtypes = [vp, cp, pp, sz, u32, u64, vp, vp, u64, vp,
                                          ctypes.POINTER(Times), cp, sz]
        L.refgpu_myers_run.restype = ctypes.c_int
        L.refgpu_myers_run.argtypes = [vp, cp, cp, pp, sz, sz, u32, vp, u64, vp,
                                       ctypes.POINTER(Times), cp, sz]
        L.refgpu_myers_lines.restype = vp
        L.refgpu_myers_lines.argtypes = [vp, pp, pp, sz, sz, vp, vp, ctypes.POINTER(u64),
                                         ctypes.POINTER(u64)]
        L.refgpu_free.argtypes = [vp]
        _lib = L
    return _lib


class RefGpuError(RuntimeError):
    pass


def _pats(patterns):
    enc = [p.encode() for p in patterns]
    return enc, (ctypes.c_char_p * len(enc))(*enc)


class RefGpu:
    """The reference's device loops over one genome's chunks.  `chunks` is a
    list of (name, bit4 bytes, start, end) as the reader yields them."""

    def __init__(self, chunks, chunks_per_search=0, device=0):
        self.chunks = chunks
        self._bufs = [ctypes.create_string_buffer(bytes(c[1]), max(len(c[1]), 1))
                      for c in chunks]
        n = len(chunks)
        self._ptrs = (ctypes.c_void_p * max(n, 1))(*[ctypes.addressof(b) for b in self._bufs])
        self._start = (ctypes.c_uint64 * max(n, 1))(*[c[2] for c in chunks])
        self._end = (ctypes.c_uint64 * max(n, 1))(*[c[3] for c in chunks])
        err = ctypes.create_string_buffer(512)
        self._h = lib().refgpu_open(self._ptrs, self._start, self._end, n, chunks_per_search,
                                    device, err, 512)
        if not self._h:
            raise RefGpuError(err.value.decode())
        self.batches = []
        for b in range(lib().refgpu_n_batches(self._h)):
            f, m, h = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_int()
            lib().refgpu_batch(self._h, b, ctypes.byref(f), ctypes.byref(m), ctypes.byref(h))
            self.batches.append((f.value, m.value, bool(h.value)))

    def close(self):
        if getattr(self, "_h", None):
            lib().refgpu_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- popcount ---------------------------------------------------------
    def popcount_counts(self, patterns, max_mm, count_cap=1 << 26):
        L = len(patterns[0])
        enc, arr = _pats(patterns)
        counts = (ctypes.c_uint64 * max(len(self.batches), 1))()
        err = ctypes.create_string_buffer(512)
        if lib().refgpu_popcount_count(self._h, popcount_cubin(L).encode(), arr, len(enc),
                                       max_mm, count_cap, counts, err, 512):
            raise RefGpuError(err.value.decode())
        return [counts[i] for i in range(len(self.batches))]

    def popcount(self, patterns, max_mm, counts=None, keep=True):
        """find_matches over every batch; returns (matches per batch, times).
        Matches are (loc, pattern, mm) with loc relative to the batch."""
        if counts is None:
            counts = self.popcount_counts(patterns, max_mm)
        L = len(patterns[0])
        enc, arr = _pats(patterns)
        nb = len(self.batches)
        cnt = (ctypes.c_uint64 * max(nb, 1))(*counts)
        total = sum(counts)
        out = (PMatch * max(total, 1))() if keep else None
        offs = (ctypes.c_uint64 * (nb + 1))()
        t = Times()
        err = ctypes.create_string_buffer(512)
        cap = max(counts) if counts else 0
        if lib().refgpu_popcount_run(self._h, popcount_cubin(L).encode(), arr, len(enc), max_mm,
                                     cap, cnt, out, total if keep else 0, offs, ctypes.byref(t),
                                     err, 512):
            raise RefGpuError(err.value.decode())
        per = []
        if keep:
            raw = np.frombuffer(out, dtype=np.uint32).reshape(-1, 4)[:total]
            for b in range(nb):
                per.append(raw[offs[b]:offs[b + 1], :3].copy())
        return per, t.as_dict()

    # -- Myers ------------------------------------------------------------
    def myers(self, search_filter, patterns, n_fwd, mm, db, rb, keep=True, out_cap=1 << 20):
        L = len(patterns[0])
        pam_len = max(sum(1 for ch in p if ch in "Nn") for p in patterns)
        cub = myers_cubin(L, pam_len, mm, db, rb)
        if not os.path.exists(cub):
            raise RefGpuError(f"no reference Myers cubin for {os.path.basename(cub)}")
        enc, arr = _pats(patterns)
        nb = len(self.batches)
        out = (MMatch * out_cap)() if keep else None
        offs = (ctypes.c_uint64 * (nb + 1))()
        t = Times()
        err = ctypes.create_string_buffer(512)
        if lib().refgpu_myers_run(self._h, cub.encode(), search_filter.encode(), arr, len(enc),
                                  n_fwd, OUT_BUF_SIZE, out, out_cap if keep else 0, offs,
                                  ctypes.byref(t), err, 512):
            raise RefGpuError(err.value.decode())
        per = []
        if keep:
            for b in range(nb):
                per.append([out[i] for i in range(offs[b], offs[b + 1])])
        return per, t.as_dict()

    def myers_text(self, search_filter, patterns, n_fwd, mm, db, rb, out_cap):
        """find_matches_myers over every batch, decoded in C into search()'s
        raw Match lines (refgpu_myers_lines: the decode of myers_raw_lines
        below, for millions of records).  Returns (text, lines, times)."""
        L = len(patterns[0])
        pam_len = max(sum(1 for ch in p if ch in "Nn") for p in patterns)
        cub = myers_cubin(L, pam_len, mm, db, rb)
        if not os.path.exists(cub):
            raise RefGpuError(f"no reference Myers cubin for {os.path.basename(cub)}")
        enc, arr = _pats(patterns)
        nb = len(self.batches)
        out = (MMatch * out_cap)()
        offs = (ctypes.c_uint64 * (nb + 1))()
        t = Times()
        err = ctypes.create_string_buffer(512)
        if lib().refgpu_myers_run(self._h, cub.encode(), search_filter.encode(), arr, len(enc),
                                  n_fwd, OUT_BUF_SIZE, out, out_cap, offs, ctypes.byref(t),
                                  err, 512):
            raise RefGpuError(err.value.decode())
        names = [c[0].encode() for c in self.chunks]
        name_arr = (ctypes.c_char_p * max(len(names), 1))(*names)
        n_text, n_lines = ctypes.c_uint64(), ctypes.c_uint64()
        p = lib().refgpu_myers_lines(self._h, name_arr, arr, len(enc), n_fwd, out, offs,
                                     ctypes.byref(n_text), ctypes.byref(n_lines))
        if not p:
            raise RefGpuError("out of host memory for the decoded lines")
        try:
            text = ctypes.string_at(p, n_text.value).decode("latin-1")
        finally:
            lib().refgpu_free(p)
        return text, n_lines.value, t.as_dict()


# -- host-side decode into search()'s raw Match lines -----------------------
_UP = {"G": 8, "C": 2, "A": 4, "T": 1, "R": 12, "Y": 3, "S": 10, "W": 5, "K": 9, "M": 6,
       "B": 11, "D": 13, "H": 7, "V": 14, "N": 15}
_DEC = {v: c for c, v in _UP.items()}
_DEC[0] = "\0"


def _comp(c):
    pairs = {"A": "T", "T": "A", "C": "G", "G": "C", "R": "Y", "Y": "R", "K": "M", "M": "K",
             "B": "V", "V": "B", "D": "H", "H": "D", "S": "S", "W": "W", "N": "N"}
    u = pairs.get(c.upper())
    if u is None:
        return c
    return u.lower() if c.islower() else u


def _revcomp(s):
    return "".join(_comp(c) for c in reversed(s))


class _BatchView:
    def __init__(self, chunks, first, n):
        self.meta = chunks[first:first + n]
        self.offs = [0]
        parts = []
        for name, data, s, e in self.meta:
            nb = (e - s + 1) // 2
            parts.append(bytes(data[:nb]))
            self.offs.append(self.offs[-1] + nb)
        self.buf = b"".join(parts)

    def nib(self, i):
        if i // 2 >= len(self.buf):
            return 0
        b = self.buf[i // 2]
        return (b >> 4) & 0xF if i & 1 else b & 0xF

    def owner(self, start):
        idx = bisect.bisect_right(self.offs, start // 2) - 1
        return min(idx, len(self.meta) - 1)

    def place(self, start, extent):
        """(name, position) of a window, or None past a record end."""
        idx = self.owner(start)
        name, _d, cs, ce = self.meta[idx]
        pos = cs + (start - self.offs[idx] * 2)
        end_chrom = idx == len(self.meta) - 1 or self.meta[idx + 1][2] == 0
        if end_chrom and pos + extent > ce:
            return None
        return name, pos


def popcount_raw_lines(ref, per_batch, patterns, masked=True):
    """Raw Match lines of the popcount kernel's records (loc, pattern, mm):
    ownership and the record-end drop of convert_matches, strings from the
    N-masked batch and the pattern's bit4 cells (search.rs:1428-1488); rc
    patterns print reverse complemented."""
    L = len(patterns[0])
    n_fwd = len(patterns) // 2
    out = []
    for (first, n, _head), recs in zip(ref.batches, per_batch):
        bv = _BatchView(ref.chunks, first, n)
        for loc, p, mm in recs.tolist():
            pl = bv.place(loc, L)
            if pl is None:
                continue
            cells = [bv.nib(loc + i) for i in range(L)]
            if masked:
                cells = [0 if v == 0xF else v for v in cells]
            dna = "".join(_DEC[v] for v in cells)
            rna = "".join(_DEC[_UP.get(ch.upper(), 0)] for ch in patterns[p])
            fwd = p < n_fwd
            if not fwd:
                dna, rna = _revcomp(dna), _revcomp(rna)
            out.append(f"{pl[0]}\t{pl[1]}\t{p}\t{'+' if fwd else '-'}\t{mm}\t0\t0\t{rna}\t{dna}")
    return out


def myers_raw_lines(ref, per_batch, patterns):
    """Raw Match lines of the Myers kernel's records: decode_gpu_enum_match
    (ops read last-to-first, a zero nibble under an M/S/D op drops the
    record) and the record-end drop of convert_matches_myers with extent
    L + db - rb."""
    L = len(patterns[0])
    n_fwd = len(patterns) // 2
    out = []
    for (first, n, _head), recs in zip(ref.batches, per_batch):
        bv = _BatchView(ref.chunks, first, n)
        for r in recs:
            pat = patterns[r.pattern_idx]
            pa, ta, pi, gi, ok = [], [], 0, r.chunk_idx, True
            for k in range(r.ops_count - 1, -1, -1):
                op = (r.ops_packed >> (2 * k)) & 3
                if op in (0, 1, 2):
                    v = bv.nib(gi)
                    if v == 0:
                        ok = False
                        break
                    ta.append(_DEC[v])
                    pa.append(pat[pi] if op != 2 else "-")
                    pi += op != 2
                    gi += 1
                else:
                    pa.append(pat[pi])
                    ta.append("-")
                    pi += 1
            if not ok:
                continue
            db, rb = r.dna_bulge_size, r.rna_bulge_size
            pl = bv.place(r.chunk_idx, L + db - rb)
            if pl is None:
                continue
            rna, dna = "".join(pa), "".join(ta)
            fwd = r.pattern_idx < n_fwd
            if not fwd:
                rna, dna = _revcomp(rna), _revcomp(dna)
            out.append(f"{pl[0]}\t{pl[1]}\t{r.pattern_idx}\t{'+' if fwd else '-'}\t"
                       f"{r.mismatches}\t{db}\t{rb}\t{rna}\t{dna}")
    return out


def skipped_starts(ref):
    """(name, position) of the window starts find_matches never scans: the
    last < 32 starts of a batch past floor(bytes / 16) * 32 (search.rs:280-284;
    the CPU path scans them)."""
    out = set()
    for first, n, _head in ref.batches:
        bv = _BatchView(ref.chunks, first, n)
        for s in range(len(bv.buf) // 16 * 32, 2 * len(bv.buf)):
            idx = bv.owner(s)
            name, _d, cs, _ce = bv.meta[idx]
            out.add((name, cs + (s - bv.offs[idx] * 2)))
    return out
