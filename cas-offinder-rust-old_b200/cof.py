"""Python host binding of libcof.so (ctypes over include/cof.h).

Mirrors cas-offinder-lib's public search API:

    search(devices, max_mismatches, max_dna_bulges, max_rna_bulges,
           search_filter_ascii, pattern_len, patterns_ascii, recv, dest)
    (cas-offinder-lib/src/search.rs:1490-1500)

The genome (the `recv` channel of ChromChunkInfo) is a `Genome` object that
is filled once and stays resident on the GPU; the result (the `dest` channel,
rendered by the CLI writer, cas-offinder-cli/src/main.rs:122-247) is the
8-column row text.  The CUDA library must be present: importing this module
without libcof.so raises, there is no CPU fallback.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcof.so")

COF_OK = 0
COF_E_BADINPUT = -1
COF_E_OOM = -2
COF_E_CUDA = -3
COF_E_IO = -4
COF_E_UNSUPPORTED = -5
COF_E_STATE = -6
COF_E_TIMEOUT = -7
COF_E_CANCELLED = -8
COF_F_ADD_REVCOMP = 1
COF_F_RAW_MATCHES = 2
COF_STREAM_MATCHES = 1

HEADER = "#Bulge type\tcrRNA\tDNA\tChromosome\tPosition\tDirection\tMismatches\tBulge Size\n"

# Every symbol include/cof.h declares.
EXPORTS = (
    "cof_genome_create", "cof_genome_add_chunk", "cof_genome_load", "cof_genome_upload",
    "cof_genome_n_nucl", "cof_genome_n_chunks", "cof_genome_free", "cof_search",
    "cof_search_batch", "cof_result_free", "cof_genome_last_stats", "cof_last_error",
    "cof_abi_version", "cof_search_seq_noalloc", "cof_server_create", "cof_server_submit",
    "cof_server_wait", "cof_server_stats", "cof_server_free", "cof_genome_tuning",
    "cof_search_stream", "cof_genome_record_name", "cof_genome_n_records",
)


class CofError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"cof error {code}: {msg}")
        self.code = code


class _Request(ctypes.Structure):
    _fields_ = [
        ("search_filter", ctypes.c_char_p),
        ("pattern_len", ctypes.c_size_t),
        ("patterns", ctypes.POINTER(ctypes.c_char_p)),
        ("n_patterns", ctypes.c_size_t),
        ("max_mismatches", ctypes.c_uint32),
        ("max_dna_bulges", ctypes.c_uint32),
        ("max_rna_bulges", ctypes.c_uint32),
        ("flags", ctypes.c_uint32),
        ("chunks_per_search", ctypes.c_uint32),
    ]


class _Result(ctypes.Structure):
    _fields_ = [
        ("text", ctypes.c_void_p),
        ("text_len", ctypes.c_size_t),
        ("n_rows", ctypes.c_uint64),
        ("device_ms", ctypes.c_double),
    ]


class Match(ctypes.Structure):
    """cof_match: one Match of search()'s stream (chrom_chunk.rs:19-29)."""
    _fields_ = [
        ("chrom_idx", ctypes.c_uint64),
        ("text_offset", ctypes.c_uint64),
        ("record", ctypes.c_uint32),
        ("pattern_idx", ctypes.c_uint32),
        ("mismatches", ctypes.c_uint8),
        ("dna_bulge_size", ctypes.c_uint8),
        ("rna_bulge_size", ctypes.c_uint8),
        ("is_forward", ctypes.c_uint8),
        ("pad", ctypes.c_uint32),
    ]


class _Piece(ctypes.Structure):
    _fields_ = [
        ("request", ctypes.c_size_t),
        ("text", ctypes.c_void_p),
        ("text_len", ctypes.c_size_t),
        ("n_rows", ctypes.c_uint64),
        ("matches", ctypes.POINTER(Match)),
    ]


_SINK = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(_Piece))


class _ServerConfig(ctypes.Structure):
    _fields_ = [("max_requests_per_pass", ctypes.c_uint32),
                ("memory_budget_bytes", ctypes.c_uint64),
                ("ring_slices", ctypes.c_uint32)]


_lib = None


def load_library(path=LIB_PATH):
    """Loads libcof.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with cas-offinder-rust-old_b200/build.py")
    lib = ctypes.CDLL(path)
    vp, c = ctypes.c_void_p, ctypes
    lib.cof_genome_create.argtypes = [c.c_int, c.POINTER(vp)]
    lib.cof_genome_add_chunk.argtypes = [vp, c.c_char_p, c.c_void_p, c.c_uint64, c.c_uint64]
    lib.cof_genome_load.argtypes = [vp, c.c_char_p]
    lib.cof_genome_upload.argtypes = [vp]
    lib.cof_genome_n_nucl.argtypes = [vp]
    lib.cof_genome_n_nucl.restype = c.c_uint64
    lib.cof_genome_n_chunks.argtypes = [vp]
    lib.cof_genome_n_chunks.restype = c.c_uint64
    lib.cof_genome_free.argtypes = [vp]
    lib.cof_genome_free.restype = None
    lib.cof_search.argtypes = [vp, c.POINTER(_Request), c.POINTER(_Result)]
    lib.cof_search_batch.argtypes = [vp, c.POINTER(_Request), c.c_size_t, c.POINTER(_Result)]
    lib.cof_result_free.argtypes = [c.POINTER(_Result)]
    lib.cof_result_free.restype = None
    lib.cof_genome_last_stats.argtypes = [vp, c.POINTER(c.c_double), c.POINTER(c.c_uint64)]
    lib.cof_last_error.restype = c.c_char_p
    lib.cof_abi_version.restype = c.c_int
    lib.cof_genome_tuning.argtypes = [vp, c.c_char_p, c.c_size_t]
    lib.cof_server_create.argtypes = [vp, c.POINTER(_ServerConfig), c.POINTER(vp)]
    lib.cof_server_submit.argtypes = [vp, c.POINTER(_Request), c.POINTER(c.c_uint64)]
    lib.cof_server_wait.argtypes = [vp, c.c_uint64, c.c_int64, c.POINTER(_Result),
                                    c.POINTER(c.c_double)]
    lib.cof_server_stats.argtypes = [vp, c.POINTER(c.c_uint64)]
    lib.cof_server_free.argtypes = [vp]
    lib.cof_server_free.restype = None
    lib.cof_search_stream.argtypes = [vp, c.POINTER(_Request), c.c_size_t, c.c_uint32, _SINK,
                                      vp, c.POINTER(c.c_uint64)]
    lib.cof_genome_record_name.argtypes = [vp, c.c_uint32]
    lib.cof_genome_record_name.restype = c.c_char_p
    lib.cof_genome_n_records.argtypes = [vp]
    lib.cof_genome_n_records.restype = c.c_uint32
    lib.cof_search_seq_noalloc.argtypes = [c.c_void_p, c.c_uint64, c.c_char_p,
                                           c.POINTER(c.c_char_p), c.c_size_t, c.c_uint32,
                                           c.c_void_p, c.c_uint32, c.POINTER(c.c_uint32),
                                           c.c_void_p]
    _lib = lib
    return lib


def _check(rc):
    if rc != COF_OK:
        raise CofError(rc, _lib.cof_last_error().decode(errors="replace"))


def _make_request(filt, patterns, mm, db, rb, add_revcomp, cps, keep, raw=False):
    fb = filt.encode() if isinstance(filt, str) else bytes(filt)
    pb = [p.encode() if isinstance(p, str) else bytes(p) for p in patterns]
    arr = (ctypes.c_char_p * len(pb))(*pb)
    keep.extend([fb, pb, arr])
    r = _Request()
    r.search_filter = fb
    r.pattern_len = len(fb)
    r.patterns = arr
    r.n_patterns = len(pb)
    r.max_mismatches = mm
    r.max_dna_bulges = db
    r.max_rna_bulges = rb
    r.flags = (COF_F_ADD_REVCOMP if add_revcomp else 0) | (COF_F_RAW_MATCHES if raw else 0)
    r.chunks_per_search = cps
    return r


class Genome:
    """A genome resident on one GPU (replaces the ChromChunkInfo channel)."""

    def __init__(self, path=None, device=0):
        lib = load_library()
        h = ctypes.c_void_p()
        _check(lib.cof_genome_create(device, ctypes.byref(h)))
        self._h = h
        if path is not None:
            self.load(path)

    def load(self, path):
        _check(_lib.cof_genome_load(self._h, os.fsencode(path)))

    def add_chunk(self, name, bit4, chunk_start, chunk_end):
        buf = bytes(bit4)
        _check(_lib.cof_genome_add_chunk(self._h, name.encode() if isinstance(name, str) else name,
                                         buf, chunk_start, chunk_end))

    def upload(self):
        _check(_lib.cof_genome_upload(self._h))

    @property
    def n_nucl(self):
        return _lib.cof_genome_n_nucl(self._h)

    @property
    def n_chunks(self):
        return _lib.cof_genome_n_chunks(self._h)

    def search(self, search_filter, patterns, max_mismatches, max_dna_bulges=0,
               max_rna_bulges=0, add_revcomp=True, chunks_per_search=0, raw=False):
        """Returns (rows_text, n_rows) for one request (raw=True: search()'s
        Match lines, COF_F_RAW_MATCHES)."""
        return self.search_batch([dict(search_filter=search_filter, patterns=patterns,
                                       max_mismatches=max_mismatches,
                                       max_dna_bulges=max_dna_bulges,
                                       max_rna_bulges=max_rna_bulges, add_revcomp=add_revcomp,
                                       chunks_per_search=chunks_per_search, raw=raw)])[0]

    def prepare(self, requests):
        """Encodes requests once for repeated cof_search_batch calls."""
        keep = []
        reqs = (_Request * len(requests))()
        for i, r in enumerate(requests):
            reqs[i] = _make_request(r["search_filter"], r["patterns"], r["max_mismatches"],
                                    r.get("max_dna_bulges", 0), r.get("max_rna_bulges", 0),
                                    r.get("add_revcomp", True), r.get("chunks_per_search", 0),
                                    keep, r.get("raw", False))
        return reqs, keep

    def run_prepared(self, prepared, as_text=True):
        """One cof_search_batch call; returns [(rows, n_rows), ...] with rows
        as str (as_text), bytes, or None (result buffers freed unread)."""
        reqs, _keep = prepared
        outs = (_Result * len(reqs))()
        _check(_lib.cof_search_batch(self._h, reqs, len(reqs), outs))
        res = []
        for o in outs:
            if as_text is None:
                data = o.text_len
            else:
                data = ctypes.string_at(o.text, o.text_len) if o.text_len else b""
                if as_text:
                    data = data.decode("latin-1")
            res.append((data, o.n_rows))
            _lib.cof_result_free(ctypes.byref(o))
        return res

    def search_batch(self, requests):
        """Many requests in one pass; returns [(rows_text, n_rows), ...]."""
        return self.run_prepared(self.prepare(requests))

    def search_stream(self, requests, on_piece, matches=False, prepared=None):
        """cof_search_stream: calls on_piece(request, text_bytes, n_rows,
        match_list_or_None) for every piece of output, in order, on this
        thread; a truthy return stops the search (CofError COF_E_CANCELLED).
        Returns each request's row count.  match_list: (chrom_idx,
        text_offset, record, pattern_idx, mismatches, dna_bulge_size,
        rna_bulge_size, is_forward) tuples."""
        reqs, _keep = prepared if prepared is not None else self.prepare(requests)
        err = []

        def cb(_user, pp):
            try:
                p = pp.contents
                text = ctypes.string_at(p.text, p.text_len) if p.text_len else b""
                recs = None
                if p.matches:
                    recs = [(m.chrom_idx, m.text_offset, m.record, m.pattern_idx, m.mismatches,
                             m.dna_bulge_size, m.rna_bulge_size, m.is_forward)
                            for m in p.matches[:p.n_rows]]
                return 1 if on_piece(p.request, text, p.n_rows, recs) else 0
            except BaseException as e:  # noqa: BLE001 -- re-raised after the call
                err.append(e)
                return 1

        fn = _SINK(cb)
        n = (ctypes.c_uint64 * max(len(reqs), 1))()
        rc = _lib.cof_search_stream(self._h, reqs, len(reqs),
                                    COF_STREAM_MATCHES if matches else 0, fn, None, n)
        if err:
            raise err[0]
        _check(rc)
        return [n[i] for i in range(len(reqs))]

    def stream_count(self, prepared, matches=False):
        """cof_search_stream with a sink that only counts: returns (rows,
        text bytes, pieces).  The rows pass through page-locked staging
        buffers and are never held, so the result may exceed host memory."""
        reqs, _keep = prepared
        tot = [0, 0, 0]

        def cb(_user, pp):
            p = pp.contents
            tot[0] += p.n_rows
            tot[1] += p.text_len
            tot[2] += 1
            return 0

        fn = _SINK(cb)
        n = (ctypes.c_uint64 * max(len(reqs), 1))()
        _check(_lib.cof_search_stream(self._h, reqs, len(reqs),
                                      COF_STREAM_MATCHES if matches else 0, fn, None, n))
        return tot[0], tot[1], tot[2]

    def record_name(self, record):
        v = _lib.cof_genome_record_name(self._h, record)
        return None if v is None else v.decode()

    @property
    def n_records(self):
        return _lib.cof_genome_n_records(self._h)

    def last_stats(self):
        ms = (ctypes.c_double * 5)()
        cnt = (ctypes.c_uint64 * 5)()
        _check(_lib.cof_genome_last_stats(self._h, ms, cnt))
        return dict(scan_ms=ms[0], verify_ms=ms[1], format_ms=ms[2], d2h_ms=ms[3],
                    total_ms=ms[4], candidates=cnt[0], pairs=cnt[1], raw_hits=cnt[2],
                    rows=cnt[3], kernel_launches=cnt[4])

    def tuning(self):
        """Autotuner state (dict)."""
        import json
        buf = ctypes.create_string_buffer(1 << 16)
        _check(_lib.cof_genome_tuning(self._h, buf, len(buf)))
        return json.loads(buf.value.decode())

    def close(self):
        if getattr(self, "_h", None):
            _lib.cof_genome_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def search(devices, max_mismatches, max_dna_bulges, max_rna_bulges, search_filter_ascii,
           pattern_len, patterns_ascii, genome):
    """search() of search.rs:1490 with the genome as a resident Genome.

    `devices` is accepted for signature parity (one GPU per Genome); the
    patterns are the full fwd+rc list as main.rs passes them.  Returns the
    writer's rows (list of str, without the header)."""
    assert len(patterns_ascii) > 0
    assert all(len(p) == pattern_len for p in patterns_ascii), "All patterns must have same length"
    text, _ = genome.search(search_filter_ascii, patterns_ascii, max_mismatches, max_dna_bulges,
                            max_rna_bulges, add_revcomp=False)
    return text.splitlines()


class Server:
    """Continuous-batching request loop over a resident Genome
    (cof_server_*): the genome is walked as a ring of ring_slices slices (0:
    about one per 512 Mnt), arrivals join at slice boundaries.
    max_requests_per_pass=1 is the plain one-request-per-pass loop."""

    def __init__(self, genome, max_requests_per_pass=0, memory_budget_bytes=0, ring_slices=0):
        self.genome = genome
        cfg = _ServerConfig(max_requests_per_pass, memory_budget_bytes, ring_slices)
        h = ctypes.c_void_p()
        _check(_lib.cof_server_create(genome._h, ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self._keep = {}

    def submit(self, search_filter, patterns, max_mismatches, max_dna_bulges=0,
               max_rna_bulges=0, add_revcomp=True, chunks_per_search=0):
        keep = []
        r = _make_request(search_filter, patterns, max_mismatches, max_dna_bulges,
                          max_rna_bulges, add_revcomp, chunks_per_search, keep)
        t = ctypes.c_uint64()
        _check(_lib.cof_server_submit(self._h, ctypes.byref(r), ctypes.byref(t)))
        return t.value

    def wait(self, ticket, timeout_ms=-1, as_text=True):
        """Returns (rows, n_rows, latency_ms); rows as str, bytes or None."""
        o = _Result()
        lat = ctypes.c_double()
        _check(_lib.cof_server_wait(self._h, ticket, timeout_ms, ctypes.byref(o),
                                    ctypes.byref(lat)))
        if as_text is None:
            data = o.text_len
        else:
            data = ctypes.string_at(o.text, o.text_len) if o.text_len else b""
            if as_text:
                data = data.decode("latin-1")
        n = o.n_rows
        _lib.cof_result_free(ctypes.byref(o))
        return data, n, lat.value

    def stats(self):
        """steps (slice searches), completed, queued, and the most requests
        active in one step."""
        s = (ctypes.c_uint64 * 4)()
        _check(_lib.cof_server_stats(self._h, s))
        return dict(passes=s[0], completed=s[1], queued=s[2], largest_pass=s[3])

    def close(self):
        if getattr(self, "_h", None):
            _lib.cof_server_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

