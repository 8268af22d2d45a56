"""ctypes binding of liboracle.so -- the CPU restatement of the reference.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py as the checker.  The product never imports it.
"""
import ctypes
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def reference_src():
    """The reference's cas-offinder-lib/src directory, from the environment
    variable COF_REFERENCE_DIR (the reference project's root), or None."""
    root = os.environ.get("COF_REFERENCE_DIR")
    return os.path.join(root, "cas-offinder-lib", "src") if root else None


def build_reference_kernels():
    """Builds _ref/ (the reference's kernel.cu / kernel_myers.cu for sm_100a
    and the launcher ref_gpu.cu) when COF_REFERENCE_DIR names the reference
    tree; without it, the files built earlier (if any) are kept."""
    src = reference_src()
    if src and os.path.exists(os.path.join(src, "kernel.cu")):
        subprocess.run(["make", "-s", "-j8", "-C", _HERE, "ref", "REF=" + src], check=True)


class _Req(ctypes.Structure):
    _fields_ = [
        ("filter", ctypes.c_char_p),
        ("patterns", ctypes.POINTER(ctypes.c_char_p)),
        ("n_patterns", ctypes.c_size_t),
        ("max_mismatches", ctypes.c_uint32),
        ("max_dna_bulges", ctypes.c_uint32),
        ("max_rna_bulges", ctypes.c_uint32),
        ("chunks_per_search", ctypes.c_uint32),
        ("n_threads", ctypes.c_int),
        ("raw_matches", ctypes.c_int),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.orc_genome_load.restype = vp
        L.orc_genome_load.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t]
        L.orc_genome_new.restype = vp
        L.orc_genome_add_chunk.argtypes = [vp, ctypes.c_char_p, ctypes.c_char_p,
                                           ctypes.c_uint64, ctypes.c_uint64]
        L.orc_genome_free.argtypes = [vp]
        L.orc_genome_n_chunks.argtypes = [vp]
        L.orc_genome_n_chunks.restype = ctypes.c_size_t
        L.orc_genome_n_nucl.argtypes = [vp]
        L.orc_genome_n_nucl.restype = ctypes.c_uint64
        L.orc_chunk_name.argtypes = [vp, ctypes.c_size_t]
        L.orc_chunk_name.restype = ctypes.c_char_p
        L.orc_chunk_start.argtypes = [vp, ctypes.c_size_t]
        L.orc_chunk_start.restype = ctypes.c_uint64
        L.orc_chunk_end.argtypes = [vp, ctypes.c_size_t]
        L.orc_chunk_end.restype = ctypes.c_uint64
        L.orc_chunk_data.argtypes = [vp, ctypes.c_size_t]
        L.orc_chunk_data.restype = ctypes.c_void_p
        L.orc_genome_decode.argtypes = [vp, ctypes.POINTER(ctypes.c_size_t)]
        L.orc_genome_decode.restype = ctypes.c_void_p
        L.orc_search.argtypes = [vp, ctypes.POINTER(_Req), ctypes.POINTER(ctypes.c_void_p),
                                 ctypes.POINTER(ctypes.c_size_t),
                                 ctypes.POINTER(ctypes.c_uint64), ctypes.c_char_p,
                                 ctypes.c_size_t]
        L.orc_popcount_scan_only.argtypes = [vp, ctypes.POINTER(_Req), ctypes.c_size_t,
                                             ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint64),
                                             ctypes.c_char_p, ctypes.c_size_t]
        L.orc_n_batches.argtypes = [vp, ctypes.c_uint32]
        L.orc_n_batches.restype = ctypes.c_size_t
        L.orc_free.argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


class OracleError(RuntimeError):
    pass


def _req(filt, patterns, mm, db, rb, cps, threads, keep, raw=False):
    fb = filt.encode() if isinstance(filt, str) else filt
    pb = [p.encode() if isinstance(p, str) else p for p in patterns]
    arr = (ctypes.c_char_p * len(pb))(*pb)
    keep.extend([fb, pb, arr])
    r = _Req()
    r.filter = fb
    r.patterns = arr
    r.n_patterns = len(pb)
    r.max_mismatches = mm
    r.max_dna_bulges = db
    r.max_rna_bulges = rb
    r.chunks_per_search = cps
    r.n_threads = threads
    r.raw_matches = 1 if raw else 0
    return r


class OracleGenome:
    def __init__(self, path=None):
        L = lib()
        if path is None:
            self._h = L.orc_genome_new()
        else:
            err = ctypes.create_string_buffer(512)
            self._h = L.orc_genome_load(os.fsencode(path), err, 512)
            if not self._h:
                raise OracleError(err.value.decode())

    def add_chunk(self, name, bit4, start, end):
        if lib().orc_genome_add_chunk(self._h, name.encode(), bytes(bit4), start, end):
            raise OracleError("bad chunk")

    @property
    def n_chunks(self):
        return lib().orc_genome_n_chunks(self._h)

    @property
    def n_nucl(self):
        return lib().orc_genome_n_nucl(self._h)

    def chunks(self):
        L = lib()
        out = []
        for k in range(self.n_chunks):
            s, e = L.orc_chunk_start(self._h, k), L.orc_chunk_end(self._h, k)
            data = ctypes.string_at(L.orc_chunk_data(self._h, k), (e - s + 1) // 2)
            out.append((L.orc_chunk_name(self._h, k).decode(), data, s, e))
        return out

    def decode(self):
        n = ctypes.c_size_t()
        p = lib().orc_genome_decode(self._h, ctypes.byref(n))
        s = ctypes.string_at(p, n.value)
        lib().orc_free(p)
        return s

    def n_batches(self, cps):
        return lib().orc_n_batches(self._h, cps)

    def search(self, search_filter, patterns, max_mismatches, max_dna_bulges=0,
               max_rna_bulges=0, chunks_per_search=0, n_threads=0, raw=False):
        """Rows of main.rs's writer for user patterns (rc appended), or with
        raw=True the raw Match lines of search()."""
        keep = []
        r = _req(search_filter, patterns, max_mismatches, max_dna_bulges, max_rna_bulges,
                 chunks_per_search, n_threads, keep, raw)
        out = ctypes.c_void_p()
        n = ctypes.c_size_t()
        nr = ctypes.c_uint64()
        err = ctypes.create_string_buffer(512)
        if lib().orc_search(self._h, ctypes.byref(r), ctypes.byref(out), ctypes.byref(n),
                            ctypes.byref(nr), err, 512):
            raise OracleError(err.value.decode())
        text = ctypes.string_at(out, n.value).decode("latin-1")
        lib().orc_free(out)
        return text, nr.value

    def popcount_scan_only(self, search_filter, patterns, max_mismatches, batch_begin,
                           batch_end, chunks_per_search=64, n_threads=0):
        keep = []
        r = _req(search_filter, patterns, max_mismatches, 0, 0, chunks_per_search, n_threads,
                 keep)
        n = ctypes.c_uint64()
        err = ctypes.create_string_buffer(512)
        if lib().orc_popcount_scan_only(self._h, ctypes.byref(r), batch_begin, batch_end,
                                        ctypes.byref(n), err, 512):
            raise OracleError(err.value.decode())
        return n.value

    def close(self):
        if getattr(self, "_h", None):
            lib().orc_genome_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
