"""Seeded synthetic genomes, guides and planted sites for the benchmark shapes.

Stands in for hg38 (not available offline): i.i.d. bases at ~41% GC
(A,T = 76/256, C,G = 52/256), runs of N, and planted near-target sites with a
recorded truth list.  Genomes are produced directly as the reference's chunk
stream (bit4 one-hot nibbles in 64 Knt chunks cut at 60-column FASTA line
boundaries, i.e. 65520-nt chunks, read_fasta.rs:45-57) or written as FASTA.
"""
import bisect

import numpy as np

# bit4 one-hot codes (cas-offinder-lib/src/bit4ops.rs:1-4, 17-37)
B4 = {"T": 1, "C": 2, "A": 4, "G": 8, "N": 15, "R": 12, "Y": 3, "S": 10, "W": 5, "K": 9,
      "M": 6, "B": 11, "D": 13, "H": 7, "V": 14}
B4CHAR = {v: k for k, v in B4.items()}
COMP = {"A": "T", "C": "G", "G": "C", "T": "A", "N": "N", "R": "Y", "Y": "R", "S": "S",
        "W": "W", "K": "M", "M": "K", "B": "V", "V": "B", "D": "H", "H": "D"}
_LUT = np.array([4] * 76 + [2] * 52 + [8] * 52 + [1] * 76, dtype=np.uint8)
_CHARS = np.zeros(16, dtype=np.uint8)
for _k, _v in B4.items():
    _CHARS[_v] = ord(_k)


def revcomp(s):
    return "".join(COMP[c] for c in reversed(s.upper()))


def random_bases(rng, n):
    """n bit4 codes, i.i.d., 40.6% GC."""
    return _LUT[rng.integers(0, 256, size=n, dtype=np.uint8)]


def random_guide(rng, n):
    return "".join(rng.choice(list("ACGT"), size=n))


def iupac_instance(rng, c):
    """A concrete base matching IUPAC character c."""
    v = B4[c.upper()]
    opts = [b for b in "ACGT" if B4[b] & v]
    return opts[rng.integers(0, len(opts))]


class SynthGenome:
    """Records as bit4 code arrays (one uint8 per nucleotide)."""

    def __init__(self, names, records):
        self.names = list(names)
        self.records = list(records)

    @property
    def n_nucl(self):
        return sum(len(r) for r in self.records)

    def chunks(self, line_len=60, chunk_size=65536):
        """(name, bit4 bytes, start, end) exactly as read_fasta would emit for
        this genome written with `line_len`-column lines."""
        per = (chunk_size // line_len) * line_len
        for name, rec in zip(self.names, self.records):
            n = len(rec)
            if n == 0:
                continue
            pad = np.zeros(n + (n & 1), dtype=np.uint8)
            pad[:n] = rec
            packed = (pad[0::2] | (pad[1::2] << 4)).astype(np.uint8)
            for s in range(0, n, per):
                e = min(s + per, n)
                yield name, packed[s // 2:(e + 1) // 2].tobytes(), s, e

    def write_fasta(self, path, line_len=60):
        """FASTA with `line_len`-column lines, each record's whole lines laid
        out as one (lines x (line_len + 1)) array with a newline column."""
        with open(path, "wb") as f:
            for name, rec in zip(self.names, self.records):
                f.write(b">" + name.encode() + b"\n")
                chars = _CHARS[rec]
                full = len(chars) // line_len * line_len
                if full:
                    block = np.empty((full // line_len, line_len + 1), dtype=np.uint8)
                    block[:, :line_len] = chars[:full].reshape(-1, line_len)
                    block[:, line_len] = ord("\n")
                    f.write(block.tobytes())
                if full < len(chars):
                    f.write(chars[full:].tobytes() + b"\n")

    def write_2bit(self, path):
        """UCSC .2bit v0 (the format read_2bit.rs reads): bases packed 2 bits
        each, T=0 C=1 A=2 G=3, first base in the high bits; N runs as N
        blocks.  The synthetic records hold only A, C, G, T and N."""
        import struct
        to2 = np.zeros(16, dtype=np.uint8)
        to2[[1, 2, 4, 8]] = [0, 1, 2, 3]
        blocks = []
        for rec in self.records:
            d = np.flatnonzero(rec == 15)
            if len(d):
                br = np.flatnonzero(np.diff(d) != 1)
                starts = d[np.concatenate(([0], br + 1))]
                ends = d[np.concatenate((br, [len(d) - 1]))] + 1
            else:
                starts = ends = d
            blocks.append((starts.astype("<u4"), (ends - starts).astype("<u4")))
        off = 16 + sum(1 + len(n) + 4 for n in self.names)
        with open(path, "wb") as f:
            f.write(struct.pack("<IIII", 0x1A412743, 0, len(self.names), 0))
            for name, rec, (st, sz) in zip(self.names, self.records, blocks):
                f.write(bytes([len(name)]) + name.encode() + struct.pack("<I", off))
                off += 16 + 8 * len(st) + (len(rec) + 3) // 4
            for rec, (st, sz) in zip(self.records, blocks):
                f.write(struct.pack("<II", len(rec), len(st)) + st.tobytes() + sz.tobytes() +
                        struct.pack("<II", 0, 0))
                c = to2[rec]
                n4 = len(c) // 4 * 4
                v = c[:n4].view(">u4")
                packed = ((v >> 18) & 0xC0) | ((v >> 12) & 0x30) | ((v >> 6) & 0xC) | (v & 3)
                f.write(packed.astype(np.uint8).tobytes())
                if n4 < len(c):
                    t = np.zeros(4, dtype=np.uint8)
                    t[:len(c) - n4] = c[n4:]
                    f.write(bytes([(t[0] << 6) | (t[1] << 4) | (t[2] << 2) | t[3]]))

    def site(self, rec, pos, length):
        return bytes(_CHARS[self.records[rec][pos:pos + length]]).decode()

    def load_into(self, genome, line_len=60):
        for name, data, s, e in self.chunks(line_len):
            genome.add_chunk(name, data, s, e)
        return genome


def make_genome(rng, lengths, n_runs=(), names=None):
    """lengths: record lengths; n_runs: list of (record, length) N runs."""
    names = names or [f"chr{i + 1}" for i in range(len(lengths))]
    recs = [random_bases(rng, n) for n in lengths]
    occupied = [[] for _ in lengths]
    for r, ln in n_runs:
        if ln >= lengths[r]:
            continue
        p = int(rng.integers(0, lengths[r] - ln))
        recs[r][p:p + ln] = 15
        bisect.insort(occupied[r], (p, p + ln))
    g = SynthGenome(names, recs)
    g.occupied = occupied
    return g


def _free(occ, a, b, margin=8):
    """occ: sorted list of (start, end) intervals."""
    i = bisect.bisect_left(occ, (a, a))
    for x, y in occ[max(i - 1, 0):i + 1]:
        if not (b + margin <= x or a >= y + margin):
            return False
    # an earlier long interval (N run) may still cover [a, b)
    return all(not (x <= a < y + margin) for x, y in occ[max(i - 64, 0):i])


def plant(rng, g, pattern, pam_filter, n_sites, max_subs, truth, guide_idx,
          bulge=None):
    """Writes n_sites copies of `pattern` (guide cells substituted, PAM cells
    made concrete from pam_filter) at random free positions on a random
    strand; appends (record, pos, strand, guide_idx, n_subs) to truth.

    bulge: optional (n_ins, n_del) -- guide bases inserted into / deleted
    from the site away from the PAM-adjacent cells."""
    L = len(pattern)
    for _ in range(n_sites):
        site = []
        guide_cells = [i for i, c in enumerate(pattern) if c.upper() != "N"]
        k = int(rng.integers(0, max_subs + 1))
        subs = set(rng.choice(guide_cells, size=min(k, len(guide_cells)), replace=False).tolist())
        for i, c in enumerate(pattern):
            if c.upper() == "N":
                site.append(iupac_instance(rng, pam_filter[i]))
            elif i in subs:
                site.append(rng.choice([b for b in "ACGT" if b != c.upper()]))
            else:
                site.append(c.upper())
        if bulge:
            n_ins, n_del = bulge
            interior = guide_cells[2:-2]
            for _i in range(n_del):
                j = int(rng.choice(interior))
                site[j] = ""
            for _i in range(n_ins):
                j = int(rng.choice(interior))
                site[j] = site[j] + rng.choice(list("ACGT"))
        s = "".join(site)
        strand = int(rng.integers(0, 2))
        if strand:
            s = revcomp(s)
        for _try in range(1000):
            r = int(rng.integers(0, len(g.records)))
            if len(g.records[r]) <= len(s) + 64:
                continue
            p = int(rng.integers(16, len(g.records[r]) - len(s) - 16))
            if _free(g.occupied[r], p, p + len(s)):
                break
        else:
            raise RuntimeError("no room to plant")
        g.records[r][p:p + len(s)] = np.array([B4[c] for c in s], dtype=np.uint8)
        bisect.insort(g.occupied[r], (p, p + len(s)))
        truth.append((r, p, "-" if strand else "+", guide_idx, k, len(s)))


# ---------------------------------------------------------------------------
# benchmark shapes (scale < 1 shrinks genome sizes for tests)
# ---------------------------------------------------------------------------

def config_plain_small(seed=1, scale=1.0):
    """10 Mbp in 4 records (4/3/2/1 Mbp), 5 N-runs of 10-50 kb, 1 guide of
    20 nt + NRG, <= 3 mismatches, 20 planted sites with 0-3 substitutions."""
    rng = np.random.default_rng(seed)
    lengths = [int(x * scale) for x in (4_000_000, 3_000_000, 2_000_000, 1_000_000)]
    runs = [(int(rng.integers(0, 4)), int(rng.integers(10_000, 50_001) * scale))
            for _ in range(5)]
    g = make_genome(rng, lengths, runs)
    guide = random_guide(rng, 20)
    pattern = guide + "NNN"
    filt = "N" * 21 + "RG"
    truth = []
    plant(rng, g, pattern, "N" * 20 + "NRG", 20, 3, truth, 0)
    return dict(genome=g, filter=filt, patterns=[pattern], max_mismatches=3, truth=truth,
                name="plain 10 Mbp x 1 guide (20 nt + NRG), mm<=3")


def _genome_3g(rng, scale, n_records=24):
    total = int(3_100_000_000 * scale)
    w = rng.uniform(50, 250, size=n_records)
    lengths = [int(x) for x in (w / w.sum() * total)]
    # ~5% of bases in N-runs of 10 kb - 3 Mb
    runs, target, acc = [], 0.05 * total, 0
    while acc < target:
        ln = int(min(np.exp(rng.uniform(np.log(10_000), np.log(3_000_000))) * max(scale, 1e-3),
                     target - acc + 1))
        ln = max(ln, 10)
        runs.append((int(rng.integers(0, n_records)), ln))
        acc += ln
    return make_genome(rng, lengths, runs)


def config_full_genome(seed=2, scale=1.0, n_guides=100, planted=50):
    """3.1 Gbp, 24 records of 50-250 Mbp, ~5% N; 100 guides of 20 nt + NRG,
    <= 6 mismatches, 50 planted sites per guide with 0-6 mismatches."""
    rng = np.random.default_rng(seed)
    g = _genome_3g(rng, scale)
    guides = [random_guide(rng, 20) for _ in range(n_guides)]
    patterns = [x + "NNN" for x in guides]
    truth = []
    for i, p in enumerate(patterns):
        plant(rng, g, p, "N" * 20 + "NRG", planted, 6, truth, i)
    return dict(genome=g, filter="N" * 21 + "RG", patterns=patterns, max_mismatches=6,
                truth=truth, name="3.1 Gbp x 100 guides (20 nt + NRG), mm<=6")


def config_mixed_pam(seed=3, scale=1.0, n_each=50, planted=50):
    """Same genome shape; 50 x (25 nt + NNGRRT) and 50 x (TTTN + 25 nt), mm<=6.
    Returns two requests (the reference runs them separately)."""
    rng = np.random.default_rng(seed)
    g = _genome_3g(rng, scale)
    truth = []
    a = [random_guide(rng, 25) + "NNNNNN" for _ in range(n_each)]
    b = ["NNNN" + random_guide(rng, 25) for _ in range(n_each)]
    for i, p in enumerate(a):
        plant(rng, g, p, "N" * 25 + "NNGRRT", planted, 6, truth, i)
    for i, p in enumerate(b):
        plant(rng, g, p, "TTTN" + "N" * 25, planted, 6, truth, n_each + i)
    reqs = [dict(search_filter="N" * 25 + "NNGRRT", patterns=a, max_mismatches=6),
            dict(search_filter="TTTN" + "N" * 25, patterns=b, max_mismatches=6)]
    return dict(genome=g, requests=reqs, truth=truth,
                name="3.1 Gbp x 100 guides (50 NNGRRT + 50 TTTN, 25 nt), mm<=6, batched")


def config_bulge(seed=4, scale=1.0, n_guides=20, planted=30):
    """500 Mbp in 5 records; 20 guides of 20 nt + NRG; mm<=4, DNA/RNA bulge<=2."""
    rng = np.random.default_rng(seed)
    total = int(500_000_000 * scale)
    g = make_genome(rng, [total // 5] * 5, [])
    guides = [random_guide(rng, 20) + "NNN" for _ in range(n_guides)]
    truth = []
    for i, p in enumerate(guides):
        for _k in range(planted):
            ins = int(rng.integers(0, 3))
            dele = int(rng.integers(0 if ins else 1, 3 - ins if ins < 2 else 1))
            plant(rng, g, p, "N" * 20 + "NRG", 1, 4, truth, i, bulge=(ins, dele))
    return dict(genome=g, filter="N" * 21 + "RG", patterns=guides, max_mismatches=4,
                max_dna_bulges=2, max_rna_bulges=2, truth=truth,
                name="500 Mbp x 20 guides (20 nt + NRG), mm<=4, bulges<=2")
