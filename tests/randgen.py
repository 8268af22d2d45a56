"""Seeded random small genomes and requests for the parity tests.

Chunks are produced directly (not through FASTA) so that small genomes still
exercise intra-record chunk boundaries, odd-length chunks inside a record
(their pad nibble sits inside the record, search.rs:1400-1412), tiny chunks
at batch boundaries and IUPAC / N genome letters.
"""
import random

IUPAC = "RYSWKMBDHV"
B4 = {"T": 1, "C": 2, "A": 4, "G": 8, "N": 15, "R": 12, "Y": 3, "S": 10, "W": 5, "K": 9,
      "M": 6, "B": 11, "D": 13, "H": 7, "V": 14}

REQUEST_SHAPES = [
    # (filter, pattern maker, mm)
    ("N" * 21 + "RG", lambda g: g[:20] + "NNN", 4),          # NRG, 3' PAM
    ("TTTN" + "N" * 20, lambda g: "NNNN" + g[:20], 4),        # TTTN, 5' PAM
    ("N" * 18 + "NNGRRT", lambda g: g[:18] + "NNNNNN", 3),   # NNGRRT
    ("N" * 14, lambda g: g[:14], 3),                          # no PAM at all
    ("N" * 17 + "NGG", lambda g: g[:10] + "R" + g[11:17] + "NNN", 3),  # IUPAC in guide
    ("NNNNNNNNNNANNNNNNNNNRG", lambda g: g[:19] + "NNN", 3),  # constrained guide cell
]


def random_seq(rng, n, gc=0.41, n_rate=0.02, iupac_rate=0.01):
    out = []
    while len(out) < n:
        x = rng.random()
        if x < n_rate:
            out.extend("N" * rng.randint(1, 40))
        elif x < n_rate + iupac_rate:
            out.append(rng.choice(IUPAC))
        else:
            y = rng.random()
            out.append("G" if y < gc / 2 else "C" if y < gc else "A" if y < (1 + gc) / 2 else "T")
    return "".join(out[:n])


def pack(seq):
    nib = [B4[c] for c in seq]
    if len(nib) % 2:
        nib.append(0)
    return bytes(nib[i] | (nib[i + 1] << 4) for i in range(0, len(nib), 2)), [B4[c] for c in seq]


def random_genome(rng, n_records=3, min_len=200, max_len=1500, max_chunk=300):
    """Returns (chunks, records): chunks = [(name, bit4 bytes, nibbles, start, end)]."""
    chunks, records = [], []
    for r in range(n_records):
        n = rng.randint(min_len, max_len)
        seq = random_seq(rng, n)
        records.append(seq)
        s = 0
        while s < n:
            ln = min(rng.randint(1, max_chunk), n - s)
            data, nibs = pack(seq[s:s + ln])
            chunks.append((f"rec{r} desc {r}", data, nibs, s, s + ln))
            s += ln
    return chunks, records


def plant_sites(rng, records, pattern, filt, count, max_subs):
    """Overwrites random windows of records with near-copies of pattern
    (both strands) so that searches find rows."""
    comp = {"A": "T", "C": "G", "G": "C", "T": "A"}
    for _ in range(count):
        r = rng.randrange(len(records))
        seq = records[r]
        if len(seq) < len(pattern) + 2:
            continue
        p = rng.randrange(0, len(seq) - len(pattern))
        site = []
        for i, c in enumerate(pattern):
            f = filt[i]
            if f != "N":
                site.append(rng.choice([b for b in "ACGT" if B4[b] & B4[f]]))
            elif c == "N" or c not in "ACGT":
                opts = [b for b in "ACGT" if B4[b] & B4[f if f != "N" else "N"]]
                site.append(rng.choice(opts))
            elif rng.random() < max_subs / len(pattern):
                site.append(rng.choice([b for b in "ACGT" if b != c]))
            else:
                site.append(c)
        s = "".join(site)
        if rng.random() < 0.5:
            s = "".join(comp[c] for c in reversed(s))
        records[r] = seq[:p] + s + seq[p + len(s):]


def chunk_records(rng, records, max_chunk=300):
    chunks = []
    for r, seq in enumerate(records):
        s = 0
        while s < len(seq):
            ln = min(rng.randint(1, max_chunk), len(seq) - s)
            data, nibs = pack(seq[s:s + ln])
            chunks.append((f"rec{r} desc {r}", data, nibs, s, s + ln))
            s += ln
    return chunks


def random_case(seed, bulge=False):
    rng = random.Random(seed)
    filt, mk, mm = REQUEST_SHAPES[seed % len(REQUEST_SHAPES)]
    guides = ["".join(rng.choice("ACGT") for _ in range(25)) for _ in range(rng.randint(1, 3))]
    pats = [mk(g) for g in guides]
    if rng.random() < 0.3:
        pats = [p.lower() if rng.random() < 0.5 else p for p in pats]
    _, records = random_genome(rng, rng.randint(1, 4))
    for p in pats:
        plant_sites(rng, records, p.upper(), filt, 6, 2)
    chunks = chunk_records(rng, records, max_chunk=rng.choice([60, 300, 2000]))
    cps = rng.choice([2, 3, 5, 16384])
    db = rb = 0
    if bulge:
        db, rb = rng.choice([(1, 0), (0, 1), (1, 1), (2, 1)])
        mm = min(mm, 3)
    return dict(chunks=chunks, filter=filt, patterns=pats, mm=mm, db=db, rb=rb, cps=cps)


def write_messy_fasta(rng, path, final_newline):
    # CRLF and LF lines, lowercase and IUPAC letters, N runs, blank lines,
    # odd and varying line lengths (neighbouring lines share a bit4 byte),
    # lines that push a chunk past 65,536 nt, a header ending in '\r'
    parts = []
    for r, n in enumerate((150001, 70003, 5, 131072)):
        parts.append(f">rec{r} description {r}" + ("\r\n" if r % 2 else "\n"))
        left = n
        while left:
            ln = min(left, rng.choice([1, 59, 60, 61, 997, 4096, 65535]))
            seq = "".join(rng.choice("ACGTacgtNnRYKMSWBDHVx") for _ in range(ln))
            eol = rng.choice(["\n", "\r\n", "\n\n"])
            parts.append(seq + eol)
            left -= ln
    text = "".join(parts)
    if not final_newline:
        text = text.rstrip("\n") + "ACGTr"
    with open(path, "w", newline="") as f:
        f.write(text)
