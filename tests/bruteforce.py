"""Independent pure-Python restatement of the reference search, for small
inputs.  Test infrastructure: it cross-checks the C oracle (oracle/) with
different arithmetic -- per-character comparisons instead of u64 popcount
blocks, and for the bulge path the DP bound alone instead of the Myers sweep
(every row the reference emits has dp[m][n] <= max_edits, which bounds the
windowed Myers score from above, so the sweep never removes a row).

Follows cas-offinder-lib/src/search.rs (batcher 1531-1572, popcount path
378-546 + 1428-1488, Myers path 597-1031 + 1316-1374), traceback.rs:181-381
and cas-offinder-cli/src/main.rs:122-242.
"""
import sys

sys.setrecursionlimit(10000)

_UP = {"G": 8, "C": 2, "A": 4, "T": 1, "R": 12, "Y": 3, "S": 10, "W": 5, "K": 9, "M": 6,
       "B": 11, "D": 13, "H": 7, "V": 14, "N": 15}
MIXED = {}
PLAIN = {}
for _c, _v in _UP.items():
    MIXED[_c] = MIXED[_c.lower()] = _v
    if _c in "ACGT":
        PLAIN[_c] = PLAIN[_c.lower()] = _v
DEC = {v: c for c, v in _UP.items()}
DEC[0] = "\0"


def b4(c):
    return MIXED.get(c, 0)


def comp4(v):
    return ((v << 2) | (v >> 2)) & 0xF


def comp_char(c):
    v = MIXED.get(c, 0)
    if not v:
        return c
    out = DEC[comp4(v)]
    return out.lower() if c.islower() else out


def revcomp(s):
    return "".join(comp_char(c) for c in reversed(s))


def cmp_chars(d, r):
    return (PLAIN.get(d, 0) & MIXED.get(r, 0)) != 0


def make_batches(n, cps):
    out, buf, head = [], [], False
    for k in range(n):
        buf.append(k)
        if len(buf) == cps:
            out.append((buf[0], buf[-1], head))
            buf, head = [buf[-1]], True
    if buf and not (head and len(buf) == 1):
        out.append((buf[0], buf[-1], head))
    return out


def _batch(chunks, first, last):
    """nibble buffer (odd chunks padded with one 0 nibble) + byte offsets"""
    buf, offs = [], []
    for k in range(first, last + 1):
        name, nibs, s, e = chunks[k]
        offs.append(len(buf) // 2)
        buf.extend(nibs)
        if len(nibs) % 2:
            buf.append(0)
    offs.append(len(buf) // 2)
    return buf, offs


def _chunk_of(offs, byte_pos):
    idx = 0
    for i, o in enumerate(offs):
        if o <= byte_pos:
            idx = i
    return idx


def _tail(name, pos, fwd, db, mm, size, pam_len):
    if not fwd:
        pos += max(max(pam_len - 1, 0) - db, 0)
    return f"\t{name}\t{pos}\t{'+' if fwd else '-'}\t{mm}\t{size}"


def search(chunks, filt, user_patterns, mm, db=0, rb=0, cps=16384, raw=False):
    """chunks: list of (name, nibble list, chunk_start, chunk_end).
    Returns the sorted list of output rows."""
    pats = list(user_patterns) + [revcomp(p) for p in user_patterns]
    L = len(filt)
    pam_len = 0
    for c in reversed(user_patterns[0]):
        if c in "Nn":
            pam_len += 1
        else:
            break
    rows = []
    for first, last, head in make_batches(len(chunks), cps):
        buf, offs = _batch(chunks, first, last)
        nch = last - first + 1
        meta = [chunks[k] for k in range(first, last + 1)]
        if db == 0 and rb == 0:
            rows += _popcount_batch(buf, offs, meta, nch, head, filt, pats, mm, L, pam_len, raw)
        else:
            rows += _myers_batch(buf, offs, meta, nch, head, filt, pats, mm, db, rb, L, pam_len,
                                 raw)
    return sorted(rows)


def _popcount_batch(buf, offs, meta, nch, head, filt, pats, mm, L, pam_len, raw=False):
    out = []
    gm = [0 if v == 0xF else v for v in buf]  # mask_genome_n_to_zero_inplace
    msmin = max(offs[1] * 2 - (L - 1), 0) if head else 0
    n_fwd = len(pats) // 2
    for p, pat in enumerate(pats):
        pb = [b4(c) for c in pat]
        for s in range(msmin, len(gm)):
            matches = 0
            for i in range(L):
                g = gm[s + i] if s + i < len(gm) else 0
                matches += bin(g & pb[i]).count("1")
            if L - matches > mm:
                continue
            idx = _chunk_of(offs, s // 2)
            name, _nibs, cs, ce = meta[idx]
            pos = cs + (s - offs[idx] * 2)
            end_chrom = idx == nch - 1 or meta[idx + 1][2] == 0
            if end_chrom and pos + L > ce:
                continue
            fwd = p < n_fwd
            dna = [DEC[gm[s + i]] if s + i < len(gm) else "\0" for i in range(L)]
            rna = [DEC[v] for v in pb]
            if not fwd:
                dna = list(revcomp("".join(dna)))
                rna = list(revcomp("".join(rna)))
            if raw:  # search()'s Match, before the writer
                out.append(f"{name}\t{pos}\t{p}\t{'+' if fwd else '-'}\t{max(L - matches, 0)}"
                           f"\t0\t0\t" + "".join(rna) + "\t" + "".join(dna))
                continue
            ok, actual = True, 0
            for i in range(L):
                if filt[i] not in "Nn" and not cmp_chars(dna[i], filt[i]):
                    ok = False
                    break
                if rna[i] not in "Nn" and not cmp_chars(dna[i], rna[i]):
                    actual += 1
            if not ok or actual > mm:
                continue
            mark = []
            for d, r in zip(dna, rna):
                if d == "\0":
                    mark.append("N" if r in "Nn" else "n")
                elif r in "Nn":
                    mark.append(d)
                elif d in "Nn":
                    mark.append("n")
                elif not cmp_chars(d, r):
                    mark.append(d.lower())
                else:
                    mark.append(d)
            out.append("X\t" + "".join(rna) + "\t" + "".join(mark) +
                       _tail(name, pos, fwd, 0, actual, 0, pam_len))
    return out


def _loose(p, t):
    if t == 0:
        return False
    if p == 0xF:
        return True
    if t == 0xF:
        return False
    return (p & t) != 0


def _myers_batch(buf, offs, meta, nch, head, filt, pats, mm, db, rb, L, pam_len, raw=False):
    out = []
    total = offs[-1] * 2
    active = offs[1] * 2 if head else 0
    W = L + db
    E = mm + db + rb
    n_fwd = len(pats) // 2
    rfilt = revcomp(filt)
    INF = 1 << 40
    for p, pat in enumerate(pats):
        pb = [b4(c) for c in pat]
        isn = [c in "Nn" for c in pat]
        eff = [b4(c) for c in (filt if p < n_fwd else rfilt)]
        ps = next((i for i in range(L) if isn[i]), L)
        pf = [eff[i] for i in range(ps, L) if isn[i]]
        for t in range(active, total):
            if t + 1 < L:
                continue
            # check_pam_quick
            ranges = (db + 1, rb + 1) if ps == 0 else (1, 1)
            pam = False
            for bd in range(ranges[0]):
                for br in range(ranges[1]):
                    span = L + bd - br
                    if span <= 0 or span > t + 1:
                        continue
                    a = t + 1 - span
                    ok = True
                    for k, f in enumerate(pf):
                        gp = a + ps + k
                        if gp >= total:
                            ok = False
                            break
                        g = buf[gp]
                        good = (g != 0) if f == 0xF else (g not in (0, 0xF) and (g & f) != 0)
                        if not good:
                            ok = False
                            break
                    if ok:
                        pam = True
                        break
                if pam:
                    break
            if not pam:
                continue
            ts = max(t + 1 - W, 0)
            text = buf[ts:t + 1]
            n = len(text)
            dc = INF if db == 0 else 1
            rc = INF if rb == 0 else 1
            dp = [[0] * (n + 1) for _ in range(L + 1)]
            for i in range(L + 1):
                dp[i][0] = min(i * rc, INF)
            for i in range(1, L + 1):
                for j in range(1, n + 1):
                    if text[j - 1] == 0:
                        dp[i][j] = INF
                        continue
                    mc = 0 if _loose(pb[i - 1], text[j - 1]) else 1
                    dp[i][j] = min(dp[i - 1][j - 1] + mc, dp[i - 1][j] + rc, dp[i][j - 1] + dc)
            if dp[L][n] > E:
                continue
            aligns = []

            def rec(i, j, ops, cost, m_, d_, r_):
                if cost + dp[i][j] > E or m_ > mm or d_ > db or r_ > rb:
                    return
                if i == 0:
                    aligns.append((list(reversed(ops)), j, m_, d_, r_))
                    return
                if j > 0:
                    mc = 0 if _loose(pb[i - 1], text[j - 1]) else 1
                    if not (mc == 1 and isn[i - 1]):
                        rec(i - 1, j - 1, ops + ["S" if mc else "M"], cost + mc, m_ + mc, d_, r_)
                if r_ < rb and rb > 0:
                    if not isn[i - 1] and not (i < L and isn[i]) and not (i >= 2 and isn[i - 2]):
                        rec(i - 1, j, ops + ["R"], cost + 1, m_, d_, r_ + 1)
                if d_ < db and db > 0 and j > 0 and i < L:
                    if not (isn[i - 1] and isn[i]):
                        rec(i, j - 1, ops + ["D"], cost + 1, m_, d_ + 1, r_)

            rec(L, n, [], 0, 0, 0, 0)
            for ops, j, m_, d_, r_ in aligns:
                pa, ta, pi, ti = [], [], 0, j
                okf = True
                for op in ops:
                    if op in "MS":
                        f, g = eff[pi], text[ti]
                        good = (g != 0) if f == 0xF else (g not in (0, 0xF) and (g & f) != 0)
                        if not good:
                            okf = False
                        pa.append(DEC[pb[pi]])
                        ta.append(DEC[g])
                        pi += 1
                        ti += 1
                    elif op == "R":
                        pa.append(DEC[pb[pi]])
                        ta.append("-")
                        pi += 1
                    else:
                        pa.append("-")
                        ta.append(DEC[text[ti]])
                        ti += 1
                if not okf:
                    continue
                span = n - j
                start = t + 1 - span
                idx = _chunk_of(offs, start // 2)
                name, _nibs, cs, ce = meta[idx]
                pos = cs + (start - offs[idx] * 2)
                end_chrom = idx == nch - 1 or meta[idx + 1][2] == 0
                if end_chrom and pos + L + d_ - r_ > ce:
                    continue
                fwd = p < n_fwd
                rna_s, dna_s = "".join(pa), "".join(ta)
                if not fwd:
                    rna_s, dna_s = revcomp(rna_s), revcomp(dna_s)
                if raw:
                    out.append(f"{name}\t{pos}\t{p}\t{'+' if fwd else '-'}\t{m_}\t{d_}\t{r_}\t"
                               + rna_s + "\t" + dna_s)
                    continue
                typ = "X" if d_ + r_ == 0 else ("DNA" if d_ > 0 else "RNA")
                out.append(typ + "\t" + rna_s + "\t" + dna_s +
                           _tail(name, pos, fwd, d_, m_, d_ + r_, pam_len))
    return out


def chunks_from_fasta_text(text):
    """read_fasta.rs:9-71 over a str, returning (name, nibbles, start, end)."""
    out = []
    name, nibs, cs, ce, started = None, [], 0, 0, False
    lines = text.split("\n")
    if lines and lines[-1] == "":
        lines.pop()
    for line in lines:
        if line.endswith("\r"):
            line = line[:-1]
        if line.startswith(">"):
            if ce != cs:
                out.append((name, nibs, cs, ce))
            name, nibs, cs, ce, started = line[1:], [], 0, 0, True
        else:
            assert started and name
            if len(line) + (ce - cs) > 65536:
                out.append((name, nibs, cs, ce))
                nibs, cs = [], ce
            nibs = nibs + [b4(c) for c in line]
            ce += len(line)
    if ce > cs:
        out.append((name, nibs, cs, ce))
    return out
