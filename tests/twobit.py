"""A small .2bit writer for tests (UCSC twoBit v0: header, index, per record
its length, N blocks, mask blocks and 2-bit packed bases T=0 C=1 A=2 G=3,
first base in the high bits).  Lowercase letters become mask blocks, N runs
become N blocks."""
import struct


def write_2bit(path, records):
    """records: list of (name, sequence str over ACGTNacgtn)."""
    code = {"T": 0, "C": 1, "A": 2, "G": 3, "N": 0}
    bodies = []
    for _name, seq in records:
        up = seq.upper()
        nblocks, mblocks = [], []
        for runs, pred in ((nblocks, lambda c: c == "N"), (mblocks, lambda c: c.islower())):
            src = up if runs is nblocks else seq
            i = 0
            while i < len(src):
                if pred(src[i]):
                    j = i
                    while j < len(src) and pred(src[j]):
                        j += 1
                    runs.append((i, j - i))
                    i = j
                else:
                    i += 1
        packed = bytearray()
        for k in range(0, len(up), 4):
            v = 0
            for j in range(4):
                v = (v << 2) | (code[up[k + j]] if k + j < len(up) else 0)
            packed.append(v)
        body = struct.pack("<II", len(seq), len(nblocks))
        body += b"".join(struct.pack("<I", s) for s, _ in nblocks)
        body += b"".join(struct.pack("<I", n) for _, n in nblocks)
        body += struct.pack("<I", len(mblocks))
        body += b"".join(struct.pack("<I", s) for s, _ in mblocks)
        body += b"".join(struct.pack("<I", n) for _, n in mblocks)
        body += struct.pack("<I", 0) + bytes(packed)
        bodies.append(body)
    index_size = sum(1 + len(n) + 4 for n, _ in records)
    off = 16 + index_size
    with open(path, "wb") as f:
        f.write(struct.pack("<IIII", 0x1A412743, 0, len(records), 0))
        for (name, _), body in zip(records, bodies):
            f.write(bytes([len(name)]) + name.encode() + struct.pack("<I", off))
            off += len(body)
        for body in bodies:
            f.write(body)
