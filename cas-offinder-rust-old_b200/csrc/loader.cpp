// loader.cpp -- genome loaders and request compiler (host side).
//
// Produces the reference's ChromChunkInfo stream (64 Knt chunks of bit4
// one-hot nibbles) tight-packed into one byte stream, which is the layout the
// device keeps resident.  Semantics follow:
//   read_fasta        cas-offinder-lib/src/read_fasta.rs:9-71
//   read_2bit         cas-offinder-lib/src/read_2bit.rs:33-118
//   read_fasta_folder cas-offinder-lib/src/read_fasta_folder.rs:8-23
//   path dispatch     cas-offinder-cli/src/main.rs:106-121
#include <dirent.h>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "cof_engine.h"

namespace cof {

Bit4Tables::Bit4Tables() {
    // makebit4map / apply_lower (bit4ops.rs:17-47)
    for (int mixed = 0; mixed < 2; ++mixed) {
        uint8_t up[256] = {0};
        up['G'] = 8; up['C'] = 2; up['A'] = 4; up['T'] = 1;
        if (mixed) {
            up['R'] = 12; up['Y'] = 3; up['S'] = 10; up['W'] = 5; up['K'] = 9;
            up['M'] = 6; up['B'] = 11; up['D'] = 13; up['H'] = 7; up['V'] = 14;
            up['N'] = 15;
        }
        std::memset(str2b4[mixed], 0, 256);
        for (int i = 1; i <= 26; ++i) {
            str2b4[mixed][64 + i] = up[64 + i];
            str2b4[mixed][96 + i] = up[64 + i];
        }
    }
    // invert_chrmap (bit4ops.rs:48-59): lowest character code wins
    std::memset(b4str, 0, sizeof b4str);
    for (int c = 255; c >= 0; --c)
        if (str2b4[1][c]) b4str[str2b4[1][c]] = (char)c;
}

const Bit4Tables &bit4() {
    static const Bit4Tables t;
    return t;
}

char complement_char(char c) {
    const Bit4Tables &t = bit4();
    uint8_t v = t.str2b4[1][(uint8_t)c];
    char out = v ? t.b4str[comp4(v)] : c;
    return (char)(out | (c & 0x20));
}

bool is_mixed_base(char c) { return bit4().str2b4[1][(uint8_t)c] != 0; }

uint64_t HostGenome::n_nucl() const {
    uint64_t s = 0;
    for (size_t k = 0; k < start.size(); ++k) s += end[k] - start[k];
    return s;
}

uint32_t HostGenome::add_name(const char *s, size_t n) {
    names.emplace_back(s, n);
    return (uint32_t)(names.size() - 1);
}

int HostGenome::add_chunk(uint32_t name, uint64_t cs, uint64_t ce, const uint8_t *bytes,
                          Error &err) {
    if ((deferred || deferred_fa) && materialize(err)) return err.code;
    if (ce < cs || ce - cs > kChunkSize) {
        err = {kBadInput, "chunk must hold 0..65536 nucleotides"};
        return err.code;
    }
    if (!start.empty() && cs != 0 && end.back() != cs) {
        // search.rs:1396-1399
        err = {kBadInput, "search expects chromosome chunks to arrive in order"};
        return err.code;
    }
    size_t nb = (size_t)((ce - cs + 1) / 2);
    name_idx.push_back(name);
    start.push_back(cs);
    end.push_back(ce);
    data.insert(data.end(), bytes, bytes + nb);
    boff.push_back(data.size());
    return kOk;
}

namespace {

struct File {
    FILE *f = nullptr;
    ~File() {
        if (f) std::fclose(f);
    }
};

// Reads a whole file.
int slurp(const std::string &path, std::vector<char> &buf, Error &err) {
    File fh;
    fh.f = std::fopen(path.c_str(), "rb");
    if (!fh.f) {
        err = {kIo, "cannot open " + path + ": " + std::strerror(errno)};
        return err.code;
    }
    std::fseek(fh.f, 0, SEEK_END);
    long sz = std::ftell(fh.f);
    std::fseek(fh.f, 0, SEEK_SET);
    if (sz < 0) {
        err = {kIo, "cannot size " + path};
        return err.code;
    }
    buf.resize((size_t)sz);
    if (sz && std::fread(buf.data(), 1, (size_t)sz, fh.f) != (size_t)sz) {
        err = {kIo, "short read on " + path};
        return err.code;
    }
    return kOk;
}

// read_fasta.rs:9-71 over an in-memory file.  Lines end at '\n' with one
// preceding '\r' dropped (BufRead::lines).  Genome characters use the mixed
// base map (N -> 0xF, IUPAC -> union, anything else -> 0).
//
// Two passes.  A sequential scan of the line ends decides the chunks exactly
// as read_fasta.rs does (a record's lines fill a chunk until the next line
// would take it past 65536 nt) and records, for each chunk, its record,
// range and the file span of its lines.  Then every host thread converts a
// share of the chunks straight into the genome's byte array, at offsets known
// from the chunk sizes.
int parse_fasta(HostGenome &g, const char *buf, size_t n, Error &err) {
    struct Span {
        uint32_t name;
        uint64_t cs, ce;
        const char *fb, *fe;  // the chunk's lines: file bytes [fb, fe)
    };
    std::vector<Span> spans;
    const char *p = buf, *e = buf + n;
    bool started = false, have_name = false;
    uint32_t name = 0;
    uint64_t cs = 0, ce = 0;
    const char *fb = p;
    while (p < e) {
        const char *nl = (const char *)std::memchr(p, '\n', (size_t)(e - p));
        const char *le = nl ? nl : e;
        const char *next = nl ? nl + 1 : e;
        size_t len = (size_t)(le - p);
        if (nl && len && p[len - 1] == '\r') --len;
        if (len >= 1 && p[0] == '>') {
            if (ce != cs) spans.push_back({name, cs, ce, fb, p});
            name = g.add_name(p + 1, len - 1);
            have_name = len > 1;
            cs = ce = 0;
            fb = next;
            started = true;
        } else {
            if (!started) {
                err = {kBadInput, "fasta file needs to start with >"};
                return err.code;
            }
            if (!have_name) {
                err = {kBadInput, "> must be followed by chromosome name"};
                return err.code;
            }
            if (len + (size_t)(ce - cs) > kChunkSize) {
                spans.push_back({name, cs, ce, fb, p});
                cs = ce;
                fb = p;
            }
            if (len > kChunkSize) {
                err = {kBadInput, "line in fasta too long"};
                return err.code;
            }
            ce += len;
        }
        p = next;
    }
    if (ce > cs) spans.push_back({name, cs, ce, fb, e});

    // chunk table, then the bytes of every chunk in parallel
    const size_t k0 = g.start.size();
    uint64_t total = g.data.size();
    for (const Span &sp : spans) {
        if (!g.start.empty() && sp.cs != 0 && g.end.back() != sp.cs) {
            err = {kBadInput, "search expects chromosome chunks to arrive in order"};
            return err.code;
        }
        g.name_idx.push_back(sp.name);
        g.start.push_back(sp.cs);
        g.end.push_back(sp.ce);
        total += (sp.ce - sp.cs + 1) / 2;
        g.boff.push_back(total);
    }
    g.data.resize(total, 0);
    const uint8_t *m = bit4().str2b4[1];
    auto convert = [&](size_t a, size_t b) {
        for (size_t k = a; k < b; ++k) {
            const Span &sp = spans[k];
            uint8_t *out = g.data.data() + g.boff[k0 + k];
            uint64_t o = 0;
            for (const char *q = sp.fb; q < sp.fe;) {
                const char *nl = (const char *)std::memchr(q, '\n', (size_t)(sp.fe - q));
                const char *le = nl ? nl : sp.fe;
                size_t len = (size_t)(le - q);
                if (nl && len && q[len - 1] == '\r') --len;
                const uint8_t *s = (const uint8_t *)q;
                size_t i = 0;
                if ((o & 1) && len) {
                    out[o >> 1] |= (uint8_t)(m[s[0]] << 4);
                    i = 1;
                }
                for (; i + 1 < len; i += 2)
                    out[(o + i) >> 1] = (uint8_t)(m[s[i]] | (m[s[i + 1]] << 4));
                if (i < len) out[(o + i) >> 1] |= m[s[i]];
                o += len;
                q = nl ? nl + 1 : sp.fe;
            }
        }
    };
    const size_t nsp = spans.size();
    const unsigned nt = std::max(1u, std::min(std::thread::hardware_concurrency(), 32u));
    if (nt == 1 || nsp < 64) {
        convert(0, nsp);
    } else {
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nt; ++t) {
            const size_t a = nsp * t / nt, b = nsp * (t + 1) / nt;
            if (a < b) th.emplace_back(convert, a, b);
        }
        for (auto &x : th) x.join();
    }
    return kOk;
}

// A read-only view of a whole file (mmap; read into memory where mapping
// fails).
struct FileView {
    const char *p = nullptr;
    size_t n = 0;
    void *map = nullptr;
    std::vector<char> copy;
    ~FileView() {
        if (map) ::munmap(map, n);
    }
    int open(const std::string &path, Error &err) {
        const int fd = ::open(path.c_str(), O_RDONLY);
        if (fd < 0) {
            err = {kIo, "cannot open " + path + ": " + std::strerror(errno)};
            return err.code;
        }
        struct stat st;
        if (::fstat(fd, &st) == 0 && st.st_size > 0) {
            n = (size_t)st.st_size;
            void *m = ::mmap(nullptr, n, PROT_READ, MAP_PRIVATE, fd, 0);
            if (m != MAP_FAILED) {
                map = m;
                p = (const char *)m;
                ::madvise(m, n, MADV_SEQUENTIAL);
            }
        }
        ::close(fd);
        if (p) return kOk;
        n = 0;
        if (int rc = slurp(path, copy, err)) return rc;
        p = copy.data();
        n = copy.size();
        return kOk;
    }
};

// A byte range of a file (the .2bit reader's view of it).
struct FileBytes {
    const char *p;
    size_t n;
    size_t size() const { return n; }
    const char *data() const { return p; }
    char operator[](size_t i) const { return p[i]; }
};

uint32_t rd32(const FileBytes &b, size_t &o, bool &ok) {
    if (o + 4 > b.size()) {
        ok = false;
        return 0;
    }
    uint32_t v;
    std::memcpy(&v, b.data() + o, 4);
    o += 4;
    return v;
}

// read_fasta.rs:9-71, the chunk decisions only, for a FASTA file whose
// bases the device converts.  Every host thread measures the lines of its
// share of the file (a share ends just after a '\n'): each line's length,
// with one '\r' before its '\n' dropped, and whether it is a header.  Then
// one sequential pass over those lengths applies parse_fasta's rules -- the
// same chunks, names and errors -- and records each chunk as a range of line
// indices.
int index_fasta(HostGenome &g, const char *buf, size_t n, FastaPlan &plan, Error &err) {
    constexpr uint32_t kHdr = 0x80000000u;
    const unsigned nt = (unsigned)std::max<size_t>(
        1, std::min<size_t>(n >> 20, std::min(32u, std::max(1u, std::thread::hardware_concurrency()))));
    std::vector<size_t> cut(nt + 1, n);
    cut[0] = 0;
    for (unsigned t = 1; t < nt; ++t) {
        size_t c = std::max(cut[t - 1], n * t / nt);
        const char *nl = c < n ? (const char *)std::memchr(buf + c, '\n', n - c) : nullptr;
        cut[t] = nl ? (size_t)(nl - buf) + 1 : n;
    }
    std::vector<std::vector<uint32_t>> lens(nt);
    std::vector<std::vector<uint64_t>> hdrs(nt);  // file offsets of header lines
    std::vector<int> too_long(nt, 0);
    auto scan = [&](unsigned t) {
        const char *p = buf + cut[t], *e = buf + cut[t + 1];
        auto &L = lens[t];
        L.reserve((size_t)(e - p) / 61 + 16);
        while (p < e) {
            const char *nl = (const char *)std::memchr(p, '\n', (size_t)(e - p));
            const char *le = nl ? nl : e;
            size_t len = (size_t)(le - p);
            if (nl && len && p[len - 1] == '\r') --len;
            if (len >= kHdr) {
                too_long[t] = 1;
                return;
            }
            const bool hdr = len >= 1 && p[0] == '>';
            if (hdr) hdrs[t].push_back((uint64_t)(p - buf));
            L.push_back((uint32_t)len | (hdr ? kHdr : 0u));
            p = nl ? nl + 1 : e;
        }
    };
    if (nt == 1) {
        scan(0);
    } else {
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nt; ++t) th.emplace_back(scan, t);
        for (auto &x : th) x.join();
    }
    for (unsigned t = 0; t < nt; ++t)
        if (too_long[t]) {
            err = {kBadInput, "line in fasta too long"};
            return err.code;
        }
    struct Span {
        uint32_t name;
        uint64_t cs, ce, fl, el;  // nucleotides [cs, ce); lines [fl, el)
    };
    std::vector<Span> spans;
    bool started = false, have_name = false;
    uint32_t name = 0;
    uint64_t cs = 0, ce = 0, fl = 0, li = 0;
    for (unsigned t = 0; t < nt; ++t) {
        size_t h = 0;
        for (uint32_t v : lens[t]) {
            const size_t len = v & ~kHdr;
            if (v & kHdr) {
                if (ce != cs) spans.push_back({name, cs, ce, fl, li});
                name = g.add_name(buf + hdrs[t][h++] + 1, len - 1);
                have_name = len > 1;
                cs = ce = 0;
                fl = li + 1;
                started = true;
            } else {
                if (!started) {
                    err = {kBadInput, "fasta file needs to start with >"};
                    return err.code;
                }
                if (!have_name) {
                    err = {kBadInput, "> must be followed by chromosome name"};
                    return err.code;
                }
                if (len + (size_t)(ce - cs) > kChunkSize) {
                    spans.push_back({name, cs, ce, fl, li});
                    cs = ce;
                    fl = li;
                }
                if (len > kChunkSize) {
                    err = {kBadInput, "line in fasta too long"};
                    return err.code;
                }
                ce += len;
            }
            ++li;
        }
    }
    if (ce > cs) spans.push_back({name, cs, ce, fl, li});
    plan.file_bytes = n;
    plan.n_lines = li;
    uint64_t total = g.boff.back();
    for (const Span &sp : spans) {
        if (!g.start.empty() && sp.cs != 0 && g.end.back() != sp.cs) {
            err = {kBadInput, "search expects chromosome chunks to arrive in order"};
            return err.code;
        }
        g.name_idx.push_back(sp.name);
        g.start.push_back(sp.cs);
        g.end.push_back(sp.ce);
        plan.first_line.push_back(sp.fl);
        plan.last_line.push_back(sp.el);
        plan.out.push_back(total);
        plan.nt.push_back((uint32_t)(sp.ce - sp.cs));
        total += (sp.ce - sp.cs + 1) / 2;
        g.boff.push_back(total);
    }
    return kOk;
}

// read_2bit.rs:33-118, first half: the header, the index, and per record
// its length and N blocks.  Sequences are taken one after the other in index
// order (the stored offsets are skipped, as the reference does).  Appends the
// chunk table to g and describes every chunk's bases in plan: the file
// offset of its packed bytes, and the N ranges the reference's loop writes
// into it.  That loop keeps its N-block index across a record's chunks and
// steps back by one at each chunk; it is replayed here without touching any
// bases.
int index_2bit(HostGenome &g, const FileBytes &b, TwoBitPlan &plan, Error &err) {
    bool ok = true;
    size_t o = 0;
    auto trunc = [&]() {
        err = {kBadInput, "truncated .2bit file"};
        return err.code;
    };
    if (rd32(b, o, ok) != 0x1A412743u || !ok) {
        err = {kBadInput, ".2bit file badly formatted header"};
        return err.code;
    }
    if (rd32(b, o, ok) != 0 || !ok) {
        err = {kBadInput, "only supports version 0 of .2bit format"};
        return err.code;
    }
    uint32_t cnt = rd32(b, o, ok);
    o += 4;
    if (!ok) return trunc();
    std::vector<uint32_t> names(cnt);
    for (uint32_t i = 0; i < cnt; ++i) {
        if (o + 1 > b.size()) return trunc();
        uint8_t nl = (uint8_t)b[o++];
        if (o + nl + 4 > b.size()) return trunc();
        names[i] = g.add_name(b.data() + o, nl);
        o += nl + 4;
    }
    plan.file_bytes = b.size();
    plan.pieces.clear();
    plan.nr.clear();
    plan.raw_begin = b.size();
    plan.raw_end = 0;
    std::vector<uint32_t> piece_rec;
    std::vector<uint64_t> piece_pos;
    std::vector<std::pair<uint32_t, uint32_t>> nb;
    for (uint32_t s = 0; s < cnt; ++s) {
        uint32_t chrlen = rd32(b, o, ok);
        uint32_t nbc = rd32(b, o, ok);
        if (!ok) return trunc();
        nb.assign(nbc, {0, 0});
        for (uint32_t i = 0; i < nbc; ++i) nb[i].first = rd32(b, o, ok);
        for (uint32_t i = 0; i < nbc; ++i) nb[i].second = rd32(b, o, ok);
        if (!ok) return trunc();
        std::stable_sort(nb.begin(), nb.end(),
                         [](const std::pair<uint32_t, uint32_t> &x,
                            const std::pair<uint32_t, uint32_t> &y) { return x.first < y.first; });
        uint32_t mbc = rd32(b, o, ok);
        if (!ok) return trunc();
        o += (uint32_t)(mbc * 8u + 4u);
        size_t pos = 0;
        int64_t bmi = 0;
        while (pos < chrlen) {
            const size_t rs = std::min<size_t>(chrlen - pos, kChunkSize);
            const size_t nbytes = (rs + 3) / 4;
            if (o + nbytes > b.size()) return trunc();
            bmi = std::max<int64_t>(bmi - 1, 0);
            plan.pieces.push_back({o, 0, (uint32_t)rs, (uint32_t)(plan.nr.size() / 2)});
            piece_rec.push_back(s);
            piece_pos.push_back(pos);
            // memsetbit4 of every N block the loop reaches in this chunk,
            // clipped to the chunk (the block end wraps at 32 bits, as the
            // reference's u32 sum does)
            while (bmi < (int64_t)nbc && (int64_t)nb[bmi].first - (int64_t)pos <= (int64_t)rs) {
                const int64_t bs = (int64_t)nb[bmi].first - (int64_t)pos;
                const int64_t be =
                    (int64_t)(uint32_t)(nb[bmi].first + nb[bmi].second) - (int64_t)pos;
                const int64_t lo = std::max<int64_t>(bs, 0);
                const int64_t hi = std::min<int64_t>(std::max<int64_t>(be, 0), (int64_t)rs);
                if (lo < hi) {
                    plan.nr.push_back((uint32_t)lo);
                    plan.nr.push_back((uint32_t)hi);
                }
                ++bmi;
            }
            plan.raw_begin = std::min<uint64_t>(plan.raw_begin, o);
            plan.raw_end = std::max<uint64_t>(plan.raw_end, o + nbytes);
            o += nbytes;
            pos += rs;
        }
    }
    if (plan.pieces.empty()) plan.raw_begin = plan.raw_end = 0;
    // chunk table
    uint64_t total = g.boff.back();
    for (size_t k = 0; k < plan.pieces.size(); ++k) {
        TwoBitPlan::Piece &pc = plan.pieces[k];
        const uint64_t pos = piece_pos[k];
        if (!g.start.empty() && pos != 0 && g.end.back() != pos) {
            err = {kBadInput, "search expects chromosome chunks to arrive in order"};
            return err.code;
        }
        g.name_idx.push_back(names[piece_rec[k]]);
        g.start.push_back(pos);
        g.end.push_back(pos + pc.rs);
        pc.out = total;
        total += (pc.rs + 1) / 2;
        g.boff.push_back(total);
    }
    plan.pieces.push_back({0, total, 0, (uint32_t)(plan.nr.size() / 2)});
    return kOk;
}

// read_2bit.rs:33-118, second half, on all host threads: each chunk's bases
// (BIT2_TO_BIT4, bit4ops.rs:60-75: codes T=0 C=1 A=2 G=3, first base in the
// high bits of each byte), zero padding after the last base, then the N
// ranges, written into g.data at the chunk's byte offset.
void convert_2bit_host(HostGenome &g, const FileBytes &b, const TwoBitPlan &plan) {
    uint16_t b2b4[256];
    for (int i = 0; i < 256; ++i) {
        uint16_t v = 0;
        for (int j = 0; j < 4; ++j) v |= (uint16_t)((1u << ((i >> ((3 - j) * 2)) & 3)) << (4 * j));
        b2b4[i] = v;
    }
    g.data.resize(plan.pieces.back().out, 0);
    const size_t np = plan.pieces.size() - 1;
    auto convert = [&](size_t a, size_t z) {
        std::vector<uint8_t> cur(kChunkBytes);
        for (size_t k = a; k < z; ++k) {
            const TwoBitPlan::Piece &pc = plan.pieces[k];
            const size_t rs = pc.rs, nbytes = (rs + 3) / 4;
            const uint8_t *raw = (const uint8_t *)b.data() + pc.raw;
            std::fill(cur.begin(), cur.end(), 0);
            for (size_t i = 0; i < nbytes; ++i) {
                uint16_t v = b2b4[raw[i]];
                cur[2 * i] = (uint8_t)v;
                cur[2 * i + 1] = (uint8_t)(v >> 8);
            }
            auto setn = [&](size_t lo, size_t hi, uint8_t v) {  // memsetbit4
                for (size_t i = lo; i < hi; ++i) {
                    if (i & 1) cur[i >> 1] = (uint8_t)((cur[i >> 1] & 0x0F) | (v << 4));
                    else cur[i >> 1] = (uint8_t)((cur[i >> 1] & 0xF0) | v);
                }
            };
            if (rs % 4) setn(rs, nbytes * 4, 0);
            for (uint32_t r = pc.nr; r < plan.pieces[k + 1].nr; ++r)
                setn(plan.nr[2 * r], plan.nr[2 * r + 1], 0xF);
            std::memcpy(g.data.data() + pc.out, cur.data(), (rs + 1) / 2);
        }
    };
    const unsigned nt = std::max(1u, std::min(std::thread::hardware_concurrency(), 32u));
    if (nt == 1 || np < 64) {
        convert(0, np);
    } else {
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nt; ++t) {
            const size_t lo = np * t / nt, hi = np * (t + 1) / nt;
            if (lo < hi) th.emplace_back(convert, lo, hi);
        }
        for (auto &x : th) x.join();
    }
}

int parse_2bit(HostGenome &g, const FileBytes &b, Error &err) {
    TwoBitPlan plan;
    if (int rc = index_2bit(g, b, plan, err)) return rc;
    convert_2bit_host(g, b, plan);
    return kOk;
}

}  // namespace

int load_genome_path(HostGenome &g, const std::string &path, Error &err) {
    if ((g.deferred || g.deferred_fa) && g.materialize(err)) return err.code;  // appending to it
    struct stat st;
    if (::stat(path.c_str(), &st)) {
        err = {kIo, "cannot stat " + path};
        return err.code;
    }
    std::vector<char> buf;
    if (S_ISDIR(st.st_mode)) {
        DIR *d = ::opendir(path.c_str());
        if (!d) {
            err = {kIo, "cannot open folder " + path};
            return err.code;
        }
        int rc = kOk;
        while (struct dirent *e = ::readdir(d)) {
            std::string nm = e->d_name;
            if (nm == "." || nm == "..") continue;
            std::string p = path;
            if (p.empty() || p.back() != '/') p += '/';
            p += nm;
            struct stat fs;
            if (::stat(p.c_str(), &fs) || !S_ISREG(fs.st_mode)) continue;
            if (p.size() >= 3 && p.compare(p.size() - 3, 3, ".fa") == 0) {
                FileView fv;
                if ((rc = fv.open(p, err))) break;
                if ((rc = parse_fasta(g, fv.p, fv.n, err))) break;
            }
        }
        ::closedir(d);
        return rc;
    }
    FileView fv;
    if (int rc = fv.open(path, err)) return rc;
    if (fv.n == 0) {
        err = {kIo, "cannot read " + path};
        return err.code;
    }
    if (fv.p[0] == '>') {
        if (g.n_chunks() == 0) {
            // one FASTA file into an empty genome: the chunks are decided
            // here; the device converts the bases at upload
            auto plan = std::make_shared<FastaPlan>();
            plan->path = path;
            if (int rc = index_fasta(g, fv.p, fv.n, *plan, err)) return rc;
            if (!plan->first_line.empty()) g.deferred_fa = plan;
            return kOk;
        }
        return parse_fasta(g, fv.p, fv.n, err);
    }
    if (g.n_chunks() == 0) {
        // a .2bit file into an empty genome: only the index is read here;
        // the device decodes the bases at upload
        auto plan = std::make_shared<TwoBitPlan>();
        plan->path = path;
        if (int rc = index_2bit(g, FileBytes{fv.p, fv.n}, *plan, err)) return rc;
        if (plan->pieces.size() > 1) g.deferred = plan;
        return kOk;
    }
    return parse_2bit(g, FileBytes{fv.p, fv.n}, err);
}

int HostGenome::materialize(Error &err) {
    if (deferred_fa) {
        FileView fv;
        if (int rc = fv.open(deferred_fa->path, err)) return rc;
        if (fv.n != deferred_fa->file_bytes) {
            err = {kIo, deferred_fa->path + " changed since it was loaded"};
            return err.code;
        }
        HostGenome tmp;  // the same chunks, converted on the host
        if (int rc = parse_fasta(tmp, fv.p, fv.n, err)) return rc;
        if (tmp.n_bytes() != n_bytes()) {
            err = {kIo, deferred_fa->path + " changed since it was loaded"};
            return err.code;
        }
        data = std::move(tmp.data);
        deferred_fa.reset();
        return kOk;
    }
    if (!deferred) return kOk;
    FileView fv;
    if (int rc = fv.open(deferred->path, err)) return rc;
    if (fv.n != deferred->file_bytes) {
        err = {kIo, deferred->path + " changed since it was loaded"};
        return err.code;
    }
    convert_2bit_host(*this, FileBytes{fv.p, fv.n}, *deferred);
    deferred.reset();
    return kOk;
}

bool Tuner::enabled() const {
    const char *e = std::getenv("COF_AUTOTUNE");
    return !(e && std::strcmp(e, "0") == 0);
}

void Tuner::load() {
    if (loaded_) return;
    loaded_ = true;
    const char *path = std::getenv("COF_TUNE_CACHE");
    if (!path) return;
    FILE *f = std::fopen(path, "r");
    if (!f) return;
    char key[256];
    int v;
    while (std::fscanf(f, "%255s %d", key, &v) == 2) cache_[key] = v;
    std::fclose(f);
}

bool Tuner::lookup(const std::string &key, int &variant) {
    load();
    auto it = cache_.find(key);
    if (it == cache_.end()) return false;
    variant = it->second;
    return true;
}

void Tuner::store(const std::string &key, int variant) {
    cache_[key] = variant;
    const char *path = std::getenv("COF_TUNE_CACHE");
    if (!path) return;
    if (FILE *f = std::fopen(path, "a")) {
        std::fprintf(f, "%s %d\n", key.c_str(), variant);
        std::fclose(f);
    }
}

std::string Tuner::report() const {
    std::string out = "{";
    for (const auto &kv : cache_) {
        if (out.size() > 1) out += ", ";
        out += "\"" + kv.first + "\": " + std::to_string(kv.second);
    }
    return out + "}";
}

int make_request(const char *filter, size_t pattern_len, const char *const *patterns,
                 size_t n_patterns, uint32_t mm, uint32_t db, uint32_t rb, uint32_t flags,
                 uint32_t cps, Request &out, Error &err) {
    auto bad = [&](const std::string &m, int code = kBadInput) {
        err = {code, m};
        return code;
    };
    if (!filter || !patterns || n_patterns == 0) return bad("no patterns");  // search.rs:1502
    if (std::strlen(filter) != pattern_len) return bad("search filter length != pattern_len");
    if (pattern_len == 0) return bad("empty pattern");
    for (size_t i = 0; i < pattern_len; ++i)
        if (!is_mixed_base(filter[i])) return bad("search filter must be a mixed base string");
    out = Request();
    out.filter = filter;
    out.max_mm = mm;
    out.max_db = db;
    out.max_rb = rb;
    out.cps = cps ? cps : kDefaultCps;
    if (out.cps < 2) return bad("chunks_per_search must be >= 2");
    for (size_t i = 0; i < n_patterns; ++i) {
        if (!patterns[i]) return bad("null pattern");
        std::string p = patterns[i];
        if (p.size() != pattern_len) return bad("All patterns must have same length");  // :1503-1507
        for (char c : p)
            if (!is_mixed_base(c)) return bad("pattern must be a mixed base string");
        out.patterns.push_back(p);
    }
    out.raw = (flags & 2u) != 0;  // COF_F_RAW_MATCHES
    if (flags & 1u) {  // COF_F_ADD_REVCOMP: main.rs:253-259
        for (size_t i = 0; i < n_patterns; ++i) {
            std::string r = out.patterns[i];
            for (char &c : r) c = complement_char(c);
            std::reverse(r.begin(), r.end());
            out.patterns.push_back(r);
        }
    }
    for (size_t i = pattern_len; i > 0; --i) {  // main.rs:80-91
        char c = out.patterns[0][i - 1];
        if (c == 'N' || c == 'n') ++out.pam_len;
        else break;
    }
    bool myers = db > 0 || rb > 0;
    if (pattern_len > kMaxPatternLen)
        return bad("pattern length above 64 is not supported (at most 64 cells)", kUnsupported);
    if (!myers && mm >= pattern_len)
        return bad("max_mismatches must be below the pattern length");
    if (myers && (db > 8 || rb > 8 || mm + db + rb > 30))
        return bad("bulge / edit limits above 8 bulges or 30 edits are not supported",
                   kUnsupported);
    return kOk;
}

}  // namespace cof
