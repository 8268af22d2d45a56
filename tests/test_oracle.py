"""CPU tests of the oracle (the C restatement in oracle/) against the
reference's own golden vectors and against an independent Python
restatement (tests/bruteforce.py)."""
import os
import shutil

import pytest

import bruteforce
import randgen


def _expected(golden):
    with open(os.path.join(golden, "expected.txt"), "rb") as f:
        return f.read()


# cas-offinder-lib/tests/file_test.rs:34-73: every reader decodes
# upstream1000 to expected.txt
@pytest.mark.parametrize("name", ["upstream1000.fa", "upstream1000.2bit"])
def test_reader_golden(oracle_mod, golden, name):
    g = oracle_mod.OracleGenome(os.path.join(golden, name))
    assert g.decode() == _expected(golden)


def test_reader_golden_folder(oracle_mod, golden, tmp_path):
    shutil.copyfile(os.path.join(golden, "upstream1000.fa"), tmp_path / "upstream1000.fa")
    shutil.copyfile(os.path.join(golden, "upstream1000.2bit"), tmp_path / "upstream1000.2bit")
    shutil.copyfile(os.path.join(golden, "expected.txt"), tmp_path / "expected.txt")
    g = oracle_mod.OracleGenome(str(tmp_path))
    assert g.decode() == _expected(golden)


def test_reader_chunking(oracle_mod, golden):
    # 13 records (12 x 1000 nt + 1 x 507 nt), one chunk each
    g = oracle_mod.OracleGenome(os.path.join(golden, "upstream1000.fa"))
    ch = g.chunks()
    assert len(ch) == 13
    assert sorted(e - s for _, _, s, e in ch) == [507] + [1000] * 12


# integration_bulge.rs:156-176: the popcount path finds exactly 117 rows
@pytest.mark.parametrize("cps", [64, 16384, 2])
def test_kat_117_rows(oracle_mod, golden, cps):
    g = oracle_mod.OracleGenome(os.path.join(golden, "upstream1000.fa"))
    text, n = g.search("N" * 24, ["CCGTGGTTCAACATTTGCTTAGCA", "GATGTTGGTAAGTGGGATATGGCA"], 11,
                       chunks_per_search=cps)
    assert n == 117
    with open(os.path.join(golden, "kat_popcount_rows.txt")) as f:
        assert sorted(text.splitlines()) == f.read().splitlines()


def test_kat_2bit_same_sites(oracle_mod, golden):
    # the .2bit names drop the FASTA description; sites are identical
    fa = oracle_mod.OracleGenome(os.path.join(golden, "upstream1000.fa"))
    tb = oracle_mod.OracleGenome(os.path.join(golden, "upstream1000.2bit"))
    args = ("N" * 24, ["CCGTGGTTCAACATTTGCTTAGCA", "GATGTTGGTAAGTGGGATATGGCA"], 11)

    def strip(text):
        out = []
        for row in text.splitlines():
            c = row.split("\t")
            c[3] = c[3].split(" ")[0]
            out.append("\t".join(c))
        return sorted(out)

    assert strip(fa.search(*args)[0]) == strip(tb.search(*args)[0])


# integration_bulge.rs:208-259: the bulge path finds rows, 8 columns, types
def test_kat_bulge_rows(oracle_mod, golden):
    g = oracle_mod.OracleGenome(os.path.join(golden, "upstream1000.fa"))
    text, n = g.search("N" * 25 + "GG", ["CCGTGGTTCAACATTTGCTTAGCANNN"], 5, 1, 1,
                       chunks_per_search=64)
    rows = sorted(text.splitlines())
    assert n >= 1
    for r in rows:
        c = r.split("\t")
        assert len(c) == 8 and c[0] in ("X", "DNA", "RNA")
    with open(os.path.join(golden, "kat_bulge_rows.txt")) as f:
        assert rows == f.read().splitlines()


def _oracle_from_chunks(oracle_mod, chunks):
    g = oracle_mod.OracleGenome()
    for name, data, _nibs, s, e in chunks:
        g.add_chunk(name, data, s, e)
    return g


@pytest.mark.parametrize("seed", range(12))
def test_oracle_vs_bruteforce_popcount(oracle_mod, seed):
    case = randgen.random_case(seed)
    g = _oracle_from_chunks(oracle_mod, case["chunks"])
    text, _ = g.search(case["filter"], case["patterns"], case["mm"],
                       chunks_per_search=case["cps"])
    bf = bruteforce.search([(n, nb, s, e) for n, _d, nb, s, e in case["chunks"]],
                           case["filter"], case["patterns"], case["mm"], cps=case["cps"])
    assert sorted(text.splitlines()) == bf
    assert len(bf) > 0


@pytest.mark.parametrize("seed", range(8))
def test_oracle_vs_bruteforce_bulge(oracle_mod, seed):
    case = randgen.random_case(100 + seed, bulge=True)
    g = _oracle_from_chunks(oracle_mod, case["chunks"])
    text, _ = g.search(case["filter"], case["patterns"], case["mm"], case["db"], case["rb"],
                       chunks_per_search=case["cps"])
    bf = bruteforce.search([(n, nb, s, e) for n, _d, nb, s, e in case["chunks"]],
                           case["filter"], case["patterns"], case["mm"], case["db"],
                           case["rb"], cps=case["cps"])
    assert sorted(text.splitlines()) == bf


def test_bruteforce_fasta_chunking(oracle_mod, tmp_path):
    # the brute-force FASTA chunker and the oracle's read_fasta agree on an
    # input with odd line lengths and long records (several 64 Knt chunks)
    rng = __import__("random").Random(7)
    recs = [randgen.random_seq(rng, n) for n in (140_001, 3, 70_000)]
    lines = []
    for i, s in enumerate(recs):
        lines.append(f">r{i} x")
        w = [61, 3, 77][i]
        lines += [s[j:j + w] for j in range(0, len(s), w)]
    text = "\n".join(lines) + "\n"
    p = tmp_path / "g.fa"
    p.write_text(text)
    g = oracle_mod.OracleGenome(str(p))
    bf = bruteforce.chunks_from_fasta_text(text)
    got = [(n, s, e) for n, _d, s, e in g.chunks()]
    assert got == [(n, s, e) for n, _nb, s, e in bf]


@pytest.mark.parametrize("seed", [0, 1, 2, 3, 104, 105])
def test_oracle_raw_matches_vs_bruteforce(oracle_mod, seed):
    case = randgen.random_case(seed, bulge=seed >= 100)
    g = _oracle_from_chunks(oracle_mod, case["chunks"])
    text, _ = g.search(case["filter"], case["patterns"], case["mm"], case["db"], case["rb"],
                       chunks_per_search=case["cps"], raw=True)
    bf = bruteforce.search([(n, nb, s, e) for n, _d, nb, s, e in case["chunks"]],
                           case["filter"], case["patterns"], case["mm"], case["db"], case["rb"],
                           cps=case["cps"], raw=True)
    assert sorted(text.split("\n")[:-1]) == bf and len(bf) > 0


def test_reference_kernel_launcher_loads():
    # oracle/_ref/: the reference's kernels for sm_100a and their launcher
    import ref_gpu
    if not ref_gpu.available():
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    lib = ref_gpu.lib()
    for sym in ("refgpu_open", "refgpu_n_batches", "refgpu_batch", "refgpu_close",
                "refgpu_popcount_count", "refgpu_popcount_run", "refgpu_myers_run"):
        assert hasattr(lib, sym)
    assert os.path.exists(ref_gpu.popcount_cubin(23))
    assert os.path.exists(ref_gpu.myers_cubin(23, 3, 4, 2, 2))


def test_synth_2bit_writer(oracle_mod, tmp_path):
    # the benchmark's numpy .2bit writer: byte-identical to the plain test
    # writer, and read by the oracle as the same genome as its FASTA
    # (odd lengths, a record that is all N, N runs at both ends)
    import numpy as np
    import synth
    import twobit
    rng = np.random.default_rng(9)
    gen = synth.make_genome(rng, [70001, 7, 3, 64, 5], n_runs=[(0, 500), (0, 37), (3, 10)])
    gen.records[2][:] = 15
    gen.records[4][0] = gen.records[4][-1] = 15
    gen.write_2bit(str(tmp_path / "a.2bit"))
    twobit.write_2bit(str(tmp_path / "b.2bit"),
                      [(n, bytes(synth._CHARS[r]).decode()) for n, r in zip(gen.names, gen.records)])
    assert (tmp_path / "a.2bit").read_bytes() == (tmp_path / "b.2bit").read_bytes()
    gen.write_fasta(str(tmp_path / "a.fa"))
    a = oracle_mod.OracleGenome(str(tmp_path / "a.2bit"))
    b = oracle_mod.OracleGenome(str(tmp_path / "a.fa"))
    assert a.decode() == b.decode()
