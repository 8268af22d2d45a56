"""Regenerates the golden fixtures in this folder.

Copies the reference's own test data (cas-offinder-lib/tests/test_data:
upstream1000.fa, upstream1000.2bit and the reader golden expected.txt) and
records the oracle's rows for the reference's integration inputs
(cas-offinder-lib/tests/integration_bulge.rs:156-259) so that the GPU tests,
which run without the reference tree, compare against the same rows:

  kat_popcount_rows.txt  N x 24 filter, 2 patterns, mm 11 (117 rows, pinned
                         by integration_bulge.rs:156-176)
  kat_bulge_rows.txt     N x 25 + GG filter, db 1 rb 1, mm 5, one pattern
                         (integration_bulge.rs:208-259; CPU == GPU only)

Run from the repository root, with COF_REFERENCE_DIR naming the reference
project's root:  COF_REFERENCE_DIR=<reference> python tests/golden/make_golden.py
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

KAT_POPCOUNT = dict(search_filter="N" * 24,
                    patterns=["CCGTGGTTCAACATTTGCTTAGCA", "GATGTTGGTAAGTGGGATATGGCA"],
                    max_mismatches=11)
KAT_BULGE = dict(search_filter="N" * 25 + "GG", patterns=["CCGTGGTTCAACATTTGCTTAGCANNN"],
                 max_mismatches=5, max_dna_bulges=1, max_rna_bulges=1)


def main():
    ref = os.path.join(os.environ["COF_REFERENCE_DIR"], "cas-offinder-lib", "tests", "test_data")
    for f in ("upstream1000.fa", "upstream1000.2bit", "expected.txt"):
        shutil.copyfile(os.path.join(ref, f), os.path.join(HERE, f))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.build()
    g = oracle.OracleGenome(os.path.join(HERE, "upstream1000.fa"))
    for name, kw in (("kat_popcount_rows.txt", KAT_POPCOUNT), ("kat_bulge_rows.txt", KAT_BULGE)):
        text, n = g.search(**kw, chunks_per_search=64)
        rows = sorted(text.splitlines())
        with open(os.path.join(HERE, name), "w") as f:
            f.write("\n".join(rows) + "\n")
        print(name, n)


if __name__ == "__main__":
    main()
