"""Shared-memory sizes the bulge kernels ask for, checked against the 227 KB
a B200 block may opt into (232,448 bytes), from the constants in
csrc/bulge.cu: the host tries every tile count up to kMfMaxTiles for
myers_tile_kernel and sets that size as the kernel's dynamic shared memory,
so a size past the limit would fail the search instead of running it."""
import os
import re

SRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                   "cas-offinder-rust-old_b200", "csrc", "bulge.cu")
OPTIN_BYTES = 232448


def _const(name):
    text = open(SRC).read()
    m = re.search(r"constexpr (?:uint32_t|int) %s = ([^;]+);" % name, text)
    assert m, name
    expr = m.group(1)
    # kMfQWords = kTile / 32 + 2
    for dep in re.findall(r"k[A-Z]\w+", expr):
        expr = expr.replace(dep, str(_const(dep)))
    return int(eval(expr, {}))  # integer constant expressions only


def test_myers_tile_kernel_smem_worst_case():
    tiles, forms = _const("kMfMaxTiles"), _const("kMfMaxForms")
    qwords, stage = _const("kMfQWords"), _const("kMfStage")
    staged_patterns = _const("kSmemMyers")
    assert qwords == _const("kTile") // 32 + 2
    # smem_of(t) in Engine::run_bulge: Q and pam_ok words per tile and form,
    # the staged Eq tables (64-bit words above 32 cells), the candidate stage
    worst = tiles * forms * (qwords + 32) * 4 + staged_patterns * 16 * 8 + stage * 8 + 8
    assert worst <= OPTIN_BYTES, worst


def test_slot_traceback_fits_a_block():
    # the largest slot layout: the stack (margin + spare nodes of 24 bytes
    # for windows over 48 cells), slot records, band tables of the widest
    # band at 64 cells with two-word cells, texts and pattern arrays.  The
    # host lowers the slots, then the warps per block, while a block does
    # not fit; one warp of the default three slots must always fit
    spare, slots = _const("kTbSlotSpare"), _const("kTbSlotsShared")
    band_max = _const("kBandMax")
    text, pat = _const("kTbText"), _const("kTbPat")
    wmax = 72
    cap = 2 * max(wmax, 40) + spare
    tbl_words = (64 + 1) * band_max * 2

    def al16(x):
        return (x + 15) & ~15

    per_warp = (al16(cap * 24) + al16(slots * 64) + al16(slots * tbl_words * 8) + al16(slots * 4)
                + al16(slots * text) + al16(slots * 3 * pat))
    # with the widest tables the host may still drop to fewer warps per
    # block; one warp must always fit
    assert per_warp <= OPTIN_BYTES, per_warp
    # at the benchmark shape (23 cells, band 5, one-word cells) four warps
    # of three slots fit with room for several blocks per SM
    bench_cap = 2 * 40 + spare
    bench = 4 * (al16(bench_cap * 16) + al16(slots * 64) + al16(slots * 21 * 5 * 8)
                 + al16(slots * 4) + al16(slots * text) + al16(slots * 3 * pat))
    assert bench * 6 <= OPTIN_BYTES, bench
