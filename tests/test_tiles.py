"""The fused kernel's row bands (fg2_tile_bands, host only): for every grid height, tile
height and tail-band count, in both launch directions, the bands cover the rows exactly once,
each in as many 7-row blocks as its rows need, and the tail bands come last in the order a
launch takes the tiles."""
import pytest

import fg2_b200

HEIGHTS = list(range(1, 120)) + [203, 4095, 4096, 4097, 8192, 14336]


@pytest.mark.parametrize("reverse", [False, True])
@pytest.mark.parametrize("tail", [0, 1, 2, 3, 5])
@pytest.mark.parametrize("nb", [1, 2, 3, 4, 6, 8])
def test_bands_partition_the_rows(nb, tail, reverse):
    for n1 in HEIGHTS:
        bands = fg2_b200.tile_bands(n1, nb, tail, reverse)
        assert bands, n1
        for i0, iend, blocks in bands:
            assert 0 <= i0 < iend <= n1, (n1, i0, iend)
            assert 1 <= blocks <= nb and blocks == -(-(iend - i0) // 7), (n1, i0, iend, blocks)
        # exactly once: sorted by first row, each band starts where the previous one ended
        rows = sorted((i0, iend) for i0, iend, _ in bands)
        assert rows[0][0] == 0 and rows[-1][1] == n1, n1
        assert all(a[1] == b[0] for a, b in zip(rows, rows[1:])), (n1, rows)
        # a launch takes the bands top-down, a reverse launch bottom-up
        firsts = [i0 for i0, _, _ in bands]
        assert firsts == sorted(firsts, reverse=reverse), n1
        # at least `tail` one-block bands end the order (when the grid has the rows for them)
        if tail and nb > 1:
            k = min(tail, -(-n1 // 7))
            assert all(b[2] == 1 for b in bands[-k:]), (n1, bands[-k:])


def test_without_tail_bands_the_decomposition_is_nb_blocks():
    # 4096 rows in bands of 21: 195 whole bands and a last band of one row, one block
    bands = fg2_b200.tile_bands(4096, 3, 0, False)
    assert len(bands) == 196
    assert bands[0] == (0, 21, 3) and bands[-1] == (4095, 4096, 1)
    # the reverse launch lays them out from the last row: the one-row band is the top one
    rev = fg2_b200.tile_bands(4096, 3, 0, True)
    assert rev[0] == (4075, 4096, 3) and rev[-1] == (0, 1, 1)
    # one tail band: 194 bands of 21 rows, then 22 rows in four one-block bands
    t = fg2_b200.tile_bands(4096, 3, 1, False)
    assert len(t) == 198 and t[193] == (4053, 4074, 3)
    assert t[194:] == [(4074, 4081, 1), (4081, 4088, 1), (4088, 4095, 1), (4095, 4096, 1)]


def test_bad_arguments_are_refused():
    lib = fg2_b200.load_library("hydro")
    assert lib.fg2_tile_bands(0, 3, 0, 0, None, 0) == -1
    assert lib.fg2_tile_bands(100, -1, 0, 0, None, 0) == -1
    assert lib.fg2_tile_bands(100, 3, -2, 0, None, 0) == -1
