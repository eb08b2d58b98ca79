"""The exclusive scan of the cell counts (k_cell_scan in csrc/tbmd_kernels.cu), restated on the host
with the kernel's own index arithmetic: one block of 1024 threads over tiles of 8192 cells, each
thread scanning 8 contiguous cells of a tile, the thread totals scanned across the block, and a carry
from tile to tile.  Checked against numpy's cumulative sum for grids of one cell to several tiles,
including partial last tiles, which the GPU tests reach only through the batched systems."""
import numpy as np
import pytest

THREADS, PER_THREAD = 1024, 8
TILE = THREADS * PER_THREAD


def cell_scan(count):
    ncells = len(count)
    start = np.zeros(ncells + 1, dtype=np.int64)
    carry = 0
    for base in range(0, ncells, TILE):
        m = min(TILE, ncells - base)
        # coalesced loads: thread t reads cells k * 1024 + t of the tile (zero past its end)
        tile = np.zeros(TILE, dtype=np.int64)
        for k in range(PER_THREAD):
            i = k * THREADS + np.arange(THREADS)
            ok = i < m
            tile[i[ok]] = count[base + i[ok]]
        # thread t owns tile[8 t .. 8 t + 7]; its total, scanned over the block (warps, then warps of warps)
        own = tile.reshape(THREADS, PER_THREAD)
        s = own.sum(axis=1)
        incl = np.cumsum(s)
        run = carry + incl - s
        ex = run[:, None] + np.concatenate([np.zeros((THREADS, 1), dtype=np.int64), np.cumsum(own, axis=1)[:, :-1]], 1)
        tile = ex.reshape(-1)
        carry += int(incl[-1])
        # coalesced stores of the tile's starts
        for k in range(PER_THREAD):
            i = k * THREADS + np.arange(THREADS)
            ok = i < m
            start[base + i[ok]] = tile[i[ok]]
    start[ncells] = carry
    return start


@pytest.mark.parametrize("ncells", [1, 7, 1023, 6859, 8191, 8192, 8193, 14000, 32768, 32768 + 5])
def test_cell_scan_matches_cumsum(ncells):
    rng = np.random.default_rng(ncells)
    count = rng.poisson(19.1, size=ncells).astype(np.int64)
    count[rng.random(ncells) < 0.05] = 0  # empty cells
    want = np.concatenate([[0], np.cumsum(count)])
    assert np.array_equal(cell_scan(count), want)
