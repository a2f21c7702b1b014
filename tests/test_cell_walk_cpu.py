"""The cell walk of the grid-wide persistent kernels (``CellWalk`` in
``csrc/persistent.cuh``: ``k_pcg``, ``k_pcg1``, ``k_svof``), restated in
Python and checked on the CPU.

A thread of those kernels visits the interior cells q = tid, tid + nthr,
tid + 2 nthr, ... with q = (i - 1) + (j - 1) nx.  Instead of a division and
a remainder per cell it starts from (i0, j0) of q = tid and adds the
stride's (di, dj) = (nthr mod nx, nthr div nx) with a carry; the loop ends
when j passes ny (q >= nx ny).  ``k_svof`` takes four cells of the walk per
step, loads first.  Both must visit exactly the cells of the strided loop,
in its order, for every thread -- the sums and the max-norm of the kernels
then see the same values in the same order as before, so the bits are
unchanged.  The GPU kernels themselves are checked against the oracle in
``tests/test_gpu_routines.py`` and ``tests/test_zz_no_alloc.py``.
"""
import pytest


def strided(tid, nthr, nx, ny):
    return [(1 + q % nx, 1 + q // nx) for q in range(tid, nx * ny, nthr)]


def walk(tid, nthr, nx, ny):
    i, j = 1 + tid % nx, 1 + tid // nx
    di, dj = nthr % nx, nthr // nx
    out = []
    while j <= ny:
        out.append((i, j))
        i += di
        j += dj
        if i > nx:
            i -= nx
            j += 1
    return out


def walk4(tid, nthr, nx, ny, U=4):
    """k_svof's batches: U cells of the walk gathered, then visited"""
    i, j = 1 + tid % nx, 1 + tid // nx
    di, dj = nthr % nx, nthr // nx
    out = []
    while j <= ny:
        batch = []
        for _ in range(U):
            if j <= ny:
                batch.append((i, j))
                i += di
                j += dj
                if i > nx:
                    i -= nx
                    j += 1
        out.extend(batch)
    return out


# grids and launch widths of the grid-wide kernels (148 CTAs x 512 threads on
# a B200, fewer when the grid is small) and awkward ones: a stride below,
# equal to and just above nx, and wider than the whole grid
CASES = [(320, 640, 148 * 512), (256, 256, 148 * 512), (2048, 2048, 148 * 512), (13, 9, 7), (13, 9, 13),
         (13, 9, 14), (13, 9, 200), (1, 5, 3), (7, 1, 3), (64, 128, 64 * 512)]


@pytest.mark.parametrize("nx,ny,nthr", CASES)
def test_walk_visits_the_strided_cells_in_order(nx, ny, nthr):
    tids = sorted({0, 1, nthr // 2, nthr - 1, min(nthr - 1, nx * ny - 1), min(nthr - 1, nx * ny)})
    for tid in tids:
        ref = strided(tid, nthr, nx, ny)
        assert walk(tid, nthr, nx, ny) == ref, tid
        assert walk4(tid, nthr, nx, ny) == ref, tid


@pytest.mark.parametrize("nx,ny,nthr", [(13, 9, 7), (13, 9, 40), (10, 14, 33)])
def test_walks_of_all_threads_cover_the_interior_once(nx, ny, nthr):
    seen = [c for tid in range(nthr) for c in walk(tid, nthr, nx, ny)]
    assert sorted(seen) == sorted((i, j) for i in range(1, nx + 1) for j in range(1, ny + 1))
