"""Host side of the multigrid hierarchy: coarse level records (no GPU).

The records are checked against their definition: halved block sizes (ceil), cells of each
block and instance contiguous and in order, tiles of PHB_TILE_CELLS cells that never cross
a block, faces carried over, and coarsening refused where a connection that reverses a
tangential axis meets an odd size."""
import numpy as np

from phipict_b200 import _lib
from phipict_b200.amg import coarsen_records


def _records(sizes_per_block, ninst=1, faces=None):
    """Block and instance records of `ninst` copies of a multi-block domain."""
    nb = len(sizes_per_block)
    blocks = np.zeros((ninst * nb, _lib.BREC), dtype=np.int32)
    insts = np.zeros((ninst, _lib.IREC), dtype=np.int32)
    n_inst = sum(int(np.prod(s)) for s in sizes_per_block)
    tiles = 0
    for e in range(ninst):
        off = 0
        t0 = tiles
        for i, s in enumerate(sizes_per_block):
            r = blocks[e * nb + i]
            r[0:3] = s
            r[3] = e * n_inst + off
            r[4] = off
            r[5] = e
            r[6] = e * n_inst
            r[7] = n_inst
            for f in range(6):
                r[8 + 6 * f] = 1
            for (bi, f), rec in (faces or {}).items():
                if bi == i:
                    r[8 + 6 * f: 8 + 6 * f + 6] = rec
                    if rec[0] == 2:
                        r[8 + 6 * f + 1] = e * nb + rec[1]
            r[44] = tiles
            tiles += -(-int(np.prod(s)) // _lib.TILE)
            off += int(np.prod(s))
        insts[e, :6] = (e * n_inst, n_inst, t0, tiles - t0, e * nb, nb)
    return blocks, insts


def test_sizes_offsets_and_tiles():
    blocks, insts = _records([(64, 48, 48), (64, 48, 48), (7, 3, 1)], ninst=2)
    out, tiles, ins = coarsen_records(blocks, insts, 3)
    assert out[:, 0:3].tolist() == [[32, 24, 24], [32, 24, 24], [4, 2, 1]] * 2
    n = [32 * 24 * 24, 32 * 24 * 24, 8]
    assert ins[:, 1].tolist() == [sum(n)] * 2
    assert out[:, 3].tolist() == [0, n[0], n[0] + n[1], sum(n), sum(n) + n[0], sum(n) + n[0] + n[1]]
    assert (out[:, 7] == sum(n)).all() and out[3:, 6].tolist() == [sum(n)] * 3
    # tiles: each block cut into runs of TILE cells, in block order, none crossing a block
    expect = []
    for i in range(6):
        expect += [(i, t) for t in range(0, n[i % 3], _lib.TILE)]
    assert [tuple(t) for t in tiles] == expect
    assert ins[:, 2].tolist() == [0, len(expect) // 2] and ins[:, 3].tolist() == [len(expect) // 2] * 2
    assert out[:, 44].tolist() == [expect.index((i, 0)) for i in range(6)]
    # faces are carried over unchanged
    assert (out[:, 8:44] == blocks[:, 8:44]).all()


def test_two_dimensional_and_exhausted():
    blocks, insts = _records([(5, 1, 1)])
    out, _, ins = coarsen_records(blocks, insts, 2)
    assert out[0, 0:3].tolist() == [3, 1, 1] and ins[0, 1] == 3
    blocks, insts = _records([(1, 1, 1)])
    assert coarsen_records(blocks, insts, 2) is None


def test_reversed_connection_needs_even_tangential_sizes():
    # block 0's +x face joined to block 1 with the first tangential axis (y) reversed
    rec = (2, 1, (0 << 1) | 0, (1 << 1) | 1, (2 << 1) | 0, 0)
    blocks, insts = _records([(4, 6, 4), (4, 6, 4)], faces={(0, 1): rec})
    assert coarsen_records(blocks, insts, 3) is not None
    blocks, insts = _records([(4, 5, 4), (4, 5, 4)], faces={(0, 1): rec})
    assert coarsen_records(blocks, insts, 3) is None
    # not reversed: odd sizes line up
    rec2 = (2, 1, (0 << 1) | 0, (1 << 1) | 0, (2 << 1) | 0, 0)
    blocks, insts = _records([(4, 5, 4), (4, 5, 4)], faces={(0, 1): rec2})
    assert coarsen_records(blocks, insts, 3) is not None
