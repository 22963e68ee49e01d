"""The piece rules of the column-panel layout (specann_b200/csrc/panel.cu: pl_pieces), restated on the
CPU with their invariants.

A segment (one row block's entries of one panel, in row order) is packed into pieces of at most 256
entries: a row is added whole while it fits; when it does not fit the open piece is closed; a row
longer than the room left fills whole pieces and its remainder opens the next one. Every piece is
padded to 256 slots (one warp batch). The segment's pieces are cut into 16 contiguous runs, one per
warp: warp w starts at piece floor(P w / 16), moved forward past pieces that continue the row of the
piece before them, so the pieces of one row always belong to one warp.
"""
import numpy as np

PIECE, WARPS = 256, 16


def pieces(rows):
    """rows: the row of every entry of a segment, in order -> list of (start, length)."""
    out, fill, opened, k, e = [], 0, 0, 0, len(rows)
    while k < e:
        k2 = k + 1
        while k2 < e and rows[k2] == rows[k]:
            k2 += 1
        left = k2 - k
        if fill > 0 and fill + left > PIECE:
            out.append((opened, fill))
            fill = 0
        while left > 0:
            if fill == 0:
                opened = k
            take = min(left, PIECE - fill)
            fill += take
            k += take
            left -= take
            if fill == PIECE:
                out.append((opened, fill))
                fill = 0
    if fill > 0:
        out.append((opened, fill))
    return out


def warp_starts(rows, pcs):
    cnt = len(pcs)
    starts = []
    for w in range(WARPS):
        t = cnt * w // WARPS
        while 0 < t < cnt and pcs[t][0] > 0 and rows[pcs[t][0]] == rows[pcs[t][0] - 1]:
            t += 1
        starts.append(t)
    return starts


def check_segment(rows):
    pcs = pieces(rows)
    # the pieces cover the segment in order, each at most one batch
    pos = 0
    for start, length in pcs:
        assert start == pos and 0 < length <= PIECE
        pos += length
    assert pos == len(rows)
    # a row is split only when it does not fit in one piece, and then only across consecutive pieces
    piece_of = np.repeat(np.arange(len(pcs)), [l for _, l in pcs])
    for r in np.unique(rows):
        span = np.unique(piece_of[rows == r])
        assert np.array_equal(span, np.arange(span[0], span[-1] + 1))
        if len(span) > 1:                       # only a row that cannot fit in one piece is split
            s0, l0 = pcs[span[0]]
            room = PIECE - (l0 - np.sum(rows[s0:s0 + l0] == r))
            assert np.sum(rows == r) > room
    # a closed piece with room left was closed because the next row did not fit
    for i, (start, length) in enumerate(pcs[:-1]):
        if length < PIECE:
            nxt = rows[start + length]
            assert length + np.sum(rows == nxt) > PIECE
    # at most 2 L / 256 + 1 pieces (the layout's capacity bound)
    assert len(pcs) <= 2 * (len(rows) // PIECE) + 1
    # warp runs are non-decreasing and never separate the pieces of one row
    st = warp_starts(rows, pcs)
    assert st == sorted(st)
    for t in st:
        if 0 < t < len(pcs):
            s = pcs[t][0]
            assert rows[s] != rows[s - 1]


def test_piece_rules_on_random_segments():
    rng = np.random.default_rng(3)
    for trial in range(300):
        nrows = int(rng.integers(1, 400))
        lens = rng.choice([0, 1, 1, 1, 2, 3, 7, 40, 255, 256, 257, 600], size=nrows)
        rows = np.repeat(np.arange(nrows), lens)
        if len(rows) == 0:
            assert pieces(rows) == []
            continue
        check_segment(rows)


def test_long_row_fills_whole_pieces():
    rows = np.concatenate([np.zeros(10, int), np.ones(700, int), np.full(5, 2)])
    pcs = pieces(rows)
    # row 0 (10) closes before row 1 (700) would not fit; row 1 fills two whole pieces, its 188
    # remaining entries open the third, and row 2 joins them
    assert pcs == [(0, 10), (10, 256), (266, 256), (522, 193)]
    # warps 8-15 would start inside row 1's pieces: they move past them, so warp 4 takes all of row 1
    assert warp_starts(rows, pcs) == [0] * 4 + [1] * 4 + [4] * 8
