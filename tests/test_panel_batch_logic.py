"""The run-summation logic of one panel SpMV batch (specann_b200/csrc/panel.cuh: panel_batch), restated
on the CPU and checked against direct row sums.

A warp batch is 256 entries in row order, lane l holding entries [8 l, 8 l + 8). Runs of one row
inside a lane are summed left to right; a run that crosses lanes is summed by a segmented inclusive
scan over the lanes' tail sums (segments: equal last rows) and added by the lane where it ends, with
the carry of the lanes before it. Padding entries (row 0xFFFF) are never added. A row spanning several
batches is added once per batch. This restatement follows the kernel step by step (including the
shuffle semantics: lanes below the distance keep their own value) so that a change of the lane logic
can be checked here before it runs on a GPU.
"""
import numpy as np

PAD = 0xFFFF
LANES, PER_LANE = 32, 8


def batch(keys, prods, ys):
    K = keys.reshape(LANES, PER_LANE)
    S = prods.reshape(LANES, PER_LANE).astype(np.float64).copy()
    for j in range(1, PER_LANE):
        same = K[:, j] == K[:, j - 1]
        S[same, j] = S[same, j - 1] + S[same, j]
    k0, k7 = K[:, 0], K[:, PER_LANE - 1]
    kprev = np.concatenate([[k7[0]], k7[:-1]])      # shfl_up by 1: lane 0 keeps its own
    knext = np.concatenate([k0[1:], [k0[-1]]])      # shfl_down by 1: lane 31 keeps its own
    heads = [(l == 0) or (kprev[l] != k7[l]) for l in range(LANES)]
    seg0 = [max(i for i in range(l + 1) if heads[i]) for l in range(LANES)]
    inc = S[:, PER_LANE - 1].copy()
    d = 1
    while d < LANES:
        t = np.concatenate([inc[:d], inc[:-d]])
        new = inc.copy()
        for l in range(LANES):
            if l - d >= seg0[l]:
                new[l] = t[l] + inc[l]
        inc = new
        d <<= 1
    cin = np.concatenate([[inc[0]], inc[:-1]])
    for l in range(LANES):
        carry = cin[l] if (l > 0 and kprev[l] == k0[l]) else 0.0
        cont = l < LANES - 1 and knext[l] == k7[l]
        for j in range(PER_LANE):
            end = (not cont) if j == PER_LANE - 1 else (K[l, j + 1] != K[l, j])
            if end and K[l, j] != PAD:
                ys[K[l, j]] += S[l, j] + carry if K[l, j] == k0[l] else S[l, j]


def run_chunk(keys, prods):
    """A warp's chunk: consecutive batches, the last one padded."""
    ys = np.zeros(PAD + 1)
    per = LANES * PER_LANE
    pad = (-len(keys)) % per
    keys = np.concatenate([keys, np.full(pad, PAD)])
    prods = np.concatenate([prods, np.zeros(pad)])
    for e in range(0, len(keys), per):
        batch(keys[e:e + per], prods[e:e + per], ys)
    return ys


def test_batch_logic_matches_row_sums():
    rng = np.random.default_rng(1)
    for trial in range(400):
        nrows = int(rng.integers(1, 300))
        lens = rng.choice([1, 1, 1, 2, 3, 9, 40, 300, 700], size=nrows)
        keys = np.repeat(np.arange(nrows), lens)[: int(rng.integers(1, 2000))]
        prods = rng.standard_normal(len(keys))
        ys = run_chunk(keys, prods)
        ref = np.zeros(PAD + 1)
        np.add.at(ref, keys, prods)
        assert np.allclose(ys[:PAD], ref[:PAD], rtol=0, atol=1e-9), trial
        assert ys[PAD] == 0.0


def test_piece_padding_inside_a_batch():
    """Pieces are padded to whole batches: padding may sit inside a lane after real entries."""
    keys = np.concatenate([np.repeat(np.arange(5), [3, 1, 7, 2, 1]), np.full(256 - 14, PAD)])
    prods = np.concatenate([np.arange(1.0, 15.0), np.zeros(256 - 14)])
    ys = np.zeros(PAD + 1)
    batch(keys, prods, ys)
    ref = np.zeros(PAD + 1)
    np.add.at(ref, keys[:14], prods[:14])
    assert np.array_equal(ys[:5], ref[:5]) and ys[PAD] == 0.0
