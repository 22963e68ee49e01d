"""Counter-based node selection for the local search (oracle side). TEST INFRASTRUCTURE ONLY.

The reference draws ``cp.random.permutation(n)[:m]`` with m = max(1, int(fraction * n)) for each
pass (models/spectral_annealing.py:1083-1084) and one permutation per final-sweep round
(models/spectral_annealing.py:1008-1011). CuPy's generator cannot be reproduced, so the build
defines its own stream, identical on the GPU (specann_b200/csrc/common.cuh, ``sel_rank``) and here:

  * keys: k_r = splitmix64(splitmix64(seed ^ SEL_SALT) + 4 * stream + r), r = 0..3
  * a bijection P of [0, 2^b), b = bit length of n - 1 (at least 1): four rounds of
    x <- (x + (k_r & M)) & M ; x <- (x * ((k_r >> 32) | 1)) & M ; x <- x ^ (x >> s), s = (b + 1) // 2
    (each step is invertible on b-bit words: addition, multiplication by an odd number, xorshift)
  * rank(i) = P(i), then P again while the value is >= n (cycle walking: a bijection of [0, n))
  * node i is selected in that stream iff rank(i) < m.

Exactly m nodes are selected, as with the reference's permutation prefix. The main loop uses
stream = pass index; final-sweep round r uses stream = FINAL_STREAM_BASE + r.
splitmix64 is the published SplitMix64 finaliser (Steele, Lea and Flood, 2014).
"""
import numpy as np

MASK64 = (1 << 64) - 1
SEL_SALT = 0x5E1EC7ED5EED0001
FINAL_STREAM_BASE = 1 << 20


def splitmix64(x: int) -> int:
    x = (x + 0x9E3779B97F4A7C15) & MASK64
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
    return z ^ (z >> 31)


def stream_keys(seed: int, stream: int):
    base = splitmix64((int(seed) ^ SEL_SALT) & MASK64)
    return [splitmix64((base + 4 * int(stream) + r) & MASK64) for r in range(4)]


def domain_bits(n: int) -> int:
    return max(1, int(n - 1).bit_length())


def _perm(x: np.ndarray, keys, b: int) -> np.ndarray:
    M = np.uint64((1 << b) - 1)
    s = np.uint64((b + 1) // 2)
    for k in keys:
        add = np.uint64(k & ((1 << b) - 1))
        mul = np.uint64(((k >> 32) | 1) & 0xFFFFFFFF)
        x = (x + add) & M
        x = (x * mul) & M
        x = x ^ (x >> s)
    return x


def ranks(n: int, seed: int, stream: int) -> np.ndarray:
    """rank(i) for i in [0, n): a permutation of [0, n) as int64."""
    if n <= 0:
        return np.zeros(0, dtype=np.int64)
    b = domain_bits(n)
    keys = stream_keys(seed, stream)
    y = _perm(np.arange(n, dtype=np.uint64), keys, b)
    over = y >= np.uint64(n)
    while over.any():
        y[over] = _perm(y[over], keys, b)
        over = y >= np.uint64(n)
    return y.astype(np.int64)


def selected_mask(n: int, seed: int, stream: int, m: int) -> np.ndarray:
    """Boolean mask of the m nodes selected in this stream."""
    if m >= n:
        return np.ones(n, dtype=bool)
    return ranks(n, seed, stream) < m


def num_selected(n: int, fraction: float) -> int:
    """m = max(1, int(fraction * n)) as the reference computes it (models/spectral_annealing.py:1082)."""
    return max(1, int(fraction * n))
