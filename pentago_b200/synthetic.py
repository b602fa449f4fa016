"""Seeded synthetic inputs (the benchmark configs use random superinfo, not real data).

splitmix64 is used so that the same (seed, index) gives the same words on any
machine and any numpy version.  ``random_nodes`` produces end-engine nodes
[win, notlost] with win a subset of notlost and about 31% of notlost bits set:
per 64-bit word, notlost = r0 & (r1 | (r2 & r3)) and win = notlost & r4 & r5.
"""
import numpy as np

_G = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed, count, offset=0):
    """``count`` 64-bit words of the splitmix64 stream of ``seed``, starting at ``offset``."""
    with np.errstate(over="ignore"):
        x = np.uint64(seed) + (np.arange(offset, offset + count, dtype=np.uint64) + np.uint64(1)) * _G
        z = x
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def random_words(seed, shape):
    n = int(np.prod(shape))
    return splitmix64(seed, n).reshape(shape)


def random_nodes(seed, n):
    """``n`` nodes (n x 8 uint64): [win super, notlost super] with win subset of notlost."""
    r = splitmix64(seed, 6 * 4 * n).reshape(n, 4, 6)
    notlost = r[..., 0] & (r[..., 1] | (r[..., 2] & r[..., 3]))
    win = notlost & r[..., 4] & r[..., 5]
    return np.concatenate([win, notlost], axis=1)
