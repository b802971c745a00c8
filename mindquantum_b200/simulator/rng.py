"""The reference's random streams: std::mt19937 + std::uniform_real_distribution<double>.

The reference simulator draws measurement outcomes and sampling uniforms from
``std::mt19937`` (``RndEngine``, ccsrc/include/simulator/vector/vector_state.h:67) through
``std::uniform_real_distribution<double>``.  numpy's MT19937 with legacy seeding produces
the same 32-bit stream; two draws per double follow libstdc++'s generate_canonical
((x0 + x1 * 2^32) / 2^64).  Reproducing the streams keeps sampling results identical to the
reference for the same seed.
"""
import numpy as np

_TWO32 = 4294967296.0
_TWO64 = 18446744073709551616.0
_BELOW_ONE = np.nextafter(1.0, 0.0)


class Mt19937Uniform:
    """uniform_real_distribution<double>(low, high) over std::mt19937(seed)."""

    def __init__(self, seed):
        self._bg = np.random.MT19937(0)
        self._bg._legacy_seeding(int(seed) & 0xFFFFFFFF)  # pylint: disable=protected-access

    def draw(self, n=None, low=0.0, high=1.0):
        k = 1 if n is None else int(n)
        raw = self._bg.random_raw(2 * k).astype(np.float64)
        r = (raw[0::2] + raw[1::2] * _TWO32) / _TWO64
        r = np.minimum(r, _BELOW_ONE)
        out = r * (high - low) + low
        return float(out[0]) if n is None else out


class UniformStreams:
    """Several Mt19937Uniform streams read in lockstep: ``take(rows)`` returns the next uniform
    (0, 1) draw of each listed stream (rows distinct), drawing exactly what it returns, so a
    stream that lives on (a simulator's own) is left where the reference would leave it."""

    def __init__(self, streams):
        self._streams = list(streams)

    def __len__(self):
        return len(self._streams)

    def take(self, rows):
        return np.fromiter((self._streams[b].draw() for b in rows), dtype=np.float64, count=len(rows))


class UniformBlocks:
    """Streams std::mt19937(seeds[b]) made for one batch of trajectories and dropped after it:
    their uniform (0, 1) draws are generated ahead in blocks, and ``take(rows)`` gathers the next
    draw of each listed stream (rows distinct) with one indexing operation."""

    def __init__(self, seeds, block=256):
        self._streams = [Mt19937Uniform(s) for s in seeds]
        self._block = int(block)
        self._buf = np.stack([s.draw(self._block) for s in self._streams]) if self._streams else np.zeros((0, 1))
        self._cur = np.zeros(len(self._streams), dtype=np.int64)

    def __len__(self):
        return len(self._streams)

    def take(self, rows):
        rows = np.asarray(rows, dtype=np.int64)
        for b in rows[self._cur[rows] >= self._block]:
            self._buf[b] = self._streams[b].draw(self._block)
            self._cur[b] = 0
        out = self._buf[rows, self._cur[rows]]
        self._cur[rows] += 1
        return out
