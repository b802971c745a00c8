"""MeasureResult: sampled bit strings per measurement key (mindquantum/core/gates/measurement.py:190-330)."""
import numpy as np


class MeasureResult:
    """Container of sampling results.

    ``keys`` lists the measurement keys in reverse order of their appearance in the circuit and
    every bit string shows the keys in that order, as the reference does.
    """

    def __init__(self):
        self.measures = []
        self._keys = []
        self._samples = np.array([])
        self.bit_string_data = {}
        self.shots = 0

    def add_measure(self, measure):
        if not isinstance(measure, (list, tuple)):
            measure = [measure]
        for meas in reversed(list(measure)):
            key = meas if isinstance(meas, str) else meas.key
            if key in self._keys:
                raise ValueError(f"Measure key {key} already defined.")
            self.measures.append(meas)
            self._keys.append(key)

    @property
    def keys(self):
        return list(self._keys)

    @property
    def keys_map(self):
        return {k: i for i, k in enumerate(self._keys)}

    @property
    def samples(self):
        return self._samples

    def collect_data(self, samples):
        samples = np.asarray(samples)
        out = {}
        self._samples = samples
        self.shots = len(samples)
        for row in samples:
            s = ''.join(str(int(i)) for i in row)
            out[s] = out.get(s, 0) + 1
        self.bit_string_data = {k: out[k] for k in sorted(out)}

    @property
    def data(self):
        return self.bit_string_data

    def __str__(self):
        return f"shots: {self.shots}\nKeys: {' '.join(self._keys)}\n{self.bit_string_data}"

    __repr__ = __str__
