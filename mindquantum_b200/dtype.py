"""Precision selection for the state-vector path (mirrors mindquantum/dtype/dtype.py).

``complex128`` keeps the state as interleaved float64 pairs and computes in FP64.
``complex64`` keeps the state as interleaved float32 pairs, computes gate updates in
FP32 and accumulates every reduction (expectations, gradients, norms) in FP64.
"""
import numpy as np

complex64 = 'complex64'
complex128 = 'complex128'
float32 = 'float32'
float64 = 'float64'

_ALIASES = {
    complex64: complex64, 'mindquantum.complex64': complex64, np.complex64: complex64,
    complex128: complex128, 'mindquantum.complex128': complex128, np.complex128: complex128,
    float32: complex64, float64: complex128, np.float32: complex64, np.float64: complex128,
}


def to_mq_type(dtype):
    """Normalise a dtype spelling to ``complex64`` / ``complex128``."""
    if dtype is None:
        return complex128
    try:
        return _ALIASES[dtype]
    except (KeyError, TypeError):
        pass
    s = str(dtype)
    if s.endswith('complex64') or s.endswith('float32'):
        return complex64
    if s.endswith('complex128') or s.endswith('float64'):
        return complex128
    raise TypeError(f"Unsupported dtype {dtype!r}; use complex64 or complex128.")


def is_double_precision(dtype):
    return to_mq_type(dtype) == complex128


def to_np_type(dtype):
    return np.complex128 if is_double_precision(dtype) else np.complex64


def precision_str(dtype):
    return 'double' if is_double_precision(dtype) else 'single'
