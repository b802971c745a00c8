"""ctypes binding of libmqb200.so (the C ABI declared in include/mqb200.h).

The library is the only compute path of this package: there is no CPU or PyTorch fallback.
Importing this module builds the library if it is missing (nvcc only, no GPU needed) and
raises if it cannot be loaded.
"""
import ctypes
import os
import threading

from .build_native import LIB, build

MQB_OK = 0
MQB_PREC_C64 = 0
MQB_PREC_C128 = 1
MQB_GATE_NONUNITARY = 1
MQB_MAX_OBJ = 6
MQB_MAX_ANGLES = 3


class GateDesc(ctypes.Structure):
    _fields_ = [
        ('gate_id', ctypes.c_int32),
        ('n_obj', ctypes.c_int32),
        ('obj', ctypes.c_int32 * MQB_MAX_OBJ),
        ('ctrl_mask', ctypes.c_uint64),
        ('n_angles', ctypes.c_int32),
        ('grad_angles', ctypes.c_int32),
        ('angle_const', ctypes.c_double * MQB_MAX_ANGLES),
        ('term_begin', ctypes.c_int32 * MQB_MAX_ANGLES),
        ('term_count', ctypes.c_int32 * MQB_MAX_ANGLES),
        ('matrix_offset', ctypes.c_int64),
        ('pauli_x', ctypes.c_uint64),
        ('pauli_y', ctypes.c_uint64),
        ('pauli_z', ctypes.c_uint64),
        ('pauli_ny', ctypes.c_int32),
        ('flags', ctypes.c_int32),
    ]


class ParamTerm(ctypes.Structure):
    _fields_ = [('param', ctypes.c_int32), ('flags', ctypes.c_int32), ('coeff', ctypes.c_double)]


class ProgramOptions(ctypes.Structure):
    _fields_ = [('fuse', ctypes.c_int32), ('tile_bits', ctypes.c_int32), ('jit', ctypes.c_int32),
                ('reserved', ctypes.c_int32 * 5)]


class ProgramInfo(ctypes.Structure):
    _fields_ = [
        ('n_qubits', ctypes.c_int32),
        ('precision', ctypes.c_int32),
        ('n_ops', ctypes.c_int32),
        ('n_params', ctypes.c_int32),
        ('n_passes', ctypes.c_int32),
        ('tile_bits', ctypes.c_int32),
        ('n_grad_slots', ctypes.c_int32),
        ('per_sample_entries', ctypes.c_int32),
        ('custom_entries', ctypes.c_int32),
        ('reserved', ctypes.c_int32 * 7),
    ]


_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_SZ = ctypes.c_size_t
_D = ctypes.c_double

# name -> argtypes; every entry point returns int (status), except mqb_last_error
SIGNATURES = {
    'mqb_version': [],
    'mqb_device_sm_count': [_P],
    'mqb_timing_begin': [],
    'mqb_timing_end': [_P, _P, _I],
    'mqb_device_error': [_P, _I],
    'mqb_inject_alloc_failure': [_I],
    'mqb_grad_norm_checks': [_P, _P, _SZ, _I64, _I, _I, _P, _I, _P, _P],
    'mqb_abi_struct_sizes': [_P, _I],
    'mqb_program_create': [_I, _I, _P, _I, _P, _I, _I, _P, _I64, _P, _P],
    'mqb_program_destroy': [_P],
    'mqb_plan_schedule': [_I, _I, _P, _I, _P, _I64, _I, _I, _P, _P, _P, _P, _P, _P],
    'mqb_jit_check': [_I, _I, _P, _I, _P, _I64, _I, _I, _P],
    'mqb_adjoint_with_lambda': [_P, _P, _I, _P, _I, _I64, _P, _I64, _P, _P, _I, _P, _SZ, _P],
    'mqb_program_get_info': [_P, _P],
    'mqb_program_grad_passes': [_P, _I, _P, _P],
    'mqb_apply_workspace_size': [_P, _I64, _P],
    'mqb_apply': [_P, _P, _I64, _P, _I64, _P, _P, _SZ, _P],
    'mqb_apply_static': [_P, _P, _I64, _P, _I64, _P, _P],
    'mqb_ham_create': [_I, _I, _P, _P, _P, _P, _P, _I, _P],
    'mqb_ham_create_csr': [_I, _I, _I64, _P, _P, _P, _P],
    'mqb_ham_destroy': [_P],
    'mqb_apply_hamiltonian': [_P, _P, _P, _I64, _P],
    'mqb_expectation': [_P, _P, _P, _I64, _P, _P],
    'mqb_apply_matrix1': [_I, _I, _P, _I64, _I, ctypes.c_uint64, _P, _P],
    'mqb_vdot': [_I, _I, _P, _P, _I64, _P, _P],
    'mqb_rows_apply_matrix1': [_I, _I, _P, _I64, _I64, _P, _P, _P, _P, _P],
    'mqb_rows_matrix1_norm': [_I, _I, _P, _I64, _I64, _P, _P, _P, _P, _P, _P],
    'mqb_grad_workspace_size': [_P, _I64, _I, _I, _P],
    'mqb_expectation_with_grad': [_P, _P, _I, _P, _I, _I64, _P, _I64, _P, _P, _P, _I, _P, _SZ, _P],
    'mqb_sample_scratch_size': [_I, _P],
    'mqb_sample_indices': [_I, _I, _P, _P, _I64, _P, _P, _SZ, _P],
    'mqb_qubit_one_probability': [_I, _I, _P, _I, _P, _P],
    'mqb_collapse': [_I, _I, _P, _I, _I, _D, _P],
}

_lib = None
_lock = threading.Lock()


class NativeError(RuntimeError):
    """A non-zero status returned by libmqb200."""


def lib():
    """Load (building first if needed) libmqb200.so; raises if it cannot be loaded."""
    global _lib  # pylint: disable=global-statement
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB) or os.environ.get('MQB200_REBUILD'):
                build()
            L = ctypes.CDLL(LIB)
            for name, args in SIGNATURES.items():
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = ctypes.c_int
            L.mqb_last_error.argtypes = []
            L.mqb_last_error.restype = ctypes.c_char_p
            sizes = (ctypes.c_int64 * 4)()
            L.mqb_abi_struct_sizes(sizes, 4)
            want = [ctypes.sizeof(GateDesc), ctypes.sizeof(ParamTerm), ctypes.sizeof(ProgramOptions),
                    ctypes.sizeof(ProgramInfo)]
            if list(sizes) != want:
                raise NativeError(f"ABI mismatch between libmqb200.so {list(sizes)} and the bindings {want}")
            _lib = L
    return _lib


def check(status, what=''):
    if status != MQB_OK:
        msg = lib().mqb_last_error().decode(errors='replace')
        raise NativeError(f"{what}: {msg} (status {status})" if what else f"{msg} (status {status})")


def call(name, *args):
    """Call an entry point and raise NativeError on a non-zero status."""
    check(getattr(lib(), name)(*args), name)


TIMING_KINDS = ('fused_forward', 'fused_backward', 'hamiltonian', 'matgen', 'gate_apply', 'gate_grad', 'grad_scatter',
                'copy', 'channel_rows')


class KernelTimer:
    """Context manager collecting per-kind kernel times (ms) and launch counts of libmqb200."""

    def __enter__(self):
        call('mqb_timing_begin')
        self.ms = {}
        self.launches = {}
        return self

    def __exit__(self, *exc):
        n = len(TIMING_KINDS)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_int64 * n)()
        call('mqb_timing_end', ms, cnt, n)
        self.ms = {k: ms[i] for i, k in enumerate(TIMING_KINDS)}
        self.launches = {k: cnt[i] for i, k in enumerate(TIMING_KINDS)}
        return False


def device_error(clear=True):
    """Error word of the generated pass kernels on the current device (0: none; 1: a tile-pipeline
    wait gave up, the results since the last check are invalid).  Synchronizes the device."""
    code = ctypes.c_int()
    call('mqb_device_error', ctypes.byref(code), 1 if clear else 0)
    return code.value
