"""NVTX ranges of the C ABI, checked on the host with a recording injection library.

libmqb200 pushes one NVTX range per C-ABI call (named after the entry point) and one per kernel
launch (named after the launch kind).  tests/nvtx/nvtx_recorder.c is a minimal NVTX injection
library that records the pushed names; a child process loads it through NVTX_INJECTION64_PATH,
calls entry points whose argument checks fail before any device work, and reports what was pushed
and popped: every call's range opens and closes, also when the call returns an error.
"""
import json
import os
import shutil
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

CHILD = r'''
import ctypes, json, os, sys
sys.path.insert(0, sys.argv[1])
from mindquantum_b200 import _native as N
L = N.lib()
p = ctypes.c_void_p(4096)
codes = [L.mqb_apply(None, p, 1, None, 0, None, None, 0, None),
         L.mqb_vdot(0, N.MQB_PREC_C64, p, p, 1, p, None),
         L.mqb_collapse(3, N.MQB_PREC_C64, p, 0, 2, 1.0, None)]
R = ctypes.CDLL(os.environ['NVTX_INJECTION64_PATH'])
R.recorder_name.restype = ctypes.c_char_p
names = [R.recorder_name(i).decode() for i in range(R.recorder_pushes())]
print(json.dumps({"codes": codes, "names": names, "pops": R.recorder_pops()}))
'''


@pytest.mark.skipif(shutil.which('gcc') is None, reason="gcc is needed to build the recorder")
def test_entry_points_push_and_pop_nvtx_ranges(tmp_path):
    lib = tmp_path / 'libnvtx_recorder.so'
    cuda = os.environ.get('CUDA_HOME', '/usr/local/cuda')
    subprocess.run(['gcc', '-O2', '-fPIC', '-shared', f'-I{cuda}/include',
                    os.path.join(HERE, 'nvtx', 'nvtx_recorder.c'), '-o', str(lib)], check=True)
    env = dict(os.environ, NVTX_INJECTION64_PATH=str(lib))
    out = subprocess.run([sys.executable, '-c', CHILD, ROOT], env=env, capture_output=True, text=True, timeout=300,
                         check=True)
    rec = json.loads(out.stdout.strip().splitlines()[-1])
    assert rec['codes'] == [-1, -1, -1]                   # MQB_ERR_INVALID, before any device work
    assert rec['names'] == ['mqb_apply', 'mqb_vdot', 'mqb_collapse']
    assert rec['pops'] == 3                                # every range closed on the error path
