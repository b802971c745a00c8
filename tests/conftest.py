"""Shared pytest configuration: the ``gpu`` marker and import paths."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)
# compiled pass kernels are cached inside the repository's build folder
os.environ.setdefault('MQB_JIT_CACHE', os.path.join(ROOT, '_build', 'jit_cache'))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def goldens():
    import json

    with open(os.path.join(HERE, 'golden', 'reference_goldens.json'), encoding='utf8') as f:
        return json.load(f)


@pytest.fixture(autouse=True)
def _device_error_word(request):
    """After every GPU test: the generated pass kernels reported no given-up wait (their error word
    is 0), so a pipeline that timed out fails the test that ran it instead of passing silently."""
    yield
    if request.node.get_closest_marker('gpu') is None:
        return
    import torch

    if not torch.cuda.is_available():
        return
    from mindquantum_b200 import _native as N

    assert N.device_error(clear=True) == 0, "a generated pass kernel gave up a wait (MQB_DEV_ERR_TIMEOUT)"
