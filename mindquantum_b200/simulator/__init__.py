"""Simulator facade and the B200 state-vector backend."""
from .backend_base import BackendBase
from .measure_result import MeasureResult
from .simulator import SUPPORTED_SIMULATOR, Simulator, inner_product
from .utils import GradOpsWrapper
