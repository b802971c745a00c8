"""PyTorch autograd integration of the expectation-with-gradient operator."""
from .operations import MQAnsatzOnlyOps, MQEncoderOnlyOps, MQOps, QRamVecOps, mq_expectation
from .layer import MQAnsatzOnlyLayer, MQLayer
