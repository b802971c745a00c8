"""PyTorch autograd integration of the expectation-with-gradient operator."""
from .operations import MQAnsatzOnlyOps, MQEncoderOnlyOps, MQOps, mq_expectation
from .layer import MQAnsatzOnlyLayer, MQLayer
