"""PyTorch autograd integration of the expectation-with-gradient operator."""
from .operations import (MQAnsatzOnlyOps, MQEncoderOnlyOps, MQN2AnsatzOnlyOps, MQN2EncoderOnlyOps, MQN2Ops, MQOps,
                         QRamVecOps, mq_expectation)
from .layer import MQAnsatzOnlyLayer, MQLayer, MQN2AnsatzOnlyLayer, MQN2Layer, QRamVecLayer
