"""B200-native (sm_100a) 3D TV-L1 optical flow and tricubic mask propagation: a drop-in for the
`opticalFlow_cuda_ext.opticalFlow` operators and the flow driver of
ajortizg/singleVentricleSegmentation.

    from singleventriclesegmentation_b200 import opticalFlow          # the operator module
    from singleventriclesegmentation_b200.tvl13d import TVL13DOpticalFlow
"""
from . import opticalFlow  # noqa: F401

__all__ = ["opticalFlow"]
