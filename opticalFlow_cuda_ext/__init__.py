"""Import-compatible alias of the reference's extension package: code that does
`from opticalFlow_cuda_ext import opticalFlow` gets the libsvsflow-backed operator module."""
from singleventriclesegmentation_b200 import opticalFlow  # noqa: F401

__all__ = ["opticalFlow"]
