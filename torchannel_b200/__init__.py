"""B200-native TorChannel time step.

Hand-written sm_100a CUDA kernels behind a C ABI (include/torchannel_b200.h),
bound with ctypes, with a ChannelFlow-compatible host class.
"""
__version__ = "0.1.0"


def __getattr__(name):
    # lazy: importing the package must not require a GPU or the built library
    if name == "Channel":
        from .core import Channel
        return Channel
    if name == "ChannelFlowB200":
        from .solver import ChannelFlowB200
        return ChannelFlowB200
    raise AttributeError(name)
