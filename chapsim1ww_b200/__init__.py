"""chapsim1ww_b200: B200 (sm_100a) implementation of CHAPSim's RK3
fractional-step substep, exposed through the C ABI in include/chapsim.h.

``TGChannel`` mirrors the reference's TG-channel entry points and
``IOChannel`` its IO-section ones; every compute
call goes to libchapsim.so (hand-written CUDA).  There is no CPU fallback.
"""
from ._lib import FP64, MIXED, ITG, IIO, load  # noqa: F401
from .solver import TGChannel, ChapsimError, default_config  # noqa: F401
from .props import PropertyEngine, synthetic_table  # noqa: F401
from .batch import ChannelBatch, batch64_configs  # noqa: F401
from .io_channel import IOChannel  # noqa: F401
