"""B200 (sm_100a) implementation of the PowerLLEL_Channel DNS time step.

The compute path is ``lib/libplc.so`` (hand-written CUDA behind the C ABI of
``include/plc.h``); this package is the host-side mirror of the reference's
module interface over that ABI (see :mod:`.channel`).
"""
from ._lib import FIELDS, PlcError, PlcParams, lib  # noqa: F401
from .channel import Channel, get_eigen_values, make_params, read_param_json  # noqa: F401
from .ensemble import Ensemble, partition  # noqa: F401

__all__ = ["Channel", "Ensemble", "PlcError", "PlcParams", "make_params", "read_param_json",
           "get_eigen_values", "lib", "FIELDS", "partition"]
