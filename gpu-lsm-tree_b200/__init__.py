"""B200-native GPU dictionary: LSM (GPULSMOpt semantics) and FliX bucket layer.

The compute path is libgpulsm.so (csrc/, sm_100a CUDA behind the C ABI in
include/gpulsm.h).  This package is the host-side mirror of the reference's
interfaces; it needs torch only for device buffers and streams.

The directory name contains hyphens, so import it with
``importlib.import_module("gpu-lsm-tree_b200")``.
"""
from . import _native  # noqa: F401
from ._native import (CapacityError, CudaError, DeviceTimeout, GpuLsmError, InvalidArgument,  # noqa: F401
                      LengthError, OutOfDeviceMemory, PublicationError, load)
from .dictionary import DictionaryConfig, GPULSMOpt, GpuLsmOptIndex, sort_pairs  # noqa: F401
from .flix import FlixIndex  # noqa: F401
from .serving import Server  # noqa: F401
from .tenants import TenantPool  # noqa: F401


def build(force: bool = False) -> str:
    """Compile libgpulsm.so in-tree for sm_100a (see build.py)."""
    from .build import build as _build

    return _build(force=force)
