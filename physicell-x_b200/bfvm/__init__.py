"""bfvm -- B200 implementation of PhysiCell-X BioFVM's 3-D diffusion-decay
LOD step with cell sources/sinks, behind the reference's interface.

The compute path is libbiofvm_b200.so (hand-written sm_100a CUDA, C ABI in
include/biofvm_b200.h); this package is the Python host mirror of it.
"""
from . import workloads
from .batch import Batch
from ._lib import BfvmError, kernel_launches, lib, status_string
from .solver import Microenvironment

__all__ = ["Batch", "BfvmError", "Microenvironment", "kernel_launches", "lib", "status_string", "workloads"]
