"""Kernel operator types (reference: numerics/kernel_op_types.py:19-30).

The reference selects a TPU stencil implementation (conv, slice or matmul).
Here every stencil is a direct CUDA stencil; the key is accepted and kept for
config compatibility only.
"""

import enum


class KernelOpType(enum.Enum):
  KERNEL_OP_CONV = 'ApplyKernelConvOp'
  KERNEL_OP_SLICE = 'ApplyKernelSliceOp'
  KERNEL_OP_MATMUL = 'ApplyKernelMulOp'
