"""Finite differences (reference: numerics/gradient.py:21-94).

forward_1: (f[i+1]-f[i])/h; backward_1: (f[i]-f[i-1])/h;
central_2: (f[i+1]-f[i-1])/(2h). Points whose stencil leaves the array are 0.
"""

from swirlc_b200.numerics import _pointwise


def forward_1(f, h, dim, kernel_op=None):
  del kernel_op
  return _pointwise.stencil(f, 0, dim, h)


def backward_1(f, h, dim, kernel_op=None):
  del kernel_op
  return _pointwise.stencil(f, 1, dim, h)


def central_2(f, h, dim, kernel_op=None):
  del kernel_op
  return _pointwise.stencil(f, 2, dim, h)
