"""The flux kernels divide through the hardware approximate reciprocal refined by
Newton-Raphson steps (two in FP64, none in FP32). Checked against CUDA's IEEE division
on 4M pseudo-random operand pairs spanning 2^-20 .. 2^20:
  FP64: max relative error <= 4 ulp (8.9e-16);  FP32: <= 4 ulp (4.8e-7)."""
import ctypes

import numpy as np
import pytest

from philip_b200 import _lib


@pytest.mark.gpu
def test_quotient_against_ieee_division():
    L = _lib.load()
    out = np.zeros(2)
    _lib.check(L.ph_quotient_selftest(20261203, 1 << 22, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    print(f"quotient max rel err: fp64 {out[0]:.3e}, fp32 {out[1]:.3e}")
    assert out[0] <= 4 * 2.0 ** -53
    assert out[1] <= 4 * 2.0 ** -24
