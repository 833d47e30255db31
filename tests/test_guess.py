"""The learned Newton initial guess: tensor-core kernels against the CPU
restatement in oracle/mlp_ref.py."""
import ctypes

import numpy as np
import pytest

from billardballraytracing3d_b200 import _capi as C
from oracle import mlp_ref as R


@pytest.mark.gpu
def test_umma_operand_layouts(built):
    """D = A B^T through tcgen05 with A and B staged K-major and MN-major."""
    lib = C.load_library()
    rng = np.random.default_rng(5)
    a = R.bf16_bits(rng.standard_normal((128, 64)))
    b = R.bf16_bits(rng.standard_normal((128, 64)))
    d = np.zeros((4, 128, 128), np.float32)
    rc = lib.bbrt_umma_check(C.ptr(a, ctypes.c_ushort), C.ptr(b, ctypes.c_ushort), C.ptr(d, ctypes.c_float))
    C.check(lib, rc, "bbrt_umma_check")
    want = R.from_bf16_bits(a) @ R.from_bf16_bits(b).T
    for v in range(4):
        err = np.max(np.abs(d[v] - want))
        assert err < 1e-3 * np.max(np.abs(want)), (v, err)
