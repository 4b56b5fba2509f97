"""tcgen05 building blocks on the device: operand layout, descriptors, TMEM reads (B200)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _selftest(n, k, split, seed=0):
    from apollo_b200.dg import load_library
    lib = load_library()
    fn = lib.apollo_dg_selftest_umma
    fn.restype = C.c_int
    fp = C.POINTER(C.c_float)
    fn.argtypes = [C.c_int, C.c_int, fp, fp, fp, C.c_int]
    rng = np.random.default_rng(seed)
    A = rng.uniform(-1, 1, (128, k)).astype(np.float32)
    B = rng.uniform(-1, 1, (n, k)).astype(np.float32)
    D = np.zeros((128, n), dtype=np.float32)
    rc = fn(n, k, A.ctypes.data_as(fp), B.ctypes.data_as(fp), D.ctypes.data_as(fp), split)
    ref = A.astype(np.float64) @ B.astype(np.float64).T
    return rc, D, ref


@pytest.mark.parametrize("n,k", [(16, 8), (96, 16), (256, 32), (48, 24)])
def test_tf32_single_product(n, k):
    rc, D, ref = _selftest(n, k, split=0)
    assert rc == 0
    err = np.abs(D - ref).max() / np.abs(ref).max()
    assert err < 5e-3, err


@pytest.mark.parametrize("n,k", [(16, 8), (96, 16), (256, 32)])
def test_tf32_three_term_split(n, k):
    """Ahi Bhi + Ahi Blo + Alo Bhi reaches fp32 accuracy."""
    rc, D, ref = _selftest(n, k, split=1, seed=1)
    assert rc == 0
    err = np.abs(D - ref).max() / np.abs(ref).max()
    assert err < 2e-6, err
