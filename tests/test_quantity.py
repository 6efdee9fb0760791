"""Strided-pointer views handed to the C-ABI (no GPU needed)."""
import numpy as np
import pytest

from pyshield_b200.quantity import field2d, field3d


class FakeCuda:
    """An object with __cuda_array_interface__ (like CuPy/Numba arrays)."""

    def __init__(self, shape, strides_bytes=None, ptr=1 << 20, typestr="<f8"):
        self.shape = shape
        self.__cuda_array_interface__ = {
            "shape": shape, "typestr": typestr, "data": (ptr, False), "strides": strides_bytes, "version": 3,
        }


class Q:
    def __init__(self, data, origin, extent):
        self.data, self.origin, self.extent = data, origin, extent


def test_c_order_storage():
    a = FakeCuda((13, 11, 80))
    f = field3d(Q(a, (3, 3, 0), (6, 4, 79)))
    assert (f.si, f.sj, f.sk) == (11 * 80, 80, 1)
    assert f.ptr == (1 << 20) + 8 * (3 * 11 * 80 + 3 * 80)


def test_ifirst_storage():
    a = FakeCuda((13, 11, 80), strides_bytes=(8, 8 * 13, 8 * 13 * 11))
    f = field3d(Q(a, (3, 3, 0), (6, 4, 79)))
    assert (f.si, f.sj, f.sk) == (1, 13, 143)
    assert f.ptr == (1 << 20) + 8 * (3 + 3 * 13)


def test_rejects_domain_outside_storage_and_wrong_dtype():
    a = FakeCuda((13, 11, 80))
    with pytest.raises(ValueError):
        field3d(Q(a, (3, 3, 0), (11, 4, 79)))
    with pytest.raises(TypeError):
        field3d(Q(FakeCuda((13, 11, 80), typestr="<f4"), (0, 0, 0), (1, 1, 1)))
    with pytest.raises(TypeError):
        field3d(Q(np.zeros((4, 4, 4)), (0, 0, 0), (4, 4, 4)))


def test_2d():
    f = field2d(Q(FakeCuda((13, 11)), (3, 3), (6, 4)))
    assert (f.si, f.sj) == (11, 1)
