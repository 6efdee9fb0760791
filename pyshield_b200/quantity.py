"""Quantity-like containers and the strided-pointer view the C-ABI takes.

pySHiELD passes NDSL ``Quantity`` objects: ``.data`` is the full storage
(compute domain plus halo), ``.origin`` / ``.extent`` locate the compute
domain. Any object with those three attributes works here, as long as
``.data`` is a float64 CUDA array: a ``torch.Tensor`` or anything exposing
``__cuda_array_interface__`` (CuPy, Numba, ...). The layout is free: the
element strides are passed to the kernels.
"""

import numpy as np

from ._lib import ShieldField2D, ShieldField3D


class Quantity:
    """Minimal NDSL-style quantity: storage + compute-domain origin/extent."""

    def __init__(self, data, dims, units, origin=None, extent=None):
        self.data = data
        self.dims = tuple(dims)
        self.units = units
        nd = len(tuple(data.shape))
        self.origin = tuple(origin) if origin is not None else (0,) * nd
        self.extent = tuple(extent) if extent is not None else tuple(data.shape)

    @property
    def view(self):
        """The compute-domain view of ``data`` (torch tensors only)."""
        sl = tuple(slice(o, o + e) for o, e in zip(self.origin, self.extent))
        return self.data[sl]


def _array_info(a):
    """(device pointer, element strides, shape) of a float64 CUDA array."""
    try:
        import torch

        if isinstance(a, torch.Tensor):
            if a.dtype != torch.float64:
                raise TypeError(f"expected float64 data, got {a.dtype}")
            if not a.is_cuda:
                raise TypeError("the microphysics kernels need device (CUDA) arrays")
            return a.data_ptr(), tuple(a.stride()), tuple(a.shape)
    except ImportError:  # pragma: no cover
        pass
    cai = getattr(a, "__cuda_array_interface__", None)
    if cai is None:
        raise TypeError(f"{type(a).__name__} is not a CUDA array (no __cuda_array_interface__)")
    if np.dtype(cai["typestr"]) != np.float64:
        raise TypeError(f"expected float64 data, got {cai['typestr']}")
    shape = tuple(cai["shape"])
    if cai.get("strides") is None:
        st = [1] * len(shape)
        for d in range(len(shape) - 2, -1, -1):
            st[d] = st[d + 1] * shape[d + 1]
        strides = tuple(st)
    else:
        if any(s % 8 for s in cai["strides"]):
            raise ValueError("strides must be whole elements")
        strides = tuple(s // 8 for s in cai["strides"])
    return cai["data"][0], strides, shape


def _unpack(q):
    data = getattr(q, "data", q)
    origin = getattr(q, "origin", None)
    ptr, strides, shape = _array_info(data)
    if origin is None:
        origin = (0,) * len(shape)
    return ptr, strides, shape, tuple(origin)


def field3d(q, extent=None):
    """ShieldField3D for a 3-D quantity: pointer at the compute-domain origin."""
    ptr, st, shape, org = _unpack(q)
    if len(shape) != 3:
        raise ValueError(f"expected a 3-D field, got shape {shape}")
    ext = tuple(extent) if extent is not None else tuple(getattr(q, "extent", shape))
    for d in range(3):
        if org[d] < 0 or org[d] + ext[d] > shape[d]:
            raise ValueError(f"domain origin {org} extent {ext} exceeds storage {shape}")
    off = org[0] * st[0] + org[1] * st[1] + org[2] * st[2]
    return ShieldField3D(ptr + 8 * off, st[0], st[1], st[2])


def field2d(q, extent=None):
    ptr, st, shape, org = _unpack(q)
    if len(shape) != 2:
        raise ValueError(f"expected a 2-D field, got shape {shape}")
    ext = tuple(extent) if extent is not None else tuple(getattr(q, "extent", shape))
    for d in range(2):
        if org[d] < 0 or org[d] + ext[d] > shape[d]:
            raise ValueError(f"domain origin {org} extent {ext} exceeds storage {shape}")
    off = org[0] * st[0] + org[1] * st[1]
    return ShieldField2D(ptr + 8 * off, st[0], st[1])
