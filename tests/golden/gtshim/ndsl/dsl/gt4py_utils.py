import numpy as np


def asarray(a):
    return np.asarray(a)


def make_storage_from_shape(shape, origin=None, backend=None):
    return np.zeros(shape)
