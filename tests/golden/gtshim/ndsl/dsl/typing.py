import numpy as np

Float = np.float64
Int = int
Bool = bool


class FloatField:
    pass


class FloatFieldIJ:
    pass


class FloatFieldI:
    pass
