class DataArray:
    def __init__(self, *a, **k):
        pass


class Dataset:
    def __init__(self, *a, **k):
        pass
