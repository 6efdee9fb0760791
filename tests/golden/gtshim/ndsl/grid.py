class GridData:
    def __init__(self, area=None, ptop=None):
        self.area = area
        self.ptop = ptop


class DriverGridData:
    pass
