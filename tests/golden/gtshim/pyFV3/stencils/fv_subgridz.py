class DryConvectiveAdjustment:
    def __init__(self, *a, **k):
        pass
