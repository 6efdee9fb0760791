class CubedToLatLon:
    def __init__(self, *a, **k):
        pass
