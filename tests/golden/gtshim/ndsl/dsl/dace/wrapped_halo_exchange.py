class WrappedHaloUpdater:
    def __init__(self, *a, **k):
        pass
