class GridSizer:
    pass


class SubtileGridSizer(GridSizer):
    pass
