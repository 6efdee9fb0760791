class TilePartitioner:
    """Stand-in for NDSL's TilePartitioner: the subtile (y, x) of each rank
    of a layout, ranks row by row."""

    def __init__(self, layout=(1, 1)):
        self.layout = tuple(layout)

    def subtile_index(self, rank):
        return (rank // self.layout[0], rank % self.layout[0])
