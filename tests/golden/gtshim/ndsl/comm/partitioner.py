class TilePartitioner:
    pass
