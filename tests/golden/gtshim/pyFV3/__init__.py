class DynamicalCoreConfig:
    pass


class DycoreState:
    pass
