class Namelist(dict):
    pass


def read(path):
    raise FileNotFoundError(path)
