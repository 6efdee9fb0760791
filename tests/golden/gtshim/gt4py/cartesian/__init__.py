from . import gtscript  # noqa: F401
