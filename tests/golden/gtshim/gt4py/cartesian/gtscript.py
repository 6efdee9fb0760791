"""gtscript names used by pySHiELD, bound to the numpy executor in ``_gtexec``."""
from _gtexec import (  # noqa: F401
    BACKWARD,
    FORWARD,
    PARALLEL,
    computation,
    exp,
    function,
    interval,
    log,
    sqrt,
)
