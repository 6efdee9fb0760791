"""NamelistDefaults mirrors the defaults chosen in pyshield_b200._config."""
import dataclasses

from pyshield_b200._config import PhysicsConfig as _PC


class NamelistDefaults:
    pass


for _f in dataclasses.fields(_PC):
    if _f.default is not dataclasses.MISSING:
        setattr(NamelistDefaults, _f.name, _f.default)


class Namelist:
    pass
