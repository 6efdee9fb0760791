from enum import Enum


class MetaEnumStr(type(Enum)):
    def __contains__(cls, item):
        if isinstance(item, cls):
            return True
        return item in {m.value for m in cls}
