"""Configuration objects with manapy's semantics (``manapy/base/base.py:8-13,65-225``).

``Struct`` is an attribute bag whose ``get(key, default, msg_if_none)`` raises
``ValueError(msg_if_none)`` when the value is missing; ``make_get_conf`` lets
keyword arguments override a ``Struct``.  Solver and domain options are read
through these exactly as manapy reads them.
"""
from __future__ import annotations

from copy import copy, deepcopy

__all__ = ["Struct", "make_get_conf", "process_conf"]


def make_get_conf(conf, kwargs):
    def _get_conf_item(name, default=None, msg_if_none=None):
        return kwargs.get(name, conf.get(name, default=default, msg_if_none=msg_if_none))
    return _get_conf_item


class Struct(object):
    def __init__(self, **kwargs):
        if kwargs:
            self.__dict__.update(kwargs)

    def __repr__(self):
        return "Struct(%s)" % ", ".join("%s=%r" % kv for kv in self.__dict__.items())

    def to_dict(self):
        return copy(self.__dict__)

    def get(self, key, default=None, msg_if_none=None):
        out = getattr(self, key, default)
        if (out is None) and (msg_if_none is not None):
            raise ValueError(msg_if_none)
        return out

    def update(self, other, **kwargs):
        if other is None:
            return
        if not isinstance(other, dict):
            other = other.to_dict()
        self.__dict__.update(other, **kwargs)

    def set_default(self, key, default=None):
        return self.__dict__.setdefault(key, default)

    def copy(self, deep=False, name=None):
        other = deepcopy(self) if deep else copy(self)
        if hasattr(self, "name"):
            other.name = name if name is not None else self.name + "_copy"
        return other


def process_conf(parameters, conf, kwargs):
    """Options from a ``(name, type, default, required, doc)`` table, as the
    ``process_conf`` classmethods of manapy's solvers build them
    (``manapy/solvers/advecdiff/system.py:37-66``)."""
    if conf is None:
        conf = Struct()
    get = make_get_conf(conf, kwargs)
    opts = Struct()
    allow_extra = False
    for name, _, default, required, _ in parameters:
        if name == "*":
            allow_extra = True
            continue
        msg = ('missing "%s" in options!' % name) if required else None
        setattr(opts, name, get(name, default, msg))
    if allow_extra:
        other = set(conf.to_dict().keys()).difference(opts.to_dict().keys())
        for name in other:
            setattr(opts, name, get(name, None, None))
    return opts
