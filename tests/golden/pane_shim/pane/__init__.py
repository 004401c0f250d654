"""Minimal stand-in for the `pane` package (py-pane), used ONLY to import the
reference phaser sources in this container when generating golden fixtures.

The real `pane` converts YAML/JSON into typed dataclasses.  The fixture
generator never parses a plan, it builds the reference's state objects and
plan dataclasses directly, so this stub only has to make the reference modules
importable and make `Dataclass` subclasses constructible with keyword
arguments and defaults.
"""
import dataclasses
import typing as t

from . import annotations, converters, errors, util, convert, io  # noqa: F401

ConvertError = errors.ConvertError


class PaneBase:
    def __init_subclass__(cls, kw_only: bool = True, allow_extra: bool = False,
                          frozen: bool = False, **kwargs: t.Any):
        super().__init_subclass__()
        # eq=False keeps identity hashing, so instances may be class-level
        # defaults and arguments of lru_cache'd functions.
        dataclasses.dataclass(kw_only=True, eq=False, frozen=False)(cls)

    def into_data(self) -> t.Dict[str, t.Any]:
        return dataclasses.asdict(self)

    def dict(self, set_only: bool = False) -> t.Dict[str, t.Any]:
        return dataclasses.asdict(self)


def field(*, default: t.Any = dataclasses.MISSING, default_factory: t.Any = dataclasses.MISSING,
          converter: t.Any = None, init: bool = True, exclude: bool = False, **kwargs: t.Any) -> t.Any:
    return dataclasses.field(default=default, default_factory=default_factory, init=init)


def from_data(data: t.Any, ty: t.Any) -> t.Any:
    if isinstance(ty, type) and isinstance(data, dict):
        return ty(**data)
    return ty(data) if callable(ty) else data


def into_data(val: t.Any) -> t.Any:
    if dataclasses.is_dataclass(val):
        return dataclasses.asdict(val)  # type: ignore
    return val
