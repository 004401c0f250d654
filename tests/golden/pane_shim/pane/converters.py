"""Stub of `pane.converters` (names only)."""
import typing as t

T = t.TypeVar('T')
ConverterHandlers = t.Any


class ErrorNode:
    pass


class Converter(t.Generic[T]):
    pass


def make_converter(ty: t.Any, handlers: t.Any = None) -> t.Any:
    return Converter()
