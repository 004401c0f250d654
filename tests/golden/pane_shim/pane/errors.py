"""Stub of `pane.errors` (names only)."""
from .converters import ErrorNode  # noqa: F401


class ConvertError(Exception):
    pass


class ParseInterrupt(Exception):
    pass


class WrongTypeError(Exception):
    def __init__(self, *args, **kwargs):
        super().__init__(*args)


class ProductErrorNode(Exception):
    def __init__(self, *args, **kwargs):
        super().__init__(*args)
