"""Stub of `pane.annotations` (names only)."""
import typing as t


class ConvertAnnotation:
    pass


class Tagged(ConvertAnnotation):
    def __init__(self, *args: t.Any, **kwargs: t.Any):
        pass


def shape(*args: t.Any, **kwargs: t.Any) -> ConvertAnnotation:
    return ConvertAnnotation()
