"""Stub of `pane.io` (names only)."""
import typing as t

FileOrPath = t.Any


def from_json(*args: t.Any, **kwargs: t.Any) -> t.Any:
    raise NotImplementedError("pane stub cannot parse files")
