"""Stub of `pane.convert` (names only)."""
import typing as t

ConverterHandlers = t.Any
DataType = t.Any
