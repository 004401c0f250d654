"""Stub of `pane.util` (names only)."""


def pluralize(word: str, plural: bool = False, article: str = '') -> str:
    return word + ('s' if plural else '')


def list_phrase(items) -> str:
    return ', '.join(map(str, items))
