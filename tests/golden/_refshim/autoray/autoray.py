"""Internal tables the reference's ``ad.py`` pokes at; empty here."""

_FUNCS = {}
_NAMESPACE_CACHE = {}
