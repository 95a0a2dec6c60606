"""Test-only NumPy subset of ``autoray`` (pinned 0.10.1 by the reference, ``uv.lock:14-15``).

Enough of ``autoray.do`` for the reference's NumPy backend: the names its ops call
(``ar.do("transpose"|"reshape"|"concatenate"|"matmul"|"linalg.svd"|...)``) resolve to the
NumPy function of the same dotted name, exactly as autoray does for the ``numpy`` backend.
Registration hooks are accepted and ignored (the reference registers its own tensor type
as a backend for user convenience; nothing on the contraction path dispatches through it).
Used only by ``tests/golden/make_golden.py``.
"""

import importlib

import numpy as np

from . import autoray as autoray  # noqa: F401  (the reference touches ar.autoray in ad.py)

_REGISTERED = {}


def _resolve(name):
    obj = np
    for part in name.split("."):
        obj = getattr(obj, part)
    return obj


def do(fn, *args, like=None, **kwargs):
    key = None
    target = like if like is not None else (args[0] if args else None)
    if isinstance(target, str):
        key = target
    elif target is not None:
        key = type(target).__module__.split(".")[0]
    if key in _REGISTERED and fn in _REGISTERED[key]:
        return _REGISTERED[key][fn](*args, **kwargs)
    if fn == "linalg.svd":
        return np.linalg.svd(*args, **kwargs)
    if fn == "astype":
        x, dtype = args
        return np.asarray(x).astype(dtype)
    if fn in ("zeros", "eye", "array", "ones", "empty"):
        kwargs.pop("like", None)
    return _resolve(fn)(*args, **kwargs)


def get_dtype_name(x):
    return np.asarray(x).dtype.name


def infer_backend(x):
    mod = type(x).__module__.split(".")[0]
    return "numpy" if mod in ("numpy", "builtins") else mod


def to_numpy(x):
    return np.asarray(x)


def register_backend(cls, name):
    return None


def register_dispatch(*args, **kwargs):
    return None


def register_function(backend, name, fn, wrap=False):
    _REGISTERED.setdefault(backend, {})[name] = fn
