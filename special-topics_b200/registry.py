"""Backend registry (js_fdtd/src/backends/registry.js:13-84) with the b200 engine registered first.

``select_backend`` keeps the reference's never-throw probing and fallback
order, but this package ships exactly one backend: when no GPU is present the
selection fails loudly instead of falling back to a CPU path.
"""
from __future__ import annotations

from .backend import B200Backend

_LOADERS = {"b200": lambda: B200Backend()}
_cache: dict = {}


def load_backend(name: str):
    if name in _cache:
        return _cache[name]
    if name not in _LOADERS:
        raise ValueError(f'Unknown backend "{name}". Known: {", ".join(_LOADERS)}')
    try:
        b = _LOADERS[name]()
    except Exception:
        b = None
    _cache[name] = b
    return b


def select_backend(preferred: str = "auto"):
    order = ["b200"] if preferred in (None, "auto") else [preferred, "b200"]
    seen = set()
    for name in order:
        if name in seen:
            continue
        seen.add(name)
        b = load_backend(name)
        if b is None:
            continue
        try:
            ok = b.is_available()
        except Exception:
            ok = False
        if ok:
            return name, b
    raise RuntimeError("No FDTD backend is available (the b200 engine needs a CUDA GPU).")


def list_backends():
    out = []
    for name in _LOADERS:
        b = load_backend(name)
        if b is None:
            out.append({"name": name, "available": False, "detail": "module failed to load"})
            continue
        try:
            out.append({"name": name, "available": bool(b.is_available())})
        except Exception as e:  # pragma: no cover - is_available never raises
            out.append({"name": name, "available": False, "detail": str(e)})
    return out
