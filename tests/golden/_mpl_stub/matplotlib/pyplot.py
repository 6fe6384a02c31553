"""Placeholder pyplot module."""


def __getattr__(name):  # pragma: no cover - placeholder
    raise RuntimeError("plotting is unavailable in this environment")
