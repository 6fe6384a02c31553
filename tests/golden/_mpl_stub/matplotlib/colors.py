"""Placeholder colors module."""


class LogNorm:  # pragma: no cover - placeholder
    def __init__(self, *args, **kwargs):
        pass
