"""Minimal stand-in for matplotlib so the reference package imports without it.

Only used by the fixture generator in tests/golden; nothing here draws.
"""
from . import cm, colors, pyplot  # noqa: F401
