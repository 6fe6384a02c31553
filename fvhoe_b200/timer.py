"""Multi-category wall-clock timer (same interface as fvhoe/timer.py:6-109)."""

import time
from typing import Iterable, Union


class Timer:
    def __init__(self, cats: Union[str, Iterable[str]] = (), precision: int = 2):
        self.cats = ()
        self._start_time = {}
        self.cum_time = {}
        self.precision = precision
        self.add_cat(cats)

    def add_cat(self, cat: Union[str, Iterable[str]]):
        for c in (cat,) if isinstance(cat, str) else cat:
            if c in self.cats:
                raise ValueError(f"Category '{c}' already exists.")
            self.cats = (*self.cats, c)
            self._start_time[c] = None
            self.cum_time[c] = 0.0

    def check_cat_existence(self, cat: str):
        if cat not in self.cats:
            raise ValueError(f"Category '{cat}' not found in timer categories.")

    def start(self, cat: str):
        self.check_cat_existence(cat)
        if self._start_time[cat] is not None:
            raise RuntimeError(f"Cannot start '{cat}' timer since it is already in progress.")
        self._start_time[cat] = time.time()

    def stop(self, cat: str):
        self.check_cat_existence(cat)
        if self._start_time[cat] is None:
            raise RuntimeError(f"Cannot stop '{cat}' timer since it is not in progress.")
        self.cum_time[cat] += time.time() - self._start_time[cat]
        self._start_time[cat] = None

    def report(self) -> str:
        width = max((len(c) for c in self.cats), default=8)
        lines = [f"{'Category':<{width}}  Time (s)"]
        for c in self.cats:
            lines.append(f"{c:<{width}}  {self.cum_time[c]:.{self.precision}f}")
        return "\n".join(lines)

    def to_dict(self, decimals: int = None) -> dict:
        d = self.precision if decimals is None else decimals
        return {c: round(t, d) for c, t in self.cum_time.items()}
