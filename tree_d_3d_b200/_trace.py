"""NVTX ranges around the solver's host phases, for nsys / ncu timelines.

The reference marks its phases as scope-profiler regions named
``tree_d_3d.<module>.<op>`` (src/tree_d_3d/_profiling.py:10-13, the ``@sp.profile``
decorators of src/tree_d_3d/flat_tree.py:124, 987, 1151, 1460 and the ``sp.region``
blocks of :672, :801), off unless a tag enables them.  Here the same names become NVTX
ranges, off unless the environment variable ``TREE_D_3D_NVTX`` is set to a non-empty
value other than ``0`` when the package is imported (or ``enable()`` is called): when
off, ``region`` costs one attribute test.
"""

from __future__ import annotations

import contextlib
import functools
import os

import torch

_ENABLED = os.environ.get("TREE_D_3D_NVTX", "") not in ("", "0")

#: every range name opened since enable(), in order (for tests and quick inspection)
opened: list = []


def enable(on: bool = True) -> None:
    """Turn the ranges on or off for the rest of the process."""
    global _ENABLED
    _ENABLED = bool(on)


def enabled() -> bool:
    return _ENABLED


@contextlib.contextmanager
def region(name: str):
    """An NVTX range named ``tree_d_3d.<name>`` while the block runs (when enabled)."""
    if not _ENABLED:
        yield
        return
    full = f"tree_d_3d.{name}"
    opened.append(full)
    torch.cuda.nvtx.range_push(full)
    try:
        yield
    finally:
        torch.cuda.nvtx.range_pop()


def profile(name: str):
    """Decorator form of ``region`` for whole methods."""

    def wrap(fn):
        @functools.wraps(fn)
        def inner(*args, **kwargs):
            if not _ENABLED:
                return fn(*args, **kwargs)
            with region(name):
                return fn(*args, **kwargs)

        return inner

    return wrap
