"""Loader of ``libtreed3d.so``, the sm_100a CUDA library behind the C ABI.

The argument types of every entry point are read from its declaration in
``include/treed3d.h``; calls go through :func:`call`, which turns a nonzero return
code into an exception.  There is no fallback: without the built library (see
``tree_d_3d_b200/build.py``) or a CUDA device every solver call raises.
"""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import torch

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "libtreed3d.so"
HEADER = HERE.parent / "include" / "treed3d.h"

OK, EINVAL, ECUDA, ENEEDMORE, EWORKSPACE, EDEPTH, ETOOLARGE = 0, 1, 2, 3, 4, 5, 6
KERNEL_COULOMB, KERNEL_LOG = 0, 1

_CTYPES = {
    "int": ctypes.c_int,
    "int64_t": ctypes.c_int64,
    "double": ctypes.c_double,
    "size_t": ctypes.c_size_t,
    "float": ctypes.c_float,
}

_lib = None


class LibraryError(RuntimeError):
    """A call of the CUDA library failed."""


def _parse_header(text: str) -> dict:
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    protos = {}
    for m in re.finditer(r"(?m)^\s*(const char\*|int|size_t|void)\s+(td3_\w+)\(([^;]*?)\);", text):
        ret, name, params = m.group(1), m.group(2), m.group(3)
        args = []
        params = " ".join(params.split())
        if params and params != "void":
            for p in params.split(","):
                p = p.strip()
                if "*" in p:
                    args.append(ctypes.c_void_p)
                else:
                    ctype = p.replace("const ", "").split()[0]
                    args.append(_CTYPES[ctype])
        restype = {"int": ctypes.c_int, "size_t": ctypes.c_size_t, "const char*": ctypes.c_char_p,
                   "void": None}[ret]
        protos[name] = (restype, args)
    return protos


def lib():
    """The loaded library (loaded once per process)."""
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            raise ImportError(
                f"{LIBRARY} is missing: build it with `python -m tree_d_3d_b200.build` "
                "(this package has no CPU fallback)"
            )
        handle = ctypes.CDLL(str(LIBRARY))
        for name, (restype, args) in _parse_header(HEADER.read_text()).items():
            fn = getattr(handle, name)
            fn.restype = restype
            fn.argtypes = args
        _lib = handle
    return _lib


def declared_symbols() -> list:
    """Names of every entry point declared in include/treed3d.h."""
    return sorted(_parse_header(HEADER.read_text()))


def call(name: str, *args) -> int:
    """Call entry point ``name``; raise LibraryError on an error code other than ENEEDMORE."""
    rc = getattr(lib(), name)(*args)
    if rc == EDEPTH:
        raise RuntimeError(
            "the quadtree is too deep for the traversal of the CUDA kernels; lower max_depth"
        )
    if rc not in (OK, ENEEDMORE):
        detail = lib().td3_last_error().decode() if rc == ECUDA else ""
        raise LibraryError(f"{name} failed with code {rc} {detail}".strip())
    return rc


def call_code(name: str, *args) -> int:
    """Call entry point ``name`` and return its code; raise LibraryError only for a CUDA
    failure (the caller interprets the other codes)."""
    rc = getattr(lib(), name)(*args)
    if rc == ECUDA:
        raise LibraryError(f"{name} failed with code {rc} {lib().td3_last_error().decode()}")
    return rc


def query(name: str, *args) -> int:
    """A size query (``*_workspace_size``)."""
    return int(getattr(lib(), name)(*args))


def ptr(t: torch.Tensor | None) -> int | None:
    """The device address of a contiguous tensor (None for None)."""
    if t is None:
        return None
    return t.data_ptr()


def stream(device: torch.device | None = None) -> int:
    """The current CUDA stream handle of ``device``."""
    return torch.cuda.current_stream(device).cuda_stream


def workspace(nbytes: int, device: torch.device) -> torch.Tensor:
    """Scratch memory for one call, from torch's caching allocator."""
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
