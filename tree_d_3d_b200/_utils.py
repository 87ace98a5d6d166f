"""Argument checks and tensor conversions shared by the solvers.

The messages are those of the reference (src/tree_d_3d/_utils.py:11-63), so code that
matches on them keeps working.  Arrays become contiguous CUDA tensors of the current
device; results are returned as CUDA tensors for tensor inputs and as NumPy arrays
otherwise (the reference returns arrays of its input's backend).
"""

from __future__ import annotations

import numpy as np
import torch

from tree_d_3d_b200 import _lib


def _finite(name: str, value: float, *, minimum=None, positive=False) -> float:
    """src/tree_d_3d/_utils.py:11-20."""
    value = float(value)
    if not np.isfinite(value):
        raise ValueError(f"{name} must be finite")
    if minimum is not None and value < minimum:
        raise ValueError(f"{name} must be >= {minimum}")
    if positive and value <= 0:
        raise ValueError(f"{name} must be positive")
    return value


def _coincident() -> ValueError:
    return ValueError("Coincident charges require positive softening")


def _check_code(code: int) -> None:
    """src/tree_d_3d/_utils.py:26-35: status > 0 coincident charges, < 0 stack overflow."""
    if code > 0:
        raise _coincident()
    if code < 0:
        raise RuntimeError(
            "the quadtree is too deep for the traversal of the CUDA kernels; lower max_depth"
        )


def _check(status: torch.Tensor) -> None:
    """Read a device status word (synchronises its stream) and raise for a failure."""
    _check_code(int(status[0].item()))


def device() -> torch.device:
    """The CUDA device the solvers run on (the current one)."""
    if not torch.cuda.is_available():
        raise RuntimeError("tree_d_3d_b200 needs a CUDA device (it has no CPU fallback)")
    return torch.device("cuda", torch.cuda.current_device())


def _device(array, dtype=torch.float64) -> torch.Tensor:
    """A contiguous CUDA tensor of ``dtype`` (src/tree_d_3d/_utils.py:38-44)."""
    dev = device()
    if isinstance(array, torch.Tensor):
        return array.to(device=dev, dtype=dtype).contiguous()
    np_dtype = np.int64 if dtype == torch.int64 else np.float64
    return torch.as_tensor(np.ascontiguousarray(np.asarray(array, dtype=np_dtype)), device=dev)


def _points(array, name: str) -> torch.Tensor:
    """``array`` as a contiguous component-major (2, N) float64 CUDA tensor
    (src/tree_d_3d/_utils.py:52-63)."""
    points = _device(array)
    if points.ndim != 2 or points.shape[0] != 2:
        raise ValueError(
            f"{name} must have shape (2, N) (component-major), got {tuple(points.shape)}"
        )
    return points


def wants_numpy(array) -> bool:
    """Whether results for this input go back as NumPy arrays (non-tensor inputs)."""
    return not isinstance(array, torch.Tensor)


def out(result, as_numpy: bool):
    """Results as CUDA tensors, or NumPy arrays for NumPy callers."""
    if not as_numpy:
        return result
    if isinstance(result, tuple):
        return tuple(r.cpu().numpy() for r in result)
    return result.cpu().numpy()


def status_word(dev: torch.device) -> torch.Tensor:
    return torch.zeros(1, dtype=torch.int64, device=dev)


__all__ = ["_finite", "_check", "_check_code", "_device", "_points", "device", "out",
           "wants_numpy", "status_word", "_lib"]
