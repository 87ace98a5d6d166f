"""The stable radix sort (td3_radix_sort_pairs) against NumPy's stable argsort.

Sizes straddle the 2048-item tile and twice it (empty, single, ragged tails, many tiles); keys cover
heavy duplication, a single repeated key, and sorts on fewer bits than the keys hold
(the high bits must then be ignored, equal low bits kept in input order).
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _sort(keys: np.ndarray, bits: int):
    from tree_d_3d_b200 import _lib

    n = keys.size
    dev = torch.device("cuda", 0)
    k = torch.tensor(keys.astype(np.int64), device=dev).to(torch.int32)
    v = torch.arange(n, dtype=torch.int32, device=dev)
    k_alt, v_alt = torch.empty_like(k), torch.empty_like(v)
    ws = _lib.workspace(_lib.query("td3_radix_sort_workspace_size", n), dev)
    in_alt = ctypes.c_int(0)
    _lib.call("td3_radix_sort_pairs", k.data_ptr(), k_alt.data_ptr(), v.data_ptr(),
              v_alt.data_ptr(), n, bits, ctypes.addressof(in_alt), ws.data_ptr(), ws.numel(),
              _lib.stream(dev))
    ko, vo = (k_alt, v_alt) if in_alt.value else (k, v)
    return (ko.cpu().numpy().astype(np.int64) & 0xFFFFFFFF), vo.cpu().numpy().astype(np.int64)


@pytest.mark.parametrize("n", [0, 1, 2, 4095, 4096, 4097, 100_003, 3_000_001])
@pytest.mark.parametrize("kind", ["uniform32", "few", "same", "bits19"])
def test_radix_sort_is_stable_and_matches_numpy(n, kind):
    rng = np.random.default_rng(n + len(kind))
    bits = 32
    if kind == "uniform32":
        keys = rng.integers(0, 2**32, n, dtype=np.uint64)
    elif kind == "few":
        keys = rng.integers(0, 7, n, dtype=np.uint64) * 0x01010101
    elif kind == "same":
        keys = np.full(n, 0xDEADBEEF, dtype=np.uint64)
    else:
        keys = rng.integers(0, 2**32, n, dtype=np.uint64)
        bits = 19
    ko, vo = _sort(keys, bits)
    low = keys & np.uint64((1 << bits) - 1) if bits < 32 else keys
    order = np.argsort(low, kind="stable")
    assert np.array_equal(vo, order)
    assert np.array_equal(ko, keys[order].astype(np.int64))


@pytest.mark.parametrize("bits", [1, 5, 8, 9, 11, 12, 16, 20, 22, 23, 27, 31])
def test_radix_sort_digit_widths(bits):
    """Key widths that end on a full and on a partial digit: stable against NumPy on
    keys whose high bits must be ignored."""
    rng = np.random.default_rng(bits)
    n = 250_007
    keys = rng.integers(0, 2**32, n, dtype=np.uint64)
    ko, vo = _sort(keys, bits)
    order = np.argsort(keys & np.uint64((1 << bits) - 1), kind="stable")
    assert np.array_equal(vo, order)
    assert np.array_equal(ko, keys[order].astype(np.int64))
