"""The allocation-free sort entry point (yb_sort_pairs_noalloc).

It exists for callers that may not allocate device memory where they sort (code hosted in
another framework that owns the device-memory budget, or fixed-budget loops where an
allocation is an error): it sorts caller-owned device buffers using only a fixed scratch
array compiled into the library.  This test calls it through the C ABI on two different
inputs in a row (the scratch keeps the previous call's contents, so the second call checks
that everything that must start at zero is cleared) and compares each result with the
allocating entry point's, bit for bit (an integer sort has no tolerance).  It also checks
that a request above the fixed limit is refused with its own status code.  This file is
named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

import yarnball_b200 as yb
from yarnball_b200 import _abi


MAX_N = 262144  # YB_SORT_NOALLOC_MAX_N
SCRATCH_TOO_SMALL = 13  # YB_ERR_SCRATCH_TOO_SMALL


def _noalloc_sort(keys, vals, bits):
    import torch

    kin = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    vin = torch.from_numpy(vals.copy()).cuda()
    kout = torch.empty_like(kin)
    vout = torch.empty_like(vin)
    stream = torch.cuda.current_stream()
    st = _abi.load().yb_sort_pairs_noalloc(
        ctypes.c_void_p(kin.data_ptr()), ctypes.c_void_p(vin.data_ptr()), ctypes.c_void_p(kout.data_ptr()),
        ctypes.c_void_p(vout.data_ptr()), len(keys), bits, ctypes.c_void_p(stream.cuda_stream))
    return st, kout.cpu().numpy().view(np.uint64), vout.cpu().numpy()


def _stable_order(keys, bits):
    """Reference order: a stable argsort on the low `bits` key bits (numpy, on the host)."""
    mask = np.uint64((1 << bits) - 1) if bits < 64 else np.uint64(0xFFFFFFFFFFFFFFFF)
    return np.argsort(keys & mask, kind="stable")


@pytest.mark.gpu
def test_noalloc_sort_matches_allocating_sort_twice():
    rng = np.random.default_rng(11)
    # calls in a row with different sizes and key widths: a full 5-pass key at the size limit,
    # an 8-pass key, a 1-pass key (odd pass count: the only pass writes the caller's output),
    # a single pair, and bits = 0 (nothing to sort: a copy)
    cases = [(MAX_N, 39), (100003, 64), (5000, 8), (1, 30), (777, 0)]
    for n, bits in cases:
        # keys below 2**bits, as the BVH build passes them (bits = 0: any keys, left in place)
        keys = rng.integers(0, 2**min(bits, 63) if bits else 2**63, size=n, dtype=np.uint64)
        keys[: n // 4] = keys[n // 2]  # duplicates exercise stability
        vals = rng.permutation(n).astype(np.int32)
        st, ko, vo = _noalloc_sort(keys, vals, bits)
        assert st == 0, (n, bits)
        order = _stable_order(keys, bits)
        assert np.array_equal(ko, keys[order]), (n, bits)
        assert np.array_equal(vo, vals[order]), (n, bits)
        rk, rv = yb.sort_pairs(keys, vals, bits)  # the existing (allocating) entry point
        assert np.array_equal(ko, rk), (n, bits)
        assert np.array_equal(vo, rv), (n, bits)


@pytest.mark.gpu
def test_noalloc_sort_rejects_sizes_above_its_scratch():
    keys = np.zeros(MAX_N + 1, np.uint64)
    vals = np.zeros(MAX_N + 1, np.int32)
    st, _, _ = _noalloc_sort(keys, vals, 30)
    assert st == SCRATCH_TOO_SMALL


@pytest.mark.parametrize("alias", ["keys", "vals"])
def test_noalloc_sort_refuses_output_overlapping_input(alias):
    """An in-place call is refused before any device work: the argument check reads no
    memory, so placeholder addresses are enough and this runs without a GPU."""
    lib = _abi.load()
    n = 1000
    kin, vin, kout, vout = 0x100000, 0x200000, 0x300000, 0x400000
    if alias == "keys":
        kout = kin + 8 * 10  # overlaps the tail of the input keys
    else:
        vout = vin
    st = lib.yb_sort_pairs_noalloc(ctypes.c_void_p(kin), ctypes.c_void_p(vin), ctypes.c_void_p(kout),
                                   ctypes.c_void_p(vout), n, 30, None)
    assert st == 1  # YB_ERR_INVALID_ARGUMENT
