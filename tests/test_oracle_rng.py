"""Known-answer checks of the oracle's random-number building blocks
(KernelHelpers.h:10-116; the host seed stream std::mt19937_64,
SyclBridge.cpp:83)."""
import numpy as np

from oracle_lib import lib

import ctypes as C


def test_mt19937_64_known_answer():
    # C++ [rand.predef]: the 10000th output of a default-constructed
    # mt19937_64 (seed 5489) is 9981545732273789042.
    out = (C.c_uint64 * 10000)()
    lib().orc_mt19937_64(5489, 10000, out)
    assert out[9999] == 9981545732273789042


def test_splitmix64_known_answer():
    # SplitMix64 from state 0: first output 0xE220A8397B1DCDAF.  The per-item
    # seed mixes the base as base ^ (golden + id) before one step, so with
    # base = golden and id = 0 the state is 0.
    golden = 0x9E3779B97F4A7C15
    assert lib().orc_per_item_seed(golden ^ golden, (2**64 - golden) % 2**64) == 0xE220A8397B1DCDAF


def test_xorshift128_known_answer():
    # Marsaglia (2003), xor128 with x,y,z,w = 123456789, 362436069,
    # 521288629, 88675123: first output 3701687786.
    out = np.zeros(2, np.uint32)
    lib().orc_xorshift128_raw(123456789, 362436069, 521288629, 88675123, 2, out.ctypes.data_as(C.POINTER(C.c_uint32)))
    assert int(out[0]) == 3701687786


def test_xorshift_float_range_and_grid():
    n = 4096
    out = np.zeros(n, np.float32)
    lib().orc_xorshift_floats(12345, n, out.ctypes.data_as(C.POINTER(C.c_float)))
    assert out.min() >= 0.0 and out.max() < 1.0
    # (u >> 8) * 2^-24: every value is a multiple of 2^-24
    assert np.all(np.mod(out.astype(np.float64) * 2**24, 1.0) == 0.0)
