"""C-ABI library: loads without a GPU, exports every declared symbol, host
helpers agree with the oracle, compute entry points fail loudly without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

import ts_b200 as T
from ts_b200 import _capi as C
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "ts_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ts_[a-z_0-9]+)\s*\(", src)))


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(C.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(C.EXPORTS) == names


def test_library_metadata():
    L = T.lib()
    assert L.ts_abi_version() == 1
    for i, name in enumerate(C.STRUCT_NAMES):
        assert L.ts_struct_from_name(name.encode()) == i
        assert L.ts_struct_name(i).decode() == name
    assert L.ts_struct_from_name(b"bogus") == -1
    assert L.ts_status_string(0) == b"ok"


@pytest.mark.parametrize("seed", [0, 1, 7, 123456789, 2**32 - 1])
def test_mdp_random_start_matches_glibc_rand(seed):
    for n, m in ((2000, 200), (50, 49), (10, 1)):
        a = T.random_start(T.PROBLEM_MDP, n, m, seed)
        b = O.mdp_random_initial(n, m, seed)
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("seed", [0, 3, 99, 2**31 + 5])
def test_maxbs_random_partition_and_draws(seed):
    for n in (2, 41, 1000, 100_001):
        a = T.random_start(T.PROBLEM_MAXBS, n, 0, seed)
        b = O.maxbs_random_partition(n, seed)
        np.testing.assert_array_equal(a, b)
        assert (a == 0).sum() == n // 2
    for init_random in (False, True):
        d = T.perturb_draws(1001, seed, 150, init_random, 7)
        e = O.maxbs_perturb_draws(1001, seed, init_random, 7, 75)
        np.testing.assert_array_equal(d, e)
        assert all(len(set(r.tolist())) == len(r) for r in d)


def test_draws_beyond_int32_pair_space():
    # n=100,000 -> 2.5e9 pairs (> int32): the library draws 64-bit indices in range
    d = T.perturb_draws(100_000, 5, 150, True, 3)
    assert d.max() < 50_000 * 50_000 and d.min() >= 0
    np.testing.assert_array_equal(d, O.maxbs_perturb_draws(100_000, 5, True, 3, 75))


def test_compute_without_device_fails_loudly():
    if T.lib() and _has_device():
        pytest.skip("a CUDA device is visible")
    with pytest.raises(T.TsError) as e:
        T.Graph(10, np.array([0], np.int32), np.array([1], np.int32), np.array([1], np.int32))
    assert e.value.status == C.ERR_NO_DEVICE


def _has_device():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_bad_host_helper_args():
    with pytest.raises(T.TsError):
        T.random_start(T.PROBLEM_MDP, 10, 10, 1)
    with pytest.raises(T.TsError):
        T.random_start(5, 10, 1, 1)
