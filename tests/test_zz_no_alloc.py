"""thorx_device_sum_noalloc: the allocation-free device sum against thorx_device_sum.

Collected last on purpose (file name), so it runs both after every other test in the session and,
when run alone, in a fresh process; it holds in either order because the only state it keeps is
the scratch address of each device, looked up on the first call.
"""
import math

import numpy as np
import pytest

import thor_b200

EPS = np.finfo(np.float64).eps


def _cancelling(n, seed):
    rng = np.random.default_rng(seed)
    big = rng.standard_normal(n) * 1e12
    x = np.concatenate([big, -big[::-1], rng.standard_normal(n)])
    rng.shuffle(x)
    return x


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 2049, 1_000_003])
def test_noalloc_sum_equals_the_allocating_sum_on_two_calls_in_a_row(n):
    import torch
    x = _cancelling(n, 11 + n)
    xd = torch.from_numpy(x).cuda()
    torch.cuda.synchronize()
    first = thor_b200.device_sum_noalloc(xd.data_ptr(), x.size)
    second = thor_b200.device_sum_noalloc(xd.data_ptr(), x.size)
    want = thor_b200.device_sum(xd.data_ptr(), x.size)
    exact = math.fsum(x)
    # same kernels, same order of addition: identical bits (tolerance 0)
    assert first == want and second == want, (first, second, want)
    assert abs(first - exact) <= 2 * EPS * abs(exact) + 4 * x.size * EPS ** 2 * math.fsum(
        np.abs(x))


@pytest.mark.gpu
def test_noalloc_sum_at_its_limit_and_beyond():
    import torch
    nmax = thor_b200.NOALLOC_SUM_MAX_N
    g = torch.Generator(device="cuda").manual_seed(5)
    xd = torch.rand(nmax + 1, dtype=torch.float64, device="cuda", generator=g)
    torch.cuda.synchronize()
    a = thor_b200.device_sum_noalloc(xd.data_ptr(), nmax)
    b = thor_b200.device_sum_noalloc(xd.data_ptr(), nmax)
    want = thor_b200.device_sum(xd.data_ptr(), nmax)
    assert a == want and b == want, (a, b, want)
    assert abs(a - float(xd[:nmax].sum())) <= 1e-12 * a
    # one element more than the scratch holds: refused before any launch, buffer is big enough
    with pytest.raises(thor_b200.ThorxError) as e:
        thor_b200.device_sum_noalloc(xd.data_ptr(), nmax + 1)
    assert e.value.code == thor_b200.E_ARG
    assert "exceeds the fixed scratch limit" in str(e.value)
    del xd
    torch.cuda.empty_cache()


@pytest.mark.gpu
def test_noalloc_sum_rejects_bad_arguments_and_stays_usable():
    import torch
    xd = torch.ones(1000, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    assert thor_b200.device_sum_noalloc(xd.data_ptr(), 0) == 0.0
    host = np.ones(10)
    for ptr, n in [(host.ctypes.data, 10), (xd.data_ptr(), 10_000_000), (xd.data_ptr(), -1)]:
        with pytest.raises(thor_b200.ThorxError) as e:
            thor_b200.device_sum_noalloc(ptr, n)
        assert e.value.code == thor_b200.E_ARG
    assert thor_b200.device_sum_noalloc(xd.data_ptr(), 1000) == 1000.0
