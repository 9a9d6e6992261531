"""The allocation-free CRT entry point agrees with the allocating one.

dr_crt_batch_device_noalloc serves callers that cannot call cudaMalloc (for
example code whose device memory is owned by a framework's allocator): its
tables live in a static device array instead of library allocations.  Here
the test (not the entry point) allocates the input and output buffers with
torch, then checks two calls in a row -- different K, so the shared array is
rebuilt between them -- against dr_crt_batch_device, bit for bit.  The file
sorts last so a run that stops at the first failure has run everything else.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call_both(N, torch, K, n, seed):
    rng = np.random.default_rng(seed)
    primes = N.prime_table(K).astype(np.int64)
    res = np.stack([rng.integers(0, p, size=n) for p in primes], axis=1).astype(np.uint32)
    res[0, :] = 0
    res[1, :] = [p - 1 for p in primes]
    stride = (31 * K + 31) // 32 + 2
    dev = torch.device("cuda")
    r_d = torch.from_numpy(res.view(np.int32)).to(dev)
    out = {}
    for name in ("alloc", "noalloc"):
        limbs = torch.zeros((n, stride), dtype=torch.int32, device=dev)
        signs = torch.zeros(n, dtype=torch.int32, device=dev)
        if name == "alloc":
            nl = torch.zeros(n, dtype=torch.int32, device=dev)
            rc = N.lib().dr_crt_batch_device(r_d.data_ptr(), K, n, None, limbs.data_ptr(), stride,
                                             signs.data_ptr(), nl.data_ptr(), None)
        else:
            rc = N.lib().dr_crt_batch_device_noalloc(r_d.data_ptr(), K, n, limbs.data_ptr(), stride,
                                                     signs.data_ptr(), None)
        N.check(rc, name)
        torch.cuda.synchronize()
        out[name] = (limbs.cpu().numpy(), signs.cpu().numpy())
    return out


def test_noalloc_crt_matches_allocating_entry_point():
    torch = pytest.importorskip("torch")
    from dreams_rns import _native as N
    N.init()
    first = _call_both(N, torch, 100, 300, seed=1)
    second = _call_both(N, torch, 32, 1000, seed=2)
    for got in (first, second):
        assert np.array_equal(got["alloc"][0], got["noalloc"][0])
        assert np.array_equal(got["alloc"][1], got["noalloc"][1])
        assert (got["noalloc"][1] != 0).any()


def test_noalloc_rejects_oversized_K():
    from dreams_rns import _native as N
    rc = N.lib().dr_crt_batch_device_noalloc(None, 129, 1, None, 200, None, None)
    assert rc == N.DR_ERR_UNSUPPORTED
