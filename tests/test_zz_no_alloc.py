"""The allocation-free CRT entry point agrees with the allocating one.

dr_crt_batch_device_noalloc serves callers that cannot call cudaMalloc (for
example code whose device memory is owned by a framework's allocator): its
tables live in a static device array instead of library allocations.  Here
the test (not the entry point) allocates the input and output buffers with
torch, then checks calls in a row -- different K, so the shared array is
rebuilt between them, up to K = 128 where its tables reach the array's last
word -- against dr_crt_batch_device bit for bit, and the centred values
against the CRT oracle.  The file sorts last so a run that stops at the
first failure has run everything else.
"""

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
        out[name] = (limbs.cpu().numpy().view(np.uint32), signs.cpu().numpy())
    out["residues"] = res
    out["primes"] = [int(p) for p in primes]
    return out


def _value(limbs_row, sign):
    mag = int.from_bytes(np.ascontiguousarray(limbs_row, dtype=np.uint32).tobytes(), "little")
    return -mag if sign < 0 else mag


def test_noalloc_crt_matches_allocating_entry_point():
    torch = pytest.importorskip("torch")
    from dreams_rns import _native as N
    from oracle.walk_np import centered, crt
    N.init()
    runs = [_call_both(N, torch, 100, 300, seed=1), _call_both(N, torch, 32, 1000, seed=2),
            _call_both(N, torch, 128, 257, seed=3), _call_both(N, torch, 1, 64, seed=4)]
    for got in runs:
        assert np.array_equal(got["alloc"][0], got["noalloc"][0])
        assert np.array_equal(got["alloc"][1], got["noalloc"][1])
        assert (got["noalloc"][1] != 0).any()
        limbs, signs = got["noalloc"]
        for i in range(0, len(signs), max(1, len(signs) // 16)):
            x, M = crt([int(v) for v in got["residues"][i]], got["primes"])
            assert _value(limbs[i], int(signs[i])) == centered(x, M)
    # one prime: the centred residue itself
    p = runs[3]["primes"][0]
    limbs, signs = runs[3]["noalloc"]
    for i, r in enumerate(runs[3]["residues"][:, 0]):
        r = int(r)
        assert _value(limbs[i], int(signs[i])) == (r - p if r > p // 2 else r)


def test_noalloc_rejects_oversized_K():
    from dreams_rns import _native as N
    rc = N.lib().dr_crt_batch_device_noalloc(None, 129, 1, None, 200, None, None)
    assert rc == N.DR_ERR_UNSUPPORTED
