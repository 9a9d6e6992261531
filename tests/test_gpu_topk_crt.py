"""GPU CRT and top-k at sizes where their fast paths decide.

CRT (reference runner.py:57-81): the lane-per-value kernel (standard prime
table, K <= 256) and the warp-per-value kernel (larger K, custom moduli)
against the oracle's crt_reconstruct/centered, bit for bit, including raw
residues at or above their modulus (the reference reduces a_i mod p_i for
i >= 1 and starts from the raw a_0).

Top-k by delta: highest first, NaN last, ties by lower index; the threshold
filter (from 2^18 values) must give exactly the full sort's answer,
including on inputs that defeat its threshold (ties, NaNs) and fall back.
"""

import ctypes

import numpy as np
import pytest

import dreams_rns as dr
from dreams_rns import _native as N
from oracle.walk_np import centered, crt

pytestmark = pytest.mark.gpu


def _residues(rng, K, n, raw=False):
    pr = [int(p) for p in N.prime_table(K)]
    res = np.stack([rng.integers(0, p, size=n) for p in pr], axis=1).astype(np.uint64)
    res[0, :] = 0
    res[1, :] = [p - 1 for p in pr]
    res[2, :] = res[2, 0]
    if raw and n > 6:
        res[3:6, :] = rng.integers(0, 1 << 32, size=(3, K), dtype=np.uint64)
    return res.astype(np.uint32), pr


@pytest.mark.parametrize("K", [1, 2, 7, 31, 32, 33, 64, 100, 128, 200, 256, 300])
def test_crt_batch_both_kernels_vs_oracle(K):
    rng = np.random.default_rng(K)
    res, pr = _residues(rng, K, 70, raw=True)
    got = dr.crt_batch(res, K)
    for i in range(res.shape[0]):
        x, M = crt([int(v) for v in res[i]], pr)
        assert got[i] == centered(x, M), (K, i)
    # unsigned values too (the reference's x itself)
    cen, uns = dr.crt_batch(res[:8], K, unsigned=True)
    for i in range(8):
        assert uns[i] == crt([int(v) for v in res[i]], pr)[0]


def test_crt_custom_moduli_take_the_general_kernel():
    rng = np.random.default_rng(9)
    mods = [2147483647, 1000000007, 998244353, 12345679, 3, 65537, 2147483629, 999999937]
    res = np.stack([rng.integers(0, m, size=50) for m in mods], axis=1).astype(np.uint32)
    got = dr.crt_batch(res, len(mods), mods)
    for i in range(res.shape[0]):
        x, M = crt([int(v) for v in res[i]], mods)
        assert got[i] == centered(x, M)


def test_crt_device_large_batch_spot_checks():
    torch = pytest.importorskip("torch")
    K, n = 32, 1 << 18
    rng = np.random.default_rng(5)
    res, pr = _residues(rng, K, n)
    stride = (31 * K + 31) // 32 + 2
    dev = torch.device("cuda")
    r_d = torch.from_numpy(res.view(np.int32)).to(dev)
    limbs = torch.zeros((n, stride), dtype=torch.int32, device=dev)
    sign = torch.zeros(n, dtype=torch.int32, device=dev)
    nl = torch.zeros(n, dtype=torch.int32, device=dev)
    N.check(N.lib().dr_crt_batch_device(r_d.data_ptr(), K, n, None, limbs.data_ptr(), stride,
                                        sign.data_ptr(), nl.data_ptr(), None), "crt device")
    torch.cuda.synchronize()
    L = limbs.cpu().numpy().view(np.uint32)
    S = sign.cpu().numpy()
    NL = nl.cpu().numpy()
    for i in list(range(0, n, 4099)) + [n - 1]:
        x, M = crt([int(v) for v in res[i]], pr)
        want = centered(x, M)
        mag = int.from_bytes(L[i].tobytes(), "little")
        assert (-mag if S[i] < 0 else mag) == want, i
        assert NL[i] == (abs(want).bit_length() + 31) // 32


def _ref_topk(d, k):
    key = np.where(np.isnan(d), -np.inf, d)
    nan = np.isnan(d)
    order = np.lexsort((np.arange(len(d)), -key, nan))   # NaN last, then -value, then index
    return order[:k]


@pytest.mark.parametrize("case", ["normal", "ties", "nan_inf", "small"])
def test_topk_filter_matches_full_order(case):
    rng = np.random.default_rng(hash(case) % 1000)
    n = (1 << 20) + 123 if case != "small" else 5000
    if case == "normal":
        d = rng.normal(-1.0, 0.01, size=n)
    elif case == "ties":
        d = np.round(rng.normal(0, 1, size=n), 1)          # heavy ties: falls back or filters exactly
        d[:300000] = 5.0                                   # more ties than any k at the top
    elif case == "nan_inf":
        d = rng.normal(0, 1, size=n)
        d[rng.integers(0, n, size=5000)] = np.nan
        d[rng.integers(0, n, size=50)] = np.inf
        d[rng.integers(0, n, size=50)] = -np.inf
    else:
        d = rng.normal(0, 1, size=n)
    for k in (1, 100, 256, 2048):
        idx = np.zeros(k, dtype=np.int32)
        val = np.zeros(k, dtype=np.float64)
        N.check(N.lib().dr_topk(N.ptr(d), n, k, N.ptr(idx), N.ptr(val)), "dr_topk")
        want = _ref_topk(d, k)
        assert list(idx) == list(want), (case, k)
        assert np.array_equal(val, d[want], equal_nan=True)


def test_topk_device_reports_the_filter():
    torch = pytest.importorskip("torch")
    n, k = 1 << 22, 256
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    d = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    idx = torch.zeros(k, dtype=torch.int32, device="cuda")
    val = torch.zeros(k, dtype=torch.float64, device="cuda")
    flag = ctypes.c_int32(-1)
    N.check(N.lib().dr_topk_device(d.data_ptr(), n, k, idx.data_ptr(), val.data_ptr(), None,
                                   ctypes.byref(flag)), "dr_topk_device")
    assert flag.value == 1
    h = d.cpu().numpy()
    want = _ref_topk(h, k)
    assert list(idx.cpu().numpy()) == list(want)
    assert np.array_equal(val.cpu().numpy(), h[want])


@pytest.mark.parametrize("n", [1, 7, 100, 4096, 8192])
def test_topk_small_inputs_with_ties(n):
    """Small inputs (the tile sort): the order of a full sort -- value
    descending, NaN last, ties by lower index, -0.0 equal to +0.0 -- with heavy
    ties, NaNs and infinities, and k above n."""
    rng = np.random.default_rng(n)
    d = np.round(rng.normal(0, 1, size=n), 1)          # many ties
    d[rng.integers(0, n, size=max(1, n // 50))] = np.nan
    d[rng.integers(0, n, size=max(1, n // 200))] = np.inf
    d[rng.integers(0, n, size=max(1, n // 200))] = -np.inf
    if n > 100:
        d[: n // 4] = 0.5                              # a block of equal values near the top
    for k in (1, 5, 100, 2048):
        keep = min(k, n)
        idx = np.zeros(keep, dtype=np.int32)
        val = np.zeros(keep, dtype=np.float64)
        N.check(N.lib().dr_topk(N.ptr(d), n, k, N.ptr(idx), N.ptr(val)), "dr_topk")
        want = _ref_topk(d, keep)
        assert list(idx) == list(want), (n, k)
        assert np.array_equal(val, d[want], equal_nan=True)
