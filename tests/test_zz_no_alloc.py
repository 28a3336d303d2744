"""The allocation-free sort, gcs_sort_pairs_static, called through the C ABI.

It exists for callers that cannot allocate device memory where they sort
(a real-time loop or host callback that must not trigger an allocation's
implicit synchronisation, or a plug-in whose host application owns the
device memory budget); its working state lives in one static device array.
Checked here against the engine's own sort stage on the same Morton keys,
on two calls in a row (each call must clear what the previous one left in
the shared array); at exactly the array's limit (1,048,576 pairs, every
look-back slot in use) against the oracle's stable sort, with and without a
caller status word; plus the rejection of sizes beyond the limit.
Collected last so that a stop-at-first-failure run has run everything else.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import small_collision

pytestmark = pytest.mark.gpu

STATIC_SORT_MAX = 1 << 20


def _engine_sort(gcs, stars):
    p = gcs.reference_params(bounds_mode=gcs.BOUNDS_DEVICE, theta=0.5, epsilon_sq=4e-4)
    with gcs.Context(len(stars)) as ctx:
        ctx.upload(stars)
        ctx.run_stages(p, gcs.STAGE_BOUNDS, gcs.STAGE_ENCODE)
        unsorted = ctx.read(gcs.BUF_KEYS_UNSORTED)
        ctx.run_stages(p, gcs.STAGE_SORT, gcs.STAGE_SORT)
        return unsorted, ctx.read(gcs.BUF_KEYS), ctx.read(gcs.BUF_INDEX)


def test_static_sort_matches_engine_sort_on_two_calls(gcs_mod):
    import torch

    gcs = gcs_mod
    L = gcs.lib()
    stars = small_collision(60000, 15000, 7000, seed=21)  # 164,000 pairs: 41 tiles
    n = len(stars)
    unsorted, ref_keys, ref_idx = _engine_sort(gcs, stars)
    assert not np.array_equal(unsorted, ref_keys)  # the input really needs sorting
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    for _ in range(2):
        keys = torch.from_numpy(unsorted.view(np.int64).copy()).to(dev)
        vals = torch.arange(n, dtype=torch.int32, device=dev)
        keys_alt = torch.empty_like(keys)
        vals_alt = torch.empty_like(vals)
        rc = L.gcs_sort_pairs_static(C.c_void_p(keys.data_ptr()), C.c_void_p(vals.data_ptr()),
                                     C.c_void_p(keys_alt.data_ptr()), C.c_void_p(vals_alt.data_ptr()), n,
                                     C.c_void_p(status.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert rc == 0, gcs.lib().gcs_status_string(rc)
        torch.cuda.synchronize(dev)
        np.testing.assert_array_equal(keys.cpu().numpy().view(np.uint64), ref_keys)
        np.testing.assert_array_equal(vals.cpu().numpy().view(np.uint32), ref_idx)
        assert int(status.item()) == 0


def _static_sort(L, torch, keys_np, with_status):
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    n = len(keys_np)
    keys = torch.from_numpy(keys_np.view(np.int64).copy()).to(dev)
    vals = torch.arange(n, dtype=torch.int32, device=dev)
    keys_alt = torch.empty_like(keys)
    vals_alt = torch.empty_like(vals)
    status = torch.zeros(1, dtype=torch.int32, device=dev) if with_status else None
    rc = L.gcs_sort_pairs_static(C.c_void_p(keys.data_ptr()), C.c_void_p(vals.data_ptr()),
                                 C.c_void_p(keys_alt.data_ptr()), C.c_void_p(vals_alt.data_ptr()), n,
                                 C.c_void_p(status.data_ptr()) if with_status else None,
                                 C.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize(dev)
    st = int(status.item()) if with_status else 0
    return rc, st, keys.cpu().numpy().view(np.uint64), vals.cpu().numpy().view(np.uint32)


def test_static_sort_at_its_limit_matches_oracle(gcs_mod, oracle_mod):
    import torch

    L = gcs_mod.lib()
    rng = np.random.default_rng(5)
    n = STATIC_SORT_MAX
    # 63-bit Morton keys of a 1,048,576-particle collision, and a second set
    # with heavy duplication (4,096 distinct keys) so the position tie-break
    # decides most of the order
    stars = gcs_mod.collision_equal(384000, 96000, 44288, seed=3)
    pos, _ = gcs_mod.pos_vel_from_stars(stars)
    lo, hi = oracle_mod.bounds(pos)
    morton = oracle_mod.encode(pos, lo, hi)
    dup = (rng.integers(0, 4096, n, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)) >> np.uint64(1)
    for keys_np, with_status in ((morton, True), (dup, False)):
        assert len(keys_np) == n
        ref_k, ref_i = oracle_mod.sort(keys_np)
        rc, st, k, v = _static_sort(L, torch, keys_np, with_status)
        assert rc == 0, L.gcs_status_string(rc)
        assert st == 0
        np.testing.assert_array_equal(k, ref_k)
        np.testing.assert_array_equal(v, ref_i)


def test_static_sort_rejects_sizes_beyond_its_array(gcs_mod):
    L = gcs_mod.lib()
    p = C.c_void_p(16)  # never dereferenced: the size check comes first
    assert L.gcs_sort_pairs_static(p, p, p, p, STATIC_SORT_MAX + 1, None, None) == -4  # GCS_ERR_CAPACITY
    assert L.gcs_sort_pairs_static(None, None, None, None, 0, None, None) == 0
    assert L.gcs_sort_pairs_static(None, None, None, None, 5, None, None) == -1  # GCS_ERR_ARG
