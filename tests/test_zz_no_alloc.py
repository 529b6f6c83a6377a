"""cuapss_feature_remap_noalloc (the allocation-free frequency remap) called
through the C ABI with CUDA buffers, checked against cuapss_feature_remap and
the CPU oracle's remap on the same inputs. Integer outputs, so the tolerance
is exact equality.

The file name sorts last so that the test also runs after every other test
in one process (the scratch array then holds earlier calls' leftovers)."""
import ctypes

import numpy as np
import pytest

import cuapss
from cuapss import synth
from oracle import oracle

pytestmark = pytest.mark.gpu

MAX_FEATURES = 65536  # the entry point's stated limit


def _noalloc():
    L = cuapss.lib()
    f = L.cuapss_feature_remap_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.POINTER(cuapss.CsrDesc), ctypes.c_void_p,
                  ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _device_csr(x, torch):
    return {"rowptr": torch.from_numpy(x.rowptr).cuda(), "col": torch.from_numpy(x.col).cuda(),
            "val": torch.from_numpy(x.val).cuda(), "d": x.d}


def _call(ctx, dx, perm, counts):
    desc, keep = cuapss._desc(dx)
    return _noalloc()(ctx._h, ctypes.byref(desc), perm.data_ptr(), counts.data_ptr())


@pytest.fixture(scope="module")
def torch_cuda():
    from tests.conftest import HAS_GPU
    if not HAS_GPU:
        pytest.skip("no CUDA device")
    import torch
    return torch


@pytest.mark.parametrize("cfg,n,d", [("plain_20k", 20_000, 10_000),
                                     ("plain_800k", 50_000, 50_000),
                                     ("plain_800k", 3_000, MAX_FEATURES)])
def test_noalloc_matches_remap_twice(torch_cuda, cfg, n, d):
    torch = torch_cuda
    x = synth.generate(cfg, n=n, d=d, seed=11)
    y = synth.generate(cfg, n=n // 2, d=d, seed=12)
    with cuapss.Context() as ctx:
        for inp in (x, y, x):  # three calls in a row, outputs start dirty
            want_perm, want_counts = ctx.feature_remap(inp)
            dx = _device_csr(inp, torch)
            perm = torch.full((inp.d,), -7, dtype=torch.int32, device="cuda")
            counts = torch.full((inp.d,), 123, dtype=torch.int32, device="cuda")
            s = _call(ctx, dx, perm, counts)
            assert s == cuapss.OK, cuapss.status_string(s)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(counts.cpu().numpy(), want_counts)
            np.testing.assert_array_equal(perm.cpu().numpy(), want_perm)
            # and directly against the oracle's remap
            o_perm, o_counts = oracle.feature_remap(inp)
            np.testing.assert_array_equal(counts.cpu().numpy(), o_counts)
            np.testing.assert_array_equal(perm.cpu().numpy(), o_perm)
            # a permutation of 0..d-1 ordered by (count desc, id asc)
            p = perm.cpu().numpy()
            order = np.argsort(p)
            c = want_counts[order]
            assert np.all(np.diff(c) <= 0)
            ties = np.diff(c) == 0
            assert np.all(np.diff(order)[ties] > 0)


def test_noalloc_rejects_beyond_limit_and_host_input(torch_cuda):
    torch = torch_cuda
    x = synth.generate("plain_20k", n=100, d=MAX_FEATURES + 1, seed=3)
    with cuapss.Context() as ctx:
        dx = _device_csr(x, torch)
        perm = torch.empty(x.d, dtype=torch.int32, device="cuda")
        counts = torch.empty(x.d, dtype=torch.int32, device="cuda")
        assert _call(ctx, dx, perm, counts) == cuapss.EINVAL
        # host arrays are refused (they would need a device staging copy)
        desc, keep = cuapss._desc(synth.generate("plain_20k", n=100, seed=3))
        assert _noalloc()(ctx._h, ctypes.byref(desc), perm.data_ptr(),
                          counts.data_ptr()) == cuapss.EINVAL
        # an unsorted row is refused, and a valid call afterwards still works
        bad = synth.generate("plain_20k", n=100, seed=4)
        r = int(np.argmax(np.diff(bad.rowptr) >= 2))
        lo = int(bad.rowptr[r])
        bad.col[lo], bad.col[lo + 1] = bad.col[lo + 1], bad.col[lo]
        small_perm = torch.empty(bad.d, dtype=torch.int32, device="cuda")
        small_counts = torch.empty(bad.d, dtype=torch.int32, device="cuda")
        assert _call(ctx, _device_csr(bad, torch), small_perm, small_counts) == cuapss.EINVAL
        good = synth.generate("plain_20k", n=100, seed=5)
        assert _call(ctx, _device_csr(good, torch), small_perm, small_counts) == cuapss.OK
        want_perm, _ = ctx.feature_remap(good)
        np.testing.assert_array_equal(small_perm.cpu().numpy(), want_perm)
