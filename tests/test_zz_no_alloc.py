"""rg_filter_roundtrip_noalloc against rg_debug_filter_roundtrip, through the C ABI.

The allocation-free entry point works in a static device array instead of context
buffers; its output must match the context path within the round trip's tolerance
(relative L2 <= 1e-6: the only difference is how the twiddle table is rounded), on two
calls in a row, and a call must not change the device's free memory.
"""

import ctypes as C

import numpy as np
import pytest

import rg_b200 as rg
import workloads as wl
from helpers import rel_l2

pytestmark = pytest.mark.gpu


def _noalloc(p, d_in, d_out, R, ftype, stream=None):
    err = C.create_string_buffer(256)
    rc = rg.load().rg_filter_roundtrip_noalloc(C.byref(p), d_in.data_ptr(), d_out.data_ptr(), R, ftype, stream,
                                                err, len(err))
    return rc, err.value.decode()


@pytest.mark.parametrize("n,box", [(8, 10.0), (16, 20.0), (24, 30.0), (32, 40.0), (48, 48.0), (64, 80.0)])
@pytest.mark.parametrize("ftype", [-1, 0, 1, 2])
def test_noalloc_matches_context_path_twice(n, box, ftype):
    import torch
    rng = np.random.default_rng(1000 + n + ftype)
    x = wl.to_padded(rng.standard_normal((n, n, n)).astype(np.float32))
    d_in = torch.from_numpy(x.ravel()).cuda()
    want_d = torch.zeros_like(d_in)
    p = rg.make_params(n, box)
    R = box / 6.1
    ctx = rg.Context(n)
    ctx.call("rg_debug_filter_roundtrip", C.byref(p), d_in.data_ptr(), want_d.data_ptr(), R, ftype)
    ctx.close()
    want = wl.from_padded(want_d.cpu().numpy().reshape(n, n, -1))
    outs = []
    for _ in range(2):
        d_out = torch.full_like(d_in, float("nan"))
        rc, msg = _noalloc(p, d_in, d_out, R, ftype)
        assert rc == rg.RG_OK, msg
        torch.cuda.synchronize()
        got = wl.from_padded(d_out.cpu().numpy().reshape(n, n, -1))
        assert np.all(np.isfinite(got))
        assert rel_l2(got, want) <= 1e-6
        outs.append(got)
    assert np.array_equal(outs[0], outs[1])


def test_noalloc_allocates_nothing_and_rejects_large_grids():
    import torch
    n, box = 64, 64.0
    p = rg.make_params(n, box)
    d_in = torch.ones(n * n * 2 * (n // 2 + 1), device="cuda")
    d_out = torch.zeros_like(d_in)
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    assert _noalloc(p, d_in, d_out, 5.0, 0, stream.cuda_stream)[0] == rg.RG_OK   # first call: set-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert _noalloc(p, d_in, d_out, 5.0, 1, stream.cuda_stream)[0] == rg.RG_OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    # a uniform field survives any filter unchanged (only k = 0 carries power)
    assert torch.allclose(d_out, torch.ones_like(d_out).masked_fill(_pad_mask(n), 0.0), atol=1e-6)
    big = rg.make_params(96, 96.0)
    d_big = torch.zeros(96 * 96 * 98, device="cuda")
    rc, msg = _noalloc(big, d_big, d_big, 5.0, 0)
    assert rc == rg.RG_EUNSUPPORTED and "RG_NOALLOC_MAX_GRID_DIM" in msg and "64" in msg
    rc, msg = _noalloc(p, d_in, d_out, 5.0, 3)
    assert rc == rg.RG_EINVAL and msg
    # errbuf may be NULL: the status alone reports the rejection
    rc = rg.load().rg_filter_roundtrip_noalloc(C.byref(big), d_big.data_ptr(), d_big.data_ptr(), 5.0, 0, None,
                                                None, 0)
    assert rc == rg.RG_EUNSUPPORTED


def _pad_mask(n):
    import torch
    m = torch.zeros((n, n, 2 * (n // 2 + 1)), dtype=torch.bool)
    m[:, :, n:] = True
    return m.ravel().cuda()
