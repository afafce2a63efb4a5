"""The split-BF16 tensor-core y pass (tcgen05) against the FP32 register y pass and FP64, through
the C ABI: rg_dft_y_pass on whole 256^3 Hermitian spectra, forward and inverse.

Gates (relative L2 against numpy's FP64 transform of the same input): the FP32 form 1e-6, the
tensor-core form 1e-5 (three BF16 products per stage, two radix-16 stages)."""

import numpy as np
import pytest

import rg_b200 as rg

pytestmark = pytest.mark.gpu

N = 256
NZ = N // 2 + 1


def spectra(ng, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((ng, NZ, N, N), dtype=np.float32) + 1j * rng.standard_normal((ng, NZ, N, N), dtype=np.float32)
    return a.astype(np.complex64)


def run(x, inverse, impl):
    import torch
    ctx = rg.Context(N)
    d = torch.from_numpy(x.copy()).cuda()
    ctx.call("rg_dft_y_pass", d.data_ptr(), x.shape[0], int(inverse), impl)
    out = d.cpu().numpy()
    ctx.close()
    return out


def want(x, inverse):
    x64 = x.astype(np.complex128)
    return np.fft.ifft(x64, axis=-1) * N if inverse else np.fft.fft(x64, axis=-1)


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.mark.parametrize("inverse", [0, 1])
def test_tensor_core_y_pass_matches_fp64(inverse):
    x = spectra(2, 11 + inverse)
    ref = want(x, inverse)
    e32 = rel_l2(run(x, inverse, rg.RG_DFT_FP32), ref)
    etc = rel_l2(run(x, inverse, rg.RG_DFT_TC_BF16X3), ref)
    assert e32 <= 1e-6, e32
    assert etc <= 1e-5, etc
    assert etc > e32   # the BF16 splits are coarser than FP32: the tensor-core path really ran


def test_tensor_core_y_pass_single_modes():
    # x[y] = exp(2 pi i m y / N) on every line: the forward transform is N at bin m, zero elsewhere
    y = np.arange(N)
    x = np.empty((1, NZ, N, N), np.complex64)
    ms = (np.arange(NZ)[:, None] * 7 + np.arange(N)[None, :] * 3) % N
    x[0] = np.exp(2j * np.pi * ms[:, :, None] * y[None, None, :] / N)
    got = run(x, 0, rg.RG_DFT_TC_BF16X3)
    peak = np.take_along_axis(got[0], ms[:, :, None], axis=-1)[..., 0]
    assert np.max(np.abs(peak - N)) <= 1e-5 * N * 4
    got[0][np.arange(NZ)[:, None], np.arange(N)[None, :], ms] = 0
    assert np.max(np.abs(got)) <= 1e-5 * N * 4


def test_tensor_core_y_pass_rejects_other_sizes():
    import torch
    ctx = rg.Context(128)
    d = torch.zeros(65 * 128 * 128, dtype=torch.complex64, device="cuda")
    with pytest.raises(rg.RGError) as e:
        ctx.call("rg_dft_y_pass", d.data_ptr(), 1, 0, rg.RG_DFT_TC_BF16X3)
    assert e.value.status == rg.RG_EUNSUPPORTED
    ctx.close()
