"""The split-BF16 arithmetic of the tensor-core y pass, emulated on the CPU.

rg_dft_y_pass's tcgen05 form (csrc/rg_dft_tc.cu) computes a 256-point line as 16 x 16: two
radix-16 stages, each a real matrix product of the 16 complex inputs (as 32 reals) with the 32 x 32
real form of the DFT-16 matrix, both operands split into BF16 hi + lo and the three products
Ahi Bhi + Alo Bhi + Ahi Blo accumulated in FP32, with the w256 twiddles applied in FP32 between
the stages.  This test does the same arithmetic in numpy (round-to-nearest-even BF16 by bit
manipulation) and checks the error model stated for it: about 4e-6 relative L2 per pass against
FP64 (the GPU measures 4.4e-6), inside the 1e-5 gate and well above the FP32 transform's 1e-7, and
that the two-part operands (about 16 significant bits), not the dropped Alo Blo term, set it."""

import numpy as np


def bf16(x):
    """Round float32 values to BF16 (nearest, ties to even), returned as float32."""
    b = np.ascontiguousarray(x, np.float32).view(np.uint32)
    r = ((b >> 16) & 1) + 0x7FFF
    return ((b + r) & 0xFFFF0000).view(np.float32)


def dft16_real(sign):
    """The 32 x 32 real form of the DFT-16 matrix: rows (k, re/im), columns (n, re/im)."""
    m = np.zeros((32, 32))
    for k in range(16):
        for n in range(16):
            c, s = np.cos(2 * np.pi * n * k / 16), sign * np.sin(2 * np.pi * n * k / 16)
            m[2 * k, 2 * n], m[2 * k, 2 * n + 1] = c, -s
            m[2 * k + 1, 2 * n], m[2 * k + 1, 2 * n + 1] = s, c
    return m


def split_product(a, b, terms=3):
    """FP32 accumulation of the hi/lo BF16 products of a (rows x 32) and b^T (b: 32 x 32)."""
    a32 = a.astype(np.float32)
    b32 = b.astype(np.float32)
    ah = bf16(a32)
    al = bf16(a32 - ah)
    bh = bf16(b32)
    bl = bf16(b32 - bh)
    d = ah @ bh.T + al @ bh.T + ah @ bl.T
    if terms == 4:
        d = d + al @ bl.T
    return d.astype(np.float32)


def as_reals(z):
    r = np.empty(z.shape[:-1] + (2 * z.shape[-1],), np.float32)
    r[..., 0::2], r[..., 1::2] = z.real, z.imag
    return r


def as_complex(r):
    return r[..., 0::2].astype(np.float64) + 1j * r[..., 1::2]


def tc_pass(x, sign=-1, terms=3):
    """One 256-point transform of each row of x by the tensor-core form's arithmetic."""
    lines = x.shape[0]
    b = dft16_real(sign)
    n1n2 = x.reshape(lines, 16, 16)                     # [line][n1][n2], n = 16 n1 + n2
    a = as_reals(np.transpose(n1n2, (0, 2, 1)))         # rows (line, n2), K = n1
    y = as_complex(split_product(a.reshape(-1, 32), b, terms)).reshape(lines, 16, 16)   # [line][n2][k1]
    n2 = np.arange(16)[:, None]
    k1 = np.arange(16)[None, :]
    w = np.exp(sign * 2j * np.pi * n2 * k1 / 256).astype(np.complex64)
    y = (y.astype(np.complex64) * w).astype(np.complex64)
    a2 = as_reals(np.transpose(y, (0, 2, 1)))           # rows (line, k1), K = n2
    out = as_complex(split_product(a2.reshape(-1, 32), b, terms)).reshape(lines, 16, 16)   # [line][k1][k2]
    return np.transpose(out, (0, 2, 1)).reshape(lines, 256)     # X[k1 + 16 k2]


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_split_bf16_pass_error_model():
    rng = np.random.default_rng(3)
    x = (rng.standard_normal((512, 256)) + 1j * rng.standard_normal((512, 256))).astype(np.complex64)
    want = np.fft.fft(x.astype(np.complex128), axis=1)
    e3 = rel_l2(tc_pass(x, terms=3), want)
    e4 = rel_l2(tc_pass(x, terms=4), want)
    e32 = rel_l2(np.fft.fft(x, axis=1).astype(np.complex64), want)
    assert 1e-6 < e3 < 1e-5, e3          # the GPU form measures 4.4e-6
    assert 0.7 * e3 < e4 < e3             # a fourth product (Alo Blo) buys little: the splits set it
    assert e32 < 1e-6


def test_split_bf16_inverse_pass_matches_fp64():
    rng = np.random.default_rng(4)
    x = (rng.standard_normal((128, 256)) + 1j * rng.standard_normal((128, 256))).astype(np.complex64)
    want = np.fft.ifft(x.astype(np.complex128), axis=1) * 256
    assert rel_l2(tc_pass(x, sign=+1), want) < 1e-5


def test_split_bf16_errors_accumulate_over_passes():
    """A forward and inverse 2-D transform (four passes) by this arithmetic returns the input to
    about 9e-6: a 3-D forward and inverse (six passes, every filtered field of the step) would be
    above the 1e-5 gates."""
    rng = np.random.default_rng(5)
    x = (rng.standard_normal((256, 256)) + 1j * rng.standard_normal((256, 256))).astype(np.complex64)
    y = tc_pass(x)
    y = tc_pass(y.T.astype(np.complex64)).T
    z = tc_pass(y.T.astype(np.complex64), sign=+1).T
    z = tc_pass(z.astype(np.complex64), sign=+1)
    e = rel_l2(z / 256 ** 2, x.astype(np.complex128))
    assert 6e-6 < e < 1.2e-5, e
    assert e * np.sqrt(6 / 4) > 1e-5
