"""CPU: why the precision form's bars can tell 3xTF32 from plain TF32.

One 5-qubit block is a complex 32x32 matrix applied to 128 rows of a tile, i.e.
the real product X' W' (X' 128 x 64, W' 64 x 64).  TF32 keeps 10 explicit
mantissa bits (round to nearest, ties away, as the kernel rounds).  Emulated here in
numpy with exact products and FP64 sums (the tensor cores' products are exact;
their sums are FP32): plain TF32 operands leave a relative error near 2^-11,
far above the 1e-5 block bar of tests/test_gpu_tc.py, while the 3xTF32 split
(hi*hi + hi*lo + lo*hi, hi = tf32(x), lo = tf32(x - hi)) stays near 2^-21."""
import numpy as np


def tf32(x: np.ndarray) -> np.ndarray:
    """Round float32 values to TF32 (10 mantissa bits), nearest, ties away."""
    b = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x1000) & 0xFFFFE000  # add half an ulp of bit 13, clear the low 13 bits
    return b.astype(np.uint32).view(np.float32)


def block_real(rng):
    q, r = np.linalg.qr(rng.normal(size=(32, 32)) + 1j * rng.normal(size=(32, 32)))
    u = q * (np.diag(r) / np.abs(np.diag(r)))
    W = np.zeros((64, 64))
    W[0::2, 0::2] = u.real.T
    W[1::2, 0::2] = -u.imag.T
    W[0::2, 1::2] = u.imag.T
    W[1::2, 1::2] = u.real.T
    return W


def test_plain_tf32_fails_and_3xtf32_passes_the_block_bar():
    rng = np.random.default_rng(0)
    W = block_real(rng).astype(np.float32)
    X = (rng.normal(size=(128, 64)) * 2 ** -6).astype(np.float32)
    exact = X.astype(np.float64) @ W.astype(np.float64)
    scale = np.abs(exact).max()
    plain = tf32(X).astype(np.float64) @ tf32(W).astype(np.float64)
    xh, wh = tf32(X), tf32(W)
    xl, wl = tf32(X - xh), tf32(W - wh)
    split = (xh.astype(np.float64) @ wh.astype(np.float64) +
             xh.astype(np.float64) @ wl.astype(np.float64) +
             xl.astype(np.float64) @ wh.astype(np.float64))
    e_plain = np.abs(plain - exact).max() / scale
    e_split = np.abs(split - exact).max() / scale
    assert e_plain > 1e-4          # fails the 1e-5 bar by an order of magnitude
    assert e_split < 1e-6          # passes it with room for FP32 sums
    assert tf32(np.float32(1.0 + 2 ** -11)) == np.float32(1.0 + 2 ** -10)  # tie rounds away
