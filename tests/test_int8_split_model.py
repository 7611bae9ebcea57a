"""The numerical model of the int8 FP64 engine (csrc/oz.cu), restated on the
CPU: eight int8 digits per value under a per-row power-of-two scale, the
slice pairs with s + t < 8 summed exactly per diagonal, combined in FP64.

These checks pin the model the kernels implement and the bounds their
comments and tests state: digit range, the 32-bit accumulator bound of a K
range, and the worst-case error bound that tests/test_gpu_int8_contractions.py
applies to the GPU overlap. No GPU.
"""
import numpy as np

SLICES = 8


def digits(x, e):
    """Digits d_s of x 2^-e (|x| < 2^e): v <- 128 v, d = trunc(v), v <- v - d."""
    v = x * 2.0 ** (-e)
    out = []
    for _ in range(SLICES):
        t = np.trunc(v * 128.0)
        v = v * 128.0 - t
        out.append(t.astype(np.int64))
    return out, v


def scale_exp(m):
    e = np.frexp(m)[1]
    return np.where(m > 0, e, 0)


def product(A, B):
    """A (M x K) times B^T (N x K) by the split: per-row scales of A and of B."""
    eA = scale_exp(np.max(np.abs(A), axis=1))
    eB = scale_exp(np.max(np.abs(B), axis=1))
    dA, _ = digits(A, eA[:, None])
    dB, _ = digits(B, eB[:, None])
    out = np.zeros((A.shape[0], B.shape[0]))
    worst = 0
    for d in range(SLICES):
        acc = sum(dA[s] @ dB[d - s].T for s in range(d + 1))
        worst = max(worst, int(np.max(np.abs(acc))))
        out += acc * 2.0 ** (-7 * d)
    return out * 2.0 ** (eA[:, None] + eB[None, :] - 14), eA, eB, worst


def test_digits_are_int8_and_exact_to_the_remainder():
    rng = np.random.default_rng(1)
    x = rng.standard_normal((50, 300)) * np.exp(rng.uniform(-30, 30, (50, 1)))
    e = scale_exp(np.max(np.abs(x), axis=1))[:, None]
    d, rem = digits(x, e)
    assert all(np.max(np.abs(di)) <= 127 for di in d)
    back = sum(di * 2.0 ** (-7 * (s + 1)) for s, di in enumerate(d)) * 2.0 ** e
    # the remainder after eight digits is below 2^-56 of the row scale, and
    # digits plus remainder give x back exactly
    assert np.all(np.abs(rem) < 1.0)
    assert np.array_equal(back + rem * 2.0 ** (e - 56), x)


def test_accumulator_bounds():
    # a diagonal holds at most 8 slice pairs of at most 127^2 each
    assert 8 * 127 ** 2 * 16384 < 2 ** 31       # the overlap's chunk: 8192 grid points x (re, im)
    assert 8 * 127 ** 2 * 2 * 8299 < 2 ** 31    # the rotation's K = 2k for k < 8300
    assert 8 * 127 ** 2 * 2 * 8400 > 2 ** 31    # ... and not much beyond


def test_product_error_within_the_stated_bound():
    rng = np.random.default_rng(7)
    M, N, K = 40, 24, 2048
    env = np.exp(-np.linspace(-3, 3, K) ** 2)
    A = rng.standard_normal((M, K)) * env
    B = rng.standard_normal((N, K)) * env
    C, eA, eB, worst = product(A, B)
    assert worst < 2 ** 31
    ref = A @ B.T
    bound = 10.0 * 2.0 ** -56 * K * 2.0 ** (eA[:, None] + eB[None, :]).astype(float)
    diff = np.abs(C - ref)
    assert np.all(diff <= bound)
    # and in practice far below it: about the FP64 rounding of the sum
    assert np.max(diff) / np.max(np.abs(ref)) < 1e-14


def test_complex_layouts_of_the_overlap_and_rotation():
    """The interleaved real layouts give the complex products: the overlap's
    X = (re, im), Y = (im, -re) rows, and the rotation's (re, -im), (im, re)
    rows per grid point."""
    rng = np.random.default_rng(3)
    k, G = 12, 64
    psi = rng.standard_normal((k, G)) + 1j * rng.standard_normal((k, G))
    A = np.empty((k, 2 * G))
    A[:, 0::2], A[:, 1::2] = psi.real, psi.imag
    Y = np.empty((k, 2 * G))
    Y[:, 0::2], Y[:, 1::2] = psi.imag, -psi.real
    S = product(A, A)[0] + 1j * product(A, Y)[0]
    assert np.max(np.abs(S - psi.conj() @ psi.T)) < 1e-13
    W = rng.standard_normal((k, k)) + 1j * rng.standard_normal((k, k))
    Aw = np.empty((k, 2 * k))
    Aw[:, 0::2], Aw[:, 1::2] = W.T.real, W.T.imag          # A[n][(i, c)] = W[i][n].c
    Bre = np.empty((G, 2 * k))
    Bre[:, 0::2], Bre[:, 1::2] = psi.T.real, -psi.T.imag
    Bim = np.empty((G, 2 * k))
    Bim[:, 0::2], Bim[:, 1::2] = psi.T.imag, psi.T.real
    # per grid point scales shared by the two rows: take them from both
    m = np.maximum(np.max(np.abs(Bre), axis=1), np.max(np.abs(Bim), axis=1))
    assert np.array_equal(m, np.max(np.abs(Bre), axis=1))   # the same values, permuted and negated
    out = product(Aw, Bre)[0] + 1j * product(Aw, Bim)[0]
    assert np.max(np.abs(out - W.T @ psi)) < 1e-12
