"""CPU checks of the folded correlation's arithmetic (corr_fold_kernel<N> in
prestozl_b200/csrc/jerk_kernels.cu), in float64 numpy.

1. The fold identity: for a prepared chunk D of length N that repeats with
   period N/2 (the transform of data spread to even interbins) and a kernel
   row K, the inverse transform of D conj(K) splits by output parity into two
   N/2-point transforms of D A and D B, with A and B built from K alone.
2. The kernel's index flow for the half-length transform, [8, 16, R2] on
   T = N/16 threads: stage 0's butterflies with stage 1's input twiddles
   applied at stage 0's writes, stage 1 (radix 16, Ns = 8) one transform per
   thread, stage 2 (radix R2, Ns = 128) on 128 butterflies; the padded
   shared-memory addresses stay inside one plane and every slot is written
   once per stage.

The GPU parity tests compare the kernel's volumes with the oracle; these
pin the design itself for both folded lengths (2048 and 1280).
"""
import numpy as np
import pytest

FOLDED = [2048, 1280]


def _pad(i):
    return i + (i >> 4)


def _w(n, m):
    return np.exp(2j * np.pi * np.asarray(m) / n)


def _dft_inv(x):
    n = len(x)
    k = np.arange(n)
    return np.array([np.sum(x * _w(n, k * m)) for m in range(n)])


@pytest.mark.parametrize("N", FOLDED)
def test_fold_identity(N):
    rng = np.random.default_rng(N)
    H = N // 2
    # data at even interbins: its transform repeats with period N/2
    x = np.zeros(N, complex)
    x[0::2] = rng.normal(size=H) + 1j * rng.normal(size=H)
    D = np.fft.fft(x)
    assert np.allclose(D[:H], D[H:])
    K = rng.normal(size=N) + 1j * rng.normal(size=N)
    y = np.fft.ifft(D * np.conj(K)) * N
    k = np.arange(H)
    A = np.conj(K[:H]) + np.conj(K[H:])
    B = (np.conj(K[:H]) - np.conj(K[H:])) * np.exp(2j * np.pi * k / N)
    ye = np.fft.ifft(D[:H] * A) * H
    yo = np.fft.ifft(D[:H] * B) * H
    scale = np.max(np.abs(y))
    assert np.max(np.abs(y[0::2] - ye)) < 1e-12 * scale
    assert np.max(np.abs(y[1::2] - yo)) < 1e-12 * scale


@pytest.mark.parametrize("N", FOLDED)
def test_half_length_index_flow(N):
    H = N // 2
    R2 = H // 128
    T = H // 8
    NB1 = T // 2
    plane = H + H // 16
    rng = np.random.default_rng(7 + N)
    Y = rng.normal(size=H) + 1j * rng.normal(size=H)  # the products D A (or D B)
    buf = np.full(plane, np.nan, complex)
    out = np.full(plane, np.nan, complex)
    # stage 0: butterfly t on inputs t + T r; stage 1's input twiddle for
    # element 8 t + r is W_128^((t / (T/16)) r)
    for t in range(T):
        v = _dft_inv(Y[t + T * np.arange(8)])
        for r in range(8):
            row = t // (T // 16)
            assert row * 8 + r < 128  # inside stage 0's table
            a = _pad(8 * t + r)
            assert a < plane and np.isnan(buf[a])
            buf[a] = v[r] * _w(128, row * r)
    # stage 1: butterfly j of one transform, inputs j + NB1 r, outputs at
    # (j / 8) 128 + j % 8 + 8 r
    for j in range(NB1):
        x = np.array([buf[_pad(j + r * NB1)] for r in range(16)])
        assert not np.isnan(x).any()
        y = _dft_inv(x)
        for r in range(16):
            a = _pad((j >> 3) * 128 + (j & 7) + 8 * r)
            assert a < plane and np.isnan(out[a])
            out[a] = y[r]
    # stage 2: butterfly j < 128 on inputs j + 128 r, twiddles W_H^(r j)
    res = np.zeros(H, complex)
    for j in range(128):
        v = np.array([out[_pad(j + 128 * r)] for r in range(R2)])
        assert not np.isnan(v).any()
        y = _dft_inv(v * _w(H, np.arange(R2) * j))
        res[j + 128 * np.arange(R2)] = y
    ref = np.fft.ifft(Y) * H
    assert np.max(np.abs(res - ref)) < 1e-12 * np.max(np.abs(ref))
