"""Host check of the pass structure of the register-resident longitude filter
(``k_dealias_reg`` in ``zhenmode_b200/csrc/zm_fft.cu``), restated in NumPy with
the kernel's own indexing: for n = N1 N2 N3 the forward transform is
decimation in frequency over n = n1 N2 N3 + n2 N3 + n3 (passes A, B, C with
their twiddles and shared-memory layouts), the 2/3 mask and conjugation act on
X[k1 + N1 k2 + N1 N2 k3], and the second forward transform runs over
k = k3 N1 N2 + k2 N1 + k1 (passes C', B', A'), its output landing at
m = p3 + N3 p2 + N3 N2 p1.  The filtered line must equal
ifft(fft(x) * mask) for every split the kernel is built for.  The CUDA kernel
itself is checked against the float64 oracle on the GPU
(``tests/test_gpu_parity.py``, widths 180, 360, 720, 800).
"""
import numpy as np
import pytest

# (n, N1, N2, N3) of the kernel's split table (fft_reg_split)
SPLITS = [(720, 8, 9, 10), (800, 8, 10, 10), (360, 4, 9, 10), (180, 4, 9, 5)]


def _w(e, n):
    return np.exp(-2j * np.pi * (np.asarray(e) % n) / n)


def _filter(x, keep, n1, n2, n3):
    n = n1 * n2 * n3
    n12, n23 = n1 * n2, n2 * n3
    ex = np.zeros(n, complex)
    # A: DFT_N1 over n1 for column t = n2 N3 + n3, twiddle W_n^(k1 t)
    for t in range(n23):
        v = np.fft.fft(x[t + n23 * np.arange(n1)]) * _w(np.arange(n1) * t, n)
        ex[np.arange(n1) * n23 + t] = v
    # B: DFT_N2 over n2 for (k1, n3), twiddle W_n^(N1 k2 n3)
    nxt = np.empty_like(ex)
    for t in range(n1 * n3):
        k1, n3i = t // n3, t % n3
        idx = k1 * n23 + np.arange(n2) * n3 + n3i
        nxt[idx] = np.fft.fft(ex[idx]) * _w(np.arange(n2) * (n1 * n3i), n)
    ex = nxt
    # C, mask and conjugation, C': for (k1, k2) with kp = k1 + N1 k2
    nxt = np.empty_like(ex)
    for t in range(n12):
        k1, k2 = t % n1, t // n1
        v = np.fft.fft(ex[k1 * n23 + k2 * n3 + np.arange(n3)])
        kk = t + n12 * np.arange(n3)
        v = np.where(keep[kk], np.conj(v), 0)
        v = np.fft.fft(v) * _w(np.arange(n3) * t, n)
        nxt[np.arange(n3) * n12 + t] = v
    ex = nxt
    # B': DFT_N2 over k2 for (k1, p3), twiddle W_n^(N3 k1 p2)
    nxt = np.empty_like(ex)
    for t in range(n1 * n3):
        k1, p3 = t % n1, t // n1
        idx = p3 * n12 + np.arange(n2) * n1 + k1
        nxt[idx] = np.fft.fft(ex[idx]) * _w(np.arange(n2) * (n3 * k1), n)
    ex = nxt
    # A': DFT_N1 over k1 for (p3, p2), output m = t + N2 N3 p1
    out = np.empty(n, complex)
    for t in range(n23):
        p3, p2 = t % n3, t // n3
        out[t + n23 * np.arange(n1)] = np.fft.fft(ex[p3 * n12 + p2 * n1 + np.arange(n1)])
    return np.conj(out) / n


@pytest.mark.parametrize("n,n1,n2,n3", SPLITS)
def test_register_split_filters_like_the_fft(n, n1, n2, n3):
    assert n1 * n2 * n3 == n
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    # the reference's 2/3-rule mask (factory.py:529-533)
    keep = np.abs(np.fft.fftfreq(n) * n) <= int(n // 2 * 2.0 / 3.0)
    want = np.fft.ifft(np.fft.fft(x) * keep)
    got = _filter(x, keep, n1, n2, n3)
    assert np.abs(got - want).max() < 1e-12 * np.abs(want).max()
