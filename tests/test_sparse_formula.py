"""The sparse-mask temporal kernels' algebra (temporal_sparse_kernel,
temporal_sparse_big_kernel), restated in FP64 numpy and checked on the CPU
against the oracle's masked Wiener-Khinchin pass (analyzeFull,
motility-ddm/src/ddm_ref.js:229-288, 450-463):

  A(tau) + B(tau) = S(T - tau) + S(T) - S(tau) - sum_{d in Z} (p(d - tau) + p(d + tau))
      with p = m |x|^2 (0 outside [0, T)), S its prefix sums, Z the masked indices;
  G_a, G_b from ONE inverse transform W = n IFFT(|Y_a|^2 + i |Y_b|^2):
      G_a = (W(tau) + conj W(-tau)) / 2n,  G_b = (W(tau) - conj W(-tau)) / 2in
      (the kernels' gx, gy expressions);
  D = (A + B - 2 Re G) / N(tau), C = G / N(tau), 0 where N(tau) = 0.
"""
import numpy as np
import pytest

import oracle as O


def _sparse_pair(xa, xb, mask, L, TPAD):
    T = mask.size
    m = (mask != 0).astype(np.float64)
    xa, xb = xa * m, xb * m
    Z = np.nonzero(m == 0)[0]
    Ya, Yb = np.fft.fft(xa, TPAD), np.fft.fft(xb, TPAD)
    W = np.fft.ifft(np.abs(Ya) ** 2 + 1j * np.abs(Yb) ** 2) * TPAD  # unnormalised inverse
    tau = np.arange(L)
    w0, w1 = W[tau], W[(TPAD - tau) % TPAD]
    inv2n = 0.5 / TPAD
    G = [((w0.real + w1.real) + 1j * (w0.imag - w1.imag)) * inv2n,  # mode a
         ((w0.imag + w1.imag) + 1j * (w1.real - w0.real)) * inv2n]  # mode b
    npairs = np.array([np.sum(m[:T - t] * m[t:]) for t in tau])
    inv = np.where(npairs > 0.5, 1.0 / np.maximum(npairs, 1), 0.0)
    out = []
    for s, x in enumerate((xa, xb)):
        p = np.abs(x) ** 2
        S = np.concatenate([[0.0], np.cumsum(p)])
        pad = np.concatenate([np.zeros(L), p, np.zeros(L)])  # p read as 0 outside [0, T)
        corr = np.array([sum(pad[L + d - t] + pad[L + d + t] for d in Z) for t in tau])
        E = S[T - tau] + S[T] - S[tau] - corr
        D = (E - 2 * G[s].real) * inv
        C = G[s] * inv
        out.append((D, C))
    return out


@pytest.mark.parametrize("case", ["few", "ends", "run", "none", "all_but_two"])
def test_sparse_formula_matches_oracle(case):
    T, L = 96, 40
    TPAD = 256
    rng = np.random.default_rng(21)
    hist = rng.standard_normal((2, T)) + 1j * rng.standard_normal((2, T))
    mask = np.ones(T)
    if case == "few":
        mask[rng.choice(T, 7, replace=False)] = 0
    elif case == "ends":
        mask[[0, 1, T - 2, T - 1]] = 0
    elif case == "run":
        mask[20:45] = 0
    elif case == "all_but_two":
        mask[:] = 0
        mask[[3, 60]] = 1
    order = np.arange(T, dtype=np.uint32)
    D, C, P = O.analyze_modes(hist, order, mask, L, np.array([0, 1], np.int32), TPAD=TPAD)
    got = _sparse_pair(hist[0], hist[1], mask, L, TPAD)
    for s in range(2):
        sc = 2 * P[s]  # D's natural scale (harness.ts:147)
        assert sc > 0
        assert np.abs(got[s][0] - D[s]).max() <= 1e-10 * sc, (case, s)
        assert np.abs(got[s][1] - C[s]).max() <= 1e-10 * sc, (case, s)


def test_head_tail_prefix_sums():
    """temporal_sparse_big_kernel keeps only S(n) for n <= L (head) and
    n >= T - L (tail): S(T) - S(tau) + S(T - tau) for every tau < L reads
    only those."""
    T, L = 4000, 128
    p = np.random.default_rng(1).random(T)
    S = np.concatenate([[0.0], np.cumsum(p)])
    head = S[:L + 1]
    tail = S[T - L:]
    tau = np.arange(L)
    full = S[T] - S[tau] + S[T - tau]
    kept = tail[L] - head[tau] + tail[L - tau]
    assert np.array_equal(full, kept)
