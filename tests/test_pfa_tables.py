"""CPU checks of the index arithmetic of the prime-factor alpha kernels
(s2dw_b200/csrc/s2dw_kernels.cu), without a GPU.

The Rader kernels (2047 = 23 * 89 and 511 = 7 * 73) carry constant tables:
for each position L = i + 8 j of the length-(p-1) convolution layout, the
index g^-q whose value goes there and the index g^q its result goes to.  The
test recomputes them from the primitive root and the layout's input digits,
then restates each kernel's steps in numpy (the row's Good-Thomas digits, the
short DFTs, the convolution through the 8 x (p-1)/8 transform, the product
with the DFT of w, the inverse) and compares the result with a plain DFT.  The
direct prime-factor kernels (1023, 255, 63, 31, 15, 7, 3) are checked the same
way from their factors and input digits.
"""
import os
import re

import numpy as np
import pytest

SRC = os.path.join(os.path.dirname(__file__), "..", "s2dw_b200", "csrc", "s2dw_kernels.cu")


def _table(name):
    text = open(SRC).read()
    m = re.search(r"__constant__ int " + name + r"\[(\d+)\] = \{([^}]*)\};", text)
    assert m, name
    vals = [int(x) for x in m.group(2).replace("\n", " ").split(",") if x.strip()]
    assert len(vals) == int(m.group(1))
    return vals


def _dft(x, sign):
    r = len(x)
    k = np.arange(r)
    return np.exp(sign * 2j * np.pi * np.outer(k, k) / r) @ x


def _rader_tables(p, g, b):
    """src/dst for a prime p with primitive root g; convolution length
    p-1 = 8 b, layout L = i + 8 j, input digits (q u1) mod 8, (q u2) mod b."""
    m = p - 1
    u1, u2 = pow(b, -1, 8), pow(8, -1, b)
    src, dst = [0] * m, [0] * m
    for q in range(m):
        L = (q * u1) % 8 + 8 * ((q * u2) % b)
        src[L] = pow(g, -q, p)
        dst[L] = pow(g, q, p)
    return src, dst


def _rader_kernel(z, R1, p, P, g, b, src, dst, sign):
    """The steps of pfa2047_alpha_kernel / pfa511_alpha_kernel on one row."""
    n = R1 * p
    u1, u2 = pow(p, -1, R1), pow(R1, -1, p)
    X = np.zeros(P * p, complex)
    for mm in range(n):
        X[(mm * u1) % R1 + P * ((mm * u2) % p)] = z[mm]
    for d2 in range(p):
        X[P * d2:P * d2 + R1] = _dft(X[P * d2:P * d2 + R1], sign)
    m = p - 1
    w = np.array([np.exp(sign * 2j * np.pi * pow(g, j, p) / p) for j in range(m)])
    W = np.zeros(m, complex)
    for k in range(m):
        W[k % 8 + 8 * (k % b)] = (np.exp(-2j * np.pi * np.arange(m) * k / m) @ w) / m
    for c1 in range(R1):
        col = np.array([X[c1 + P * d2] for d2 in range(p)])
        S = np.zeros((8, b), complex)
        for j in range(b):
            S[:, j] = _dft(np.array([col[src[i + 8 * j]] for i in range(8)]), -1)
        x0 = col[0]
        for i in range(8):
            v = _dft(S[i, :], -1)
            if i == 0:
                y0 = x0 + v[0]
            S[i, :] = _dft(v * np.array([W[i + 8 * kk] for kk in range(b)]), +1)
        out = np.zeros(p, complex)
        out[0] = y0
        for j in range(b):
            v = _dft(S[:, j], +1)
            for i in range(8):
                out[dst[i + 8 * j]] = x0 + v[i]
        for d2 in range(p):
            X[c1 + P * d2] = out[d2]
    return np.array([X[k % R1 + P * (k % p)] for k in range(n)])


@pytest.mark.parametrize("name,R1,p,P,g,b", [("c_rader", 23, 89, 25, 3, 11), ("c_rader73", 7, 73, 9, 5, 9)])
def test_rader_tables_and_steps(name, R1, p, P, g, b):
    src, dst = _rader_tables(p, g, b)
    assert _table(name + "_src") == src and _table(name + "_dst") == dst
    rng = np.random.default_rng(p)
    z = rng.standard_normal(R1 * p) + 1j * rng.standard_normal(R1 * p)
    for sign, ref in ((+1, np.fft.ifft(z) * len(z)), (-1, np.fft.fft(z))):
        y = _rader_kernel(z, R1, p, P, g, b, src, dst, sign)
        assert np.abs(y - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("factors", [(3, 11, 31), (3, 5, 17), (7, 9, 1), (31, 1, 1), (3, 5, 1), (7, 1, 1),
                                     (3, 1, 1), (5, 7, 9, 13)])
def test_direct_prime_factor_steps(factors):
    n = int(np.prod(factors))
    u = [pow((n // r) % r, -1, r) if r > 1 else 1 for r in factors]
    strides = [int(np.prod(factors[:i])) for i in range(len(factors))]
    rng = np.random.default_rng(n)
    z = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    for sign, ref in ((+1, np.fft.ifft(z) * n), (-1, np.fft.fft(z))):
        X = np.zeros(n, complex)
        for m in range(n):
            X[sum(((m * ui) % r) * s for ui, r, s in zip(u, factors, strides))] = z[m]
        for r, s in zip(factors, strides):
            if r == 1:
                continue
            for d in range(n // r):
                base = (d % s) + (d // s) * (s * r)
                idx = [base + k * s for k in range(r)]
                X[idx] = _dft(X[idx], sign)
        y = np.array([X[sum((k % r) * s for r, s in zip(factors, strides))] for k in range(n)])
        assert np.abs(y - ref).max() <= 1e-12 * np.abs(ref).max()


def test_kernel_input_digits_match_the_factors():
    """The input digit multipliers written in the kernels are the inverses
    (n / R_i)^-1 mod R_i that the steps above use."""
    text = open(SRC).read()
    assert "(m * 15) % 23 + PFB_P * ((m * 31) % 89)" in text
    assert (pow(89, -1, 23), pow(23, -1, 89)) == (15, 31)
    assert "(m * 5) % 7 + PFD_P * ((m * 21) % 73)" in text
    assert (pow(73, -1, 7), pow(7, -1, 73)) == (5, 21)
    assert "(n * 2) % 3 + 3 * ((n * 9) % 11) + 33 * ((n * 16) % 31)" in text
    assert (pow(341 % 3, -1, 3), pow(93 % 11, -1, 11), pow(33 % 31, -1, 31)) == (2, 9, 16)
    assert "(n * 4) % 5 + 5 * ((n * 2) % 7) + 35 * ((n * 2) % 9) + 315 * ((n * 9) % 13)" in text
