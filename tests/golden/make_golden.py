"""Generates the golden fixtures under tests/golden/.

  python tests/golden/make_golden.py

dl_known.npz    d^l_{m'm}(pi/2) known answers computed in 50-digit arithmetic
                by mpmath: the Wigner sum formula for l <= 12 (all entries)
                and the three-term l recurrence, started from the closed-form
                edge value sqrt(C(2 l0, l0+k))/2^l0, for sampled pairs up to
                l = 2047.  These pin the oracle's Turok-Bucher planes and the
                library's recurrence tables independently of both.
oracle_*.npz    outputs of the CPU restatement of the reference (oracle/) at
                small sizes: a regression pin for the oracle and a parity
                target for the CUDA library.

The reference itself (Fortran + FFTW) cannot be compiled on this machine and
publishes no vectors, so no fixture here comes from running it.
"""
import os
import sys

import mpmath as mp
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

mp.mp.dps = 50


def wigner_sum(l, a, b):
    """d^l_{ab}(pi/2) by the Wigner sum formula (first index a)."""
    c = s = mp.sqrt(mp.mpf(1) / 2)
    tot = mp.mpf(0)
    for k in range(max(0, b - a), min(l + b, l - a) + 1):
        num = mp.sqrt(mp.factorial(l + a) * mp.factorial(l - a) * mp.factorial(l + b) * mp.factorial(l - b))
        den = mp.factorial(l + b - k) * mp.factorial(k) * mp.factorial(a - b + k) * mp.factorial(l - a - k)
        tot += (-1) ** (a - b + k) * num / den * c ** (2 * l + b - a - 2 * k) * s ** (a - b + 2 * k)
    return tot


def lwalk_mp(a, b, lmax):
    """{l: d^l_{ab}(pi/2)} for l in [max(a,b), lmax] (a, b >= 0) by the
    three-term recurrence in l at beta = pi/2."""
    l0, k = max(a, b), min(a, b)
    e = mp.sqrt(mp.binomial(2 * l0, l0 + k)) / mp.mpf(2) ** l0
    if a >= b and (l0 - b) % 2:
        e = -e
    out = {l0: e}
    dp, d = mp.mpf(0), e
    for l in range(l0, lmax):
        if l == 0:
            dn = mp.mpf(0)
        else:
            R = lambda ll, x: mp.sqrt(mp.mpf(ll * ll - x * x))
            u = mp.mpf(2 * l + 1) * a * b / (l * R(l + 1, a) * R(l + 1, b))
            v = mp.mpf(l + 1) * R(l, a) * R(l, b) / (l * R(l + 1, a) * R(l + 1, b))
            dn = -u * d - v * dp
        dp, d = d, dn
        out[l + 1] = d
    return out


def make_dl():
    rows = []
    for l in range(0, 13):
        for a in range(-l, l + 1):
            for b in range(-l, l + 1):
                rows.append((l, a, b, float(wigner_sum(l, a, b))))
    rng = np.random.default_rng(1234)
    pairs = [(0, 0), (3, 700), (500, 501), (1000, 20), (900, 1000), (1023, 1023), (1500, 100),
             (1200, 1300), (2047, 5), (7, 2047)]
    pairs += [tuple(int(x) for x in rng.integers(0, 1024, 2)) for _ in range(6)]
    for a, b in pairs:
        vals = lwalk_mp(a, b, 2047)
        for l in sorted(set([max(a, b), max(a, b) + 1, 1023, 2047] + list(rng.integers(max(a, b), 2048, 4)))):
            if l in vals:
                rows.append((int(l), a, b, float(vals[l])))
    arr = np.array(rows, dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, "dl_known.npz"), l=arr[:, 0].astype(np.int64),
                        a=arr[:, 1].astype(np.int64), b=arr[:, 2].astype(np.int64), d=arr[:, 3])
    print("dl_known.npz:", len(rows), "values")


def make_oracle(B, N, alpha, seed):
    from oracle import oracle as O

    from s2dw_b200.workload import gaussian_flm

    J = O.comp_jmax(B, alpha)
    K, P, bs = O.init_kernels(J, B, alpha)
    S = O.init_directionality(B, N)
    flm = gaussian_flm(B, seed=seed)
    wav, sc = O.analysis_dynamic(flm, K, S, J, B, N, bs, alpha)
    f2 = O.synthesis_dynamic(wav, sc, K, P, S, J, B, N, bs, alpha)
    name = f"oracle_B{B}_N{N}_a{alpha:g}.npz"
    d = {"B": B, "N": N, "alpha": alpha, "J": J, "seed": seed, "K_gamma": K, "Phi2": P, "bl_scoeff": bs,
         "Slm": S, "flm": flm, "scoeff": sc, "flm_syn": f2}
    for j, w in enumerate(wav):
        d[f"wav{j}"] = w
    np.savez_compressed(os.path.join(HERE, name), **d)
    print(name, "recon", np.abs(f2 - flm).max())


if __name__ == "__main__":
    make_dl()
    make_oracle(16, 3, 2.0, 11)
    make_oracle(32, 4, 2.0, 12)
    make_oracle(27, 2, 3.0, 13)
