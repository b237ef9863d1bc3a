"""Generates tests/golden/oracle_B2048_N8_samples.npz: oracle outputs at the
large configuration B=2048, N=8, alpha=2, J=Jmax=11, for the GPU parity test
of the full-band scales (tests/test_gpu_headline_parity.py).

  python tests/golden/make_b2048_fixture.py [threads] [--add-accurate]

The oracle (oracle/, the CPU restatement of the reference loops) runs
unsampled on every scale; it takes tens of minutes on 8 cores.  The full
outputs (2.5 GB of wavelet coefficients) are too large to commit, so the
fixture keeps:

analysis of flm = gaussian_flm(2048, seed=0, power=1.2) (C_l = (1/(l(l+1)))^1.2):
  for every scale j, the rows w_j(:, b, g) at the (b, g) pairs ROWS_J (a
  fixed, seeded choice that always includes the edges b = 0, 2bl-1 and
  g = 0, N-1), and max|w_j| over the whole scale;
synthesis of seeded random coefficients (scale by scale, in scale order,
  rng = numpy default_rng(SYN_SEED), rng.standard_normal((2bl-1)*2bl*N) read
  in the dynamic layout, a fastest; then scoeff with real and imaginary
  parts from the same stream):
  the rows flm(l, 0:l) for l in SYN_ROWS, and max|flm| over all (l, m).

Tables come from the oracle's init_kernels / init_directionality.

Each output is stored twice: from the oracle as it restates the reference
(keys ana_rows_j, ana_max_j, syn_row_l, syn_max), and from the oracle with its
d(pi/2) planes replaced by the accurate long-double planes of
oracle.dl_plane_accurate (keys with the suffix _acc).  At l ~ 2000 the
reference's Turok-Bucher planes carry up to 1.4e-13 absolute error (measured
against 50-digit values), so the second set separates that error from any
other difference.  --add-accurate computes only the second set and adds it to
an existing fixture.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

B, N, ALPHA, POWER, SYN_SEED = 2048, 8, 2.0, 1.2, 2048
SYN_ROWS = [2, 3, 31, 64, 255, 256, 511, 512, 700, 1023, 1024, 1300, 1500, 1800, 2000, 2046, 2047]
OUT = os.path.join(HERE, "oracle_B2048_N8_samples.npz")


def rows_for_scale(j, bl, n_rows=4):
    """(b, g) pairs kept for scale j: the four corners plus seeded interior
    picks."""
    rng = np.random.default_rng(1000 + j)
    pairs = [(0, 0), (2 * bl - 1, N - 1)]
    while len(pairs) < n_rows:
        p = (int(rng.integers(0, 2 * bl)), int(rng.integers(0, N)))
        if p not in pairs:
            pairs.append(p)
    return pairs


def synthesis_inputs(J, bls, bs):
    """The seeded random wavelet and scaling coefficients of the synthesis
    case (the GPU test regenerates them the same way)."""
    rng = np.random.default_rng(SYN_SEED)
    wav = []
    for bl in bls:
        n = (2 * bl - 1) * 2 * bl * N
        wav.append(np.asfortranarray(rng.standard_normal(n).reshape((2 * bl - 1, 2 * bl, N), order="F")))
    sc = rng.standard_normal((bs, bs)) + 1j * rng.standard_normal((bs, bs))
    return wav, np.asfortranarray(sc)


def run(O, K, P, S, J, bls, bs, suffix, out):
    from s2dw_b200.workload import gaussian_flm

    flm = gaussian_flm(B, seed=0, power=POWER)
    t0 = time.time()
    for j in range(J + 1):
        w = O.analysis_scale(j, flm, K, S, J, B, N, ALPHA)
        pairs = rows_for_scale(j, bls[j])
        out[f"ana_pairs_{j}"] = np.array(pairs)
        out[f"ana_rows_{j}{suffix}"] = np.stack([w[:, b, g] for b, g in pairs])
        out[f"ana_max_{j}{suffix}"] = np.abs(w).max()
        print(f"analysis{suffix} scale {j} (bl={bls[j]}): {time.time() - t0:.0f} s", flush=True)
        del w
    wav, sc = synthesis_inputs(J, bls, bs)
    f = O.synthesis_dynamic(wav, sc, K, P, S, J, B, N, bs, ALPHA)
    print(f"synthesis{suffix}: {time.time() - t0:.0f} s", flush=True)
    for l in SYN_ROWS:
        out[f"syn_row_{l}{suffix}"] = f[l, :l + 1].copy()
    out[f"syn_max{suffix}"] = np.abs(f).max()


def main():
    from oracle import oracle as O

    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    threads = int(args[0]) if args else (os.cpu_count() or 1)
    O.set_num_threads(threads)
    J = O.comp_jmax(B, ALPHA)
    K, P, bs = O.init_kernels(J, B, ALPHA)
    S = O.init_directionality(B, N)
    bls = [O.band_limits(j, B, ALPHA)[0] for j in range(J + 1)]
    if "--add-accurate" in sys.argv:
        out = dict(np.load(OUT))
    else:
        out = {"B": B, "N": N, "alpha": ALPHA, "J": J, "power": POWER, "syn_seed": SYN_SEED,
               "syn_rows": np.array(SYN_ROWS), "bl": np.array(bls)}
        O.set_dl_method(0)
        run(O, K, P, S, J, bls, bs, "", out)
    O.set_dl_method(1)
    run(O, K, P, S, J, bls, bs, "_acc", out)
    O.set_dl_method(0)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
