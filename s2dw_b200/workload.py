"""Seeded synthetic inputs with the shapes and statistics of the benchmark
workloads (no public dataset is involved).

gaussian_flm: harmonic coefficients of a real signal with angular power
spectrum C_l = (1/(l(l+1)))^power for l >= 2 and f_00 = f_1m = 0.  Only m >= 0
is stored (flm(l, m), l fastest, entries with m > l are zero), the layout of
the reference's flm(0:B-1, 0:B-1).  f_l0 ~ N(0, C_l) is real; for m > 0 the
real and imaginary parts are each N(0, C_l/2).  Draws come from numpy's
PCG64 Generator seeded with `seed`, in l-major order, then m, real part before
imaginary part, one standard-normal stream for the whole array.
"""
import numpy as np


def gaussian_flm(B, seed=0, power=1.0):
    rng = np.random.default_rng(seed)
    flm = np.zeros((B, B), dtype=np.complex128, order="F")
    if B <= 2:
        return flm
    ls = np.arange(2, B)
    counts = 2 * ls + 1  # re(l,0), then (re, im) for m = 1..l
    z = rng.standard_normal(int(counts.sum()))
    pos = 0
    for l in ls:
        cl = (1.0 / (l * (l + 1.0))) ** power
        s = np.sqrt(cl)
        h = np.sqrt(cl / 2.0)
        flm[l, 0] = z[pos] * s
        re = z[pos + 1:pos + 2 * l + 1:2]
        im = z[pos + 2:pos + 2 * l + 1:2]
        flm[l, 1:l + 1] = h * (re + 1j * im)
        pos += 2 * l + 1
    return flm


def transform_setup(B, N, alpha=2.0, J=None):
    """Kernel tables of the library for (B, N, alpha, J=Jmax by default):
    returns dict with J, K_gamma, Phi2, bl_scoeff, Slm."""
    from . import core

    if J is None:
        J = core.s2dw_core_comp_Jmax(B, alpha)
    K, P, bs = core.s2dw_core_init_kernels(J, B, alpha)
    S = core.s2dw_core_init_directionality(B, N)
    return {"B": B, "N": N, "alpha": alpha, "J": J, "K_gamma": K, "Phi2": P, "bl_scoeff": bs, "Slm": S}


def run_pairs(B, N, alpha=2.0, pairs=2, seed=0):
    """Runs `pairs` device analysis+synthesis pairs of one seeded map through a
    plan on cuda:0 and returns the reconstruction error max|f' - f|.  This is
    the small fixed workload that kernel profiles are captured on:
    python -m s2dw_b200.workload B N pairs."""
    import torch

    from .device import Plan

    t = transform_setup(B, N, alpha)
    plan = Plan(B, N, alpha, t["J"])
    plan.set_tables(t["K_gamma"], t["Phi2"], t["Slm"], t["bl_scoeff"])
    flm = gaussian_flm(B, seed=seed)
    d_flm = torch.from_numpy(np.ascontiguousarray(flm.T)).cuda()
    d_wav = torch.empty(plan.wav_size, dtype=torch.float64, device="cuda")
    d_sc = torch.empty(max(1, t["bl_scoeff"] ** 2), dtype=torch.complex128, device="cuda")
    d_out = torch.empty_like(d_flm)
    for _ in range(pairs):
        plan.analysis(d_flm, d_wav, d_sc)
        plan.synthesis(d_wav, d_sc, d_out)
    torch.cuda.synchronize()
    err = float(np.abs(d_out.cpu().numpy().T - flm).max())
    plan.close()
    return err


def run_batch(B, N, alpha=2.0, maps=32, form=1, repeats=1):
    """Runs `repeats` batched analyses of `maps` seeded maps through a plan of
    `form` (0 FP64, 1 split) on cuda:0, then one batched synthesis of the last
    batch through the same plan; returns the worst reconstruction error over
    the maps."""
    import torch

    from .device import Plan

    t = transform_setup(B, N, alpha)
    plan = Plan(B, N, alpha, t["J"], form=form)
    plan.set_tables(t["K_gamma"], t["Phi2"], t["Slm"], t["bl_scoeff"])
    flms = [gaussian_flm(B, seed=k) for k in range(maps)]
    d_flm = torch.from_numpy(np.stack([np.ascontiguousarray(f.T) for f in flms])).cuda()
    d_wav = torch.empty((maps, plan.wav_size), dtype=torch.float64, device="cuda")
    d_sc = torch.empty((maps, max(1, t["bl_scoeff"] ** 2)), dtype=torch.complex128, device="cuda")
    for _ in range(repeats):
        plan.analysis_batch(d_flm, d_wav, d_sc)
    plan.check()
    d_out = torch.empty_like(d_flm)
    plan.synthesis_batch(d_wav, d_sc, d_out)
    plan.check()
    torch.cuda.synchronize()
    err = max(float(np.abs(d_out[k].cpu().numpy().T - flms[k]).max()) for k in range(maps))
    plan.close()
    return err


if __name__ == "__main__":
    # python -m s2dw_b200.workload B N pairs            one-map FP64 pairs
    # python -m s2dw_b200.workload B N repeats maps     split-form batched analyses
    import sys

    a = [int(x) for x in sys.argv[1:5]] + [None] * 4
    B, N, P, M = a[0] or 1024, a[1] or 4, a[2] or 2, a[3]
    if M:
        print(f"B={B} N={N} maps={M} split analyses={P} + synthesis, recon {run_batch(B, N, 2.0, M, 1, P):.3e}")
    else:
        print(f"B={B} N={N} pairs={P} recon {run_pairs(B, N, 2.0, P):.3e}")
