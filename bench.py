"""Headline benchmark: S2DW analysis+synthesis pairs/s at B=1024, N=4, alpha=2,
J=Jmax on one B200 (one map per pair, FP64 plain form).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one analysis (flm -> wav) followed by one synthesis (wav -> flm) of
a seeded synthetic map, all inputs resident in HBM.  Prints one JSON line.
Under torchrun each rank runs an independent replica (the transform has no
cross-GPU exchange): scaling is weak, value = pairs of all ranks / max time.

`e2e` times the same pair through the C-ABI host-buffer entry points
(s2dwc_analysis_flm2wav_dynamic + s2dwc_synthesis_wav2flm_dynamic) with pinned
host buffers, so every step includes the host<->device copies.

`--impl reference` times the CPU restatement of the reference's algorithm
(oracle/, the reference's Fortran cannot be compiled here) on the host cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "B=1024 N=4 analysis+synthesis pairs/s at recon err<=1e-10"


def _hbm_gbs():
    """Measured HBM copy bandwidth of this pool's B200s (MEASURED_PEAKS.json,
    hbm_gbs), else the earlier measured fallback of 6650 GB/s."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except Exception:
        return 6650.0


HBM_GBS = _hbm_gbs()
UNIT = "pairs/s"

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per launch of each
# kernel kind, averaged over the 11 launches of each kind in one
# analysis+synthesis pair at B=1024 N=4 alpha=2 J=10, from the ncu launch list
# of `python -m s2dw_b200.workload 1024 4 1` (profiles/launches_B1024_N4.md).
# Used only for the roofline "traffic" entry of that workload.
NCU_TRAFFIC = {(1024, 4, 2.0): {"lwalk": 7.18e6, "mwalk": 10.89e6, "ana_beta": 27.22e6,
                                "ana_alpha": 44.23e6, "syn_alpha": 44.30e6, "syn_beta": 31.00e6}}
NCU_TRAFFIC_SOURCE = ("ncu --metrics gpu__time_duration.sum,dram__bytes_read.sum,dram__bytes_write.sum "
                      "--clock-control none of `python -m s2dw_b200.workload 1024 4 1` (one pair, 11 launches of "
                      "each kind), profiles/launches_B1024_N4.md")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 300; 10 for --impl reference, whose steps are CPU pairs)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--B", type=int, default=1024)
    ap.add_argument("--N", type=int, default=4)
    ap.add_argument("--alpha", type=float, default=2.0)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serving-requests", type=int, default=4096,
                    help="mixed request stream for the serving p50/p99 (0 = skip)")
    ap.add_argument("--no-graph", action="store_true", help="launch kernels directly instead of replaying a CUDA graph")
    ap.add_argument("--no-large", action="store_true", help="skip the B=2048 N=8 single-transform section")
    ap.add_argument("--serving-split-requests", type=int, default=1024,
                    help="requests of the stream served again by the split-precision server (0 = skip)")
    ap.add_argument("--large-split-maps", type=int, default=8,
                    help="maps per split-form batch in the B=2048 N=8 section (0: skip)")
    ap.add_argument("--no-b256", action="store_true", help="skip the B=256 N=5 split-vs-FP64 section")
    ap.add_argument("--split-maps", type=int, default=32,
                    help="maps per batch for the split-precision measurement (0: skip)")
    return ap.parse_args()


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
                power.append(float(r[3]))
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


def contraction_flops_per_scale(B, N, alpha, J):
    """Algorithmic FLOPs of the l-contractions per scale (analysis, synthesis):
    4 flops per complex-by-real MAC, (l+1)^2 (m, m') pairs per l, times the
    number of n with N+n odd (|n| <= min(N-1,l) for analysis, 0 <= n for
    synthesis)."""
    from s2dw_b200.core import band_limits

    ana, syn = [], []
    for j in range(J + 1):
        hi, lo = band_limits(j, B, alpha)
        fa = fs = 0.0
        for l in range(lo + 1, hi):
            k = min(N - 1, l)
            na = sum(1 for n in range(-k, k + 1) if (N + n) % 2)
            ns = sum(1 for n in range(0, k + 1) if (N + n) % 2)
            fa += 4.0 * (l + 1) ** 2 * na
            fs += 4.0 * (l + 1) ** 2 * ns
        ana.append(fa)
        syn.append(fs)
    return ana, syn


def pair_roofline(B, N, alpha, J, t_ms, fp64_peak_tflops):
    """Whole-pair roofline: t_min = max(F / P_FP64, Q / BW_HBM) with F the
    contraction flops of an analysis+synthesis pair (4 per complex-by-real MAC)
    and Q its compulsory HBM bytes (the wavelet array written then read, flm
    read then written: 2*8*samples + 2*16*B(B+1)/2); frac = t_min / t."""
    from s2dw_b200 import core

    ana_f, syn_f = contraction_flops_per_scale(B, N, alpha, J)
    F = sum(ana_f) + sum(syn_f)
    samples = sum(int(np.prod(core.wav_scale_shape(j, B, N, alpha))) for j in range(J + 1))
    Q = 2 * 8 * samples + 2 * 16 * B * (B + 1) / 2
    t_f = F / (fp64_peak_tflops * 1e12) * 1e3
    t_q = Q / (HBM_GBS * 1e9) * 1e3
    t_min = max(t_f, t_q)
    return {"flops": F, "bytes": Q, "t_flops_ms": t_f, "t_hbm_ms": t_q, "t_min_ms": t_min, "t_ms": t_ms,
            "frac": t_min / t_ms, "bound": "fp64" if t_f >= t_q else "hbm",
            "peaks": f"FP64 {fp64_peak_tflops:.1f} TFLOP/s (measured DGEMM), HBM {HBM_GBS:.0f} GB/s (measured copy)"}


def _serve(srv, reqs, rate=None):
    """Warm-up (the whole stream at once, untimed: every slot the stream
    needs is created and every graph captured, as in a server that has been
    running), then the whole stream at once (saturation throughput), then
    Poisson arrivals at `rate` (default 70% of the saturation throughput) for
    the latency percentiles."""
    for r in reqs:
        r.arrival = 0.0
    srv.run(reqs)
    cap = srv.run(reqs)["throughput_rps"]
    rate = 0.7 * cap if rate is None else rate
    rng = np.random.default_rng(7)
    t = 0.0
    for r in reqs:
        t += rng.exponential(1.0 / rate)
        r.arrival = t
    st = srv.run(reqs)
    st.update({"offered_rate_rps": rate, "saturation_rps": cap})
    return st


def serving_stats(n_requests, device, split_requests=1024):
    """The mixed serving stream: Poisson arrivals, B uniform over
    {32,...,1024}, N uniform over 1..8, alpha in {2,3}, J=Jmax, half analyses
    and half syntheses (inputs from analyses of seeded maps).  The arrival
    rate is 70% of the FP64 server's throughput with every request arriving
    at once, so that queues stay finite and the percentiles reflect overlap.
    The split-precision server then serves the first `split_requests`
    requests of the same stream at the same offered rate, batching the
    waiting requests of a configuration and kind (up to 1 GB of packed
    wavelets per batch); a subset, because the split form serves single maps
    far slower than FP64 and the whole stream would take minutes."""
    from s2dw_b200.serving import Server, make_stream

    reqs, inputs = make_stream(n_requests, seed=2026, rate_hz=1e9)
    srv = Server(hbm_budget_bytes=60 << 30, slots_per_config=2, use_graphs=True, device=device, priorities=True)
    st = _serve(srv, reqs)
    # the stream's device time with the requests run one at a time: the
    # saturation span against it is the overlap the server achieves
    serial = srv.device_time(reqs)
    srv.close()
    st["serial_device_s"] = serial
    st["overlap_vs_serial"] = serial * st["saturation_rps"] / len(reqs)
    st.update({"form": "fp64",
               "stream": f"{n_requests} requests, Poisson, B in 32..1024, N in 1..8, alpha in {{2,3}}, J=Jmax, "
                         "half analysis / half synthesis, device-resident inputs, graph replay, slot stream "
                         "priorities by B (smaller first)"})
    # the same stream and offered rate with every slot at the default priority (first come, first served)
    srv = Server(hbm_budget_bytes=60 << 30, slots_per_config=2, use_graphs=True, device=device, priorities=False)
    fifo = _serve(srv, reqs, rate=st["offered_rate_rps"])
    srv.close()
    st["fifo"] = {k: fifo[k] for k in ("p50_ms", "p99_ms", "mean_ms", "throughput_rps", "saturation_rps")}
    if split_requests > 0:
        try:
            sub = reqs[:split_requests]
            srv = Server(hbm_budget_bytes=80 << 30, slots_per_config=2, use_graphs=True, device=device,
                         form="auto", batch_bytes=12 << 30, split_min_batch=16, priorities=True)
            sp = _serve(srv, sub, rate=st["offered_rate_rps"])
            srv.close()
            sp["note"] = (f"form auto: split-precision slots (waiting requests of one configuration and kind as "
                          f"one tensor-core batch of up to 32 maps) where 16 or more of one configuration and kind "
                          f"wait, FP64 slots otherwise; the first {len(sub)} requests of the FP64 server's stream "
                          f"at its offered rate")
            st["split"] = sp
        except Exception as ex:  # reported, not fatal to the bench line
            st["split"] = {"error": str(ex)[:300]}
        try:
            st["burst"] = burst_stats(device)
        except Exception as ex:
            st["burst"] = {"error": str(ex)[:300]}
    del inputs
    return st


def burst_stats(device, n=512):
    """A burst of one configuration (B=1024, N=4, alpha=2, half analyses and
    half syntheses, all arriving at once), served by the FP64 server and by
    the split server (batches of up to 32 maps of one configuration and kind;
    under 16 maps in FP64): where the split form pays in serving."""
    from s2dw_b200.serving import Server, make_stream

    reqs, inputs = make_stream(n, seed=11, rate_hz=1e9, Bs=(1024,), Ns=(4,), alphas=(2.0,))
    out = {"stream": f"{n} requests of B=1024 N=4 alpha=2 J=10, half analysis / half synthesis, all at once"}
    for name, kw in (("fp64", {}), ("split", {"form": "auto", "batch_bytes": 12 << 30, "split_min_batch": 16})):
        srv = Server(hbm_budget_bytes=80 << 30, slots_per_config=2, use_graphs=True, device=device, **kw)
        for r in reqs:
            r.arrival = 0.0
        srv.run(reqs)  # warm-up: slots and graphs of every batch size met
        st = srv.run(reqs)
        srv.close()
        out[name] = {k: st[k] for k in ("throughput_rps", "p50_ms", "p99_ms", "mean_batch")}
    out["split_vs_fp64"] = out["split"]["throughput_rps"] / out["fp64"]["throughput_rps"]
    del inputs
    return out


def split_stats(B, N, alpha, J, maps, repeats=3, power=1.0):
    """Split-precision form on a batch of `maps` seeded maps (the form's
    tensor-core contractions share their d-operand across the batch): device
    time of batched analysis+synthesis pairs per map for the split plan and for
    the FP64 plan on the same batch, the serialised contraction times of each
    form, the split form's max|w_split - w_fp64| / max|w_fp64| per scale (worst
    map) and overall, its synthesis error max|flm_split - flm_fp64| /
    max|flm_fp64| on the same coefficients, and the split pair's
    reconstruction error (absolute and relative to max|flm|).  Errors are
    reduced on the device."""
    import torch

    from s2dw_b200.device import Plan
    from s2dw_b200.workload import gaussian_flm, transform_setup

    t = transform_setup(B, N, alpha, J)
    plain = Plan(B, N, alpha, J)
    split = Plan(B, N, alpha, J, form=Plan.SPLIT)
    for p in (plain, split):
        p.set_tables(t["K_gamma"], t["Phi2"], t["Slm"], t["bl_scoeff"])
    flms = [gaussian_flm(B, seed=k, power=power) for k in range(maps)]
    d_flm = torch.from_numpy(np.stack([np.ascontiguousarray(f.T) for f in flms])).cuda()
    del flms
    bs2 = max(1, t["bl_scoeff"] ** 2)
    w_ref = torch.empty((maps, plain.wav_size), dtype=torch.float64, device="cuda")
    w_sp = torch.empty_like(w_ref)
    s_ref = torch.empty((maps, bs2), dtype=torch.complex128, device="cuda")
    s_sp = torch.empty_like(s_ref)
    out = torch.empty_like(d_flm)
    out_ref = torch.empty_like(d_flm)
    plain.analysis_batch(d_flm, w_ref, s_ref)
    split.analysis_batch(d_flm, w_sp, s_sp)
    split.synthesis_batch(w_sp, s_sp, out)
    split.check()
    plain.synthesis_batch(w_sp, s_sp, out_ref)
    torch.cuda.synchronize()
    offs = plain.wav_offsets
    per_scale = []
    for j in range(J + 1):
        a_, b_ = w_ref[:, offs[j]:offs[j + 1]], w_sp[:, offs[j]:offs[j + 1]]
        sc = a_.abs().amax(dim=1)
        d = (a_ - b_).abs().amax(dim=1)
        r = torch.where(sc > 0, d / sc.clamp_min(1e-300), torch.zeros_like(d))
        per_scale.append(float(r.max()))
    werr = max(per_scale)
    fmax = d_flm.abs().amax(dim=(1, 2))
    dev = (out - d_flm).abs().amax(dim=(1, 2))
    recon = float(dev.max())
    recon_rel = float((dev / fmax).max())
    synerr = float(((out - out_ref).abs().amax(dim=(1, 2)) / out_ref.abs().amax(dim=(1, 2))).max())
    del w_ref, s_ref, out_ref
    torch.cuda.empty_cache()

    def timed(ana, syn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(repeats):
            ana.analysis_batch(d_flm, w_sp, s_sp)
            syn.synthesis_batch(w_sp, s_sp, out)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / repeats

    t_split = timed(split, split)
    t_fp64 = timed(plain, plain)
    contraction = {}
    for name, p in (("split", split), ("fp64", plain)):
        p.set_timing(True)
        p.timing(reset=True)
        p.analysis_batch(d_flm, w_sp, s_sp)
        p.synthesis_batch(w_sp, s_sp, out)
        torch.cuda.synchronize()
        kt = p.timing(reset=True)
        contraction[name] = {"analysis_ms_per_map": kt["lwalk"][1] / maps, "synthesis_ms_per_map": kt["mwalk"][1] / maps,
                             "serialised_pair_ms_per_map": sum(v[1] for v in kt.values()) / maps}
        p.set_timing(False)
    split.check()
    plain.close()
    split.close()
    return {"maps_per_batch": maps, "value": maps / t_split, "unit": "pairs/s",
            "fp64_same_batch": maps / t_fp64, "speedup_vs_fp64": t_fp64 / t_split,
            "kernels": contraction,
            "max_w_err": werr, "max_w_err_per_scale": per_scale, "max_flm_err_synthesis": synerr,
            "recon_err": recon, "recon_err_rel_max_flm": recon_rel,
            "form": "split analysis and synthesis contractions (tcgen05 int8 digits, 6 bytes, 26 exact products); FP64 recurrences, tables and FFTs",
            "workload": f"B={B} N={N} alpha={alpha:g} J={J}, {maps} seeded maps per batch"
                        + (f", C_l=(1/(l(l+1)))^{power:g}" if power != 1.0 else "") + ", device-resident"}


def large_stats(B=2048, N=8, alpha=2.0, power=1.2, steps=6, warmup=2):
    """The large single transform: B=2048, N=8, alpha=2, J=Jmax, one map with
    C_l = (1/(l(l+1)))^1.2, FP64 form: device time per analysis+synthesis
    pair (scales on the plan's streams), reconstruction error, and the
    serialised time of each kernel kind."""
    import torch

    from s2dw_b200.core import s2dw_core_comp_Jmax
    from s2dw_b200.device import Plan
    from s2dw_b200.workload import gaussian_flm, transform_setup

    J = s2dw_core_comp_Jmax(B, alpha)
    t = transform_setup(B, N, alpha, J)
    plan = Plan(B, N, alpha, J)
    plan.set_tables(t["K_gamma"], t["Phi2"], t["Slm"], t["bl_scoeff"])
    flm = gaussian_flm(B, seed=0, power=power)
    d_flm = torch.from_numpy(np.ascontiguousarray(flm.T)).cuda()
    d_wav = torch.empty(plan.wav_size, dtype=torch.float64, device="cuda")
    d_sc = torch.empty(max(1, t["bl_scoeff"] ** 2), dtype=torch.complex128, device="cuda")
    d_out = torch.empty_like(d_flm)
    for _ in range(warmup):
        plan.analysis(d_flm, d_wav, d_sc)
        plan.synthesis(d_wav, d_sc, d_out)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        plan.analysis(d_flm, d_wav, d_sc)
        plan.synthesis(d_wav, d_sc, d_out)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    recon = float(np.abs(d_out.cpu().numpy().T - flm).max() / np.abs(flm).max())
    plan.set_timing(True)
    plan.timing(reset=True)
    plan.analysis(d_flm, d_wav, d_sc)
    plan.synthesis(d_wav, d_sc, d_out)
    torch.cuda.synchronize()
    kt = plan.timing(reset=True)
    plan.close()
    return {"workload": f"B={B} N={N} alpha={alpha:g} J={J}, one map, C_l=(1/(l(l+1)))^{power}, FP64 form",
            "value": 1e3 / ms, "unit": "pairs/s", "ms_per_pair": ms, "recon_err_rel_max_flm": recon,
            "wav_bytes": 8 * plan.wav_size, "steps": steps,
            "kernels_ms": {k: v[1] for k, v in kt.items() if v[0]}}


def fft_flops_per_pair(B, N, alpha, J):
    """Algorithmic FLOPs of the transform stages per pair, counted as
    5 L log2 L per complex transform of the length L the stage needs:
    alpha stages: N*bl complex transforms of length 2bl-1 (two real rows
    each); beta stages: N*bl (analysis) or ceil(N/2)*bl (synthesis)
    transforms with 2bl outputs (L = 2bl)."""
    import math

    from s2dw_b200.core import band_limits

    npos = sum(1 for n in range(N) if (N + n) % 2)
    out = {"ana_alpha": 0.0, "syn_alpha": 0.0, "ana_beta": 0.0, "syn_beta": 0.0}
    for j in range(J + 1):
        bl, _ = band_limits(j, B, alpha)
        n = 2 * bl - 1
        fa = 5.0 * n * math.log2(max(n, 2))
        fb = 5.0 * (2 * bl) * math.log2(2 * bl)
        out["ana_alpha"] += N * bl * fa
        out["syn_alpha"] += N * bl * fa
        out["ana_beta"] += N * bl * fb
        out["syn_beta"] += npos * bl * fb
    return out


def measured_fp64_peak():
    """FP64 reference rate on this GPU: best of 10 torch.matmul float64 4096^3
    (cuBLAS DGEMM), TFLOP/s."""
    import torch

    n = 4096
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(3):
        torch.matmul(a, b)
    best = 1e30
    for _ in range(10):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


def _generator():
    """The seeded flm generator (s2dw_b200/workload.py, numpy only), loaded by
    file path so that the CPU legs do not import the s2dw_b200 package."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("s2dw_workload_gen", os.path.join(ROOT, "s2dw_b200", "workload.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.gaussian_flm


def _cpu_threads():
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    return max(1, min(n, 64))


class CpuPair:
    """The CPU restatement of the reference (oracle/, C + OpenMP, the
    reference's loops including its naive beta sums) on one configuration:
    tables from the oracle's own init_kernels / init_directionality, the
    seeded flm of the benchmark.  Nothing of the CUDA library is loaded."""

    def __init__(self, B, N, alpha, seed=0, threads=None):
        from oracle import oracle as O

        self.O = O
        self.threads = threads or _cpu_threads()
        O.set_num_threads(self.threads)
        J = O.comp_jmax(B, alpha)
        K, P, bs = O.init_kernels(J, B, alpha)
        S = O.init_directionality(B, N)
        self.flm = _generator()(B, seed=seed)
        self.a = (K, S, J, B, N, bs, alpha)
        self.s = (K, P, S, J, B, N, bs, alpha)
        self.B, self.N, self.J = B, N, J

    def pair(self):
        """One full analysis + synthesis; returns (seconds, recon error)."""
        t0 = time.perf_counter()
        w, sc = self.O.analysis_dynamic(self.flm, *self.a)
        f = self.O.synthesis_dynamic(w, sc, *self.s)
        dt = time.perf_counter() - t0
        return dt, float(np.abs(f - self.flm).max())


def cpu_baseline(B, N, alpha):
    """The CPU restatement timed on the host cores: one full, unsampled
    analysis+synthesis pair of the benchmark configuration (every scale,
    every loop iteration), after one untimed warm-up pair at B=128."""
    CpuPair(128, N, alpha).pair()
    cp = CpuPair(B, N, alpha)
    dt, err = cp.pair()
    return {"value": 1.0 / dt, "unit": UNIT, "cores": cp.threads, "kind": "port",
            "sample": (f"one full unsampled analysis+synthesis pair at B={B} N={N} alpha={alpha:g} J={cp.J} "
                       f"(all scales; CPU restatement of the reference loops in C/OpenMP, {cp.threads} threads): "
                       f"{dt:.1f} s, reconstruction error {err:.1e}"),
            "recon_err": err}


def run_reference(args):
    """The reference arm: the CPU restatement of the reference (oracle/,
    the reference's Fortran/FFTW cannot be compiled here) on the host cores.
    Warm-up steps are pairs at B=128 (threads and pages warm); each timed
    step is one full unsampled analysis+synthesis pair of the benchmark
    configuration.  Only the oracle's library is loaded."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    B, N, alpha = args.B, args.N, args.alpha
    warm = CpuPair(128, N, alpha)
    for _ in range(args.warmup):
        warm.pair()
    cp = CpuPair(B, N, alpha)
    times, errs = [], []
    for _ in range(args.steps):
        dt, err = cp.pair()
        times.append(dt)
        errs.append(err)
    total = sum(times)
    v = args.steps / total
    cb = {"value": v, "unit": UNIT, "cores": cp.threads, "kind": "port",
          "sample": (f"{args.steps} full unsampled analysis+synthesis pairs at B={B} N={N} alpha={alpha:g} "
                     f"J={cp.J} (all scales; CPU restatement of the reference loops in C/OpenMP, {cp.threads} "
                     f"threads), {total:.1f} s in all, {min(times):.1f}-{max(times):.1f} s per pair; "
                     f"warm-up: {args.warmup} pairs at B=128")}
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Gaussian C_l=1/(l(l+1)) flm)", "impl": "reference",
            "config": {"workload": f"B={B} N={N} alpha={alpha:g} J=Jmax={cp.J} analysis+synthesis of one map",
                       "B": B, "N": N, "alpha": alpha, "J": cp.J, "recon_err": max(errs)},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.steps is None:
        args.steps = 10 if args.impl == "reference" else 300
    if args.impl == "reference":
        run_reference(args)
        return
    import torch

    from s2dw_b200 import core
    from s2dw_b200.device import Plan
    from s2dw_b200.workload import gaussian_flm, transform_setup

    from s2dw_b200 import replicas

    world, rank, local = replicas.init_group("nccl")
    torch.cuda.set_device(local)
    barrier, max_over_ranks = replicas.barrier, replicas.max_over_ranks
    B, N, alpha = args.B, args.N, args.alpha
    t = transform_setup(B, N, alpha)
    J = t["J"]
    plan = Plan(B, N, alpha, J, device=local)
    plan.set_tables(t["K_gamma"], t["Phi2"], t["Slm"], t["bl_scoeff"])
    bs = t["bl_scoeff"]
    # a ring of inputs so consecutive steps never reuse the same flm
    nring = 4
    flms = [gaussian_flm(B, seed=rank * 1000 + i) for i in range(nring)]
    d_flm = [torch.from_numpy(np.ascontiguousarray(f.T)).cuda() for f in flms]
    d_wav = torch.empty(plan.wav_size, dtype=torch.float64, device="cuda")
    d_sc = torch.empty(max(1, bs * bs), dtype=torch.complex128, device="cuda")
    d_out = torch.empty_like(d_flm[0])
    stream = torch.cuda.current_stream()

    def direct_step(i):
        plan.analysis(d_flm[i % nring], d_wav, d_sc, stream)
        plan.synthesis(d_wav, d_sc, d_out, stream)

    graphs = []
    if not args.no_graph:
        direct_step(0)  # kernel attributes are set outside capture
        torch.cuda.synchronize()
        cap_stream = torch.cuda.Stream()  # capture needs a non-default stream
        for i in range(nring):
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=cap_stream):
                plan.analysis(d_flm[i], d_wav, d_sc, torch.cuda.current_stream())
                plan.synthesis(d_wav, d_sc, d_out, torch.cuda.current_stream())
            graphs.append(g)

    def step(i):
        if graphs:
            graphs[i % nring].replay()
        else:
            direct_step(i)

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    # reconstruction check of the last warm-up pair
    recon = float(np.abs(d_out.cpu().numpy().T - flms[(args.warmup - 1) % nring]).max())

    clocks = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(args.steps):
        step(i)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    elapsed = e0.elapsed_time(e1) / 1e3
    elapsed = max_over_ranks(elapsed, world)
    pairs = args.steps * world
    value = pairs / elapsed
    la, ls = plan.launch_counts()

    # ---- per-kernel device times: a second timed loop in which the plan
    # brackets every launch with CUDA events (scales serialised on `stream`)
    ksteps = max(3, min(args.steps, 10))
    plan.set_timing(True)
    plan.timing(reset=True)
    for i in range(ksteps):
        direct_step(i)
    torch.cuda.synchronize()
    kt = plan.timing(reset=True)
    plan.set_timing(False)

    # ---- roofline of the dominant kernel (largest device-time share)
    fp64_peak = measured_fp64_peak()
    ana_f, syn_f = contraction_flops_per_scale(B, N, alpha, J)
    dom = max(kt.items(), key=lambda kv: kv[1][1])
    algo = dict(fft_flops_per_pair(B, N, alpha, J))
    algo["lwalk"], algo["mwalk"] = sum(ana_f), sum(syn_f)
    n_launch, ms = dom[1]
    roofline = None
    if dom[0] in algo and n_launch:
        per_launch_ms = ms / n_launch
        launches_per_pair = n_launch / ksteps
        achieved = algo[dom[0]] / launches_per_pair / (per_launch_ms / 1e3) / 1e12
        traffic = NCU_TRAFFIC.get((B, N, float(alpha)), {}).get(dom[0])
        roofline = {"kernel": dom[0], "bound": "fp64", "achieved": achieved, "peak": fp64_peak,
                    "unit": "TFLOP/s", "frac": achieved / fp64_peak, "traffic": traffic,
                    "traffic_unit": "bytes per launch (ncu, mean over a pair's launches)",
                    "traffic_source": NCU_TRAFFIC_SOURCE,
                    "peak_source": "measured cuBLAS DGEMM 4096^3 on this GPU (MEASURED_PEAKS.json has no fp64 entry)",
                    "flops_per_pair": algo[dom[0]], "launches_per_pair": launches_per_pair,
                    "avg_launch_ms": per_launch_ms,
                    "pair": pair_roofline(B, N, alpha, J, 1e3 * elapsed / args.steps, fp64_peak)}
    kernel_tflops = {k: (algo[k] * ksteps / (v[1] / 1e3) / 1e12 if k in algo and v[1] > 0 else None)
                     for k, v in kt.items()}
    # achieved DRAM bandwidth per kind: the ncu traffic per launch of this
    # workload (when known) times the launches, over the CUDA-event time
    trf = NCU_TRAFFIC.get((B, N, float(alpha)), {})
    kernel_gbs = {k: (trf[k] * v[0] / (v[1] / 1e3) / 1e9 if k in trf and v[1] > 0 else None) for k, v in kt.items()}
    kernel_ms = {k: {"launches_per_step": v[0] / ksteps, "ms_per_step": v[1] / ksteps,
                     "tflops": kernel_tflops[k], "dram_gbs": kernel_gbs[k],
                     "dram_frac_of_hbm": (kernel_gbs[k] / HBM_GBS if kernel_gbs[k] else None)}
                 for k, v in kt.items()}

    # ---- end to end through the C ABI with pinned host buffers
    e2e = None
    if rank == 0 or world > 1:
        a_ = (t["K_gamma"], t["Slm"], J, B, N, bs, alpha)
        wav_h = [torch.empty(core.wav_scale_shape(j, B, N, alpha)[::-1], dtype=torch.float64,
                             pin_memory=True).numpy().T for j in range(J + 1)]
        flm_h = [torch.empty((B, B), dtype=torch.complex128, pin_memory=True).numpy().T for _ in range(nring)]
        for i in range(nring):
            flm_h[i][...] = flms[i]
        out_h = torch.empty((B, B), dtype=torch.complex128, pin_memory=True).numpy().T
        sc_h = np.zeros((bs, bs), dtype=np.complex128, order="F")
        import ctypes

        from s2dw_b200._lib import check, lib

        dp = ctypes.POINTER(ctypes.c_double)
        L = lib()
        wptr = (dp * (J + 1))(*[w.ctypes.data_as(dp) for w in wav_h])
        K = np.asfortranarray(t["K_gamma"])
        P = np.ascontiguousarray(t["Phi2"])
        S = np.asfortranarray(t["Slm"])

        def e2e_step(i):
            check(L.s2dwc_analysis_flm2wav_dynamic(wptr, sc_h.ctypes.data_as(dp), flm_h[i % nring].ctypes.data_as(dp),
                                                   K.ctypes.data_as(dp), S.ctypes.data_as(dp), J, B, N, bs, alpha))
            check(L.s2dwc_synthesis_wav2flm_dynamic(out_h.ctypes.data_as(dp), wptr, sc_h.ctypes.data_as(dp),
                                                    K.ctypes.data_as(dp), P.ctypes.data_as(dp), S.ctypes.data_as(dp),
                                                    J, B, N, bs, alpha))

        for i in range(2):
            e2e_step(i)
        barrier(world)
        t0 = time.perf_counter()
        for i in range(args.e2e_steps):
            e2e_step(i)
        te = time.perf_counter() - t0
        te = max_over_ranks(te, world)
        e2e_recon = float(np.abs(out_h - flm_h[(args.e2e_steps - 1) % nring]).max())
        wav_bytes = 8 * plan.wav_size
        e2e = {"value": args.e2e_steps * world / te, "unit": UNIT,
               "h2d_bytes_per_step": 16 * B * B + wav_bytes + 16 * bs * bs,
               "d2h_bytes_per_step": wav_bytes + 16 * bs * bs + 16 * B * B,
               "recon_err": e2e_recon,
               "api": "s2dwc_analysis_flm2wav_dynamic + s2dwc_synthesis_wav2flm_dynamic, pinned host buffers"}
        # PCIe floor: plain page-locked copies of the same bytes, one direction
        # at a time as a pair of calls moves them (the analysis output leaves
        # before the synthesis input arrives)
        nb = wav_bytes // 8
        hbuf = torch.empty(nb, dtype=torch.float64, pin_memory=True)
        dbuf = torch.empty(nb, dtype=torch.float64, device=f"cuda:{local}")
        rates = {}
        for name, dst, src in (("h2d", dbuf, hbuf), ("d2h", hbuf, dbuf)):
            dst.copy_(src, non_blocking=True)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(4):
                dst.copy_(src, non_blocking=True)
            torch.cuda.synchronize()
            rates[name] = 4 * wav_bytes / (time.perf_counter() - t0) / 1e9
        floor_s = e2e["h2d_bytes_per_step"] / (rates["h2d"] * 1e9) + e2e["d2h_bytes_per_step"] / (rates["d2h"] * 1e9)
        e2e["copy_floor"] = {"h2d_gbs": rates["h2d"], "d2h_gbs": rates["d2h"], "pairs_per_s": 1.0 / floor_s,
                             "frac": e2e["value"] / world / (1.0 / floor_s),
                             "what": "pinned cudaMemcpy of the step's bytes, no kernels: the bound of e2e"}
        del hbuf, dbuf
        # the same with ordinary (pageable) arrays, as Fortran callers pass them
        pg = [np.zeros(core.wav_scale_shape(j, B, N, alpha), order="F") for j in range(J + 1)]
        wptr = (dp * (J + 1))(*[w.ctypes.data_as(dp) for w in pg])
        flm_p = [np.asfortranarray(f) for f in flms]
        out_p = np.zeros((B, B), dtype=np.complex128, order="F")

        def e2e_step_p(i):
            check(L.s2dwc_analysis_flm2wav_dynamic(wptr, sc_h.ctypes.data_as(dp), flm_p[i % nring].ctypes.data_as(dp),
                                                   K.ctypes.data_as(dp), S.ctypes.data_as(dp), J, B, N, bs, alpha))
            check(L.s2dwc_synthesis_wav2flm_dynamic(out_p.ctypes.data_as(dp), wptr, sc_h.ctypes.data_as(dp),
                                                    K.ctypes.data_as(dp), P.ctypes.data_as(dp), S.ctypes.data_as(dp),
                                                    J, B, N, bs, alpha))

        for i in range(2):
            e2e_step_p(i)
        barrier(world)
        t0 = time.perf_counter()
        for i in range(args.e2e_steps):
            e2e_step_p(i)
        tp = max_over_ranks(time.perf_counter() - t0, world)
        e2e["pageable"] = {"value": args.e2e_steps * world / tp, "unit": UNIT,
                           "recon_err": float(np.abs(out_p - flms[(args.e2e_steps - 1) % nring]).max()),
                           "api": "same entry points, pageable numpy arrays (staged through page-locked buffers)"}
        del pg

    graphs.clear()
    serving = None
    if args.serving_requests > 0:
        try:
            serving = serving_stats(args.serving_requests, local, args.serving_split_requests)
        except Exception as ex:
            serving = {"error": str(ex)[:300]}

    large = None
    if not args.no_large and rank == 0:
        try:
            large = large_stats()
        except Exception as ex:
            large = {"error": str(ex)[:300]}
        if args.large_split_maps > 0 and "error" not in large:
            from s2dw_b200.core import s2dw_core_comp_Jmax
            try:
                large["split"] = split_stats(2048, 8, 2.0, s2dw_core_comp_Jmax(2048, 2.0), args.large_split_maps,
                                             repeats=1, power=1.2)
            except Exception as ex:
                large["split"] = {"error": str(ex)[:300]}

    split_b256 = None
    if args.split_maps > 0 and not args.no_b256 and rank == 0:
        from s2dw_b200.core import s2dw_core_comp_Jmax
        try:
            split_b256 = split_stats(256, 5, 2.0, s2dw_core_comp_Jmax(256, 2.0), args.split_maps)
        except Exception as ex:
            split_b256 = {"error": str(ex)[:300]}

    split = None
    if args.split_maps > 0:
        try:
            split = split_stats(B, N, alpha, J, args.split_maps)
            split["pair_roofline"] = pair_roofline(B, N, alpha, J, 1e3 / split["value"], fp64_peak)
        except Exception as ex:
            split = {"error": str(ex)[:300]}
    # the benchmark configuration itself in the split form: one map per pair
    split_one = None
    if args.split_maps > 0 and rank == 0:
        try:
            split_one = split_stats(B, N, alpha, J, 1, repeats=10)
            split_one["pair_roofline"] = pair_roofline(B, N, alpha, J, 1e3 / split_one["value"], fp64_peak)
        except Exception as ex:
            split_one = {"error": str(ex)[:300]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(B, N, alpha)
        except Exception as ex:  # keep the GPU line even if the oracle is absent
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "port", "sample": f"unavailable: {ex}"}

    if rank == 0:
        def g(d, *ks):
            for k in ks:
                if not isinstance(d, dict) or k not in d:
                    return None
                d = d[k]
            return d

        # compact figures last: a reader of the line's tail sees them
        summary = {
            "fp64_pairs_s": value, "e2e_pairs_s": g(e2e, "value"), "cpu_pairs_s": g(cpu, "value"),
            "roofline_frac_dominant_kernel": g(roofline, "frac"), "roofline_frac_pair": g(roofline, "pair", "frac"),
            "split_one_map_pairs_s": g(split_one, "value"), "split_one_map_vs_fp64": g(split_one, "speedup_vs_fp64"),
            "split_32maps_pairs_s_per_map": g(split, "value"), "split_32maps_vs_fp64": g(split, "speedup_vs_fp64"),
            "split_max_w_err": g(split, "max_w_err"), "split_b256_vs_fp64": g(split_b256, "speedup_vs_fp64"),
            "large_b2048_pairs_s": g(large, "value"), "large_split_vs_fp64": g(large, "split", "speedup_vs_fp64"),
            "serving_saturation_rps": g(serving, "saturation_rps"),
            "serving_serial_device_s": g(serving, "serial_device_s"),
            "serving_rps": g(serving, "throughput_rps"), "serving_p50_ms": g(serving, "p50_ms"),
            "serving_p99_ms": g(serving, "p99_ms"), "serving_split_p50_ms": g(serving, "split", "p50_ms"),
            "serving_split_p99_ms": g(serving, "split", "p99_ms"),
            "serving_burst_split_vs_fp64": g(serving, "burst", "split_vs_fp64"),
        }
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Gaussian C_l=1/(l(l+1)) flm, no dataset)",
            "config": {"workload": f"B={B} N={N} alpha={alpha:g} J=Jmax={J} analysis+synthesis of one map per step",
                       "B": B, "N": N, "alpha": alpha, "J": J, "form": "fp64 plain",
                       "parallelism": f"replicas x{world} (no collective)",
                       "launch": "direct" if args.no_graph else "CUDA graph replay of the pair",
                       "l2": f"each step reads/writes a {8 * plan.wav_size / 1e6:.0f} MB wavelet array (> 126 MB L2); flm from a ring of {nring}",
                       "recon_err": recon},
            "gpu_launches": (la + ls) * args.steps, "clocks": clk, "roofline": roofline, "cpu_baseline": cpu,
            "e2e": e2e, "kernels": kernel_ms, "large": large, "split_b256": split_b256, "split": split,
            "split_one_map": split_one, "serving": serving, "summary": summary,
        }
        print(json.dumps(line), flush=True)
    plan.close()
    replicas.finish(world)


if __name__ == "__main__":
    main()
