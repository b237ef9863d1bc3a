"""Continuous-batching server for mixed S2DW transform requests on one GPU.

Requests are analyses (flm -> wav) or syntheses (wav -> flm) of any supported
(B, N, alpha, J).  A request is admitted as soon as a *slot* for its
configuration is free: a slot is a plan (cached recurrence and chirp tables,
workspaces, per-scale streams) with its own output buffers and CUDA stream.
Slots are created on demand while the device memory they hold stays within
an HBM budget; when the budget is full an idle slot of another configuration
is evicted (least recently used) or the request waits.  Admitted requests run
concurrently on their slots' streams, so work of requests that arrive while
others are on the GPU overlaps on the device.  Each slot replays a CUDA graph
captured once per (kind, input buffer), which removes the per-kernel launch
cost of the ~20-70 kernels a transform issues.

With ``form="split"`` the slots run the split-precision plan, whose
tensor-core pass shares the Wigner-d digits among up to 32 maps: a free slot
takes every waiting request of its configuration and kind (up to the slot's
batch capacity) as one batch.  The batch's inputs are copied into the slot's
staging buffers, so one CUDA graph per (kind, batch size) serves every batch.
With ``form="auto"`` a request goes to a split slot when at least
``split_min_batch`` requests of its configuration and kind are waiting (the
batch size from which the split form is faster, about 17 maps at B=1024,
N=4), and to an FP64 slot otherwise.

Results are identical alone and in a mix: the kernels are deterministic (no
atomics; the synthesis sums scales in a fixed order), a slot's buffers are
owned by one batch at a time, and in the split form each map's digits are
scaled by that map's own exponents, so a map's result does not depend on the
other maps of its batch.

Latency of a request = device time of its completion event minus its arrival
time, both relative to the stream's start (an event recorded when the first
request is admitted).
"""
import collections
import dataclasses
import time

import numpy as np

from .device import Plan
from .workload import transform_setup


@dataclasses.dataclass
class Request:
    rid: int
    kind: str                 # "analysis" or "synthesis"
    B: int
    N: int
    alpha: float
    J: int
    arrival: float            # seconds after the stream start
    inp: tuple = ()           # device tensors: (flm,) or (wav, scoeff)
    # filled by the server
    slot_key: tuple = None
    done_event: object = None
    t_done: float = None      # seconds after the stream start (device clock)
    out: object = None        # host copy of the output when keep_outputs


def split_batch_capacity(B, N, alpha, J, max_batch=32, batch_bytes=2 << 30):
    """Maps per batch of a split-form slot: up to `max_batch`, with the
    slot's packed wavelet buffer within `batch_bytes`."""
    return max(1, min(max_batch, int(batch_bytes) // (8 * _wav_size(B, N, alpha, J))))


def size_priority(B):
    """CUDA stream priority of a slot by band limit (lower runs first): the
    small transforms, a few microseconds of latency-bound kernels each, take
    SMs ahead of the full-band scales of large ones (shortest job first)."""
    return 0 if B >= 1024 else -1 if B >= 512 else -2 if B >= 256 else -3


class Slot:
    def __init__(self, key, tables, device, form="fp64", max_batch=32, batch_bytes=2 << 30, priority=None,
                 split_min_batch=1):
        import torch

        B, N, alpha, J = key
        self.key = key
        self.split = form == "split"
        self.cap = split_batch_capacity(B, N, alpha, J, max_batch, batch_bytes) if self.split else 1
        self.plan = Plan(B, N, alpha, J, device=device, form=Plan.SPLIT if self.split else Plan.FP64)
        self.plan.set_tables(tables["K_gamma"], tables["Phi2"], tables["Slm"], tables["bl_scoeff"])
        if self.split and split_min_batch > 1:
            self.plan.set_split_min_batch(split_min_batch)
        bs = tables["bl_scoeff"]
        if priority is not None:
            self.plan.set_priority(priority)
            self.stream = torch.cuda.Stream(device=device, priority=priority)
        else:
            self.stream = torch.cuda.Stream(device=device)
        c = self.cap
        self.d_wav = torch.empty((c, self.plan.wav_size), dtype=torch.float64, device=device)
        self.d_sc = torch.empty((c, max(1, bs * bs)), dtype=torch.complex128, device=device)
        self.d_flm = torch.empty((c, B, B), dtype=torch.complex128, device=device)
        staged = 0
        if self.split:
            # analysis inputs are staged here; synthesis inputs in d_wav / d_sc
            self.in_flm = torch.empty((c, B, B), dtype=torch.complex128, device=device)
            staged = 16 * c * B * B
            self.plan.reserve(c, stream=self.stream)
            self.stream.synchronize()
        self.bytes = (self.plan.workspace_bytes() + 8 * c * self.plan.wav_size + 16 * c * (max(1, bs * bs) + B * B)
                      + staged)
        self.graphs = {}
        self.busy = False
        self.last_used = 0.0
        # recorded just before the slot's last batch starts (its device time
        # when the batch runs alone: Server.device_time)
        self.ev_start = torch.cuda.Event(enable_timing=True)

    def run(self, reqs, use_graphs):
        """Enqueue the transform of a batch of requests (one request in the
        FP64 form; same kind, at most `cap`) on this slot's stream."""
        import torch

        kind, k = reqs[0].kind, len(reqs)
        if self.split:
            with torch.cuda.stream(self.stream):
                for i, r in enumerate(reqs):
                    if kind == "analysis":
                        self.in_flm[i].copy_(r.inp[0], non_blocking=True)
                    else:
                        self.d_wav[i].copy_(r.inp[0], non_blocking=True)
                        self.d_sc[i].copy_(r.inp[1].reshape(-1), non_blocking=True)

        def body():
            cs = torch.cuda.current_stream()
            if self.split:
                if kind == "analysis":
                    self.plan.analysis_batch(self.in_flm[:k], self.d_wav[:k], self.d_sc[:k], stream=cs)
                else:
                    self.plan.synthesis_batch(self.d_wav[:k], self.d_sc[:k], self.d_flm[:k], stream=cs)
            elif kind == "analysis":
                self.plan.analysis(reqs[0].inp[0], self.d_wav[0], self.d_sc[0], stream=cs)
            else:
                self.plan.synthesis(reqs[0].inp[0], reqs[0].inp[1], self.d_flm[0], stream=cs)

        with torch.cuda.stream(self.stream):
            if use_graphs:
                if self.split:
                    gkey = (kind, k)
                else:
                    gkey = (kind,) + tuple(t.data_ptr() for t in reqs[0].inp)
                g = self.graphs.get(gkey)
                if g is None:
                    body()  # warm-up launch outside capture (lazy kernel attributes)
                    g = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(g, stream=self.stream):
                        body()
                    self.graphs[gkey] = g
                self.ev_start.record(self.stream)
                g.replay()
            else:
                self.ev_start.record(self.stream)
                body()
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(self.stream)
        return ev

    def output(self, req, i=0):
        """Output tensors of the i-th request of the batch that just ran."""
        return (self.d_wav[i], self.d_sc[i]) if req.kind == "analysis" else (self.d_flm[i],)

    def close(self):
        self.graphs.clear()
        self.plan.close()


class Server:
    def __init__(self, hbm_budget_bytes=40 << 30, max_inflight=64, slots_per_config=2, use_graphs=True,
                 device=0, keep_outputs=False, form="fp64", max_batch=32, batch_bytes=2 << 30,
                 priorities=False, split_min_batch=1):
        if form not in ("fp64", "split", "auto"):
            raise ValueError(f"form must be 'fp64', 'split' or 'auto', not {form!r}")
        self.form = form
        # split slots: batches smaller than this run the FP64 path (the split
        # form pays from ~17 maps of one configuration at B=1024, N=4)
        self.split_min_batch = split_min_batch
        self.priorities = priorities  # slots' stream priorities by size (size_priority)
        self.max_batch = max_batch
        self.batch_bytes = batch_bytes
        self.budget = int(hbm_budget_bytes)
        self.max_inflight = max_inflight
        self.slots_per_config = slots_per_config
        self.use_graphs = use_graphs
        self.device = device
        self.keep_outputs = keep_outputs
        self.slots = collections.defaultdict(list)  # key -> [Slot]
        self.tables = {}
        self.used = 0

    def config_tables(self, B, N, alpha, J):
        key = (B, N, alpha, J)
        if key not in self.tables:
            self.tables[key] = transform_setup(B, N, alpha, J)
        return self.tables[key]

    def _evict_one(self, keep_key):
        idle = [s for k, lst in self.slots.items() if k != keep_key for s in lst if not s.busy]
        if not idle:
            return False
        victim = min(idle, key=lambda s: s.last_used)
        self.slots[victim.key].remove(victim)
        self.used -= victim.bytes
        victim.close()
        return True

    def _acquire(self, key, now, form=None):
        """A free slot of `key` in `form` (the server's form by default),
        created within the HBM budget if needed; None if there is none."""
        form = form or ("split" if self.form == "split" else "fp64")
        mine = [s for s in self.slots[key] if (s.split == (form == "split"))]
        for s in mine:
            if not s.busy:
                return s
        if len(mine) >= self.slots_per_config:
            return None
        B, N, alpha, J = key
        # size estimate of a new slot; evict idle slots of other configs if needed
        est = Slot.estimate_bytes(B, N, alpha, J, form, self.max_batch, self.batch_bytes)
        while self.used + est > self.budget:
            if not self._evict_one(key):
                return None
        s = Slot(key, self.config_tables(B, N, alpha, J), self.device, form, self.max_batch, self.batch_bytes,
                 priority=size_priority(B) if self.priorities else None, split_min_batch=self.split_min_batch)
        self.slots[key].append(s)
        self.used += s.bytes
        return s

    def run(self, requests, poll_sleep=0.0):
        """Serves `requests` (sorted by arrival) with wall-clock arrivals.
        Returns a dict of latency/throughput statistics."""
        import torch

        torch.cuda.set_device(self.device)
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        waiting = collections.deque()
        inflight = []
        done = []
        batches = []
        base = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        base.record()
        while pending or waiting or inflight:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                waiting.append(pending.popleft())
            # admit in arrival order; a request whose config has no free slot
            # does not block requests of other configs
            still = collections.deque()
            while waiting:
                r = waiting.popleft()
                if len(inflight) >= self.max_inflight:
                    still.append(r)
                    continue
                key = (r.B, r.N, r.alpha, r.J)
                form = None
                if self.form == "auto":
                    # a split slot only for a batch the split form serves faster
                    same = 1 + sum(1 for r2 in waiting if r2.kind == r.kind and (r2.B, r2.N, r2.alpha, r2.J) == key)
                    form = "split" if same >= self.split_min_batch else "fp64"
                s = self._acquire(key, now, form)
                if s is None:
                    still.append(r)
                    continue
                batch = [r]
                if s.cap > 1:
                    # the later waiting requests of the same configuration and kind
                    rest_w = collections.deque()
                    for r2 in waiting:
                        if (len(batch) < s.cap and r2.kind == r.kind
                                and (r2.B, r2.N, r2.alpha, r2.J) == key):
                            batch.append(r2)
                        else:
                            rest_w.append(r2)
                    waiting = rest_w
                s.busy = True
                s.last_used = now
                ev = s.run(batch, self.use_graphs)
                for rb in batch:
                    rb.slot_key = key
                    rb.done_event = ev
                inflight.append((batch, s))
                batches.append(len(batch))
            waiting = still
            rest = []
            for batch, s in inflight:
                ev = batch[0].done_event
                if ev.query():
                    t_done = base.elapsed_time(ev) / 1e3
                    for i, rb in enumerate(batch):
                        rb.t_done = t_done
                        if self.keep_outputs:
                            rb.out = tuple(t.detach().cpu().numpy().copy() for t in s.output(rb, i))
                        done.append(rb)
                    s.busy = False
                else:
                    rest.append((batch, s))
            inflight = rest
            if not inflight and not waiting and pending:
                delay = pending[0].arrival - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
            elif poll_sleep:
                time.sleep(poll_sleep)
        torch.cuda.synchronize()
        t_end = time.perf_counter() - t0
        lat = np.array([r.t_done - r.arrival for r in done]) * 1e3
        span = max(r.t_done for r in done) - min(r.arrival for r in done)
        return {"requests": len(done), "p50_ms": float(np.percentile(lat, 50)),
                "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
                "throughput_rps": len(done) / span, "wall_s": t_end, "form": self.form,
                "batches": len(batches), "mean_batch": float(np.mean(batches)) if batches else 0.0,
                "slots": sum(len(v) for v in self.slots.values()), "hbm_bytes": self.used}

    def device_time(self, requests):
        """Sum over `requests` of each one's device time run alone (one at a
        time, graphs and slots already warm): the stream's GPU work with no
        overlap between requests, against which a saturation span shows how
        much the server overlaps requests and whether the host loop limits it."""
        import torch

        torch.cuda.set_device(self.device)
        total = 0.0
        for r in requests:
            key = (r.B, r.N, r.alpha, r.J)
            s = self._acquire(key, 0.0)
            ev = s.run([r], self.use_graphs)
            ev.synchronize()
            total += s.ev_start.elapsed_time(ev) / 1e3
        return total

    def close(self):
        for lst in self.slots.values():
            for s in lst:
                s.close()
        self.slots.clear()
        self.used = 0


def _wav_size(B, N, alpha, J):
    from .core import band_limits

    return sum((2 * bl - 1) * 2 * bl * N for bl, _ in (band_limits(j, B, alpha) for j in range(J + 1)))


def _estimate_bytes(B, N, alpha, J, form="fp64", max_batch=32, batch_bytes=2 << 30):
    """Device bytes a slot of (B, N, alpha, J) holds (plan + buffers); for
    the split form with the map workspaces and staging of its batch."""
    from .core import band_limits

    wav = _wav_size(B, N, alpha, J)
    tg = ta = sq = 0
    for j in range(J + 1):
        bl, _ = band_limits(j, B, alpha)
        tg += N * bl * bl
        ta += N * bl * 2 * bl
        sq += bl * bl
    Bp = (B + 31) // 32 * 32
    tables = B * Bp * 8 * 6 + B * B * 8 * 8 + B * B * 16
    fp64 = 8 * wav + 16 * (tg + ta) * 3 // 2 + tables + 16 * B * B * 3
    if form != "split":
        return fp64
    c = split_batch_capacity(B, N, alpha, J, max_batch, batch_bytes)
    digits = 2 * 12 * 64 * sq + 2 * 2 * N * sq  # map digits of both directions, exponent tables
    return fp64 + digits + c * (8 * wav + 16 * (tg + 2 * ta) + 16 * 2 * B * B)


Slot.estimate_bytes = staticmethod(_estimate_bytes)


def make_stream(n_requests, seed=0, rate_hz=2000.0, Bs=(32, 64, 128, 256, 512, 1024), Ns=range(1, 9),
                alphas=(2.0, 3.0), device="cuda", pool=2):
    """The benchmark's mixed request stream: Poisson arrivals at `rate_hz`,
    B uniform over `Bs`, N uniform over `Ns`, alpha over `alphas`, J = Jmax,
    half analyses and half syntheses.  Inputs are device-resident: `pool`
    seeded maps per configuration (analysis inputs from the Gaussian
    generator; synthesis inputs from an analysis of such a map), shared by the
    requests of that configuration.  Returns (requests, inputs) where inputs
    maps config -> list of (flm, wav, scoeff) device tensors."""
    import torch

    from . import core
    from .workload import gaussian_flm

    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    inputs = {}
    for i in range(n_requests):
        t += rng.exponential(1.0 / rate_hz)
        B = int(rng.choice(Bs))
        N = int(rng.choice(list(Ns)))
        alpha = float(rng.choice(alphas))
        J = core.s2dw_core_comp_Jmax(B, alpha)
        kind = "analysis" if rng.random() < 0.5 else "synthesis"
        key = (B, N, alpha, J)
        if key not in inputs:
            inputs[key] = None
        reqs.append(Request(rid=i, kind=kind, B=B, N=N, alpha=alpha, J=J, arrival=t,
                            inp=(int(rng.integers(pool)),)))
    # device-resident inputs per configuration
    for key in inputs:
        B, N, alpha, J = key
        tab = transform_setup(B, N, alpha, J)
        plan = Plan(B, N, alpha, J)
        plan.set_tables(tab["K_gamma"], tab["Phi2"], tab["Slm"], tab["bl_scoeff"])
        lst = []
        for k in range(pool):
            flm = gaussian_flm(B, seed=1000 * k + B + 17 * N)
            d_flm = torch.from_numpy(np.ascontiguousarray(flm.T)).to(device)
            d_wav = torch.empty(plan.wav_size, dtype=torch.float64, device=device)
            d_sc = torch.empty(max(1, tab["bl_scoeff"] ** 2), dtype=torch.complex128, device=device)
            plan.analysis(d_flm, d_wav, d_sc)
            lst.append((d_flm, d_wav, d_sc, flm))
        torch.cuda.synchronize()
        plan.close()
        inputs[key] = lst
    for r in reqs:
        d_flm, d_wav, d_sc, _ = inputs[(r.B, r.N, r.alpha, r.J)][r.inp[0]]
        r.inp = (d_flm,) if r.kind == "analysis" else (d_wav, d_sc)
    return reqs, inputs
