"""Device-resident API: a plan for (B, N, alpha, J) and transforms on CUDA
tensors (torch is used only to own device memory and streams).

Layouts on the device (all contiguous):
  flm     complex128, B*B values, flm[l + B*m]          (torch shape (B, B) = flm^T)
  scoeff  complex128, bs*bs values, scoeff[l + bs*m]
  wav     float64, packed per-scale layout; scale jj occupies
          [offsets[jj], offsets[jj+1]) in coeff(a, b, g) order (a fastest).
"""
import ctypes

import numpy as np

from ._lib import check, lib
from .core import band_limits


def plan_footprint(B, N, alpha, J, form=0):
    """Device bytes a plan for (B, N, alpha, J, form) allocates when created,
    computed on the host (no device is touched)."""
    out = ctypes.c_longlong(0)
    check(lib().s2dwc_plan_footprint(int(B), int(N), float(alpha), int(J), int(form), ctypes.byref(out)))
    return int(out.value)


def set_plan_memory_limit(nbytes):
    """Process-wide limit on one plan's device memory (0: none).  Plans above
    it are refused with S2DW_ERROR_MEM_ALLOC_FAIL (4) before any device call."""
    check(lib().s2dwc_set_plan_memory_limit(int(nbytes)))


class Plan:
    FP64, SPLIT = 0, 1

    def __init__(self, B, N, alpha, J, device=0, form=0):
        import torch

        self.B, self.N, self.alpha, self.J, self.device = int(B), int(N), float(alpha), int(J), int(device)
        self.form = int(form)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            check(lib().s2dwc_plan_create(ctypes.byref(h), self.B, self.N, self.alpha, self.J, self.form,
                                          self.device))
        self._h = h
        offs = (ctypes.c_longlong * (J + 2))()
        check(lib().s2dwc_plan_wav_offsets(self._h, offs))
        self.wav_offsets = [int(v) for v in offs]
        self.bl = [band_limits(j, B, alpha)[0] for j in range(J + 1)]
        self.bl_scoeff = None

    def close(self):
        if getattr(self, "_h", None):
            lib().s2dwc_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def wav_size(self):
        return self.wav_offsets[-1]

    def workspace_bytes(self):
        return int(lib().s2dwc_plan_workspace_bytes(self._h))

    def launch_counts(self):
        a, s = ctypes.c_int(0), ctypes.c_int(0)
        check(lib().s2dwc_plan_launch_count(self._h, ctypes.byref(a), ctypes.byref(s)))
        return a.value, s.value

    def set_timing(self, enable=True):
        check(lib().s2dwc_plan_set_timing(self._h, int(bool(enable))))

    def timing(self, reset=False):
        """{kind: (launches, total_ms)} accumulated since the last reset."""
        from ._lib import KERNEL_KINDS

        out = {}
        for k, name in enumerate(KERNEL_KINDS):
            n, ms = ctypes.c_longlong(0), ctypes.c_double(0.0)
            check(lib().s2dwc_plan_timing(self._h, k, ctypes.byref(n), ctypes.byref(ms)))
            out[name] = (n.value, ms.value)
        if reset:
            check(lib().s2dwc_plan_timing_reset(self._h))
        return out

    def set_tables(self, K_gamma, Phi2, Slm, bl_scoeff):
        dp = ctypes.POINTER(ctypes.c_double)
        K = np.asfortranarray(K_gamma, dtype=np.float64)
        S = np.asfortranarray(Slm, dtype=np.complex128)
        P = None if Phi2 is None else np.ascontiguousarray(Phi2, dtype=np.float64)
        check(lib().s2dwc_plan_set_tables(self._h, K.ctypes.data_as(dp),
                                          None if P is None else P.ctypes.data_as(dp),
                                          S.ctypes.data_as(dp), int(bl_scoeff)))
        self.bl_scoeff = int(bl_scoeff)

    def scale_view(self, wav, jj):
        """View of scale jj of a packed wav tensor as (N, 2bl, 2bl-1) in C
        order, i.e. coeff(a, b, g) at [g, b, a]."""
        b = self.bl[jj]
        return wav[self.wav_offsets[jj]:self.wav_offsets[jj + 1]].view(self.N, 2 * b, 2 * b - 1)

    @staticmethod
    def _ptr(t, dtype, numel):
        import torch

        if t is None:
            return None
        if not t.is_cuda or not t.is_contiguous() or t.dtype != dtype or t.numel() < numel:
            raise ValueError(f"expected a contiguous CUDA {dtype} tensor of >= {numel} elements")
        return ctypes.c_void_p(t.data_ptr())

    @staticmethod
    def _stream(stream):
        import torch

        s = stream if stream is not None else torch.cuda.current_stream()
        return ctypes.c_void_p(s.cuda_stream)

    def analysis(self, flm, wav, scoeff, stream=None):
        import torch

        check(lib().s2dwc_plan_analysis(self._h, self._ptr(wav, torch.float64, self.wav_size),
                                        self._ptr(scoeff, torch.complex128, self.bl_scoeff ** 2),
                                        self._ptr(flm, torch.complex128, self.B * self.B),
                                        self._stream(stream)))

    def analysis_noalloc(self, flm, wav, scoeff, stream=None):
        """The analysis of `analysis` through s2dwc_plan_analysis_noalloc: its
        workspace is the library's static device scratch, so the call
        allocates nothing (plans up to the scratch's size only)."""
        import torch

        check(lib().s2dwc_plan_analysis_noalloc(self._h, self._ptr(wav, torch.float64, self.wav_size),
                                                self._ptr(scoeff, torch.complex128, self.bl_scoeff ** 2),
                                                self._ptr(flm, torch.complex128, self.B * self.B),
                                                self._stream(stream)))

    def analysis_batch(self, flm, wav, scoeff, stream=None):
        """Analysis of flm.shape[0] maps: flm (n, B, B) complex128 (each map
        stored as the reference's column-major flm), wav (n, wav_size), scoeff
        (n, bl_scoeff**2)."""
        import torch

        n = int(flm.shape[0])
        check(lib().s2dwc_plan_analysis_batch(self._h, n, self._ptr(wav, torch.float64, n * self.wav_size),
                                              self._ptr(scoeff, torch.complex128, n * self.bl_scoeff ** 2),
                                              self._ptr(flm, torch.complex128, n * self.B * self.B),
                                              self._stream(stream)))

    def synthesis_batch(self, wav, scoeff, flm, stream=None):
        import torch

        n = int(flm.shape[0])
        check(lib().s2dwc_plan_synthesis_batch(self._h, n, self._ptr(flm, torch.complex128, n * self.B * self.B),
                                               self._ptr(wav, torch.float64, n * self.wav_size),
                                               self._ptr(scoeff, torch.complex128, n * self.bl_scoeff ** 2),
                                               self._stream(stream)))

    def stat_moments(self, wav, moments, mask=None, stream=None):
        """Moments per scale of wav.shape[0] device maps (packed layout) into
        moments (n, J+1, 6): mean, var, skew, kur, five, six."""
        import torch

        n = int(wav.shape[0]) if wav.dim() > 1 else 1
        check(lib().s2dwc_plan_stat_moments(self._h, n, self._ptr(wav, torch.float64, n * self.wav_size),
                                            self._ptr(mask, torch.float64, self.wav_size),
                                            self._ptr(moments, torch.float64, n * (self.J + 1) * 6),
                                            self._stream(stream)))

    def reserve(self, nmaps, stream=None):
        """Sizes the split form's workspaces for batches of up to `nmaps`
        maps (call before capturing batches in a CUDA graph)."""
        check(lib().s2dwc_plan_reserve(self._h, int(nmaps), self._stream(stream)))

    def check(self):
        """Raises S2DWError if a split-form kernel gave up waiting since the
        last check (synchronises; the flag is cleared when reported)."""
        check(lib().s2dwc_plan_check(self._h))

    def set_split_min_batch(self, nmaps):
        """Split-form plans: batches of fewer than `nmaps` maps run the FP64
        path (default 1)."""
        check(lib().s2dwc_plan_set_split_min_batch(self._h, int(nmaps)))

    def set_priority(self, priority):
        """CUDA stream priority of the plan's per-scale streams (lower runs
        first); graphs captured afterwards keep it."""
        check(lib().s2dwc_plan_set_priority(self._h, int(priority)))

    def set_wait_limit(self, ns):
        """Bound in nanoseconds on every wait of the split-form kernels'
        pipeline (default 2e9)."""
        check(lib().s2dwc_plan_set_wait_limit(self._h, int(ns)))

    def synthesis(self, wav, scoeff, flm, stream=None):
        import torch

        check(lib().s2dwc_plan_synthesis(self._h, self._ptr(flm, torch.complex128, self.B * self.B),
                                         self._ptr(wav, torch.float64, self.wav_size),
                                         self._ptr(scoeff, torch.complex128, self.bl_scoeff ** 2),
                                         self._stream(stream)))
