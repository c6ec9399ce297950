"""Batched ensembles: many member models (uneven grids, mixed KL/ML/physics)
advanced together by the library's batched launches (wamgpu_batch_* in
include/wamgpu.h), optionally replayed from a captured CUDA graph."""
import ctypes

from ._lib import WamgpuError, load


class WamBatch:
    """Members are prepared WamModel objects of one precision on one device."""

    def __init__(self, models):
        self.L = load()
        self.models = list(models)
        arr = (ctypes.c_void_p * len(self.models))(*[m.h.value for m in self.models])
        h = ctypes.c_void_p()
        rc = self.L.wamgpu_batch_create(arr, len(self.models), ctypes.byref(h))
        self.h = h
        if rc != 0:
            msg = self.L.wamgpu_batch_last_error(h).decode() if h else "wamgpu_batch_create failed"
            if h:
                self.L.wamgpu_batch_destroy(h)
            self.h = None
            raise WamgpuError(f"wamgpu_batch_create: {msg} ({rc})")
        self._keep = {}

    def close(self):
        if getattr(self, "h", None):
            self.L.wamgpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != 0:
            raise WamgpuError(f"{what}: {self.L.wamgpu_batch_last_error(self.h).decode()} ({rc})")

    def set_member(self, g, fl3, scratch, u10, udir, tauw, ustar, z0, roairn, wstar, ld=None):
        """Device state of member g (torch CUDA tensors; fl3 and scratch shaped (ML, KL, ld))."""
        ld = fl3.shape[-1] if ld is None else ld
        self._keep[g] = (fl3, scratch, u10, udir, tauw, ustar, z0, roairn, wstar)
        rest = [t.data_ptr() for t in (scratch, u10, udir, tauw, ustar, z0, roairn, wstar)]
        self._check(self.L.wamgpu_batch_set_member(self.h, g, fl3.data_ptr(), ld, *rest), "batch_set_member")

    def tune(self, stream=None):
        """Autotune the CTA shapes; returns (sea points per IMPLSCH CTA, points per PROPAGS CTA)."""
        P, bs = ctypes.c_int(), ctypes.c_int()
        s = None if stream is None else ctypes.c_void_p(stream)
        self._check(self.L.wamgpu_batch_tune(self.h, s, ctypes.byref(P), ctypes.byref(bs)), "batch_tune")
        return P.value, bs.value

    def step(self, stream=None):
        """One pass for every member (replays the captured graph after capture())."""
        s = None if stream is None else ctypes.c_void_p(stream)
        self._check(self.L.wamgpu_batch_step(self.h, s), "batch_step")

    def capture(self, stream=None):
        s = None if stream is None else ctypes.c_void_p(stream)
        self._check(self.L.wamgpu_batch_capture(self.h, s), "batch_capture")

    def sync(self):
        self._check(self.L.wamgpu_batch_sync(self.h), "batch_sync")
