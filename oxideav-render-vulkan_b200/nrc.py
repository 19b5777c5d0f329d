"""Neural radiance cache on a path tracer (include/oxpt_nrc.h).

`RadianceCache(tracer)` holds the network (BF16 tensor-core MLP, FP32
master weights, Adam) on the tracer's device. `refine(n)` renders n frames
of one sample per pixel into the tracer's accumulator: rendering paths end
into the cache after `query_bounce` bounces, one path in `train_one_in` is
traced to the end and trains the cache (one Adam step per frame). With
`enabled=False` the frames are the plain tracer's (the ablation and the
fallback). The tracer's sample count advances like its own refine.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _native as N
from .pathtracer import _raise


class RadianceCache:
    def __init__(self, tracer, seed: int = 1):
        self.tracer = tracer
        h = C.c_void_p()
        st = N.lib().oxpt_nrc_create(tracer.ctx, seed, C.byref(h))
        if st != N.OK:
            _raise(st, "cannot create the radiance cache")
        self._h = h.value
        self.cfg = N.NrcConfig()
        N.lib().oxpt_nrc_config_default(C.byref(self.cfg))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and N is not None:  # None while the interpreter shuts down
            N.lib().oxpt_nrc_destroy(h)
            self._h = None

    def _check(self, st):
        if st != N.OK:
            _raise(st, N.lib().oxpt_nrc_last_error(self._h).decode() or N.lib().oxpt_last_error(
                self.tracer.ctx).decode())

    def configure(self, **kw):
        for k, v in kw.items():
            setattr(self.cfg, k, float(v) if k == "spread" else int(v))

    def weights(self) -> np.ndarray:
        w = np.zeros(N.NRC_PARAMS, np.float32)
        self._check(N.lib().oxpt_nrc_get_weights(self._h, w.ctypes.data))
        return w

    def set_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        assert w.size == N.NRC_PARAMS
        self._check(N.lib().oxpt_nrc_set_weights(self._h, w.ctypes.data))

    def set_adam(self, lr=1e-2, beta1=0.9, beta2=0.99, eps=1e-8):
        self._check(N.lib().oxpt_nrc_set_adam(self._h, lr, beta1, beta2, eps))

    def refine(self, frames: int, loss: bool = False) -> Optional[float]:
        """`frames` cache frames on the tracer (bound to its scene and
        options); returns the last frame's training loss when asked."""
        t = self.tracer
        l = C.c_float()
        st = N.lib().oxpt_tracer_refine_nrc(t._h, self._h, frames, C.byref(self.cfg),
                                             C.byref(l) if loss else None)
        if st != N.OK:
            _raise(st, N.lib().oxpt_tracer_last_error(t._h).decode())
        return l.value if loss else None

    def refine_training(self, frames: int, loss: bool = False) -> Optional[float]:
        """`frames` frames whose every path is a training path that runs to
        its end: the frames are the plain tracer's (bit for bit) while the
        cache learns from all of them. Rendering the first frames this way
        keeps an untrained cache's predictions out of the average."""
        saved = (self.cfg.train_one_in, self.cfg.train_suffix)
        self.configure(train_one_in=1, train_suffix=0)
        try:
            return self.refine(frames, loss)
        finally:
            self.configure(train_one_in=saved[0], train_suffix=saved[1])

    def frame_counts(self):
        q, s = N.u32(), N.u32()
        self._check(N.lib().oxpt_nrc_frame_counts(self._h, C.byref(q), C.byref(s)))
        return int(q.value), int(s.value)
