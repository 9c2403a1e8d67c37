"""Horizontal statistics on the GPU: the reductions ParallelMPI provides to
the statistics output (ParallelMPI.pyx:196-540), under the reference's
method names, returning device tensors of nlg2 values (a float for
HorizontalMeanSurface).  Writing the statistics files is not part of this
library; a caller copies the profiles it writes to the host.
"""
from __future__ import annotations

import ctypes

import torch

from . import _capi


class HorizontalStatistics:
    def __init__(self, Gr):
        self.Gr = Gr
        self._ws = None

    def _run(self, kind, v1, v2=None, v3=None, mask=None, stream=None):
        Gr = self.Gr
        L = _capi.load()
        dev = v1.device
        n = int(L.pb_stat_workspace_bytes(ctypes.byref(Gr.dims)))
        if self._ws is None or self._ws.numel() < n or self._ws.device != dev:
            self._ws = torch.empty(n, dtype=torch.uint8, device=dev)
        out = torch.empty(Gr.dims.nlg[2] if kind != _capi.PB_STAT_MEAN_SURFACE else 1, dtype=torch.float64,
                          device=dev)
        rc = L.pb_horizontal_stat(ctypes.byref(Gr.dims), kind, _capi.ptr(v1), _capi.ptr(v2), _capi.ptr(v3),
                                  _capi.ptr(mask), _capi.ptr(out), _capi.ptr(self._ws), n,
                                  _capi.stream_handle(stream))
        _capi.check(rc, "pb_horizontal_stat")
        return out

    def HorizontalMean(self, Gr, values, stream=None):
        return self._run(_capi.PB_STAT_MEAN, values, stream=stream)

    def HorizontalMeanofSquares(self, Gr, values1, values2, stream=None):
        return self._run(_capi.PB_STAT_MEAN_SQUARES, values1, values2, stream=stream)

    def HorizontalMeanofCubes(self, Gr, values1, values2, values3, stream=None):
        return self._run(_capi.PB_STAT_MEAN_CUBES, values1, values2, values3, stream=stream)

    def HorizontalMaximum(self, Gr, values, stream=None):
        return self._run(_capi.PB_STAT_MAX, values, stream=stream)

    def HorizontalMinimum(self, Gr, values, stream=None):
        return self._run(_capi.PB_STAT_MIN, values, stream=stream)

    def HorizontalMeanSurface(self, Gr, values, stream=None):
        return float(self._run(_capi.PB_STAT_MEAN_SURFACE, values, stream=stream)[0])

    def HorizontalMeanConditional(self, Gr, values, mask, stream=None):
        return self._run(_capi.PB_STAT_MEAN_CONDITIONAL, values, mask=mask, stream=stream)

    def HorizontalMeanofSquaresConditional(self, Gr, values1, values2, mask, stream=None):
        return self._run(_capi.PB_STAT_MEAN_SQUARES_CONDITIONAL, values1, values2, mask=mask, stream=stream)
