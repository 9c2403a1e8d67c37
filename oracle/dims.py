"""Single-rank grid geometry for the oracle (test infrastructure).

Follows Grid.pyx:17-159 with one MPI rank: nl = n, indx_lo = 0,
nlg = n + 2 gw, uniform spacing.  ``DimStructC`` is the ctypes mirror of
``struct DimStruct`` (Csrc/grid.h:2-24) used to call the reference C.
"""
from __future__ import annotations

import ctypes

import numpy as np

_L3 = ctypes.c_long * 3
_D3 = ctypes.c_double * 3


class DimStructC(ctypes.Structure):
    _fields_ = [
        ("dims", ctypes.c_long),
        ("n", _L3), ("ng", _L3), ("nl", _L3), ("nlg", _L3),
        ("npd", ctypes.c_long), ("npl", ctypes.c_long), ("npg", ctypes.c_long),
        ("gw", ctypes.c_long),
        ("indx_lo", _L3), ("indx_lo_g", _L3),
        ("nbuffer", _L3), ("ghosted_stride", _L3),
        ("dx", _D3), ("dxi", _D3),
    ]


class Dims:
    """Geometry of one rank holding the whole domain (Grid.pyx:17-123)."""

    def __init__(self, n, gw, dx):
        self.n = tuple(int(v) for v in n)
        self.gw = int(gw)
        self.dx = tuple(float(v) for v in dx)
        self.dxi = tuple(1.0 / v for v in self.dx)
        self.nl = self.n
        self.nlg = tuple(v + 2 * self.gw for v in self.n)
        self.ng = self.nlg
        self.npl = self.n[0] * self.n[1] * self.n[2]
        self.npg = self.nlg[0] * self.nlg[1] * self.nlg[2]
        self.shape = self.nlg
        # Grid.compute_coordinates (Grid.pyx:125-159)
        idx = np.arange(-self.gw, self.n[2] + self.gw, dtype=np.float64)
        self.z = (idx + 1) * self.dx[2]
        self.z_half = (idx + 0.5) * self.dx[2]

    def c(self) -> DimStructC:
        d = DimStructC()
        d.dims = 3
        nlg = self.nlg
        for i in range(3):
            d.n[i] = self.n[i]
            d.ng[i] = self.ng[i]
            d.nl[i] = self.nl[i]
            d.nlg[i] = nlg[i]
            d.indx_lo[i] = 0
            d.indx_lo_g[i] = 0
            d.dx[i] = self.dx[i]
            d.dxi[i] = self.dxi[i]
        d.npd = self.npl
        d.npl = self.npl
        d.npg = self.npg
        d.gw = self.gw
        d.nbuffer[0] = self.gw * max(nlg[1] * nlg[2], nlg[1], nlg[2])
        d.nbuffer[1] = self.gw * max(nlg[0] * nlg[2], nlg[0], nlg[2])
        d.nbuffer[2] = self.gw * max(nlg[0] * nlg[1], nlg[0], nlg[1])
        d.ghosted_stride[0] = max(nlg[1] * nlg[2], nlg[1], nlg[2])
        d.ghosted_stride[1] = max(1, nlg[0])
        d.ghosted_stride[2] = 1
        return d

    def interior(self):
        g = self.gw
        return (slice(g, self.nlg[0] - g), slice(g, self.nlg[1] - g), slice(g, self.nlg[2] - g))
