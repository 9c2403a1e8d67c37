"""Grid (Grid.pyx:17-159) for one GPU holding the whole domain."""
from __future__ import annotations

import numpy as np

from ._capi import PbDims


class Grid:
    """Uniform grid, periodic in x and y.  ``dims`` is the C struct passed to
    every kernel; it has the layout of the reference's DimStruct.  Like the
    reference's single-rank case, nl == n and indx_lo == 0."""

    def __init__(self, namelist, Parallel=None):
        gn = namelist["grid"]
        d = PbDims()
        d.dims = int(gn.get("dims", 3))
        for i, key in enumerate(("dx", "dy", "dz")):
            d.dx[i] = float(gn[key])
            d.dxi[i] = 1.0 / d.dx[i]
        d.gw = int(gn["gw"])
        for i, key in enumerate(("nx", "ny", "nz")):
            d.n[i] = int(gn[key])
            d.ng[i] = d.n[i] + 2 * d.gw
            d.nl[i] = d.n[i]
            d.nlg[i] = d.nl[i] + 2 * d.gw
            d.indx_lo[i] = 0
            d.indx_lo_g[i] = 0
        d.npd = max(d.n[0], 1) * max(d.n[1], 1) * max(d.n[2], 1)
        d.npl = d.nl[0] * d.nl[1] * d.nl[2]
        d.npg = d.nlg[0] * d.nlg[1] * d.nlg[2]
        nlg = d.nlg
        d.nbuffer[0] = d.gw * max(nlg[1] * nlg[2], nlg[1], nlg[2])
        d.nbuffer[1] = d.gw * max(nlg[0] * nlg[2], nlg[0], nlg[2])
        d.nbuffer[2] = d.gw * max(nlg[0] * nlg[1], nlg[0], nlg[1])
        d.ghosted_stride[0] = max(nlg[1] * nlg[2], nlg[1], nlg[2])
        d.ghosted_stride[1] = max(1, nlg[0])
        d.ghosted_stride[2] = 1
        self.dims = d
        self.compute_coordinates()

    def compute_coordinates(self):
        """Grid.compute_coordinates (Grid.pyx:125-159)."""
        d = self.dims
        out = {}
        for ax, name in enumerate(("x", "y", "z")):
            idx = np.arange(-d.gw, d.n[ax] + d.gw, dtype=np.float64)
            out[name] = (idx + 1) * d.dx[ax]
            out[name + "_half"] = (idx + 0.5) * d.dx[ax]
        self.x, self.x_half = out["x"], out["x_half"]
        self.y, self.y_half = out["y"], out["y_half"]
        self.z, self.z_half = out["z"], out["z_half"]
        # Grid.pyx:162-163: zl_half is extracted from zl, not from z_half, so on
        # one rank it holds the face heights (z); the wall-adjusted and ILES
        # Smagorinsky length scales read it
        self.zl = self.z.copy()
        self.zl_half = self.zl.copy()

    # convenience --------------------------------------------------------
    @property
    def shape(self):
        return tuple(self.dims.nlg)

    @property
    def npg(self):
        return self.dims.npg

    @property
    def npl(self):
        return self.dims.npl

    def interior(self):
        g = self.dims.gw
        n = self.dims.nlg
        return (slice(g, n[0] - g), slice(g, n[1] - g), slice(g, n[2] - g))
