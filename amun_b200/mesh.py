"""Uniform single-level block mesh on the host.

Describes the leaf blocks of a periodic domain refined uniformly to one
level, like the reference's base block array (src/domains.F90:136-360,
periodic neighbours by cshift) refined to ``maxlev`` everywhere
(minlev == maxlev).  Blocks are numbered b = bx + nbx (by + nby bz).

Arrays:
  global field      (NZ, NY, NX, nv)          C order == Fortran (nv,NX,NY,NZ)
  block arrays      (nb, km, jm, im, nv)      C order == Fortran (nv,im,jm,km)
                                               per block, back to back
"""
from __future__ import annotations

import numpy as np

from . import _native as N


class UniformMesh:
    def __init__(self, geo: dict):
        self.ndims = int(geo["ndims"])
        self.nc = int(geo["ncells"])
        self.ng = int(geo["nghosts"])
        lev = int(geo["maxlev"])
        ff = 2 ** (lev - 1)
        self.level = lev
        self.nbx = int(geo["xblocks"]) * ff
        self.nby = int(geo["yblocks"]) * ff
        self.nbz = int(geo["zblocks"]) * ff if self.ndims == 3 else 1
        # adx(l) = xlen / (ir * ni), src/coordinates.F90:339-345
        self.dx = (geo["xmax"] - geo["xmin"]) / (int(geo["xblocks"]) * (self.nc * ff))
        self.dy = (geo["ymax"] - geo["ymin"]) / (int(geo["yblocks"]) * (self.nc * ff))
        self.dz = ((geo["zmax"] - geo["zmin"]) / (int(geo["zblocks"]) * (self.nc * ff))
                   if self.ndims == 3 else 1.0)
        self.xmin, self.ymin, self.zmin = geo["xmin"], geo["ymin"], geo["zmin"]
        self.im = self.nc + 2 * self.ng
        self.jm = self.im
        self.km = self.im if self.ndims == 3 else 1
        self.nblocks = self.nbx * self.nby * self.nbz
        self.shape = (self.nbz * (self.nc if self.ndims == 3 else 1), self.nby * self.nc, self.nbx * self.nc)

    @property
    def ncells_total(self) -> int:
        return int(np.prod(self.shape))

    def block_coords(self, b: int):
        bx = b % self.nbx
        by = (b // self.nbx) % self.nby
        bz = b // (self.nbx * self.nby)
        return bx, by, bz

    def descriptors(self):
        arr = (N.amun_block_desc * self.nblocks)()
        for b in range(self.nblocks):
            bx, by, bz = self.block_coords(b)
            d = arr[b]
            d.level = self.level
            d.dx[0], d.dx[1], d.dx[2] = self.dx, self.dy, self.dz
            d.coord[0], d.coord[1], d.coord[2] = bx, by, bz
            for oz in (-1, 0, 1):
                for oy in (-1, 0, 1):
                    for ox in (-1, 0, 1):
                        n = (ox + 1) + 3 * (oy + 1) + 9 * (oz + 1)
                        if self.ndims == 2 and oz != 0:
                            d.neighbor[n] = -1
                            continue
                        nx = (bx + ox) % self.nbx
                        ny = (by + oy) % self.nby
                        nz = (bz + oz) % self.nbz
                        d.neighbor[n] = nx + self.nbx * (ny + self.nby * nz)
        return arr

    def cell_centres(self):
        """Global cell-centre coordinates (x, y, z) of the interior cells:
        block xmin + ((i - ng) - 1/2) dx (src/coordinates.F90:351-356)."""
        NZ, NY, NX = self.shape
        x = self.xmin + (np.arange(NX) + 0.5) * self.dx
        y = self.ymin + (np.arange(NY) + 0.5) * self.dy
        z = self.zmin + (np.arange(NZ) + 0.5) * self.dz if self.ndims == 3 else np.zeros(1)
        return x, y, z

    def to_blocks(self, field: np.ndarray) -> np.ndarray:
        """Global interior field -> block arrays with periodic ghost cells."""
        nv = field.shape[-1]
        ng, nc = self.ng, self.nc
        if self.ndims == 3:
            padded = np.pad(field, ((ng, ng), (ng, ng), (ng, ng), (0, 0)), mode="wrap")
        else:
            padded = np.pad(field, ((0, 0), (ng, ng), (ng, ng), (0, 0)), mode="wrap")
        out = np.empty((self.nblocks, self.km, self.jm, self.im, nv))
        for b in range(self.nblocks):
            bx, by, bz = self.block_coords(b)
            if self.ndims == 3:
                out[b] = padded[bz * nc:bz * nc + self.km, by * nc:by * nc + self.jm, bx * nc:bx * nc + self.im]
            else:
                out[b] = padded[:, by * nc:by * nc + self.jm, bx * nc:bx * nc + self.im]
        return out

    def to_blocks_torch(self, field):
        """to_blocks for a torch tensor, on the tensor's device."""
        import torch
        ng, nc = self.ng, self.nc
        if self.ndims == 3:
            idx = [torch.arange(-ng, n + ng, device=field.device) % n for n in field.shape[:3]]
            padded = field[idx[0]][:, idx[1]][:, :, idx[2]]
        else:
            iy = torch.arange(-ng, field.shape[1] + ng, device=field.device) % field.shape[1]
            ix = torch.arange(-ng, field.shape[2] + ng, device=field.device) % field.shape[2]
            padded = field[:, iy][:, :, ix]
        blocks = []
        for b in range(self.nblocks):
            bx, by, bz = self.block_coords(b)
            if self.ndims == 3:
                blocks.append(padded[bz * nc:bz * nc + self.km, by * nc:by * nc + self.jm, bx * nc:bx * nc + self.im])
            else:
                blocks.append(padded[:, by * nc:by * nc + self.jm, bx * nc:bx * nc + self.im])
        return torch.stack(blocks).contiguous()

    def from_blocks_torch(self, blocks):
        """from_blocks for a torch tensor, on the tensor's device."""
        import torch
        ng, nc = self.ng, self.nc
        out = torch.empty(self.shape + (blocks.shape[-1],), dtype=blocks.dtype, device=blocks.device)
        for b in range(self.nblocks):
            bx, by, bz = self.block_coords(b)
            if self.ndims == 3:
                out[bz * nc:(bz + 1) * nc, by * nc:(by + 1) * nc, bx * nc:(bx + 1) * nc] = \
                    blocks[b, ng:ng + nc, ng:ng + nc, ng:ng + nc]
            else:
                out[:, by * nc:(by + 1) * nc, bx * nc:(bx + 1) * nc] = blocks[b, :, ng:ng + nc, ng:ng + nc]
        return out

    def from_blocks(self, blocks: np.ndarray) -> np.ndarray:
        """Block arrays -> global interior field."""
        nv = blocks.shape[-1]
        ng, nc = self.ng, self.nc
        out = np.empty(self.shape + (nv,))
        for b in range(self.nblocks):
            bx, by, bz = self.block_coords(b)
            if self.ndims == 3:
                out[bz * nc:(bz + 1) * nc, by * nc:(by + 1) * nc, bx * nc:(bx + 1) * nc] = \
                    blocks[b, ng:ng + nc, ng:ng + nc, ng:ng + nc]
            else:
                out[:, by * nc:(by + 1) * nc, bx * nc:(bx + 1) * nc] = blocks[b, :, ng:ng + nc, ng:ng + nc]
        return out
