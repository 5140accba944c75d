"""Block mesh with refinement levels on the host.

The leaves of a 2:1 balanced block tree on a periodic domain, as the
reference's meta tree holds them (src/blocks.F90:109-228, refined by
src/mesh.F90:436-756): level 1 is the base grid of xblocks x yblocks
(x zblocks) blocks; a block at level l has the same number of cells as any
other and half the size of its parent.  A leaf is (level, cx, cy, cz), its
position at its level in blocks, zero based.

The library receives the leaves as block descriptors (level, cell size,
position) and derives every ghost-cell relation itself; neighbours across
a face, edge or corner differ by at most one level.
"""
from __future__ import annotations

import itertools

import numpy as np

from . import _native as N


class BlockView:
    """One block seen as a small uniform mesh (for initial conditions)."""

    def __init__(self, amr, level, cx, cy, cz):
        self.ndims = amr.ndims
        self.nc = amr.nc
        self.dx, self.dy, self.dz = amr.level_dx(level)
        self.x0 = amr.xmin + cx * self.nc * self.dx
        self.y0 = amr.ymin + cy * self.nc * self.dy
        self.z0 = amr.zmin + cz * self.nc * self.dz if self.ndims == 3 else 0.0
        n = self.nc
        self.shape = (n if self.ndims == 3 else 1, n, n)

    def cell_centres(self):
        n = self.nc
        x = self.x0 + (np.arange(n) + 0.5) * self.dx
        y = self.y0 + (np.arange(n) + 0.5) * self.dy
        z = self.z0 + (np.arange(n) + 0.5) * self.dz if self.ndims == 3 else np.zeros(1)
        return x, y, z


class AMRMesh:
    def __init__(self, geo: dict):
        self.ndims = int(geo["ndims"])
        self.nc = int(geo["ncells"])
        self.ng = int(geo["nghosts"])
        self.base = (int(geo["xblocks"]), int(geo["yblocks"]), int(geo["zblocks"]) if self.ndims == 3 else 1)
        self.xmin, self.ymin, self.zmin = geo["xmin"], geo["ymin"], geo.get("zmin", 0.0)
        self.xlen = geo["xmax"] - geo["xmin"]
        self.ylen = geo["ymax"] - geo["ymin"]
        self.zlen = geo["zmax"] - geo["zmin"] if self.ndims == 3 else 1.0
        self.maxlev = int(geo["maxlev"])
        self.im = self.nc + 2 * self.ng
        self.jm = self.im
        self.km = self.im if self.ndims == 3 else 1
        nbx, nby, nbz = self.base
        self.leaves = {(1, x, y, z) for x in range(nbx) for y in range(nby) for z in range(nbz)}

    # ---- geometry ---------------------------------------------------------------
    def level_dx(self, level):
        f = 2 ** (level - 1)
        dx = self.xlen / (self.base[0] * self.nc * f)
        dy = self.ylen / (self.base[1] * self.nc * f)
        dz = self.zlen / (self.base[2] * self.nc * f) if self.ndims == 3 else 1.0
        return dx, dy, dz

    def extent(self, level):
        """Blocks per direction at `level`."""
        f = 2 ** (level - 1)
        return (self.base[0] * f, self.base[1] * f, self.base[2] * f if self.ndims == 3 else 1)

    def box(self, leaf):
        """(lower corner, upper corner) of a leaf."""
        l, cx, cy, cz = leaf
        dx, dy, dz = self.level_dx(l)
        lo = np.array([self.xmin + cx * self.nc * dx, self.ymin + cy * self.nc * dy,
                       self.zmin + cz * self.nc * dz if self.ndims == 3 else 0.0])
        hi = lo + np.array([self.nc * dx, self.nc * dy, self.nc * dz if self.ndims == 3 else 0.0])
        return lo, hi

    # ---- refinement -------------------------------------------------------------
    def _children(self, leaf):
        l, cx, cy, cz = leaf
        zs = (0, 1) if self.ndims == 3 else (0,)
        return [(l + 1, 2 * cx + a, 2 * cy + b, 2 * cz + c) for c in zs for b in (0, 1) for a in (0, 1)]

    def refine(self, leaf):
        self.leaves.discard(leaf)
        self.leaves.update(self._children(leaf))

    def cover(self, level, x, y, z):
        """The leaf covering block position (x, y, z) of `level` (periodic),
        or None when that position is subdivided further."""
        ex, ey, ez = self.extent(level)
        x, y, z = x % ex, y % ey, z % ez
        for m in range(level, 0, -1):
            s = level - m
            key = (m, x >> s, y >> s, z >> s)
            if key in self.leaves:
                return key
        return None

    def balance(self):
        """Refine until neighbours across faces, edges and corners differ by at
        most one level (the reference's 2:1 rule, src/mesh.F90)."""
        offs = [o for o in itertools.product((-1, 0, 1), repeat=3) if any(o)]
        if self.ndims == 2:
            offs = [o for o in offs if o[2] == 0]
        while True:
            marked = set()
            for leaf in self.leaves:
                l, cx, cy, cz = leaf
                for ox, oy, oz in offs:
                    c = self.cover(l, cx + ox, cy + oy, cz + oz)
                    if c is not None and c[0] < l - 1:
                        marked.add(c)
            if not marked:
                return
            for c in marked:
                if c in self.leaves:
                    self.refine(c)

    def refine_where(self, pred):
        """Refine every leaf below maxlev for which pred(lower, upper, level)
        holds, level by level, keeping the mesh balanced."""
        for level in range(1, self.maxlev):
            for leaf in sorted(x for x in self.leaves if x[0] == level):
                lo, hi = self.box(leaf)
                if pred(lo, hi, level):
                    self.refine(leaf)
            self.balance()

    # ---- blocks -----------------------------------------------------------------
    @property
    def order(self):
        """Leaves in block-index order: by level, then z, y, x."""
        return sorted(self.leaves, key=lambda t: (t[0], t[3], t[2], t[1]))

    @property
    def nblocks(self) -> int:
        return len(self.leaves)

    @property
    def ncells_total(self) -> int:
        return self.nblocks * self.nc ** self.ndims

    def levels(self):
        return np.array([t[0] for t in self.order], dtype=np.int32)

    def coords(self):
        return np.array([t[1:] for t in self.order], dtype=np.int32)

    def descriptors(self):
        order = self.order
        index = {t: b for b, t in enumerate(order)}
        arr = (N.amun_block_desc * len(order))()
        for b, (l, cx, cy, cz) in enumerate(order):
            d = arr[b]
            d.level = l
            d.dx[0], d.dx[1], d.dx[2] = self.level_dx(l)
            d.coord[0], d.coord[1], d.coord[2] = cx, cy, cz
            ex, ey, ez = self.extent(l)
            for oz in (-1, 0, 1):
                for oy in (-1, 0, 1):
                    for ox in (-1, 0, 1):
                        n = (ox + 1) + 3 * (oy + 1) + 9 * (oz + 1)
                        if self.ndims == 2 and oz != 0:
                            d.neighbor[n] = -1
                            continue
                        key = (l, (cx + ox) % ex, (cy + oy) % ey, (cz + oz) % ez)
                        d.neighbor[n] = index.get(key, -1)
        return arr

    def view(self, b):
        l, cx, cy, cz = self.order[b]
        return BlockView(self, l, cx, cy, cz)

    def blocks_from(self, fn, nv):
        """Block arrays (nblocks, km, jm, im, nv) whose interiors are fn(view)
        ((nz, ny, nx, nv) of each block); ghost entries are zero."""
        out = np.zeros((self.nblocks, self.km, self.jm, self.im, nv))
        ng, nc = self.ng, self.nc
        for b in range(self.nblocks):
            q = fn(self.view(b))
            if self.ndims == 3:
                out[b, ng:ng + nc, ng:ng + nc, ng:ng + nc] = q
            else:
                out[b, 0, ng:ng + nc, ng:ng + nc] = q[0]
        return out

    def interior(self, blocks):
        """Interior cells of block arrays: (nblocks, nz, ny, nx, nv)."""
        ng, nc = self.ng, self.nc
        if self.ndims == 3:
            return blocks[:, ng:ng + nc, ng:ng + nc, ng:ng + nc]
        return blocks[:, :, ng:ng + nc, ng:ng + nc]

    def cell_volumes(self):
        """Cell volume of every block (nblocks,)."""
        return np.array([np.prod(self.level_dx(t[0])[:self.ndims]) for t in self.order])
