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

import copy
import ctypes as C
import itertools

import numpy as np

from . import _native as N


class BlockView:
    """One block seen as a small uniform mesh (for initial conditions): its
    interior cells, or with `ghosts` layers of ghost cells around them (the
    cells setup_problem fills, at their own unwrapped coordinates)."""

    def __init__(self, amr, level, cx, cy, cz, ghosts=0):
        self.ndims = amr.ndims
        self.nc = amr.nc
        self.dx, self.dy, self.dz = amr.level_dx(level)
        self.x0 = amr.xmin + (cx * self.nc - ghosts) * self.dx
        self.y0 = amr.ymin + (cy * self.nc - ghosts) * self.dy
        self.z0 = amr.zmin + (cz * self.nc - ghosts) * self.dz if self.ndims == 3 else 0.0
        n = self.n = self.nc + 2 * ghosts
        self.shape = (n if self.ndims == 3 else 1, n, n)

    def cell_centres(self):
        n = self.n
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
        self.minlev = int(geo.get("minlev", 1))
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

    # ---- mesh update ------------------------------------------------------------
    def _offsets(self):
        offs = [o for o in itertools.product((-1, 0, 1), repeat=3) if any(o)]
        return [o for o in offs if o[2] == 0] if self.ndims == 2 else offs

    def _touching(self, level, x, y, z, o):
        """Leaves inside the subdivided position (level, x, y, z) that touch
        the block it neighbours in direction -o."""
        ex, ey, ez = self.extent(level + 1)
        subs = [(0,) if d == 1 else ((1,) if d == -1 else (0, 1)) for d in o]
        if self.ndims == 2:
            subs[2] = (0,)
        out = set()
        for c in subs[2]:
            for b in subs[1]:
                for a in subs[0]:
                    key = (level + 1, (2 * x + a) % ex, (2 * y + b) % ey, (2 * z + c) % ez)
                    if key in self.leaves:
                        out.add(key)
                    elif level + 1 < self.maxlev:
                        out |= self._touching(level + 1, key[1], key[2], key[3], o)
        return out

    def neighbours(self, leaf):
        """Leaves touching `leaf` across a face, an edge or a corner (the
        faces / edges / corners pointers of src/blocks.F90:4369-4463)."""
        l, cx, cy, cz = leaf
        out = set()
        for o in self._offsets():
            c = self.cover(l, cx + o[0], cy + o[1], cz + o[2])
            if c is not None:
                out.add(c)
            else:
                ex, ey, ez = self.extent(l)
                out |= self._touching(l, (cx + o[0]) % ex, (cy + o[1]) % ey, (cz + o[2]) % ez, o)
        out.discard(leaf)
        return out

    def neighbour_lists(self):
        """For every leaf in block-index order, the block indices of the
        leaves touching it across faces, edges and corners, ascending (the
        same sets as neighbours(), looked up for all leaves at once: the
        same level, the coarser level, or the finer leaves next to it, as a
        2:1 balanced mesh has them)."""
        order = self.order
        nb = len(order)
        t = np.array(order, dtype=np.int64).reshape(nb, 4)
        lev = t[:, 0]
        maxl = int(lev.max())
        ext = np.stack([np.array(self.extent(l)) for l in range(1, maxl + 2)])

        def enc(l, x, y, z):
            return ((l * 65536 + x) * 65536 + y) * 65536 + z

        keys = enc(lev, t[:, 1], t[:, 2], t[:, 3])
        srt = np.argsort(keys)
        skeys = keys[srt]

        def look(k):
            pos = np.minimum(np.searchsorted(skeys, k), nb - 1)
            return np.where(skeys[pos] == k, srt[pos], -1)

        found = [[] for _ in range(nb)]
        rows, cols = [], []
        for o in self._offsets():
            e = ext[lev - 1]
            p = [(t[:, 1 + a] + o[a]) % e[:, a] for a in range(3)]
            hit = look(enc(lev, p[0], p[1], p[2]))
            miss = hit < 0
            coarse = np.where(miss & (lev > 1), look(enc(lev - 1, p[0] // 2, p[1] // 2, p[2] // 2)), -1)
            rows.append(np.nonzero(hit >= 0)[0]); cols.append(hit[hit >= 0])
            rows.append(np.nonzero(coarse >= 0)[0]); cols.append(coarse[coarse >= 0])
            fine = miss & (coarse < 0)
            if fine.any():
                subs = [(0,) if d == 1 else ((1,) if d == -1 else (0, 1)) for d in o]
                if self.ndims == 2:
                    subs[2] = (0,)
                idx = np.nonzero(fine)[0]
                for c in subs[2]:
                    for b in subs[1]:
                        for a in subs[0]:
                            f = look(enc(lev[idx] + 1, 2 * p[0][idx] + a, 2 * p[1][idx] + b, 2 * p[2][idx] + c))
                            for r in idx[f < 0]:  # deeper than one level: the general search
                                found[r].extend(self.neighbours(order[r]))
                            rows.append(idx[f >= 0]); cols.append(f[f >= 0])
        index = {tt: b for b, tt in enumerate(order)}
        for r in range(nb):
            for x in found[r]:
                rows.append(np.array([r]))
                cols.append(np.array([index[x]]))
        rows = np.concatenate(rows).astype(np.int64)
        cols = np.concatenate(cols).astype(np.int64)
        pair = np.unique(rows * nb + cols)  # sorted by leaf, then neighbour
        r, c = pair // nb, pair % nb
        keep = r != c
        r, c = r[keep], c[keep]
        cut = np.searchsorted(r, np.arange(nb + 1))
        cl = c.tolist()
        return [cl[cut[b]:cut[b + 1]] for b in range(nb)]

    def is_balanced(self) -> bool:
        """Neighbours across faces, edges and corners differ by at most one level."""
        return all(abs(n[0] - t[0]) <= 1 for t in self.leaves for n in self.neighbours(t))

    def update_plan(self, criterion):
        """The mesh after update_mesh (src/mesh.F90:756-821) for the per-block
        criterion (-1 derefine, 0 keep, 1 refine, block-index order) and, per
        new block, where its data comes from: (new AMRMesh, src (n, 9) int32)
        with rows {0, old} kept, {1, parent, px + 2 py + 4 pz} prolonged and
        {2, children by position} restricted.

        The flags follow check_data_block_refinement (src/mesh.F90:1455-1680:
        the minlev / maxlev clamps), update_neighbor_refinement (1694-1748
        with reset_neighbors_refinement, src/blocks.F90:4297-4352, from the
        finest level down) and prepare_sibling_derefinement (1768-2055: a
        parent derefines only when all its children are leaves flagged -1).
        Within a level the leaves are visited in block-index order."""
        order = self.order
        index = {t: b for b, t in enumerate(order)}
        crit = np.asarray(criterion).reshape(-1)
        if len(crit) != len(order):
            raise ValueError("one criterion per block")
        ref = {}
        for t, c in zip(order, crit):
            r, l = int(c), t[0]
            if l < self.minlev:
                r = 1
            if l == self.minlev:
                r = max(0, r)
            if l == self.maxlev:
                r = min(0, r)
            if l > self.maxlev:
                r = -1
            ref[t] = r
        nbrs = self.neighbour_lists()
        by_level = {}
        for t in order:
            by_level.setdefault(t[0], []).append(t)
        for l in range(self.maxlev, 0, -1):
            for t in by_level.get(l, []):
                for n in (order[k] for k in nbrs[index[t]]):
                    if ref[t] == 1:
                        ref[n] = max(0, ref[n])
                        if n[0] < l:
                            ref[n] = 1
                    elif ref[t] == 0:
                        if n[0] < l:
                            ref[n] = max(0, ref[n])
                    else:
                        if n[0] < l:
                            ref[n] = max(0, ref[n])
                        if ref[n] == 1:
                            ref[t] = 0
        derefine = set()
        for l in range(2, self.maxlev + 1):
            for t in order:
                if t[0] != l or ref[t] != -1:
                    continue
                parent = (l - 1, t[1] // 2, t[2] // 2, t[3] // 2)
                sibs = self._children(parent)
                if all(ref.get(s) == -1 for s in sibs):
                    derefine.add(parent)
                else:
                    for s in sibs:
                        if s in ref:
                            ref[s] = max(0, ref[s])
        new = set(self.leaves)
        for parent in derefine:
            new.difference_update(self._children(parent))
            new.add(parent)
        for t in order:
            if ref[t] == 1 and t[0] < self.maxlev and t in new:
                new.discard(t)
                new.update(self._children(t))
        mesh = copy.copy(self)
        mesh.leaves = new
        src = np.zeros((len(new), 9), dtype=np.int32)
        for b, t in enumerate(mesh.order):
            if t in index:
                src[b, :2] = (0, index[t])
            elif t in derefine:
                src[b, 0] = 2
                for c, ch in enumerate(self._children(t)):
                    src[b, 1 + c] = index[ch]
            else:
                l, cx, cy, cz = t
                src[b, :3] = (1, index[(l - 1, cx // 2, cy // 2, cz // 2)], (cx & 1) + 2 * (cy & 1) + 4 * (cz & 1))
        return mesh, src

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
        """The block descriptors of the leaves in block-index order: level,
        cell size, position, and the same-level neighbour across every face,
        edge and corner (-1 where the neighbour is at another level; z
        neighbours -1 in 2D).  Vectorised: the neighbour keys of all leaves
        are looked up at once in the sorted leaf keys."""
        order = self.order
        nb = len(order)
        t = np.array(order, dtype=np.int64).reshape(nb, 4)
        lev = t[:, 0]
        ext = np.stack([np.array(self.extent(int(l))) for l in range(1, int(lev.max()) + 1)])[lev - 1]

        def enc(l, x, y, z):
            return ((l * 65536 + x) * 65536 + y) * 65536 + z

        keys = enc(lev, t[:, 1], t[:, 2], t[:, 3])
        srt = np.argsort(keys)
        skeys = keys[srt]
        nbr = np.full((nb, 27), -1, dtype=np.int32)
        for oz in (-1, 0, 1):
            if self.ndims == 2 and oz != 0:
                continue
            for oy in (-1, 0, 1):
                for ox in (-1, 0, 1):
                    n = (ox + 1) + 3 * (oy + 1) + 9 * (oz + 1)
                    k = enc(lev, (t[:, 1] + ox) % ext[:, 0], (t[:, 2] + oy) % ext[:, 1], (t[:, 3] + oz) % ext[:, 2])
                    pos = np.minimum(np.searchsorted(skeys, k), nb - 1)
                    hit = skeys[pos] == k
                    nbr[:, n] = np.where(hit, srt[pos], -1)
        D = N.amun_block_desc
        dt = np.dtype({"names": ["level", "dx", "neighbor", "coord"],
                       "formats": [np.int32, (np.float64, 3), (np.int32, 27), (np.int32, 3)],
                       "offsets": [D.level.offset, D.dx.offset, D.neighbor.offset, D.coord.offset],
                       "itemsize": C.sizeof(D)})
        arr = (D * nb)()
        view = np.frombuffer(arr, dtype=dt)
        view["level"] = lev
        dxs = np.array([self.level_dx(l) for l in range(1, int(lev.max()) + 1)])
        view["dx"] = dxs[lev - 1]
        view["neighbor"] = nbr
        view["coord"] = t[:, 1:]
        return arr

    def view(self, b, ghosts=False):
        l, cx, cy, cz = self.order[b]
        return BlockView(self, l, cx, cy, cz, self.ng if ghosts else 0)

    def blocks_from(self, fn, nv, ghosts=False, only=None):
        """Block arrays (nblocks, km, jm, im, nv) whose interiors are fn(view)
        ((nz, ny, nx, nv) of each block); ghost entries are zero, or with
        `ghosts` fn of the whole padded block.  With `only` (one flag per
        block) the other blocks stay zero."""
        out = np.zeros((self.nblocks, self.km, self.jm, self.im, nv))
        ng, nc = self.ng, self.nc
        for b in range(self.nblocks):
            if only is not None and not only[b]:
                continue
            q = fn(self.view(b, ghosts))
            if ghosts:
                out[b] = q
            elif self.ndims == 3:
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
