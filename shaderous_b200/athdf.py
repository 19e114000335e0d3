"""Snapshots of a run as Athena++ HDF5 files (.athdf), and runs restarted from them.

Restates the reference's snapshot path:
  - ``Snapshot`` and the block/variable conventions: src/io/snapshot.ts:8-112;
  - ``primitives_from``: primitivesFrom and pressureOf for the ideal gas (snapshot.ts:121-155);
  - ``write_athdf`` / ``read_athdf`` / ``open_athdf``: src/io/athdf.ts:112-407;
  - ``SnapshotSampler``: snapshot.ts:162-260;
  - ``capture`` and ``restart``: src/io/capture.ts:16-150 and restartFrom (:158-250), with the
    blocks' mesh rebuilt by the AMR entry point shz_amr_reset_mesh (amr_sim.ts:1867-1971).

The HDF5 container comes from :mod:`shaderous_b200.hdf5` (the format restated; the reference
uses the HDF5 library through h5wasm). Layout, attribute and dataset names, types and shapes are
the reference's:

  root attributes  NumCycles <i4, Time <f4, Coordinates S<len>, RootGridX1..3 <f4[3],
                   RootGridSize <i4[3], NumMeshBlocks <i4, MeshBlockSize <i4[3], MaxLevel <i4,
                   NumVariables <i4[1], DatasetNames S21[1], VariableNames S21[n], Shaderous (JSON)
  Levels           <i4 [blocks]
  LogicalLocations <i8 [blocks, 3]
  x1f..x3f         <f4 [blocks, n + 1];  x1v..x3v <f4 [blocks, n]
  prim             <f4 [variables, blocks, nz, ny, nx]

One difference in storage, invisible to readers: without compression ``prim`` is stored
contiguously (the reference always chunks it, to grow it one variable at a time).
"""
from __future__ import annotations

import json
import math
from dataclasses import dataclass, field

import numpy as np

from .hdf5 import H5Error, H5File, H5Writer

VARIABLES = ("rho", "press", "vel1", "vel2", "vel3", "r0")
SNAPSHOT_FORMAT = 2
BS = 16  # cells per block side on the adaptive grid


@dataclass
class Snapshot:
    """The gas as blocks of primitive variables (snapshot.ts:20-112).

    ``locations`` holds 3 ints per block (its position in blocks at its level); every array in
    ``data`` holds the blocks in order, each as [z][y][x] (float32, block_cells per block).
    """

    ndim: int
    root_size: list
    block_size: list
    lo: list
    hi: list
    time: float
    steps: int
    levels: np.ndarray
    locations: np.ndarray
    data: dict = field(default_factory=dict)
    meta: dict | None = None
    geometry: str | None = None  # 'cylindrical' | 'spherical' | None (Cartesian)
    x1rat: float | None = None


def block_cells(s: Snapshot) -> int:
    return int(s.block_size[0] * s.block_size[1] * s.block_size[2])


def block_count(s: Snapshot) -> int:
    return int(len(s.levels))


def max_level(s: Snapshot) -> int:
    return int(max((int(v) for v in s.levels), default=0))


def primitives_from(gamma: float, u1: np.ndarray, u2: np.ndarray, chunk: int = 1 << 22) -> dict:
    """Primitive variables from interleaved conserved state (snapshot.ts:121-137): the pressure
    from the ideal-gas equation of state on the stored internal energy, (gamma - 1) e_int
    (eos.ts:398-400), each value formed in float64 and stored as float32. The cells are taken
    `chunk` at a time, so the float64 work arrays stay small for a state of billions of cells."""
    chunk = int(chunk)
    if chunk < 1:
        raise ValueError(f"chunk must be at least 1 cell, got {chunk}")
    u1 = np.asarray(u1, np.float32).reshape(-1, 4)
    u2 = np.asarray(u2, np.float32).reshape(-1, 4)
    n = u1.shape[0]
    out = {k: np.empty(n, np.float32) for k in VARIABLES}
    for i in range(0, n, chunk):
        a = u1[i:i + chunk].astype(np.float64)
        b = u2[i:i + chunk].astype(np.float64)
        rho = a[:, 0]
        with np.errstate(divide="ignore", invalid="ignore"):
            out["rho"][i:i + chunk] = rho
            out["press"][i:i + chunk] = (gamma - 1) * b[:, 1]
            out["vel1"][i:i + chunk] = a[:, 1] / rho
            out["vel2"][i:i + chunk] = a[:, 2] / rho
            out["vel3"][i:i + chunk] = a[:, 3] / rho
            out["r0"][i:i + chunk] = b[:, 2] / rho
    return out


def _swap_axes23(s: Snapshot, to_file: bool) -> Snapshot:
    """An axisymmetric snapshot (x = R, y = z, v_z = v_phi) relabelled into Athena++'s cylindrical
    order (R, phi, z), one cell in phi spanning 2 pi, and back (athdf.ts:79-99)."""
    def at(v, phi):
        return [v[0], phi, v[1]] if to_file else [v[0], v[2], phi]

    loc = np.asarray(s.locations, np.int32).reshape(-1, 3)
    new = np.zeros_like(loc)
    if to_file:
        new[:, 0], new[:, 2] = loc[:, 0], loc[:, 1]
    else:
        new[:, 0], new[:, 1] = loc[:, 0], loc[:, 2]
    data = dict(s.data)
    data["vel2"], data["vel3"] = s.data.get("vel3"), s.data.get("vel2")
    return Snapshot(s.ndim, at(s.root_size, 1), at(s.block_size, 1), at(s.lo, 0), at(s.hi, 2 * math.pi if to_file else 0),
                    s.time, s.steps, s.levels, new, data, s.meta, s.geometry, s.x1rat)


# ---------------------------------------------------------------------------------------------
# Writing (athdf.ts:112-236)
# ---------------------------------------------------------------------------------------------

def write_athdf(s0: Snapshot, path=None, gzip: int = 0):
    """Write a snapshot as an .athdf file to ``path`` (a name or a binary file), or return its
    bytes. ``gzip``: deflate level 1-9 for the cell data, 0 for none (writeAthdf)."""
    cyl = s0.geometry == "cylindrical"
    s = _swap_axes23(s0, True) if cyl else s0
    nb = block_count(s)
    nx, ny, nz = (int(v) for v in s.block_size)
    present = [v for v in VARIABLES if s.data.get(v) is not None]
    present += [k for k in s.data if k not in VARIABLES and s.data[k] is not None]
    if not present:
        raise ValueError("a snapshot needs at least one variable")
    cells = block_cells(s)
    for k in present:
        if np.asarray(s.data[k]).size != nb * cells:
            raise ValueError(f"variable {k!r} holds {np.asarray(s.data[k]).size} values, not {nb} blocks of {cells}")
    levels = np.asarray(s.levels, np.int32)
    loc = np.asarray(s.locations, np.int64).reshape(nb, 3)

    w = H5Writer()
    w.attr("NumCycles", int(s.steps), "<i4")
    w.attr("Time", float(s.time), "<f4")
    sph = s0.geometry == "spherical"
    coords = "spherical_polar" if sph else "cylindrical" if cyl else "cartesian"
    w.attr("Coordinates", coords, f"S{len(coords)}")
    for a in range(3):
        rat = (s.x1rat or 1.0) if (a == 0 and sph) else 1.0
        w.attr(f"RootGridX{a + 1}", np.array([s.lo[a], s.hi[a], rat], np.float32))
    w.attr("RootGridSize", np.array(s.root_size, np.int32))
    w.attr("NumMeshBlocks", nb, "<i4")
    w.attr("MeshBlockSize", np.array(s.block_size, np.int32))
    w.attr("MaxLevel", max_level(s), "<i4")
    w.attr("NumVariables", np.array([len(present)], np.int32))
    w.attr("DatasetNames", ["prim"], "S21")
    w.attr("VariableNames", present, "S21")
    if s.meta is not None:
        w.attr("Shaderous", json.dumps(s.meta, separators=(",", ":"), ensure_ascii=False))

    w.dataset("Levels", levels)
    w.dataset("LogicalLocations", loc)
    for a in range(3):
        n = int(s.block_size[a])
        # float64 positions rounded once to float32, as the reference's Float32Array stores them
        dx = (s.hi[a] - s.lo[a]) / (np.int64(s.root_size[a]) << levels.astype(np.int64))
        x0 = s.lo[a] + loc[:, a] * n * dx
        i = np.arange(n + 1, dtype=np.float64)
        faces = x0[:, None] + i[None, :] * dx[:, None]
        centers = x0[:, None] + (i[None, :n] + 0.5) * dx[:, None]
        if sph and a < 2:
            rat = s.x1rat or 1.0

            def ff(b, k):
                if a == 1 or rat == 1:
                    return x0[b] + k * dx[b]
                return s.lo[0] * rat ** (int(loc[b, 0]) * n + k)

            for b in range(nb):
                for k in range(n + 1):
                    faces[b, k] = ff(b, k)
                for k in range(n):
                    l, h = ff(b, k), ff(b, k + 1)
                    centers[b, k] = (0.75 * (h ** 4 - l ** 4)) / (h ** 3 - l ** 3) if a == 0 else (
                        (math.sin(h) - h * math.cos(h) - math.sin(l) + l * math.cos(l)) / (math.cos(l) - math.cos(h)))
        w.dataset(f"x{a + 1}f", faces.astype(np.float32))
        w.dataset(f"x{a + 1}v", centers.astype(np.float32))

    prim = np.empty((len(present), nb, nz, ny, nx), np.float32)
    for v, k in enumerate(present):
        prim[v] = np.asarray(s.data[k], np.float32).reshape(nb, nz, ny, nx)
    if gzip:
        chunk_blocks = max(1, min(nb, (1 << 22) // cells))
        w.dataset("prim", prim, chunks=(1, chunk_blocks, nz, ny, nx), gzip=gzip)
    else:
        w.dataset("prim", prim)
    return w.write(path)


# ---------------------------------------------------------------------------------------------
# Reading (athdf.ts:238-407)
# ---------------------------------------------------------------------------------------------

class AthdfReader:
    """An .athdf file open for reading in parts (athdf.ts:264-297): its header as a snapshot
    without data, and any variable over a range of blocks."""

    def __init__(self, src):
        try:
            self._f = H5File(src)
        except H5Error as e:
            raise ValueError("this is not an HDF5 file") from e
        f = self._f
        try:
            self._open(f)
        except Exception:
            f.close()
            raise

    def _attr(self, key):
        if key not in self._f.attrs:
            raise ValueError(f'not an Athena++ HDF5 file: it has no "{key}" attribute')
        return self._f.attrs[key]

    def _numbers(self, key):
        v = self._attr(key)
        return [float(x) if isinstance(x, (float, np.floating)) else int(x) for x in np.atleast_1d(v)]

    def _strings(self, key):
        v = self._attr(key)
        items = v if isinstance(v, list) else [v]
        return [str(x).rstrip("\0").strip() for x in items]

    def _dataset(self, key):
        d = self._f.get(key)
        if d is None or not hasattr(d, "shape"):
            raise ValueError(f'not an Athena++ HDF5 file: it has no "{key}" dataset')
        return d

    def _open(self, f):
        coords = self._strings("Coordinates")[0].lower()
        root_size = [int(v) for v in self._numbers("RootGridSize")]
        cyl = coords == "cylindrical" and root_size[1] == 1
        if coords != "cartesian" and not cyl:
            raise ValueError("only Cartesian grids, and axisymmetric cylindrical ones, can be read "
                             f"(this file is {self._strings('Coordinates')[0]})")
        block_size = [int(v) for v in self._numbers("MeshBlockSize")]
        nb = int(self._numbers("NumMeshBlocks")[0])
        grid = [[float(x) for x in self._numbers(f"RootGridX{a}")] for a in (1, 2, 3)]
        if any(abs(g[2] - 1) > 1e-6 for g in grid):
            raise ValueError("only uniformly spaced grids can be read")
        levels = np.asarray(self._dataset("Levels").read(), np.int32).reshape(-1)
        locations = np.asarray(self._dataset("LogicalLocations").read()).astype(np.int32).reshape(-1)
        ndim = 3 if root_size[2] != 1 else 2 if root_size[1] != 1 else 1
        head = Snapshot(ndim, root_size, block_size, [g[0] for g in grid], [g[1] for g in grid],
                        float(self._numbers("Time")[0]), int(self._numbers("NumCycles")[0]) if "NumCycles" in f.attrs else 0,
                        levels, locations.reshape(-1, 3))
        if len(levels) != nb or len(locations) != 3 * nb:
            raise ValueError("the block tables do not match NumMeshBlocks")
        meta = f.attrs.get("Shaderous")
        if isinstance(meta, str):
            try:
                parsed = json.loads(meta)
                if isinstance(parsed, dict) and parsed.get("program") == "shaderous" and isinstance(parsed.get("query"), str):
                    head.meta = parsed
            except ValueError:
                pass  # not ours after all: read it as any other file
        names = self._strings("VariableNames")
        counts = [int(v) for v in self._numbers("NumVariables")]
        sets = self._strings("DatasetNames")
        cells = block_cells(head)
        where = {}
        first = 0
        for d, set_name in enumerate(sets):
            for v in range(counts[d] if d < len(counts) else 0):
                var = names[first + v] if first + v < len(names) else ""
                if not var or var in where:
                    continue
                ds = self._dataset(set_name)
                sh = ds.shape
                if len(sh) != 5 or sh[1] != nb or sh[2] * sh[3] * sh[4] != cells:
                    raise ValueError(f'"{set_name}" does not have the shape the header describes')
                where[var] = (ds, v)
            first += counts[d] if d < len(counts) else 0
        self._head, self._where, self._cyl = head, where, cyl
        self.blocks, self.cells = nb, cells
        self.variables = list(where.keys())

    def header(self) -> Snapshot:
        h = self._head
        return Snapshot(h.ndim, list(h.root_size), list(h.block_size), list(h.lo), list(h.hi), h.time, h.steps,
                        h.levels.copy(), h.locations.copy(), {}, h.meta)

    def read(self, name: str, b0: int, b1: int) -> np.ndarray:
        """Variable ``name`` for blocks b0 to b1 (exclusive), each block as [z][y][x]."""
        if name not in self._where:
            raise ValueError(f'the file has no variable "{name}"')
        ds, v = self._where[name]
        got = np.asarray(ds[v, b0:b1], np.float32).reshape(-1)
        if got.size != (b1 - b0) * self.cells:
            raise ValueError(f'"{name}" does not have the shape the header describes')
        return np.ascontiguousarray(got)

    def read_slab(self, name: str, block: int, z, y, x) -> np.ndarray:
        """Variable ``name`` in one block, cells [z0, z1) x [y0, y1) x [x0, x1), as [z][y][x]."""
        if name not in self._where:
            raise ValueError(f'the file has no variable "{name}"')
        ds, v = self._where[name]
        return np.ascontiguousarray(np.asarray(ds[v, block, z[0]:z[1], y[0]:y[1], x[0]:x[1]], np.float32).reshape(-1))

    def finish(self, s: Snapshot) -> Snapshot:
        """A snapshot read from this file in the program's axis order (a cylindrical file's)."""
        if not self._cyl:
            return s
        out = _swap_axes23(s, False)
        out.ndim, out.geometry = 2, "cylindrical"
        return out

    def close(self):
        self._f.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def open_athdf(src) -> AthdfReader:
    return AthdfReader(src)


def read_athdf(src) -> Snapshot:
    """The whole snapshot in a file (a path, or the file's bytes) (readAthdf)."""
    if isinstance(src, (bytes, bytearray, memoryview)):
        b = bytes(src[:8])
        if len(src) < 8 or b != b"\x89HDF\r\n\x1a\n":
            raise ValueError("this is not an HDF5 file")
    r = open_athdf(src)
    try:
        snap = r.header()
        for v in r.variables:
            snap.data[v] = r.read(v, 0, r.blocks)
        return r.finish(snap)
    finally:
        r.close()


# ---------------------------------------------------------------------------------------------
# Point lookup (snapshot.ts:162-260)
# ---------------------------------------------------------------------------------------------

class SnapshotSampler:
    """The cell of a snapshot that holds a position given as fractions of its box: the finest
    leaf whose block covers it. ``prim``/``level`` take one point; ``lookup`` takes arrays."""

    def __init__(self, snap: Snapshot):
        self.snap = snap
        self.top = max_level(snap)
        self.root_blocks = [int(snap.root_size[a] // snap.block_size[a]) for a in range(3)]
        self.cells = block_cells(snap)
        loc = np.asarray(snap.locations, np.int64).reshape(-1, 3)
        lv = np.asarray(snap.levels, np.int64)
        self._keys = self._key(lv, loc[:, 0], loc[:, 1], loc[:, 2])
        self._order = np.argsort(self._keys, kind="stable")
        self._sorted = self._keys[self._order]
        for v in ("rho", "press", "vel1", "vel2", "vel3"):
            if snap.data.get(v) is None:
                raise ValueError(f'the file has no "{v}" variable')

    @staticmethod
    def _key(level, i, j, k):
        return ((np.asarray(level, np.int64) * 4096 + k) * 4096 + j) * 4096 + i

    def lookup(self, fx, fy, fz):
        """(block, cell) index arrays for points given as fractions of the box, clamped into it; an
        axis of one cell is the same at every point along it."""
        s = self.snap

        def clamp(v):
            return np.minimum(np.maximum(np.asarray(v, np.float64), 0.0), 1 - 1e-7)

        f = [clamp(fx), np.zeros_like(clamp(fy)) if s.root_size[1] == 1 else clamp(fy),
             np.zeros_like(clamp(fz)) if s.root_size[2] == 1 else clamp(fz)]
        f = np.broadcast_arrays(*f)
        shape = f[0].shape
        f = [np.ravel(v) for v in f]
        block = np.full(f[0].shape, -1, np.int64)
        for l in range(self.top, -1, -1):
            todo = block < 0
            if not todo.any():
                break
            at = [np.minimum(np.floor(f[a][todo] * (self.root_blocks[a] << l)).astype(np.int64),
                             (self.root_blocks[a] << l) - 1) for a in range(3)]
            key = self._key(l, at[0], at[1], at[2])
            pos = np.searchsorted(self._sorted, key)
            pos = np.minimum(pos, len(self._sorted) - 1)
            hit = self._sorted[pos] == key
            idx = np.flatnonzero(todo)
            block[idx[hit]] = self._order[pos[hit]]
        if (block < 0).any():
            raise ValueError("the file does not cover the whole domain")
        lv = np.asarray(s.levels, np.int64)[block]
        loc = np.asarray(s.locations, np.int64).reshape(-1, 3)[block]
        cell = np.zeros(block.shape, np.int64)
        stride = 1
        for a in range(3):
            g = np.minimum(np.floor(f[a] * (np.int64(s.root_size[a]) << lv)).astype(np.int64), (np.int64(s.root_size[a]) << lv) - 1)
            local = g - loc[..., a] * s.block_size[a]
            cell += local * stride
            stride *= int(s.block_size[a])
        return block.reshape(shape), cell.reshape(shape)

    def prim(self, fx, fy, fz, species=None) -> dict:
        b, c = self.lookup(fx, fy, fz)
        o = int(b) * self.cells + int(c)
        d = self.snap.data
        w = {"rho": float(d["rho"][o]), "vx": float(d["vel1"][o]), "vy": float(d["vel2"][o]), "vz": float(d["vel3"][o]),
             "p": float(d["press"][o]), "s": float(d["r0"][o]) if d.get("r0") is not None else 0.0}
        if species and all(d.get(k) is not None for k in species):
            w["X"] = [float(d[k][o]) for k in species]
        return w

    def level(self, fx, fy, fz) -> int:
        return int(self.snap.levels[int(self.lookup(fx, fy, fz)[0])])

    def prims(self, fx, fy, fz) -> np.ndarray:
        """Float64 (rho, vx, vy, vz, p, s) at many points, shape (npoints, 6)."""
        b, c = self.lookup(fx, fy, fz)
        o = (b * self.cells + c).reshape(-1)
        d = self.snap.data
        cols = [d["rho"], d["vel1"], d["vel2"], d["vel3"], d["press"], d["r0"] if d.get("r0") is not None else None]
        out = np.zeros((o.size, 6), np.float64)
        for i, col in enumerate(cols):
            if col is not None:
                out[:, i] = np.asarray(col, np.float32)[o]
        return out


# ---------------------------------------------------------------------------------------------
# Runs: capture and restart (capture.ts)
# ---------------------------------------------------------------------------------------------

def _uniform_box(cfg):
    """lo, hi of a uniform grid: the box centred on 0, cells of dx; an axis of one cell spans
    the x side (the reference's box along a collapsed axis)."""
    n = [int(v) for v in (list(cfg.n) + [1, 1])[:3]]
    dx = cfg.dx if cfg.dx is not None else 1.0 / n[0]
    side = [(n[a] if n[a] > 1 else n[0]) * dx for a in range(3)]
    return [-s / 2 for s in side], [s / 2 for s in side]


def capture(sim, meta: dict | None = None) -> Snapshot:
    """The state of a run as blocks of primitive variables (capture.ts:16-150): a uniform grid is
    one block; on blocks, the leaves in the tree's order, each as [z][y][x]."""
    from .amr import AmrSim
    from .sim import Sim

    if isinstance(sim, AmrSim):
        c = sim.cfg
        _, levels, coords = sim.leaves()
        u1, u2 = sim.leaves_state()
        n0 = c.nr * BS
        flat = c.ndim < 3
        root_size = [n0, n0, 1 if flat else n0]
        block_size = [BS, BS, 1 if flat else BS]
        locations = np.asarray(coords, np.int32).reshape(-1, 3).copy()
        if flat:
            locations[:, 2] = 0
        lo, hi = [-c.box / 2] * 3, [c.box / 2] * 3
        gamma = c.hydro.gamma
        ndim = c.ndim
        t, _, steps = sim.clock()
    elif isinstance(sim, Sim):
        cfg = sim.cfg
        n = [int(v) for v in (list(cfg.n) + [1, 1])[:3]]
        root_size, block_size = n, list(n)
        levels = np.zeros(1, np.int32)
        locations = np.zeros((1, 3), np.int32)
        u1, u2 = sim.read_state()
        lo, hi = _uniform_box(cfg)
        gamma = cfg.gamma
        ndim = 3 if n[2] > 1 else 2 if n[1] > 1 else 1
        t, _, steps = sim.clock()
    else:
        raise TypeError("this kind of simulation cannot be exported")
    m = None
    if meta is not None:
        m = {"format": SNAPSHOT_FORMAT, **meta}
    return Snapshot(ndim, root_size, block_size, lo, hi, float(t), int(round(steps)), np.asarray(levels, np.int32),
                    locations, primitives_from(gamma, u1, u2), m)


def _fractions(snap: Snapshot, box_lo, box_hi, x, a):
    """restartFrom's frac (capture.ts:164-168): a position as a fraction of the file's own box."""
    flo = snap.lo[a] if snap.lo is not None else box_lo[a]
    side = (snap.hi[a] - flo) if snap.hi is not None else (box_hi[a] - box_lo[a])
    return (np.asarray(x, np.float64) - flo) / side


def restart(sim, snap: Snapshot) -> None:
    """Start ``sim`` from a snapshot (restartFrom, capture.ts:158-250): every cell of the run takes
    the primitives of the snapshot's cell that holds its centre (the run's grid may differ from the
    file's), turned into conserved state as the run's initial conditions are, and the clock takes
    the file's time and step count. On blocks the mesh is first rebuilt where the file is finer
    (shz_amr_reset_mesh)."""
    from .amr import AmrSim
    from .sim import Sim, prims_to_state

    if snap.geometry not in (None, "cartesian"):
        raise ValueError(f"a {snap.geometry} snapshot cannot start a Cartesian run")
    sampler = SnapshotSampler(snap)
    if isinstance(sim, AmrSim):
        c = sim.cfg
        n0 = c.nr * BS
        shift = int(round(math.log2(snap.root_size[0] / n0)))
        sim.reset_mesh(snap.levels, np.asarray(snap.locations).reshape(-1, 3), snap.root_size, snap.block_size,
                       snap.lo, snap.hi, shift)
        _, levels, coords = sim.leaves()
        nd = c.ndim
        dx0 = c.box / n0
        half = c.box / 2
        t = np.arange(BS ** nd)
        i, j = t % BS, (t // BS) % BS
        k = t // (BS * BS) if nd == 3 else np.zeros_like(t)
        dx = dx0 / (2.0 ** np.asarray(levels, np.float64))[:, None]
        co = np.asarray(coords, np.int64)
        x = ((co[:, 0:1] * BS + i[None, :]) + 0.5) * dx - half
        y = ((co[:, 1:2] * BS + j[None, :]) + 0.5) * dx - half
        z = ((co[:, 2:3] * BS + k[None, :]) + 0.5) * dx - half if nd == 3 else np.zeros_like(x)
        box = ([-half] * 3, [half] * 3)
        w = sampler.prims(_fractions(snap, *box, x, 0), _fractions(snap, *box, y, 1), _fractions(snap, *box, z, 2))
        u1, u2 = prims_to_state(w, c.hydro.gamma)
        sim.set_leaves_state(u1, u2)
        sim.set_clock(float(snap.time), int(snap.steps))
        return
    if isinstance(sim, Sim):
        cfg = sim.cfg
        n = [int(v) for v in (list(cfg.n) + [1, 1])[:3]]
        dx = cfg.dx if cfg.dx is not None else 1.0 / n[0]
        box = _uniform_box(cfg)
        gx = (np.arange(n[0]) + 0.5 - n[0] / 2.0) * dx
        gy = (np.arange(n[1]) + 0.5 - n[1] / 2.0) * dx
        gz = (np.arange(n[2]) + 0.5 - n[2] / 2.0) * dx
        fx = _fractions(snap, *box, gx, 0)[None, None, :]
        fy = _fractions(snap, *box, gy, 1)[None, :, None]
        fz = _fractions(snap, *box, gz, 2)[:, None, None]
        w = sampler.prims(fx, fy, fz)
        u1, u2 = prims_to_state(w, cfg.gamma)
        sim.set_state(u1, u2)
        sim.set_clock(float(snap.time), int(snap.steps))
        return
    raise TypeError("this kind of simulation cannot be restarted")
