"""Athena++ HDF5 snapshots (.athdf) on the CPU: the reference's own checks of the format
(tests/unit/athdf.test.ts) restated, and the HDF5 layer pinned to a file written by the HDF5
library itself (scipy's test file testhdf5_7.4_GLNX86.mat, an HDF5 file behind a 512-byte user
block, holding the 9 x 1 float64 dataset "testdouble" = k pi / 4 with a MATLAB_class attribute)."""
import math
import os
import struct

import numpy as np
import pytest

from shaderous_b200 import hdf5 as H
from shaderous_b200.athdf import (VARIABLES, Snapshot, SnapshotSampler, open_athdf, read_athdf, write_athdf)


def library_file():
    import scipy

    p = os.path.join(os.path.dirname(scipy.__file__), "io", "matlab", "tests", "data", "testhdf5_7.4_GLNX86.mat")
    if not os.path.exists(p):
        pytest.skip("the HDF5 library's test file is not in this image")
    return p


def sample() -> Snapshot:
    """Two root blocks along x; the second refined once in the plane (a 2D mesh, 4-cell blocks)."""
    blocks = [[0, 0, 0, 0], [1, 2, 0, 0], [1, 3, 0, 0], [1, 2, 1, 0], [1, 3, 1, 0]]
    cells = 16
    data = {v: (q * 1000 + np.arange(len(blocks) * cells) + 0.25).astype(np.float32) for q, v in enumerate(VARIABLES)}
    return Snapshot(2, [8, 4, 1], [4, 4, 1], [-1, -0.5, -0.5], [1, 0.5, 0.5], 1.5, 42,
                    np.array([b[0] for b in blocks], np.int32), np.array([b[1:] for b in blocks], np.int32), data,
                    {"program": "shaderous", "build": "test", "query": "problem=sedov&dim=2&n=128",
                     "perturber": {"pos": [1, 2, 3], "vel": [4, 5, 6]}})


# -- the reference's athdf.test.ts --------------------------------------------------------------

def test_round_trips_blocks_variables_grid_and_settings():
    s = sample()
    back = read_athdf(write_athdf(s))
    assert back.ndim == 2
    assert back.root_size == s.root_size and back.block_size == s.block_size
    assert back.lo == s.lo and back.hi == s.hi
    assert (back.time, back.steps) == (1.5, 42)
    assert back.levels.tolist() == s.levels.tolist()
    assert back.locations.tolist() == s.locations.tolist()
    for v in VARIABLES:
        assert np.array_equal(back.data[v], s.data[v])
    assert back.meta == s.meta


def test_axisymmetric_run_as_cylindrical_and_back():
    data = {v: (q * 1000 + np.arange(4 * 16) + 0.25).astype(np.float32) for q, v in enumerate(VARIABLES)}
    s = Snapshot(2, [8, 8, 1], [4, 4, 1], [0, -0.5, -0.5], [1, 0.5, 0.5], 1, 3, np.zeros(4, np.int32),
                 np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0]], np.int32), data, geometry="cylindrical")
    raw = write_athdf(s)
    f = H.H5File(raw)
    assert f.attrs["Coordinates"] == "cylindrical"
    assert f.attrs["RootGridSize"].tolist() == [8, 1, 8]
    back = read_athdf(raw)
    assert back.geometry == "cylindrical"
    assert [back.ndim, back.root_size, back.block_size, back.lo[:2], back.hi[:2]] == [2, [8, 8, 1], [4, 4, 1], [0, -0.5], [1, 0.5]]
    assert back.locations.tolist() == s.locations.tolist()
    for v in VARIABLES:
        assert np.array_equal(back.data[v], s.data[v])


def test_round_trips_species_as_variables_named_after_them():
    s = sample()
    n = len(s.levels) * 16
    s.data["he4"] = (np.arange(n) / n).astype(np.float32)
    s.data["c12"] = (1 - np.arange(n) / n).astype(np.float32)
    raw = write_athdf(s)
    back = read_athdf(raw)
    assert np.array_equal(back.data["he4"], s.data["he4"])
    assert np.array_equal(back.data["c12"], s.data["c12"])
    sampler = SnapshotSampler(back)
    # root block, cell (1, 2) is cell 9 of block 0
    assert sampler.prim(0.1875, 0.625, 0, ["c12", "he4"])["X"] == [float(back.data["c12"][9]), float(back.data["he4"][9])]
    # a species the file lacks: none of them are read
    assert "X" not in sampler.prim(0.1875, 0.625, 0, ["c12", "o16"])
    assert H.H5File(raw).attrs["VariableNames"] == [*VARIABLES, "he4", "c12"]


def test_writes_the_layout_other_tools_expect():
    f = H.H5File(write_athdf(sample()))
    assert f["prim"].shape == (6, 5, 1, 4, 4)
    assert f["x1f"].shape == (5, 5)
    assert f["LogicalLocations"].shape == (5, 3)
    assert f["LogicalLocations"].dtype == np.dtype("<i8") and f["Levels"].dtype == np.dtype("<i4")
    assert f.attrs["DatasetNames"] == ["prim"]
    assert f.attrs["VariableNames"] == list(VARIABLES)
    assert f.attrs["NumVariables"].tolist() == [6]
    assert f.attrs["NumMeshBlocks"] == 5 and f.attrs["MaxLevel"] == 1
    assert f.attrs["Time"].dtype == np.float32 and f.attrs["NumCycles"] == 42
    # the refined block at (2, 0) starts at x = 0 and its cells are 0.125 wide
    assert f["x1f"].read()[1].tolist() == [0, 0.125, 0.25, 0.375, 0.5]
    assert f["x1v"].read()[1].tolist() == [0.0625, 0.1875, 0.3125, 0.4375]


def test_spherical_run_as_spherical_polar_with_logarithmic_radial_faces():
    data = {v: np.ones(2 * 16, np.float32) for v in VARIABLES}
    rat = math.exp(math.log(8) / 8)
    s = Snapshot(2, [8, 4, 1], [4, 4, 1], [1, 0, 0], [8, math.pi, 2 * math.pi], 0, 0, np.zeros(2, np.int32),
                 np.array([[0, 0, 0], [1, 0, 0]], np.int32), data, geometry="spherical", x1rat=rat)
    f = H.H5File(write_athdf(s))
    assert f.attrs["Coordinates"] == "spherical_polar"
    assert f.attrs["RootGridX1"].tolist() == np.float32([1, 8, rat]).tolist()
    x1f = f["x1f"].read().reshape(-1)
    # the second block's faces go on from the first's: r = rat^4 to rat^8 = 8
    assert x1f[5] == pytest.approx(rat ** 4, abs=5e-6)
    assert x1f[9] == pytest.approx(8, abs=5e-6)
    assert f["x2f"].read().reshape(-1)[4] == pytest.approx(math.pi, abs=5e-7)
    with pytest.raises(ValueError, match="only Cartesian grids"):
        read_athdf(write_athdf(s))


def test_samples_the_finest_block_that_covers_a_point():
    s = SnapshotSampler(sample())
    assert s.level(0.1, 0.5, 0.5) == 0
    assert s.level(0.9, 0.9, 0.5) == 1
    # root block, cell (1, 2): fractions 0.5 * (1.5 / 4), (2.5 / 4)
    assert s.prim(0.1875, 0.625, 0)["rho"] == 2 * 4 + 1 + 0.25
    # refined block 3 at (2, 1): its cell (0, 0) sits at fractions (0.5 + 1/32, 0.5 + 1/16)
    assert s.prim(0.5 + 1 / 32, 0.5 + 1 / 16, 0)["rho"] == 3 * 16 + 0.25


def test_reads_back_compressed_files_which_are_smaller():
    s = sample()
    for v in VARIABLES:
        s.data[v][16:] = 1.5  # mostly uniform, as a quiet region of a run would be
    plain = write_athdf(s)
    packed = write_athdf(s, gzip=1)
    assert len(packed) < len(plain)
    back = read_athdf(packed)
    for v in VARIABLES:
        assert np.array_equal(back.data[v], s.data[v])


def test_rejects_files_that_are_not_snapshots():
    with pytest.raises(ValueError, match="not an HDF5 file"):
        read_athdf(bytes([1, 2, 3, 4]))
    with pytest.raises(ValueError, match='it has no "Coordinates" attribute'):
        read_athdf(library_file())


# -- beyond the reference's tests ---------------------------------------------------------------

def test_reader_reads_a_file_the_hdf5_library_wrote():
    f = H.H5File(library_file())
    assert f.keys() == ["testdouble"]
    d = f["testdouble"]
    assert d.shape == (9, 1) and d.dtype == np.float64
    assert d.attrs == {"MATLAB_class": "double"}
    assert np.array_equal(d.read()[:, 0], np.pi / 4 * np.arange(9))


def test_writer_encodes_as_the_hdf5_library_does():
    """The writer's datatype, dataspace, attribute and symbol-table encodings equal the library's
    for the same objects (the library null-terminates strings where this writer null-pads them:
    both are HDF5's, and readers take either)."""
    f = H.H5File(library_file())
    msgs = {mt: d for mt, d, _ in f._messages(f._root["testdouble"])}
    assert msgs[0x0003][:20] == H._datatype(np.float64)
    assert msgs[0x0001] == H._dataspace((9, 1))
    w = H.H5Writer()
    w.attr("MATLAB_class", "double", "S6")
    ours = w.attrs[0][1][8:]  # the message body, after its 8-byte header
    lib = msgs[0x000C]
    assert len(ours) == len(lib)
    k = 8 + 16 + 1  # the string type's first bit-field byte: padding type and character set
    assert ours[:k] == lib[:k] and ours[k + 1:] == lib[k + 1:]
    assert (ours[k] & 0xF0, lib[k] & 0x0F, ours[k] & 0x0F) == (lib[k] & 0xF0, 0, 1)
    # the root group: a symbol-table message, a v1 B-tree of symbol-table nodes over a local heap
    ours_file = H.H5File(write_athdf(sample()))
    root = {mt: d for mt, d, _ in ours_file._messages(ours_file._root_addr)}
    assert set(root) == {0x0011, 0x000C}
    lib_root = {mt: d for mt, d, _ in f._messages(f._root_addr)}
    assert len(root[0x0011]) == len(lib_root[0x0011]) == 16


def test_writer_structures_many_objects_and_chunks():
    """More datasets than one symbol-table node holds and more chunks than one B-tree node holds."""
    rng = np.random.default_rng(7)
    w = H.H5Writer()
    arrays = {f"set{i:02d}": rng.random((i + 1, 3)).astype(np.float64) for i in range(20)}
    for k, a in arrays.items():
        w.dataset(k, a)
    big = rng.random((9, 70, 6)).astype(np.float32)
    w.dataset("chunked", big, chunks=(1, 4, 6), gzip=3)  # 9 x 18 = 162 chunks
    w.dataset("ints", np.arange(-5, 5, dtype=np.int16))
    raw = w.write()
    f = H.H5File(raw)
    assert sorted(f.keys()) == sorted([*arrays, "chunked", "ints"])
    for k, a in arrays.items():
        assert np.array_equal(f[k].read(), a)
    assert np.array_equal(f["chunked"].read(), big)
    assert np.array_equal(f["chunked"][3, 10:20], big[3, 10:20])
    assert np.array_equal(f["ints"].read(), np.arange(-5, 5, dtype=np.int16))
    # the superblock: version 1 (a chunk-index K of 81 to hold 162 chunks in one node), 8-byte
    # offsets and lengths, the end-of-file address = the size
    assert raw[:8] == H.SIGNATURE and raw[8] == 1 and raw[13:15] == b"\x08\x08"
    assert struct.unpack_from("<H", raw, 24)[0] == 81
    assert struct.unpack_from("<Q", raw, 44)[0] == len(raw)
    # more chunks than the largest node holds: a B-tree of two levels
    w2 = H.H5Writer()
    many = rng.random((3 * H.MAX_CHUNK_K,)).astype(np.float32)
    w2.dataset("many", many, chunks=(1,), gzip=1)
    f2 = H.H5File(w2.write())
    assert np.array_equal(f2["many"].read(), many)
    # no chunked data: a version 0 superblock
    w3 = H.H5Writer()
    w3.dataset("a", np.arange(3.0))
    assert w3.write()[8] == 0


def test_file_round_trip_through_a_path(tmp_path):
    s = sample()
    p = tmp_path / "snap.athdf"
    assert write_athdf(s, p) is None
    back = read_athdf(str(p))
    for v in VARIABLES:
        assert np.array_equal(back.data[v], s.data[v])
    with open_athdf(str(p)) as r:
        assert r.variables == list(VARIABLES)
        assert np.array_equal(r.read("press", 1, 3), s.data["press"][16:48])
        # block 0, cells z 0, y [1, 3), x [2, 4)
        assert r.read_slab("rho", 0, [0, 1], [1, 3], [2, 4]).tolist() == [6.25, 7.25, 10.25, 11.25]


def test_primitives_in_chunks_equal_the_whole():
    """The primitives of a state taken a chunk of cells at a time are those formed all at once, and
    each is the float32 rounding of the float64 value (snapshot.ts primitivesFrom)."""
    from shaderous_b200.athdf import primitives_from

    rng = np.random.default_rng(3)
    n = 10007
    u1 = np.column_stack([rng.uniform(0.1, 3, n), rng.normal(size=(n, 3))]).astype(np.float32)
    u2 = np.column_stack([rng.uniform(1, 5, n), rng.uniform(0.5, 2, n), rng.uniform(0, 1, n), np.zeros(n)]).astype(np.float32)
    whole = primitives_from(1.4, u1, u2, chunk=n)
    parts = primitives_from(1.4, u1, u2, chunk=1000)
    for k in VARIABLES:
        assert parts[k].dtype == np.float32 and np.array_equal(parts[k], whole[k])
    rho = u1[:, 0].astype(np.float64)
    assert np.array_equal(whole["vel2"], (u1[:, 2].astype(np.float64) / rho).astype(np.float32))
    assert np.array_equal(whole["press"], (0.4 * u2[:, 1].astype(np.float64)).astype(np.float32))
