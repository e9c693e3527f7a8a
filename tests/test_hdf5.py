"""manapy's HDF5 mesh directories without h5py (``manapy_b200.hdf5``).

The reader follows the HDF5 file format specification for the subset manapy's
partitioner writes.  It is pinned on a file written by the HDF5 library itself (a
MATLAB v7.3 file from scipy's test data, when present: superblock 0 behind a 512-byte
user block, version-1 object headers, a symbol-table group, a contiguous dataset) and
on round trips through this module's writer, which writes the datasets manapy's
partitioner writes (``manapy/partitions/meshpartitioning.py:238-275``).
"""
import os

import numpy as np
import pytest

import manapy_b200 as M
from manapy_b200 import hdf5, meshgen


def test_reads_a_file_written_by_the_hdf5_library():
    import scipy
    p = os.path.join(os.path.dirname(scipy.__file__), "io", "matlab", "tests", "data", "testhdf5_7.4_GLNX86.mat")
    if not os.path.exists(p):
        pytest.skip("scipy's HDF5 test file is not installed")
    f = hdf5.H5File(p)
    assert f.base == 512 and f.names() == ["testdouble"]
    a = f.read("testdouble")
    assert a.dtype == np.float64 and a.shape == (9, 1)
    assert np.array_equal(a.ravel(), np.arange(9) * (np.pi / 4))      # MATLAB's 0:pi/4:2*pi


def test_round_trip_of_integer_and_float_datasets(tmp_path):
    rng = np.random.default_rng(0)
    data = {"elements": rng.integers(0, 99, (25, 4)).astype(np.int32), "nodes": rng.random((13, 4)),
            "neigh1": np.array([1, 3], np.int32), "empty": np.zeros((0, 2), np.int32),
            **{"d%02d" % k: np.arange(k + 2, dtype=np.int64) for k in range(10)}}   # 14 links: two SNODs
    p = str(tmp_path / "m.hdf5")
    hdf5.write_datasets(p, data)
    got = hdf5.read_datasets(p)
    assert sorted(got) == sorted(data)
    for k, a in data.items():
        assert got[k].dtype == a.dtype and np.array_equal(got[k], a), k


def _write_partitioned(mesh_dir, el, vx, nparts, seed=3):
    """Rank files with manapy's datasets: elements with global node ids, nodes =
    vertices[localnodetoglobal], localcelltoglobal / localnodetoglobal maps."""
    os.makedirs(mesh_dir)
    owner = np.random.default_rng(seed).integers(0, nparts, len(el))
    k = int(el[0, -1])
    for r in range(nparts):
        cells = np.nonzero(owner == r)[0].astype(np.int32)
        nodes = np.unique(el[cells, :k]).astype(np.int32)
        hdf5.write_datasets(os.path.join(mesh_dir, "mesh%d.hdf5" % r), {
            "elements": el[cells], "nodes": vx[nodes], "nparts": np.zeros((len(nodes), 3), np.int32),
            "centvol": np.zeros((2, 2)), "localnodetoglobal": nodes, "localcelltoglobal": cells,
            "neigh1": np.zeros(0, np.int32), "neigh2": np.zeros(0, np.int32),
            "halosext": np.zeros((2, 2), np.int32), "halosint": np.zeros(2, np.int32),
            **({"GtoL": np.arange(len(el), dtype=np.int32)} if r == 0 else {})})


def test_single_and_partitioned_mesh_directories_give_the_same_domain(tmp_path):
    el, vx = meshgen.square_triangles(9, seed=4)
    one = str(tmp_path / "meshes1PROC")
    os.makedirs(one)
    hdf5.write_datasets(os.path.join(one, "mesh0.hdf5"), {"elements": el, "nodes": vx})
    four = str(tmp_path / "meshes4PROC")
    _write_partitioned(four, el, vx, 4)
    for d in (one, four):
        e2, v2 = hdf5.read_mesh_dir(d)
        assert np.array_equal(e2, el) and np.array_equal(v2, vx)
    a = M.Domain.from_hdf5(four, 2).host_arrays
    b = M.Domain(dim=2, mesh=(el, vx)).host_arrays
    for key in ("faces_cellid", "faces_name", "cells_volume", "faces_normal"):
        assert np.array_equal(a[key], b[key]), key


def test_unsupported_features_are_named(tmp_path):
    p = str(tmp_path / "x.hdf5")
    hdf5.write_datasets(p, {"a": np.arange(3.0)})
    raw = bytearray(open(p, "rb").read())
    raw[8] = 7                                   # an unknown superblock version
    open(p, "wb").write(bytes(raw))
    with pytest.raises(NotImplementedError):
        hdf5.H5File(p)
    with pytest.raises(ValueError):
        open(str(tmp_path / "y.hdf5"), "wb").write(b"not hdf5 at all")
        hdf5.H5File(str(tmp_path / "y.hdf5"))
