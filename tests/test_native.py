"""The native host builder (C++) reproduces the Python builder's device tables bit for bit."""
import numpy as np
import pytest

from manapy_b200 import boundary as B, device as D, geometry as G, meshgen
from manapy_b200.serving import SIDES


@pytest.mark.parametrize("n,seed,reorder", [(7, 0, True), (23, 5, True), (16, 2, False), (40, 9, True)])
def test_tables_match_the_python_builder(n, seed, reorder):
    el, vx = meshgen.square_triangles(n, seed=seed)
    ref = D.DeviceMesh(G.build(el, vx, 2), device=None, reorder=reorder)
    nat = D.DeviceMesh.from_native(el, vx, reorder=reorder)
    assert sorted(ref.t) == sorted(nat.t)
    for k, v in ref.t.items():
        assert v.dtype == nat.t[k].dtype and v.shape == nat.t[k].shape, k
        assert v.tobytes() == nat.t[k].tobytes(), k
    for kind in ("cell", "face", "node"):
        assert np.array_equal(ref.perm[kind], nat.perm[kind])
        assert np.array_equal(ref.inv[kind], nat.inv[kind])
    # boundary rules from the native builder's manapy-numbered arrays
    A = G.build(el, vx, 2)
    bc = {s: "dirichlet" for s in SIDES}
    vals = {s: 1.5 for s in SIDES}
    b_ref = D.DeviceBC(A, B.resolve(A, bc, vals), device=None, mesh=ref)
    b_nat = D.DeviceBC(nat.A, B.resolve(nat.A, bc, vals), device=None, mesh=nat)
    for a in ("kind", "value", "face_grad_on"):
        assert np.array_equal(getattr(b_ref, a), getattr(b_nat, a)), a


def test_rejects_unmatched_boundary_faces():
    el, vx = meshgen.square_triangles(4, seed=1)
    vx = vx.copy()
    vx[:, 3] = 0  # no boundary tags at all
    with pytest.raises(ValueError, match="match no boundary side"):
        D.DeviceMesh.from_native(el, vx)


@pytest.mark.parametrize("n,seed", [(7, 1), (33, 5), (200, 4)])   # 200: 80,000 cells, threaded union
def test_native_full_geometry_is_bit_identical(n, seed):
    """With full=True the native builder also returns every geometry.build array (what a
    Domain exposes): same keys, dtypes, shapes and bits (signs of zeros included)."""
    import numpy as np
    from manapy_b200 import geometry as G, meshgen
    from manapy_b200.device import DeviceMesh
    el, vx = meshgen.square_triangles(n, seed=seed)
    A = G.build(el, vx, 2)
    B = DeviceMesh.from_native(el, vx, full=True).A
    assert set(A) == set(B)
    for k, a in A.items():
        b = B[k]
        if isinstance(a, (int, np.integer)):
            assert int(a) == int(b), k
            continue
        assert a.dtype == b.dtype and a.shape == b.shape, k
        assert np.array_equal(a, b), k
        if a.dtype.kind == "f":
            assert np.array_equal(np.signbit(a), np.signbit(b)), k


def test_domain_uses_the_native_builder_for_triangles():
    import manapy_b200 as M
    from manapy_b200 import geometry as G, meshgen
    el, vx = meshgen.square_triangles(9, seed=2)
    dom = M.Domain(dim=2, mesh=(el, vx))
    assert dom._host_dm is not None                     # tables built natively, uploaded on first use
    A = G.build(el, vx, 2)
    assert all(np.array_equal(np.asarray(dom.host_arrays[k]), np.asarray(A[k])) for k in A)


@pytest.mark.parametrize("n,seed", [(2, 1), (6, 7), (24, 2)])   # 24: 82,944 cells, threaded union
def test_native_3d_geometry_is_bit_identical(n, seed):
    """host/geom3d.cpp: every geometry.build array of a tetrahedral mesh, bit for bit."""
    from manapy_b200 import native
    el, vx = meshgen.cube_tetrahedra(n, seed=seed)
    A = G.build(el, vx, 3)
    B = native.geometry3d(el, vx)
    assert set(A) == set(B)
    for k, a in A.items():
        b = B[k]
        if isinstance(a, (int, np.integer)):
            assert int(a) == int(b), k
            continue
        assert a.dtype == b.dtype and a.shape == b.shape, k
        assert np.array_equal(a, b), k
        if a.dtype.kind == "f":
            assert np.array_equal(np.signbit(a), np.signbit(b)), k


@pytest.mark.filterwarnings("ignore::RuntimeWarning")
def test_native_3d_rejects_untagged_boundaries_like_the_python_builder():
    import manapy_b200 as M
    from manapy_b200 import native
    el, vx = meshgen.cube_tetrahedra(2, seed=1)
    vx = vx.copy()
    vx[:, 3] = 0                                    # no boundary tags at all
    with pytest.raises(ValueError):
        native.geometry3d(el, vx)
    with pytest.raises(ValueError, match="match no boundary side"):
        M.Domain(dim=3, mesh=(el, vx))


def test_native_builder_writes_either_stencil_layout():
    """The builder's slot-shared stencil equals the layout ``lsq_sell`` forms from its own
    vertex-neighbour tables; every other table does not depend on the layout."""
    from manapy_b200 import native
    el, vx = meshgen.square_triangles(60, seed=8)
    a = native.tables2d(el, vx, stencil="shared")
    b = native.tables2d(el, vx)
    gp, gi = D.lsq_sell(b["cellnid_ptr"], b["cellnid_idx"], "shared")
    assert np.array_equal(a["lsq_sell_ptr"], gp) and np.array_equal(a["lsq_sell_idx"], gi)
    mp, mi = D.lsq_sell(b["cellnid_ptr"], b["cellnid_idx"], "manapy")
    assert np.array_equal(b["lsq_sell_ptr"], mp) and np.array_equal(b["lsq_sell_idx"], mi)
    for k in a:
        if not k.startswith("lsq_sell"):
            assert np.array_equal(a[k], b[k]), k
    with pytest.raises(ValueError):
        native.tables2d(el, vx, stencil="sorted")


def test_native_builder_threads_do_not_change_the_tables(monkeypatch):
    """Every threaded path of the builder (per-element loops, unions, the SELL layouts, the
    counting sorts, which switch to threads above 2^18 entries) gives the bytes of the
    one-thread build."""
    from manapy_b200 import native
    el, vx = meshgen.square_triangles(230, seed=12)          # 105,800 triangles
    monkeypatch.setenv("MANAPY_B200_HOST_THREADS", "1")
    one = native.tables2d(el, vx, stencil="shared", full=True)
    monkeypatch.setenv("MANAPY_B200_HOST_THREADS", "7")
    many = native.tables2d(el, vx, stencil="shared", full=True)
    assert one.keys() == many.keys()
    for k in one:
        assert one[k].dtype == many[k].dtype and one[k].shape == many[k].shape, k
        assert one[k].tobytes() == many[k].tobytes(), k
