"""Host side of the serving loop, on the CPU: the seeded request stream and the per-request
preparation a worker process runs (native tables, boundary rules, initial state)."""
import numpy as np

from manapy_b200 import serving as SV
from manapy_b200.device import DeviceMesh


def test_request_stream_is_seeded_and_within_bounds():
    a = SV.make_requests(400, rate=20.0, seed=7)
    b = SV.make_requests(400, rate=20.0, seed=7)
    assert [(r.kind, r.n, r.seed, r.steps, r.arrival) for r in a] == [(r.kind, r.n, r.seed, r.steps, r.arrival)
                                                                       for r in b]
    arr = np.array([r.arrival for r in a])
    assert np.all(np.diff(arr) >= 0) and 10 < arr[-1] < 30          # Poisson, mean gap 0.05 s
    assert all(2e3 * 0.8 <= r.cells <= 5e5 * 1.2 for r in a)
    assert all(100 <= r.steps <= 2000 for r in a)
    frac = np.mean([r.kind == "advdiff" for r in a])
    assert 0.6 < frac < 0.8
    for r in a:
        if r.kind == "advdiff":
            assert 0.2 <= np.hypot(r.ux, r.uy) <= 1.5 + 1e-12 and 1e-4 <= r.D <= 1e-2
        else:
            assert 1.2 <= r.ratio <= 3.0
    assert all(r.arrival == 0 for r in SV.make_requests(5, rate=0.0))


def test_prepare_gives_host_tables_in_device_order():
    for kind in ("advdiff", "sw"):
        req = SV.Request(rid=0, kind=kind, n=12, seed=3, steps=10, ux=0.3, uy=0.1, D=1e-3)
        _, dm, bc, init = SV.prepare(req)
        assert set(dm.t) <= set(DeviceMesh.SERVE_TABLES)
        assert all(isinstance(v, np.ndarray) for v in dm.t.values())
        assert dm.A is None and dm.nbcells == 2 * 12 * 12
        assert (bc is not None) == (kind == "advdiff")
        assert len(init) == (1 if kind == "advdiff" else 5)
        # the initial state is manapy's, permuted into the device (Morton) numbering
        from manapy_b200 import geometry as G, meshgen
        el, vx = meshgen.square_triangles(12, seed=3)
        A = G.build(el, vx, 2)
        ref = SV.initial_state(req, A["cells_center"])
        for a, r in zip(init, ref):
            assert np.array_equal(a, r[dm.R.cperm])


def _struct_of(dm):
    """An MbMesh whose pointer fields are non-NULL exactly for the tables ``dm`` holds."""
    from manapy_b200 import _lib
    s = _lib.MbMesh()
    for name, _ in _lib.MbMesh._fields_:
        if name in dm.t:
            setattr(s, name, 1)
    return s


def test_batched_items_are_checked_for_the_tables_their_step_reads():
    """The batched kernels read mesh tables through pointers held in device memory, which no
    kernel can check: the server checks each item on the host.  A mesh prepared for the FP32c
    batches lacks the FP64 centre->vertex weights of the FP64 batches."""
    import pytest
    for kind in ("advdiff", "sw"):
        req = SV.Request(rid=0, kind=kind, n=10, seed=5, steps=10, ux=0.3, uy=0.1, D=1e-3)
        for prec in ("fp32c", "fp64"):
            _, dm, _, _ = SV.prepare(req, prec)
            SV.check_item_tables(kind, prec, _struct_of(dm))
        _, dm32, _, _ = SV.prepare(req, "fp32c")
        if kind == "advdiff":
            with pytest.raises(ValueError, match="n2c_sell_alpha"):
                SV.check_item_tables(kind, "fp64", _struct_of(dm32))
