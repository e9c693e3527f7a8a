"""Host side of the serving loop, on the CPU: the seeded request stream, the per-request
preparation a worker process runs (native tables, boundary rules, initial state), and its
hand-over back to the serving process through shared memory."""
import os

import numpy as np
import pytest

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
    for kind in ("advdiff", "sw"):
        req = SV.Request(rid=0, kind=kind, n=10, seed=5, steps=10, ux=0.3, uy=0.1, D=1e-3)
        for prec in ("fp32c", "fp64"):
            _, dm, _, _ = SV.prepare(req, prec)
            SV.check_item_tables(kind, prec, _struct_of(dm))
        _, dm32, _, _ = SV.prepare(req, "fp32c")
        if kind == "advdiff":
            with pytest.raises(ValueError, match="n2c_sell_alpha"):
                SV.check_item_tables(kind, "fp64", _struct_of(dm32))

def _arrays(obj, path="x"):
    """Every numpy array reachable from obj, by path."""
    if isinstance(obj, np.ndarray):
        return {path: obj}
    out = {}
    if isinstance(obj, (list, tuple)):
        for i, v in enumerate(obj):
            out.update(_arrays(v, "%s[%d]" % (path, i)))
    elif isinstance(obj, dict):
        for k, v in obj.items():
            out.update(_arrays(v, "%s.%s" % (path, k)))
    elif hasattr(obj, "__dict__") and not isinstance(obj, type):
        out.update(_arrays(vars(obj), path))
    return out


@pytest.mark.skipif(not os.path.isdir(SV._SHM_DIR), reason="no tmpfs at /dev/shm")
@pytest.mark.parametrize("kind_seed", [3, 4])
def test_prepared_request_crosses_shared_memory(kind_seed):
    req = SV.make_requests(1, 0.0, seed=kind_seed, cells=(3e3, 6e3))[0]
    a = SV.prepare(req)
    x = SV._ship(a)
    assert isinstance(x, SV._Shipped) and os.path.exists(x.path) and len(x.head) < 16384
    b = SV._receive(x)
    assert not os.path.exists(x.path)
    aa, bb = _arrays(a), _arrays(b)
    assert aa.keys() == bb.keys() and len(aa) > 30
    for k in aa:
        assert aa[k].dtype == bb[k].dtype and aa[k].shape == bb[k].shape, k
        assert np.array_equal(aa[k], bb[k], equal_nan=True), k
        if bb[k].nbytes:
            assert bb[k].ctypes.data % 64 == 0, k
    assert b[0].prep_window is not None and b[0].rid == req.rid


def test_hand_over_without_tmpfs(monkeypatch, tmp_path):
    monkeypatch.setattr(SV, "_SHM_DIR", str(tmp_path / "absent"))
    req = SV.make_requests(1, 0.0, seed=5, cells=(2e3, 3e3))[0]
    a = SV.prepare(req)
    assert SV._ship(a) is a
    assert SV._receive(a) is a


@pytest.mark.skipif(not os.path.isdir(SV._SHM_DIR), reason="no tmpfs at /dev/shm")
def test_unreceived_preparation_leaves_no_file():
    """A preparation that nobody admits (the serving loop ended by an error) has its
    shared-memory file removed when it finishes."""
    import concurrent.futures as cf
    req = SV.make_requests(1, 0.0, seed=6, cells=(2e3, 3e3))[0]
    with cf.ThreadPoolExecutor(1) as ex:
        fut = ex.submit(SV.prepare_shipped, req)
        x = fut.result()
        assert isinstance(x, SV._Shipped) and os.path.exists(x.path)
        fut.add_done_callback(SV._discard)     # runs at once: the future is done
    assert not os.path.exists(x.path)


def test_admission_order():
    """Arrival order while the budget allows; a request that does not fit lets later ones
    that fit pass it until it has waited ``max_skip_wait``; nothing admitted: the first goes
    in whatever its size; never more than the free slots."""
    ao = SV.admission_order
    w = [(0.0, 10.0), (0.1, 10.0), (0.2, 10.0)]
    assert ao(w, used=0.0, budget=100.0, slots=8, active=0, now=0.3) == [0, 1, 2]
    assert ao(w, used=0.0, budget=100.0, slots=2, active=0, now=0.3) == [0, 1]
    big = [(0.0, 80.0), (0.1, 10.0), (0.2, 5.0), (0.3, 40.0)]
    # 50 bytes in use: the 80-byte head does not fit, the two small ones pass it, the 40-byte
    # one no longer fits after them
    assert ao(big, used=50.0, budget=100.0, slots=8, active=3, now=0.5) == [1, 2]
    # the head has waited long enough: nothing passes it
    assert ao(big, used=50.0, budget=100.0, slots=8, active=3, now=1.5, max_skip_wait=1.0) == []
    assert ao(big, used=50.0, budget=100.0, slots=8, active=3, now=0.5, max_skip_wait=0.0) == []
    # nothing admitted: the oversize head goes in alone, then the budget counts it
    assert ao([(0.0, 150.0), (0.1, 10.0)], used=0.0, budget=100.0, slots=8, active=0, now=0.2) == [0]
    assert ao([], used=0.0, budget=100.0, slots=8, active=0, now=0.0) == []
