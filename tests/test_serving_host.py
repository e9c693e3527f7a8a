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
