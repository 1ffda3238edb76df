"""Serving form: results of a run served in a mix equal the run alone.

The serving loop admits many independent runs, keeps them resident
together and advances each in slices of time steps interleaved with the
others.  Every run must come back with what the plain drop-in call returns
for the same inputs: relative L2 error <= 1e-4 on every output (the bound
the FP32 path meets against the FP64 oracle), and in fact bit-identical,
since each run executes the same kernels on the same data in the same
order whatever else is resident.
"""
import numpy as np
import pytest

from cases import CASES, make_case

TOL = 1e-4


def _grid(mod, shape, dx, Nt, dt):
    args = []
    for s in shape:
        args += [s, dx]
    g = mod.kWaveGrid(*args)
    g.setTime(Nt, dt)
    return g


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (d if d > 0 else 1.0))


def _flat(out):
    if out is None:
        return {}
    if isinstance(out, np.ndarray):
        return {"": out}
    if isinstance(out, list):
        return {"%d.%s" % (i, k): v for i, d in enumerate(out) for k, v in d.items()}
    return dict(out)


def _alone(kw, name):
    dim, shape, dx, Nt, dt, med, src, sen, opts = make_case(name)
    run = kw.kspaceFirstOrder2D if dim == 2 else kw.kspaceFirstOrder3D
    return run(_grid(kw, shape, dx, Nt, dt), med, src, sen, **opts)


def _submit(kw, server, name):
    dim, shape, dx, Nt, dt, med, src, sen, opts = make_case(name)
    return server.submit(dim, _grid(kw, shape, dx, Nt, dt), med, src, sen, **opts)


def _compare(name, served, alone):
    a, b = _flat(served), _flat(alone)
    assert set(a) == set(b), (name, sorted(a), sorted(b))
    for k in b:
        assert a[k].shape == b[k].shape, (name, k)
        e = _rel(a[k], b[k])
        assert e <= TOL, "%s %s: served vs alone rel-L2 %.3e" % (name, k, e)
        assert np.array_equal(a[k], b[k]), "%s %s: served result not bit-identical (rel-L2 %.3e)" % (name, k, e)


@pytest.mark.gpu
@pytest.mark.parametrize("max_active,slice_steps,budget", [(4, 5, 0), (32, 32, 0), (32, 16, 1)])
def test_mix_equals_alone(max_active, slice_steps, budget):
    """Every case of the parity suite, submitted at once, against its plain run.
    (4, 5): few slots, short slices -- runs queue and interleave finely;
    (32, 32): everything resident at once; budget 1 byte: one run at a time."""
    import kwave_b200 as kw
    alone = {n: _alone(kw, n) for n in CASES}
    with kw.Server(max_active=max_active, steps_per_slice=slice_steps, hbm_budget_bytes=budget) as srv:
        tickets = [(n, _submit(kw, srv, n)) for n in CASES + CASES[::-1]]
        for n, t in tickets:
            _compare(n, srv.result(t), alone[n])
        st = srv.stats()
    assert st["completed"] == 2 * len(CASES) and st["failed"] == 0
    assert st["active"] == 0 and st["pending"] == 0
    assert 0 < st["p50_ms"] <= st["p99_ms"]


@pytest.mark.gpu
def test_failed_request_does_not_disturb_others():
    """A request the library rejects at admission (an axis of 4100 points,
    above the 4096-point line of one transform tile) fails alone; the runs
    around it finish unchanged."""
    import kwave_b200 as kw
    name = "2d_hetero_abs_nl"
    ref = _alone(kw, name)
    bad = kw.kWaveGrid(22, 1e-4, 4100, 1e-4)
    bad.setTime(10, 2e-8)
    with kw.Server(max_active=2, steps_per_slice=3) as srv:
        t0 = _submit(kw, srv, name)
        tb = srv.submit(2, bad, {"sound_speed": 1500.0}, {"p0": np.ones((22, 4100))}, {"mask": np.ones((22, 4100))},
                        PMLSize=2)
        t1 = _submit(kw, srv, name)
        with pytest.raises(kw.KWaveError, match="outside 2..4096"):
            srv.result(tb)
        _compare(name, srv.result(t0), ref)
        _compare(name, srv.result(t1), ref)
        st = srv.stats()
    assert st["completed"] == 2 and st["failed"] == 1


@pytest.mark.gpu
def test_deadline_watchdog_and_bounded_wait():
    """The serving watchdog: a request still running request_timeout_ms after
    its admission gets no further steps, drains and fails with KW_ERR_TIMEOUT,
    while the run beside it finishes unchanged; a bounded wait on an
    unfinished request returns KW_ERR_TIMEOUT and leaves its ticket valid.
    The stall is a host-side one (a run far longer than the deadline); no
    device wait is involved."""
    import kwave_b200 as kw
    from kwave_b200 import _abi
    name = "2d_hetero_abs_nl"
    ref = _alone(kw, name)
    N = 512
    long_grid = kw.kWaveGrid(N, 1e-4, N, 1e-4)
    long_grid.setTime(200000, 2e-8)      # tens of seconds alone
    mask = np.zeros((N, N))
    mask[40, :] = 1
    with kw.Server(max_active=4, steps_per_slice=16, request_timeout_ms=2000) as srv:
        t_long = srv.submit(2, long_grid, {"sound_speed": 1500.0, "density": 1000.0},
                            {"p0": kw.makeDisc(N, N, N // 2, N // 2, 8)}, {"mask": mask, "record": ["p_max"]},
                            PMLSize=10)
        t0 = _submit(kw, srv, name)
        with pytest.raises(kw.KWaveError) as e:
            srv.result(t_long, timeout_ms=5)
        assert e.value.status == _abi.KW_ERR_TIMEOUT
        _compare(name, srv.result(t0), ref)
        with pytest.raises(kw.KWaveError, match="deadline") as e:
            srv.result(t_long)
        assert e.value.status == _abi.KW_ERR_TIMEOUT
        st = srv.stats()
    assert st["completed"] == 1 and st["failed"] == 1
    assert st["active"] == 0 and st["pending"] == 0
