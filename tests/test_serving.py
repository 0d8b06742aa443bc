"""Serving loop (kumo_server_*): a burst of requests of different molecules,
sizes, request types and precisions runs concurrently on the GPU; each result
must equal the same request evaluated alone through the regular entry points
(the kernels are deterministic and padding repeats the last point, so equality
is exact; the stated tolerance is 1e-12 scaled for FP64 and for the mixed
form against its own lone run)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, scaled_error

import kumo_b200 as K
from kumo_b200 import synth

P = K.PropertyKind
FIELDS = [K.density(P.Density), K.density(P.Gradient), K.density(P.Laplacian), K.density(P.Tau), K.density(P.Elf)]


def _line(m, npts):
    _, _, xyz = m.atoms()
    a, b = xyz.min(0) - 2.0, xyz.max(0) + 2.0
    step = (b - a) / (npts - 1)
    return K.Grid(a, np.column_stack([step, [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]]), (npts, 1, 1))


def _requests(mols, rng):
    reqs = []
    for name, m in mols.items():
        _, _, xyz = m.atoms()
        lo, hi = xyz.min(0) - 2.5, xyz.max(0) + 2.5
        for prec in (K.Precision.FP64, K.Precision.Mixed):
            n = int(rng.integers(1, 1000))
            reqs.append(("points", name, dict(points=rng.uniform(lo, hi, (n, 3))), FIELDS, prec))
            reqs.append(("points", name, dict(points=rng.uniform(lo, hi, (n, 3))), FIELDS, prec))  # same bucket
            reqs.append(("grid", name, dict(grid=_line(m, 1000)), FIELDS, prec))
            plane = K.Grid(lo, np.diag([0.2, 0.2, 1.0]), (60, 60, 1))
            reqs.append(("grid", name, dict(grid=plane), FIELDS, prec))
        reqs.append(("grid", name, dict(grid=m.grid_around(2.0, 0.25)), FIELDS, K.Precision.Mixed))
        info = m.info()
        homo = int(info["nalpha"])
        reqs.append(("points", name, dict(points=rng.uniform(lo, hi, (300, 3))),
                     [K.orbital(homo), K.orbital(homo + 1)], K.Precision.FP64))
        reqs.append(("points", name, dict(points=rng.uniform(lo, hi, (200, 3))),
                     [K.density(P.ElectrostaticPotential)], K.Precision.FP64))
    return reqs


def _alone(m, kind, arg, props, prec):
    ev = K.Evaluator(m, precision=prec)
    if kind == "grid":
        return ev.evaluate_grid(arg["grid"], props)[0]
    return ev.evaluate_points(arg["points"], props)[0]


@pytest.mark.gpu
def test_serving_mix_equals_alone(synth_cache):
    mols = {n: K.Molecule.from_fchk(os.path.join(GOLDEN, n)) for n in ("o2.fchk.gz", "acrolein.fchk.gz")}
    mols["water_28"] = K.Molecule.from_fchk(synth.workload_fchk("water_28", synth_cache))
    rng = np.random.default_rng(11)
    reqs = _requests(mols, rng)
    srv = K.Server(max_active=4)

    def burst():
        tickets = []
        for kind, name, arg, props, prec in reqs:
            if kind == "grid":
                t, outs = srv.submit_grid(mols[name], arg["grid"], props, precision=int(prec))
            else:
                t, outs = srv.submit_points(mols[name], arg["points"], props, precision=int(prec))
            tickets.append((t, outs))
        for t, _ in tickets:
            assert srv.wait(t, 120.0)
        return tickets

    first = burst()
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["graph_captures"] >= 1 and st["direct_runs"] >= 1
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    assert st["peak_bytes"] <= st["budget_bytes"]
    # A shape met again is captured into a graph (second meeting) and then
    # replayed.  Requests of one shape that run at the same time take separate
    # graph instances, so a later burst may still capture an instance when
    # more of them overlap than before.
    second = burst()
    st2 = srv.stats()
    third = burst()
    st3 = srv.stats()
    assert st2["graph_captures"] > st["graph_captures"]
    assert st3["graph_replays"] > st2["graph_replays"]
    for (kind, name, arg, props, prec), (_, o1), (_, o2), (_, o3) in zip(reqs, first, second, third):
        ref = _alone(mols[name], kind, arg, props, prec)
        for p, a, b, c, r in zip(props, o1, o2, o3, ref):
            assert scaled_error(a, r) <= 1e-12, (kind, name, p, prec, scaled_error(a, r))
            for x in (a, b, c):
                assert np.array_equal(x, r), (kind, name, p, prec)
    srv.close()


@pytest.mark.gpu
def test_serving_admission_under_small_budget():
    # A budget smaller than the requests' footprints together: requests wait
    # for memory instead of failing, every one completes, and the admitted
    # footprint never exceeds the budget.
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, "acrolein.fchk.gz"))
    # A 1 MiB staging arena: most staging falls back to page-locking on demand.
    srv = K.Server(hbm_budget_bytes=1.5e9, max_active=8, request_scratch_bytes=256 * 2**20, staging_bytes=2**20)
    grid = m.grid_around(3.0, 0.15)
    tickets = [srv.submit_grid(m, grid, FIELDS, precision=int(K.Precision.Mixed)) for _ in range(3)]
    tickets += [srv.submit_points(m, np.random.default_rng(i).uniform(-3, 3, (500, 3)), FIELDS) for i in range(5)]
    srv.drain()
    st = srv.stats()
    assert st["completed"] == 8 and st["peak_bytes"] <= st["budget_bytes"]
    ref = K.Evaluator(m, precision=K.Precision.Mixed).evaluate_grid(grid, FIELDS)[0]
    for a, r in zip(tickets[0][1], ref):
        assert np.array_equal(a, r)
    srv.close()


@pytest.mark.gpu
def test_kernel_preload_then_evaluation():
    # Loading every listed kernel succeeds (each name resolves to a kernel of
    # this device's code), a second call does nothing, and evaluations after
    # it give the same bits as before.
    m = K.Molecule.from_fchk(os.path.join(GOLDEN, "acrolein.fchk.gz"))
    grid = m.grid_around(3.0, 0.3)
    ev = K.Evaluator(m, precision=K.Precision.Mixed)
    before = ev.evaluate_grid(grid, FIELDS)[0]
    assert K.registered_kernels() >= 60
    K.preload_kernels()
    K.preload_kernels()
    after = ev.evaluate_grid(grid, FIELDS)[0]
    for a, b in zip(after, before):
        assert np.array_equal(a, b)


def test_serving_rejects_bad_requests_before_device_work():
    # Validation happens at submit, with the evaluator's exception types; no
    # GPU is needed to see it (creating the server needs one, so this only
    # checks that creation fails cleanly where there is none).
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        srv = K.Server()
        m = K.Molecule.from_fchk(os.path.join(GOLDEN, "o2.fchk.gz"))
        with pytest.raises(K.InvalidArgument):
            srv.submit_points(m, np.zeros((4, 3)), FIELDS, block_size=0)
        with pytest.raises(K.OutOfRange):
            srv.submit_points(m, np.zeros((4, 3)), [K.orbital(10**6)])
        srv.close()
    else:
        with pytest.raises(K.KumoError):
            K.Server()
