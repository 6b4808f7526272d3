"""Run server (continuous batching of NRG runs on one GPU): every result is
the same alone and in the mix, admission respects the memory budget, and a
failing run does not take the others down.

Tolerance of "the same": the merged eigensolver call splits the cooperative
panel work of a block over a different number of CTAs than a solo call, so
sums are taken in another order.  Thermodynamics (td, printed with 10
significant digits) agree to 1e-8 relative, the accuracy target for chi(T)
and S(T) (plus 1e-13 of the column scale for columns that vanish by
symmetry); spectral weights per bin (raw doubles) to 1e-9 of the largest
bin."""
import glob
import os

import numpy as np
import pytest

import inputgen
import nrg_cases as cases

pytestmark = pytest.mark.gpu

TD_RTOL = 1e-8
BIN_RTOL = 1e-9

# small runs of the served workload's kind (SIAM, z-shifts, FDM), different Nkeep
RUNS = [
    dict(z=0.25, eps_d=-0.05, keep=120, Nmax=18),
    dict(z=0.5, eps_d=-0.12, keep=200, Nmax=18),
    dict(z=0.75, eps_d=-0.02, keep=160, Nmax=20),
    dict(z=1.0, eps_d=-0.1, keep=240, Nmax=16),
    dict(z=0.625, eps_d=-0.07, keep=100, Nmax=20),
]


def make_run(root, i, r, T=1e-4):
    wd = os.path.join(root, "in%d" % i)
    inputgen.make_siam(wd, 0.2, r["eps_d"], 0.02, 2.0, r["Nmax"], z=r["z"],
                       params={"keep": r["keep"], "fdm": True, "T": T, "specd": "A_d-A_d", "bins": 40,
                               "savebins": True, "broaden": False})
    return wd


def compare_outputs(da, db):
    ta, tb = cases.read_table(os.path.join(da, "td")), cases.read_table(os.path.join(db, "td"))
    assert ta.shape == tb.shape
    colmax = np.max(np.abs(ta), axis=0)
    assert np.all(np.abs(ta - tb) <= TD_RTOL * np.abs(ta) + 1e-13 * (1 + colmax))
    fa = sorted(glob.glob(os.path.join(da, "*.bin")))
    assert fa and [os.path.basename(x) for x in fa] == [os.path.basename(x) for x in
                                                         sorted(glob.glob(os.path.join(db, "*.bin")))]
    for f in fa:
        a, b = cases.read_bins(f), cases.read_bins(os.path.join(db, os.path.basename(f)))
        xa, xb = dict(zip(a[:, 0], a[:, 1])), dict(zip(b[:, 0], b[:, 1]))
        wmax = max(abs(v) for v in xa.values())
        err = max(abs(xa.get(k, 0.0) - xb.get(k, 0.0)) for k in set(xa) | set(xb))
        assert err <= BIN_RTOL * wmax, (f, err, wmax)


def test_results_same_alone_and_in_the_mix(tmp_path):
    import nrgb
    wds = [make_run(str(tmp_path), i, r) for i, r in enumerate(RUNS)]
    alone = []
    ctx = nrgb.Context(0)
    for i, wd in enumerate(wds):
        od = str(tmp_path / ("alone%d" % i))
        os.makedirs(od)
        ctx.run(wd, od)
        alone.append(od)
    ctx.close()
    srv = nrgb.Server(0, max_runs=len(wds), batch_window_us=5000)
    mix = []
    tickets = []
    for i, wd in enumerate(wds):
        od = str(tmp_path / ("mix%d" % i))
        os.makedirs(od)
        mix.append(od)
        tickets.append(srv.submit(wd, od))
    stats = [srv.wait(t, 600) for t in tickets]
    cnt = srv.counters()
    srv.close()
    assert cnt["done"] == len(wds) and cnt["failed"] == 0
    # the runs overlapped and their eigensolves were merged
    assert cnt["peak_running"] >= 2
    assert cnt["eig_requests"] > cnt["eig_calls"]
    for s in stats:
        assert 0 < s["peak_bytes"] <= s["projected_bytes"]
        assert s["latency_s"] >= s["queue_s"] >= 0
    for a, b in zip(alone, mix):
        compare_outputs(a, b)


def test_admission_respects_memory_budget(tmp_path):
    import nrgb
    wds = [make_run(str(tmp_path), i, r) for i, r in enumerate(RUNS[:4])]
    proj = [nrgb.project_bytes(wd) for wd in wds]
    budget = 1.05 * max(proj)  # no two of these runs fit together
    assert budget < 2 * min(proj)
    srv = nrgb.Server(0, max_runs=4, mem_budget_bytes=budget)
    tickets = []
    for i, wd in enumerate(wds):
        od = str(tmp_path / ("o%d" % i))
        os.makedirs(od)
        tickets.append(srv.submit(wd, od))
    stats = [srv.wait(t, 600) for t in tickets]
    cnt = srv.counters()
    srv.close()
    assert cnt["done"] == 4
    assert cnt["peak_admitted_bytes"] <= budget
    # while no run had finished, projections were the bounds and the second
    # run waited for the first; first come, first served throughout
    assert stats[1]["queue_s"] >= stats[0]["latency_s"] - 0.05
    assert [s["order"] for s in stats] == [1, 2, 3, 4]


def test_projection_is_learned_from_finished_runs(tmp_path):
    """A budget that holds one run by its bound holds several once a run of
    the same shape has finished and its measured peak is known."""
    import nrgb
    r = dict(RUNS[0])
    wds = [make_run(str(tmp_path), i, dict(r, eps_d=r["eps_d"] - 0.01 * i)) for i in range(4)]
    bound = nrgb.project_bytes(wds[0])
    srv = nrgb.Server(0, max_runs=4, mem_budget_bytes=1.5 * bound)
    outs = []
    for i in range(4):
        od = str(tmp_path / ("o%d" % i))
        os.makedirs(od)
        outs.append(od)
    first = srv.wait(srv.submit(wds[0], outs[0]), 600)
    assert first["projected_bytes"] == bound and 0 < first["peak_bytes"] <= bound
    rest = [srv.submit(wd, od) for wd, od in zip(wds[1:], outs[1:])]
    stats = [srv.wait(t, 600) for t in rest]
    cnt = srv.counters()
    srv.close()
    assert cnt["done"] == 4 and cnt["failed"] == 0
    for s_ in stats:
        # learned: twice the measured peak ratio, below the bound
        assert s_["projected_bytes"] == pytest.approx(2.0 * first["peak_bytes"], rel=1e-9)
        assert s_["peak_bytes"] <= s_["projected_bytes"]
    assert cnt["peak_running"] >= 2


def test_failing_run_is_isolated(tmp_path):
    import nrgb
    good = [make_run(str(tmp_path), i, r) for i, r in enumerate(RUNS[:2])]
    # a density-matrix run at T = 0 is rejected by the driver after admission
    bad = make_run(str(tmp_path), 9, RUNS[2], T=0.0)
    srv = nrgb.Server(0, max_runs=3)
    outs = []
    for i, wd in enumerate([good[0], bad, good[1]]):
        od = str(tmp_path / ("o%d" % i))
        os.makedirs(od)
        outs.append(od)
    tickets = [srv.submit(wd, od) for wd, od in zip([good[0], bad, good[1]], outs)]
    srv.wait(tickets[0], 600)
    with pytest.raises(RuntimeError, match="T > 0"):
        srv.wait(tickets[1], 600)
    srv.wait(tickets[2], 600)
    # unreadable input is refused at submission
    with pytest.raises(RuntimeError):
        srv.submit(str(tmp_path / "missing"), outs[0])
    cnt = srv.counters()
    srv.close()
    assert cnt["done"] == 2 and cnt["failed"] == 1
