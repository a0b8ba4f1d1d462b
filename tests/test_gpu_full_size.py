"""The full-size workloads: the benchmark's 512x512x40 storm domain, the
1024x1024x50 storm domain and the 256-domain ensemble.

The oracle cannot run these sizes within a test's time, so they are checked
through properties that do not depend on size: the discrete water balance of
the conservative moisture update closes to 1e-8 of the rain that fell, every
value stays finite, a CUDA-graph replay equals eager launches bit for bit, and
the result does not depend on the block schedule (Krylov blocks per SM, a
resident or a streaming overland solve) bit for bit.  The same kernels are
checked against the oracle at small sizes in test_gpu_parity.py.
"""
import numpy as np
import pytest

import dhara_b200 as db
from dhara_b200 import inputs

pytestmark = pytest.mark.gpu

FIELDS = ("psi", "theta", "ponding", "waterelev")


def advance(dom, nsteps, graph=False, schedule=None):
    """State and diagnostics of one domain after nsteps; schedule =
    (Krylov blocks per SM, overland resident, overland blocks per SM)."""
    with db.Solver(dom.params) as s:
        s.load(dom)
        s.prepare()
        if schedule is not None:
            s.set_launch_config(*schedule)
        s.step(nsteps, graph=graph)
        s.synchronize()
        return {k: s.download(k) for k in FIELDS}, s.diagnostics()


def water_balance_error(dg):
    return abs(dg["storage_change_cum"] - (dg["top_inflow_cum"] - dg["bottom_outflow_cum"]))


def check_domain(st, dg):
    assert dg["nonfinite"] == 0
    for k in FIELDS:
        assert np.isfinite(st[k]).all(), k
    assert dg["rain_cum"] > 0
    assert water_balance_error(dg) <= 1e-8 * dg["rain_cum"], (water_balance_error(dg), dg["rain_cum"])


def test_storm_512x512x40():
    """The benchmark domain: balance and finiteness, graph replay = eager, and
    the smallest schedule (one Krylov block per SM, streaming overland solve)
    = the default one."""
    dom = inputs.mixed_512x512x40(nsteps=4)
    a, ad = advance(dom, 4)
    check_domain(a, ad)
    b, bd = advance(dom, 4, graph=True)
    c, cd = advance(dom, 4, schedule=(1, 0, 1))
    for k in FIELDS:
        assert np.array_equal(a[k], b[k]), ("graph", k)
        assert np.array_equal(a[k], c[k]), ("schedule", k)
    for key in ("krylov_iters_total", "refine_iters_total", "overland_iters_total"):
        assert ad[key] == bd[key] == cd[key], key


def test_storm_1024x1024x50():
    """52 million cells under the storm's peak rain rate (50 mm/h, dt 120 s)."""
    dom = inputs.large_1024x1024x50(nsteps=3)
    dom.rain_mm = np.full(3, 50.0 * dom.params.dt / 3600.0)
    st, dg = advance(dom, 3)
    check_domain(st, dg)
    assert dg["krylov_nonconverged"] == 0


def test_ensemble_256_domains():
    """All 256 domains of the ensemble in one handle, graph-replayed: every
    domain's own balance, and the batch equals an eager run bit for bit."""
    doms = inputs.ensemble(256, nsteps=3)
    out = []
    for graph in (True, False):
        with db.Solver([d.params for d in doms]) as s:
            for i, d in enumerate(doms):
                s.load(d, i)
            s.prepare()
            s.step(3, graph=graph)
            s.synchronize()
            out.append([({k: s.download(k, i) for k in FIELDS}, s.diagnostics(i)) for i in range(len(doms))])
    for (st, dg), (st2, dg2) in zip(*out):
        check_domain(st, dg)
        for k in FIELDS:
            assert np.array_equal(st[k], st2[k]), k


def test_ensemble_shards_equal_one_handle():
    """The ensemble split as two ranks would split it (dhara_b200.ensemble),
    each share advanced by its own handle one after the other on this GPU:
    every domain ends bit for bit where the single 256-domain handle puts it,
    so sharding over GPUs changes nothing but the time."""
    from dhara_b200 import ensemble as ens
    doms = inputs.ensemble(256, nsteps=2)

    def advance_share(idx):
        with db.Solver([doms[i].params for i in idx]) as s:
            for j, i in enumerate(idx):
                s.load(doms[i], j)
            s.prepare()
            s.step(2, graph=True)
            s.synchronize()
            return {i: ({k: s.download(k, j) for k in FIELDS}, s.diagnostics(j)) for j, i in enumerate(idx)}

    whole = advance_share(list(range(len(doms))))
    shares = ens.partition([d.ncells for d in doms], 2)
    assert ens.balance([d.ncells for d in doms], 2) < 1.01
    for share in shares:
        part = advance_share(share)
        for i, (st, dg) in part.items():
            for k in FIELDS:
                assert np.array_equal(st[k], whole[i][0][k]), (i, k)
            assert dg["krylov_iters_total"] == whole[i][1]["krylov_iters_total"], i
