"""Checkpoint and restart (dhara_checkpoint / dhara_restore): a handle rebuilt
from the same inputs and restored from a checkpoint continues exactly where
the original handle was, bit for bit, for every domain; a checkpoint of other
domains, or bytes that are not a checkpoint, are rejected.  And the failure
detection under them: a bounded device-side wait gives up and reports."""
import numpy as np
import pytest

import dhara_b200 as db
from dhara_b200 import inputs

pytestmark = pytest.mark.gpu

FIELDS = ("psi", "theta", "ponding", "waterelev")


def domains(nz0=10):
    mk = dict(rain_mm_per_h=30.0, nsteps=12, theta_update=db.THETA_CONSERVATIVE, precision=db.MIXED,
              krylov_tol=1e-10, krylov_maxiter=400)
    return [inputs.make_domain(24, 20, nz0, seed=3, **mk), inputs.make_domain(9, 37, 7, seed=4, **mk)]


def fresh(doms):
    s = db.Solver([d.params for d in doms])
    for i, d in enumerate(doms):
        s.load(d, i)
    s.prepare()
    return s


def state(s, n):
    return [({k: s.download(k, i) for k in FIELDS}, s.diagnostics(i)) for i in range(n)]


@pytest.mark.parametrize("graph", [False, True])
def test_restart_continues_bit_for_bit(graph):
    doms = domains()
    with fresh(doms) as a:
        a.step(4)
        ck = a.checkpoint()
        a.step(5)
        a.synchronize()
        want = state(a, len(doms))
    with fresh(doms) as b:
        b.step(2)          # whatever the new handle did before is overwritten
        b.restore(ck)
        b.step(5, graph=graph)
        b.synchronize()
        got = state(b, len(doms))
    for (ws, wd), (gs, gd) in zip(want, got):
        for k in FIELDS:
            assert np.array_equal(ws[k], gs[k]), k
        assert wd == gd


def test_restore_rejects_other_domains_and_garbage():
    with fresh(domains()) as a:
        a.step(1)
        ck = a.checkpoint()
    with fresh(domains(nz0=11)) as b:
        with pytest.raises(db.DharaError) as e:
            b.restore(ck)
        assert e.value.code == 1
        with pytest.raises(db.DharaError):
            b.restore(np.zeros(64, np.uint8))
        with pytest.raises(db.DharaError):
            b.restore(ck[:100])


def test_bounded_wait_gives_up_and_context_survives():
    """Failure detection without a fault: a device-side wait that nothing can
    satisfy gives up after its 200 ms limit, flags the error and returns; the
    same process then runs a solver normally."""
    import time
    t0 = time.perf_counter()
    assert db.selftest_bounded_wait(200.0)
    assert 0.2 <= time.perf_counter() - t0 < 10.0
    doms = domains()
    with fresh(doms) as s:
        s.step(1)
        s.synchronize()
        assert s.diagnostics(0)["nonfinite"] == 0
