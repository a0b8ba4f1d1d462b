"""Block schedules: results do not depend on them (reductions run over tiles
and segments in a fixed order), and the autotuner leaves the state as it was."""
import numpy as np
import pytest

import dhara_b200 as db
from dhara_b200 import inputs

pytestmark = pytest.mark.gpu


def domain():
    return inputs.make_domain(40, 36, 12, seed=21, rain_mm_per_h=40.0, nsteps=6, krylov_tol=1e-11,
                              krylov_maxiter=2000, precision=db.MIXED)


def run_with(cfg, nsteps=4):
    d = domain()
    s = db.Solver(d.params)
    s.load(d)
    s.prepare()
    if cfg is not None:
        s.set_launch_config(*cfg)
    s.step(nsteps)
    out = {k: s.download(k) for k in ("psi", "theta", "ponding", "waterelev")}
    s.close()
    return out


def test_results_do_not_depend_on_the_schedule(gpu):
    base = run_with(None)
    for cfg in ((1, 0, 1), (2, 1, 2), (3, 0, 3)):
        other = run_with(cfg)
        for k in base:
            assert np.array_equal(base[k], other[k]), (cfg, k)


def test_autotune_restores_state(gpu):
    d = domain()
    s = db.Solver(d.params)
    s.load(d)
    s.prepare()
    s.step(1)
    before = {k: s.download(k) for k in ("psi", "theta", "ponding", "waterelev")}
    dg = s.diagnostics()
    chosen = s.autotune(2)
    after = {k: s.download(k) for k in before}
    for k in before:
        assert np.array_equal(before[k], after[k]), k
    assert s.diagnostics()["steps"] == dg["steps"]
    assert chosen["krylov_blocks_per_sm"] >= 1 and chosen["krylov_ms"] > 0
    assert s.launch_config()["krylov_blocks_per_sm"] == chosen["krylov_blocks_per_sm"]
    s.step(2)
    s.close()
