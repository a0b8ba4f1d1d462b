"""Time-step halving (dhara_params.dt_halvings), the opt-in alternative to
the reference's acceptance of a step whose modified Picard iteration ended
at its cap (src/subsurface.cu:762-789): a failed step is undone and retried
as two half steps, per domain.  Off (0) the path is the reference's scheme;
on, a domain whose Picard iteration converges at full dt is unchanged bit
for bit, a batch equals its domains run alone, the water balance closes
over the sub-steps, and a domain that diverges under the reference scheme
(rain on dry, strongly capillary soil) stays bounded.
"""
import numpy as np
import pytest

import dhara_b200 as db
from dhara_b200 import inputs

pytestmark = pytest.mark.gpu


def with_halvings(d, k):
    p = type(d.params).from_buffer_copy(d.params)
    p.dt_halvings = k
    return inputs.Domain(params=p, fields=d.fields, int_fields=d.int_fields, rain_mm=d.rain_mm)


def run(doms, nsteps):
    s = db.Solver([d.params for d in doms])
    for i, d in enumerate(doms):
        s.load(d, i)
    s.prepare()
    s.step(nsteps)
    out = [({k: s.download(k, i) for k in ("psi", "theta", "ponding", "waterelev")}, s.diagnostics(i))
           for i in range(len(doms))]
    s.close()
    return out


def mass_error(dg):
    return abs(dg["storage_change_cum"] - (dg["top_inflow_cum"] - dg["bottom_outflow_cum"])) / dg["top_inflow_cum"]


def converging_domain():
    """Light rain (5 mm/h) on a domain whose Picard iteration converges at full
    dt every step (the oracle needs 52 iterations over the 6 steps, cap 20)."""
    return inputs.make_domain(24, 20, 12, seed=3, nsteps=6, precision=db.FP64, rain_mm_per_h=5.0,
                              picard_maxiter=20, picard_rule=db._abi.PICARD_PSI_ABSOLUTE, picard_tol=1e-6,
                              krylov_tol=1e-10, krylov_maxiter=2000)


def test_converging_domain_is_unchanged(gpu):
    d = converging_domain()
    (a, da), = run([d], 6)
    (b, dbb), = run([with_halvings(d, 4)], 6)
    assert da["picard_nonconverged"] == 0
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert dbb["substeps_total"] == dbb["step_attempts_total"] == dbb["steps"] == 6


def test_diverging_domain_stays_bounded(gpu):
    # ensemble domain 20 (16 x 123 x 21, alpha 4.25 /m, n 2.04): under the
    # reference scheme every step ends at the Picard cap and the heads run
    # away (hundreds of metres within 12 steps, ~1e9 m later)
    d = inputs.ensemble(256, nsteps=12)[20]
    (a, da), = run([d], 12)
    (b, dbb), = run([with_halvings(d, 10)], 12)
    print("reference scheme: max |psi|", np.abs(a["psi"]).max(), "capped steps", da["picard_nonconverged"])
    print("halving: max |psi|", np.abs(b["psi"]).max(), "capped", dbb["picard_nonconverged"],
          "sub-steps", dbb["substeps_total"], "attempts", dbb["step_attempts_total"], "mass", mass_error(dbb))
    assert da["picard_nonconverged"] == 12 and np.abs(a["psi"]).max() > 1e2
    assert np.abs(b["psi"]).max() < 5.0
    # only sub-steps at the smallest length (dt / 1024) may end at the cap
    assert dbb["picard_nonconverged"] < 0.1 * dbb["substeps_total"]
    assert dbb["steps"] == 12 and dbb["substeps_total"] > 12
    assert mass_error(dbb) < 1e-8


def test_halving_batch_equals_individual(gpu):
    ens = inputs.ensemble(256, nsteps=4)
    doms = [with_halvings(ens[i], 6) for i in (20, 3, 57)]
    both = run(doms, 4)
    for i, d in enumerate(doms):
        (alone, da), = run([d], 4)
        for k in alone:
            assert np.array_equal(alone[k], both[i][0][k]), (i, k)
        assert da["substeps_total"] == both[i][1]["substeps_total"], i
