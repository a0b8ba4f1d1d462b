"""The fused subsurface step (dhara_launch_config.fused_step: prologue, every
Picard iteration's assembly, Dirichlet passes, linear solve and check, and
the epilogue in one persistent launch, k_step) against the launch-per-kernel
sequence it replaces: the same per-tile code in the same order, so states,
water balances and iteration counts agree bit for bit -- for a batch of
uneven domains, with Dirichlet faces, eagerly and replayed from a CUDA graph --
and a graph-replayed step of the batch is four launches (the step and the
three overland kernels)."""
import numpy as np
import pytest

import dhara_b200 as db
from dhara_b200 import inputs

from test_gpu_dirichlet import domain_with_faces

pytestmark = pytest.mark.gpu


def batch(prec):
    return [inputs.make_domain(17, 9, 7, seed=1, precision=prec, rain_mm_per_h=30.0, nsteps=4),
            inputs.make_domain(40, 33, 12, seed=2, precision=prec, rain_mm_per_h=30.0, nsteps=4),
            inputs.make_domain(5, 70, 4, seed=3, precision=prec, rain_mm_per_h=30.0, nsteps=4)]


def run(doms, fused, nsteps, graph):
    s = db.Solver([d.params for d in doms])
    for i, d in enumerate(doms):
        s.load(d, i)
    s.prepare()
    c = s.launch_config()
    s.set_launch_config(c["krylov_blocks_per_sm"], c["overland_resident"], c["overland_blocks_per_sm"],
                        fused_step=fused)
    assert s.launch_config()["fused_step"] == fused
    n0 = s.launch_count()
    s.step(nsteps, graph=graph)
    s.synchronize()
    launches = s.launch_count() - n0
    out = [({k: s.download(k, i) for k in ("psi", "theta", "ponding", "waterelev")}, s.diagnostics(i))
           for i in range(len(doms))]
    s.close()
    return out, launches


@pytest.mark.parametrize("prec", [db.FP64, db.MIXED])
@pytest.mark.parametrize("graph", [False, True])
def test_fused_step_equals_launch_per_kernel(gpu, prec, graph):
    doms = batch(prec)
    a, _ = run(doms, 0, 3, graph)
    b, launches = run(doms, 1, 3, graph)
    for (sa, da), (sb, dbg) in zip(a, b):
        for k in sa:
            assert np.array_equal(sa[k], sb[k]), k
        for k in ("picard_iters_total", "krylov_iters_total", "refine_iters_total", "mb_subsurface_cum"):
            assert da[k] == dbg[k], k
    if graph:
        assert launches == 3 * 4


def test_fused_step_with_dirichlet_faces(gpu):
    d = domain_with_faces({"west": 0.2, "bottom": -0.1})
    a, _ = run([d], 0, 3, False)
    b, _ = run([d], 1, 3, False)
    for k in a[0][0]:
        assert np.array_equal(a[0][0][k], b[0][0][k]), k
