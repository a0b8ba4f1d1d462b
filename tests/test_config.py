"""The reference's configuration file onto dhara_params (no GPU needed):
key mapping and units (src/io.cc:236-274), the boundary keys with the
reference's top/bottom exchange (src/host.cc:101-114), comments, first
occurrence wins, missing keys keep the defaults."""
import os

import pytest

import dhara_b200 as db
from dhara_b200 import _abi

CFG = """# flow model settings
TIME_STEP_DATA          = 0.25
GRID_SIZE.DX            = 2.0
GRID_SIZE.DY            = 1.5
GRID_SIZE.DZ            = 0.1
# overland
DELTA                   = 2e-7
KZERO                   = 3e-5
WATERDEPTH_MINIMUM      = 2e-5
WATERDEPTH_CRITICAL     = 0.0
MAXIMUM_ITERATIONS      = 7
MINIMUM_PRESSURE_HEAD   = 4e-3
PICARD_METHOD           = 1
TOLERANCE_PRESSURE      = 1e-8
TOLERANCE_THETA         = 2e-4
WEIGHTED_SCHEME         = 0.3
ALPHA                   = 0.035
PORE_SIZE_DISTRIBUTION  = 1.6
POROSITY                = 0.44
SPECIFIC_STORAGE        = 4e-4
RESIDUAL_WATER_CONTENT  = 0.05
SATURATED_WATER_CONTENT = 0.44
ALPHA                   = 0.5
BOUNDARY_TYPE_TOP       = 1
BOUNDARY_TYPE_BOTTOM    = 0
BOUNDARY_TYPE_NORTH     = 2
BOUNDARY_TYPE_WEST      = 0
PRESSURE_HEAD_TOP       = -0.7
PRESSURE_HEAD_BOTTOM    = -1.5
FLUX_TOP                = 1e-6
FLUX_BOTTOM             = 2e-6
FLUX_EAST               = 3e-7
"""


@pytest.fixture
def cfg(tmp_path):
    path = tmp_path / "model.cfg"
    path.write_text(CFG)
    return str(path)


def test_keys_and_units(cfg):
    p, faces, bc = db.params_from_config(cfg, 16, 12, 10)
    assert (p.nx, p.ny, p.nz) == (16, 12, 10)
    assert (p.dx, p.dy, p.dz) == (2.0, 1.5, 0.1)
    assert p.dt == 0.25 and abs(p.sec_p_mm2dt_p_m - 0.25 * 3.6) < 1e-15
    assert p.alpha == pytest.approx(3.5)          # first ALPHA wins, 1/cm -> 1/m
    assert p.n == 1.6 and p.porosity == 0.44 and p.Ss == 4e-4
    assert p.theta_r == 0.05 and p.theta_s == 0.44
    assert p.picard_maxiter == 7 and p.am == 0.3 and p.psimin == 4e-3
    assert p.picard_rule == _abi.PICARD_THETA_RELATIVE and p.picard_tol == 2e-4
    assert p.delta == 2e-7 and p.K0 == 3e-5 and p.hmin == 2e-5


def test_boundary_keys_follow_the_reference(cfg):
    _, faces, bc = db.params_from_config(cfg, 16, 12, 10)
    assert faces["top"] == (1, -1.5, 2e-6)        # *_BOTTOM values land on the top face
    assert faces["bottom"] == (0, -0.7, 1e-6)     # *_TOP values land on the bottom face
    assert faces["north"][0] == 2 and faces["east"] == (1, 0.0, 3e-7)
    assert faces["west"] == (0, 0.0, 0.0)
    assert faces["south"] == (1, 0.0, 0.0)        # missing: free flow, zero values


def test_missing_keys_keep_defaults(tmp_path):
    path = tmp_path / "empty.cfg"
    path.write_text("# nothing\nUNRELATED_KEY = 5\n")
    p, _, bc = db.params_from_config(str(path), 8, 8, 8)
    d = db.default_params(8, 8, 8, 1.2, 1.2, 0.2, 0.5)
    for name, _ in _abi.Params._fields_:
        if name in ("reserved_i", "reserved_d"):
            continue
        assert getattr(p, name) == getattr(d, name), name
    assert bc.found == 0


def test_unreadable_file(tmp_path):
    with pytest.raises(db.DharaError):
        db.params_from_config(str(tmp_path / "missing.cfg"), 8, 8, 8)


@pytest.mark.gpu
def test_boundary_config_on_the_gpu(gpu, cfg):
    """Faces set from the configuration file give the same steps as the same
    faces uploaded as arrays to the oracle."""
    import numpy as np
    import oracle
    from dhara_b200 import inputs
    _, faces, bc = db.params_from_config(cfg, 12, 10, 8)
    d = inputs.make_domain(12, 10, 8, seed=3, krylov_tol=1e-13, krylov_maxiter=4000, nsteps=3,
                           rain_mm_per_h=20.0, picard_rule=_abi.PICARD_PSI_ABSOLUTE, picard_tol=1e-9,
                           overland_tol=1e-13, overland_maxiter=4000)
    nx, ny, nz = 12, 10, 8
    C, WE, SN = nx * ny, nz * ny, nz * nx
    ints = dict(d.int_fields)
    fields = dict(d.fields)
    for face, n, tkey, pkey, qkey in (("bottom", C, "bcb", "bcpsib", "bcqb"), ("north", SN, "bcn", "bcpsin", "bcqn"),
                                      ("south", SN, "bcs", "bcpsis", "bcqs"), ("east", WE, "bce", "bcpsie", "bcqe"),
                                      ("west", WE, "bcw", "bcpsiw", "bcqw")):
        t, psi, q = faces[face]
        ints[tkey] = np.full(n, t, np.int32)
        fields[pkey] = np.full(n, psi)
        fields[qkey] = np.full(n, q)
    ref = inputs.Domain(params=d.params, fields=fields, int_fields=ints, rain_mm=d.rain_mm)
    so, _, _ = oracle.run(ref, nsteps=3, solver3d=oracle.SOLVER_CG)
    s = db.Solver(d.params)
    s.load(d)
    s.apply_boundary_config(bc)
    s.prepare()
    s.step(3)
    for k in ("psi", "theta", "ponding"):
        g = s.download(k)
        assert np.max(np.abs(g - so[k])) <= 1e-6 * np.max(np.abs(so[k])), k
    s.close()
