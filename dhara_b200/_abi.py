"""ctypes mirror of include/dhara_gpu.h (structs, enums, field ids).

The layouts here must match the C header byte for byte; tests/test_abi.py
checks the sizes against the compiled library.
"""
import ctypes as ct

DHARA_OK = 0
STATUS_NAMES = {
    0: "OK", 1: "INVALID", 2: "CUDA", 3: "NOMEM", 4: "UNSUPPORTED",
    5: "NONFINITE", 6: "TIMEOUT", 7: "STATE",
}

FP64, MIXED = 0, 1
PICARD_PSI_RELATIVE, PICARD_THETA_RELATIVE, PICARD_PSI_ABSOLUTE = 0, 1, 2
THETA_REFERENCE, THETA_FINAL, THETA_CONSERVATIVE = 0, 1, 2

# field ids (dhara_field)
F = dict(
    psi=0, theta=1, ksat=2, alpha=3, nvg=4, K=5, C=6, theta_new=7,
    ztopo=16, mann=17, waterdepth=18, waterelev=19, ponding=20, ppt=21, esoil=22, tr=23,
    hpoten=24, qtop=25,
    bcqw=32, bcqe=33, bcqs=34, bcqn=35, bcqb=36,
    bcpsiw=40, bcpsie=41, bcpsis=42, bcpsin=43, bcpsib=44,
)
FI = dict(bcw=64, bce=65, bcs=66, bcn=67, bcb=68, bct=69, procmap=70)

# which extent each field has: "N" cells, "C" columns, "WE" nz*ny, "SN" nz*nx
FIELD_EXTENT = {
    **{k: "N" for k in ("psi", "theta", "ksat", "alpha", "nvg", "K", "C", "theta_new")},
    **{k: "C" for k in ("ztopo", "mann", "waterdepth", "waterelev", "ponding", "ppt", "esoil",
                         "tr", "hpoten", "qtop", "bcqb", "bcpsib", "bcb", "bct", "procmap")},
    **{k: "WE" for k in ("bcqw", "bcqe", "bcpsiw", "bcpsie", "bcw", "bce")},
    **{k: "SN" for k in ("bcqs", "bcqn", "bcpsis", "bcpsin", "bcs", "bcn")},
}


class Params(ct.Structure):
    _fields_ = [
        ("struct_size", ct.c_int32), ("nx", ct.c_int32), ("ny", ct.c_int32), ("nz", ct.c_int32),
        ("dx", ct.c_double), ("dy", ct.c_double), ("dz", ct.c_double), ("dt", ct.c_double),
        ("alpha", ct.c_double), ("n", ct.c_double), ("theta_s", ct.c_double),
        ("theta_r", ct.c_double), ("porosity", ct.c_double), ("Ss", ct.c_double),
        ("airdry", ct.c_double), ("psimin", ct.c_double), ("am", ct.c_double),
        ("delta", ct.c_double), ("hmin", ct.c_double), ("hcri", ct.c_double), ("K0", ct.c_double),
        ("sec_p_mm2dt_p_m", ct.c_double),
        ("picard_maxiter", ct.c_int32), ("picard_rule", ct.c_int32), ("picard_tol", ct.c_double),
        ("krylov_maxiter", ct.c_int32), ("theta_update", ct.c_int32), ("krylov_tol", ct.c_double),
        ("overland_maxiter", ct.c_int32), ("precision", ct.c_int32), ("overland_tol", ct.c_double),
        ("inner_tol", ct.c_double), ("inner_maxiter", ct.c_int32), ("closure_fp32", ct.c_int32),
        ("record_branches", ct.c_int32), ("overland_solver", ct.c_int32), ("dt_halvings", ct.c_int32),
        ("reserved_i", ct.c_int32 * 3), ("reserved_d", ct.c_double * 8),
    ]


class Diagnostics(ct.Structure):
    _fields_ = [
        ("steps", ct.c_int64), ("picard_iters_total", ct.c_int64),
        ("krylov_iters_total", ct.c_int64), ("refine_iters_total", ct.c_int64),
        ("overland_iters_total", ct.c_int64),
        ("picard_iters_last", ct.c_int32), ("krylov_iters_last", ct.c_int32),
        ("picard_nonconverged", ct.c_int32), ("krylov_nonconverged", ct.c_int32),
        ("overland_nonconverged", ct.c_int32), ("nonfinite", ct.c_int32),
        ("mb_subsurface_last", ct.c_double), ("mb_subsurface_cum", ct.c_double),
        ("storage_change_cum", ct.c_double), ("top_inflow_cum", ct.c_double),
        ("bottom_outflow_cum", ct.c_double), ("rain_cum", ct.c_double),
        ("overland_boundary_out_cum", ct.c_double), ("overland_clip_cum", ct.c_double),
        ("ponded_volume", ct.c_double), ("picard_err_last", ct.c_double),
        ("krylov_relres_last", ct.c_double), ("branch_signature", ct.c_uint64),
        ("substeps_total", ct.c_int64), ("step_attempts_total", ct.c_int64), ("reserved", ct.c_double * 3),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved"}


class LaunchConfig(ct.Structure):
    _fields_ = [("krylov_blocks_per_sm", ct.c_int32), ("overland_resident", ct.c_int32),
                ("overland_blocks_per_sm", ct.c_int32), ("tile_shape", ct.c_int32),
                ("krylov_ms", ct.c_double), ("overland_ms", ct.c_double), ("fused_step", ct.c_int32),
                ("pad", ct.c_int32)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_ if n != "pad"}


class ConfigBC(ct.Structure):
    """dhara_config_bc: faces top, bottom, north, south, east, west."""
    _fields_ = [("type", ct.c_int32 * 6), ("psi", ct.c_double * 6), ("flux", ct.c_double * 6),
                ("found", ct.c_int32), ("pad", ct.c_int32)]


class AdjointDesc(ct.Structure):
    _fields_ = [
        ("struct_size", ct.c_int32), ("nsteps", ct.c_int32), ("checkpoint_every", ct.c_int32),
        ("pad", ct.c_int32), ("theta_target", ct.POINTER(ct.c_double)), ("q_target", ct.POINTER(ct.c_double)),
        ("w_q", ct.c_double), ("reserved", ct.c_double * 4),
    ]


def make_params(nx, ny, nz, dx=1.0, dy=1.0, dz=0.05, dt=60.0, **kw):
    """Parameters with the reference's device defaults (include/devconst.h:6-31,
    converted to SI: alpha 0.02 /cm -> 2.0 /m, dt in seconds) overridden by kw."""
    p = Params()
    p.struct_size = ct.sizeof(Params)
    p.nx, p.ny, p.nz = nx, ny, nz
    p.dx, p.dy, p.dz, p.dt = dx, dy, dz, dt
    defaults = dict(
        alpha=2.0, n=1.8, theta_s=0.45, theta_r=0.1, porosity=0.45, Ss=5e-4,
        airdry=-5.0, psimin=5e-3, am=0.0,
        delta=1e-7, hmin=1e-5, hcri=0.0, K0=1e-5,
        sec_p_mm2dt_p_m=dt / 1000.0,
        picard_maxiter=10, picard_rule=PICARD_PSI_RELATIVE, picard_tol=1e-8,
        krylov_maxiter=100, theta_update=THETA_REFERENCE, krylov_tol=1e-8,
        overland_maxiter=100, precision=FP64, overland_tol=1e-9,
        inner_tol=1e-4, inner_maxiter=60, closure_fp32=0,
    )
    defaults.update(kw)
    for k, v in defaults.items():
        setattr(p, k, v)
    return p


def extent(p, field):
    e = FIELD_EXTENT[field]
    if e == "N":
        return p.nx * p.ny * p.nz
    if e == "C":
        return p.nx * p.ny
    if e == "WE":
        return p.nz * p.ny
    return p.nz * p.nx
