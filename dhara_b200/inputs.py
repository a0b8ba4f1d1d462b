"""Seeded synthetic inputs for the benchmark and test domains.

The reference's example inputs are NetCDF4/HDF5 files that cannot be read in
this environment, and no public dataset exists for the path, so every domain
is generated from a seed: a Gaussian random field of micro-topography on a
plane slope, lognormal per-cell saturated conductivity, a hydrostatic initial
head with a water table, and a rain schedule.  The same arrays feed the GPU
library and the CPU oracle.
"""
from dataclasses import dataclass, field
import numpy as np

from . import _abi


@dataclass
class Domain:
    params: _abi.Params
    fields: dict            # name -> np.ndarray (float64) in reference layout
    int_fields: dict        # name -> np.ndarray (int32)
    rain_mm: np.ndarray     # mm per step, uniform over the domain, one entry per step
    seed: int = 0
    meta: dict = field(default_factory=dict)

    @property
    def ncells(self):
        p = self.params
        return p.nx * p.ny * p.nz


def gaussian_random_field(nx, ny, dx, dy, sigma, corr, rng):
    """Stationary field with Gaussian covariance sigma^2 exp(-(r/corr)^2),
    synthesised spectrally on a periodic grid padded to avoid wrap-around,
    then rescaled to the exact sample standard deviation sigma."""
    if sigma == 0.0:
        return np.zeros((ny, nx))
    pad = int(np.ceil(3 * corr / min(dx, dy)))
    mx, my = nx + pad, ny + pad
    kx = 2 * np.pi * np.fft.fftfreq(mx, d=dx)
    ky = 2 * np.pi * np.fft.fftfreq(my, d=dy)
    k2 = ky[:, None] ** 2 + kx[None, :] ** 2
    spec = np.exp(-k2 * corr * corr / 8.0)   # sqrt of the covariance's spectrum
    noise = rng.standard_normal((my, mx))
    f = np.real(np.fft.ifft2(np.fft.fft2(noise) * spec))[:ny, :nx]
    f = f - f.mean()
    s = f.std()
    return f * (sigma / s) if s > 0 else f


def make_domain(nx, ny, nz, *, dx=1.0, dy=1.0, dz=0.05, dt=60.0, seed=0,
                topo_sigma=0.05, topo_corr=3.0, slope=0.01,
                theta_s=0.45, theta_r=0.05, alpha=3.5, n=1.6, Ss=5e-4,
                ks_median=1e-5, ks_sigma_ln=0.5, water_table=0.8, manning=0.03,
                rain_mm_per_h=10.0, rain_hours=1.0, nsteps=60, dry_hours=0.0,
                per_cell_vg=False, am=0.25, overland_maxiter=2000, overland_tol=1e-12,
                **param_kw):
    """One seeded hillslope domain.  Surface: GRF(sigma, corr) on a plane that
    falls by `slope` per metre in +x.  Soil: van Genuchten (alpha in 1/m),
    ln Ks = ln(median) + sigma_ln * xi per cell.  Initial head hydrostatic
    with the water table `water_table` m below the surface.  Sides no-flux,
    bottom free drainage, top switching per the reference.

    am = 0.25 is the Picard relaxation of the reference's example config
    (WEIGHTED_SCHEME, examples/1-EBI/ebi.cfg); with the device default am = 0
    the modified Picard iteration oscillates with period two in the saturated
    layers of a domain with a water table and never converges.  The overland
    solve is converged tightly (the reference's 100-iteration cap leaves it
    unconverged on these domains)."""
    rng = np.random.default_rng(seed)
    p = _abi.make_params(nx, ny, nz, dx=dx, dy=dy, dz=dz, dt=dt,
                         alpha=alpha, n=n, theta_s=theta_s, theta_r=theta_r,
                         porosity=theta_s, Ss=Ss, am=am, overland_maxiter=overland_maxiter,
                         overland_tol=overland_tol, **param_kw)
    N, C = nx * ny * nz, nx * ny
    grf = gaussian_random_field(nx, ny, dx, dy, topo_sigma, topo_corr, rng)
    xs = np.arange(nx) * dx
    z = 1.0 + slope * (xs[-1] - xs)[None, :] + grf       # [ny, nx]
    ksat = ks_median * np.exp(ks_sigma_ln * rng.standard_normal(N))
    depth = (np.arange(nz) + 0.5) * dz
    psi = np.repeat(depth - water_table, C)               # k-major: k*C + j*nx + i
    f = dict(
        psi=psi.astype(np.float64),
        ksat=ksat.astype(np.float64),
        ztopo=z.reshape(-1).astype(np.float64),
        mann=np.full(C, manning),
        waterdepth=np.zeros(C),
        ponding=np.zeros(C),
        ppt=np.zeros(C),
        esoil=np.zeros(C),
        tr=np.zeros(C),
    )
    if per_cell_vg:
        f["alpha"] = np.full(N, alpha)
        f["nvg"] = np.full(N, n)
    ints = dict(
        bcw=np.ones(nz * ny, np.int32), bce=np.ones(nz * ny, np.int32),
        bcs=np.ones(nz * nx, np.int32), bcn=np.ones(nz * nx, np.int32),
        bcb=np.ones(C, np.int32), bct=np.ones(C, np.int32),
        procmap=np.zeros(C, np.int32),
    )
    per_step = rain_mm_per_h * dt / 3600.0
    rain_steps = int(round(rain_hours * 3600.0 / dt))
    rain = np.array([per_step if t < rain_steps else 0.0 for t in range(nsteps)])
    return Domain(params=p, fields=f, int_fields=ints, rain_mm=rain, seed=seed,
                  meta=dict(nx=nx, ny=ny, nz=nz, ks_sigma_ln=ks_sigma_ln))


# ---------------------------------------------------------------------------
# The benchmark workloads.

def plain_fp64_32x32x20(seed=1, **kw):
    """32x32x20 (dx=dy=1 m, dz=0.05 m); topography sigma 5 cm / corr 3 m on a
    1% slope; theta_s .45, theta_r .05, alpha 3.5 /m, n 1.6; Ks lognormal
    (median 1e-5 m/s, sigma_ln 0.5); water table 0.8 m; rain 10 mm/h for 1 h;
    Manning 0.03; dt 60 s x 60 steps; absolute Picard tol 1e-6 m; Krylov 1e-10."""
    args = dict(seed=seed, ks_sigma_ln=0.5, rain_mm_per_h=10.0, rain_hours=1.0, nsteps=60,
                picard_rule=_abi.PICARD_PSI_ABSOLUTE, picard_tol=1e-6, picard_maxiter=10,
                krylov_tol=1e-10, krylov_maxiter=200, precision=_abi.FP64)
    args.update(kw)
    return make_domain(32, 32, 20, **args)


def mixed_512x512x40(seed=2, nx=512, ny=512, nz=40, **kw):
    """512x512x40 single domain, Ks sigma_ln 1.0, rain 20 mm/h for 2 h then
    2 h recession, dt 60 s x 240 steps, FP32 inner solve + FP64 refinement."""
    args = dict(seed=seed, ks_sigma_ln=1.0, rain_mm_per_h=20.0, rain_hours=2.0, nsteps=240,
                picard_rule=_abi.PICARD_PSI_ABSOLUTE, picard_tol=1e-6, picard_maxiter=10,
                krylov_tol=1e-10, krylov_maxiter=200, precision=_abi.MIXED,
                theta_update=_abi.THETA_CONSERVATIVE)
    args.update(kw)
    return make_domain(nx, ny, nz, **args)


def adjoint_128x128x30(seed=5, nx=128, ny=128, nz=30, **kw):
    """The calibration domain: 128x128x30 with the 32x32x20 domain's physics
    (Ks sigma_ln 0.5, rain 10 mm/h for 1 h, water table 0.8 m), dt 60 s x 120
    steps, FP32 inner solve + FP64 refinement.  The Picard loop runs its full
    10 iterations every step (tolerance 1e-300): with a convergence test the
    number of iterations, and so the computed state, jumps when a parameter
    moves the error across the tolerance, and the loss is not differentiable
    at the scale of a finite-difference step."""
    args = dict(seed=seed, ks_sigma_ln=0.5, rain_mm_per_h=10.0, rain_hours=1.0, nsteps=120,
                picard_rule=_abi.PICARD_PSI_ABSOLUTE, picard_tol=1e-300, picard_maxiter=10,
                krylov_tol=1e-10, krylov_maxiter=200, precision=_abi.MIXED,
                theta_update=_abi.THETA_CONSERVATIVE)
    args.update(kw)
    return make_domain(nx, ny, nz, **args)


def ensemble(ndomains=256, seed=3, lo=(16, 16, 20), hi=(128, 128, 40), nsteps=120, **kw):
    """Independent domains of uneven size drawn uniformly between lo and hi,
    each with its own seed, Ks sigma_ln in [0.5, 1.5], alpha in [1, 5] /m,
    n in [1.3, 2.2] and rain intensity in [5, 40] mm/h for 1 h."""
    rng = np.random.default_rng(seed)
    out = []
    for d in range(ndomains):
        nx = int(rng.integers(lo[0], hi[0] + 1))
        ny = int(rng.integers(lo[1], hi[1] + 1))
        nz = int(rng.integers(lo[2], hi[2] + 1))
        args = dict(seed=int(rng.integers(0, 2**31 - 1)),
                    ks_sigma_ln=float(rng.uniform(0.5, 1.5)),
                    alpha=float(rng.uniform(1.0, 5.0)), n=float(rng.uniform(1.3, 2.2)),
                    rain_mm_per_h=float(rng.uniform(5.0, 40.0)), rain_hours=1.0, nsteps=nsteps,
                    picard_rule=_abi.PICARD_PSI_ABSOLUTE, picard_tol=1e-6, picard_maxiter=10,
                    krylov_tol=1e-10, krylov_maxiter=200, precision=_abi.MIXED,
                    theta_update=_abi.THETA_CONSERVATIVE)
        args.update(kw)
        out.append(make_domain(nx, ny, nz, **args))
    return out


def large_1024x1024x50(seed=4, **kw):
    """1024x1024x50, topography sigma 10 cm / corr 5 m on a 0.5% slope, Ks
    sigma_ln 1.0, dt 120 s; the 24 h triangular storm (peak 50 mm/h at hour 6,
    120 mm total) is applied through the per-step rain schedule."""
    nsteps = kw.pop("nsteps", 720)
    args = dict(seed=seed, dt=120.0, topo_sigma=0.10, topo_corr=5.0, slope=0.005,
                ks_sigma_ln=1.0, rain_mm_per_h=0.0, nsteps=nsteps,
                picard_rule=_abi.PICARD_PSI_ABSOLUTE, picard_tol=1e-6, picard_maxiter=10,
                krylov_tol=1e-10, krylov_maxiter=200, precision=_abi.MIXED,
                theta_update=_abi.THETA_CONSERVATIVE)
    args.update(kw)
    d = make_domain(1024, 1024, 50, **args)
    d.rain_mm = triangular_storm(nsteps, d.params.dt)
    return d


def triangular_storm(nsteps, dt, peak_mm_h=50.0, peak_h=6.0, total_mm=120.0):
    """Triangular hyetograph with the given peak and total depth; its base is
    2*total/peak hours long, starting at peak_h - rise."""
    base_h = 2.0 * total_mm / peak_mm_h
    rise = min(peak_h, base_h / 2.0)
    t0, t1 = peak_h - rise, peak_h - rise + base_h
    out = np.zeros(nsteps)
    for s in range(nsteps):
        tm = (s + 0.5) * dt / 3600.0
        if t0 <= tm <= peak_h:
            rate = peak_mm_h * (tm - t0) / (peak_h - t0)
        elif peak_h < tm <= t1:
            rate = peak_mm_h * (t1 - tm) / (t1 - peak_h)
        else:
            rate = 0.0
        out[s] = rate * dt / 3600.0
    return out
