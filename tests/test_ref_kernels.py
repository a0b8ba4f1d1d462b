"""Pins the oracle against the reference's own kernels.

The reference's kernel files (src/global.cu, src/subsurface.cu,
src/overland.cu) are compiled from their sources by `make -C oracle ref`
(stub MPI/netCDF/Eigen/CUSP headers; the CUSP-based host drivers are never
called) into oracle/_ref/libdhara_refkernels.so.  Each test runs one of the
reference's __global__ kernels on the GPU and the oracle's restatement of it
(oracle_k_*) on the CPU, on the same seeded inputs, and requires agreement to
FP64 rounding (a few ulp; pow differs between CUDA and glibc in the last bit).
Launch shapes are chosen so that the reference kernels' in-loop
__syncthreads() is reached uniformly by every thread of a block.
"""
import ctypes as ct

import numpy as np
import pytest

import oracle
from dhara_b200 import _abi

pytestmark = pytest.mark.gpu

NX, NY, NZ, NPROC = 16, 8, 5, 3          # N = 640 (multiple of 64), C = 128 (multiple of 32)
N, C, WE, SN = NX * NY * NZ, NX * NY, NZ * NY, NZ * NX


@pytest.fixture(scope="module")
def ref(gpu):
    R = oracle.ref_lib()
    if R is None:
        pytest.skip("reference kernels not built (make -C oracle ref needs the reference tree)")
    return R


@pytest.fixture(scope="module")
def params():
    return _abi.make_params(NX, NY, NZ, dx=1.2, dy=0.9, dz=0.07, dt=600.0, alpha=3.1, n=1.7,
                            theta_s=0.43, theta_r=0.06, porosity=0.43, Ss=4e-4, am=0.0)


def close(a, b, rtol=1e-12, atol=1e-300):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = np.maximum(np.abs(b), np.max(np.abs(b)) * 1e-6 + atol)
    return float(np.max(np.abs(a - b) / scale)) if a.size else 0.0


def rng_fields(seed):
    r = np.random.default_rng(seed)
    psi = r.uniform(-2.0, 0.3, N)
    psi[::17] = 0.0
    return r, psi


def test_van_genuchten(ref, params):
    r, psi = rng_fields(1)
    ksat = r.lognormal(np.log(1e-5), 0.8, N)
    out_r = [np.empty(N) for _ in range(3)]
    dp = lambda a: a.ctypes.data_as(ct.POINTER(ct.c_double))
    assert ref.ref_k_van_genuchten(ct.byref(params), N, dp(psi), dp(ksat), *[dp(a) for a in out_r]) == 0
    C_o, th_o, K_o = oracle.van_genuchten(params, psi, ksat)
    assert close(out_r[0], C_o) < 1e-12
    assert close(out_r[1], th_o) < 1e-13
    assert close(out_r[2], K_o) < 1e-12


def test_van_genuchten_inverse(ref, params):
    r = np.random.default_rng(2)
    theta = r.uniform(params.theta_r + 1e-3, params.theta_s, N)
    theta[::11] = params.theta_s
    psi_r = np.empty(N)
    dp = lambda a: a.ctypes.data_as(ct.POINTER(ct.c_double))
    assert ref.ref_k_vg_inverse(ct.byref(params), N, dp(theta), dp(psi_r)) == 0
    assert close(psi_r, oracle.van_genuchten_inverse(params, theta)) < 1e-12


def top_arrays(seed):
    r = np.random.default_rng(seed)
    a = dict(nx=NX, ny=NY,
             ph_in=np.where(r.random(C) < 0.5, r.uniform(0, 0.02, C), 0.0),
             psinp1m=r.uniform(-1.5, 0.1, C), knp1m=r.lognormal(np.log(1e-6), 1.0, C),
             ppt=r.uniform(0, 3.0, C), et=r.uniform(0, 1e-4, C), ksat=r.lognormal(np.log(1e-5), 0.7, C),
             thetan=r.uniform(0.1, 0.43, C), psinp1mp1=r.uniform(-1.5, 0.1, C), psi_top=r.uniform(-1, 0, C))
    for k in ("hpoten", "qcapa", "topqflux", "qss", "ph_out"):
        a[k] = np.zeros(C)
    a["topbc"] = np.zeros(C, np.int32)
    return a


def test_top_boundary_and_infiltration(ref, params):
    kf = oracle.k_functions()
    ar = top_arrays(3)
    ao = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in ar.items()}
    io_r = oracle.fill(oracle.TopIO(), ar)
    io_o = oracle.fill(oracle.TopIO(), ao)
    assert ref.ref_k_top(ct.byref(params), ct.byref(io_r)) == 0
    kf["estimate_fluxes"](ct.byref(params), ct.byref(io_o))
    kf["identify_top"](ct.byref(params), ct.byref(io_o))
    for k in ("hpoten", "qcapa", "topqflux"):
        assert close(ar[k], ao[k]) < 1e-13, k
    assert np.array_equal(ar["topbc"], ao["topbc"])
    assert ref.ref_k_infiltration(ct.byref(params), ct.byref(io_r)) == 0
    kf["infiltration"](ct.byref(params), ct.byref(io_o))
    assert close(ar["qss"], ao["qss"]) < 1e-13
    assert close(ar["ph_out"], ao["ph_out"]) < 1e-13


def asm_arrays(seed, dirichlet):
    r = np.random.default_rng(seed)
    types = lambda n: (r.random(n) < 0.4).astype(np.int32) ^ 1 if dirichlet else np.ones(n, np.int32)
    a = dict(nx=NX, ny=NY, nz=NZ, nproc=NPROC,
             psinp1m=r.uniform(-2, 0.2, N), psin=r.uniform(-2, 0.2, N), thetanp1m=r.uniform(0.07, 0.43, N),
             thetan=r.uniform(0.07, 0.43, N), knp1m=r.lognormal(np.log(1e-6), 1.5, N),
             cnp1m=r.uniform(0, 0.5, N),
             wbc=types(WE), ebc=types(WE), sbc=types(SN), nbc=types(SN),
             tbc=np.ones(C, np.int32), bbc=types(C),
             psi_w=r.uniform(-1, 0, WE), psi_e=r.uniform(-1, 0, WE), psi_s=r.uniform(-1, 0, SN),
             psi_n=r.uniform(-1, 0, SN), psi_t=r.uniform(-1, 0, C), psi_b=r.uniform(-1, 0, C),
             qw=r.uniform(-1e-6, 1e-6, WE), qe=r.uniform(-1e-6, 1e-6, WE), qs=r.uniform(-1e-6, 1e-6, SN),
             qn=r.uniform(-1e-6, 1e-6, SN), qt=r.uniform(0, 3e-6, C), qb=np.zeros(C),
             tr=np.where(r.random(C) < 0.5, r.uniform(0, 1e-4, C), 0.0),
             procmap=r.integers(0, NPROC, C).astype(np.int32), root=r.uniform(0, 0.3, NPROC * NZ),
             a3d=np.zeros(7 * N), rhs=np.zeros(N))
    return a


@pytest.mark.parametrize("dirichlet", [False, True])
def test_assembly(ref, params, dirichlet):
    kf = oracle.k_functions()
    ar = asm_arrays(4 + dirichlet, dirichlet)
    ao = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in ar.items()}
    assert ref.ref_k_assemble(ct.byref(params), ct.byref(oracle.fill(oracle.AsmIO(), ar))) == 0
    kf["assemble"](ct.byref(params), ct.byref(oracle.fill(oracle.AsmIO(), ao)))
    assert close(ar["a3d"], ao["a3d"]) < 1e-13
    assert close(ar["rhs"], ao["rhs"]) < 1e-12
    assert close(ar["qb"], ao["qb"]) < 1e-15


def test_water_flux(ref, params):
    kf = oracle.k_functions()
    r = np.random.default_rng(6)
    a = dict(nx=NX, ny=NY, nz=NZ, nproc=NPROC,
             knp1m=r.lognormal(np.log(1e-6), 1.5, N), psinp1mp1=r.uniform(-2, 0.2, N), psin=r.uniform(-2, 0.2, N),
             thetanp1mp1=r.uniform(0.07, 0.43, N), thetan=r.uniform(0.07, 0.43, N),
             E_soil=r.uniform(0, 1e-4, C), TR=np.where(r.random(C) < 0.5, r.uniform(0, 1e-4, C), 0.0),
             qss=r.uniform(0, 1e-6, C), bcqw=r.uniform(-1e-6, 1e-6, WE), bcqe=r.uniform(-1e-6, 1e-6, WE),
             bcqs=r.uniform(-1e-6, 1e-6, SN), bcqn=r.uniform(-1e-6, 1e-6, SN), bcqt=r.uniform(0, 3e-6, C),
             bcqb=r.lognormal(np.log(1e-6), 1.0, C),
             wbc=np.ones(WE, np.int32), ebc=np.ones(WE, np.int32), sbc=np.ones(SN, np.int32),
             nbc=np.ones(SN, np.int32), tbc=np.ones(C, np.int32), bbc=np.ones(C, np.int32),
             procmap=r.integers(0, NPROC, C).astype(np.int32), root=r.uniform(0, 0.3, NPROC * NZ))
    outs = ("quflux", "qdflux", "qwflux", "qeflux", "qsflux", "qnflux", "dtheta", "transp", "evapo", "ssflux")
    ar = dict(a, **{k: np.zeros(N) for k in outs})
    ao = dict(a, **{k: np.zeros(N) for k in outs})
    assert ref.ref_k_water_flux(ct.byref(params), ct.byref(oracle.fill(oracle.FluxIO(), ar))) == 0
    kf["water_flux"](ct.byref(params), ct.byref(oracle.fill(oracle.FluxIO(), ao)))
    for k in outs:
        if k == "evapo":
            continue  # the reference never writes it
        assert close(ar[k], ao[k]) < 1e-13, k


def test_overland_setup_and_depth(ref, params):
    kf = oracle.k_functions()
    r = np.random.default_rng(7)
    z = 1.0 + 0.01 * np.arange(C) % 0.3 + r.normal(0, 0.02, C)
    h = np.where(r.random(C) < 0.6, r.uniform(0, 0.01, C), 0.0)
    h[::9] = 5e-6   # below WATERDEPTH_MINIMUM: the K0 branch
    base = dict(nx=NX, ny=NY, waterdepth=h, ztopo=z, mann=r.uniform(0.02, 0.05, C))
    outs = dict(waterelev=C, kw=C, ke=C, ks=C, kn=C, a2d=5 * C, rhs2d=C, waterdepth_out=C)
    ar = dict(base, **{k: np.zeros(n) for k, n in outs.items()})
    ao = dict(base, **{k: np.zeros(n) for k, n in outs.items()})
    io_r, io_o = oracle.fill(oracle.OlfIO(), ar), oracle.fill(oracle.OlfIO(), ao)
    assert ref.ref_k_overland_setup(ct.byref(params), ct.byref(io_r)) == 0
    kf["overland_setup"](ct.byref(params), ct.byref(io_o))
    for k in ("waterelev", "kw", "ke", "ks", "kn", "a2d", "rhs2d"):
        assert close(ar[k], ao[k]) < 1e-12, k
    # depth clip on a perturbed elevation (some cells below ground)
    ar["waterelev"][:] = z + r.normal(0, 0.01, C)
    ao["waterelev"][:] = ar["waterelev"]
    assert ref.ref_k_water_depth(ct.byref(params), ct.byref(io_r)) == 0
    kf["water_depth"](ct.byref(params), ct.byref(io_o))
    assert np.array_equal(ar["waterdepth_out"], ao["waterdepth_out"])
