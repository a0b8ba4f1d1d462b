"""FP64 CPU oracle of Dhara's integrated flow hot path -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
legs may import this package.  It wraps oracle/liboracle.so (built from
oracle/dhara_oracle.cc by oracle/Makefile) with ctypes.
"""
import ctypes as ct
import os
import subprocess

import numpy as np

from dhara_b200 import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
SOLVER_BICGSTAB, SOLVER_CG, SOLVER_PCG_COLUMN = 0, 1, 2

_lib = None


def build(force=False):
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ct.CDLL(LIB_PATH)
        P = ct.POINTER
        dp = P(ct.c_double)
        L.oracle_create.restype = ct.c_void_p
        L.oracle_create.argtypes = [P(_abi.Params)]
        L.oracle_destroy.argtypes = [ct.c_void_p]
        L.oracle_set_solvers.argtypes = [ct.c_void_p, ct.c_int, ct.c_int]
        L.oracle_set_threads.argtypes = [ct.c_int]
        L.oracle_get_threads.restype = ct.c_int
        L.oracle_upload.argtypes = [ct.c_void_p, ct.c_int, dp, ct.c_longlong]
        L.oracle_upload_int.argtypes = [ct.c_void_p, ct.c_int, P(ct.c_int), ct.c_longlong]
        L.oracle_download.argtypes = [ct.c_void_p, ct.c_int, dp, ct.c_longlong]
        L.oracle_set_roots.argtypes = [ct.c_void_p, dp, ct.c_int]
        for fn in ("oracle_psi_from_theta", "oracle_prepare", "oracle_overland_step"):
            getattr(L, fn).argtypes = [ct.c_void_p]
        L.oracle_subsurface_step.argtypes = [ct.c_void_p, dp]
        L.oracle_get_diagnostics.argtypes = [ct.c_void_p, P(_abi.Diagnostics)]
        L.oracle_van_genuchten.argtypes = [P(_abi.Params), dp, dp, dp, dp, ct.c_longlong, dp, dp, dp]
        L.oracle_van_genuchten_inverse.argtypes = [P(_abi.Params), dp, dp, dp, ct.c_longlong, dp]
        L.oracle_assemble.argtypes = [ct.c_void_p, dp, dp]
        L.oracle_update_k_overland.argtypes = [P(_abi.Params), dp, dp, dp, dp, dp, dp, dp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ct.POINTER(ct.c_double))


def set_threads(n):
    lib().oracle_set_threads(int(n))


def get_threads():
    return lib().oracle_get_threads()


class Oracle:
    """One domain of the reference model on the CPU, in FP64."""

    def __init__(self, params, solver3d=SOLVER_BICGSTAB, solver2d=SOLVER_CG):
        self.p = params
        self.h = lib().oracle_create(ct.byref(params))
        if not self.h:
            raise ValueError("oracle_create rejected the parameters")
        lib().oracle_set_solvers(self.h, solver3d, solver2d)

    def close(self):
        if self.h:
            lib().oracle_destroy(self.h)
            self.h = None

    __del__ = close

    def upload(self, name, arr):
        if name in _abi.FI:
            a = np.ascontiguousarray(arr, dtype=np.int32)
            rc = lib().oracle_upload_int(self.h, _abi.FI[name],
                                         a.ctypes.data_as(ct.POINTER(ct.c_int)), a.size)
        else:
            a = np.ascontiguousarray(arr, dtype=np.float64)
            rc = lib().oracle_upload(self.h, _abi.F[name], _dp(a), a.size)
        if rc != 0:
            raise ValueError(f"oracle upload of {name} failed ({rc})")

    def download(self, name):
        out = np.empty(_abi.extent(self.p, name), np.float64)
        rc = lib().oracle_download(self.h, _abi.F[name], _dp(out), out.size)
        if rc != 0:
            raise ValueError(f"oracle download of {name} failed ({rc})")
        return out

    def load(self, domain):
        for k, v in domain.fields.items():
            self.upload(k, v)
        for k, v in domain.int_fields.items():
            self.upload(k, v)

    def prepare(self):
        lib().oracle_prepare(self.h)

    def psi_from_theta(self):
        lib().oracle_psi_from_theta(self.h)

    def step(self, rain_mm=None):
        if rain_mm is None:
            rc = lib().oracle_subsurface_step(self.h, None)
        else:
            r = ct.c_double(float(rain_mm))
            rc = lib().oracle_subsurface_step(self.h, ct.pointer(r))
        if rc != 0:
            raise RuntimeError(f"oracle subsurface step failed ({rc})")
        rc = lib().oracle_overland_step(self.h)
        if rc != 0:
            raise RuntimeError(f"oracle overland step failed ({rc})")

    def diagnostics(self):
        d = _abi.Diagnostics()
        lib().oracle_get_diagnostics(self.h, ct.byref(d))
        return d.as_dict()

    def assemble(self):
        N = self.p.nx * self.p.ny * self.p.nz
        a = np.empty(7 * N)
        b = np.empty(N)
        lib().oracle_assemble(self.h, _dp(a), _dp(b))
        return a, b


def van_genuchten(params, psi, ksat, alpha=None, nvg=None):
    psi = np.ascontiguousarray(psi, np.float64)
    ksat = np.ascontiguousarray(ksat, np.float64)
    n = psi.size
    C, th, K = np.empty(n), np.empty(n), np.empty(n)
    a = None if alpha is None else np.ascontiguousarray(alpha, np.float64)
    m = None if nvg is None else np.ascontiguousarray(nvg, np.float64)
    lib().oracle_van_genuchten(ct.byref(params), _dp(psi), _dp(ksat),
                               _dp(a) if a is not None else None,
                               _dp(m) if m is not None else None, n, _dp(C), _dp(th), _dp(K))
    return C, th, K


def van_genuchten_inverse(params, theta, alpha=None, nvg=None):
    theta = np.ascontiguousarray(theta, np.float64)
    out = np.empty(theta.size)
    a = None if alpha is None else np.ascontiguousarray(alpha, np.float64)
    m = None if nvg is None else np.ascontiguousarray(nvg, np.float64)
    lib().oracle_van_genuchten_inverse(ct.byref(params), _dp(theta),
                                       _dp(a) if a is not None else None,
                                       _dp(m) if m is not None else None, theta.size, _dp(out))
    return out


def update_k_overland(params, H, h, mann):
    C = params.nx * params.ny
    H, h, mann = (np.ascontiguousarray(x, np.float64) for x in (H, h, mann))
    kw, ke, ks, kn = (np.empty(C) for _ in range(4))
    lib().oracle_update_k_overland(ct.byref(params), _dp(H), _dp(h), _dp(mann),
                                   _dp(kw), _dp(ke), _dp(ks), _dp(kn))
    return kw, ke, ks, kn


def run(domain, nsteps=None, solver3d=SOLVER_BICGSTAB, solver2d=SOLVER_CG, record=()):
    """Runs a domain for nsteps with its rain schedule; returns the final
    state, diagnostics and any recorded per-step fields."""
    o = Oracle(domain.params, solver3d, solver2d)
    o.load(domain)
    o.prepare()
    n = len(domain.rain_mm) if nsteps is None else nsteps
    rec = {k: [] for k in record}
    for t in range(n):
        o.step(domain.rain_mm[t] if t < len(domain.rain_mm) else 0.0)
        for k in record:
            rec[k].append(o.download(k))
    state = {k: o.download(k) for k in ("psi", "theta", "ponding", "waterelev", "K")}
    diag = o.diagnostics()
    o.close()
    return state, diag, rec


# ---------------------------------------------------------------------------
# Per-kernel records (oracle/kernel_io.h) and the reference's own kernels
# compiled from its sources (oracle/_ref/libdhara_refkernels.so, built by
# `make -C oracle ref` where the reference tree is available).

_dp_t = ct.POINTER(ct.c_double)
_ip_t = ct.POINTER(ct.c_int)


class AsmIO(ct.Structure):
    _fields_ = [("nx", ct.c_int), ("ny", ct.c_int), ("nz", ct.c_int), ("nproc", ct.c_int)] + [
        (n, _dp_t) for n in ("psinp1m", "psin", "thetanp1m", "thetan", "knp1m", "cnp1m")] + [
        (n, _ip_t) for n in ("wbc", "ebc", "sbc", "nbc", "tbc", "bbc")] + [
        (n, _dp_t) for n in ("psi_w", "psi_e", "psi_s", "psi_n", "psi_t", "psi_b",
                             "qw", "qe", "qs", "qn", "qt", "qb", "tr")] + [
        ("procmap", _ip_t), ("root", _dp_t), ("a3d", _dp_t), ("rhs", _dp_t)]


class FluxIO(ct.Structure):
    _fields_ = [("nx", ct.c_int), ("ny", ct.c_int), ("nz", ct.c_int), ("nproc", ct.c_int)] + [
        (n, _dp_t) for n in ("knp1m", "psinp1mp1", "psin", "thetanp1mp1", "thetan", "E_soil", "TR", "qss",
                             "bcqw", "bcqe", "bcqs", "bcqn", "bcqt", "bcqb")] + [
        (n, _ip_t) for n in ("wbc", "ebc", "sbc", "nbc", "tbc", "bbc", "procmap")] + [
        ("root", _dp_t)] + [
        (n, _dp_t) for n in ("quflux", "qdflux", "qwflux", "qeflux", "qsflux", "qnflux",
                             "dtheta", "transp", "evapo", "ssflux")]


class TopIO(ct.Structure):
    _fields_ = [("nx", ct.c_int), ("ny", ct.c_int)] + [
        (n, _dp_t) for n in ("ph_in", "psinp1m", "knp1m", "ppt", "et", "ksat", "thetan", "psinp1mp1",
                             "psi_top", "hpoten", "qcapa", "topqflux", "qss", "ph_out")] + [
        ("topbc", _ip_t)]


class OlfIO(ct.Structure):
    _fields_ = [("nx", ct.c_int), ("ny", ct.c_int)] + [
        (n, _dp_t) for n in ("waterdepth", "ztopo", "mann", "waterelev", "kw", "ke", "ks", "kn", "a2d",
                             "rhs2d", "waterdepth_out")]


def fill(record, arrays):
    """Points the record's pointer fields at the numpy arrays (kept alive by
    the caller) and sets the integer fields."""
    for name, typ in record._fields_:
        if name in arrays:
            v = arrays[name]
            if typ is ct.c_int:
                setattr(record, name, int(v))
            elif typ is _ip_t:
                setattr(record, name, v.ctypes.data_as(_ip_t))
            else:
                setattr(record, name, v.ctypes.data_as(_dp_t))
    return record


REF_LIB_PATH = os.path.join(HERE, "_ref", "libdhara_refkernels.so")
_ref = None


def ref_lib():
    """The reference's own kernels (None when they were not built)."""
    global _ref
    if _ref is None and os.path.exists(REF_LIB_PATH):
        R = ct.CDLL(REF_LIB_PATH)
        P = ct.POINTER
        R.ref_k_van_genuchten.argtypes = [P(_abi.Params), ct.c_longlong, _dp_t, _dp_t, _dp_t, _dp_t, _dp_t]
        R.ref_k_vg_inverse.argtypes = [P(_abi.Params), ct.c_longlong, _dp_t, _dp_t]
        R.ref_k_top.argtypes = [P(_abi.Params), P(TopIO)]
        R.ref_k_infiltration.argtypes = [P(_abi.Params), P(TopIO)]
        R.ref_k_assemble.argtypes = [P(_abi.Params), P(AsmIO)]
        R.ref_k_water_flux.argtypes = [P(_abi.Params), P(FluxIO)]
        R.ref_k_overland_setup.argtypes = [P(_abi.Params), P(OlfIO)]
        R.ref_k_water_depth.argtypes = [P(_abi.Params), P(OlfIO)]
        _ref = R
    return _ref


def _k(name, *argtypes):
    fn = getattr(lib(), name)
    fn.argtypes = list(argtypes)
    fn.restype = None
    return fn


def k_functions():
    """The oracle's stateless per-kernel restatements."""
    P = ct.POINTER
    return dict(
        assemble=_k("oracle_k_assemble", P(_abi.Params), P(AsmIO)),
        estimate_fluxes=_k("oracle_k_estimate_fluxes", P(_abi.Params), P(TopIO)),
        identify_top=_k("oracle_k_identify_top", P(_abi.Params), P(TopIO)),
        infiltration=_k("oracle_k_infiltration", P(_abi.Params), P(TopIO)),
        water_flux=_k("oracle_k_water_flux", P(_abi.Params), P(FluxIO)),
        overland_setup=_k("oracle_k_overland_setup", P(_abi.Params), P(OlfIO)),
        water_depth=_k("oracle_k_water_depth", P(_abi.Params), P(OlfIO)),
    )
