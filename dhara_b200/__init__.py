"""dhara_b200 -- B200-native solver for Dhara's integrated surface-subsurface
flow hot path (3D mixed-form Richards + 2D diffusive-wave overland).

The compute lives in the CUDA library libdhara_b200.so behind the C ABI of
include/dhara_gpu.h.  This module is a thin ctypes mirror of that ABI for
Python callers (tests, benchmarks, notebooks); there is no CPU path: if the
library cannot be loaded, every entry point raises.
"""
import ctypes as ct
import os

import numpy as np

from . import _abi
from ._abi import (FP64, MIXED, PICARD_PSI_RELATIVE, PICARD_THETA_RELATIVE, PICARD_PSI_ABSOLUTE,
                   THETA_REFERENCE, THETA_FINAL, THETA_CONSERVATIVE, Params, Diagnostics, make_params)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdhara_b200.so")

KERNELS = {"krylov": 0, "assemble": 1, "picard_check": 2, "epilogue": 3, "overland_solve": 4,
           "overland_aux": 5, "prologue": 6, "adjoint": 7, "step": 8}

_lib = None


class DharaError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"dhara error {code} ({_abi.STATUS_NAMES.get(code, '?')}): {msg}")
        self.code = code


def lib():
    """Loads libdhara_b200.so (building it first if only the sources exist)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _build
        _build.build()
    L = ct.CDLL(LIB_PATH)
    P = ct.POINTER
    vp, dp, i64p = ct.c_void_p, P(ct.c_double), P(ct.c_int64)
    sig = {
        "dhara_abi_version": (ct.c_int, []),
        "dhara_last_error": (ct.c_char_p, []),
        "dhara_default_params": (None, [P(Params), ct.c_int, ct.c_int, ct.c_int, ct.c_double,
                                        ct.c_double, ct.c_double, ct.c_double]),
        "dhara_create": (ct.c_int, [P(Params), ct.c_int, ct.c_int, P(vp)]),
        "dhara_destroy": (ct.c_int, [vp]),
        "dhara_upload": (ct.c_int, [vp, ct.c_int, ct.c_int, dp, ct.c_int64]),
        "dhara_upload_int": (ct.c_int, [vp, ct.c_int, ct.c_int, P(ct.c_int32), ct.c_int64]),
        "dhara_download": (ct.c_int, [vp, ct.c_int, ct.c_int, dp, ct.c_int64]),
        "dhara_set_roots": (ct.c_int, [vp, ct.c_int, dp, ct.c_int]),
        "dhara_set_rain_schedule": (ct.c_int, [vp, ct.c_int, dp, ct.c_int]),
        "dhara_psi_from_theta": (ct.c_int, [vp]),
        "dhara_prepare": (ct.c_int, [vp]),
        "dhara_subsurface_step": (ct.c_int, [vp]),
        "dhara_overland_step": (ct.c_int, [vp]),
        "dhara_step": (ct.c_int, [vp, ct.c_int, ct.c_int]),
        "dhara_synchronize": (ct.c_int, [vp]),
        "dhara_get_diagnostics": (ct.c_int, [vp, ct.c_int, P(Diagnostics)]),
        "dhara_get_stream": (ct.c_int, [vp, P(vp)]),
        "dhara_set_kernel_timing": (ct.c_int, [vp, ct.c_int]),
        "dhara_get_kernel_timing": (ct.c_int, [vp, ct.c_int, i64p, dp]),
        "dhara_reset_kernel_timing": (ct.c_int, [vp]),
        "dhara_get_launch_count": (ct.c_int, [vp, i64p]),
        "dhara_get_krylov_traffic": (ct.c_int, [vp, dp, i64p]),
        "dhara_adjoint": (ct.c_int, [vp, P(_abi.AdjointDesc), dp, dp, dp, dp]),
        "dhara_get_params": (ct.c_int, [vp, ct.c_int, P(Params)]),
        "dhara_enable_statistics": (ct.c_int, [vp, ct.c_int]),
        "dhara_autotune": (ct.c_int, [vp, ct.c_int, P(_abi.LaunchConfig)]),
        "dhara_get_launch_config": (ct.c_int, [vp, P(_abi.LaunchConfig)]),
        "dhara_set_launch_config": (ct.c_int, [vp, P(_abi.LaunchConfig)]),
        "dhara_get_statistics": (ct.c_int, [vp, ct.c_int, i64p, dp, dp, dp]),
        "dhara_snapshot": (ct.c_int, [vp, ct.c_int, dp, dp, dp, dp]),
        "dhara_snapshot_wait": (ct.c_int, [vp]),
        "dhara_params_from_config": (ct.c_int, [ct.c_char_p, ct.c_int, ct.c_int, ct.c_int, P(Params),
                                                P(_abi.ConfigBC)]),
        "dhara_apply_boundary_config": (ct.c_int, [vp, ct.c_int, P(_abi.ConfigBC)]),
        "dhara_checkpoint_size": (ct.c_int, [vp, i64p]),
        "dhara_checkpoint": (ct.c_int, [vp, vp, ct.c_int64]),
        "dhara_restore": (ct.c_int, [vp, vp, ct.c_int64]),
        "dhara_selftest_bounded_wait": (ct.c_int, [ct.c_int, ct.c_double, P(ct.c_int)]),
        "dhara_write_netcdf_state": (ct.c_int, [ct.c_char_p, ct.c_char_p, ct.c_int, ct.c_int, ct.c_int,
                                                dp, dp, dp, dp]),
        "dhara_write_netcdf_statistics": (ct.c_int, [ct.c_char_p, ct.c_char_p, ct.c_int, ct.c_int, dp, dp, dp]),
        "dhara_save_netcdf_state": (ct.c_int, [vp, ct.c_int, ct.c_char_p, ct.c_char_p]),
        "dhara_save_netcdf_statistics": (ct.c_int, [vp, ct.c_int, ct.c_char_p, ct.c_char_p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _check(rc):
    if rc != 0:
        raise DharaError(rc, lib().dhara_last_error().decode())


def default_params(nx, ny, nz, dx, dy, dz, dt):
    p = Params()
    lib().dhara_default_params(ct.byref(p), nx, ny, nz, dx, dy, dz, dt)
    return p


def _dp(a):
    return a.ctypes.data_as(ct.POINTER(ct.c_double))


FACES = ("top", "bottom", "north", "south", "east", "west")


def params_from_config(path, nx, ny, nz):
    """The reference's configuration file (src/io.cc:236-274, src/host.cc:93-112)
    as dhara_params plus per-face boundary settings {face: (type, psi, flux)}."""
    p = Params()
    bc = _abi.ConfigBC()
    _check(lib().dhara_params_from_config(os.fsencode(path), nx, ny, nz, ct.byref(p), ct.byref(bc)))
    faces = {f: (bc.type[i], bc.psi[i], bc.flux[i]) for i, f in enumerate(FACES)}
    return p, faces, bc


class Solver:
    """One handle: ndomains independent domains advanced together on one GPU."""

    def __init__(self, params, device=0):
        plist = list(params) if isinstance(params, (list, tuple)) else [params]
        arr = (Params * len(plist))(*plist)
        h = ct.c_void_p()
        _check(lib().dhara_create(arr, len(plist), device, ct.byref(h)))
        self.h = h
        self.params = plist

    def close(self):
        if getattr(self, "h", None):
            lib().dhara_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- data
    def upload(self, name, arr, domain=0):
        if name in _abi.FI:
            a = np.ascontiguousarray(arr, dtype=np.int32)
            _check(lib().dhara_upload_int(self.h, domain, _abi.FI[name],
                                          a.ctypes.data_as(ct.POINTER(ct.c_int32)), a.size))
        else:
            a = np.ascontiguousarray(arr, dtype=np.float64)
            _check(lib().dhara_upload(self.h, domain, _abi.F[name], _dp(a), a.size))

    def download(self, name, domain=0):
        out = np.empty(_abi.extent(self.params[domain], name), np.float64)
        _check(lib().dhara_download(self.h, domain, _abi.F[name], _dp(out), out.size))
        return out

    def load(self, dom, domain=0, schedule=True):
        """Uploads a dhara_b200.inputs.Domain (fields, BC types, rain schedule)."""
        for k, v in dom.fields.items():
            self.upload(k, v, domain)
        for k, v in dom.int_fields.items():
            if k == "procmap":
                continue
            self.upload(k, v, domain)
        if schedule and len(dom.rain_mm):
            self.set_rain_schedule(dom.rain_mm, domain)

    def autotune(self, trial_steps=2):
        """Times the persistent solvers' block schedules on this handle's data
        (state restored afterwards) and keeps the fastest."""
        c = _abi.LaunchConfig()
        _check(lib().dhara_autotune(self.h, int(trial_steps), ct.byref(c)))
        return c.as_dict()

    def launch_config(self):
        c = _abi.LaunchConfig()
        _check(lib().dhara_get_launch_config(self.h, ct.byref(c)))
        return c.as_dict()

    def set_launch_config(self, krylov_blocks_per_sm, overland_resident, overland_blocks_per_sm, tile_shape=None,
                          fused_step=None):
        """Sets the block schedule; tile_shape 0 (per domain), 1 (32 x 4) or 2
        (16 x 8), fused_step 0/1; None keeps the current value."""
        cur = self.launch_config()
        c = _abi.LaunchConfig()
        c.krylov_blocks_per_sm, c.overland_resident = krylov_blocks_per_sm, overland_resident
        c.overland_blocks_per_sm = overland_blocks_per_sm
        c.tile_shape = cur["tile_shape"] if tile_shape is None else tile_shape
        c.fused_step = cur["fused_step"] if fused_step is None else fused_step
        _check(lib().dhara_set_launch_config(self.h, ct.byref(c)))

    def enable_statistics(self, max_steps):
        _check(lib().dhara_enable_statistics(self.h, int(max_steps)))

    def statistics(self, domain=0, max_steps=100000):
        """Per-step mb_subsurfaceW and layer sums of the head and moisture
        (the reference's CopyLayers), as arrays [nsteps] and [nsteps, nz]."""
        nz = self.params[domain].nz
        n = ct.c_int64()
        _check(lib().dhara_get_statistics(self.h, domain, ct.byref(n), None, None, None))
        mb = np.zeros(max(n.value, 1))
        ps = np.zeros(max(n.value, 1) * nz)
        th = np.zeros(max(n.value, 1) * nz)
        _check(lib().dhara_get_statistics(self.h, domain, ct.byref(n), _dp(mb), _dp(ps), _dp(th)))
        k = n.value
        return {"mb_subsurfaceW": mb[:k], "pressure_sum": ps[:k * nz].reshape(k, nz),
                "moisture_sum": th[:k * nz].reshape(k, nz)}

    def snapshot(self, buffers, domain=0):
        """Queues a copy of the state into the given host arrays (keys
        water_elevation, water_depth, pressure_head, moisture; pinned for
        overlap); valid after snapshot_wait()."""
        ptr = [(_dp(buffers[k]) if k in buffers else None)
               for k in ("water_elevation", "water_depth", "pressure_head", "moisture")]
        _check(lib().dhara_snapshot(self.h, domain, *ptr))

    def snapshot_wait(self):
        _check(lib().dhara_snapshot_wait(self.h))

    def save_netcdf(self, file2d=None, file3d=None, domain=0):
        """The reference's snapshot files (SaveModelResults, src/io.cc:854-906)
        of the current state: water_elevation/water_depth and/or
        pressure_head/moisture in NetCDF classic format."""
        enc = lambda f: None if f is None else os.fsencode(f)
        _check(lib().dhara_save_netcdf_state(self.h, domain, enc(file2d), enc(file3d)))

    def save_netcdf_statistics(self, file1d=None, file_stat=None, domain=0):
        """The reference's mb_subsurfaceW and pressure_mean/moisture_mean files
        (SaveResultEntirePeriod, src/io.cc:962-996) from the statistics kept
        since enable_statistics()."""
        enc = lambda f: None if f is None else os.fsencode(f)
        _check(lib().dhara_save_netcdf_statistics(self.h, domain, enc(file1d), enc(file_stat)))

    def apply_boundary_config(self, bc, domain=0):
        """Uploads the per-face settings of params_from_config's third result."""
        _check(lib().dhara_apply_boundary_config(self.h, domain, ct.byref(bc)))

    def set_roots(self, rda, nproc, domain=0):
        a = np.ascontiguousarray(rda, np.float64)
        _check(lib().dhara_set_roots(self.h, domain, _dp(a), int(nproc)))

    def set_rain_schedule(self, mm_per_step, domain=0):
        a = np.ascontiguousarray(mm_per_step, np.float64)
        _check(lib().dhara_set_rain_schedule(self.h, domain, _dp(a), a.size))

    # -- the hot path
    def psi_from_theta(self):
        _check(lib().dhara_psi_from_theta(self.h))

    def prepare(self):
        _check(lib().dhara_prepare(self.h))

    def subsurface_step(self):
        _check(lib().dhara_subsurface_step(self.h))

    def overland_step(self):
        _check(lib().dhara_overland_step(self.h))

    def step(self, nsteps=1, graph=False):
        _check(lib().dhara_step(self.h, int(nsteps), 1 if graph else 0))

    def synchronize(self):
        _check(lib().dhara_synchronize(self.h))

    def diagnostics(self, domain=0):
        d = Diagnostics()
        _check(lib().dhara_get_diagnostics(self.h, domain, ct.byref(d)))
        return d.as_dict()

    @property
    def stream(self):
        s = ct.c_void_p()
        _check(lib().dhara_get_stream(self.h, ct.byref(s)))
        return s.value or 0

    # -- instrumentation
    def set_kernel_timing(self, enable):
        _check(lib().dhara_set_kernel_timing(self.h, 1 if enable else 0))

    def kernel_timing(self, kernel):
        n = ct.c_int64()
        ms = ct.c_double()
        _check(lib().dhara_get_kernel_timing(self.h, KERNELS.get(kernel, kernel), ct.byref(n),
                                             ct.byref(ms)))
        return n.value, ms.value

    def reset_kernel_timing(self):
        _check(lib().dhara_reset_kernel_timing(self.h))

    def launch_count(self):
        n = ct.c_int64()
        _check(lib().dhara_get_launch_count(self.h, ct.byref(n)))
        return n.value

    def adjoint(self, theta_target, q_target, nsteps, checkpoint_every=10, w_q=1.0, gradients=True):
        """Runs nsteps from the current state and returns the loss (and, with
        gradients, dL/dlog Ks, dL/dalpha, dL/dn in the reference 3D layout) of
        the theta / outflow misfit; see dhara_adjoint in include/dhara_gpu.h."""
        p = self.params[0]
        C, N = p.nx * p.ny, p.nx * p.ny * p.nz
        th = np.ascontiguousarray(theta_target, dtype=np.float64).reshape(-1)
        q = np.ascontiguousarray(q_target, dtype=np.float64).reshape(-1)
        if th.size != nsteps * 3 * C or q.size != nsteps:
            raise ValueError("targets must be [nsteps][3][nx*ny] and [nsteps]")
        d = _abi.AdjointDesc()
        d.struct_size = ct.sizeof(_abi.AdjointDesc)
        d.nsteps, d.checkpoint_every, d.w_q = nsteps, checkpoint_every, w_q
        d.theta_target, d.q_target = _dp(th), _dp(q)
        loss = ct.c_double()
        if gradients:
            g = [np.zeros(N) for _ in range(3)]
            _check(lib().dhara_adjoint(self.h, ct.byref(d), ct.byref(loss), *[_dp(a) for a in g]))
            return loss.value, g[0], g[1], g[2]
        _check(lib().dhara_adjoint(self.h, ct.byref(d), ct.byref(loss), None, None, None))
        return loss.value

    def checkpoint(self):
        """The state a step starts from, for every domain, as a host byte
        array (dhara_checkpoint); restore() puts it back."""
        n = ct.c_int64()
        _check(lib().dhara_checkpoint_size(self.h, ct.byref(n)))
        buf = np.empty(n.value, np.uint8)
        _check(lib().dhara_checkpoint(self.h, buf.ctypes.data_as(ct.c_void_p), buf.size))
        return buf

    def restore(self, buf):
        """Restores a checkpoint() of a handle with the same domains, after
        this handle's inputs were loaded and prepare() was called."""
        b = np.ascontiguousarray(buf, dtype=np.uint8)
        _check(lib().dhara_restore(self.h, b.ctypes.data_as(ct.c_void_p), b.size))

    def krylov_traffic(self):
        b = ct.c_double()
        n = ct.c_int64()
        _check(lib().dhara_get_krylov_traffic(self.h, ct.byref(b), ct.byref(n)))
        return b.value, n.value


def selftest_bounded_wait(limit_ms=200.0, device=0):
    """Runs a device-side wait that nothing satisfies (dhara_selftest_bounded_wait);
    True when it gave up after limit_ms, flagged the error and returned."""
    out = ct.c_int(0)
    _check(lib().dhara_selftest_bounded_wait(device, float(limit_ms), ct.byref(out)))
    return bool(out.value)


def write_netcdf_state(file2d, file3d, nx, ny, nz, water_elevation=None, water_depth=None,
                       pressure_head=None, moisture=None):
    """Writes host arrays (reference layout) as the reference's snapshot files;
    host code only, no GPU needed."""
    arrs = [None if a is None else np.ascontiguousarray(a, np.float64)
            for a in (water_elevation, water_depth, pressure_head, moisture)]
    enc = lambda f: None if f is None else os.fsencode(f)
    _check(lib().dhara_write_netcdf_state(enc(file2d), enc(file3d), nx, ny, nz,
                                          *[None if a is None else _dp(a) for a in arrs]))


def write_netcdf_statistics(file1d, file_stat, nz, mb_subsurfaceW, pressure_sum, moisture_sum):
    """Writes the reference's time-series and layer-statistics files from host
    arrays ([nsteps] and [nsteps, nz]); host code only."""
    mb = np.ascontiguousarray(mb_subsurfaceW, np.float64)
    ps = np.ascontiguousarray(pressure_sum, np.float64)
    th = np.ascontiguousarray(moisture_sum, np.float64)
    enc = lambda f: None if f is None else os.fsencode(f)
    _check(lib().dhara_write_netcdf_statistics(enc(file1d), enc(file_stat), mb.size, nz, _dp(mb), _dp(ps),
                                               _dp(th)))


def run(domains, nsteps=None, graph=False, record=(), device=0):
    """Runs one or several inputs.Domain objects together; returns per-domain
    final states and diagnostics."""
    doms = domains if isinstance(domains, (list, tuple)) else [domains]
    s = Solver([d.params for d in doms], device=device)
    for i, d in enumerate(doms):
        s.load(d, i)
    s.prepare()
    n = nsteps if nsteps is not None else max(len(d.rain_mm) for d in doms)
    rec = [{k: [] for k in record} for _ in doms]
    if record:
        for _ in range(n):
            s.step(1, graph)
            for i in range(len(doms)):
                for k in record:
                    rec[i][k].append(s.download(k, i))
    else:
        s.step(n, graph)
    s.synchronize()
    out = []
    for i in range(len(doms)):
        st = {k: s.download(k, i) for k in ("psi", "theta", "ponding", "waterelev", "K")}
        out.append((st, s.diagnostics(i), rec[i]))
    s.close()
    return out if isinstance(domains, (list, tuple)) else out[0]
