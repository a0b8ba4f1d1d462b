"""The allocation-free overland step (dhara_overland_step_noalloc).

It exists for callers that cannot allocate device memory when they step --
a host model that owns every GPU buffer and hands the library only its own
arrays, a loop that forbids allocation after start-up.  This test calls it
through the C ABI on device arrays the test owns and checks it against the
handle-based dhara_overland_step on the same inputs, for two calls in a row
(the second starting from the first one's output), at the tolerances of the
other GPU parity tests, on a small surface and on one at the 16,384-column
limit of the fixed scratch array.  It lives in its own file, collected last, and passes alone in
a fresh process as well as after the other tests.
"""
import ctypes as ct

import numpy as np
import pytest

import dhara_b200 as db
from dhara_b200 import inputs

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _noalloc():
    L = db.lib()
    fn = L.dhara_overland_step_noalloc
    fn.restype = ct.c_int
    fn.argtypes = [ct.POINTER(db.Params), ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]
    return fn


def _ponded_domain(nx=48, ny=40, seed=21):
    d = inputs.make_domain(nx, ny, 6, seed=seed, overland_tol=1e-12, overland_maxiter=5000)
    rng = np.random.default_rng(seed)
    h = np.where(rng.random(nx * ny) < 0.6, rng.uniform(0.0, 0.02, nx * ny), 0.0)
    return d, h


@pytest.mark.parametrize("nx,ny", [(48, 40), (128, 128)])
def test_noalloc_matches_handle_path_two_calls(gpu, nx, ny):
    import torch
    d, h0 = _ponded_domain(nx, ny)
    p = d.params
    # the existing entry point: a handle, two overland steps
    s = db.Solver(p)
    s.load(d, schedule=False)
    s.upload("waterdepth", h0)
    s.upload("ponding", h0)
    s.prepare()
    ref = []
    for _ in range(2):
        s.overland_step()
        s.synchronize()
        ref.append((s.download("waterdepth"), s.download("waterelev")))
    s.close()
    # the allocation-free entry point on arrays the test allocated
    dev = torch.device("cuda", 0)
    h = torch.tensor(h0, dtype=torch.float64, device=dev)
    z = torch.tensor(d.fields["ztopo"], dtype=torch.float64, device=dev)
    m = torch.tensor(d.fields["mann"], dtype=torch.float64, device=dev)
    H = torch.zeros_like(h)
    stream = torch.cuda.current_stream(dev).cuda_stream
    fn = _noalloc()
    for call in range(2):
        rc = fn(ct.byref(p), h.data_ptr(), z.data_ptr(), m.data_ptr(), H.data_ptr(), stream)
        assert rc == 0, db.lib().dhara_last_error().decode()
        torch.cuda.synchronize(dev)
        h_ref, H_ref = ref[call]
        assert rel_err(H.cpu().numpy(), H_ref) < 1e-8, call
        assert rel_err(h.cpu().numpy(), h_ref) < 1e-6, call


def test_noalloc_rejects_oversize(gpu):
    import torch
    n = int(np.ceil(np.sqrt(16384))) + 1
    p = db.make_params(n, n, 4)
    dev = torch.device("cuda", 0)
    buf = torch.zeros(n * n, dtype=torch.float64, device=dev)
    rc = _noalloc()(ct.byref(p), buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), None)
    assert rc == 4
    assert "exceeds" in db.lib().dhara_last_error().decode()


def test_noalloc_rejects_overlapping_arrays(gpu):
    import torch
    d, _ = _ponded_domain()
    p = d.params
    C = p.nx * p.ny
    dev = torch.device("cuda", 0)
    buf = torch.zeros(3 * C, dtype=torch.float64, device=dev)
    base = buf.data_ptr()
    fn = _noalloc()
    # waterelev overlapping waterdepth (shifted by one cell)
    rc = fn(ct.byref(p), base, base + 2 * C * 8, base + 2 * C * 8, base + 8, None)
    assert rc == 1
    assert "overlap" in db.lib().dhara_last_error().decode()
