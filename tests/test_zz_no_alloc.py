"""The allocation-free inverse-mass entry point, called through the C ABI.

sfb_assemble_inverse_mass_noalloc serves callers that cannot allocate device
memory where they need the mass matrix (a host framework that hands out all
device buffers from its own pool, a real-time loop that must not touch the
allocator): it keeps its FP64 accumulation scratch in a fixed device array
instead of allocating.
Here the test itself provides the device inputs and output (through torch)
and compares the result with the inverse mass the regular path computes, on
two calls in a row (the second call must clear the scratch the first one
left behind).  The file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-6  # relative; both paths accumulate in FP64 and round once


def _medium_inputs(sim, medium):
    """Device arrays of one medium's local points, from the problem view."""
    import torch
    v = sim.problem_view()
    info = sim.info()
    n = info.ngll
    nn = n * n
    nspec = info.nspec
    nloc = nspec * nn
    med = np.ctypeslib.as_array(v.medium, shape=(nspec,))
    sel = np.nonzero(med == medium)[0]
    idx = (sel[:, None] * nn + np.arange(nn)[None, :]).reshape(-1)

    def arr(ptr, dtype):
        return np.ctypeslib.as_array(ptr, shape=(nloc,)).astype(dtype)[idx]

    iglob = arr(v.iglob, np.int32)
    jac = arr(v.jacobian, np.float32)
    kappa, mu, rho, rho_inv = (arr(p, np.float32) for p in (v.kappa, v.mu, v.rho, v.rho_inverse))
    if medium == 0:
        m0, m1, m2 = kappa, mu, rho
    elif medium == 1:
        m0, m1, m2 = mu, rho, np.zeros_like(rho)
    else:
        m0, m1, m2 = rho_inv, kappa, np.zeros_like(rho)
    bnd = arr(v.bnd, np.uint8)
    bnx, bnz, bw = (arr(p, np.float32) for p in (v.bnd_nx, v.bnd_nz, v.bnd_w))
    dev = {k: torch.from_numpy(np.ascontiguousarray(a)).cuda()
           for k, a in dict(iglob=iglob, jac=jac, m0=m0, m1=m1, m2=m2, bnd=bnd, bnx=bnx, bnz=bnz, bw=bw).items()}
    w = np.ctypeslib.as_array(v.wgll, shape=(n,)).astype(np.float64).copy()
    return dev, w, len(sel), info.nglob[medium], info.dt


def _problem(medium):
    from specfempp_b200 import workloads as W
    if medium == 0:
        return W.plain_elastic(scale=0.3, nstep=10)
    if medium == 1:
        p = W.plain_elastic(scale=0.3, nstep=10)
        p.elastic_sh = True
        return p
    return W.coupled(scale=0.08, nstep=10)


def _call(lib, medium, ngll, nelem, npoints, dev, w, dt, out, stream):
    ptr = lambda t: C.c_void_p(t.data_ptr())
    return lib.sfb_assemble_inverse_mass_noalloc(
        medium, ngll, nelem, npoints, ptr(dev["iglob"]), ptr(dev["jac"]), ptr(dev["m0"]),
        ptr(dev["m1"]), ptr(dev["m2"]), ptr(dev["bnd"]), ptr(dev["bnx"]), ptr(dev["bnz"]),
        ptr(dev["bw"]), w.ctypes.data_as(C.POINTER(C.c_double)), dt, ptr(out), C.c_void_p(stream))


@pytest.mark.parametrize("medium", [0, 1, 3])
def test_noalloc_inverse_mass_matches_regular_path(medium):
    import torch
    from specfempp_b200 import Simulation, _capi as A

    p = _problem(medium)
    sim = Simulation.structured(p)
    sim.initialize()
    expected = sim.field(medium, 3)  # [ncomp][npoints] from the regular path
    nc = expected.shape[0]
    lib = A.load()
    dev, w, nelem, npoints, dt = _medium_inputs(sim, medium)
    out = torch.empty(npoints * nc, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        out.fill_(float("nan"))
        rc = _call(lib, medium, p.ngll, nelem, npoints, dev, w, dt, out, stream)
        assert rc == 0, lib.sfb_noalloc_last_error().decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy().reshape(npoints, nc).T
        err = float(np.max(np.abs(got - expected) / np.abs(expected)))
        assert np.isfinite(got).all()
        assert err <= TOL, (call, err)


def test_noalloc_out_of_range_index_poisons_output_only():
    """An index past the caller's points is skipped on the device (nothing is
    written outside the caller's range) and the call's output becomes NaN;
    the next call with good indices is correct again."""
    import torch
    from specfempp_b200 import Simulation, _capi as A

    p = _problem(0)
    sim = Simulation.structured(p)
    sim.initialize()
    expected = sim.field(0, 3)
    nc = expected.shape[0]
    lib = A.load()
    dev, w, nelem, npoints, dt = _medium_inputs(sim, 0)
    out = torch.empty(npoints * nc + 64, dtype=torch.float32, device="cuda")
    out.fill_(7.0)
    bad = dict(dev)
    bad["iglob"] = dev["iglob"].clone()
    bad["iglob"][5] = npoints + 3
    stream = torch.cuda.current_stream().cuda_stream
    assert _call(lib, 0, p.ngll, nelem, npoints, bad, w, dt, out, stream) == 0
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert np.isnan(got[:npoints * nc]).all()
    assert (got[npoints * nc:] == 7.0).all()  # the guard words past the output are untouched
    assert _call(lib, 0, p.ngll, nelem, npoints, dev, w, dt, out, stream) == 0
    torch.cuda.synchronize()
    good = out.cpu().numpy()[:npoints * nc].reshape(npoints, nc).T
    assert float(np.max(np.abs(good - expected) / np.abs(expected))) <= TOL


def test_noalloc_rejects_oversized_problem():
    from specfempp_b200 import _capi as A
    lib = A.load()
    w = (C.c_double * 5)(*([1.0] * 5))
    dummy = C.c_void_p(1)
    rc = lib.sfb_assemble_inverse_mass_noalloc(0, 5, 1, (1 << 21), dummy, dummy, dummy, dummy, dummy,
                                               None, None, None, None, w, 1e-3, dummy, None)
    assert rc == -1
    assert "exceeds" in lib.sfb_noalloc_last_error().decode()
