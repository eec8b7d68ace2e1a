"""Moment-tensor point sources (src/source/moment_tensor_source.cpp:18-143).

The source array the library builds is checked against an independent
restatement of the reference's formula: Lagrange interpolants h and their
derivatives h' at the source's reference coordinates (computed here from the
GLL points by the product rule), the element's partial derivatives
interpolated to the source point, and
    dsrc/dx(iz, ix) = h'_xi(ix) xix_s h_ga(iz) + h_xi(ix) h'_ga(iz) gammax_s
    dsrc/dz(iz, ix) = h'_xi(ix) xiz_s h_ga(iz) + h_xi(ix) h'_ga(iz) gammaz_s
    array = (Mxx dsrc/dx + Mxz dsrc/dz,  Mxz dsrc/dx + Mzz dsrc/dz).
The reference's sources-file entry (`moment-tensor` with Mxx, Mzz, Mxz;
src/io/sources.cpp:84-86) gives the same array, and a moment tensor in a
fluid element is an error, as in the reference.  GPU parity of runs driven
by moment tensors is in test_gpu_moment_tensor.py."""
import os

import numpy as np
import pytest

from specfempp_b200 import ForceSource, Material, SfbError, Simulation, Station, StructuredProblem

NX, NZ, LX, LZ = 12, 10, 1200.0, 1000.0


def lagrange(xi_nodes, x):
    """Values and derivatives of the Lagrange basis of `xi_nodes` at x."""
    n = len(xi_nodes)
    h = np.ones(n)
    hp = np.zeros(n)
    for j in range(n):
        others = [m for m in range(n) if m != j]
        den = np.prod([xi_nodes[j] - xi_nodes[m] for m in others])
        h[j] = np.prod([x - xi_nodes[m] for m in others]) / den
        hp[j] = sum(np.prod([x - xi_nodes[m] for m in others if m != k]) for k in others) / den
    return h, hp


def restated_array(sim, x, z, mxx, mzz, mxz):
    """The reference's source array for a source at (x, z) of the structured
    mesh (element (ix, iz) = ispec iz * NX + ix, affine map)."""
    v = sim.problem_view()
    n = sim.info().ngll
    nodes = np.ctypeslib.as_array(v.xi, shape=(n,)).copy()
    dx, dz = LX / NX, LZ / NZ
    ex, ez = int(x // dx), int(z // dz)
    ispec = ez * NX + ex
    xi = 2.0 * (x - ex * dx) / dx - 1.0
    ga = 2.0 * (z - ez * dz) / dz - 1.0
    hx, hpx = lagrange(nodes, xi)
    hz, hpz = lagrange(nodes, ga)
    nloc = sim.info().nspec * n * n
    geo = {k: np.ctypeslib.as_array(getattr(v, k), shape=(nloc,)).reshape(-1, n, n)[ispec].astype(np.float64)
           for k in ("xix", "xiz", "gammax", "gammaz")}
    w = np.outer(hz, hx)  # [iz][ix]
    s = {k: float(np.sum(w * g)) for k, g in geo.items()}
    dsdx = np.outer(hz, hpx) * s["xix"] + np.outer(hpz, hx) * s["gammax"]
    dsdz = np.outer(hz, hpx) * s["xiz"] + np.outer(hpz, hx) * s["gammaz"]
    return ispec, np.stack([mxx * dsdx + mxz * dsdz, mxz * dsdx + mzz * dsdz])


def problem(sources, materials=None, element_material=None):
    return StructuredProblem(nx=NX, nz=NZ, x0=0.0, x1=LX, z0=0.0, z1=LZ,
                             materials=materials or [Material(2700.0, 3000.0, 1732.0)],
                             element_material=element_material, dt=2.5e-4, nstep=50,
                             sources=sources, stations=[Station(x=600.0, z=900.0)])


@pytest.mark.parametrize("mt", [(1.0, 1.0, 0.0), (0.3, -0.7, 0.45), (0.0, 0.0, 1.0)])
def test_source_array_matches_restated_formula(native_lib, mt):
    x, z = 537.0, 463.0
    sim = Simulation.structured(problem([ForceSource(x=x, z=z, f0=10.0, kind="moment_tensor", mxx=mt[0],
                                                     mzz=mt[1], mxz=mt[2])]))
    v = sim.problem_view()
    n = sim.info().ngll
    ispec, ref = restated_array(sim, x, z, *mt)
    assert v.nsources == 1 and v.src_ispec[0] == ispec
    arr = np.ctypeslib.as_array(v.src_array, shape=(2 * n * n,)).reshape(2, n, n).astype(np.float64)
    err = np.abs(arr - ref).max() / np.abs(ref).max()
    print("moment tensor %s: source array vs restated formula %.2e" % (mt, err))
    assert err <= 1e-6


def test_sources_file_entry(native_lib, tmp_path):
    """`moment-tensor` entries of a reference sources file give the same
    array as the structured description."""
    import workflow_util as WU
    root = str(tmp_path)
    WU.write_mesh_and_stations(root)
    src = os.path.join(root, "sources.yaml")
    with open(src, "w") as f:
        f.write("""number-of-sources: 1
sources:
  - moment-tensor:
      x: 413.0
      z: 287.0
      Mxx: 0.3
      Mzz: -0.7
      Mxz: 0.45
      angle: 0.0
      Ricker:
        factor: 1e10
        tshift: 0.0
        f0: 10.0
""")
    mode = """      forward:
        writer:
          seismogram:
            format: ascii
            directory: %s""" % root
    cfg = os.path.join(root, "config.yaml")
    with open(cfg, "w") as f:
        f.write(WU.config(root, 50, 2.5e-4, mode, src))
    a = Simulation.from_yaml(cfg)
    b = Simulation.structured(StructuredProblem(
        nx=WU.NX, nz=WU.NZ, x0=0.0, x1=WU.LX, z0=0.0, z1=WU.LZ, materials=[Material(*WU.MAT)],
        absorb=WU.ABSORB, dt=2.5e-4, nstep=50,
        sources=[ForceSource(x=413.0, z=287.0, f0=10.0, factor=1e10, kind="moment_tensor", mxx=0.3, mzz=-0.7,
                             mxz=0.45)],
        stations=[Station(x=x, z=z) for x, z in WU.STATIONS]))
    n = a.info().ngll
    va, vb = a.problem_view(), b.problem_view()
    assert va.src_ispec[0] == vb.src_ispec[0]
    xa = np.ctypeslib.as_array(va.src_array, shape=(2 * n * n,))
    xb = np.ctypeslib.as_array(vb.src_array, shape=(2 * n * n,))
    assert np.array_equal(xa, xb)
    sa = np.ctypeslib.as_array(va.src_stf, shape=(100,))
    sb = np.ctypeslib.as_array(vb.src_stf, shape=(100,))
    assert np.array_equal(sa, sb)


def test_moment_tensor_in_fluid_is_an_error(native_lib):
    em = np.zeros((NZ, NX), np.int32)
    em[NZ // 2:, :] = 1
    p = problem([ForceSource(x=600.0, z=900.0, f0=10.0, kind="moment_tensor", mxx=1.0, mzz=1.0)],
                materials=[Material(2700.0, 3000.0, 1732.0), Material(1020.0, 1500.0, 0.0)],
                element_material=em.ravel())
    with pytest.raises(SfbError) as e:
        Simulation.structured(p)
    assert "Moment tensor" in str(e.value)


def test_oracle_runs_moment_tensor_source(native_lib, oracle_lib):
    from oracle import bridge
    sim = Simulation.structured(problem([ForceSource(x=537.0, z=463.0, f0=10.0, factor=1e10,
                                                     kind="moment_tensor", mxx=1.0, mzz=1.0)]))
    out = bridge.forward(sim, 64, threads=2)["seismograms"]
    assert np.isfinite(out).all() and np.abs(out).max() > 0
