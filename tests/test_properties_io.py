"""Model files in the reference's property layout (include/io/property/
{writer,reader}.tpp, io/impl/medium_writer.tpp): structure, element order,
round trip, and the parameter-file keys databases.writer.properties (write
and stop, src/execute.cpp:115-125) and databases.reader.properties."""
import os

import numpy as np
import pytest

from specfempp_b200 import Simulation, StructuredProblem, Material, ForceSource, Station
from workflow_util import reference_element_order, write_forward


def problem(gll_model=None, coupled=False):
    nx, nz = 8, 6
    mats, emat = [Material(2700.0, 3000.0, 1732.0)], None
    if coupled:
        mats.append(Material(1020.0, 1500.0, 0.0))
        emat = np.zeros((nz, nx), np.int32)
        emat[4:, :] = 1
        emat = emat.ravel()
    return StructuredProblem(nx=nx, nz=nz, x0=0.0, x1=400.0, z0=0.0, z1=300.0, materials=mats,
                             element_material=emat, gll_model=gll_model, dt=2.5e-4, nstep=10,
                             sources=[ForceSource(x=200.0, z=100.0, f0=10.0)],
                             stations=[Station(x=100.0, z=120.0)])


def model_arrays(sim):
    info, view = sim.info(), sim.problem_view()
    nloc = info.nspec * info.ngll * info.ngll
    return {name: np.ctypeslib.as_array(getattr(view, name), shape=(nloc,)).copy()
            for name in ("kappa", "mu", "rho", "rho_inverse")}


def perturbed_model(nspec, n, seed=0):
    rng = np.random.default_rng(seed)
    shape = (nspec, n, n)
    return (2700.0 * (1 + 0.05 * rng.standard_normal(shape)), 3000.0 * (1 + 0.05 * rng.standard_normal(shape)),
            1732.0 * (1 + 0.05 * rng.standard_normal(shape)))


def read_meta(path):
    lines = open(path).read().split("\n")
    assert lines[0].split() == ["rank", "3"]
    return [int(x) for x in lines[1].split()[1:]]


@pytest.mark.parametrize("chunk", [1, 32])
def test_round_trip_and_layout(native_lib, tmp_path, chunk):
    n, nspec = 5, 48
    sim = Simulation.structured(problem(gll_model=perturbed_model(nspec, n), coupled=True))
    sim.write_properties(str(tmp_path), chunk)
    root = tmp_path / "Properties"
    info = sim.info()
    for group, names, medium in (("elastic_psv_isotropic", ("X", "Z", "kappa", "mu", "rho"), 0),
                                 ("acoustic_isotropic", ("X", "Z", "rho_inverse", "kappa"), 3),
                                 ("elastic_sh_isotropic", ("X", "Z", "kappa", "mu", "rho"), 1)):
        ne = info.nelements[medium]
        span = -(-ne // chunk) * chunk * n * n
        for name in names:
            assert read_meta(root / group / (name + ".meta")) == [ne, n, n]
            text = open(root / group / (name + ".txt")).read().split()
            assert len(text) == span
    # read back into a context with another (homogeneous) model
    other = Simulation.structured(problem(coupled=True))
    before = model_arrays(other)
    other.read_properties(str(tmp_path), chunk)
    after, ref = model_arrays(other), model_arrays(sim)
    for name in ("kappa", "mu", "rho", "rho_inverse"):
        np.testing.assert_allclose(after[name], ref[name], rtol=2e-7, err_msg=name)
    assert not np.allclose(before["rho"], after["rho"])
    with pytest.raises(Exception):
        other.read_properties(str(tmp_path / "missing"), chunk)


def test_element_order_is_the_reference_compute_order(native_lib, tmp_path):
    """Elements without boundary points first, then the Stacey elements
    (compute_mesh.cpp:239-279); the X dataset shows the order."""
    n = 5
    sim = Simulation.structured(problem())
    sim.write_properties(str(tmp_path), 1)
    x = np.loadtxt(tmp_path / "Properties" / "elastic_psv_isotropic" / "X.txt").reshape(-1, n * n)
    info, view = sim.info(), sim.problem_view()
    order = reference_element_order(sim, 0)
    nloc = info.nspec * n * n
    bnd = np.ctypeslib.as_array(view.bnd, shape=(nloc,)).reshape(info.nspec, n * n)
    assert (bnd[order[0]] == 0).all() and (bnd[order[-1]] & 1).any()
    # first element: its GLL points' x in (i, iz, ix) tile order, i.e. x[iz + ix n]
    xs = x[0].reshape(n, n).T  # [iz][ix]
    assert np.ptp(xs[0]) > 0 and np.allclose(xs[:, 0], xs[0, 0])
    assert order.size == info.nelements[0]


def with_property_key(cfg_path, key, directory):
    text = open(cfg_path).read()
    anchor = "  databases:\n"
    assert anchor in text
    text = text.replace(anchor, anchor + "    %s:\n      properties:\n        format: ascii\n        directory: %s\n"
                        % (key, directory))
    out = cfg_path.replace(".yaml", "_%s.yaml" % key)
    open(out, "w").write(text)
    return out


def test_parameter_file_writer_then_reader(native_lib, tmp_path):
    from specfempp_b200.__main__ import run
    root = str(tmp_path)
    cfg = write_forward(root, 20, 2.5e-4)
    model_dir = tmp_path / "model"
    model_dir.mkdir()
    # writer mode: the model files, and no simulation (no seismograms)
    run(with_property_key(cfg, "writer", str(model_dir)))
    assert (model_dir / "Properties" / "elastic_psv_isotropic" / "rho.txt").exists()
    assert not (tmp_path / "seismograms").exists() or not os.listdir(tmp_path / "seismograms")
    base = model_arrays(Simulation.from_yaml(cfg))
    # scale the density in the files; reader mode picks it up
    path = model_dir / "Properties" / "elastic_psv_isotropic" / "rho.txt"
    rho = np.loadtxt(path)
    with open(path, "w") as f:
        for v in 1.25 * rho:
            f.write("%.10e\n" % v)
    sim = Simulation.from_yaml(with_property_key(cfg, "reader", str(model_dir)))
    got = model_arrays(sim)
    np.testing.assert_allclose(got["rho"], 1.25 * base["rho"], rtol=1e-6)
    np.testing.assert_allclose(got["rho_inverse"], 1.0 / (1.25 * base["rho"]), rtol=1e-6)
    np.testing.assert_allclose(got["mu"], base["mu"], rtol=1e-7)
    # a missing model folder is an error, as in the reference
    with pytest.raises(Exception):
        Simulation.from_yaml(with_property_key(cfg, "reader", str(tmp_path / "nowhere")))
