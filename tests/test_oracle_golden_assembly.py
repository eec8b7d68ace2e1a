"""The oracle's (and the host assembly's) inverse mass, partial derivatives
and global numbering against the reference's own golden arrays
(tests/unit-tests/domain/serial/test{1,2}: rmass_inverse_*.bin with
index_mapping.bin, compared with the reference's metric and 1e-5 tolerance,
domain/rmass_inverse_tests.cpp:140-230; compute/partial_derivatives/serial/
*_00000.bin, compute_partial_derivatives_tests.cpp:88-120, tolerance 1e-2
absolute there, checked tighter here; compute/index/serial/ibool_00000.bin,
compute/index/compute_tests.cpp).  The golden files are Fortran sequential
records of one value each.  Reads the reference tree; skipped without it."""
import os
import re

import numpy as np
import pytest

from specfempp_b200 import Simulation


def frec(path, dtype):
    raw = np.fromfile(path, dtype=np.uint8)
    size = np.dtype(dtype).itemsize
    rec = raw.reshape(-1, 8 + size)
    assert (rec[:, :4].copy().view(np.int32) == size).all()
    return rec[:, 4:4 + size].copy().view(dtype).ravel()


def config_with_local_paths(ref_root, config, tmp_path, database, sources=None):
    """The reference's test config with absolute mesh / sources paths and a
    one-station STATIONS file (receivers do not enter these arrays)."""
    text = open(os.path.join(ref_root, config)).read()
    text = re.sub(r'mesh-database: .*', 'mesh-database: "%s"' % os.path.join(ref_root, database), text)
    if sources is None:
        src = tmp_path / "sources.yaml"
        src.write_text("number-of-sources: 1\nsources:\n  - force:\n      x : 0.0\n      z : 0.0\n"
                       "      angle : 0.0\n      Ricker:\n        factor: 1e10\n        tshift: 0.0\n        f0: 1.0\n")
        sources = str(src)
    else:
        sources = os.path.join(ref_root, sources)
    text = re.sub(r'\n  sources: .*', '\n  sources: "%s"' % sources, text)
    stations = tmp_path / "STATIONS"
    stations.write_text("S0001 AA 0.0 0.0 0.0 0.0\n")
    text = re.sub(r'stations: .*', 'stations: "%s"' % stations, text)
    out = tmp_path / "config.yaml"
    out.write_text(text)
    return str(out)


def minimal_config(ref_root, database, tmp_path):
    text = """parameters:
  header:
    title: golden arrays
    description: none
  simulation-setup:
    quadrature:
      quadrature-type: GLL4
    solver:
      time-marching:
        time-scheme:
          type: Newmark
          dt: 1e-3
          nstep: 10
  receivers:
    stations: "STATIONS_PLACEHOLDER"
    angle: 0.0
    seismogram-type:
      - displacement
    nstep_between_samples: 1
  run-setup:
    number-of-processors: 1
    number-of-runs: 1
  databases:
    mesh-database: "%s"
  sources: "SOURCES_PLACEHOLDER"
""" % os.path.join(ref_root, database)
    cfg = tmp_path / "base.yaml"
    cfg.write_text(text)
    return config_with_local_paths(str(tmp_path), "base.yaml", tmp_path, os.path.join(ref_root, database))


@pytest.mark.parametrize("test,mass_file,medium", [("test1", "rmass_inverse_elastic.bin", 0),
                                                   ("test2", "rmass_inverse_acoustic.bin", 3)])
def test_oracle_inverse_mass_matches_reference(reference_tests_dir, oracle_lib, tmp_path, test, mass_file, medium):
    from oracle import bridge
    folder = "domain/serial/%s" % test
    cfg = config_with_local_paths(reference_tests_dir, folder + "/specfem_config.yaml", tmp_path,
                                  folder + "/database.bin", folder + "/source.yaml")
    sim = Simulation.from_yaml(cfg)
    info = sim.info()
    n, nspec = info.ngll, info.nspec
    view = sim.problem_view()
    iglob = np.ctypeslib.as_array(view.iglob, shape=(nspec * n * n,)).reshape(nspec, n, n)
    nc = 2 if medium == 0 else 1
    name = {0: "psv", 3: "acoustic"}[medium]
    minv = bridge.forward(sim, 64, nstep=1, threads=8, want_fields=True)[name][3]  # [nc][nglob]
    mapping = frec(os.path.join(reference_tests_dir, folder, "index_mapping.bin"), np.int32).reshape(nspec, n, n)
    ref = frec(os.path.join(reference_tests_dir, folder, mass_file), np.float64)
    ref = ref.reshape(-1, 2 if medium == 0 else 1)
    err = norm = 0.0
    for c in range(nc):
        ours = minv[c][iglob]
        theirs = ref[mapping, c]
        err += np.sum(np.abs(ours - theirs))
        norm += np.sum(np.abs(theirs))
    print("%s inverse mass: sum|diff| / sum|ref| = %.2e" % (test, err / norm))
    assert err / norm < 1e-5


def test_partial_derivatives_match_reference(reference_tests_dir, native_lib, tmp_path):
    folder = os.path.join(reference_tests_dir, "compute/partial_derivatives/serial")
    sim = Simulation.from_yaml(minimal_config(reference_tests_dir, "compute/partial_derivatives/serial/Database00000.bin",
                                              tmp_path))
    info = sim.info()
    n, nspec = info.ngll, info.nspec
    view = sim.problem_view()
    for name, field in (("xix", "xix"), ("gammax", "gammax"), ("gammaz", "gammaz"), ("jacobian", "jacobian")):
        ours = np.ctypeslib.as_array(getattr(view, field), shape=(nspec * n * n,)).astype(np.float64)
        ref = frec(os.path.join(folder, "%s_00000.bin" % name), np.float64)
        assert np.max(np.abs(ours - ref)) < 1e-2  # the reference's tolerance
        rel = np.max(np.abs(ours - ref)) / np.max(np.abs(ref))
        print("%s: max |diff| / max |ref| = %.2e" % (name, rel))
        assert rel < 1e-6


def test_global_numbering_matches_reference_partition(reference_tests_dir, native_lib, tmp_path):
    """ibool: the same local points share a global point as in the
    reference (the numbering order itself is this library's own)."""
    sim = Simulation.from_yaml(minimal_config(reference_tests_dir, "compute/index/serial/Database00000.bin", tmp_path))
    info = sim.info()
    n, nspec = info.ngll, info.nspec
    view = sim.problem_view()
    ours = np.ctypeslib.as_array(view.iglob, shape=(nspec * n * n,)).astype(np.int64)
    ref = frec(os.path.join(reference_tests_dir, "compute/index/serial/ibool_00000.bin"), np.int32).astype(np.int64)
    assert ours.size == ref.size
    assert len(np.unique(ours)) == len(np.unique(ref))
    pairs = np.unique(np.stack([ours, ref], axis=1), axis=0)
    assert len(pairs) == len(np.unique(ref))  # one-to-one
