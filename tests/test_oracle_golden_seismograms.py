"""Receiver location, Lagrange interpolation and the seismogram formula
against the reference's seismogram unit tests
(tests/unit-tests/seismogram/{elastic,acoustic}/seismogram_tests.cpp): a
wavefield read from files (*_00000.bin, Fortran records of one FP64 value,
[nglob][ncomp]) is interpolated at four stations for displacement, velocity
and acceleration, and compared with the ground-truth vector in the test
source (elastic :134-148, tolerance 1e-6 relative; acoustic, tolerance
1e-5 relative).  Both tests are switched off in the reference's own build
(tests/unit-tests/CMakeLists.txt:517-518); their data still pin the path.

The field files are indexed by the reference's point numbering, restated
here from the host side of this library (same partition of local points
into global points, pinned by the ibool golden test):
  * elastic: the per-medium field numbering of field_impl.tpp:37-58, first
    appearance over (element chunk, ix, iz, element in chunk) in compute
    element order (compute_mesh.cpp:239-279: mesh order within each element
    type; every element of this mesh has the same type);
  * acoustic: the global numbering of compute_mesh.cpp:115-150, first
    appearance over (element chunk, iz, ix, element in chunk) in mesh order;
    the file predates the per-medium field numbering.
The storage chunk is 1 element, as in the reference's serial build
(parallel_configuration/chunk_config.hpp:14-27).
The seismograms are the oracle's (FP64), from the problem view this
library's host code assembles.  Reads the reference tree; skipped without it.
"""
import os
import re

import numpy as np
import pytest

from specfempp_b200 import Simulation
from test_oracle_golden_assembly import frec

CASES = {
    # kind: (medium, ncomp, field files, tolerance, traversal)
    "elastic": (0, 2, ("displs", "veloc", "accel"), 1e-6, "field"),
    "acoustic": (3, 1, ("potential_acoustic", "potential_acoustic_dot", "potential_acoustic_dot_dot"), 1e-5,
                 "global"),
}


def ground_truth(test_source):
    """The `ground_truth = { ... }` vector of the reference test, read as text."""
    body = re.search(r"ground_truth\s*=\s*\{([^}]*)\}", open(test_source).read()).group(1)
    return np.array([float(x) for x in body.replace("\n", " ").split(",") if x.strip()])


def local_config(folder, tmp_path):
    """The test's parameter file with absolute paths and a placeholder source
    (the reference test builds its assembly without sources)."""
    text = open(os.path.join(folder, "specfem_config.yaml")).read()
    text = re.sub(r"mesh-database: .*", 'mesh-database: "%s"' % os.path.join(folder, "database.bin"), text)
    text = re.sub(r"stations: .*", 'stations: "%s"' % os.path.join(folder, "STATIONS"), text)
    src = tmp_path / "sources.yaml"
    src.write_text("number-of-sources: 1\nsources:\n  - force:\n      x : 100.0\n      z : 100.0\n"
                   "      angle : 0.0\n      Ricker:\n        factor: 1e10\n        tshift: 0.0\n        f0: 1.0\n")
    text = re.sub(r"\n *sources: .*", "", text).rstrip("\n") + '\n  sources: "%s"\n' % src
    out = tmp_path / "config.yaml"
    out.write_text(text)
    return str(out)


def reference_index(iglob, medium_of, medium, traversal, chunk=1):
    """Map this library's global index -> the reference file's index: first
    appearance of each point over the traversal the reference numbers with
    (elements in mesh order; with one element type that is also the compute
    order)."""
    nspec, n, _ = iglob.shape
    nglob = int(iglob[medium_of == medium].max()) + 1
    out = -np.ones(nglob, np.int64)
    count = 0
    for c0 in range(0, nspec, chunk):
        for a in range(n):
            for b in range(n):
                iz, ix = (b, a) if traversal == "field" else (a, b)
                for e in range(c0, min(c0 + chunk, nspec)):
                    if medium_of[e] != medium:
                        continue
                    g = iglob[e, iz, ix]
                    if out[g] < 0:
                        out[g] = count
                        count += 1
    assert count == nglob
    return out


@pytest.mark.parametrize("kind", sorted(CASES))
def test_seismograms_of_loaded_fields_match_reference(reference_tests_dir, oracle_lib, tmp_path, kind):
    from oracle import bridge
    medium, nc, files, tol, traversal = CASES[kind]
    folder = os.path.join(reference_tests_dir, "seismogram", kind, "serial")
    sim = Simulation.from_yaml(local_config(folder, tmp_path))
    info = sim.info()
    view = sim.problem_view()
    n, nspec = info.ngll, info.nspec
    iglob = np.ctypeslib.as_array(view.iglob, shape=(nspec * n * n,)).reshape(nspec, n, n)
    medium_of = np.ctypeslib.as_array(view.medium, shape=(nspec,))
    assert (medium_of == medium).all()
    # one element type: no Stacey elements (and, for the acoustic mesh, the
    # order is mesh order whatever the tags)
    if kind == "elastic":
        bnd = np.ctypeslib.as_array(view.bnd, shape=(nspec * n * n,))
        assert not (bnd & 1).any()
    idx = reference_index(iglob, medium_of, medium, traversal)
    nglob = idx.size
    fields = []
    for f in files:
        raw = frec(os.path.join(folder, f + "_00000.bin"), np.float64).reshape(nglob, nc)
        fields.append(raw[idx].T.copy())  # [nc][nglob] in this library's numbering
    seis = bridge.seismograms(sim, {"psv" if medium == 0 else "acoustic": tuple(fields)}, 64)
    ours = seis.ravel().astype(np.float64)  # [type][receiver][2], the reference test's order
    truth = ground_truth(os.path.join(reference_tests_dir, "seismogram", kind, "seismogram_tests.cpp"))
    assert ours.size == truth.size == 3 * 4 * 2
    rel = np.abs(ours - truth) / np.where(truth != 0, np.abs(truth), 1.0)
    print("%s: max relative difference %.2e over %d values (tolerance %.0e)" % (kind, rel.max(), truth.size, tol))
    assert np.all(np.abs(ours - truth) <= tol * np.abs(truth))
