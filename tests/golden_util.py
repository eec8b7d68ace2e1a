"""Helpers comparing seismograms with the reference's golden traces using the
reference's own metric (tests/unit-tests/displacement_tests/Newmark/
newmark_tests.cpp:304-346): per station, sum|u - u_ref| / sum|u_ref| over
all components and seismogram types, and |t - t_ref| <= 1e-3."""
import os

import numpy as np

CASES = [
    "HomogeneousElasticDomain",
    "HomogeneousElasticDomainStaceyBC",
    "HomogeneousElasticDomainStaceyDirichletBC",
    "HomogeneousAcousticDomain",
    "HomogeneousAcousticDomainDirichletBC",
    "HomogeneousAcousticDomainCompositeStaceyDirichletBC",
    "AcousticElasticCoupledDomain",
    "HomogeneousElasticIsotropicDomainSH",
]
EXT = {0: "semd", 1: "semv", 2: "sema", 3: "semp"}


def trace_names(case, network, station, stype):
    if stype == 3:
        return ["%s.%s.S2.PRE.%s" % (network, station, EXT[stype])]
    if case.endswith("SH"):
        return ["%s.%s.S2.BXY.%s" % (network, station, EXT[stype])]
    return ["%s.%s.S2.BX%s.%s" % (network, station, c, EXT[stype]) for c in "XZ"]


def station_errors(case, traces, stations, types, seis, times):
    """traces: callable(name) -> (n, 2) array.  Returns per-station errors."""
    errs = []
    for r, (net, sta) in enumerate(stations):
        err = 0.0
        norm = 0.0
        for it, ty in enumerate(types):
            for ic, name in enumerate(trace_names(case, net, sta, ty)):
                tr = traces(name)
                n = min(len(tr), seis.shape[0])
                assert np.all(np.abs(times[:n] - tr[:n, 0]) <= 1e-3), "time axis mismatch"
                err += np.abs(seis[:n, it, r, ic].astype(np.float64) - tr[:n, 1]).sum()
                norm += np.abs(tr[:n, 1]).sum()
        errs.append(err / norm)
    return np.array(errs)


FIXTURES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "newmark")


def fixture_case(case, workdir):
    """Unpack the committed fixture of `case` (tests/golden/newmark/<case>,
    made by tests/golden/make_newmark_fixtures.py) into `workdir`; returns
    the parameter file, a trace loader (name -> (n, 2) array) and the
    (network, station) pairs of its STATIONS file."""
    import gzip
    import shutil
    src = os.path.join(FIXTURES, case)
    for name in ("specfem_config.yaml", "sources.yaml", "STATIONS"):
        shutil.copy(os.path.join(src, name), os.path.join(workdir, name))
    with gzip.open(os.path.join(src, "database.bin.gz"), "rb") as f:
        data = f.read()
    with open(os.path.join(workdir, "database.bin"), "wb") as f:
        f.write(data)
    traces = np.load(os.path.join(src, "traces.npz"))
    stations = [tuple(l.split()[:2][::-1]) for l in open(os.path.join(src, "STATIONS")) if l.strip()]
    return os.path.join(workdir, "specfem_config.yaml"), (lambda n: traces[n].astype(np.float64)), stations
