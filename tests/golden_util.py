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
