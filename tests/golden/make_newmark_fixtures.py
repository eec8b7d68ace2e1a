"""Generate tests/golden/newmark/: the reference's golden Newmark cases
(tests/unit-tests/displacement_tests/Newmark/serial/<case> in the reference
checkout) as self-contained fixtures, so that machines without the
reference (the GPU test hosts) can run the device path on the reference's
own meshes and compare with its golden traces.

Per case it writes
  database.bin.gz      the case's mesh, byte for byte, gzip-compressed
  sources.yaml         the case's sources file, unchanged (renamed)
  STATIONS             the case's stations file, unchanged
  specfem_config.yaml  the case's parameter file with the stations, mesh
                       and sources paths pointing at the files beside it
  traces.npz           the golden traces the reference's metric reads
                       (newmark_tests.cpp:304-346): for every file name
                       under traces/, its (time, value) columns as float32
                       (the metric's tolerance is 1e-3)

Run from the repository root:
  python tests/golden/make_newmark_fixtures.py [reference checkout]
(default: $SPECFEMPP_REFERENCE or /root/reference).
"""
import gzip
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from golden_util import CASES  # noqa: E402

OUT = os.path.join(HERE, "newmark")


def make(reference):
    src_root = os.path.join(reference, "tests", "unit-tests", "displacement_tests", "Newmark", "serial")
    for case in CASES:
        src = os.path.join(src_root, case)
        dst = os.path.join(OUT, case)
        os.makedirs(dst, exist_ok=True)
        with open(os.path.join(src, "database.bin"), "rb") as f:
            data = f.read()
        # fixed mtime: regenerating gives identical bytes
        with open(os.path.join(dst, "database.bin.gz"), "wb") as f:
            with gzip.GzipFile(fileobj=f, mode="wb", compresslevel=9, mtime=0) as g:
                g.write(data)
        with open(os.path.join(src, "specfem_config.yaml")) as f:
            cfg = f.read()
        # the files the parameter file names (their base names vary by case)
        named = {key: os.path.basename(re.search(key + r': *"([^"]*)"', cfg).group(1))
                 for key in ("stations", "sources")}
        for key, name in (("sources", "sources.yaml"), ("stations", "STATIONS")):
            with open(os.path.join(src, named[key])) as f:
                text = f.read()
            with open(os.path.join(dst, name), "w") as f:
                f.write(text)
        cfg = re.sub(r'stations: *"[^"]*"', 'stations: "STATIONS"', cfg)
        cfg = re.sub(r'mesh-database: *"[^"]*"', 'mesh-database: "database.bin"', cfg)
        cfg = re.sub(r'sources: *"[^"]*"', 'sources: "sources.yaml"', cfg)
        with open(os.path.join(dst, "specfem_config.yaml"), "w") as f:
            f.write(cfg)
        traces = {}
        tdir = os.path.join(src, "traces")
        for name in sorted(os.listdir(tdir)):
            traces[name] = np.loadtxt(os.path.join(tdir, name), dtype=np.float64).astype(np.float32)
        np.savez_compressed(os.path.join(dst, "traces.npz"), **traces)
        print(case, len(traces), "traces")


if __name__ == "__main__":
    make(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SPECFEMPP_REFERENCE", "/root/reference"))
