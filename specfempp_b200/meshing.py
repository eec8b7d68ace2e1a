"""Structured quad meshes written as the reference's 2D mesh database
(`database.bin`, Fortran unformatted sequential records as the reference's
reader takes them: src/io/mesh/impl/fortran/dim2/read_mesh_database.cpp,
read_material_properties.cpp, read_elements.cpp, read_boundaries.cpp,
read_interfaces.cpp), so a parameter file can name a mesh made here the way
it names one made by xmeshfem2D.

Element e = iz * nx + ix, 4 control nodes counter-clockwise from the
bottom-left corner; absorbing sides in the order (bottom, right, top, left);
the top edge of acoustic elements is a free surface unless it absorbs;
fluid-solid edges between neighbouring acoustic and elastic elements.
"""
from __future__ import annotations

import struct
from typing import Sequence

import numpy as np


def _record(f, payload: bytes):
    f.write(struct.pack("<i", len(payload)))
    f.write(payload)
    f.write(struct.pack("<i", len(payload)))


def _ints(*v):
    return struct.pack("<%di" % len(v), *v)


def write_database(path: str, nx: int, nz: int, x0: float, x1: float, z0: float, z1: float,
                   materials: Sequence, element_material=None, absorb=(True, True, False, True),
                   free_top_acoustic: bool = True, deform=None):
    """materials: (rho, vp, vs) per material (vs = 0: acoustic);
    element_material: 0-based material of each element [nz * nx];
    deform: optional (x, z) -> (x, z) map of the control nodes (e.g. a
    topography), which makes the elements general bilinear quads."""
    nspec = nx * nz
    npx, npz = nx + 1, nz + 1
    npgeo = npx * npz
    em = np.zeros(nspec, dtype=np.int64) if element_material is None else np.asarray(element_material, dtype=np.int64)
    if em.shape != (nspec,):
        raise ValueError("element_material must have nx * nz entries")
    acoustic = [float(m[2]) == 0.0 for m in materials]

    def knods(e):
        iz, ix = divmod(e, nx)
        bl = iz * npx + ix
        return (bl, bl + 1, bl + npx + 1, bl + npx)

    absorbing, surface, fluid_solid = [], [], []
    for iz in range(nz):
        for ix in range(nx):
            e = iz * nx + ix
            on = (iz == 0, ix == nx - 1, iz == nz - 1, ix == 0)
            for side in range(4):
                if not on[side]:
                    continue
                if absorb[side]:
                    absorbing.append((e, side))
                if side == 2 and free_top_acoustic and not absorb[2] and acoustic[em[e]]:
                    surface.append(e)
            for nb in ((e + nx) if iz + 1 < nz else -1, (e + 1) if ix + 1 < nx else -1):
                if nb >= 0 and acoustic[em[e]] != acoustic[em[nb]]:
                    fluid_solid.append((e, nb) if acoustic[em[e]] else (nb, e))
    with open(path, "wb") as f:
        # 64 header records of run flags (the reader uses nspec and npgeo only)
        for i in range(64):
            _record(f, _ints(nspec if i == 2 else npgeo if i == 3 else 0))
        for j in range(npz):
            for i in range(npx):
                ip = j * npx + i + 1
                x, z = x0 + (x1 - x0) * i / nx, z0 + (z1 - z0) * j / nz
                if deform is not None:
                    x, z = deform(x, z)
                _record(f, struct.pack("<idd", ip, float(x), float(z)))
        _record(f, _ints(len(materials), 4, nspec))
        _record(f, _ints(len(absorbing), 0, len(surface), len(fluid_solid), 0, 0, 0, 0))
        _record(f, struct.pack("<idi", 0, 0.0, 0))  # attenuation: n_sls, f0, read_velocities_at_f0
        for k, (rho, vp, vs) in enumerate(materials):
            v = [rho, vp, vs, 0.0, 0.0, 9999.0, 9999.0] + [0.0] * 6
            _record(f, struct.pack("<ii13d", k + 1, 1, *v))
        for e in range(nspec):
            _record(f, _ints(e + 1, int(em[e]) + 1, *[n + 1 for n in knods(e)], 0))
        _record(f, _ints(0, 0))  # ninterfaces, max_interface_size
        for e, side in absorbing:
            codes = [0, 0, 0, 0]
            codes[side] = 1
            _record(f, _ints(e + 1, *codes, 1, *([0] * 8)))
        for e in surface:
            kn = knods(e)
            _record(f, _ints(e + 1, 2, kn[2] + 1, kn[3] + 1))  # the top edge's two control nodes
        for a, b in fluid_solid:
            _record(f, _ints(a + 1, b + 1))
        _record(f, _ints(0, 0))  # tangential-curve flags
    return path
