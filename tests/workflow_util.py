"""Parameter files, sources files, STATIONS and a database.bin for a small
elastic case, in the reference's formats (a forward run that writes its
wavefield, then a combined run that reads it and writes kernels)."""
import os

import numpy as np

from specfempp_b200 import StructuredProblem, Material, ForceSource, Station
from specfempp_b200.meshing import write_database

NX, NZ, LX, LZ = 20, 16, 800.0, 600.0
MAT = (2700.0, 3000.0, 1732.0)
ABSORB = (True, True, False, True)
SOURCE = (400.0, 300.0, 10.0)
STATIONS = [(100.0 + 150.0 * k, 500.0) for k in range(5)]


def structured(nstep, dt):
    """The same case as a StructuredProblem (the ABI path)."""
    return StructuredProblem(nx=NX, nz=NZ, x0=0.0, x1=LX, z0=0.0, z1=LZ, materials=[Material(*MAT)],
                             absorb=ABSORB, dt=dt, nstep=nstep,
                             sources=[ForceSource(x=SOURCE[0], z=SOURCE[1], f0=SOURCE[2], factor=1e10)],
                             stations=[Station(x=x, z=z, network="AA", station="S%04d" % (k + 1))
                                       for k, (x, z) in enumerate(STATIONS)],
                             seismogram_types=("displacement",), save_boundary_values=True)


def force_entry():
    return """  - force:
      x : %r
      z : %r
      source_surf: false
      angle : 0.0
      vx : 0.0
      vz : 0.0
      Ricker:
        factor: 1e10
        tshift: 0.0
        f0: %r
""" % SOURCE


def write_mesh_and_stations(root, deform=None):
    write_database(os.path.join(root, "database.bin"), NX, NZ, 0.0, LX, 0.0, LZ, [MAT], absorb=ABSORB,
                   deform=deform)
    with open(os.path.join(root, "STATIONS"), "w") as f:
        for k, (x, z) in enumerate(STATIONS):
            f.write("S%04d    AA    %.7f    %.7f    0.0    0.0\n" % (k + 1, x, z))


def config(root, nstep, dt, mode_block, sources_file):
    return """parameters:
  header:
    title: workflow test
    description: small elastic case
  simulation-setup:
    quadrature:
      quadrature-type: GLL4
    solver:
      time-marching:
        time-scheme:
          type: Newmark
          dt: %r
          nstep: %d
    simulation-mode:
%s
  receivers:
    stations: %s
    angle: 0.0
    seismogram-type:
      - displacement
    nstep_between_samples: 1
  run-setup:
    number-of-processors: 1
    number-of-runs: 1
  databases:
    mesh-database: %s
  sources: %s
""" % (dt, nstep, mode_block, os.path.join(root, "STATIONS"), os.path.join(root, "database.bin"), sources_file)


def write_forward(root, nstep, dt, deform=None):
    write_mesh_and_stations(root, deform)
    src = os.path.join(root, "forward_sources.yaml")
    with open(src, "w") as f:
        f.write("number-of-sources: 1\nsources:\n" + force_entry())
    mode = """      forward:
        writer:
          wavefield:
            format: ascii
            directory: %s
          seismogram:
            format: ascii
            directory: %s""" % (root, os.path.join(root, "seismograms"))
    path = os.path.join(root, "forward_config.yaml")
    with open(path, "w") as f:
        f.write(config(root, nstep, dt, mode, src))
    return path


def write_combined(root, nstep, dt, adj_folder, names):
    src = os.path.join(root, "adjoint_sources.yaml")
    with open(src, "w") as f:
        f.write("number-of-sources: %d\nsources:\n" % (1 + len(names)))
        f.write(force_entry())
        for k, ((x, z), name) in enumerate(zip(STATIONS, names)):
            f.write("""  - adjoint-source:
      station_name: %s
      network_name: AA
      x: %r
      z: %r
      source_surf: false
      angle: 0.0
      vx: 0.0
      vz: 0.0
      External:
        format: ascii
        stf:
          X-component: %s
          Z-component: %s
""" % (name.split(".")[1], x, z, os.path.join(adj_folder, name + ".BXX.adj"), os.path.join(adj_folder, name + ".BXZ.adj")))
    mode = """      combined:
        reader:
          wavefield:
            format: ascii
            directory: %s
        writer:
          kernels:
            format: ascii
            directory: %s""" % (root, os.path.join(root, "kernels"))
    path = os.path.join(root, "adjoint_config.yaml")
    with open(path, "w") as f:
        f.write(config(root, nstep, dt, mode, src))
    return path


def reference_element_order(sim, medium):
    """Elements of `medium` in the reference's compute order, which the
    kernel and property writers follow: by boundary tag (none, acoustic free
    surface, Stacey, both; from the points' boundary bits), mesh order within
    a tag."""
    info, view = sim.info(), sim.problem_view()
    n, nspec = info.ngll, info.nspec
    med = np.ctypeslib.as_array(view.medium, shape=(nspec,))
    bits = np.bitwise_or.reduce(np.ctypeslib.as_array(view.bnd, shape=(nspec * n * n,)).reshape(nspec, n * n), axis=1)
    stacey, surface = (bits & 1) != 0, (bits & 2) != 0
    tag = np.where(stacey & surface, 3, np.where(stacey, 2, np.where(surface, 1, 0)))
    return np.concatenate([np.nonzero((med == medium) & (tag == t))[0] for t in range(4)])


def read_kernel(folder, medium_group, name, nspec_medium, ngll, order=None):
    """A kernel dataset written with element tile 1: value (i, iz, ix) at
    i * n * n + iz + ix * n, element i of the writer's order; with `order`
    (reference_element_order) the result is in mesh element order."""
    v = np.loadtxt(os.path.join(folder, "Kernels", medium_group, name + ".txt"))
    out = np.zeros((nspec_medium, ngll, ngll))
    for i in range(nspec_medium):
        for iz in range(ngll):
            for ix in range(ngll):
                out[i, iz, ix] = v[i * ngll * ngll + iz + ix * ngll]
    if order is not None:
        mesh = np.zeros_like(out)
        mesh[order] = out
        out = mesh
    return out
