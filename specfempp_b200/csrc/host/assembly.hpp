// Host-side assembly: everything the time-marching kernels read, built once
// from a Mesh2D.  It restates what the reference's `specfem::compute::assembly`
// computes (src/compute/assembly/assembly.cpp:6-101) in flat arrays indexed
// by local GLL point  p = (ispec * ngll + iz) * ngll + ix.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "mesh.hpp"
#include "quadrature.hpp"

namespace sfb {

// One point of a fluid-solid coupling edge as seen by the medium that
// receives the contribution ("self"): self += factor * f(normal, coupled).
struct CouplingPoint {
  int self_iglob;     // index in the self medium's field
  int coupled_iglob;  // index in the coupled medium's field
  float factor;       // GLL weight along the edge
  float nx, nz;       // edge normal (carries the 1D Jacobian)
};

struct Source {
  enum Kind { FORCE = 0, MOMENT_TENSOR = 1, EXTERNAL = 2, ADJOINT = 3 };
  enum Stf { RICKER = 0, DIRAC = 1, DGAUSSIAN = 2, TABLE = 3 };
  int kind = FORCE;
  double x = 0, z = 0;
  double angle = 0;                    // force direction (degrees)
  double mxx = 0, mzz = 0, mxz = 0;    // moment tensor
  int stf = RICKER;
  double f0 = 0, tshift = 0, factor = 1;
  bool use_trick_for_better_pressure = false;
  std::vector<double> stf_table;       // TABLE: [nstep][ncomp] user samples
  double table_t0 = 0;                 // TABLE read from files: time of the first sample
  int wavefield = 0;                   // 0 forward/backward, 1 adjoint
  std::string station, network;        // ADJOINT: the station it stands for

  double t0() const;                   // reference rule: -1.2 / f0 + tshift
  double value(double t) const;        // source time function at time t
};

struct Receiver {
  std::string network, station;
  double x = 0, z = 0, angle = 0;
};

// Located point source / receiver (element-local Lagrange arrays).
struct LocatedSource {
  int ispec = -1;
  int medium = 0;
  std::vector<float> array;  // [ncomp][ngll][ngll]
  std::vector<float> stf;    // [nstep][ncomp]
};
struct LocatedReceiver {
  int ispec = -1;
  int medium = 0;
  std::vector<float> lagrange;  // [ngll][ngll]
  float sin_angle = 0, cos_angle = 1;
};

struct Assembly {
  int ngll = 0;
  int nspec = 0;
  Quadrature quad;
  std::vector<int> medium;          // [nspec] MediumTag
  std::vector<int> elem_boundary;   // [nspec] BoundaryTag of the element
  std::vector<double> coord;        // [nloc][2] GLL point coordinates
  // Partial derivatives of the reference-to-physical map, per local point.
  std::vector<float> xix, xiz, gammax, gammaz, jacobian;
  // Material per local point.  Elastic: kappa, mu, rho.  Acoustic: kappa and
  // rho_inverse (rho holds 1/rho_inverse for convenience).
  std::vector<float> kappa, mu, rho, rho_inverse;
  // Mesh-global numbering (all media) and per-medium compact numbering.
  int nglob_mesh = 0;
  std::vector<int> ibool;           // [nloc] mesh-global point
  int nglob[4] = {0, 0, 0, 0};      // per MediumTag
  std::vector<int> iglob;           // [nloc] index within its medium's field
  // Boundary data per local point: bit 0 Stacey, bit 1 acoustic free
  // surface; Stacey edge normal (with 1D Jacobian) and edge weight.
  std::vector<uint8_t> bnd;
  std::vector<float> bnd_nx, bnd_nz, bnd_w;
  // Fluid-solid coupling, per receiving medium.
  std::vector<CouplingPoint> couple_acoustic;  // acoustic <- elastic displacement
  std::vector<CouplingPoint> couple_elastic;   // elastic  <- acoustic acceleration
  std::vector<int> mesh_knods;                 // control nodes (for locating)
  std::vector<double> mesh_coorg;
  int ngnod = 4;

  size_t nloc() const { return static_cast<size_t>(nspec) * ngll * ngll; }
  int ncomp(int m) const { return m == MEDIUM_ELASTIC_PSV ? 2 : 1; }
  int count_elements(int m) const;
};

Assembly build_assembly(const Mesh2D &mesh, int ngll);

// Point location: (ispec, xi, gamma) of a physical point
// (reference: src/algorithms/locate_point.cpp).
struct LocalCoord {
  int ispec;
  double xi, gamma;
};
LocalCoord locate_point(const Assembly &a, double x, double z);

// t0 rule of src/io/sources.cpp:128-158: without a user start time the
// simulation starts at min over sources of t0, and every source's time shift
// becomes its t0 minus that minimum.  Returns the simulation t0.
double resolve_t0(std::vector<Source> &sources, double user_t0);

LocatedSource locate_source(const Assembly &a, const Source &s, double t0,
                            double dt, int nstep);
LocatedReceiver locate_receiver(const Assembly &a, const Receiver &r);

// STATIONS file (name network x z elevation burial per line).
std::vector<Receiver> read_stations(const std::string &path, double angle);

}  // namespace sfb
