// Output / checkpoint files in the reference's ASCII layout
// (include/io/ASCII/impl/*): a "file" is a folder, a group a sub-folder, a
// dataset <name>.meta ("rank R" / "dims d0 d1 ...") plus <name>.txt (one
// value per line, 10-digit scientific for floating point).
#pragma once
#include <string>
#include <vector>

#include "problem.hpp"

namespace sfb {

// Create `dir` afresh (an existing folder of that name is removed first, as
// the reference's writer does) and return it.
std::string ascii_group(const std::string &dir);
void ascii_write(const std::string &group, const std::string &name, const std::vector<long> &dims,
                 const float *data, size_t n);
void ascii_write(const std::string &group, const std::string &name, const std::vector<long> &dims,
                 const double *data, size_t n);
void ascii_write(const std::string &group, const std::string &name, const std::vector<long> &dims, const int *data,
                 size_t n);
// Read a dataset, checking its rank and dims against `dims`.
std::vector<double> ascii_read(const std::string &group, const std::string &name, const std::vector<long> &dims);

// One shot's forward state for the combined run: the fields after the last
// step (per medium tag, [ncomp][nglob]: u, v, a) and the boundary store:
// the element-local accelerations of the elements whose boundary tag is
// stacey (not composite Stacey / Dirichlet), per step; `slot` gives each
// mesh element's slot, -1 where none.
struct ForwardSnapshot {
  int step = 0;
  std::vector<float> field[4][3];
  std::vector<int> slot;        // [nspec]
  int nstacey = 0;
  std::vector<float> store;     // [nstep][nstacey][ngll*ngll][2] (slot order)
};

// <dir>/ForwardWavefield/{Coordinates,StepNNNNNN} as the reference's
// wavefield writer lays it out (include/io/wavefield/writer.tpp:14-150):
// Coordinates/<medium>/{X,Z,mapping}; StepNNNNNN/<medium>/{Displacement,
// Velocity,Acceleration} (acoustic: Potential, PotentialDot,
// PotentialDotDot), [nglob][ncomp] column-major, with empty groups for the
// poroelastic and elastic_psv_t media the reference also visits;
// StepNNNNNN/Boundary/Stacey/{IndexMapping, ElasticAcceleration,
// AcousticAcceleration, PoroelasticAcceleration}: the reference's Stacey
// containers (compute/boundary_values/*): per medium the stacey-tagged
// elements in mesh order, values (nelements, nz, nx, nstep, ncomp)
// column-major.  Files written by either program are read by the other.
// fresh: start the file anew (coordinates and this step); otherwise add or
// replace this step's group (periodic snapshots, time_interval).
void write_forward_wavefield(const Problem &P, const std::string &dir, const ForwardSnapshot &s, bool fresh = true);
// `slot`: this context's store slot per mesh element (the layout the file
// must match).
ForwardSnapshot read_forward_wavefield(const Problem &P, const std::string &dir, const std::vector<int> &slot,
                                       int nstacey);

// <dir>/Kernels/<medium>_isotropic/{X, Z, rho, mu, kappa, rhop, alpha, beta}
// (acoustic: rho, kappa, rhop, alpha), include/io/kernel/writer.tpp and
// include/io/impl/medium_writer.tpp:14-70.  Each dataset has dims
// (nelements, ngllz, ngllx) and the reference's storage order for an element
// tile of `chunk` elements (domain_view.hpp:100-160; chunk 1 is the
// reference's CPU build): tile (i / chunk), then i % chunk, iz, ix, element
// fastest within a tile; the last tile is padded with zeros.  kern[q] holds
// kernel q (rho, mu, kappa, rhop, alpha, beta) per local point, reference
// element order.
void write_kernels(const Problem &P, const std::string &dir, const std::vector<double> kern[6], int chunk);

// <dir>/Properties/<medium>_isotropic/{X, Z, kappa, mu, rho} (acoustic: X, Z,
// rho_inverse, kappa): the model per local point, the reference's property
// writer / reader (include/io/property/{writer,reader}.tpp with
// io/impl/medium_writer.tpp), same element order and tile layout as the
// kernels.  read_properties replaces the assembly's model (and the rho /
// rho_inverse it derives); groups of media the mesh does not hold are not
// read.
void write_properties(const Problem &P, const std::string &dir, int chunk);
void read_properties(Problem &P, const std::string &dir, int chunk);

}  // namespace sfb
