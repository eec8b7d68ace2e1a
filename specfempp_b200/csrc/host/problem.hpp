// A complete simulation problem on the host: assembly, located sources and
// receivers, time stepping and output settings.  Built either from the
// reference's YAML parameter file (src/parameter_parser/setup.cpp) or from a
// structured-mesh description (the benchmark workloads).
#pragma once
#include <string>
#include <vector>

#include "../../../include/specfem_b200.h"
#include "assembly.hpp"

namespace sfb {

struct Problem {
  Assembly asmb;
  double dt = 0, t0 = 0;
  int nstep = 0;
  int nshots = 1;
  int simulation = 0;  // 0 forward, 1 combined
  int nstep_between_samples = 1;
  std::vector<int> seismogram_types;
  std::vector<Source> sources;             // as described
  std::vector<int> source_shot;            // [nsources]
  std::vector<LocatedSource> located_sources;
  std::vector<Receiver> receivers;
  std::vector<LocatedReceiver> located_receivers;
  // adjoint sources given in the sources file (combined runs), located like
  // point sources with Lagrange weights in both components and their own
  // [nstep][2] time functions; empty: adjoint sources at the stations, set
  // through sfb_set_adjoint_sources
  std::vector<Source> adjoint_sources;
  std::vector<LocatedSource> located_adjoint;
  bool save_boundary_values = false;
  bool elastic_sh = false;
  // Output settings from the YAML file.
  std::string seismogram_dir;
  bool write_seismograms = false;
  std::string wavefield_dir;   // forward: writer.wavefield; combined: reader
  // forward writer.wavefield: a snapshot every time_interval steps (0: none)
  // and one of the last step when include_last_step
  // (src/parameter_parser/writer/wavefield.cpp:36-66)
  int wavefield_time_interval = 0;
  bool wavefield_include_last_step = true;
  std::string kernel_dir;      // combined: writer.kernels
  // databases.writer.properties / databases.reader.properties (ASCII):
  // 1 write the model under property_dir and stop (the reference's driver
  // does the same, src/execute.cpp:115-125), 2 read it from there
  int property_mode = 0;
  std::string property_dir;

  int max_sig_step() const { return nstep / nstep_between_samples; }

  // Flattened copies backing sfb_problem_view.
  std::vector<int> v_src_ispec, v_src_shot, v_src_wavefield;
  std::vector<float> v_src_array, v_src_stf;
  std::vector<int> v_rec_ispec;
  std::vector<float> v_rec_lagrange, v_rec_sin, v_rec_cos;
  std::vector<int> v_cp_ac_self, v_cp_ac_other, v_cp_el_self, v_cp_el_other;
  std::vector<float> v_cp_ac_f, v_cp_ac_nx, v_cp_ac_nz, v_cp_el_f, v_cp_el_nx, v_cp_el_nz;
  // Element-private points (P-SV): elements with no boundary points and no
  // source, receiver or adjoint source get elem_private = 1; their interior
  // (N-2)^2 points belong to them alone.  finalize() renumbers the P-SV
  // field so that the other (shared) points come first: [0, nshared_psv).
  std::vector<uint8_t> elem_private;  // [nspec]
  int nshared_psv = 0;
  void finalize();  // locate sources / receivers, private points, flat copies
  void fill_view(sfb_problem_view *v) const;
};

Problem problem_from_yaml_text(const std::string &parameter_text, const std::string &default_text);
Problem problem_from_yaml(const std::string &parameter_file,
                          const std::string &default_file);
Problem problem_from_structured(const sfb_structured_desc &d);

}  // namespace sfb
