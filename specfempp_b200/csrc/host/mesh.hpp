// In-memory 2D spectral-element mesh: control nodes, element connectivity,
// materials, absorbing / free-surface edges and fluid-solid coupling edges.
// It is what the reference's `specfem::mesh::mesh<dim2>` holds after
// `specfem::io::read_2d_mesh` (src/io/mesh/impl/fortran/dim2/mesh.cpp:26-195),
// reduced to the element types on the time-marching path.
#pragma once
#include <string>
#include <vector>

namespace sfb {

// Medium / boundary / wavefield tag values equal the reference's enum ordinals
// (include/enumerations/medium.hpp:39-69, include/enumerations/wavefield.hpp:17)
// so that integers crossing the C ABI mean the same thing on both sides.
enum MediumTag : int {
  MEDIUM_ELASTIC_PSV = 0,
  MEDIUM_ELASTIC_SH = 1,
  MEDIUM_ELASTIC_PSV_T = 2,
  MEDIUM_ACOUSTIC = 3,
};
enum BoundaryTag : int {
  BOUNDARY_NONE = 0,
  BOUNDARY_ACOUSTIC_FREE_SURFACE = 1,
  BOUNDARY_STACEY = 2,
  BOUNDARY_COMPOSITE_STACEY_DIRICHLET = 3,
};
enum SeismogramType : int {
  SEIS_DISPLACEMENT = 0,
  SEIS_VELOCITY = 1,
  SEIS_ACCELERATION = 2,
  SEIS_PRESSURE = 3,
  SEIS_ROTATION = 4,
};
// Element edge / corner identifiers (reference: specfem::enums::boundaries).
enum EdgeType : int {
  EDGE_BOTTOM = 0,
  EDGE_RIGHT = 1,
  EDGE_TOP = 2,
  EDGE_LEFT = 3,
  CORNER_BOTTOM_LEFT = 4,
  CORNER_BOTTOM_RIGHT = 5,
  CORNER_TOP_RIGHT = 6,
  CORNER_TOP_LEFT = 7,
};

struct Material {
  bool acoustic = false;  // indic == 1 and cs == 0
  double rho = 0, cp = 0, cs = 0;
  double qkappa = 9999, qmu = 9999;
};

struct Mesh2D {
  int nspec = 0;
  int ngnod = 4;
  std::vector<double> coorg;   // [npgeo][2] control-node coordinates (x, z)
  std::vector<int> knods;      // [nspec][ngnod] 0-based control-node ids
  std::vector<int> material;   // [nspec] index into `materials`
  std::vector<Material> materials;
  bool sh = false;             // elastic materials are SH (else P-SV)
  // Absorbing (Stacey) edges in file order: (ispec, EdgeType).
  std::vector<int> abs_ispec, abs_type;
  // Acoustic free-surface edges / corners in file order: (ispec, EdgeType).
  std::vector<int> afs_ispec, afs_type;
  // Fluid-solid edges: (elastic ispec, acoustic ispec).
  std::vector<int> fs_elastic, fs_acoustic;
  // Optional per-GLL-point model override, [nspec][ngll][ngll] each; empty
  // means the element material is used (reference: property reader,
  // include/io/property/reader.tpp:17-44).
  std::vector<float> gll_rho, gll_vp, gll_vs;
  int gll_ngll = 0;

  int npgeo() const { return static_cast<int>(coorg.size() / 2); }
  int medium_of(int ispec) const {
    const Material &m = materials[material[ispec]];
    if (m.acoustic) return MEDIUM_ACOUSTIC;
    return sh ? MEDIUM_ELASTIC_SH : MEDIUM_ELASTIC_PSV;
  }
};

// Reads a 2D xmeshfem2D `database.bin` (Fortran unformatted records).
// Reference: src/io/mesh/impl/fortran/dim2/{mesh,read_mesh_database,
// read_parameters,read_material_properties,read_boundaries,
// read_interfaces,read_elements}.cpp.
Mesh2D read_database(const std::string &path, bool elastic_sh);

// Structured rectangle mesher standing in for xmeshfem2D on the benchmark
// workloads: nx * nz straight-edged 4-node quads over [x0, x1] x [z0, z1],
// element ispec = iz * nx + ix.  `absorb` flags the (bottom, right, top,
// left) sides as Stacey; `free_top_acoustic` marks the top edge of acoustic
// elements as an acoustic free surface.
struct StructuredSpec {
  int nx = 0, nz = 0;
  double x0 = 0, x1 = 1, z0 = 0, z1 = 1;
  bool absorb[4] = {false, false, false, false};
  bool free_top_acoustic = true;
};
Mesh2D structured_mesh(const StructuredSpec &spec,
                       const std::vector<Material> &materials,
                       const std::vector<int> &element_material, bool sh);

}  // namespace sfb
