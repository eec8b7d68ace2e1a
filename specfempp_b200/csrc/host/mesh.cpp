#include "mesh.hpp"

#include <cstdint>
#include <cstring>
#include <fstream>
#include <map>
#include <stdexcept>
#include <string>

namespace sfb {

namespace {

// One Fortran unformatted sequential record: int32 length, payload, int32
// length (reference: include/io/fortranio/fortran_io.tpp:45-64).
struct RecordReader {
  std::vector<char> buf;
  size_t pos = 0;

  explicit RecordReader(const std::string &path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("Could not open database file: " + path);
    buf.assign(std::istreambuf_iterator<char>(f),
               std::istreambuf_iterator<char>());
  }
  bool eof() const { return pos >= buf.size(); }
  int32_t peek_length() const {
    if (pos + 4 > buf.size()) throw std::runtime_error("database truncated");
    int32_t n;
    std::memcpy(&n, &buf[pos], 4);
    return n;
  }
  // Returns the payload of the next record and advances past it.
  std::vector<char> next() {
    const int32_t n = peek_length();
    if (n < 0 || pos + 8 + static_cast<size_t>(n) > buf.size())
      throw std::runtime_error("corrupt Fortran record in database");
    std::vector<char> rec(buf.begin() + pos + 4, buf.begin() + pos + 4 + n);
    int32_t tail;
    std::memcpy(&tail, &buf[pos + 4 + n], 4);
    if (tail != n) throw std::runtime_error("record length mismatch");
    pos += 8 + n;
    return rec;
  }
};

template <typename T> T get(const std::vector<char> &rec, size_t off) {
  if (off + sizeof(T) > rec.size())
    throw std::runtime_error("short Fortran record in database");
  T v;
  std::memcpy(&v, rec.data() + off, sizeof(T));
  return v;
}

// Boundary type of an acoustic free-surface entry given by control nodes
// (reference: read_boundaries.cpp get_boundary_type).
int free_surface_type(int kind, int e1, int e2, const int *cn) {
  if (kind == 1) {
    if (e1 == cn[0]) return CORNER_BOTTOM_LEFT;
    if (e1 == cn[1]) return CORNER_BOTTOM_RIGHT;
    if (e1 == cn[2]) return CORNER_TOP_RIGHT;
    if (e1 == cn[3]) return CORNER_TOP_LEFT;
  } else {
    auto is = [&](int a, int b) {
      return (e1 == cn[a] && e2 == cn[b]) || (e1 == cn[b] && e2 == cn[a]);
    };
    if (is(0, 1)) return EDGE_BOTTOM;
    if (is(0, 3)) return EDGE_LEFT;
    if (is(1, 2)) return EDGE_RIGHT;
    if (is(2, 3)) return EDGE_TOP;
  }
  throw std::invalid_argument(
      "Could not generate type of acoustic free surface boundary");
}

}  // namespace

Mesh2D read_database(const std::string &path, bool elastic_sh) {
  RecordReader rd(path);
  Mesh2D mesh;
  mesh.sh = elastic_sh;

  // Header: 64 records of run-time flags the solver does not use (the
  // reference reads and discards them, read_mesh_database.cpp:13-150), with
  // one optional 16-byte record (ATTENUATION_PERMITTIVITY) after record 42.
  std::vector<std::vector<char>> header;
  for (int i = 0; i < 42; ++i) header.push_back(rd.next());
  if (rd.peek_length() == 16) rd.next();
  for (int i = 42; i < 64; ++i) header.push_back(rd.next());
  const int nspec = get<int32_t>(header[2], 0);
  const int npgeo = get<int32_t>(header[3], 0);
  mesh.nspec = nspec;

  mesh.coorg.assign(2 * npgeo, 0.0);
  for (int i = 0; i < npgeo; ++i) {
    auto r = rd.next();
    const int ip = get<int32_t>(r, 0);
    if (ip < 1 || ip > npgeo) throw std::runtime_error("Error reading coordinates");
    mesh.coorg[2 * (ip - 1)] = get<double>(r, 4);
    mesh.coorg[2 * (ip - 1) + 1] = get<double>(r, 12);
  }

  auto p1 = rd.next();
  const int numat = get<int32_t>(p1, 0);
  const int ngnod = get<int32_t>(p1, 4);
  if (get<int32_t>(p1, 8) != nspec) throw std::runtime_error("nspec mismatch");
  mesh.ngnod = ngnod;
  auto p2 = rd.next();
  const int nelemabs = get<int32_t>(p2, 0);
  const int nelem_acforcing = get<int32_t>(p2, 4);
  const int nelem_acoustic_surface = get<int32_t>(p2, 8);
  const int num_fluid_solid = get<int32_t>(p2, 12);
  const int num_fluid_poro = get<int32_t>(p2, 16);
  const int num_solid_poro = get<int32_t>(p2, 20);
  const int nnodes_tangential = get<int32_t>(p2, 24);
  const int nelem_on_axis = get<int32_t>(p2, 28);
  if (num_fluid_poro || num_solid_poro)
    throw std::runtime_error("poroelastic interfaces are not on this path");

  rd.next();  // attenuation: n_sls, f0_reference, read_velocities_at_f0

  // Materials: n, indic, 13 doubles (read_material_properties.cpp).
  mesh.materials.resize(numat);
  for (int i = 0; i < numat; ++i) {
    auto r = rd.next();
    const int n = get<int32_t>(r, 0);
    const int indic = get<int32_t>(r, 4);
    if (n < 1 || n > numat) throw std::runtime_error("Wrong material set number");
    double v[13];
    for (int k = 0; k < 13; ++k) v[k] = get<double>(r, 8 + 8 * k);
    if (indic != 1)
      throw std::runtime_error(
          "only isotropic elastic/acoustic materials are on this path");
    Material &m = mesh.materials[n - 1];
    m.rho = v[0];
    m.cp = v[1];
    m.cs = v[2];
    m.qkappa = v[5];
    m.qmu = v[6];
    m.acoustic = (v[2] == 0.0);
  }

  // Elements: n, kmato, knods[ngnod], pml.
  mesh.knods.assign(static_cast<size_t>(nspec) * ngnod, -1);
  mesh.material.assign(nspec, -1);
  for (int i = 0; i < nspec; ++i) {
    auto r = rd.next();
    const int n = get<int32_t>(r, 0);
    const int kmato = get<int32_t>(r, 4);
    if (n < 1 || n > nspec || kmato < 1 || kmato > numat)
      throw std::runtime_error("Error reading material indices");
    for (int k = 0; k < ngnod; ++k) {
      const int kn = get<int32_t>(r, 8 + 4 * k);
      if (kn == 0) throw std::runtime_error("Error reading knods");
      mesh.knods[static_cast<size_t>(n - 1) * ngnod + k] = kn - 1;
    }
    mesh.material[n - 1] = kmato - 1;
  }

  auto mpi = rd.next();  // ninterfaces, max_interface_size (MPI, unused)
  if (get<int32_t>(mpi, 0) != 0)
    throw std::runtime_error("partitioned (MPI) databases are not supported");

  // Absorbing edges: numabs, 4 logical codes, type, iedge[8].  Exactly one
  // code is set per record (read_boundaries.cpp read_absorbing_boundaries).
  for (int i = 0; i < nelemabs; ++i) {
    auto r = rd.next();
    const int num = get<int32_t>(r, 0);
    if (num < 1 || num > nspec) throw std::runtime_error("Wrong absorbing element number");
    int code[4];
    for (int k = 0; k < 4; ++k) code[k] = get<int32_t>(r, 4 + 4 * k);
    int ncode = (code[0] != 0) + (code[1] != 0) + (code[2] != 0) + (code[3] != 0);
    if (ncode != 1)
      throw std::runtime_error(
          "must have one and only one absorbing edge per absorbing line cited");
    int type = code[0] ? EDGE_BOTTOM : code[1] ? EDGE_RIGHT : code[2] ? EDGE_TOP : EDGE_LEFT;
    mesh.abs_ispec.push_back(num - 1);
    mesh.abs_type.push_back(type);
  }
  // The reference's corner search (find_corners) never matches, so only the
  // edge entries are kept; corner GLL points inherit the tag of every edge
  // through them and the normal/weight of the last such edge.

  for (int i = 0; i < nelem_acoustic_surface; ++i) {
    auto r = rd.next();
    const int ispec = get<int32_t>(r, 0) - 1;
    const int kind = get<int32_t>(r, 4);
    const int e1 = get<int32_t>(r, 8) - 1;
    const int e2 = get<int32_t>(r, 12) - 1;
    const int *cn = &mesh.knods[static_cast<size_t>(ispec) * ngnod];
    mesh.afs_ispec.push_back(ispec);
    mesh.afs_type.push_back(free_surface_type(kind, e1, e2, cn));
  }
  for (int i = 0; i < nelem_acforcing; ++i) rd.next();  // acoustic forcing: not on this path

  // Fluid-solid edges: (acoustic ispec, elastic ispec), 1-based
  // (read_interfaces.cpp reads medium2 then medium1).
  for (int i = 0; i < num_fluid_solid; ++i) {
    auto r = rd.next();
    const int a = get<int32_t>(r, 0) - 1;
    const int b = get<int32_t>(r, 4) - 1;
    mesh.fs_acoustic.push_back(a);
    mesh.fs_elastic.push_back(b);
  }

  rd.next();  // tangential-curve flags
  for (int i = 0; i < nnodes_tangential; ++i) rd.next();
  for (int i = 0; i < nelem_on_axis; ++i) rd.next();
  if (!rd.eof())
    throw std::runtime_error(
        "The Database file wasn't fully read. Is there anything written after "
        "axial elements?");

  // Fluid-solid pairs may be listed either way round; normalise to
  // (elastic, acoustic) by medium.
  for (size_t i = 0; i < mesh.fs_elastic.size(); ++i) {
    if (mesh.medium_of(mesh.fs_elastic[i]) == MEDIUM_ACOUSTIC)
      std::swap(mesh.fs_elastic[i], mesh.fs_acoustic[i]);
    if (mesh.medium_of(mesh.fs_acoustic[i]) != MEDIUM_ACOUSTIC ||
        mesh.medium_of(mesh.fs_elastic[i]) == MEDIUM_ACOUSTIC)
      throw std::runtime_error(
          "Coupled Interfaces: Interface is not between the correct mediums");
  }
  return mesh;
}

Mesh2D structured_mesh(const StructuredSpec &s,
                       const std::vector<Material> &materials,
                       const std::vector<int> &element_material, bool sh) {
  if (s.nx < 1 || s.nz < 1) throw std::invalid_argument("structured mesh needs nx, nz >= 1");
  Mesh2D m;
  m.nspec = s.nx * s.nz;
  m.ngnod = 4;
  m.sh = sh;
  m.materials = materials;
  if (static_cast<int>(element_material.size()) != m.nspec)
    throw std::invalid_argument("element_material must have nx*nz entries");
  m.material = element_material;
  const int npx = s.nx + 1, npz = s.nz + 1;
  m.coorg.resize(2 * static_cast<size_t>(npx) * npz);
  for (int j = 0; j < npz; ++j)
    for (int i = 0; i < npx; ++i) {
      const size_t id = static_cast<size_t>(j) * npx + i;
      m.coorg[2 * id] = s.x0 + (s.x1 - s.x0) * i / s.nx;
      m.coorg[2 * id + 1] = s.z0 + (s.z1 - s.z0) * j / s.nz;
    }
  m.knods.resize(4 * static_cast<size_t>(m.nspec));
  for (int iz = 0; iz < s.nz; ++iz)
    for (int ix = 0; ix < s.nx; ++ix) {
      const size_t e = static_cast<size_t>(iz) * s.nx + ix;
      const int bl = iz * npx + ix;
      m.knods[4 * e + 0] = bl;            // bottom-left
      m.knods[4 * e + 1] = bl + 1;        // bottom-right
      m.knods[4 * e + 2] = bl + npx + 1;  // top-right
      m.knods[4 * e + 3] = bl + npx;      // top-left
    }
  for (int iz = 0; iz < s.nz; ++iz)
    for (int ix = 0; ix < s.nx; ++ix) {
      const int e = iz * s.nx + ix;
      const bool on[4] = {iz == 0, ix == s.nx - 1, iz == s.nz - 1, ix == 0};
      for (int side = 0; side < 4; ++side) {
        if (!on[side]) continue;
        if (s.absorb[side]) {
          m.abs_ispec.push_back(e);
          m.abs_type.push_back(side);
        }
        if (side == EDGE_TOP && s.free_top_acoustic &&
            m.medium_of(e) == MEDIUM_ACOUSTIC) {
          m.afs_ispec.push_back(e);
          m.afs_type.push_back(EDGE_TOP);
        }
      }
    }
  // Fluid-solid edges between vertically or horizontally adjacent elements.
  for (int iz = 0; iz < s.nz; ++iz)
    for (int ix = 0; ix < s.nx; ++ix) {
      const int e = iz * s.nx + ix;
      const int nb[2] = {iz + 1 < s.nz ? e + s.nx : -1, ix + 1 < s.nx ? e + 1 : -1};
      for (int k = 0; k < 2; ++k) {
        if (nb[k] < 0) continue;
        const bool a1 = m.medium_of(e) == MEDIUM_ACOUSTIC;
        const bool a2 = m.medium_of(nb[k]) == MEDIUM_ACOUSTIC;
        if (a1 == a2) continue;
        m.fs_elastic.push_back(a1 ? nb[k] : e);
        m.fs_acoustic.push_back(a1 ? e : nb[k]);
      }
    }
  return m;
}

}  // namespace sfb
