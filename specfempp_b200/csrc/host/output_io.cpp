// ASCII output / checkpoint files in the reference's layout; see output_io.hpp.
#include "output_io.hpp"

#include <cstdint>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <functional>
#include <type_traits>
#include <sstream>
#include <stdexcept>

namespace fs = std::filesystem;

namespace sfb {
namespace {

const char *medium_name(int m) {
  return m == MEDIUM_ELASTIC_PSV ? "elastic_psv" : m == MEDIUM_ELASTIC_SH ? "elastic_sh" : "acoustic";
}
constexpr int kMediaTags[3] = {MEDIUM_ELASTIC_PSV, MEDIUM_ELASTIC_SH, MEDIUM_ACOUSTIC};

void write_meta(const std::string &group, const std::string &name, const std::vector<long> &dims) {
  std::ofstream m(fs::path(group) / (name + ".meta"));
  if (!m) throw std::runtime_error("could not open " + (fs::path(group) / (name + ".meta")).string());
  m << "rank " << dims.size() << "\n";
  m << "dims ";
  for (long d : dims) m << d << " ";
  m << "\n";
}

size_t product(const std::vector<long> &dims) {
  size_t n = 1;
  for (long d : dims) n *= static_cast<size_t>(d);
  return n;
}

template <typename T> void write_values(const std::string &group, const std::string &name, const T *data, size_t n) {
  const std::string path = (fs::path(group) / (name + ".txt")).string();
  FILE *f = std::fopen(path.c_str(), "w");
  if (!f) throw std::runtime_error("could not open " + path);
  for (size_t i = 0; i < n; ++i) {
    if constexpr (std::is_integral_v<T>)
      std::fprintf(f, "%d\n", static_cast<int>(data[i]));
    else
      std::fprintf(f, "%.10e\n", static_cast<double>(data[i]));  // setprecision(10), scientific
  }
  std::fclose(f);
}

template <typename T>
void write_dataset(const std::string &group, const std::string &name, const std::vector<long> &dims, const T *data,
                   size_t n) {
  if (n != product(dims)) throw std::invalid_argument("dataset " + name + ": size does not match its dims");
  write_meta(group, name, dims);
  write_values(group, name, data, n);
}

}  // namespace

std::string ascii_group(const std::string &dir) {
  std::error_code ec;
  if (fs::exists(dir)) fs::remove_all(dir, ec);
  fs::create_directories(dir);
  return dir;
}

void ascii_write(const std::string &g, const std::string &n, const std::vector<long> &d, const float *p, size_t k) {
  write_dataset(g, n, d, p, k);
}
void ascii_write(const std::string &g, const std::string &n, const std::vector<long> &d, const double *p, size_t k) {
  write_dataset(g, n, d, p, k);
}
void ascii_write(const std::string &g, const std::string &n, const std::vector<long> &d, const int *p, size_t k) {
  write_dataset(g, n, d, p, k);
}

std::vector<double> ascii_read(const std::string &group, const std::string &name, const std::vector<long> &dims) {
  const fs::path meta = fs::path(group) / (name + ".meta");
  std::ifstream m(meta);
  if (!m) throw std::runtime_error("missing dataset metadata " + meta.string());
  std::string tok;
  size_t rank = 0;
  m >> tok >> rank;
  if (tok != "rank") throw std::runtime_error("corrupted metadata " + meta.string());
  m >> tok;
  if (tok != "dims" || rank != dims.size()) throw std::runtime_error("dataset " + meta.string() + ": rank mismatch");
  for (size_t i = 0; i < rank; ++i) {
    long d = 0;
    m >> d;
    if (d != dims[i]) throw std::runtime_error("dataset " + meta.string() + ": dims mismatch");
  }
  const size_t n = product(dims);
  std::vector<double> out(n);
  const std::string path = (fs::path(group) / (name + ".txt")).string();
  FILE *f = std::fopen(path.c_str(), "r");
  if (!f) throw std::runtime_error("could not open " + path);
  for (size_t i = 0; i < n; ++i)
    if (std::fscanf(f, "%lf", &out[i]) != 1) {
      std::fclose(f);
      throw std::runtime_error("dataset " + path + " has fewer values than its dims");
    }
  std::fclose(f);
  return out;
}

namespace {

// Elements of medium m in reference (ispec) order, and each global point's
// coordinates.
std::vector<int> medium_elements(const Assembly &a, int m) {
  // the reference's compute element order (compute_mesh.cpp:239-279): by
  // element type in the order of material_definitions.hpp ELEMENT_TYPES --
  // within a medium boundary tag none, then acoustic_free_surface, stacey,
  // composite_stacey_dirichlet -- and mesh order within a type.  The tag of
  // an element follows from its points' boundary bits (bit 0 Stacey, bit 1
  // acoustic free surface).
  const int nn = a.ngll * a.ngll;
  auto tag = [&](int e) {
    uint8_t bits = 0;
    for (int k = 0; k < nn; ++k) bits |= a.bnd[static_cast<size_t>(e) * nn + k];
    const bool stacey = bits & 1, surface = bits & 2;
    return stacey && surface ? 3 : stacey ? 2 : surface ? 1 : 0;
  };
  std::vector<int> el;
  for (int t : {0, 1, 2, 3})
    for (int e = 0; e < a.nspec; ++e)
      if (a.medium[e] == m && tag(e) == t) el.push_back(e);
  return el;
}

// Raw values of a dataset whose .meta gives `dims` (the file may hold more
// values than the dims' product: padded element tiles).
std::vector<double> read_values(const std::string &group, const std::string &name, const std::vector<long> &dims,
                                size_t count) {
  ascii_read(group, name, dims);  // checks the metadata
  std::vector<double> out(count);
  const std::string path = (fs::path(group) / (name + ".txt")).string();
  FILE *f = std::fopen(path.c_str(), "r");
  if (!f) throw std::runtime_error("could not open " + path);
  for (size_t i = 0; i < count; ++i)
    if (std::fscanf(f, "%lf", &out[i]) != 1) {
      std::fclose(f);
      throw std::runtime_error("dataset " + path + " has fewer values than its element tiles");
    }
  std::fclose(f);
  return out;
}

// Position of value (i, iz, ix) of an element-tiled dataset
// (domain_view.hpp:100-160): tile i / chunk, then i % chunk + iz chunk +
// ix chunk nz.
size_t tile_index(long i, int iz, int ix, int chunk, int n) {
  return static_cast<size_t>(i / chunk) * chunk * n * n + (i % chunk) + static_cast<size_t>(iz) * chunk +
         static_cast<size_t>(ix) * chunk * n;
}

std::string step_group(int step) {
  char buf[32];
  std::snprintf(buf, sizeof(buf), "Step%06d", step);  // utilities::to_zero_lead(istep, 6)
  return buf;
}

const char *field_name(int m, int which) {
  static const char *el[3] = {"Displacement", "Velocity", "Acceleration"};
  static const char *ac[3] = {"Potential", "PotentialDot", "PotentialDotDot"};
  return m == MEDIUM_ACOUSTIC ? ac[which] : el[which];
}

}  // namespace

namespace {
// Media the reference's wavefield writer and reader visit besides the three
// this library computes (include/io/wavefield/{writer,reader}.tpp): their
// groups are written empty, with the reference's component counts
// (enumerations/medium.hpp: poroelastic 4, elastic_psv_t 3).
struct ExtraMedium {
  const char *name;
  int ncomp;
};
constexpr ExtraMedium kExtraMedia[2] = {{"poroelastic", 4}, {"elastic_psv_t", 3}};

// The reference's Stacey store (compute/boundary_values/*): per medium with a
// container (elastic_psv, acoustic) the elements whose boundary tag is
// stacey, numbered in mesh order (IndexMapping, -1 elsewhere); values
// (nelements, nz, nx, nstep, ncomp) column-major.  `slot` gives this
// library's store slot per mesh element (exactly those elements; SH
// elements have no reference container and are left out).
struct RefStacey {
  std::vector<int> mapping;  // [nspec]
  long count[4] = {0, 0, 0, 0};
};
RefStacey ref_stacey(const Assembly &a, const std::vector<int> &slot) {
  RefStacey r;
  r.mapping.assign(a.nspec, -1);
  for (int e = 0; e < a.nspec; ++e) {
    const int m = a.medium[e];
    if (slot[e] < 0 || m == MEDIUM_ELASTIC_SH) continue;
    r.mapping[e] = static_cast<int>(r.count[m]++);
  }
  return r;
}
}  // namespace

void write_forward_wavefield(const Problem &P, const std::string &dir, const ForwardSnapshot &s, bool fresh) {
  const Assembly &a = P.asmb;
  const int n = a.ngll, nn = n * n;
  const fs::path rootp = fs::path(dir) / "ForwardWavefield";
  // a fresh file starts empty; a periodic snapshot adds its step group
  const std::string root = fresh ? ascii_group(rootp.string()) : (fs::create_directories(rootp), rootp.string());
  const bool coordinates = fresh || !fs::exists(rootp / "Coordinates");
  const std::string coords = coordinates ? ascii_group((rootp / "Coordinates").string()) : std::string();
  for (int m : kMediaTags) {
    if (!coordinates) break;
    const std::string g = ascii_group((fs::path(coords) / medium_name(m)).string());
    const std::vector<int> el = medium_elements(a, m);
    const long ne = static_cast<long>(el.size()), ng = a.nglob[m];
    std::vector<float> x(ng, 0.f), z(ng, 0.f);
    std::vector<int> mapping(static_cast<size_t>(ne) * nn);
    for (long i = 0; i < ne; ++i)
      for (int iz = 0; iz < n; ++iz)
        for (int ix = 0; ix < n; ++ix) {
          const size_t p = static_cast<size_t>(el[i]) * nn + iz * n + ix;
          const int ig = a.iglob[p];
          mapping[i + ne * (iz + static_cast<size_t>(n) * ix)] = ig;  // (nelem, nz, nx), column-major
          x[ig] = static_cast<float>(a.coord[p * 2]);
          z[ig] = static_cast<float>(a.coord[p * 2 + 1]);
        }
    ascii_write(g, "X", {ng}, x.data(), x.size());
    ascii_write(g, "Z", {ng}, z.data(), z.size());
    ascii_write(g, "mapping", {ne, n, n}, mapping.data(), mapping.size());
  }
  for (const ExtraMedium &x : kExtraMedia) {
    if (!coordinates) break;
    const std::string g = ascii_group((fs::path(coords) / x.name).string());
    ascii_write(g, "X", {0}, static_cast<const float *>(nullptr), 0);
    ascii_write(g, "Z", {0}, static_cast<const float *>(nullptr), 0);
    ascii_write(g, "mapping", {0, n, n}, static_cast<const int *>(nullptr), 0);
  }
  const std::string step = ascii_group((fs::path(root) / step_group(s.step)).string());
  for (int m : kMediaTags) {
    const std::string g = ascii_group((fs::path(step) / medium_name(m)).string());
    const long ng = a.nglob[m], nc = a.ncomp(m);
    for (int w = 0; w < 3; ++w) {
      const std::vector<float> &f = s.field[m][w];
      if (f.size() != static_cast<size_t>(ng * nc)) throw std::invalid_argument("snapshot field has the wrong size");
      ascii_write(g, field_name(m, w), {ng, nc}, f.data(), f.size());  // [c][g] = (nglob, ncomp) column-major
    }
  }
  for (const ExtraMedium &x : kExtraMedia) {
    const std::string g = ascii_group((fs::path(step) / x.name).string());
    for (int w = 0; w < 3; ++w) ascii_write(g, field_name(0, w), {0, x.ncomp}, static_cast<const float *>(nullptr), 0);
  }
  const std::string stacey =
      ascii_group((fs::path(ascii_group((fs::path(step) / "Boundary").string())) / "Stacey").string());
  const RefStacey r = ref_stacey(a, s.slot);
  ascii_write(stacey, "IndexMapping", {static_cast<long>(a.nspec)}, r.mapping.data(), r.mapping.size());
  const long T = P.nstep, K = s.nstacey;
  if (!s.store.empty() && s.store.size() != static_cast<size_t>(T) * K * nn * 2)
    throw std::invalid_argument("snapshot store has the wrong size");
  for (const auto &[m, name] : {std::pair<int, const char *>{MEDIUM_ELASTIC_PSV, "ElasticAcceleration"},
                                std::pair<int, const char *>{MEDIUM_ACOUSTIC, "AcousticAcceleration"}}) {
    const long ne = r.count[m], nc = a.ncomp(m);
    std::vector<float> v(static_cast<size_t>(ne) * nn * T * nc, 0.f);
    if (!s.store.empty())
      for (int e = 0; e < a.nspec; ++e) {
        if (a.medium[e] != m || r.mapping[e] < 0) continue;
        const long i = r.mapping[e], k = s.slot[e];
        for (long t = 0; t < T; ++t)
          for (int iz = 0; iz < n; ++iz)
            for (int ix = 0; ix < n; ++ix)
              for (int c = 0; c < nc; ++c)
                v[i + ne * (iz + n * (ix + static_cast<size_t>(n) * (t + T * c)))] =
                    s.store[(((static_cast<size_t>(t) * K + k) * nn) + iz * n + ix) * 2 + c];
      }
    ascii_write(stacey, name, {ne, n, n, T, nc}, v.data(), v.size());
  }
  ascii_write(stacey, "PoroelasticAcceleration", {0, n, n, T, 4}, static_cast<const float *>(nullptr), 0);
}

ForwardSnapshot read_forward_wavefield(const Problem &P, const std::string &dir, const std::vector<int> &slot,
                                       int nstacey) {
  const Assembly &a = P.asmb;
  const int n = a.ngll, nn = n * n;
  ForwardSnapshot s;
  s.step = P.nstep;
  s.nstacey = nstacey;
  s.slot = slot;
  const fs::path step = fs::path(dir) / "ForwardWavefield" / step_group(P.nstep);
  if (!fs::exists(step)) throw std::runtime_error("no forward wavefield at " + step.string());
  for (int m : kMediaTags) {
    const std::string g = (step / medium_name(m)).string();
    const long ng = a.nglob[m], nc = a.ncomp(m);
    for (int w = 0; w < 3; ++w) {
      const std::vector<double> d = ascii_read(g, field_name(m, w), {ng, nc});
      s.field[m][w].assign(d.begin(), d.end());
    }
  }
  const std::string stacey = (step / "Boundary" / "Stacey").string();
  const std::vector<double> map = ascii_read(stacey, "IndexMapping", {static_cast<long>(a.nspec)});
  const RefStacey r = ref_stacey(a, slot);
  for (int e = 0; e < a.nspec; ++e)
    if (static_cast<int>(map[e]) != r.mapping[e])
      throw std::runtime_error("the stored boundary layout does not match this mesh");
  const long T = P.nstep, K = nstacey;
  s.store.assign(static_cast<size_t>(T) * K * nn * 2, 0.f);
  for (const auto &[m, name] : {std::pair<int, const char *>{MEDIUM_ELASTIC_PSV, "ElasticAcceleration"},
                                std::pair<int, const char *>{MEDIUM_ACOUSTIC, "AcousticAcceleration"}}) {
    const long ne = r.count[m], nc = a.ncomp(m);
    const std::vector<double> v = ascii_read(stacey, name, {ne, n, n, T, nc});
    for (int e = 0; e < a.nspec; ++e) {
      if (a.medium[e] != m || r.mapping[e] < 0) continue;
      const long i = r.mapping[e], k = slot[e];
      for (long t = 0; t < T; ++t)
        for (int iz = 0; iz < n; ++iz)
          for (int ix = 0; ix < n; ++ix)
            for (int c = 0; c < nc; ++c)
              s.store[(((static_cast<size_t>(t) * K + k) * nn) + iz * n + ix) * 2 + c] =
                  static_cast<float>(v[i + ne * (iz + n * (ix + static_cast<size_t>(n) * (t + T * c)))]);
    }
  }
  return s;
}

void write_kernels(const Problem &P, const std::string &dir, const std::vector<double> kern[6], int chunk) {
  const Assembly &a = P.asmb;
  const int n = a.ngll, nn = n * n;
  if (chunk < 1) throw std::invalid_argument("element chunk must be >= 1");
  const std::string root = ascii_group((fs::path(dir) / "Kernels").string());
  for (int m : kMediaTags) {
    const std::string g = ascii_group((fs::path(root) / (std::string(medium_name(m)) + "_isotropic")).string());
    const std::vector<int> el = medium_elements(a, m);
    const long ne = static_cast<long>(el.size());
    const long ntiles = (ne + chunk - 1) / chunk;
    const size_t span = static_cast<size_t>(ntiles) * chunk * nn;
    // domain_view.hpp:100-160: tile (i / chunk), then (i % chunk) + iz chunk + ix chunk nz
    auto place = [&](const std::function<double(size_t)> &value, std::vector<double> &out) {
      out.assign(span, 0.0);
      for (long i = 0; i < ne; ++i)
        for (int iz = 0; iz < n; ++iz)
          for (int ix = 0; ix < n; ++ix)
            out[tile_index(i, iz, ix, chunk, n)] = value(static_cast<size_t>(el[i]) * nn + iz * n + ix);
    };
    std::vector<double> buf;
    std::vector<float> fbuf;
    auto write_float = [&](const char *name, const std::function<double(size_t)> &value) {
      place(value, buf);
      fbuf.assign(buf.begin(), buf.end());
      // the .meta carries the logical dims; the values are the padded tiles
      write_meta(g, name, {ne, n, n});
      write_values(g, name, fbuf.data(), fbuf.size());
    };
    write_float("X", [&](size_t p) { return a.coord[p * 2]; });
    write_float("Z", [&](size_t p) { return a.coord[p * 2 + 1]; });
    const std::vector<std::pair<const char *, int>> names =
        m == MEDIUM_ACOUSTIC ? std::vector<std::pair<const char *, int>>{{"rho", 0}, {"kappa", 2}, {"rhop", 3}, {"alpha", 4}}
                             : std::vector<std::pair<const char *, int>>{{"rho", 0}, {"mu", 1}, {"kappa", 2},
                                                                         {"rhop", 3}, {"alpha", 4}, {"beta", 5}};
    for (const auto &[name, q] : names) write_float(name, [&](size_t p) { return kern[q][p]; });
  }
}

namespace {
// Property datasets per medium (the reference's properties containers:
// medium/dim2/elastic/isotropic/properties_container.hpp, kappa mu rho;
// acoustic/isotropic/properties_container.hpp, rho_inverse kappa).
std::vector<const char *> property_names(int m) {
  if (m == MEDIUM_ACOUSTIC) return {"rho_inverse", "kappa"};
  return {"kappa", "mu", "rho"};
}
template <typename A> auto property_array(A &a, const std::string &name) -> decltype(a.kappa.data()) {
  if (name == "kappa") return a.kappa.data();
  if (name == "mu") return a.mu.data();
  if (name == "rho") return a.rho.data();
  if (name == "rho_inverse") return a.rho_inverse.data();
  throw std::invalid_argument("unknown property " + name);
}
}  // namespace

void write_properties(const Problem &P, const std::string &dir, int chunk) {
  const Assembly &a = P.asmb;
  const int n = a.ngll, nn = n * n;
  if (chunk < 1) throw std::invalid_argument("element chunk must be >= 1");
  const std::string root = ascii_group((fs::path(dir) / "Properties").string());
  for (int m : kMediaTags) {
    const std::string g = ascii_group((fs::path(root) / (std::string(medium_name(m)) + "_isotropic")).string());
    const std::vector<int> el = medium_elements(a, m);
    const long ne = static_cast<long>(el.size());
    const size_t span = static_cast<size_t>((ne + chunk - 1) / chunk) * chunk * nn;
    std::vector<float> buf;
    auto write_float = [&](const char *name, const std::function<float(size_t)> &value) {
      buf.assign(span, 0.f);
      for (long i = 0; i < ne; ++i)
        for (int iz = 0; iz < n; ++iz)
          for (int ix = 0; ix < n; ++ix)
            buf[tile_index(i, iz, ix, chunk, n)] = value(static_cast<size_t>(el[i]) * nn + iz * n + ix);
      write_meta(g, name, {ne, n, n});
      write_values(g, name, buf.data(), buf.size());
    };
    write_float("X", [&](size_t p) { return static_cast<float>(a.coord[p * 2]); });
    write_float("Z", [&](size_t p) { return static_cast<float>(a.coord[p * 2 + 1]); });
    for (const char *name : property_names(m)) {
      const float *v = property_array(a, name);
      write_float(name, [&](size_t p) { return v[p]; });
    }
  }
}

void read_properties(Problem &P, const std::string &dir, int chunk) {
  Assembly &a = P.asmb;
  const int n = a.ngll, nn = n * n;
  if (chunk < 1) throw std::invalid_argument("element chunk must be >= 1");
  const fs::path root = fs::path(dir) / "Properties";
  if (!fs::is_directory(root)) throw std::runtime_error("no Properties folder under " + dir);
  for (int m : kMediaTags) {
    const std::vector<int> el = medium_elements(a, m);
    const long ne = static_cast<long>(el.size());
    if (ne == 0) continue;
    const std::string g = (root / (std::string(medium_name(m)) + "_isotropic")).string();
    const size_t span = static_cast<size_t>((ne + chunk - 1) / chunk) * chunk * nn;
    for (const char *name : property_names(m)) {
      const std::vector<double> v = read_values(g, name, {ne, n, n}, span);
      float *dst = property_array(a, name);
      for (long i = 0; i < ne; ++i)
        for (int iz = 0; iz < n; ++iz)
          for (int ix = 0; ix < n; ++ix)
            dst[static_cast<size_t>(el[i]) * nn + iz * n + ix] = static_cast<float>(v[tile_index(i, iz, ix, chunk, n)]);
    }
    // the quantities the kernels derive from the stored ones
    for (long i = 0; i < ne; ++i)
      for (int k = 0; k < nn; ++k) {
        const size_t p = static_cast<size_t>(el[i]) * nn + k;
        if (m == MEDIUM_ACOUSTIC) {
          if (!(a.rho_inverse[p] > 0.f)) throw std::runtime_error("acoustic rho_inverse must be positive");
          a.rho[p] = 1.0f / a.rho_inverse[p];
        } else {
          if (!(a.rho[p] > 0.f)) throw std::runtime_error("elastic rho must be positive");
          a.rho_inverse[p] = 1.0f / a.rho[p];
        }
      }
  }
}

}  // namespace sfb
