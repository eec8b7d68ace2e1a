#include "assembly.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <fstream>
#include <limits>
#include <map>
#include <numeric>
#include <sstream>
#include <stdexcept>

namespace sfb {

namespace {

// 4- and 9-node shape functions and their (xi, gamma) derivatives
// (reference: src/jacobian/shape_functions.cpp).  Control-node order:
// corners BL, BR, TR, TL; then mid-edges B, R, T, L; then centre.
void shape_functions(int ngnod, double xi, double ga, double *N, double *dNdxi,
                     double *dNdga) {
  const double sp = xi + 1, sm = xi - 1, tp = ga + 1, tm = ga - 1;
  if (ngnod == 4) {
    N[0] = 0.25 * sm * tm;
    N[1] = -0.25 * sp * tm;
    N[2] = 0.25 * sp * tp;
    N[3] = -0.25 * sm * tp;
    dNdxi[0] = 0.25 * tm;
    dNdxi[1] = -0.25 * tm;
    dNdxi[2] = 0.25 * tp;
    dNdxi[3] = -0.25 * tp;
    dNdga[0] = 0.25 * sm;
    dNdga[1] = -0.25 * sp;
    dNdga[2] = 0.25 * sp;
    dNdga[3] = -0.25 * sm;
  } else if (ngnod == 9) {
    const double s2 = 2 * xi, t2 = 2 * ga, ss = xi * xi, tt = ga * ga, st = xi * ga;
    N[0] = 0.25 * sm * st * tm;
    N[1] = 0.25 * sp * st * tm;
    N[2] = 0.25 * sp * st * tp;
    N[3] = 0.25 * sm * st * tp;
    N[4] = 0.5 * tm * ga * (1 - ss);
    N[5] = 0.5 * sp * xi * (1 - tt);
    N[6] = 0.5 * tp * ga * (1 - ss);
    N[7] = 0.5 * sm * xi * (1 - tt);
    N[8] = (1 - ss) * (1 - tt);
    dNdxi[0] = 0.25 * tm * ga * (s2 - 1);
    dNdxi[1] = 0.25 * tm * ga * (s2 + 1);
    dNdxi[2] = 0.25 * tp * ga * (s2 + 1);
    dNdxi[3] = 0.25 * tp * ga * (s2 - 1);
    dNdga[0] = 0.25 * sm * xi * (t2 - 1);
    dNdga[1] = 0.25 * sp * xi * (t2 - 1);
    dNdga[2] = 0.25 * sp * xi * (t2 + 1);
    dNdga[3] = 0.25 * sm * xi * (t2 + 1);
    dNdxi[4] = -st * tm;
    dNdxi[5] = 0.5 * (1 - tt) * (s2 + 1);
    dNdxi[6] = -st * tp;
    dNdxi[7] = 0.5 * (1 - tt) * (s2 - 1);
    dNdga[4] = 0.5 * (1 - ss) * (t2 - 1);
    dNdga[5] = -st * sp;
    dNdga[6] = 0.5 * (1 - ss) * (t2 + 1);
    dNdga[7] = -st * sm;
    dNdxi[8] = -s2 * (1 - tt);
    dNdga[8] = -t2 * (1 - ss);
  } else {
    throw std::invalid_argument("wrong number of control nodes");
  }
}

struct Map2D {
  double x, z, xxi, zxi, xga, zga;
};

Map2D element_map(const Assembly &a, int ispec, double xi, double ga) {
  double N[9], dx[9], dg[9];
  shape_functions(a.ngnod, xi, ga, N, dx, dg);
  Map2D m{0, 0, 0, 0, 0, 0};
  for (int k = 0; k < a.ngnod; ++k) {
    const int n = a.mesh_knods[static_cast<size_t>(ispec) * a.ngnod + k];
    const double X = a.mesh_coorg[2 * n], Z = a.mesh_coorg[2 * n + 1];
    m.x += N[k] * X;
    m.z += N[k] * Z;
    m.xxi += dx[k] * X;
    m.zxi += dx[k] * Z;
    m.xga += dg[k] * X;
    m.zga += dg[k] * Z;
  }
  return m;
}

// Outward edge normal scaled by the element Jacobian
// (reference: core/specfem/point/partial_derivatives.hpp:369-396).
void edge_normal(int edge, float xix, float xiz, float gax, float gaz, float J,
                 float &nx, float &nz) {
  switch (edge) {
  case EDGE_BOTTOM: nx = -1.0f * gax * J; nz = -1.0f * gaz * J; break;
  case EDGE_TOP: nx = gax * J; nz = gaz * J; break;
  case EDGE_LEFT: nx = -1.0f * xix * J; nz = -1.0f * xiz * J; break;
  case EDGE_RIGHT: nx = xix * J; nz = xiz * J; break;
  default: throw std::invalid_argument("Invalid edge type");
  }
}

bool on_boundary(int type, int iz, int ix, int n) {
  switch (type) {
  case EDGE_TOP: return iz == n - 1;
  case EDGE_BOTTOM: return iz == 0;
  case EDGE_LEFT: return ix == 0;
  case EDGE_RIGHT: return ix == n - 1;
  case CORNER_BOTTOM_RIGHT: return iz == 0 && ix == n - 1;
  case CORNER_BOTTOM_LEFT: return iz == 0 && ix == 0;
  case CORNER_TOP_RIGHT: return iz == n - 1 && ix == n - 1;
  case CORNER_TOP_LEFT: return iz == n - 1 && ix == 0;
  }
  return false;
}

// (ix, iz) of the ip-th point of an edge, in increasing order along it
// (reference: interface_container.tpp get_points_on_edge).
void edge_point(int edge, int ip, int n, int &ix, int &iz) {
  switch (edge) {
  case EDGE_BOTTOM: ix = ip; iz = 0; return;
  case EDGE_TOP: ix = ip; iz = n - 1; return;
  case EDGE_LEFT: ix = 0; iz = ip; return;
  case EDGE_RIGHT: ix = n - 1; iz = ip; return;
  }
  throw std::invalid_argument("Invalid edge type");
}

// Point index of the ip-th edge point as walked by the reference's edge
// iterator for the receiving ("self") element and for the other ("coupled")
// element (reference: include/policies/edge.hpp:119-170).  The coupled map
// for LEFT/RIGHT addresses the opposite column, exactly as the reference
// does; horizontal interfaces (TOP/BOTTOM) address the shared edge.
void self_point(int edge, int ip, int n, int &iz, int &ix) {
  switch (edge) {
  case EDGE_BOTTOM: iz = 0; ix = ip; return;
  case EDGE_TOP: iz = n - 1; ix = n - 1 - ip; return;
  case EDGE_LEFT: iz = ip; ix = 0; return;
  case EDGE_RIGHT: iz = n - 1 - ip; ix = n - 1; return;
  }
  throw std::invalid_argument("Invalid edge type");
}
void coupled_point(int edge, int ip, int n, int &iz, int &ix) {
  switch (edge) {
  case EDGE_BOTTOM: iz = 0; ix = n - 1 - ip; return;
  case EDGE_TOP: iz = n - 1; ix = ip; return;
  case EDGE_LEFT: iz = n - 1 - ip; ix = n - 1; return;
  case EDGE_RIGHT: iz = ip; ix = 0; return;
  }
  throw std::invalid_argument("Invalid edge type");
}

}  // namespace

int Assembly::count_elements(int m) const {
  return static_cast<int>(std::count(medium.begin(), medium.end(), m));
}

Assembly build_assembly(const Mesh2D &mesh, int ngll) {
  Assembly a;
  a.ngll = ngll;
  a.nspec = mesh.nspec;
  a.quad = Quadrature(ngll);
  a.ngnod = mesh.ngnod;
  a.mesh_knods = mesh.knods;
  a.mesh_coorg = mesh.coorg;
  const int n = ngll;
  const size_t nloc = a.nloc();
  a.medium.resize(a.nspec);
  for (int e = 0; e < a.nspec; ++e) a.medium[e] = mesh.medium_of(e);

  // Geometry (reference: src/compute/compute_partial_derivatives.cpp,
  // src/jacobian/jacobian.cpp).
  a.coord.resize(2 * nloc);
  a.xix.resize(nloc);
  a.xiz.resize(nloc);
  a.gammax.resize(nloc);
  a.gammaz.resize(nloc);
  a.jacobian.resize(nloc);
  for (int e = 0; e < a.nspec; ++e)
    for (int iz = 0; iz < n; ++iz)
      for (int ix = 0; ix < n; ++ix) {
        const size_t p = (static_cast<size_t>(e) * n + iz) * n + ix;
        const Map2D m = element_map(a, e, a.quad.xi[ix], a.quad.xi[iz]);
        const double J = m.xxi * m.zga - m.xga * m.zxi;
        if (J <= 0.0) {
          std::ostringstream os;
          os << "non-positive Jacobian in element " << e;
          throw std::runtime_error(os.str());
        }
        a.coord[2 * p] = m.x;
        a.coord[2 * p + 1] = m.z;
        a.xix[p] = static_cast<float>(m.zga / J);
        a.gammax[p] = static_cast<float>(-m.zxi / J);
        a.xiz[p] = static_cast<float>(-m.xga / J);
        a.gammaz[p] = static_cast<float>(m.xxi / J);
        a.jacobian[p] = static_cast<float>(J);
      }

  // Mesh-global numbering: merge coincident GLL points (reference:
  // src/compute/compute_mesh.cpp:46-110, tolerance 1e-6 of the typical
  // element size).
  {
    double xmin = 1e300, xmax = -1e300, zmin = 1e300, zmax = -1e300;
    for (size_t p = 0; p < nloc; ++p) {
      xmin = std::min(xmin, a.coord[2 * p]);
      xmax = std::max(xmax, a.coord[2 * p]);
      zmin = std::min(zmin, a.coord[2 * p + 1]);
      zmax = std::max(zmax, a.coord[2 * p + 1]);
    }
    const double typ = std::max(xmax - xmin, zmax - zmin) /
                       std::sqrt(static_cast<double>(std::max(a.nspec, 1)));
    const double tol = 1e-6 * typ;
    std::vector<size_t> order(nloc);
    std::iota(order.begin(), order.end(), size_t(0));
    std::sort(order.begin(), order.end(), [&](size_t i, size_t j) {
      return a.coord[2 * i] < a.coord[2 * j];
    });
    a.ibool.assign(nloc, -1);
    int ig = 0;
    size_t g0 = 0;
    while (g0 < nloc) {
      size_t g1 = g0 + 1;
      while (g1 < nloc && a.coord[2 * order[g1]] - a.coord[2 * order[g1 - 1]] <= tol) ++g1;
      std::sort(order.begin() + g0, order.begin() + g1, [&](size_t i, size_t j) {
        return a.coord[2 * i + 1] < a.coord[2 * j + 1];
      });
      for (size_t k = g0; k < g1; ++k) {
        if (k > g0 && a.coord[2 * order[k] + 1] - a.coord[2 * order[k - 1] + 1] > tol) ++ig;
        a.ibool[order[k]] = ig;
      }
      ++ig;
      g0 = g1;
    }
    a.nglob_mesh = ig;
  }

  // Per-medium compact numbering, first touch in element order (reference:
  // include/compute/fields/impl/field_impl.tpp:32-60 numbers per medium in
  // its own traversal order; only the layout differs).
  {
    std::vector<int> map(static_cast<size_t>(a.nglob_mesh) * 4, -1);
    a.iglob.assign(nloc, -1);
    for (int e = 0; e < a.nspec; ++e) {
      const int m = a.medium[e];
      for (int k = 0; k < n * n; ++k) {
        const size_t p = static_cast<size_t>(e) * n * n + k;
        int &slot = map[static_cast<size_t>(a.ibool[p]) * 4 + m];
        if (slot < 0) slot = a.nglob[m]++;
        a.iglob[p] = slot;
      }
    }
  }

  // Material per local point (reference: include/medium/dim2/*/isotropic/
  // material.hpp; elastic kappa = rho (vp^2 - 4/3 vs^2), mu = rho vs^2;
  // acoustic kappa = rho vp^2, rho_inverse = 1 / rho).
  a.kappa.resize(nloc);
  a.mu.resize(nloc);
  a.rho.resize(nloc);
  a.rho_inverse.resize(nloc);
  const bool per_point = !mesh.gll_rho.empty();
  if (per_point && mesh.gll_ngll != n)
    throw std::invalid_argument("per-GLL-point model has the wrong NGLL");
  for (int e = 0; e < a.nspec; ++e) {
    const Material &mat = mesh.materials[mesh.material[e]];
    for (int k = 0; k < n * n; ++k) {
      const size_t p = static_cast<size_t>(e) * n * n + k;
      double rho = mat.rho, vp = mat.cp, vs = mat.cs;
      if (per_point) {
        rho = mesh.gll_rho[p];
        vp = mesh.gll_vp[p];
        vs = mat.acoustic ? 0.0 : static_cast<double>(mesh.gll_vs[p]);
      }
      if (a.medium[e] == MEDIUM_ACOUSTIC) {
        a.kappa[p] = static_cast<float>(rho * vp * vp);
        a.rho_inverse[p] = 1.0f / static_cast<float>(rho);
        a.rho[p] = static_cast<float>(rho);
        a.mu[p] = 0.0f;
      } else {
        a.kappa[p] = static_cast<float>(rho * (vp * vp - (4.0 / 3.0) * vs * vs));
        a.mu[p] = static_cast<float>(rho * vs * vs);
        a.rho[p] = static_cast<float>(rho);
        a.rho_inverse[p] = 1.0f / static_cast<float>(rho);
      }
    }
  }

  // Boundaries (reference: src/compute/boundaries/impl/{stacey,
  // acoustic_free_surface}.cpp).  Entries are applied in file order grouped
  // by element; for a corner point the last Stacey edge through it sets the
  // normal and weight.
  a.bnd.assign(nloc, 0);
  a.bnd_nx.assign(nloc, 0.f);
  a.bnd_nz.assign(nloc, 0.f);
  a.bnd_w.assign(nloc, 0.f);
  a.elem_boundary.assign(a.nspec, BOUNDARY_NONE);
  auto add_tag = [&](int e, int tag) {
    int &t = a.elem_boundary[e];
    if (t == BOUNDARY_NONE) t = tag;
    else if (t != tag) t = BOUNDARY_COMPOSITE_STACEY_DIRICHLET;
  };
  {
    std::map<int, std::vector<int>> by_elem;
    for (size_t i = 0; i < mesh.afs_ispec.size(); ++i)
      by_elem[mesh.afs_ispec[i]].push_back(static_cast<int>(i));
    for (auto &kv : by_elem)
      for (int i : kv.second) {
        const int e = kv.first;
        add_tag(e, BOUNDARY_ACOUSTIC_FREE_SURFACE);
        for (int iz = 0; iz < n; ++iz)
          for (int ix = 0; ix < n; ++ix)
            if (on_boundary(mesh.afs_type[i], iz, ix, n))
              a.bnd[(static_cast<size_t>(e) * n + iz) * n + ix] |= 2;
      }
  }
  {
    std::map<int, std::vector<int>> by_elem;
    for (size_t i = 0; i < mesh.abs_ispec.size(); ++i)
      by_elem[mesh.abs_ispec[i]].push_back(static_cast<int>(i));
    for (auto &kv : by_elem)
      for (int i : kv.second) {
        const int e = kv.first;
        const int type = mesh.abs_type[i];
        add_tag(e, BOUNDARY_STACEY);
        for (int iz = 0; iz < n; ++iz)
          for (int ix = 0; ix < n; ++ix) {
            if (!on_boundary(type, iz, ix, n)) continue;
            const size_t p = (static_cast<size_t>(e) * n + iz) * n + ix;
            a.bnd[p] |= 1;
            int edge = type;
            if (type == CORNER_BOTTOM_LEFT || type == CORNER_TOP_LEFT) edge = EDGE_LEFT;
            if (type == CORNER_BOTTOM_RIGHT || type == CORNER_TOP_RIGHT) edge = EDGE_RIGHT;
            const bool vertical = (edge == EDGE_LEFT || edge == EDGE_RIGHT);
            a.bnd_w[p] = static_cast<float>(vertical ? a.quad.w[iz] : a.quad.w[ix]);
            edge_normal(edge, a.xix[p], a.xiz[p], a.gammax[p], a.gammaz[p],
                        a.jacobian[p], a.bnd_nx[p], a.bnd_nz[p]);
          }
      }
  }

  // Fluid-solid coupling (reference: include/compute/coupled_interfaces/
  // interface_container.tpp:349-428, 540-587; medium 1 = elastic).
  for (size_t ie = 0; ie < mesh.fs_elastic.size(); ++ie) {
    const int e1 = mesh.fs_elastic[ie], e2 = mesh.fs_acoustic[ie];
    int found = 0, edge1 = -1, edge2 = -1;
    for (int c1 = 0; c1 < 4; ++c1)
      for (int c2 = 0; c2 < 4; ++c2) {
        if (c1 == c2) continue;
        int ix, iz;
        edge_point(c1, 1, n, ix, iz);
        int jx, jz;
        edge_point(c1, 0, n, jx, jz);
        const size_t q1 = (static_cast<size_t>(e1) * n + iz) * n + ix;
        const size_t q0 = (static_cast<size_t>(e1) * n + jz) * n + jx;
        const double size = std::hypot(a.coord[2 * q1] - a.coord[2 * q0],
                                       a.coord[2 * q1 + 1] - a.coord[2 * q0 + 1]);
        bool ok = true;
        for (int ip = 0; ip < n && ok; ++ip) {
          int ax, az, bx, bz;
          edge_point(c1, ip, n, ax, az);
          edge_point(c2, ip, n, bx, bz);
          const size_t pa = (static_cast<size_t>(e1) * n + az) * n + ax;
          const size_t pb = (static_cast<size_t>(e2) * n + bz) * n + bx;
          const double d = std::hypot(a.coord[2 * pa] - a.coord[2 * pb],
                                      a.coord[2 * pa + 1] - a.coord[2 * pb + 1]);
          if (d / size > 1e-6) ok = false;
        }
        if (ok) {
          ++found;
          edge1 = c1;
          edge2 = c2;
        }
      }
    if (found != 1) throw std::runtime_error("Number of connected edges is not 1");
    std::vector<float> factor(n), nx(n), nz(n);
    for (int ip = 0; ip < n; ++ip) {
      int ix, iz;
      edge_point(edge1, ip, n, ix, iz);
      const size_t p = (static_cast<size_t>(e1) * n + iz) * n + ix;
      edge_normal(edge1, a.xix[p], a.xiz[p], a.gammax[p], a.gammaz[p],
                  a.jacobian[p], nx[ip], nz[ip]);
      const bool vertical = (edge1 == EDGE_LEFT || edge1 == EDGE_RIGHT);
      factor[ip] = static_cast<float>(vertical ? a.quad.w[iz] : a.quad.w[ix]);
    }
    for (int ip = 0; ip < n; ++ip) {
      int sz, sx, cz, cx;
      // elastic receives: self = elastic (edge1), coupled = acoustic (edge2)
      self_point(edge1, ip, n, sz, sx);
      coupled_point(edge2, ip, n, cz, cx);
      a.couple_elastic.push_back(
          {a.iglob[(static_cast<size_t>(e1) * n + sz) * n + sx],
           a.iglob[(static_cast<size_t>(e2) * n + cz) * n + cx], factor[ip],
           nx[ip], nz[ip]});
      // acoustic receives: self = acoustic (edge2), coupled = elastic (edge1)
      self_point(edge2, ip, n, sz, sx);
      coupled_point(edge1, ip, n, cz, cx);
      a.couple_acoustic.push_back(
          {a.iglob[(static_cast<size_t>(e2) * n + sz) * n + sx],
           a.iglob[(static_cast<size_t>(e1) * n + cz) * n + cx], factor[ip],
           -nx[ip], -nz[ip]});
    }
  }
  return a;
}

// ---------------------------------------------------------------------------
// Point location (reference: src/algorithms/locate_point.cpp).  The rough
// search for the closest GLL point uses a bucket grid instead of a linear
// scan; ties keep the lowest (ispec, iz, ix) like the reference's scan.
// ---------------------------------------------------------------------------
namespace {
struct PointGrid {
  double x0, z0, h;
  int nx, nz;
  std::vector<std::vector<uint32_t>> cells;
};

const PointGrid &grid_for(const Assembly &a) {
  static thread_local const Assembly *cached = nullptr;
  static thread_local size_t cached_n = 0;
  static thread_local PointGrid g;
  if (cached == &a && cached_n == a.nloc()) return g;
  const size_t nloc = a.nloc();
  double xmin = 1e300, xmax = -1e300, zmin = 1e300, zmax = -1e300;
  for (size_t p = 0; p < nloc; ++p) {
    xmin = std::min(xmin, a.coord[2 * p]);
    xmax = std::max(xmax, a.coord[2 * p]);
    zmin = std::min(zmin, a.coord[2 * p + 1]);
    zmax = std::max(zmax, a.coord[2 * p + 1]);
  }
  const double area = std::max((xmax - xmin) * (zmax - zmin), 1e-30);
  g.h = std::max(std::sqrt(area / std::max<double>(a.nspec, 1)), 1e-12);
  g.x0 = xmin;
  g.z0 = zmin;
  g.nx = static_cast<int>((xmax - xmin) / g.h) + 1;
  g.nz = static_cast<int>((zmax - zmin) / g.h) + 1;
  g.cells.assign(static_cast<size_t>(g.nx) * g.nz, {});
  for (size_t p = 0; p < nloc; ++p) {
    int cx = std::min(g.nx - 1, std::max(0, static_cast<int>((a.coord[2 * p] - g.x0) / g.h)));
    int cz = std::min(g.nz - 1, std::max(0, static_cast<int>((a.coord[2 * p + 1] - g.z0) / g.h)));
    g.cells[static_cast<size_t>(cz) * g.nx + cx].push_back(static_cast<uint32_t>(p));
  }
  cached = &a;
  cached_n = nloc;
  return g;
}

size_t closest_point(const Assembly &a, double x, double z) {
  const PointGrid &g = grid_for(a);
  const int cx = std::min(g.nx - 1, std::max(0, static_cast<int>((x - g.x0) / g.h)));
  const int cz = std::min(g.nz - 1, std::max(0, static_cast<int>((z - g.z0) / g.h)));
  double best = std::numeric_limits<double>::max();
  size_t bestp = 0;
  for (int r = 0;; ++r) {
    for (int jz = cz - r; jz <= cz + r; ++jz)
      for (int jx = cx - r; jx <= cx + r; ++jx) {
        if (std::max(std::abs(jz - cz), std::abs(jx - cx)) != r) continue;
        if (jx < 0 || jz < 0 || jx >= g.nx || jz >= g.nz) continue;
        for (uint32_t p : g.cells[static_cast<size_t>(jz) * g.nx + jx]) {
          const double d = std::hypot(x - a.coord[2 * p], z - a.coord[2 * p + 1]);
          if (d < best || (d == best && p < bestp)) {
            best = d;
            bestp = p;
          }
        }
      }
    // Every unvisited cell is at least r*h away from the query point.
    if (best < r * g.h || r > std::max(g.nx, g.nz)) break;
  }
  return bestp;
}
}  // namespace

LocalCoord locate_point(const Assembly &a, double x, double z) {
  const int n = a.ngll;
  const size_t p = closest_point(a, x, z);
  const int eg = static_cast<int>(p / (n * n));
  int iz_guess = static_cast<int>((p / n) % n), ix_guess = static_cast<int>(p % n);
  // Candidates: the guess element, then elements sharing one of its corners.
  std::vector<int> corners = {a.ibool[(static_cast<size_t>(eg) * n + 0) * n + 0],
                              a.ibool[(static_cast<size_t>(eg) * n + n - 1) * n + 0],
                              a.ibool[(static_cast<size_t>(eg) * n + 0) * n + n - 1],
                              a.ibool[(static_cast<size_t>(eg) * n + n - 1) * n + n - 1]};
  std::vector<int> cand = {eg};
  {
    const PointGrid &g = grid_for(a);
    std::vector<int> seen;
    for (int c = 0; c < 4; ++c) {
      const int cp = (c & 1) ? n - 1 : 0, cq = (c & 2) ? n - 1 : 0;
      const size_t q = (static_cast<size_t>(eg) * n + cq) * n + cp;
      const double qx = a.coord[2 * q], qz = a.coord[2 * q + 1];
      const int cx = std::min(g.nx - 1, std::max(0, static_cast<int>((qx - g.x0) / g.h)));
      const int cz = std::min(g.nz - 1, std::max(0, static_cast<int>((qz - g.z0) / g.h)));
      for (int jz = cz - 1; jz <= cz + 1; ++jz)
        for (int jx = cx - 1; jx <= cx + 1; ++jx) {
          if (jx < 0 || jz < 0 || jx >= g.nx || jz >= g.nz) continue;
          for (uint32_t r : g.cells[static_cast<size_t>(jz) * g.nx + jx]) {
            const int e = static_cast<int>(r / (n * n));
            const int k = static_cast<int>(r % (n * n));
            const int kz = k / n, kx = k % n;
            if (e == eg || !((kz == 0 || kz == n - 1) && (kx == 0 || kx == n - 1))) continue;
            if (std::find(corners.begin(), corners.end(), a.ibool[r]) != corners.end())
              seen.push_back(e);
          }
        }
    }
    std::sort(seen.begin(), seen.end());
    seen.erase(std::unique(seen.begin(), seen.end()), seen.end());
    cand.insert(cand.end(), seen.begin(), seen.end());
  }
  double final_dist = std::numeric_limits<double>::max();
  LocalCoord best{eg, 0, 0};
  for (int e : cand) {
    double xi = a.quad.xi[ix_guess], ga = a.quad.xi[iz_guess];
    for (int it = 0; it < 100; ++it) {
      const Map2D m = element_map(a, e, xi, ga);
      const double J = m.xxi * m.zga - m.xga * m.zxi;
      const double xix = m.zga / J, gax = -m.zxi / J, xiz = -m.xga / J, gaz = m.xxi / J;
      const double dx = -(m.x - x), dz = -(m.z - z);
      xi += xix * dx + xiz * dz;
      ga += gax * dx + gaz * dz;
      xi = std::min(1.01, std::max(-1.01, xi));
      ga = std::min(1.01, std::max(-1.01, ga));
    }
    const Map2D m = element_map(a, e, xi, ga);
    const double d = std::hypot(m.x - x, m.z - z);
    if (d < final_dist) {
      final_dist = d;
      best = {e, xi, ga};
    }
    ix_guess = n / 2;
    iz_guess = n / 2;
  }
  return best;
}

// ---------------------------------------------------------------------------
// Source time functions (reference: src/source_time_function/{ricker,dirac,
// dgaussian}.cpp and utilities.cpp).
// ---------------------------------------------------------------------------
namespace {
double gaussian_d(int order, double t, double f0) {
  const double a = M_PI * M_PI * f0 * f0;
  const double e = std::exp(-a * t * t);
  switch (order) {
  case 0: return -e / (2.0 * a);
  case 1: return t * e;
  case 2: return (1.0 - 2.0 * a * t * t) * e;
  case 3: return -2.0 * a * t * (3.0 - 2.0 * a * t * t) * e;
  case 4: return -2.0 * a * (3.0 - 12.0 * a * t * t + 4.0 * a * a * t * t * t * t) * e;
  }
  return 0.0;
}
}  // namespace

double Source::t0() const {
  if (stf == TABLE) return table_t0 + tshift;
  return -1.2 / f0 + tshift;
}

double Source::value(double t) const {
  const double tt = t - tshift;
  switch (stf) {
  case RICKER:
    return -factor * gaussian_d(use_trick_for_better_pressure ? 4 : 2, tt, f0);
  case DIRAC:
    return -factor * gaussian_d(use_trick_for_better_pressure ? 2 : 0, tt, f0);
  case DGAUSSIAN:
    return -factor * gaussian_d(use_trick_for_better_pressure ? 3 : 1, tt, f0);
  }
  return 0.0;
}

double resolve_t0(std::vector<Source> &sources, double user_t0) {
  if (sources.empty()) return user_t0;
  double min_t0 = std::numeric_limits<double>::max();
  double min_tshift = std::numeric_limits<double>::max();
  for (auto &s : sources) {
    min_t0 = std::min(min_t0, s.t0());
    min_tshift = std::min(min_tshift, s.tshift);
  }
  if (std::abs(user_t0) > std::numeric_limits<float>::epsilon()) {
    if (user_t0 > min_t0 - min_tshift)
      throw std::runtime_error(
          "User defined start time is less than minimum required for stability");
    return user_t0;
  }
  for (auto &s : sources) {
    if (s.stf != Source::TABLE) s.tshift = s.t0() - min_t0;
  }
  return min_t0;
}

LocatedSource locate_source(const Assembly &a, const Source &s, double t0,
                            double dt, int nstep) {
  const int n = a.ngll;
  LocatedSource out;
  const LocalCoord lc = locate_point(a, s.x, s.z);
  out.ispec = lc.ispec;
  out.medium = a.medium[lc.ispec];
  const int nc = a.ncomp(out.medium);
  std::vector<double> hx(n), hpx(n), hz(n), hpz(n);
  lagrange_interpolants(a.quad, lc.xi, hx.data(), hpx.data());
  lagrange_interpolants(a.quad, lc.gamma, hz.data(), hpz.data());
  out.array.assign(static_cast<size_t>(nc) * n * n, 0.f);
  const double rad = M_PI / 180.0 * s.angle;
  if (s.kind == Source::FORCE) {
    // reference: src/source/force_source.cpp:18-100
    for (int iz = 0; iz < n; ++iz)
      for (int ix = 0; ix < n; ++ix) {
        const double h = hx[ix] * hz[iz];
        if (nc == 1) {
          out.array[iz * n + ix] = static_cast<float>(h);
        } else {
          out.array[iz * n + ix] = static_cast<float>(std::sin(rad) * h);
          out.array[n * n + iz * n + ix] = static_cast<float>(-1.0 * std::cos(rad) * h);
        }
      }
  } else if (s.kind == Source::MOMENT_TENSOR) {
    // reference: src/source/moment_tensor_source.cpp; the element's
    // partial derivatives are interpolated to the source point.
    if (out.medium != MEDIUM_ELASTIC_PSV)
      throw std::runtime_error("Moment tensor source requires an elastic P-SV element");
    double dxix = 0, dxiz = 0, dgax = 0, dgaz = 0;
    for (int iz = 0; iz < n; ++iz)
      for (int ix = 0; ix < n; ++ix) {
        const size_t p = (static_cast<size_t>(lc.ispec) * n + iz) * n + ix;
        const double h = hx[ix] * hz[iz];
        dxix += h * a.xix[p];
        dxiz += h * a.xiz[p];
        dgax += h * a.gammax[p];
        dgaz += h * a.gammaz[p];
      }
    for (int iz = 0; iz < n; ++iz)
      for (int ix = 0; ix < n; ++ix) {
        const double dsdx = (hpx[ix] * dxix) * hz[iz] + hx[ix] * (hpz[iz] * dgax);
        const double dsdz = (hpx[ix] * dxiz) * hz[iz] + hx[ix] * (hpz[iz] * dgaz);
        out.array[iz * n + ix] = static_cast<float>(s.mxx * dsdx + s.mxz * dsdz);
        out.array[n * n + iz * n + ix] = static_cast<float>(s.mxz * dsdx + s.mzz * dsdz);
      }
  } else if (s.kind == Source::ADJOINT || s.kind == Source::EXTERNAL) {
    // reference: src/source/adjoint_source.cpp, src/source/external.cpp
    // (Lagrange weights in every component)
    for (int c = 0; c < nc; ++c)
      for (int iz = 0; iz < n; ++iz)
        for (int ix = 0; ix < n; ++ix) out.array[static_cast<size_t>(c) * n * n + iz * n + ix] = static_cast<float>(hx[ix] * hz[iz]);
  } else {
    throw std::runtime_error("unsupported source kind");
  }
  // STF table sampled at t0 + i dt, identical in every component
  // (reference: ricker.cpp compute_source_time_function).
  out.stf.assign(static_cast<size_t>(nstep) * nc, 0.f);
  for (int i = 0; i < nstep; ++i) {
    double v;
    if (s.stf == Source::TABLE) {
      const size_t ncol = s.stf_table.size() / std::max(nstep, 1);
      v = (static_cast<size_t>(i) * std::max<size_t>(ncol, 1) < s.stf_table.size())
              ? s.stf_table[static_cast<size_t>(i) * std::max<size_t>(ncol, 1)]
              : 0.0;
      for (int c = 0; c < nc; ++c) {
        const size_t k = static_cast<size_t>(i) * ncol + std::min<size_t>(c, ncol ? ncol - 1 : 0);
        out.stf[static_cast<size_t>(i) * nc + c] =
            static_cast<float>(k < s.stf_table.size() ? s.stf_table[k] : 0.0);
      }
      continue;
    }
    v = s.value(t0 + i * dt);
    for (int c = 0; c < nc; ++c) out.stf[static_cast<size_t>(i) * nc + c] = static_cast<float>(v);
  }
  return out;
}

LocatedReceiver locate_receiver(const Assembly &a, const Receiver &r) {
  // reference: src/compute/compute_receivers.cpp:59-90
  const int n = a.ngll;
  LocatedReceiver out;
  const LocalCoord lc = locate_point(a, r.x, r.z);
  out.ispec = lc.ispec;
  out.medium = a.medium[lc.ispec];
  std::vector<double> hx(n), hz(n);
  lagrange_interpolants(a.quad, lc.xi, hx.data(), nullptr);
  lagrange_interpolants(a.quad, lc.gamma, hz.data(), nullptr);
  out.lagrange.resize(static_cast<size_t>(n) * n);
  for (int iz = 0; iz < n; ++iz)
    for (int ix = 0; ix < n; ++ix) out.lagrange[iz * n + ix] = static_cast<float>(hx[ix] * hz[iz]);
  out.sin_angle = static_cast<float>(std::sin(M_PI / 180.0 * r.angle));
  out.cos_angle = static_cast<float>(std::cos(M_PI / 180.0 * r.angle));
  return out;
}

std::vector<Receiver> read_stations(const std::string &path, double angle) {
  // reference: src/io/receivers.cpp (station network x z elevation burial)
  std::ifstream f(path);
  if (!f) throw std::runtime_error("Could not open STATIONS file: " + path);
  std::vector<Receiver> out;
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream is(line);
    Receiver r;
    if (!(is >> r.station >> r.network >> r.x >> r.z)) continue;
    r.angle = angle;
    out.push_back(r);
  }
  return out;
}

}  // namespace sfb
