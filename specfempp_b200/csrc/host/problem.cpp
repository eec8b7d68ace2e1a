#include "problem.hpp"

#include <cctype>
#include <cmath>
#include <filesystem>
#include <fstream>
#include <stdexcept>
#include <sys/stat.h>

#include "output_io.hpp"
#include "yaml_lite.hpp"

namespace sfb {

namespace {

bool file_exists(const std::string &p) {
  struct stat st;
  return stat(p.c_str(), &st) == 0;
}

std::string dirname_of(const std::string &p) {
  const size_t k = p.find_last_of('/');
  return k == std::string::npos ? std::string(".") : p.substr(0, k);
}

// Paths in the reference's files are relative to the directory the solver is
// started from; accept them relative to the working directory or to any
// ancestor of the parameter file's directory.
std::string resolve(const std::string &path, const std::string &config_file) {
  if (path.empty() || path[0] == '/' || file_exists(path)) return path;
  std::string dir = dirname_of(config_file);
  for (int depth = 0; depth < 12; ++depth) {
    const std::string cand = dir + "/" + path;
    if (file_exists(cand)) return cand;
    if (dir == "." || dir == "/" || dir.empty()) break;
    const size_t k = dir.find_last_of('/');
    if (k == std::string::npos) dir = ".";
    else if (k == 0) dir = "/";
    else dir = dir.substr(0, k);
  }
  return path;
}

int seismogram_type_of(const std::string &s) {
  if (s == "displacement") return SEIS_DISPLACEMENT;
  if (s == "velocity") return SEIS_VELOCITY;
  if (s == "acceleration") return SEIS_ACCELERATION;
  if (s == "pressure") return SEIS_PRESSURE;
  if (s == "rotation") return SEIS_ROTATION;
  throw std::runtime_error("Invalid seismogram type: " + s);
}

// One entry of a sources file (reference: src/io/sources.cpp:54-90,
// src/source/source.cpp, force_source.cpp, moment_tensor_source.cpp).
// External source time function (src/source_time_function/external.cpp):
// two-column "time value" ASCII files for the X and Z components; t0 is the
// first file time, dt the spacing of the first two lines (checked against
// the simulation's dt), then one sample per step.
void read_external_stf(const YNode &ext, int nstep, double dt, const std::string &config, Source &s) {
  if (const YNode *f = ext.get("format")) {
    std::string fmt = f->str();
    for (auto &ch : fmt) ch = static_cast<char>(std::tolower(ch));
    if (fmt != "ascii") throw std::runtime_error("Only ASCII format is supported");
  }
  const YNode *stf = ext.get("stf");
  if (!stf) throw std::runtime_error("Error: External source time function requires at least one component");
  std::string files[2];
  if (const YNode *x = stf->get("X-component")) files[0] = x->str();
  if (const YNode *z = stf->get("Z-component")) files[1] = z->str();
  if (files[0].empty() && files[1].empty()) {
    if (stf->get("Y-component")) throw std::runtime_error("External source time function only supports 2 components");
    throw std::runtime_error("Error: External source time function requires at least one component");
  }
  s.stf = Source::TABLE;
  s.stf_table.assign(static_cast<size_t>(nstep) * 2, 0.0);
  bool first = true;
  for (int c = 0; c < 2; ++c) {
    if (files[c].empty()) continue;
    const std::string path = resolve(files[c], config);
    std::ifstream in(path);
    if (!in) throw std::runtime_error("Error: External source time function file " + path + " does not exist");
    std::vector<std::pair<double, double>> rows;
    double t, v;
    while (in >> t >> v) rows.emplace_back(t, v);
    if (rows.size() < 2) throw std::runtime_error("Seismogram file " + path + " is not formatted correctly");
    if (first) {
      s.table_t0 = rows[0].first;
      if (std::abs((rows[1].first - rows[0].first) - dt) > 1e-6)
        throw std::runtime_error("The time step of the external source time function does not match the simulation time step");
      first = false;
    }
    if (rows.size() < static_cast<size_t>(nstep))
      throw std::runtime_error("External source time function file " + path + " has fewer samples than nstep");
    for (int i = 0; i < nstep; ++i) s.stf_table[static_cast<size_t>(i) * 2 + c] = rows[i].second;
  }
}

Source parse_source(const YNode &entry, double dt, int nstep, const std::string &config) {
  Source s;
  const YNode *body = nullptr;
  if ((body = entry.get("force"))) {
    s.kind = Source::FORCE;
    if (const YNode *a = body->get("angle")) s.angle = a->num();
  } else if ((body = entry.get("moment-tensor"))) {
    s.kind = Source::MOMENT_TENSOR;
    s.mxx = body->get("Mxx")->num();
    s.mzz = body->get("Mzz")->num();
    s.mxz = body->get("Mxz")->num();
  } else if ((body = entry.get("user-defined"))) {
    // src/io/sources.cpp:88-91, src/source/external.cpp: Lagrange weights in
    // every component, any source time function
    s.kind = Source::EXTERNAL;
  } else if ((body = entry.get("adjoint-source"))) {
    // src/io/sources.cpp:92-99, src/source/adjoint_source.cpp
    if (!body->get("station_name") || !body->get("network_name"))
      throw std::runtime_error("Station name and network name are required for adjoint source");
    s.kind = Source::ADJOINT;
    s.station = body->get("station_name")->str();
    s.network = body->get("network_name")->str();
    s.wavefield = 1;
  } else {
    throw std::runtime_error("Unknown source type (this path supports force, moment-tensor, user-defined and adjoint-source)");
  }
  s.x = body->get("x")->num();
  s.z = body->get("z")->num();
  if (const YNode *ext = body->get("External")) {
    read_external_stf(*ext, nstep, dt, config, s);
    return s;
  }
  if (s.kind == Source::ADJOINT) throw std::runtime_error("adjoint sources need an External source time function");
  const YNode *stf = nullptr;
  if ((stf = body->get("Ricker"))) {
    s.stf = Source::RICKER;
    s.f0 = stf->get("f0")->num();
  } else if ((stf = body->get("Dirac"))) {
    s.stf = Source::DIRAC;
    s.f0 = 1.0 / (10.0 * dt);  // reference: dirac.cpp:23
  } else if ((stf = body->get("dGaussian"))) {
    s.stf = Source::DGAUSSIAN;
    s.f0 = stf->get("f0")->num();
  } else {
    throw std::runtime_error("Error: source time function not recognized");
  }
  s.factor = stf->get("factor")->num();
  if (const YNode *t = stf->get("tshift")) s.tshift = t->num();
  return s;
}

// See Problem::elem_private.  The permutation keeps the relative order of
// the shared points and of the private points, so applying it again is the
// identity.
void mark_private_points(Problem &P) {
  Assembly &a = P.asmb;
  const int n = a.ngll, nn = n * n, m = MEDIUM_ELASTIC_PSV;
  P.elem_private.assign(a.nspec, 0);
  P.nshared_psv = a.nglob[m];
  if (n <= 2 || a.nglob[m] == 0) return;
  std::vector<int> refs(a.nglob[m], 0);
  std::vector<uint8_t> busy(a.nspec, 0);
  for (int e = 0; e < a.nspec; ++e) {
    if (a.medium[e] != m) continue;
    for (int k = 0; k < nn; ++k) {
      const size_t p = static_cast<size_t>(e) * nn + k;
      ++refs[a.iglob[p]];
      if (a.bnd[p]) busy[e] = 1;
    }
  }
  for (const auto &s : P.located_sources) busy[s.ispec] = 1;
  for (const auto &s : P.located_adjoint) busy[s.ispec] = 1;
  for (const auto &r : P.located_receivers) busy[r.ispec] = 1;
  std::vector<uint8_t> priv(a.nglob[m], 0);
  for (int e = 0; e < a.nspec; ++e) {
    if (a.medium[e] != m || busy[e]) continue;
    bool ok = true;
    for (int iz = 1; iz < n - 1 && ok; ++iz)
      for (int ix = 1; ix < n - 1; ++ix)
        if (refs[a.iglob[static_cast<size_t>(e) * nn + iz * n + ix]] != 1) { ok = false; break; }
    if (!ok) continue;
    P.elem_private[e] = 1;
    for (int iz = 1; iz < n - 1; ++iz)
      for (int ix = 1; ix < n - 1; ++ix) priv[a.iglob[static_cast<size_t>(e) * nn + iz * n + ix]] = 1;
  }
  std::vector<int> perm(a.nglob[m]);
  int next = 0;
  for (int g = 0; g < a.nglob[m]; ++g)
    if (!priv[g]) perm[g] = next++;
  P.nshared_psv = next;
  for (int g = 0; g < a.nglob[m]; ++g)
    if (priv[g]) perm[g] = next++;
  for (int e = 0; e < a.nspec; ++e)
    if (a.medium[e] == m)
      for (int k = 0; k < nn; ++k) {
        int &ig = a.iglob[static_cast<size_t>(e) * nn + k];
        ig = perm[ig];
      }
  for (auto &c : a.couple_acoustic) c.coupled_iglob = perm[c.coupled_iglob];
  for (auto &c : a.couple_elastic) c.self_iglob = perm[c.self_iglob];
}

}  // namespace

void Problem::finalize() {
  const Assembly &a = asmb;
  const int n = a.ngll;
  located_sources.clear();
  for (auto &s : sources) located_sources.push_back(locate_source(a, s, t0, dt, nstep));
  located_adjoint.clear();
  for (auto &s : adjoint_sources) {
    located_adjoint.push_back(locate_source(a, s, t0, dt, nstep));
    if (located_adjoint.back().medium != MEDIUM_ELASTIC_PSV)
      throw std::runtime_error("adjoint sources from files are supported in elastic P-SV elements");
  }
  located_receivers.clear();
  for (auto &r : receivers) located_receivers.push_back(locate_receiver(a, r));
  mark_private_points(*this);
  // flat copies
  const size_t ns = sources.size();
  v_src_ispec.assign(ns, 0);
  v_src_shot.assign(ns, 0);
  v_src_wavefield.assign(ns, 0);
  v_src_array.assign(ns * 2 * n * n, 0.f);
  v_src_stf.assign(ns * static_cast<size_t>(nstep) * 2, 0.f);
  for (size_t i = 0; i < ns; ++i) {
    const LocatedSource &L = located_sources[i];
    v_src_ispec[i] = L.ispec;
    v_src_shot[i] = source_shot.empty() ? 0 : source_shot[i];
    v_src_wavefield[i] = sources[i].wavefield;
    const int nc = a.ncomp(L.medium);
    for (int c = 0; c < nc; ++c)
      for (int k = 0; k < n * n; ++k)
        v_src_array[(i * 2 + c) * n * n + k] = L.array[static_cast<size_t>(c) * n * n + k];
    for (int t = 0; t < nstep; ++t)
      for (int c = 0; c < nc; ++c)
        v_src_stf[(i * nstep + t) * 2 + c] = L.stf[static_cast<size_t>(t) * nc + c];
  }
  const size_t nr = receivers.size();
  v_rec_ispec.assign(nr, 0);
  v_rec_lagrange.assign(nr * n * n, 0.f);
  v_rec_sin.assign(nr, 0.f);
  v_rec_cos.assign(nr, 1.f);
  for (size_t i = 0; i < nr; ++i) {
    const LocatedReceiver &L = located_receivers[i];
    v_rec_ispec[i] = L.ispec;
    std::copy(L.lagrange.begin(), L.lagrange.end(), v_rec_lagrange.begin() + i * n * n);
    v_rec_sin[i] = L.sin_angle;
    v_rec_cos[i] = L.cos_angle;
  }
  auto split = [](const std::vector<CouplingPoint> &cp, std::vector<int> &s,
                  std::vector<int> &o, std::vector<float> &f, std::vector<float> &x,
                  std::vector<float> &z) {
    s.clear(); o.clear(); f.clear(); x.clear(); z.clear();
    for (auto &p : cp) {
      s.push_back(p.self_iglob);
      o.push_back(p.coupled_iglob);
      f.push_back(p.factor);
      x.push_back(p.nx);
      z.push_back(p.nz);
    }
  };
  split(a.couple_acoustic, v_cp_ac_self, v_cp_ac_other, v_cp_ac_f, v_cp_ac_nx, v_cp_ac_nz);
  split(a.couple_elastic, v_cp_el_self, v_cp_el_other, v_cp_el_f, v_cp_el_nx, v_cp_el_nz);
}

void Problem::fill_view(sfb_problem_view *v) const {
  const Assembly &a = asmb;
  *v = sfb_problem_view{};
  v->ngll = a.ngll;
  v->nspec = a.nspec;
  v->nshots = nshots;
  v->nstep = nstep;
  v->nstep_between_samples = nstep_between_samples;
  v->dt = dt;
  v->t0 = t0;
  v->xi = a.quad.xi.data();
  v->wgll = a.quad.w.data();
  v->hprime = a.quad.hprime.data();
  v->medium = a.medium.data();
  v->iglob = a.iglob.data();
  for (int m = 0; m < 4; ++m) v->nglob[m] = a.nglob[m];
  v->xix = a.xix.data();
  v->xiz = a.xiz.data();
  v->gammax = a.gammax.data();
  v->gammaz = a.gammaz.data();
  v->jacobian = a.jacobian.data();
  v->kappa = a.kappa.data();
  v->mu = a.mu.data();
  v->rho = a.rho.data();
  v->rho_inverse = a.rho_inverse.data();
  v->bnd = a.bnd.data();
  v->bnd_nx = a.bnd_nx.data();
  v->bnd_nz = a.bnd_nz.data();
  v->bnd_w = a.bnd_w.data();
  v->ncouple_acoustic = static_cast<int>(v_cp_ac_self.size());
  v->couple_acoustic_self = v_cp_ac_self.data();
  v->couple_acoustic_other = v_cp_ac_other.data();
  v->couple_acoustic_factor = v_cp_ac_f.data();
  v->couple_acoustic_nx = v_cp_ac_nx.data();
  v->couple_acoustic_nz = v_cp_ac_nz.data();
  v->ncouple_elastic = static_cast<int>(v_cp_el_self.size());
  v->couple_elastic_self = v_cp_el_self.data();
  v->couple_elastic_other = v_cp_el_other.data();
  v->couple_elastic_factor = v_cp_el_f.data();
  v->couple_elastic_nx = v_cp_el_nx.data();
  v->couple_elastic_nz = v_cp_el_nz.data();
  v->nsources = static_cast<int>(v_src_ispec.size());
  v->src_ispec = v_src_ispec.data();
  v->src_shot = v_src_shot.data();
  v->src_wavefield = v_src_wavefield.data();
  v->src_array = v_src_array.data();
  v->src_stf = v_src_stf.data();
  v->nreceivers = static_cast<int>(v_rec_ispec.size());
  v->rec_ispec = v_rec_ispec.data();
  v->rec_lagrange = v_rec_lagrange.data();
  v->rec_sin = v_rec_sin.data();
  v->rec_cos = v_rec_cos.data();
  v->nseismogram_types = static_cast<int>(seismogram_types.size());
  v->seismogram_types = seismogram_types.data();
}

namespace {
Problem problem_from_nodes(std::shared_ptr<YNode> root, std::shared_ptr<YNode> defaults,
                           const std::string &parameter_file);
}

Problem problem_from_yaml(const std::string &parameter_file,
                          const std::string &default_file) {
  auto root = yaml_load_file(parameter_file);
  std::shared_ptr<YNode> defaults;
  if (!default_file.empty() && file_exists(default_file)) defaults = yaml_load_file(default_file);
  return problem_from_nodes(root, defaults, parameter_file);
}

// The reference's Python entry point takes the parameter and default
// dictionaries as YAML text (src/python/core.cpp:46-66); file paths in them
// are relative to the working directory.
Problem problem_from_yaml_text(const std::string &parameter_text, const std::string &default_text) {
  auto root = yaml_parse(parameter_text);
  std::shared_ptr<YNode> defaults;
  if (!default_text.empty()) defaults = yaml_parse(default_text);
  return problem_from_nodes(root, defaults, "");
}

namespace {
Problem problem_from_nodes(std::shared_ptr<YNode> root, std::shared_ptr<YNode> defaults,
                           const std::string &parameter_file) {
  const YNode *params = root->get("parameters");
  if (!params) throw std::runtime_error("parameter file has no 'parameters' node");

  const YNode *setup = params->get("simulation-setup");
  if (!setup) throw std::runtime_error("parameter file has no 'simulation-setup'");
  Problem P;
  // quadrature (parameter_parser/quadrature.cpp): GLL4 -> 5 points, GLL7 -> 8
  std::string qtype = "GLL4";
  if (const YNode *q = setup->path({"quadrature", "quadrature-type"})) qtype = q->str();
  else if (defaults) {
    if (const YNode *q = defaults->path({"default-parameters", "quadrature", "quadrature-type"}))
      qtype = q->str();
  }
  int ngll;
  if (qtype == "GLL4") ngll = 5;
  else if (qtype == "GLL7") ngll = 8;
  else throw std::runtime_error("unsupported quadrature-type: " + qtype);

  if (const YNode *ew = setup->get("elastic-wave")) {
    const std::string s = ew->str();
    P.elastic_sh = (s == "SH" || s == "sh");
  }
  const YNode *ts = setup->path({"solver", "time-marching", "time-scheme"});
  if (!ts) throw std::runtime_error("missing solver.time-marching.time-scheme");
  if (const YNode *t = ts->get("type"))
    if (t->str() != "Newmark") throw std::runtime_error("only the Newmark time scheme is supported");
  P.dt = ts->get("dt")->num();
  P.nstep = ts->get("nstep")->integer();
  double user_t0 = 0.0;
  if (const YNode *t = ts->get("t0")) user_t0 = t->num();

  const YNode *mode = setup->get("simulation-mode");
  std::string sources_key;
  if (mode && mode->get("combined")) {
    P.simulation = 1;
    if (const YNode *r = mode->path({"combined", "reader", "wavefield", "directory"}))
      P.wavefield_dir = resolve(r->str(), parameter_file);
    if (const YNode *k = mode->path({"combined", "writer", "kernels", "directory"}))
      P.kernel_dir = k->str();
    if (const YNode *s = mode->path({"combined", "writer", "seismogram"})) {
      P.write_seismograms = true;
      const YNode *d = s->get("directory") ? s->get("directory") : s->get("output-folder");
      P.seismogram_dir = d ? d->str() : ".";
    }
  } else if (mode && mode->get("forward")) {
    if (const YNode *s = mode->path({"forward", "writer", "seismogram"})) {
      P.write_seismograms = true;
      const YNode *d = s->get("directory") ? s->get("directory") : s->get("output-folder");
      P.seismogram_dir = d ? d->str() : ".";
    }
    if (const YNode *w = mode->path({"forward", "writer", "wavefield"})) {
      // src/parameter_parser/writer/wavefield.cpp:10-76: the folder must
      // exist (default: the working directory); time_interval and the
      // (parsed, otherwise unused) time_interval_by_memory exclude each
      // other; include_last_step defaults to true
      P.save_boundary_values = true;
      const YNode *d = w->get("directory");
      P.wavefield_dir = d ? d->str() : ".";
      if (!std::filesystem::is_directory(P.wavefield_dir))
        throw std::runtime_error("Output folder : " + P.wavefield_dir + " does not exist.");
      if (const YNode *t = w->get("time_interval")) P.wavefield_time_interval = t->integer();
      if (w->get("time_interval_by_memory") && P.wavefield_time_interval != 0)
        throw std::runtime_error("time_interval and time_interval_by_memory cannot be used simultaneously");
      if (const YNode *l = w->get("include_last_step")) P.wavefield_include_last_step = l->boolean();
      if (P.wavefield_time_interval < 0) throw std::runtime_error("time_interval must be >= 0");
    }
  }

  // mesh
  const YNode *db = params->path({"databases", "mesh-database"});
  if (!db) throw std::runtime_error("missing databases.mesh-database");
  Mesh2D mesh = read_database(resolve(db->str(), parameter_file), P.elastic_sh);
  P.asmb = build_assembly(mesh, ngll);

  // model files (src/parameter_parser/setup.cpp:114-122,
  // src/parameter_parser/writer/property.cpp:9-38)
  for (const auto &[key, mode] : {std::pair<const char *, int>{"writer", 1}, {"reader", 2}}) {
    const YNode *node = params->path({"databases", key, "properties"});
    if (!node) continue;
    std::string format = "ASCII";
    if (const YNode *f = node->get("format")) format = f->str();
    for (auto &ch : format) ch = static_cast<char>(std::tolower(static_cast<unsigned char>(ch)));
    if (format != "ascii") throw std::runtime_error("model format " + format + " is not supported (ASCII only)");
    std::string dir = ".";
    if (const YNode *d = node->get("directory")) dir = resolve(d->str(), parameter_file);
    if (!std::filesystem::is_directory(dir)) throw std::runtime_error("Model folder : " + dir + " does not exist.");
    P.property_mode = mode;
    P.property_dir = dir;
    break;
  }
  if (P.property_mode == 2) read_properties(P, P.property_dir, 1);

  // sources
  const YNode *src = params->get("sources");
  if (!src) throw std::runtime_error("missing sources");
  std::shared_ptr<YNode> sroot;
  const YNode *sdict = src;
  if (src->is_scalar()) {
    sroot = yaml_load_file(resolve(src->str(), parameter_file));
    sdict = sroot.get();
  }
  const YNode *list = sdict->get("sources");
  if (!list || !list->is_seq()) throw std::runtime_error("sources file has no 'sources' list");
  const std::string src_config = src->is_scalar() ? resolve(src->str(), parameter_file) : parameter_file;
  for (auto &e : list->seq) P.sources.push_back(parse_source(*e, P.dt, P.nstep, src_config));
  if (const YNode *ns = sdict->get("number-of-sources"))
    if (ns->integer() != static_cast<int>(P.sources.size()))
      throw std::runtime_error("Found only " + std::to_string(P.sources.size()) +
                               " number of sources; the file announces " + ns->str());
  int nadjoint = 0;
  for (const Source &s : P.sources) nadjoint += s.kind == Source::ADJOINT;
  if (nadjoint == static_cast<int>(P.sources.size())) throw std::runtime_error("No sources found in the sources file");
  if (P.simulation == 1 && nadjoint == 0) throw std::runtime_error("No adjoint sources found in the sources file");
  if (P.simulation == 0 && nadjoint > 0)
    throw std::runtime_error("Adjoint sources found in the sources file for forward simulation");
  P.t0 = resolve_t0(P.sources, user_t0);
  for (const Source &s : P.sources)
    if (s.stf == Source::TABLE && std::abs(P.t0 - s.table_t0) > 1e-6)
      throw std::runtime_error("The start time of the external source time function does not match the simulation start time");
  // adjoint sources drive the adjoint wavefield; the others the forward
  // (forward run) or backward (combined run) wavefield
  {
    std::vector<Source> keep;
    for (Source &s : P.sources) (s.kind == Source::ADJOINT ? P.adjoint_sources : keep).push_back(s);
    P.sources = keep;
  }
  P.source_shot.assign(P.sources.size(), 0);

  // receivers
  const YNode *rec = params->get("receivers");
  if (!rec) throw std::runtime_error("missing receivers");
  double angle = 0.0;
  if (const YNode *an = rec->get("angle")) angle = an->num();
  const YNode *st = rec->get("stations");
  if (st && st->is_scalar()) {
    P.receivers = read_stations(resolve(st->str(), parameter_file), angle);
  } else if (st && st->is_seq()) {
    for (auto &e : st->seq) {
      Receiver r;
      r.network = e->get("network")->str();
      r.station = e->get("station")->str();
      r.x = e->get("x")->num();
      r.z = e->get("z")->num();
      r.angle = e->get("angle") ? e->get("angle")->num() : angle;
      P.receivers.push_back(r);
    }
  }
  if (P.receivers.empty()) throw std::runtime_error("Stations file does not contain any receivers");
  if (const YNode *types = rec->get("seismogram-type")) {
    if (types->is_seq())
      for (auto &t : types->seq) P.seismogram_types.push_back(seismogram_type_of(t->str()));
    else
      P.seismogram_types.push_back(seismogram_type_of(types->str()));
  }
  for (int t : P.seismogram_types)
    if (t == SEIS_ROTATION) throw std::runtime_error("rotation seismograms are not on this path");
  if (const YNode *k = rec->get("nstep_between_samples")) P.nstep_between_samples = k->integer();
  if (P.nstep_between_samples < 1) throw std::runtime_error("nstep_between_samples must be >= 1");
  P.finalize();
  return P;
}
}  // namespace

Problem problem_from_structured(const sfb_structured_desc &d) {
  if (d.ngll != 5 && d.ngll != 8) throw std::invalid_argument("ngll must be 5 or 8");
  if (d.nstep < 1 || d.dt <= 0) throw std::invalid_argument("need nstep >= 1 and dt > 0");
  if (d.nshots < 1) throw std::invalid_argument("nshots must be >= 1");
  StructuredSpec s;
  s.nx = d.nx;
  s.nz = d.nz;
  s.x0 = d.x0;
  s.x1 = d.x1;
  s.z0 = d.z0;
  s.z1 = d.z1;
  for (int k = 0; k < 4; ++k) s.absorb[k] = d.absorb[k] != 0;
  std::vector<Material> mats;
  for (int i = 0; i < d.nmaterials; ++i) {
    Material m;
    m.rho = d.materials[i].rho;
    m.cp = d.materials[i].vp;
    m.cs = d.materials[i].vs;
    m.acoustic = d.materials[i].vs == 0.0;
    mats.push_back(m);
  }
  const int nspec = d.nx * d.nz;
  std::vector<int> em(nspec, 0);
  if (d.element_material)
    for (int e = 0; e < nspec; ++e) {
      em[e] = d.element_material[e];
      if (em[e] < 0 || em[e] >= d.nmaterials) throw std::invalid_argument("element_material out of range");
    }
  Mesh2D mesh = structured_mesh(s, mats, em, d.elastic_sh != 0);
  if (d.gll_rho) {
    const size_t nloc = static_cast<size_t>(nspec) * d.ngll * d.ngll;
    mesh.gll_rho.assign(d.gll_rho, d.gll_rho + nloc);
    mesh.gll_vp.assign(d.gll_vp, d.gll_vp + nloc);
    mesh.gll_vs.assign(d.gll_vs, d.gll_vs + nloc);
    mesh.gll_ngll = d.ngll;
  }
  Problem P;
  P.elastic_sh = d.elastic_sh != 0;
  P.asmb = build_assembly(mesh, d.ngll);
  P.dt = d.dt;
  P.nstep = d.nstep;
  P.nshots = d.nshots;
  P.simulation = d.simulation;
  P.save_boundary_values = d.save_boundary_values != 0;
  P.nstep_between_samples = d.nstep_between_samples > 0 ? d.nstep_between_samples : 1;
  for (int i = 0; i < d.nseismogram_types; ++i) P.seismogram_types.push_back(d.seismogram_types[i]);
  for (int i = 0; i < d.nsources; ++i) {
    const sfb_source_desc &sd = d.sources[i];
    Source s;
    if (sd.kind < Source::FORCE || sd.kind > Source::EXTERNAL) throw std::runtime_error("unknown source kind");
    s.kind = sd.kind;
    s.x = sd.x;
    s.z = sd.z;
    s.angle = sd.angle;
    s.mxx = sd.mxx;
    s.mzz = sd.mzz;
    s.mxz = sd.mxz;
    s.stf = sd.stf;
    s.f0 = sd.f0;
    s.tshift = sd.tshift;
    s.factor = sd.factor;
    s.wavefield = sd.wavefield;
    if (sd.stf == Source::TABLE) {
      if (!sd.stf_table) throw std::invalid_argument("stf table missing");
      s.stf_table.assign(sd.stf_table, sd.stf_table + static_cast<size_t>(d.nstep) * 2);
    }
    if (sd.shot < 0 || sd.shot >= d.nshots) throw std::invalid_argument("source shot out of range");
    P.sources.push_back(s);
    P.source_shot.push_back(sd.shot);
  }
  // Every shot is its own simulation: t0 follows the reference rule per shot
  // unless the caller fixes it.  Shots share one time axis, so the common t0
  // is the earliest over shots and each source keeps its own time shift.
  if (d.t0 != 0.0) {
    P.t0 = d.t0;
  } else {
    double tmin = 0.0;
    bool first = true;
    for (int shot = 0; shot < d.nshots; ++shot) {
      std::vector<Source> ss;
      std::vector<int> idx;
      for (size_t i = 0; i < P.sources.size(); ++i)
        if (P.source_shot[i] == shot && P.sources[i].wavefield == 0) {
          ss.push_back(P.sources[i]);
          idx.push_back(static_cast<int>(i));
        }
      if (ss.empty()) continue;
      const double t = resolve_t0(ss, 0.0);
      for (size_t k = 0; k < idx.size(); ++k) P.sources[idx[k]] = ss[k];
      if (first || t < tmin) tmin = t;
      first = false;
    }
    P.t0 = tmin;
  }
  for (int i = 0; i < d.nreceivers; ++i) {
    Receiver r;
    r.network = d.receivers[i].network ? d.receivers[i].network : "AA";
    r.station = d.receivers[i].station ? d.receivers[i].station : ("S" + std::to_string(i + 1));
    r.x = d.receivers[i].x;
    r.z = d.receivers[i].z;
    r.angle = d.receivers[i].angle;
    P.receivers.push_back(r);
  }
  P.finalize();
  return P;
}

}  // namespace sfb
