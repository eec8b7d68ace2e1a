// C ABI of the SEM time-marching path (include/specfem_b200.h): context life
// cycle, device upload, the reference-granularity entry points and the fused
// CUDA-graph driver.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../../../include/specfem_b200.h"
#include "../host/output_io.hpp"
#include "../host/problem.hpp"
#include "kernels.cuh"

namespace sfb {
void write_seismograms_ascii(const Problem &P, const float *seis, int ntypes, int nrec,
                             int max_sig, const std::string &dir);
}

using namespace sfb;
using dev::real;

namespace {

thread_local std::string g_create_error;

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct StateError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct NonFiniteError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void ck(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

// Copies between host buffers of type H and device values of type `real`
// (FP32 in the product library, FP64 in the verification library): a plain
// copy when the types agree, through a converted host copy otherwise.
template <typename H> void copy_d2h(H *host, const real *dev, size_t n, const char *what) {
  if (!n) return;
  if constexpr (std::is_same<H, real>::value) {
    ck(cudaMemcpy(host, dev, n * sizeof(real), cudaMemcpyDeviceToHost), what);
  } else {
    std::vector<real> tmp(n);
    ck(cudaMemcpy(tmp.data(), dev, n * sizeof(real), cudaMemcpyDeviceToHost), what);
    for (size_t i = 0; i < n; ++i) host[i] = static_cast<H>(tmp[i]);
  }
}
template <typename H> void copy_h2d(real *dev, const H *host, size_t n, const char *what) {
  if (!n) return;
  if constexpr (std::is_same<H, real>::value) {
    ck(cudaMemcpy(dev, host, n * sizeof(real), cudaMemcpyHostToDevice), what);
  } else {
    std::vector<real> tmp(host, host + n);
    ck(cudaMemcpy(dev, tmp.data(), n * sizeof(real), cudaMemcpyHostToDevice), what);
  }
}

template <typename T> struct DBuf {
  T *p = nullptr;
  size_t n = 0;
  void alloc(size_t count, size_t *total) {
    free();
    n = count;
    if (count == 0) return;
    ck(cudaMalloc(&p, count * sizeof(T)), "cudaMalloc");
    // zeroed on the legacy default stream, which the contexts' non-blocking
    // streams do not wait for: finish it before any kernel can read the
    // buffer (reused memory still holds a freed buffer's data)
    ck(cudaMemset(p, 0, count * sizeof(T)), "cudaMemset");
    ck(cudaStreamSynchronize(0), "cudaMemset");
    if (total) *total += count * sizeof(T);
  }
  template <typename U> void upload(const std::vector<U> &h, size_t *total) {
    if constexpr (std::is_same<U, T>::value) {
      alloc(h.size(), total);
      if (!h.empty()) ck(cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
    } else {
      upload(std::vector<T>(h.begin(), h.end()), total);
    }
  }
  void free() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  ~DBuf() { free(); }
};

constexpr int kMedia[3] = {dev::MED_PSV, dev::MED_SH, dev::MED_AC};

struct WavefieldSet {
  bool allocated = false;
  dev::MediumFields f[4];
  DBuf<real> u[4], v[4], a[4];
  DBuf<real> cu[4], cv[4];  // Kahan compensation of u and v (forward, when enabled)
  DBuf<real> seis;
  DBuf<dev::Control> ctrl;
  bool initialized = false;
  int step = 0;  // host copy of the next step index
};

}  // namespace

struct sfb_context {
  Problem P;
  std::string err;
  bool on_device = false;
  int device = 0;
  cudaStream_t stream = nullptr;
  size_t device_bytes = 0;
  // element permutation: device element d holds mesh element perm[d]
  std::vector<int> perm, inv;
  int med_begin[4] = {0, 0, 0, 0}, med_count[4] = {0, 0, 0, 0}, med_interior[4] = {0, 0, 0, 0};
  DBuf<int> iglob;
  DBuf<real> xix, xiz, gax, gaz, jac, mat0[4], mat1[4], mat2[4];
  DBuf<real> mat0_all, mat1_all, mat2_all;
  DBuf<uint8_t> eflag, bnd;
  DBuf<real> bnd_nx, bnd_nz, bnd_w;
  DBuf<real> pack;  // [nspec][8][N*N] static block of the stiffness kernels
  DBuf<float> pack_aff;  // compact block of affine elements (single-shot FP32 contexts)
  DBuf<int> dflag;   // device error word (dev::kErrWaitTimeout | dev::kErrNonFinite)
  int *h_err = nullptr;  // pinned host copy of it, refreshed asynchronously after entry points
  DBuf<real> minv[4];
  DBuf<double> mass[4];
  // sources (forward / backward wavefield) and receivers
  DBuf<int> src_elem, src_shot, src_medium;
  DBuf<real> src_array, src_stf;
  int nsrc = 0;
  DBuf<int> rec_elem;
  DBuf<real> rec_lag, rec_sin, rec_cos;
  DBuf<int> cp_ac_self, cp_ac_other, cp_el_self, cp_el_other;
  DBuf<real> cp_ac_f, cp_ac_nx, cp_ac_nz, cp_el_f, cp_el_nx, cp_el_nz;
  DBuf<int> step_scratch;  // host-driven step index for the unfused path
  WavefieldSet wf[3];
  dev::Static st{};
  bool mass_ready = false;
  // Stacey replay store
  DBuf<real> stacey_data;  // [S][nstep][nstacey][N*N][2]
  DBuf<int> stacey_slot;
  std::vector<int> h_stacey_slot;  // host copy, per device element
  int nstacey = 0;
  // adjoint sources: one per (shot, receiver), receiver Lagrange arrays
  DBuf<int> adj_elem, adj_shot, adj_medium;
  DBuf<real> adj_array, adj_stf;
  int nadj = 0;
  DBuf<double> kern;        // Frechet accumulators [nspec][N*N][3], device element order
  // Stacey-traction model derivatives [nspec][N*N][2] (sfb_set_stacey_kernels)
  bool stacey_kernels = false;
  DBuf<double> kern_b;
  std::map<int, cudaGraphExec_t> graphs_combined;  // combined-run graphs by step count
  std::vector<float> host_seis;
  // seismogram taps per medium (fused path)
  struct Taps {
    DBuf<uint32_t> mask;
    DBuf<int> sup_g, sup_begin, slot, which;
    DBuf<real> w;
    int nsup = 0;
  } taps[4];
  bool taps_ready = false;
  DBuf<unsigned> done;  // CTA completion counter of the update kernel
  // P-SV points updated inside the stiffness launch of the forward run are
  // numbered last; the update kernel then walks [0, nshared_points)
  int nshared_points = 0, nprivate_points = 0;
  // batched stiffness kernel per medium (dev::kShots*), chosen by
  // autotune_stiffness or set by the caller
  int shots_variant[4] = {0, 0, 0, 0};
  bool tuned = false;
  bool compensated = false;  // Kahan-compensated Newmark sums in the fused forward
  // forward snapshots restored into the backward wavefield of the combined
  // run every ck_interval steps (0: pure reconstruction)
  int ck_interval = 0, ck_count = 0;
  DBuf<real> ck_u[4], ck_v[4];
  size_t ck_stride[4] = {0, 0, 0, 0};
  // forward CUDA graphs by the number of fused steps they hold (the full
  // chunk and the remainders met so far)
  std::map<int, cudaGraphExec_t> graphs;
  uint64_t launches = 0;  // kernels launched so far (graph replays included)
  // Deterministic assembly (sfb_set_deterministic): each medium's elements
  // are coloured so that no two elements of a colour share a point, one
  // stiffness launch per colour (device elements [col_begin, +col_count)),
  // sources and coupling through owner-computes maps, seismograms from the
  // receiver kernel: the same inputs give the same bits on every run.
  bool deterministic = false;
  int ncolor[4] = {0, 0, 0, 0};
  std::vector<int> col_begin[4], col_count[4];
  struct DetTailBuf {
    DBuf<int> g, begin, ent;
    int n = 0;
    bool ready = false;
  } det_tail[2][4];  // [forward sources / adjoint sources][medium]
  std::vector<int> h_adj_elem, h_adj_medium;  // adjoint sources: device element, medium

  void drop_forward_graphs() {
    for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
    graphs.clear();
  }
  void drop_combined_graphs() {
    for (auto &kv : graphs_combined) cudaGraphExecDestroy(kv.second);
    graphs_combined.clear();
  }
  ~sfb_context() {
    if (h_err) cudaFreeHost(h_err);
    drop_forward_graphs();
    drop_combined_graphs();
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

int fail(sfb_context *ctx, int code, const std::string &msg) {
  if (ctx) ctx->err = msg;
  else g_create_error = msg;
  return code;
}

template <typename F> int guarded(sfb_context *ctx, F &&fn) {
  try {
    return fn();
  } catch (const CudaError &e) {
    return fail(ctx, SFB_E_CUDA, e.what());
  } catch (const StateError &e) {
    return fail(ctx, SFB_E_STATE, e.what());
  } catch (const NonFiniteError &e) {
    return fail(ctx, SFB_E_NONFINITE, e.what());
  } catch (const std::invalid_argument &e) {
    return fail(ctx, SFB_E_INVALID, e.what());
  } catch (const std::bad_alloc &e) {
    return fail(ctx, SFB_E_NOMEM, e.what());
  } catch (const std::exception &e) {
    const std::string m = e.what();
    const bool io = m.find("open") != std::string::npos || m.find("database") != std::string::npos ||
                    m.find("YAML") != std::string::npos;
    return fail(ctx, io ? SFB_E_IO : SFB_E_INVALID, m);
  }
}

int medium_index_ok(int m) { return m == 0 || m == 1 || m == 3; }

// New contexts use the deterministic assembly when the environment sets
// SFB_DETERMINISTIC=1 (file-driven runs, sfb_execute); sfb_set_deterministic
// chooses per context.
bool deterministic_default() {
  const char *e = std::getenv("SFB_DETERMINISTIC");
  return e && e[0] == '1';
}

// Greedy colouring of each medium's elements in mesh order: an element takes
// the smallest colour none of the elements sharing one of its points has
// (four colours on a structured quad mesh).
std::vector<int> element_colours(const Assembly &a) {
  const int nspec = a.nspec, nn = a.ngll * a.ngll;
  std::vector<int> colour(nspec, -1);
  for (int m : kMedia) {
    const int np = a.nglob[m];
    if (np == 0) continue;
    std::vector<int> start(static_cast<size_t>(np) + 1, 0);
    for (int e = 0; e < nspec; ++e)
      if (a.medium[e] == m)
        for (int k = 0; k < nn; ++k) ++start[a.iglob[static_cast<size_t>(e) * nn + k] + 1];
    for (int g = 0; g < np; ++g) start[g + 1] += start[g];
    std::vector<int> fill(start.begin(), start.end() - 1), elems(start[np]);
    for (int e = 0; e < nspec; ++e)
      if (a.medium[e] == m)
        for (int k = 0; k < nn; ++k) elems[fill[a.iglob[static_cast<size_t>(e) * nn + k]]++] = e;
    for (int e = 0; e < nspec; ++e) {
      if (a.medium[e] != m) continue;
      uint64_t used = 0;
      for (int k = 0; k < nn; ++k) {
        const int g = a.iglob[static_cast<size_t>(e) * nn + k];
        for (int q = start[g]; q < start[g + 1]; ++q)
          if (colour[elems[q]] >= 0) used |= uint64_t(1) << colour[elems[q]];
      }
      int col = 0;
      while (col < 64 && ((used >> col) & 1)) ++col;
      if (col == 64) throw std::runtime_error("element colouring needs more than 64 colours");
      colour[e] = col;
    }
  }
  return colour;
}

void build_permutation(sfb_context *c) {
  const Assembly &a = c->P.asmb;
  const int nspec = a.nspec, nn = a.ngll * a.ngll;
  std::vector<int> has_b(nspec, 0);
  for (int e = 0; e < nspec; ++e)
    for (int k = 0; k < nn; ++k)
      if (a.bnd[static_cast<size_t>(e) * nn + k]) has_b[e] = 1;
  // deterministic mode: colour ranges inside each medium
  std::vector<int> colour(nspec, 0);
  if (c->deterministic) colour = element_colours(a);
  c->perm.resize(nspec);
  for (int e = 0; e < nspec; ++e) c->perm[e] = e;
  auto rank = [](int m) { return m == 0 ? 0 : m == 1 ? 1 : 2; };
  std::stable_sort(c->perm.begin(), c->perm.end(), [&](int x, int y) {
    if (rank(a.medium[x]) != rank(a.medium[y])) return rank(a.medium[x]) < rank(a.medium[y]);
    if (colour[x] != colour[y]) return colour[x] < colour[y];
    return has_b[x] < has_b[y];
  });
  for (int m : kMedia) {
    c->ncolor[m] = 0;
    c->col_begin[m].clear();
    c->col_count[m].clear();
  }
  for (int d = 0; d < nspec; ++d) {
    const int e = c->perm[d], m = a.medium[e];
    if (colour[e] >= c->ncolor[m]) {
      c->ncolor[m] = colour[e] + 1;
      c->col_begin[m].resize(c->ncolor[m], d);
      c->col_count[m].resize(c->ncolor[m], 0);
    }
    ++c->col_count[m][colour[e]];
  }
  c->inv.assign(nspec, 0);
  for (int d = 0; d < nspec; ++d) c->inv[c->perm[d]] = d;
  for (int m : kMedia) {
    c->med_begin[m] = 0;
    c->med_count[m] = 0;
    c->med_interior[m] = 0;
  }
  for (int d = nspec - 1; d >= 0; --d) c->med_begin[a.medium[c->perm[d]]] = d;
  for (int d = 0; d < nspec; ++d) {
    const int m = a.medium[c->perm[d]];
    c->med_count[m]++;
    if (!has_b[c->perm[d]]) c->med_interior[m]++;
  }
}

void ensure_device(sfb_context *c) {
  if (c->on_device) return;
  int ndev = 0;
  const cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    throw CudaError(std::string("no CUDA device available: ") + cudaGetErrorString(e));
  ck(cudaGetDevice(&c->device), "cudaGetDevice");
  ck(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
  const Assembly &a = c->P.asmb;
  const int n = a.ngll, nn = n * n;
  const size_t nloc = a.nloc();
  build_permutation(c);
  // permuted static arrays
  std::vector<int> iglob(nloc);
  std::vector<float> xix(nloc), xiz(nloc), gax(nloc), gaz(nloc), jac(nloc), m0(nloc), m1(nloc),
      m2(nloc), bnx(nloc), bnz(nloc), bw(nloc);
  std::vector<uint8_t> bnd(nloc), eflag(a.nspec, 0);
  for (int d = 0; d < a.nspec; ++d) {
    const int e = c->perm[d];
    const int m = a.medium[e];
    for (int k = 0; k < nn; ++k) {
      const size_t p = static_cast<size_t>(e) * nn + k, q = static_cast<size_t>(d) * nn + k;
      iglob[q] = a.iglob[p];
      xix[q] = a.xix[p];
      xiz[q] = a.xiz[p];
      gax[q] = a.gammax[p];
      gaz[q] = a.gammaz[p];
      jac[q] = a.jacobian[p];
      if (m == MEDIUM_ELASTIC_PSV) {
        m0[q] = a.kappa[p];
        m1[q] = a.mu[p];
        m2[q] = a.rho[p];
      } else if (m == MEDIUM_ELASTIC_SH) {
        m0[q] = a.mu[p];
        m1[q] = a.rho[p];
        m2[q] = 0.f;
      } else {
        m0[q] = a.rho_inverse[p];
        m1[q] = a.kappa[p];
        m2[q] = 0.f;
      }
      bnd[q] = a.bnd[p];
      bnx[q] = a.bnd_nx[p];
      bnz[q] = a.bnd_nz[p];
      bw[q] = a.bnd_w[p];
      eflag[d] |= a.bnd[p];
    }
  }
  // Element-private points (Problem::elem_private): the P-SV field is
  // numbered shared points first, so the update kernel can stop at
  // nshared_points when the stiffness launch has updated the rest.
  {
    const int m = MEDIUM_ELASTIC_PSV;
    const Problem &P0 = c->P;
    for (int d = c->med_begin[m]; d < c->med_begin[m] + c->med_count[m]; ++d)
      if (!P0.elem_private.empty() && P0.elem_private[c->perm[d]]) eflag[d] |= dev::kElemPrivate;
    c->nshared_points = P0.nshared_psv;
    c->nprivate_points = a.nglob[m] - P0.nshared_psv;
  }
  // packed per-element static block: iglob, xix, xiz, gammax, gammaz, jac, mat0, mat1
  std::vector<real> pack(nloc * dev::kPackFields);
  for (int d = 0; d < a.nspec; ++d)
    for (int k = 0; k < nn; ++k) {
      const size_t q = static_cast<size_t>(d) * nn + k;
      real *blk = &pack[static_cast<size_t>(d) * dev::kPackFields * nn];
      const int gi = iglob[q];
#ifdef SFB_FP64
      blk[0 * nn + k] = static_cast<real>(gi);  // the index as a value (exact below 2^53)
#else
      std::memcpy(&blk[0 * nn + k], &gi, 4);  // the index's bits
#endif
      blk[1 * nn + k] = xix[q];
      blk[2 * nn + k] = xiz[q];
      blk[3 * nn + k] = gax[q];
      blk[4 * nn + k] = gaz[q];
      blk[5 * nn + k] = jac[q];
      blk[6 * nn + k] = m0[q];
      blk[7 * nn + k] = m1[q];
    }
  size_t *tot = &c->device_bytes;
  c->pack.upload(pack, tot);
  // Compact block for media whose elements are all affine (the Jacobian
  // matrix and determinant constant over the element to 4e-7 relative, i.e.
  // equal up to rounding): the single-shot compact-block kernel then streams
  // the per-point index and material and five constants per element instead
  // of five geometry words per point; the batched kernels keep the five
  // constants in registers instead of staging geometry per point.  Chunks of
  // dev::kAffineChunk elements per medium, chunk-major (see
  // dev::Static::pack_aff).  FP32 contexts only: the compact-block kernels
  // are FP32 kernels.  The deterministic mode launches colour ranges, which
  // the chunked compact block does not follow: it reads the full block.
#ifndef SFB_FP64
  if (!c->deterministic) {
    const int words = dev::affine_chunk_words(n);
    const int E = dev::kAffineChunk;
    std::vector<float> aff;
    int chunks = 0;
    for (int m : kMedia) {
      if (c->med_count[m] == 0) continue;
      bool all = true;
      for (int d = c->med_begin[m]; all && d < c->med_begin[m] + c->med_count[m]; ++d) {
        const size_t q0 = static_cast<size_t>(d) * nn;
        const double scale = std::max(std::max(std::fabs(xix[q0]), std::fabs(xiz[q0])),
                                      std::max(std::fabs(gax[q0]), std::fabs(gaz[q0])));
        for (int k = 1; all && k < nn; ++k) {
          const size_t q = q0 + k;
          all = std::fabs(xix[q] - xix[q0]) <= 4e-7 * scale && std::fabs(xiz[q] - xiz[q0]) <= 4e-7 * scale &&
                std::fabs(gax[q] - gax[q0]) <= 4e-7 * scale && std::fabs(gaz[q] - gaz[q0]) <= 4e-7 * scale &&
                std::fabs(jac[q] - jac[q0]) <= 4e-7 * std::fabs(jac[q0]);
        }
      }
      if (!all) continue;
      const int mchunks = (c->med_count[m] + E - 1) / E;
      c->st.affine[m] = 1;
      c->st.aff_chunk0[m] = chunks;
      aff.resize(static_cast<size_t>(chunks + mchunks) * words, 0.f);
      for (int i = 0; i < c->med_count[m]; ++i) {
        const int d = c->med_begin[m] + i;
        float *chunk = &aff[static_cast<size_t>(chunks + i / E) * words];
        const int el = i % E;
        const size_t q0 = static_cast<size_t>(d) * nn;
        double mean[5] = {0, 0, 0, 0, 0};
        for (int k = 0; k < nn; ++k) {
          const size_t q = q0 + k;
          int gi = iglob[q];
          std::memcpy(&chunk[el * nn + k], &gi, 4);
          chunk[E * nn + el * nn + k] = m0[q];
          chunk[2 * E * nn + el * nn + k] = m1[q];
          mean[0] += xix[q];
          mean[1] += xiz[q];
          mean[2] += gax[q];
          mean[3] += gaz[q];
          mean[4] += jac[q];
        }
        for (int j = 0; j < 5; ++j) chunk[3 * E * nn + j * E + el] = static_cast<float>(mean[j] / nn);
      }
      chunks += mchunks;
    }
    if (!aff.empty()) c->pack_aff.upload(aff, tot);
  }
#endif
  c->dflag.alloc(1, tot);
  ck(cudaHostAlloc(reinterpret_cast<void **>(&c->h_err), sizeof(int), cudaHostAllocDefault), "cudaHostAlloc");
  *c->h_err = 0;
  c->iglob.upload(iglob, tot);
  c->xix.upload(xix, tot);
  c->xiz.upload(xiz, tot);
  c->gax.upload(gax, tot);
  c->gaz.upload(gaz, tot);
  c->jac.upload(jac, tot);
  c->mat0_all.upload(m0, tot);
  c->mat1_all.upload(m1, tot);
  c->mat2_all.upload(m2, tot);
  c->bnd.upload(bnd, tot);
  c->eflag.upload(eflag, tot);
  c->bnd_nx.upload(bnx, tot);
  c->bnd_nz.upload(bnz, tot);
  c->bnd_w.upload(bw, tot);
  c->st.ngll = n;
  c->st.nspec = a.nspec;
  c->st.iglob = c->iglob.p;
  c->st.xix = c->xix.p;
  c->st.xiz = c->xiz.p;
  c->st.gax = c->gax.p;
  c->st.gaz = c->gaz.p;
  c->st.jac = c->jac.p;
  c->st.mat0 = c->mat0_all.p;
  c->st.mat1 = c->mat1_all.p;
  c->st.mat2 = c->mat2_all.p;
  c->st.eflag = c->eflag.p;
  c->st.bnd = c->bnd.p;
  c->st.bnd_nx = c->bnd_nx.p;
  c->st.bnd_nz = c->bnd_nz.p;
  c->st.bnd_w = c->bnd_w.p;
  c->st.pack = c->pack.p;
  c->st.pack_aff = c->pack_aff.p;
  c->st.err = c->dflag.p;
  for (int m : kMedia) {
    const size_t ld = static_cast<size_t>(a.nglob[m] + (a.nglob[m] & 1)) * a.ncomp(m);
    c->minv[m].alloc(ld, tot);
    c->mass[m].alloc(ld, tot);
  }
  // quadrature tables
  std::vector<real> hp(nn), w(n);
  for (int i = 0; i < nn; ++i) hp[i] = static_cast<real>(static_cast<float>(a.quad.hprime[i]));
  for (int i = 0; i < n; ++i) w[i] = static_cast<real>(static_cast<float>(a.quad.w[i]));
  dev::set_quadrature(n, hp.data(), w.data());
  ck(cudaGetLastError(), "set_quadrature");
  dev::init_kernel_attributes();
  ck(cudaGetLastError(), "kernel attributes");
  // sources (element ids translated to device order)
  const Problem &P = c->P;
  c->nsrc = static_cast<int>(P.v_src_ispec.size());
  {
    std::vector<int> el(c->nsrc), sh(c->nsrc), md(c->nsrc);
    for (int i = 0; i < c->nsrc; ++i) {
      el[i] = c->inv[P.v_src_ispec[i]];
      sh[i] = P.v_src_shot[i];
      md[i] = a.medium[P.v_src_ispec[i]];
    }
    c->src_elem.upload(el, tot);
    c->src_shot.upload(sh, tot);
    c->src_medium.upload(md, tot);
    c->src_array.upload(P.v_src_array, tot);
    c->src_stf.upload(P.v_src_stf, tot);
  }
  {
    std::vector<int> el(P.v_rec_ispec.size());
    for (size_t i = 0; i < el.size(); ++i) el[i] = c->inv[P.v_rec_ispec[i]];
    c->rec_elem.upload(el, tot);
    c->rec_lag.upload(P.v_rec_lagrange, tot);
    c->rec_sin.upload(P.v_rec_sin, tot);
    c->rec_cos.upload(P.v_rec_cos, tot);
  }
  c->cp_ac_self.upload(P.v_cp_ac_self, tot);
  c->cp_ac_other.upload(P.v_cp_ac_other, tot);
  c->cp_ac_f.upload(P.v_cp_ac_f, tot);
  c->cp_ac_nx.upload(P.v_cp_ac_nx, tot);
  c->cp_ac_nz.upload(P.v_cp_ac_nz, tot);
  c->cp_el_self.upload(P.v_cp_el_self, tot);
  c->cp_el_other.upload(P.v_cp_el_other, tot);
  c->cp_el_f.upload(P.v_cp_el_f, tot);
  c->cp_el_nx.upload(P.v_cp_el_nx, tot);
  c->cp_el_nz.upload(P.v_cp_el_nz, tot);
  c->step_scratch.alloc(4, tot);
  // Stacey replay slots: one per device element whose boundary tag is
  // stacey -- Stacey points and no acoustic free-surface point; composite
  // Stacey / Dirichlet elements are computed in the backward run, not
  // replayed (compute_stiffness_interaction.tpp:123-137 replays the stacey
  // tag only; enumerations/boundary.hpp:50-105 combines the tags)
  {
    std::vector<int> slot(a.nspec, -1);
    c->nstacey = 0;
    for (int d = 0; d < a.nspec; ++d)
      if ((eflag[d] & 3) == 1) slot[d] = c->nstacey++;
    c->stacey_slot.upload(slot, tot);
    c->h_stacey_slot = slot;
  }
  c->on_device = true;
}

// Stiffness autotuner: with the freshly allocated (all zero)
// forward fields, time every applicable kernel variant of each medium (one
// warm-up and three timed launches, no sources, coupling or store) and keep
// the fastest.  The launches add zero forces; the force arrays are cleared
// afterwards all the same.
void autotune_stiffness(sfb_context *c, WavefieldSet &W) {
  const Problem &P = c->P;
  const int S = P.nshots, n = P.asmb.ngll;
  if (c->tuned) return;
  c->tuned = true;
  cudaEvent_t e0, e1;
  ck(cudaEventCreate(&e0), "event");
  ck(cudaEventCreate(&e1), "event");
  const dev::StaceyStore none{};
  for (int m : kMedia) {
    // a pinned compact-block variant on a medium that is not all affine
    // runs (and reports) the full block of the same chunk size
    if (S == 1 && (!c->st.affine[m] || n != 5))
      c->shots_variant[m] = dev::row_variant_without_affine(c->shots_variant[m]);
    if (c->shots_variant[m] != dev::kShotsAuto || W.f[m].nelem == 0) continue;
    int cand[3], nc = 0;
    if (S == 1) {
      cand[nc++] = dev::kRowFullChunk;
      if (n == 5) cand[nc++] = dev::kRowHalfChunk;
      if (n == 5 && c->st.affine[m] && c->st.pack_aff) cand[nc++] = dev::kRowAffine;
    } else {
      if (S % 2 == 0 && n <= 5) {
        cand[nc++] = dev::kShotsPacked;
        cand[nc++] = dev::kShotsPair;
      }
      cand[nc++] = dev::kShotsSingle;
    }
    float best = 0.f;
    int choice = cand[0];
    for (int i = 0; i < nc && nc > 1; ++i) {
      dev::launch_stiffness(m, n, c->st, W.f[m], S, none, &W.ctrl.p->istep, c->stream, nullptr, nullptr, cand[i]);
      ck(cudaEventRecord(e0, c->stream), "event record");
      for (int r = 0; r < 3; ++r)
        dev::launch_stiffness(m, n, c->st, W.f[m], S, none, &W.ctrl.p->istep, c->stream, nullptr, nullptr, cand[i]);
      ck(cudaEventRecord(e1, c->stream), "event record");
      ck(cudaEventSynchronize(e1), "event sync");
      float ms = 0.f;
      ck(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
      c->launches += 4;
      if (i == 0 || ms < best) {
        best = ms;
        choice = cand[i];
      }
    }
    c->shots_variant[m] = choice;
    const dev::MediumFields &f = W.f[m];
    const size_t ld = static_cast<size_t>(f.nglob + (f.nglob & 1)) * f.nc * S;
    ck(cudaMemsetAsync(f.a, 0, ld * sizeof(real), c->stream), "clear force");
  }
  ck(cudaGetLastError(), "autotune");
  ck(cudaStreamSynchronize(c->stream), "autotune");
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
}

WavefieldSet &ensure_wavefield(sfb_context *c, int w) {
  ensure_device(c);
  WavefieldSet &W = c->wf[w];
  if (W.allocated) return W;
  const Assembly &a = c->P.asmb;
  size_t *tot = &c->device_bytes;
  const int S = c->P.nshots;
  for (int m : kMedia) {
    const size_t ld = static_cast<size_t>(a.nglob[m] + (a.nglob[m] & 1)) * a.ncomp(m);
    W.u[m].alloc(ld * S, tot);
    W.v[m].alloc(ld * S, tot);
    W.a[m].alloc(ld * S, tot);
    dev::MediumFields &f = W.f[m];
    f.nglob = a.nglob[m];
    f.nc = a.ncomp(m);
    f.elem_begin = c->med_begin[m];
    f.nelem = c->med_count[m];
    f.nelem_interior = c->med_interior[m];
    f.u = W.u[m].p;
    f.v = W.v[m].p;
    f.a = W.a[m].p;
    f.minv = c->minv[m].p;
    f.mass = c->mass[m].p;
  }
  const Problem &P = c->P;
  const size_t nseis = static_cast<size_t>(S) * P.max_sig_step() * P.seismogram_types.size() *
                       P.receivers.size() * 2;
  W.seis.alloc(std::max<size_t>(nseis, 1), tot);
  W.ctrl.alloc(1, tot);
  W.allocated = true;
  if (w == SFB_WAVEFIELD_FORWARD) autotune_stiffness(c, W);
  return W;
}

dev::SourceSet source_set(sfb_context *c) {
  dev::SourceSet s{};
  s.n = c->nsrc;
  s.elem = c->src_elem.p;
  s.shot = c->src_shot.p;
  s.medium = c->src_medium.p;
  s.array = c->src_array.p;
  s.stf = c->src_stf.p;
  s.nstep = c->P.nstep;
  return s;
}

dev::ReceiverSet receiver_set(sfb_context *c, WavefieldSet &W) {
  dev::ReceiverSet r{};
  const Problem &P = c->P;
  r.n = static_cast<int>(P.receivers.size());
  r.elem = c->rec_elem.p;
  r.lagrange = c->rec_lag.p;
  r.sinv = c->rec_sin.p;
  r.cosv = c->rec_cos.p;
  r.ntypes = static_cast<int>(P.seismogram_types.size());
  for (int i = 0; i < r.ntypes && i < 5; ++i) r.types[i] = P.seismogram_types[i];
  r.max_sig = P.max_sig_step();
  r.nsbs = P.nstep_between_samples;
  r.seis = W.seis.p;
  return r;
}

dev::CouplingSet coupling_acoustic(sfb_context *c) {
  return {static_cast<int>(c->P.v_cp_ac_self.size()), c->cp_ac_self.p, c->cp_ac_other.p,
          c->cp_ac_f.p, c->cp_ac_nx.p, c->cp_ac_nz.p};
}
dev::CouplingSet coupling_elastic(sfb_context *c) {
  return {static_cast<int>(c->P.v_cp_el_self.size()), c->cp_el_self.p, c->cp_el_other.p,
          c->cp_el_f.p, c->cp_el_nx.p, c->cp_el_nz.p};
}

void initialize_mass(sfb_context *c, double dt) {
  ensure_device(c);
  const Assembly &a = c->P.asmb;
  for (int m : kMedia) {
    dev::MediumFields f{};
    f.nglob = a.nglob[m];
    f.nc = a.ncomp(m);
    f.elem_begin = c->med_begin[m];
    f.nelem = c->med_count[m];
    f.minv = c->minv[m].p;
    f.mass = c->mass[m].p;
    if (c->mass[m].n) ck(cudaMemsetAsync(c->mass[m].p, 0, c->mass[m].n * sizeof(double), c->stream), "memset mass");
    if (c->deterministic) {
      // one launch per element colour: a fixed order of the FP64 sums
      for (int k = 0; k < c->ncolor[m]; ++k) {
        dev::MediumFields fk = f;
        fk.elem_begin = c->col_begin[m][k];
        fk.nelem = c->col_count[m][k];
        dev::launch_mass(m, a.ngll, c->st, fk, static_cast<real>(dt), c->stream);
      }
    } else {
      dev::launch_mass(m, a.ngll, c->st, f, static_cast<real>(dt), c->stream);
    }
    dev::launch_invert_mass(f, c->stream);
  }
  ck(cudaGetLastError(), "mass kernels");
  c->mass_ready = true;
}

void set_step(sfb_context *c, WavefieldSet &W, int istep) {
  dev::Control h{istep};
  ck(cudaMemcpyAsync(W.ctrl.p, &h, sizeof(h), cudaMemcpyHostToDevice, c->stream), "set step");
  W.step = istep;
}


// Seismograms of the fused path as a sparse linear map of nodal values:
// for every receiver, seismogram type and output component, the weights of
// the element's nodal (field, component) values.  They fold the Lagrange
// interpolant, the gradient operator and material of the pressure /
// acoustic-displacement transforms (include/medium/dim2/*/isotropic/
// wavefield.hpp) and the receiver rotation (receivers.hpp:126-141).
void build_taps(sfb_context *c) {
  if (c->taps_ready) return;
  const Problem &P = c->P;
  const Assembly &a = P.asmb;
  const int n = a.ngll, nn = n * n;
  const int nrec = static_cast<int>(P.receivers.size());
  const int ntypes = static_cast<int>(P.seismogram_types.size());
  struct E { int g, slot, which; double w; };
  std::vector<E> ent[4];
  // the derivative table as the kernels and the reference hold it (FP32)
  auto hp32 = [&](int i) { return static_cast<double>(static_cast<float>(a.quad.hprime[i])); };
  for (int r = 0; r < nrec; ++r) {
    const LocatedReceiver &L = P.located_receivers[r];
    const int e = L.ispec, m = a.medium[e];
    const double cs = L.cos_angle, sn = L.sin_angle;
    for (int it = 0; it < ntypes; ++it) {
      const int type = P.seismogram_types[it];
      std::vector<double> W(static_cast<size_t>(nn) * 4, 0.0);  // [q][ic][oc]
      auto add = [&](int q, int ic, double v0, double v1) {
        W[(q * 2 + ic) * 2 + 0] += cs * v0 - sn * v1;
        W[(q * 2 + ic) * 2 + 1] += sn * v0 + cs * v1;
      };
      int which = type;
      for (int k = 0; k < nn; ++k) {
        const double h = L.lagrange[k];
        const size_t p = static_cast<size_t>(e) * nn + k;
        const int kz = k / n, kx = k % n;
        if (m != MEDIUM_ACOUSTIC && type <= 2) {
          add(k, 0, h, 0.0);  // wavefield = (u0, u1): out = R (sum h u0, sum h u1)
          if (m == MEDIUM_ELASTIC_PSV) add(k, 1, 0.0, h);
        } else if (m == MEDIUM_ELASTIC_PSV && type == 3) {
          which = 0;
          // 4/3 as the reference's FP32 constant
          const double l2m = a.kappa[p] + static_cast<double>(static_cast<float>(4.0 / 3.0)) * a.mu[p];
          const double cf = -((l2m - 2.0 * a.mu[p]) + (2.0 / 3.0) * a.mu[p]) * h;
          for (int l = 0; l < n; ++l) {
            const double hx = hp32(kx * n + l), hz = hp32(kz * n + l);
            add(kz * n + l, 0, cf * a.xix[p] * hx, 0.0);
            add(l * n + kx, 0, cf * a.gammax[p] * hz, 0.0);
            add(kz * n + l, 1, cf * a.xiz[p] * hx, 0.0);
            add(l * n + kx, 1, cf * a.gammaz[p] * hz, 0.0);
          }
        } else if (m == MEDIUM_ACOUSTIC && type == 3) {
          which = 2;
          add(k, 0, -h, 0.0);
        } else if (m == MEDIUM_ACOUSTIC) {
          const double ri = a.rho_inverse[p];
          for (int l = 0; l < n; ++l) {
            const double hx = hp32(kx * n + l), hz = hp32(kz * n + l);
            add(kz * n + l, 0, h * ri * a.xix[p] * hx, h * ri * a.xiz[p] * hx);
            add(l * n + kx, 0, h * ri * a.gammax[p] * hz, h * ri * a.gammaz[p] * hz);
          }
        }
      }
      const int nc = a.ncomp(m);
      for (int q = 0; q < nn; ++q)
        for (int ic = 0; ic < nc; ++ic)
          for (int oc = 0; oc < 2; ++oc) {
            const double w = W[(q * 2 + ic) * 2 + oc];
            if (w == 0.0) continue;
            ent[m].push_back({a.iglob[static_cast<size_t>(e) * nn + q], (it * nrec + r) * 2 + oc, which * 2 + ic, w});
          }
    }
  }
  size_t *tot = &c->device_bytes;
  for (int m : kMedia) {
    auto &T = c->taps[m];
    auto &v = ent[m];
    std::sort(v.begin(), v.end(), [](const E &x, const E &y) { return x.g < y.g; });
    std::vector<int> sup_g, sup_begin, slot, which;
    std::vector<real> w;
    for (size_t i = 0; i < v.size(); ++i) {
      if (sup_g.empty() || sup_g.back() != v[i].g) {
        sup_g.push_back(v[i].g);
        sup_begin.push_back(static_cast<int>(slot.size()));
      }
      slot.push_back(v[i].slot);
      which.push_back(v[i].which);
      w.push_back(static_cast<real>(v[i].w));
    }
    sup_begin.push_back(static_cast<int>(slot.size()));
    const int nglob = a.nglob[m];
    std::vector<uint32_t> mask((nglob + 2 + 31) / 32, 0u);
    for (int g : sup_g) mask[g >> 5] |= 1u << (g & 31);
    T.nsup = static_cast<int>(sup_g.size());
    T.mask.upload(mask, tot);
    T.sup_g.upload(sup_g, tot);
    T.sup_begin.upload(sup_begin, tot);
    T.slot.upload(slot, tot);
    T.which.upload(which, tot);
    T.w.upload(w, tot);
  }
  c->done.alloc(1, tot);
  c->taps_ready = true;
}

dev::UpdateParams update_params(sfb_context *c, WavefieldSet &W, int last, bool advance, bool taps,
                                bool private_done = false, bool snapshots = false) {
  const Problem &P = c->P;
  dev::UpdateParams u{};
  u.nm = 0;
  u.begin[0] = 0;
  for (int m : kMedia) {
    const dev::MediumFields &f = W.f[m];
    if (f.nglob == 0) continue;
    dev::UpdateMedium &M = u.m[u.nm];
    M.u = f.u;
    M.v = f.v;
    M.a = f.a;
    M.minv = f.minv;
    M.ld2 = static_cast<size_t>(f.nglob + (f.nglob & 1)) * f.nc * P.nshots / 2;
    M.nc = f.nc;
    M.cu = W.cu[m].p;
    M.cv = W.cv[m].p;
    if (snapshots && c->ck_count > 0) {
      M.ck_u = c->ck_u[m].p;
      M.ck_v = c->ck_v[m].p;
      M.ck_stride = c->ck_stride[m];
    }
    if (private_done && m == MEDIUM_ELASTIC_PSV && c->nprivate_points > 0)
      M.ld2 = static_cast<size_t>(c->nshared_points) * P.nshots;  // shared points only, a float2 pair each
    if (taps && c->taps[m].nsup > 0) {
      const auto &T = c->taps[m];
      M.taps = {T.nsup, T.mask.p, T.sup_g.p, T.sup_begin.p, T.slot.p, T.which.p, T.w.p};
    }
    u.begin[u.nm + 1] = u.begin[u.nm] + M.ld2;
    ++u.nm;
  }
  u.nshots = P.nshots;
  u.sdiv = dev::FastDiv::make(static_cast<uint32_t>(P.nshots));
  if (u.begin[u.nm] * 2 >= (1ull << 32)) throw std::invalid_argument("field too large for 32-bit update indexing");
  u.dt = static_cast<real>(P.dt);
  u.dt2 = static_cast<real>(P.dt / 2.0);
  u.dtsq2 = static_cast<real>(P.dt * P.dt / 2.0);
  u.last = last;
  u.ctrl = advance ? W.ctrl.p : nullptr;
  u.dir = 1;
  u.done = c->done.p;
  u.seis = taps ? W.seis.p : nullptr;
  u.slots = static_cast<int>(P.seismogram_types.size() * P.receivers.size() * 2);
  u.max_sig = P.max_sig_step();
  u.nsbs = P.nstep_between_samples;
  u.nstep = P.nstep;
  if (snapshots && c->ck_count > 0) {
    u.ck_interval = c->ck_interval;
    u.ck_count = c->ck_count;
  }
  return u;
}

// The owner-computes map of the sources (kind 0: the forward sources, kind 1:
// the adjoint sources) and coupling points that medium m receives (see
// dev::DetTail); built once per context.
const dev::DetTail det_tail(sfb_context *c, int kind, int m) {
  auto &T = c->det_tail[kind][m];
  if (!T.ready) {
    const Problem &P = c->P;
    const Assembly &a = P.asmb;
    const int nn = a.ngll * a.ngll;
    std::vector<std::pair<int, int>> pairs;  // (target point, entry)
    if (kind == 0) {
      for (size_t i = 0; i < P.v_src_ispec.size(); ++i) {
        const int e = P.v_src_ispec[i];
        if (a.medium[e] != m) continue;
        for (int k = 0; k < nn; ++k)
          pairs.push_back({a.iglob[static_cast<size_t>(e) * nn + k], static_cast<int>(i) * nn + k});
      }
    } else {
      for (size_t i = 0; i < c->h_adj_elem.size(); ++i) {
        if (c->h_adj_medium[i] != m) continue;
        const int e = c->perm[c->h_adj_elem[i]];
        for (int k = 0; k < nn; ++k)
          pairs.push_back({a.iglob[static_cast<size_t>(e) * nn + k], static_cast<int>(i) * nn + k});
      }
    }
    const std::vector<int> *self = m == MEDIUM_ACOUSTIC ? &P.v_cp_ac_self : m == MEDIUM_ELASTIC_PSV ? &P.v_cp_el_self : nullptr;
    if (self)
      for (size_t i = 0; i < self->size(); ++i) pairs.push_back({(*self)[i], -static_cast<int>(i) - 1});
    std::stable_sort(pairs.begin(), pairs.end(),
                     [](const std::pair<int, int> &x, const std::pair<int, int> &y) { return x.first < y.first; });
    std::vector<int> g, begin, ent;
    for (size_t q = 0; q < pairs.size(); ++q) {
      if (g.empty() || g.back() != pairs[q].first) {
        g.push_back(pairs[q].first);
        begin.push_back(static_cast<int>(q));
      }
      ent.push_back(pairs[q].second);
    }
    begin.push_back(static_cast<int>(pairs.size()));
    T.n = static_cast<int>(g.size());
    T.g.upload(g, &c->device_bytes);
    T.begin.upload(begin, &c->device_bytes);
    T.ent.upload(ent, &c->device_bytes);
    T.ready = true;
  }
  return dev::DetTail{T.n, T.g.p, T.begin.p, T.ent.p};
}

// The stiffness of one medium with its sources and coupling (`tw`, may be
// null): one launch in the atomic assembly, or, in the deterministic mode,
// one launch per element colour and then the owner-computes tail launch.
void stiffness_medium(sfb_context *c, int medium, const dev::MediumFields &f, const dev::StaceyStore &ss,
                      const int *istep, const dev::TailWork *tw, const dev::FusedUpdate *fu, int src_kind) {
  const int S = c->P.nshots, n = c->P.asmb.ngll;
  if (!c->deterministic) {
    dev::launch_stiffness(medium, n, c->st, f, S, ss, istep, c->stream, tw, fu, c->shots_variant[medium]);
    return;
  }
  for (int k = 0; k < c->ncolor[medium]; ++k) {
    dev::MediumFields fk = f;
    fk.elem_begin = c->col_begin[medium][k];
    fk.nelem = c->col_count[medium][k];
    dev::launch_stiffness(medium, n, c->st, fk, S, ss, istep, c->stream, nullptr, fu, c->shots_variant[medium]);
  }
  if (tw && f.nelem > 0) dev::launch_tail_det(medium, n, c->st, f, S, istep, *tw, det_tail(c, src_kind, medium), c->stream);
}

// Element-private points are updated inside the batched P-SV stiffness launch
// of the forward run unless an option needs every point in the update kernel.
bool private_update_on(sfb_context *c) {
  return c->nprivate_points > 0 && !c->compensated && c->ck_count == 0;
}

// One fused forward step: sources, coupling and stiffness per medium in the
// reference order, seismograms, then the update kernels.
void enqueue_fused_step(sfb_context *c, WavefieldSet &W, int last) {
  const Problem &P = c->P;
  const int S = P.nshots, n = P.asmb.ngll;
  const real dt = static_cast<real>(P.dt);
  const real dt2 = static_cast<real>(P.dt / 2.0), dtsq2 = static_cast<real>(P.dt * P.dt / 2.0);
  const int *istep = &W.ctrl.p->istep;
  dev::StaceyStore ss{};
  if (P.save_boundary_values && c->stacey_data.p) {
    ss.data = c->stacey_data.p;
    ss.slot = c->stacey_slot.p;
    ss.nstacey = c->nstacey;
    ss.nstep = P.nstep;
    ss.mode = 1;
  }
  dev::SourceSet src = source_set(c);
  // acoustic first (time_marching.tpp:48-52): stiffness + sources + coupling
  // from the predicted elastic displacement, in one launch
  // single shot with both media: the elastic launch starts while the
  // acoustic one finishes (its element loop does not depend on it)
  const bool overlap = S == 1 && W.f[dev::MED_AC].nelem > 0 && W.f[dev::MED_PSV].nelem > 0 && !c->deterministic;
  dev::TailWork ta{};
  ta.src = src;
  ta.cp = coupling_acoustic(c);
  ta.other = W.f[dev::MED_PSV];
  ta.cp_mode = ta.cp.n > 0 ? 1 : 0;
  ta.overlap = overlap ? dev::kOverlapFirst : 0;
  stiffness_medium(c, dev::MED_AC, W.f[dev::MED_AC], ss, istep, &ta, nullptr, 0);
  // elastic: coupling reads the final acoustic acceleration = force * minv
  dev::TailWork te{};
  te.src = src;
  te.cp = coupling_elastic(c);
  te.other = W.f[dev::MED_AC];
  te.cp_mode = te.cp.n > 0 ? 2 : 0;
  te.other_divided = 0;
  te.overlap = overlap ? dev::kOverlapSecond : 0;
  dev::FusedUpdate fu{};
  const bool fused = private_update_on(c);
  if (fused) {
    fu.enabled = 1;
    fu.minv = c->minv[dev::MED_PSV].p;
    fu.v = W.f[dev::MED_PSV].v;
    fu.dt = dt;
    fu.dt2 = dt2;
    fu.dtsq2 = dtsq2;
    fu.last = last;
  }
  stiffness_medium(c, dev::MED_PSV, W.f[dev::MED_PSV], ss, istep, &te, fused ? &fu : nullptr, 0);
  dev::TailWork tsh{};
  tsh.src = src;
  stiffness_medium(c, dev::MED_SH, W.f[dev::MED_SH], ss, istep, &tsh, nullptr, 0);
  build_taps(c);
  if (c->deterministic) {
    // seismograms in the receiver kernel's fixed summation order, from
    // (u, v*, force) before the update
    dev::launch_receivers(n, c->st, receiver_set(c, W), W.f, S, dt2, 1, istep, c->stream);
    dev::launch_update_all(update_params(c, W, last, true, false, fused, true), c->stream);
  } else {
    dev::launch_update_all(update_params(c, W, last, true, true, fused, true), c->stream);
  }
}

// Number of kernels one fused step launches (mirrors the skip conditions of
// the launchers in kernels.cu).
int fused_step_launches(sfb_context *c, WavefieldSet &W) {
  int n = 0;
  for (int m : {dev::MED_AC, dev::MED_PSV, dev::MED_SH}) {
    if (W.f[m].nelem == 0) continue;
    if (!c->deterministic) {
      ++n;  // stiffness (+ sources + coupling)
    } else {
      n += c->ncolor[m];                   // one stiffness launch per colour
      if (det_tail(c, 0, m).ntarget) ++n;  // sources + coupling
    }
  }
  if (c->deterministic && !c->P.receivers.empty() && !c->P.seismogram_types.empty()) ++n;  // receivers
  return n + 1;  // one update launch for all media
}

void predictor_all(sfb_context *c, WavefieldSet &W, double sgn) {
  const Problem &P = c->P;
  for (int m : kMedia)
    dev::launch_predictor(W.f[m], P.nshots, static_cast<real>(sgn * P.dt), static_cast<real>(sgn * P.dt / 2.0),
                          static_cast<real>(P.dt * P.dt / 2.0), c->stream, W.cu[m].p, W.cv[m].p);
}

void ensure_store(sfb_context *c) {
  const Problem &P = c->P;
  if (c->stacey_data.p || c->nstacey == 0) return;
  const size_t n = static_cast<size_t>(P.nshots) * P.nstep * c->nstacey * P.asmb.ngll * P.asmb.ngll * 2;
  c->stacey_data.alloc(n, &c->device_bytes);
}

// Everything the deterministic mode's launches allocate, built before any
// stream capture (no allocation may happen inside one).
void prepare_deterministic(sfb_context *c) {
  if (!c->deterministic) return;
  for (int m : kMedia) {
    det_tail(c, 0, m);
    if (!c->h_adj_elem.empty()) det_tail(c, 1, m);
  }
}

// Enqueue a capture's work; if it throws, end the capture (discarding the
// partial graph) so that the stream is usable again, and rethrow.
template <typename F> void capture_steps(sfb_context *c, F &&enqueue) {
  try {
    enqueue();
  } catch (...) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(c->stream, &g);
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    throw;
  }
}

void run_forward_fused(sfb_context *c, int nstep, int use_graph) {
  WavefieldSet &W = ensure_wavefield(c, SFB_WAVEFIELD_FORWARD);
  if (c->P.save_boundary_values) ensure_store(c);
  if (!c->mass_ready) initialize_mass(c, c->P.dt);
  if (nstep <= 0) return;
  if (W.step + nstep > c->P.nstep)
    throw std::invalid_argument("run would pass the configured number of steps");
  build_taps(c);
  set_step(c, W, W.step);
  predictor_all(c, W, 1.0);
  for (int m : kMedia)
    if (W.f[m].nglob > 0) ++c->launches;
  c->launches += static_cast<uint64_t>(fused_step_launches(c, W)) * nstep;
  // the body runs as graph launches of K fused steps plus one graph of the
  // remainder, each captured on first use and kept (a run of any length is
  // graph-launched once its chunk sizes have been seen)
  const int body = nstep - 1;
  constexpr int K = 25;  // fused steps per full CUDA graph
  prepare_deterministic(c);
  auto graph_of = [&](int steps) {
    auto it = c->graphs.find(steps);
    if (it != c->graphs.end()) return it->second;
    cudaGraph_t g;
    cudaGraphExec_t ex = nullptr;
    ck(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    capture_steps(c, [&]() {
      for (int k = 0; k < steps; ++k) enqueue_fused_step(c, W, 0);
    });
    ck(cudaStreamEndCapture(c->stream, &g), "end capture");
    ck(cudaGraphInstantiate(&ex, g, 0), "graph instantiate");
    cudaGraphDestroy(g);
    c->graphs[steps] = ex;
    return ex;
  };
  if (use_graph && body > 0) {
    int done = 0;
    while (done + K <= body) {
      ck(cudaGraphLaunch(graph_of(K), c->stream), "graph launch");
      done += K;
    }
    if (done < body) ck(cudaGraphLaunch(graph_of(body - done), c->stream), "graph launch");
  } else {
    for (int k = 0; k < body; ++k) enqueue_fused_step(c, W, 0);
  }
  enqueue_fused_step(c, W, 1);
  ck(cudaGetLastError(), "forward step kernels");
  W.step += nstep;
}

dev::SourceSet adjoint_source_set(sfb_context *c);
void ensure_adjoint_sources(sfb_context *c);
dev::StaceyStore replay_store(sfb_context *c);
void ensure_store(sfb_context *c);

// domain_kernels<W>::update_wavefields<medium>(istep): coupling, sources
// (forward and backward: the forward sources; adjoint: the adjoint sources),
// stiffness (forward: storing the Stacey elements' contributions when
// save_boundary_values; backward: replaying them), divide by mass.
int update_wavefields(sfb_context *c, int w, int medium, int istep) {
  WavefieldSet &W = ensure_wavefield(c, w);
  const Problem &P = c->P;
  const int S = P.nshots, n = P.asmb.ngll;
  set_step(c, W, istep);
  const int *is = &W.ctrl.p->istep;
  dev::StaceyStore ss{};
  if (w == SFB_WAVEFIELD_FORWARD && P.save_boundary_values && c->nstacey > 0) {
    ensure_store(c);
    ss.data = c->stacey_data.p;
    ss.slot = c->stacey_slot.p;
    ss.nstacey = c->nstacey;
    ss.nstep = P.nstep;
    ss.mode = 1;
  } else if (w == SFB_WAVEFIELD_BACKWARD) {
    ss = replay_store(c);
  }
  if (w == SFB_WAVEFIELD_ADJOINT) ensure_adjoint_sources(c);
  dev::SourceSet src = w == SFB_WAVEFIELD_ADJOINT ? adjoint_source_set(c) : source_set(c);
  if (c->deterministic) {
    // colour launches, then sources and coupling (the acoustic medium is
    // already divided by its mass here) through the owner-computes map
    dev::TailWork tw{};
    tw.src = src;
    if (medium == dev::MED_AC) {
      tw.cp = coupling_acoustic(c);
      tw.other = W.f[dev::MED_PSV];
      tw.cp_mode = tw.cp.n > 0 ? 1 : 0;
    } else if (medium == dev::MED_PSV) {
      tw.cp = coupling_elastic(c);
      tw.other = W.f[dev::MED_AC];
      tw.cp_mode = tw.cp.n > 0 ? 2 : 0;
      tw.other_divided = 1;
    }
    stiffness_medium(c, medium, W.f[medium], ss, is, &tw, nullptr, w == SFB_WAVEFIELD_ADJOINT ? 1 : 0);
    dev::launch_divide(W.f[medium], S, c->stream);
    ck(cudaGetLastError(), "update_wavefields");
    return W.f[medium].nelem;
  }
  if (medium == dev::MED_AC) {
    dev::launch_coupling_acoustic(coupling_acoustic(c), W.f[dev::MED_AC], W.f[dev::MED_PSV], S, c->stream);
  } else if (medium == dev::MED_PSV) {
    dev::launch_coupling_elastic(coupling_elastic(c), W.f[dev::MED_PSV], W.f[dev::MED_AC], S, 1, c->stream);
  }
  dev::launch_sources(n, c->st, src, W.f, S, medium, is, 0, c->stream);
  dev::launch_stiffness(medium, n, c->st, W.f[medium], S, ss, is, c->stream, nullptr, nullptr,
                        c->shots_variant[medium]);
  dev::launch_divide(W.f[medium], S, c->stream);
  ck(cudaGetLastError(), "update_wavefields");
  return W.f[medium].nelem;
}


// ===========================================================================
// Combined (adjoint + backward) loop, time_marching<combined>::run
// (include/solver/time_marching.tpp:126-247), fused per step:
//   adjoint stiffness (acoustic, elastic) with adjoint sources and coupling,
//   backward stiffness (elastic, acoustic) replaying the Stacey store, with
//   the forward sources; the backward elastic update sees a zero acoustic
//   acceleration (the reference predicts both media before updating the
//   elastic one), so that coupling term is absent, as in the reference;
//   Frechet accumulation from the adjoint displacement / acceleration and
//   the backward displacement; then both updates (+dt adjoint, -dt
//   backward); one step counter counts down.
// ===========================================================================
dev::SourceSet adjoint_source_set(sfb_context *c) {
  dev::SourceSet s{};
  s.n = c->nadj;
  s.elem = c->adj_elem.p;
  s.shot = c->adj_shot.p;
  s.medium = c->adj_medium.p;
  s.array = c->adj_array.p;
  s.stf = c->adj_stf.p;
  s.nstep = c->P.nstep;
  return s;
}

void ensure_adjoint_sources(sfb_context *c) {
  if (c->nadj > 0) return;
  if (!c->P.located_adjoint.empty()) {
    // adjoint sources from the sources file, with their own time functions
    ensure_device(c);
    const Problem &P = c->P;
    const int nn = P.asmb.ngll * P.asmb.ngll;
    c->nadj = static_cast<int>(P.located_adjoint.size());
    std::vector<int> el(c->nadj), sh(c->nadj, 0), md(c->nadj);
    std::vector<real> arr(static_cast<size_t>(c->nadj) * 2 * nn, 0), stf(static_cast<size_t>(c->nadj) * P.nstep * 2);
    for (int i = 0; i < c->nadj; ++i) {
      const LocatedSource &L = P.located_adjoint[i];
      el[i] = c->inv[L.ispec];
      md[i] = L.medium;
      for (int cc = 0; cc < 2; ++cc)
        for (int k = 0; k < nn; ++k) arr[(static_cast<size_t>(i) * 2 + cc) * nn + k] = L.array[static_cast<size_t>(cc) * nn + k];
      for (int t = 0; t < P.nstep; ++t)
        for (int cc = 0; cc < 2; ++cc)
          stf[(static_cast<size_t>(i) * P.nstep + t) * 2 + cc] = L.stf[static_cast<size_t>(t) * 2 + cc];
    }
    size_t *tot = &c->device_bytes;
    c->adj_elem.upload(el, tot);
    c->adj_shot.upload(sh, tot);
    c->adj_medium.upload(md, tot);
    c->adj_array.upload(arr, tot);
    c->adj_stf.upload(stf, tot);
    c->h_adj_elem = el;
    c->h_adj_medium = md;
    return;
  }
  if (c->P.receivers.empty()) return;
  ensure_device(c);
  const Problem &P = c->P;
  const Assembly &a = P.asmb;
  const int nn = a.ngll * a.ngll, nrec = static_cast<int>(P.receivers.size()), S = P.nshots;
  c->nadj = S * nrec;
  std::vector<int> el(c->nadj), sh(c->nadj), md(c->nadj);
  std::vector<real> arr(static_cast<size_t>(c->nadj) * 2 * nn, 0);
  for (int s = 0; s < S; ++s)
    for (int r = 0; r < nrec; ++r) {
      const int i = s * nrec + r;
      const LocatedReceiver &L = P.located_receivers[r];
      el[i] = c->inv[L.ispec];
      sh[i] = s;
      md[i] = a.medium[L.ispec];
      // reference: src/source/adjoint_source.cpp (lagrange in every component)
      for (int cc = 0; cc < 2; ++cc)
        for (int k = 0; k < nn; ++k) arr[(static_cast<size_t>(i) * 2 + cc) * nn + k] = L.lagrange[k];
    }
  size_t *tot = &c->device_bytes;
  c->adj_elem.upload(el, tot);
  c->adj_shot.upload(sh, tot);
  c->adj_medium.upload(md, tot);
  c->adj_array.upload(arr, tot);
  c->adj_stf.alloc(static_cast<size_t>(c->nadj) * P.nstep * 2, tot);
  c->h_adj_elem = el;
  c->h_adj_medium = md;
}

dev::StaceyStore replay_store(sfb_context *c) {
  dev::StaceyStore ss{};
  if (c->stacey_data.p) {
    ss.data = c->stacey_data.p;
    ss.slot = c->stacey_slot.p;
    ss.nstacey = c->nstacey;
    ss.nstep = c->P.nstep;
    ss.mode = 2;
  }
  return ss;
}

// Adjoint stiffness (both media) for the step held by the adjoint counter.
void enqueue_adjoint_stiffness(sfb_context *c, WavefieldSet &A) {
  const int S = c->P.nshots, n = c->P.asmb.ngll;
  const int *istep = &A.ctrl.p->istep;
  dev::StaceyStore none{};
  dev::SourceSet src = adjoint_source_set(c);
  dev::TailWork ta{};
  ta.src = src;
  ta.cp = coupling_acoustic(c);
  ta.other = A.f[dev::MED_PSV];
  ta.cp_mode = ta.cp.n > 0 ? 1 : 0;
  stiffness_medium(c, dev::MED_AC, A.f[dev::MED_AC], none, istep, &ta, nullptr, 1);
  dev::TailWork te{};
  te.src = src;
  te.cp = coupling_elastic(c);
  te.other = A.f[dev::MED_AC];
  te.cp_mode = te.cp.n > 0 ? 2 : 0;
  stiffness_medium(c, dev::MED_PSV, A.f[dev::MED_PSV], none, istep, &te, nullptr, 1);
  (void)S;
  (void)n;
}

// The batched P-SV backward stiffness carries the Frechet kernels of its
// medium (one launch instead of two, the backward gathers shared).
bool frechet_fused(sfb_context *c) {
  return c->med_count[MEDIUM_ELASTIC_PSV] > 0 &&
         dev::frechet_fusable(dev::MED_PSV, c->P.asmb.ngll, c->P.nshots);
}

// In the fused backward launch the backward wavefield's element-private
// points also finish their step (their Frechet contribution is taken first).
bool backward_private_on(sfb_context *c) { return frechet_fused(c) && c->nprivate_points > 0; }

void enqueue_backward_stiffness(sfb_context *c, WavefieldSet &A, WavefieldSet &B, int last) {
  const int S = c->P.nshots, n = c->P.asmb.ngll;
  const int *istep = &A.ctrl.p->istep;
  dev::StaceyStore ss = replay_store(c);
  dev::SourceSet src = source_set(c);
  dev::TailWork te{};
  te.src = src;  // elastic first; acoustic acceleration is zero at this point
  if (frechet_fused(c)) {
    dev::FrechetFuse fr{};
    fr.enabled = 1;
    fr.au = A.f[dev::MED_PSV].u;
    fr.aa = A.f[dev::MED_PSV].a;
    fr.minv = c->minv[dev::MED_PSV].p;
    fr.kern = c->kern.p;
    fr.dt = static_cast<real>(c->P.dt);
    if (backward_private_on(c)) {
      fr.adjoint_update = 1;
      fr.av = A.f[dev::MED_PSV].v;
      fr.adt = static_cast<real>(c->P.dt);
      fr.adt2 = static_cast<real>(c->P.dt / 2.0);
      fr.adtsq2 = static_cast<real>(c->P.dt * c->P.dt / 2.0);
      fr.last = last;
    }
    dev::FusedUpdate fu{};
    if (backward_private_on(c)) {
      fu.enabled = 1;
      fu.minv = c->minv[dev::MED_PSV].p;
      fu.v = B.f[dev::MED_PSV].v;
      fu.dt = static_cast<real>(-c->P.dt);
      fu.dt2 = static_cast<real>(-c->P.dt / 2.0);
      fu.dtsq2 = static_cast<real>(c->P.dt * c->P.dt / 2.0);
      fu.last = last;
    }
    if (!c->deterministic) {
      dev::launch_stiffness_frechet(n, c->st, B.f[dev::MED_PSV], S, ss, istep, te, fr, fu, c->stream);
    } else {
      const dev::MediumFields &f = B.f[dev::MED_PSV];
      for (int k = 0; k < c->ncolor[dev::MED_PSV]; ++k) {
        dev::MediumFields fk = f;
        fk.elem_begin = c->col_begin[dev::MED_PSV][k];
        fk.nelem = c->col_count[dev::MED_PSV][k];
        dev::launch_stiffness_frechet(n, c->st, fk, S, ss, istep, dev::TailWork{}, fr, fu, c->stream);
      }
      if (f.nelem > 0)
        dev::launch_tail_det(dev::MED_PSV, n, c->st, f, S, istep, te, det_tail(c, 0, dev::MED_PSV), c->stream);
    }
  } else {
    stiffness_medium(c, dev::MED_PSV, B.f[dev::MED_PSV], ss, istep, &te, nullptr, 0);
  }
  dev::TailWork ta{};
  ta.src = src;
  ta.cp = coupling_acoustic(c);
  ta.other = B.f[dev::MED_PSV];
  ta.cp_mode = ta.cp.n > 0 ? 1 : 0;
  stiffness_medium(c, dev::MED_AC, B.f[dev::MED_AC], ss, istep, &ta, nullptr, 0);
}

void enqueue_frechet(sfb_context *c, WavefieldSet &A, const dev::MediumFields *bwd_fields, int a_is_force,
                     bool psv_done = false, real vcorr = 0) {
  const real dt = static_cast<real>(c->P.dt);
  if (c->stacey_kernels)
    dev::launch_stacey_frechet(c->P.asmb.ngll, c->st, A.f[dev::MED_PSV], bwd_fields[dev::MED_PSV], c->P.nshots, dt,
                               vcorr, c->kern_b.p, c->stream);
  for (int m : {dev::MED_PSV, dev::MED_AC}) {
    if (m == dev::MED_PSV && psv_done) continue;
    dev::launch_frechet(m, c->P.asmb.ngll, c->st, A.f[m], bwd_fields[m], c->P.nshots, dt, c->kern.p, a_is_force,
                        c->stream);
  }
}

dev::UpdateParams update_params_signed(sfb_context *c, WavefieldSet &W, int last, bool advance, bool taps,
                                       double sgn, bool private_done = false) {
  dev::UpdateParams u = update_params(c, W, last, advance, taps, private_done);
  u.dt = static_cast<real>(sgn * c->P.dt);
  u.dt2 = static_cast<real>(sgn * c->P.dt / 2.0);
  u.dir = -1;
  return u;
}

void enqueue_restore(sfb_context *c, WavefieldSet &A, WavefieldSet &B) {
  if (c->ck_count == 0) return;
  dev::RestoreParams r{};
  for (int m : kMedia) {
    if (!B.u[m].n) continue;
    r.u[r.nm] = B.u[m].p;
    r.v[r.nm] = B.v[m].p;
    r.ck_u[r.nm] = c->ck_u[m].p;
    r.ck_v[r.nm] = c->ck_v[m].p;
    r.n[r.nm] = B.u[m].n;
    r.ck_stride[r.nm] = c->ck_stride[m];
    ++r.nm;
  }
  r.ctrl = A.ctrl.p;
  r.interval = c->ck_interval;
  r.count = c->ck_count;
  dev::launch_restore(r, c->stream);
}

void enqueue_combined_step(sfb_context *c, WavefieldSet &A, WavefieldSet &B, int last) {
  enqueue_restore(c, A, B);
  enqueue_adjoint_stiffness(c, A);
  enqueue_backward_stiffness(c, A, B, last);
  // the backward fields hold (u, v*, force) here: the step's final velocity
  // is v* - dt/2 force M^-1
  enqueue_frechet(c, A, B.f, 1, frechet_fused(c), static_cast<real>(-c->P.dt / 2.0));
  // with the fused Frechet launch, both wavefields' private points are done
  dev::UpdateParams ua = update_params_signed(c, A, last, false, false, 1.0, backward_private_on(c));
  dev::launch_update_all(ua, c->stream);
  // the backward update records the backward seismograms and counts the
  // shared step counter (held by the adjoint set) down; the deterministic
  // mode records them with the receiver kernel first
  if (c->deterministic) {
    dev::ReceiverSet rs = receiver_set(c, B);
    rs.backward_nstep = c->P.nstep;
    dev::launch_receivers(c->P.asmb.ngll, c->st, rs, B.f, c->P.nshots, static_cast<real>(-c->P.dt / 2.0), 1,
                          &A.ctrl.p->istep, c->stream);
  }
  dev::UpdateParams ub = update_params_signed(c, B, last, false, !c->deterministic, -1.0, backward_private_on(c));
  ub.ctrl = A.ctrl.p;
  dev::launch_update_all(ub, c->stream);
}

void copy_fields(sfb_context *c, WavefieldSet &dst, const WavefieldSet &src) {
  for (int m : kMedia) {
    const size_t n = dst.u[m].n;
    if (!n) continue;
    ck(cudaMemcpyAsync(dst.u[m].p, src.u[m].p, n * sizeof(real), cudaMemcpyDeviceToDevice, c->stream), "copy u");
    ck(cudaMemcpyAsync(dst.v[m].p, src.v[m].p, n * sizeof(real), cudaMemcpyDeviceToDevice, c->stream), "copy v");
    ck(cudaMemcpyAsync(dst.a[m].p, src.a[m].p, n * sizeof(real), cudaMemcpyDeviceToDevice, c->stream), "copy a");
  }
}

void zero_fields(sfb_context *c, WavefieldSet &W) {
  for (int m : kMedia) {
    const size_t n = W.u[m].n;
    if (!n) continue;
    ck(cudaMemsetAsync(W.u[m].p, 0, n * sizeof(real), c->stream), "zero u");
    ck(cudaMemsetAsync(W.v[m].p, 0, n * sizeof(real), c->stream), "zero v");
    ck(cudaMemsetAsync(W.a[m].p, 0, n * sizeof(real), c->stream), "zero a");
  }
  if (W.seis.n) ck(cudaMemsetAsync(W.seis.p, 0, W.seis.n * sizeof(real), c->stream), "zero seis");
}

void run_combined_fused(sfb_context *c, int use_graph) {
  const Problem &P = c->P;
  for (int e = 0; e < P.asmb.nspec; ++e)
    if (P.asmb.medium[e] == MEDIUM_ELASTIC_SH)
      throw std::invalid_argument("combined SH runs are not supported (the reference's combined loop has no SH backward predictor)");
  WavefieldSet &F = ensure_wavefield(c, SFB_WAVEFIELD_FORWARD);
  if (F.step != P.nstep)
    throw StateError("the combined run needs the forward run's final state: run " + std::to_string(P.nstep) +
                     " forward steps first (done: " + std::to_string(F.step) + ")");
  if (c->nstacey > 0 && !c->stacey_data.p)
    throw StateError("the forward run did not keep the Stacey store (save_boundary_values)");
  WavefieldSet &A = ensure_wavefield(c, SFB_WAVEFIELD_ADJOINT);
  WavefieldSet &B = ensure_wavefield(c, SFB_WAVEFIELD_BACKWARD);
  ensure_adjoint_sources(c);
  if (!c->mass_ready) initialize_mass(c, P.dt);
  build_taps(c);
  prepare_deterministic(c);
  const size_t nk = P.asmb.nloc() * 3;
  if (!c->kern.p) c->kern.alloc(nk, &c->device_bytes);
  ck(cudaMemsetAsync(c->kern.p, 0, nk * sizeof(double), c->stream), "zero kernels");
  if (c->stacey_kernels) {
    if (!c->kern_b.p) c->kern_b.alloc(P.asmb.nloc() * 2, &c->device_bytes);
    ck(cudaMemsetAsync(c->kern_b.p, 0, c->kern_b.n * sizeof(double), c->stream), "zero boundary kernels");
  }
  zero_fields(c, A);
  zero_fields(c, B);
  const int N = P.nstep;
  set_step(c, A, N - 1);
  // step N-1: adjoint from rest; the backward state is the forward run's last
  // state (the reference overwrites its first backward step with it)
  enqueue_adjoint_stiffness(c, A);
  enqueue_frechet(c, A, F.f, 1);
  {
    dev::UpdateParams ua = update_params_signed(c, A, N == 1, true, false, 1.0);
    dev::launch_update_all(ua, c->stream);
  }
  c->launches += 4;
  if (N > 1) {
    copy_fields(c, B, F);
    // the backward seismogram of step N-1 is the seismogram of the forward
    // run's last state, recorded from the backward fields that now hold it
    // (also when that state was read from files); it is the backward run's
    // first sample (backward samples are numbered in loop order,
    // time_marching.tpp:208-212)
    set_step(c, B, N - 1);
    dev::ReceiverSet rs = receiver_set(c, B);
    rs.backward_nstep = N;
    dev::launch_receivers(P.asmb.ngll, c->st, rs, B.f, P.nshots, real(0), 0, &B.ctrl.p->istep, c->stream);
    for (int m : kMedia)
      dev::launch_predictor(B.f[m], P.nshots, static_cast<real>(-P.dt), static_cast<real>(-P.dt / 2.0),
                            static_cast<real>(P.dt * P.dt / 2.0), c->stream);
  }
  const int per_step = 7 + (c->ck_count > 0 ? 1 : 0) - (frechet_fused(c) ? 1 : 0);
  const int body = N - 2;  // steps N-2 .. 1 in the body, step 0 closes
  constexpr int K = 25;
  int done = 0;
  auto graph_of = [&](int steps) {
    auto it = c->graphs_combined.find(steps);
    if (it != c->graphs_combined.end()) return it->second;
    cudaGraph_t g;
    cudaGraphExec_t ex = nullptr;
    ck(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    capture_steps(c, [&]() {
      for (int k = 0; k < steps; ++k) enqueue_combined_step(c, A, B, 0);
    });
    ck(cudaStreamEndCapture(c->stream, &g), "end capture");
    ck(cudaGraphInstantiate(&ex, g, 0), "graph instantiate");
    cudaGraphDestroy(g);
    c->graphs_combined[steps] = ex;
    return ex;
  };
  if (use_graph && body > 0) {
    while (done + K <= body) {
      ck(cudaGraphLaunch(graph_of(K), c->stream), "graph launch");
      done += K;
    }
    if (done < body) {
      ck(cudaGraphLaunch(graph_of(body - done), c->stream), "graph launch");
      done = body;
    }
  }
  for (; done < body; ++done) enqueue_combined_step(c, A, B, 0);
  if (N > 1) enqueue_combined_step(c, A, B, 1);
  c->launches += static_cast<uint64_t>(per_step) * (N > 1 ? N - 1 : 0);
  ck(cudaGetLastError(), "combined step kernels");
  A.step = N;
  B.step = N;
}
}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================

namespace {
// The device error word: bit kErrWaitTimeout (a bounded device-side wait
// expired) and bit kErrNonFinite (the watchdog saw NaN or Inf).  Entry
// points report it without a device synchronisation: each one starts by
// reading the pinned host copy that the previous one's asynchronous copy
// left (poll_device_flag) and ends by enqueueing a new copy
// (note_device_flag); the synchronising calls read it directly.
void raise_device_error(sfb_context *c, int h) {
  const int zero = 0;
  cudaMemcpy(c->dflag.p, &zero, sizeof(int), cudaMemcpyHostToDevice);
  if (c->h_err) *c->h_err = 0;
  if (h & dev::kErrWaitTimeout)
    throw CudaError("a device-side wait timed out (bounded mbarrier wait in a device kernel)");
  throw NonFiniteError("non-finite values (NaN or Inf) in the wavefields or kernels");
}
void note_device_flag(sfb_context *c) {
  if (c->dflag.p && c->h_err)
    ck(cudaMemcpyAsync(c->h_err, c->dflag.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "error word");
}
void poll_device_flag(sfb_context *c) {
  if (!c->h_err) return;
  const int h = *static_cast<volatile int *>(c->h_err);
  if (h != 0) {
    ck(cudaStreamSynchronize(c->stream), "sync");
    raise_device_error(c, h);
  }
}
void check_device_flag(sfb_context *c) {
  if (!c->dflag.p) return;
  int h = 0;
  ck(cudaStreamSynchronize(c->stream), "sync");
  ck(cudaMemcpy(&h, c->dflag.p, sizeof(int), cudaMemcpyDeviceToHost), "error flag");
  if (h != 0) raise_device_error(c, h);
}
// Watchdog over a wavefield set (u and v of every medium).
void enqueue_nonfinite(sfb_context *c, WavefieldSet &W) {
  for (int m : kMedia) {
    dev::launch_nonfinite_check(W.u[m].p, W.u[m].n, c->dflag.p, c->stream);
    dev::launch_nonfinite_check(W.v[m].p, W.v[m].n, c->dflag.p, c->stream);
  }
}

}  // namespace

SFB_API const char *sfb_last_error(const sfb_context *ctx) {
  return ctx ? ctx->err.c_str() : g_create_error.c_str();
}

SFB_API int sfb_create_from_yaml(const char *parameter_file, const char *default_file, sfb_context **out) {
  if (!parameter_file || !out) return fail(nullptr, SFB_E_INVALID, "null argument");
  *out = nullptr;
  return guarded(nullptr, [&]() {
    std::unique_ptr<sfb_context> c(new sfb_context());
    c->P = problem_from_yaml(parameter_file, default_file ? default_file : "");
    c->deterministic = deterministic_default();
    *out = c.release();
    return SFB_OK;
  });
}

SFB_API int sfb_create_from_yaml_text(const char *parameter_yaml, const char *default_yaml, sfb_context **out) {
  if (!parameter_yaml || !out) return fail(nullptr, SFB_E_INVALID, "null argument");
  *out = nullptr;
  return guarded(nullptr, [&]() {
    std::unique_ptr<sfb_context> c(new sfb_context());
    c->P = problem_from_yaml_text(parameter_yaml, default_yaml ? default_yaml : "");
    c->deterministic = deterministic_default();
    *out = c.release();
    return SFB_OK;
  });
}

SFB_API int sfb_create_structured(const sfb_structured_desc *desc, sfb_context **out) {
  if (!desc || !out) return fail(nullptr, SFB_E_INVALID, "null argument");
  *out = nullptr;
  return guarded(nullptr, [&]() {
    std::unique_ptr<sfb_context> c(new sfb_context());
    c->P = problem_from_structured(*desc);
    c->deterministic = deterministic_default();
    *out = c.release();
    return SFB_OK;
  });
}

SFB_API void sfb_destroy(sfb_context *ctx) { delete ctx; }

SFB_API int sfb_get_info(const sfb_context *ctx, sfb_info *info) {
  if (!ctx || !info) return SFB_E_INVALID;
  const Problem &P = ctx->P;
  *info = sfb_info{};
  info->ngll = P.asmb.ngll;
  info->nspec = P.asmb.nspec;
  info->nshots = P.nshots;
  info->nstep = P.nstep;
  info->nstep_between_samples = P.nstep_between_samples;
  info->max_sig_step = P.max_sig_step();
  for (int m = 0; m < 4; ++m) {
    info->nglob[m] = P.asmb.nglob[m];
    info->nelements[m] = P.asmb.count_elements(m);
  }
  info->nreceivers = static_cast<int>(P.receivers.size());
  info->nseismogram_types = static_cast<int>(P.seismogram_types.size());
  info->nsources = static_cast<int>(P.sources.size());
  info->simulation = P.simulation;
  info->dt = P.dt;
  info->t0 = P.t0;
  info->device_bytes = ctx->device_bytes;
  info->kernel_launches = ctx->launches;
  for (int m = 0; m < 4; ++m) info->stiffness_variant[m] = ctx->shots_variant[m];
  info->private_points = ctx->nprivate_points;
  info->nadjoint_sources = static_cast<int>(P.adjoint_sources.size());
  return SFB_OK;
}

SFB_API int sfb_set_newmark_compensation(sfb_context *ctx, int enable) {
  if (!ctx) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    WavefieldSet &W = ensure_wavefield(ctx, SFB_WAVEFIELD_FORWARD);
    for (int m : kMedia) {
      if (enable) {
        if (!W.cu[m].p && W.u[m].n) {
          W.cu[m].alloc(W.u[m].n, &ctx->device_bytes);
          W.cv[m].alloc(W.v[m].n, &ctx->device_bytes);
        }
      } else {
        if (W.cu[m].p) ctx->device_bytes -= 2 * W.cu[m].n * sizeof(real);
        W.cu[m].free();
        W.cv[m].free();
      }
    }
    ctx->compensated = enable != 0;
    ctx->drop_forward_graphs();  // captured launches hold the old pointers
    return SFB_OK;
  });
}

SFB_API int sfb_set_checkpoint_interval(sfb_context *ctx, int interval) {
  if (!ctx) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    if (interval < 0) throw std::invalid_argument("checkpoint interval must be >= 0");
    WavefieldSet &F = ensure_wavefield(ctx, SFB_WAVEFIELD_FORWARD);
    if (F.step != 0) throw StateError("set the checkpoint interval before the forward run");
    const int N = ctx->P.nstep;
    const int count = (interval > 0 && N >= 2) ? (N - 2) / interval : 0;
    for (int m : kMedia) {
      if (ctx->ck_u[m].p) ctx->device_bytes -= 2 * ctx->ck_u[m].n * sizeof(real);
      ctx->ck_u[m].free();
      ctx->ck_v[m].free();
      ctx->ck_stride[m] = 0;
      if (count > 0 && F.u[m].n) {
        const size_t stride = (F.u[m].n + 3) & ~static_cast<size_t>(3);  // 16-byte aligned slots
        ctx->ck_u[m].alloc(stride * count, &ctx->device_bytes);
        ctx->ck_v[m].alloc(stride * count, &ctx->device_bytes);
        ctx->ck_stride[m] = stride;
      }
    }
    ctx->ck_interval = count > 0 ? interval : 0;
    ctx->ck_count = count;
    ctx->drop_forward_graphs();
    ctx->drop_combined_graphs();
    return SFB_OK;
  });
}

SFB_API int sfb_set_stacey_kernels(sfb_context *ctx, int enable) {
  if (!ctx) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    if (ctx->stacey_kernels != (enable != 0)) ctx->drop_combined_graphs();  // captured steps hold the old launches
    ctx->stacey_kernels = enable != 0;
    return SFB_OK;
  });
}

SFB_API int sfb_set_deterministic(sfb_context *ctx, int enable) {
  if (!ctx) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    if (ctx->on_device && (enable != 0) != ctx->deterministic)
      throw StateError("choose the assembly mode before the context's first device use");
    ctx->deterministic = enable != 0;
    return SFB_OK;
  });
}

SFB_API int sfb_set_stiffness_variant(sfb_context *ctx, int medium, int variant) {
  if (!ctx) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    if (!medium_index_ok(medium)) throw std::invalid_argument("unsupported medium tag");
    const int top = ctx->P.nshots == 1 ? dev::kRowAffine : dev::kShotsSingle;
    if (variant < dev::kShotsAuto || variant > top) throw std::invalid_argument("unknown stiffness variant");
    ctx->shots_variant[medium] = variant;
    ctx->drop_forward_graphs();  // captured launches use the old kernel
    ctx->drop_combined_graphs();
    return SFB_OK;
  });
}

SFB_API int sfb_get_problem_view(const sfb_context *ctx, sfb_problem_view *view) {
  if (!ctx || !view) return SFB_E_INVALID;
  ctx->P.fill_view(view);
  return SFB_OK;
}

SFB_API int sfb_domain_initialize(sfb_context *ctx, int wavefield, double dt) {
  if (!ctx) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    if (wavefield < 0 || wavefield > 2) throw std::invalid_argument("bad wavefield");
    ensure_wavefield(ctx, wavefield);
    initialize_mass(ctx, dt);
    ctx->wf[wavefield].initialized = true;
    return SFB_OK;
  });
}

SFB_API int sfb_domain_update_wavefields(sfb_context *ctx, int wavefield, int medium, int istep,
                                         int *elements_updated) {
  if (!ctx) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    if (!medium_index_ok(medium)) throw std::invalid_argument("unsupported medium tag");
    if (!ctx->mass_ready) throw StateError("domain_kernels::initialize has not been called");
    poll_device_flag(ctx);
    const int n = update_wavefields(ctx, wavefield, medium, istep);
    note_device_flag(ctx);
    if (elements_updated) *elements_updated = n;
    return SFB_OK;
  });
}

SFB_API int sfb_domain_compute_seismograms(sfb_context *ctx, int wavefield, int isig_step) {
  if (!ctx) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    WavefieldSet &W = ensure_wavefield(ctx, wavefield);
    poll_device_flag(ctx);
    // the kernel derives isig from the step counter: isig * nsbs
    set_step(ctx, W, isig_step * ctx->P.nstep_between_samples);
    dev::launch_receivers(ctx->P.asmb.ngll, ctx->st, receiver_set(ctx, W), W.f, ctx->P.nshots, real(0), 0,
                          &W.ctrl.p->istep, ctx->stream);
    ck(cudaGetLastError(), "compute_seismograms");
    note_device_flag(ctx);
    return SFB_OK;
  });
}

SFB_API int sfb_newmark_predictor(sfb_context *ctx, int wavefield, int medium, int *dofs) {
  if (!ctx) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    if (!medium_index_ok(medium)) throw std::invalid_argument("unsupported medium tag");
    WavefieldSet &W = ensure_wavefield(ctx, wavefield);
    const double sgn = wavefield == SFB_WAVEFIELD_BACKWARD ? -1.0 : 1.0;
    const Problem &P = ctx->P;
    poll_device_flag(ctx);
    dev::launch_predictor(W.f[medium], P.nshots, static_cast<real>(sgn * P.dt),
                          static_cast<real>(sgn * P.dt / 2.0), static_cast<real>(P.dt * P.dt / 2.0),
                          ctx->stream);
    ck(cudaGetLastError(), "predictor");
    if (dofs) *dofs = W.f[medium].nglob * W.f[medium].nc;
    return SFB_OK;
  });
}

SFB_API int sfb_newmark_corrector(sfb_context *ctx, int wavefield, int medium, int *dofs) {
  if (!ctx) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    if (!medium_index_ok(medium)) throw std::invalid_argument("unsupported medium tag");
    WavefieldSet &W = ensure_wavefield(ctx, wavefield);
    const double sgn = wavefield == SFB_WAVEFIELD_BACKWARD ? -1.0 : 1.0;
    poll_device_flag(ctx);
    dev::launch_corrector(W.f[medium], ctx->P.nshots, static_cast<real>(sgn * ctx->P.dt / 2.0), ctx->stream);
    ck(cudaGetLastError(), "corrector");
    if (dofs) *dofs = W.f[medium].nglob * W.f[medium].nc;
    return SFB_OK;
  });
}

SFB_API int sfb_synchronize(sfb_context *ctx) {
  if (!ctx) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    if (!ctx->on_device) return SFB_OK;
    for (int w = 0; w < 3; ++w)
      if (ctx->wf[w].allocated) enqueue_nonfinite(ctx, ctx->wf[w]);
    check_device_flag(ctx);
    return SFB_OK;
  });
}

SFB_API int sfb_probe_device_wait(sfb_context *ctx, long long limit_cycles) {
  if (!ctx) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    if (limit_cycles < 0 || limit_cycles > (1LL << 32)) throw std::invalid_argument("limit_cycles must be in [0, 2^32]");
    ensure_device(ctx);
    dev::launch_wait_probe(limit_cycles, ctx->dflag.p, ctx->stream);
    ck(cudaGetLastError(), "wait probe");
    note_device_flag(ctx);
    return SFB_OK;
  });
}

SFB_API int sfb_run_forward(sfb_context *ctx, int nstep, int use_graph) {
  if (!ctx) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    run_forward_fused(ctx, nstep, use_graph);
    enqueue_nonfinite(ctx, ctx->wf[SFB_WAVEFIELD_FORWARD]);
    ck(cudaStreamSynchronize(ctx->stream), "forward run");
    check_device_flag(ctx);
    return SFB_OK;
  });
}

SFB_API int sfb_run_forward_unfused(sfb_context *ctx, int nstep) {
  if (!ctx) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    ctx->err.clear();  // the loop below detects failures of its own calls by the message
    WavefieldSet &W = ensure_wavefield(ctx, SFB_WAVEFIELD_FORWARD);
    if (!ctx->mass_ready) initialize_mass(ctx, ctx->P.dt);
    const Problem &P = ctx->P;
    int total_dofs = 0;
    for (int m : kMedia) total_dofs += 2 * P.asmb.nglob[m] * P.asmb.ncomp(m);
    const int start = W.step;
    if (start + nstep > P.nstep) throw std::invalid_argument("run would pass the configured number of steps");
    int isig = start / P.nstep_between_samples;
    for (int istep = start; istep < start + nstep; ++istep) {
      int dofs = 0, elements = 0, k = 0;
      for (int m : {dev::MED_AC, dev::MED_PSV, dev::MED_SH}) {
        sfb_newmark_predictor(ctx, 0, m, &k);
        dofs += k;
      }
      elements += update_wavefields(ctx, 0, dev::MED_AC, istep);
      sfb_newmark_corrector(ctx, 0, dev::MED_AC, &k);
      dofs += k;
      elements += update_wavefields(ctx, 0, dev::MED_PSV, istep);
      elements += update_wavefields(ctx, 0, dev::MED_SH, istep);
      sfb_newmark_corrector(ctx, 0, dev::MED_PSV, &k);
      dofs += k;
      sfb_newmark_corrector(ctx, 0, dev::MED_SH, &k);
      dofs += k;
      if (istep % P.nstep_between_samples == 0 && isig < P.max_sig_step()) {
        set_step(ctx, W, istep);
        dev::launch_receivers(P.asmb.ngll, ctx->st, receiver_set(ctx, W), W.f, P.nshots, real(0), 0,
                              &W.ctrl.p->istep, ctx->stream);
        ++isig;
      }
      if (!ctx->err.empty()) throw std::runtime_error(ctx->err);
      if (dofs != total_dofs || elements != P.asmb.nspec)
        return fail(ctx, SFB_E_ACCOUNTING,
                    "The time loop has not updated all the degrees of freedom (" + std::to_string(dofs) +
                        " of " + std::to_string(total_dofs) + ") or elements (" + std::to_string(elements) +
                        " of " + std::to_string(P.asmb.nspec) + ")");
    }
    enqueue_nonfinite(ctx, W);
    ck(cudaStreamSynchronize(ctx->stream), "unfused forward run");
    check_device_flag(ctx);
    W.step = start + nstep;
    return SFB_OK;
  });
}

SFB_API int sfb_get_seismograms(const sfb_context *cctx, int wavefield, int shot, float *host, size_t count) {
  sfb_context *ctx = const_cast<sfb_context *>(cctx);
  if (!ctx || !host) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    WavefieldSet &W = ensure_wavefield(ctx, wavefield);
    const Problem &P = ctx->P;
    const size_t per = static_cast<size_t>(P.max_sig_step()) * P.seismogram_types.size() * P.receivers.size() * 2;
    if (shot < 0 || shot >= P.nshots) throw std::invalid_argument("shot out of range");
    if (count < per) throw std::invalid_argument("seismogram buffer too small");
    ck(cudaStreamSynchronize(ctx->stream), "sync");
    copy_d2h(host, W.seis.p + shot * per, per, "seis d2h");
    return SFB_OK;
  });
}

SFB_API int sfb_get_seismograms_f64(const sfb_context *cctx, int wavefield, int shot, double *host, size_t count) {
  sfb_context *ctx = const_cast<sfb_context *>(cctx);
  if (!ctx || !host) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    WavefieldSet &W = ensure_wavefield(ctx, wavefield);
    const Problem &P = ctx->P;
    const size_t per = static_cast<size_t>(P.max_sig_step()) * P.seismogram_types.size() * P.receivers.size() * 2;
    if (shot < 0 || shot >= P.nshots) throw std::invalid_argument("shot out of range");
    if (count < per) throw std::invalid_argument("seismogram buffer too small");
    ck(cudaStreamSynchronize(ctx->stream), "sync");
    copy_d2h(host, W.seis.p + shot * per, per, "seis d2h");
    return SFB_OK;
  });
}

SFB_API int sfb_real_bytes(void) { return static_cast<int>(sizeof(real)); }

namespace {
template <typename H>
int get_field_impl(sfb_context *ctx, int wavefield, int medium, int which, int shot, H *host, size_t count) {
  if (!ctx || !host) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    if (!medium_index_ok(medium)) throw std::invalid_argument("unsupported medium tag");
    WavefieldSet &W = ensure_wavefield(ctx, wavefield);
    const dev::MediumFields &f = W.f[medium];
    const size_t n = static_cast<size_t>(f.nglob) * f.nc;
    if (count < n) throw std::invalid_argument("field buffer too small");
    if (shot < 0 || shot >= ctx->P.nshots) throw std::invalid_argument("shot out of range");
    const real *src = which == 0 ? f.u : which == 1 ? f.v : which == 2 ? f.a : f.minv;
    const int S = (which == 3) ? 1 : ctx->P.nshots;
    if (which == 3) shot = 0;
    std::vector<real> tmp(n);
    ck(cudaStreamSynchronize(ctx->stream), "sync");
    // device layout [g][s][c]: gather shot `shot`, then transpose to [c][g]
    if (n)
      ck(cudaMemcpy2D(tmp.data(), f.nc * sizeof(real), src + static_cast<size_t>(shot) * f.nc,
                      static_cast<size_t>(S) * f.nc * sizeof(real), f.nc * sizeof(real), f.nglob,
                      cudaMemcpyDeviceToHost),
         "field d2h");
    for (int c = 0; c < f.nc; ++c)
      for (int g = 0; g < f.nglob; ++g)
        host[static_cast<size_t>(c) * f.nglob + g] = static_cast<H>(tmp[static_cast<size_t>(g) * f.nc + c]);
    return SFB_OK;
  });
}
}  // namespace

SFB_API int sfb_get_field(const sfb_context *cctx, int wavefield, int medium, int which, int shot, float *host,
                          size_t count) {
  return get_field_impl(const_cast<sfb_context *>(cctx), wavefield, medium, which, shot, host, count);
}

SFB_API int sfb_get_field_f64(const sfb_context *cctx, int wavefield, int medium, int which, int shot, double *host,
                              size_t count) {
  return get_field_impl(const_cast<sfb_context *>(cctx), wavefield, medium, which, shot, host, count);
}

SFB_API int sfb_set_field(sfb_context *ctx, int wavefield, int medium, int which, int shot, const float *host,
                          size_t count) {
  if (!ctx || !host) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    if (!medium_index_ok(medium) || which < 0 || which > 2) throw std::invalid_argument("bad field selector");
    WavefieldSet &W = ensure_wavefield(ctx, wavefield);
    const dev::MediumFields &f = W.f[medium];
    const size_t n = static_cast<size_t>(f.nglob) * f.nc;
    if (count < n) throw std::invalid_argument("field buffer too small");
    if (shot < 0 || shot >= ctx->P.nshots) throw std::invalid_argument("shot out of range");
    std::vector<real> tmp(n);
    for (int c = 0; c < f.nc; ++c)
      for (int g = 0; g < f.nglob; ++g) tmp[static_cast<size_t>(g) * f.nc + c] = host[static_cast<size_t>(c) * f.nglob + g];
    real *dst = which == 0 ? f.u : which == 1 ? f.v : f.a;
    const int S = ctx->P.nshots;
    ck(cudaStreamSynchronize(ctx->stream), "sync");
    if (n)
      ck(cudaMemcpy2D(dst + static_cast<size_t>(shot) * f.nc, static_cast<size_t>(S) * f.nc * sizeof(real),
                      tmp.data(), f.nc * sizeof(real), f.nc * sizeof(real), f.nglob, cudaMemcpyHostToDevice),
         "field h2d");
    return SFB_OK;
  });
}

SFB_API int sfb_write_seismograms(const sfb_context *cctx, int wavefield, int shot, const char *directory) {
  sfb_context *ctx = const_cast<sfb_context *>(cctx);
  if (!ctx || !directory) return SFB_E_INVALID;
  const Problem &P = ctx->P;
  const size_t per = static_cast<size_t>(P.max_sig_step()) * P.seismogram_types.size() * P.receivers.size() * 2;
  std::vector<float> buf(std::max<size_t>(per, 1));
  const int rc = sfb_get_seismograms(ctx, wavefield, shot, buf.data(), buf.size());
  if (rc) return rc;
  return guarded(ctx, [&]() {
    write_seismograms_ascii(P, buf.data(), static_cast<int>(P.seismogram_types.size()),
                            static_cast<int>(P.receivers.size()), P.max_sig_step(), directory);
    return SFB_OK;
  });
}

namespace {
// The forward state of `shot` after the steps run so far, with the boundary
// store, in the reference's layout (fresh: a new file with coordinates;
// otherwise one more step group).
void write_snapshot(sfb_context *ctx, int shot, const char *directory, bool fresh) {
  const Problem &P = ctx->P;
  if (shot < 0 || shot >= P.nshots) throw std::invalid_argument("shot out of range");
  WavefieldSet &F = ensure_wavefield(ctx, SFB_WAVEFIELD_FORWARD);
  if (F.step < 1) throw StateError("no forward step has run");
  ForwardSnapshot snap;
  snap.step = F.step;
  for (int m : kMedia) {
    const size_t n = static_cast<size_t>(P.asmb.nglob[m]) * P.asmb.ncomp(m);
    for (int w = 0; w < 3; ++w) {
      snap.field[m][w].assign(n, 0.f);
      if (n) {
        const int rc = sfb_get_field(ctx, SFB_WAVEFIELD_FORWARD, m, w, shot, snap.field[m][w].data(), n);
        if (rc) throw std::runtime_error(ctx->err);
      }
    }
  }
  // boundary store of this shot, slots by mesh element
  snap.slot.assign(P.asmb.nspec, -1);
  for (int e = 0; e < P.asmb.nspec; ++e) snap.slot[e] = ctx->h_stacey_slot.empty() ? -1 : ctx->h_stacey_slot[ctx->inv[e]];
  snap.nstacey = ctx->nstacey;
  const size_t per = static_cast<size_t>(P.nstep) * ctx->nstacey * P.asmb.ngll * P.asmb.ngll * 2;
  if (per && ctx->stacey_data.p) {
    snap.store.resize(per);
    ck(cudaStreamSynchronize(ctx->stream), "sync");
    copy_d2h(snap.store.data(), ctx->stacey_data.p + static_cast<size_t>(shot) * per, per, "store d2h");
  } else if (per) {
    throw StateError("the forward run kept no boundary store (save_boundary_values)");
  }
  write_forward_wavefield(P, directory, snap, fresh);
}
}  // namespace

SFB_API int sfb_write_wavefield(const sfb_context *cctx, int shot, const char *directory) {
  sfb_context *ctx = const_cast<sfb_context *>(cctx);
  if (!ctx || !directory) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    if (ensure_wavefield(ctx, SFB_WAVEFIELD_FORWARD).step != ctx->P.nstep)
      throw StateError("write the forward wavefield after the whole forward run");
    write_snapshot(ctx, shot, directory, true);
    return SFB_OK;
  });
}

SFB_API int sfb_write_wavefield_step(const sfb_context *cctx, int shot, const char *directory) {
  sfb_context *ctx = const_cast<sfb_context *>(cctx);
  if (!ctx || !directory) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    write_snapshot(ctx, shot, directory, false);
    return SFB_OK;
  });
}

SFB_API int sfb_read_wavefield(sfb_context *ctx, int shot, const char *directory) {
  if (!ctx || !directory) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    const Problem &P = ctx->P;
    if (shot < 0 || shot >= P.nshots) throw std::invalid_argument("shot out of range");
    WavefieldSet &F = ensure_wavefield(ctx, SFB_WAVEFIELD_FORWARD);
    if (!ctx->mass_ready) initialize_mass(ctx, P.dt);
    std::vector<int> slot(P.asmb.nspec, -1);
    for (int e = 0; e < P.asmb.nspec; ++e)
      if (!ctx->h_stacey_slot.empty()) slot[e] = ctx->h_stacey_slot[ctx->inv[e]];
    ForwardSnapshot snap = read_forward_wavefield(P, directory, slot, ctx->nstacey);
    for (int m : kMedia) {
      const size_t n = static_cast<size_t>(P.asmb.nglob[m]) * P.asmb.ncomp(m);
      if (!n) continue;
      for (int w = 0; w < 3; ++w) {
        const int rc = sfb_set_field(ctx, SFB_WAVEFIELD_FORWARD, m, w, shot, snap.field[m][w].data(), n);
        if (rc) throw std::runtime_error(ctx->err);
      }
    }
    const size_t per = static_cast<size_t>(P.nstep) * ctx->nstacey * P.asmb.ngll * P.asmb.ngll * 2;
    if (per) {
      if (!ctx->stacey_data.p) {
        const size_t total = per * P.nshots;
        ctx->stacey_data.alloc(total, &ctx->device_bytes);
      }
      copy_h2d(ctx->stacey_data.p + static_cast<size_t>(shot) * per, snap.store.data(), per, "store h2d");
    }
    F.step = P.nstep;  // the combined run starts from this state
    return SFB_OK;
  });
}

SFB_API int sfb_write_kernels(const sfb_context *cctx, const char *directory, int element_chunk) {
  sfb_context *ctx = const_cast<sfb_context *>(cctx);
  if (!ctx || !directory) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    const size_t nloc = ctx->P.asmb.nloc();
    std::vector<double> k[6];
    for (int q = 0; q < 6; ++q) {
      k[q].assign(nloc, 0.0);
      const int rc = sfb_get_kernels(ctx, q, k[q].data(), nloc);
      if (rc) throw std::runtime_error(ctx->err);
    }
    write_kernels(ctx->P, directory, k, element_chunk);
    return SFB_OK;
  });
}

SFB_API int sfb_write_properties(const sfb_context *cctx, const char *directory, int element_chunk) {
  sfb_context *ctx = const_cast<sfb_context *>(cctx);
  if (!ctx || !directory) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    write_properties(ctx->P, directory, element_chunk);
    return SFB_OK;
  });
}

void refresh_model(sfb_context *ctx);

SFB_API int sfb_read_properties(sfb_context *ctx, const char *directory, int element_chunk) {
  if (!ctx || !directory) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    read_properties(ctx->P, directory, element_chunk);
    refresh_model(ctx);
    return SFB_OK;
  });
}

// The reference's driver (src/execute.cpp): forward runs write seismograms
// and, when asked, the forward wavefield; combined runs read that wavefield,
// run the adjoint + backward loop and write the kernels.
namespace {
int execute_context(sfb_context *ctx);
}

SFB_API int sfb_execute(const char *parameter_file, const char *default_file) {
  sfb_context *ctx = nullptr;
  const int rc = sfb_create_from_yaml(parameter_file, default_file, &ctx);
  if (rc) return rc;
  return execute_context(ctx);
}

SFB_API int sfb_execute_text(const char *parameter_yaml, const char *default_yaml) {
  sfb_context *ctx = nullptr;
  const int rc = sfb_create_from_yaml_text(parameter_yaml, default_yaml, &ctx);
  if (rc) return rc;
  return execute_context(ctx);
}

namespace {
// Runs the simulation a parameter file describes and destroys the context.
int execute_context(sfb_context *ctx) {
  int rc = 0;
  std::unique_ptr<sfb_context, void (*)(sfb_context *)> own(ctx, sfb_destroy);
  // the context goes away on return: its message moves to sfb_last_error(NULL)
  auto failed = [&](int code) { return fail(nullptr, code, ctx->err); };
  const Problem &P = ctx->P;
  // databases.writer.properties: write the model files and stop
  // (execute.cpp:115-125); the reader side was applied when the context
  // was built
  if (P.property_mode == 1) {
    if ((rc = sfb_write_properties(ctx, P.property_dir.c_str(), 1))) return failed(rc);
    return SFB_OK;
  }
  if (P.simulation == 0) {
    // the forward run, in pieces between the wavefield writer's snapshots
    // (periodic_tasks/wavefield_writer.hpp: after step k when k is a
    // multiple of time_interval, and after the last step when
    // include_last_step), the coordinates with the first
    const int K = P.wavefield_dir.empty() ? 0 : P.wavefield_time_interval;
    int done = 0;
    bool fresh = true;
    while (done < P.nstep) {
      const int next = K > 0 ? std::min(P.nstep, (done / K + 1) * K) : P.nstep;
      if ((rc = sfb_run_forward(ctx, next - done, 1))) return failed(rc);
      done = next;
      const bool periodic = K > 0 && done % K == 0;
      const bool last = done == P.nstep && P.wavefield_include_last_step;
      if (!P.wavefield_dir.empty() && (periodic || last)) {
        // the first snapshot starts the file (with the coordinates)
        rc = guarded(ctx, [&]() {
          write_snapshot(ctx, 0, P.wavefield_dir.c_str(), fresh);
          return SFB_OK;
        });
        if (rc) return failed(rc);
        fresh = false;
      }
    }
    if (P.write_seismograms)
      for (int s = 0; s < P.nshots; ++s)
        if ((rc = sfb_write_seismograms(ctx, SFB_WAVEFIELD_FORWARD, s, P.seismogram_dir.c_str()))) return failed(rc);
  } else {
    if (P.wavefield_dir.empty()) return fail(nullptr, SFB_E_INVALID, "combined run without a wavefield reader directory");
    if ((rc = sfb_read_wavefield(ctx, 0, P.wavefield_dir.c_str()))) return failed(rc);
    if ((rc = sfb_run_combined(ctx, P.nstep, 1))) return failed(rc);
    if (!P.kernel_dir.empty())
      if ((rc = sfb_write_kernels(ctx, P.kernel_dir.c_str(), 1))) return failed(rc);
    if (P.write_seismograms)
      if ((rc = sfb_write_seismograms(ctx, SFB_WAVEFIELD_BACKWARD, 0, P.seismogram_dir.c_str()))) return failed(rc);
  }
  return SFB_OK;
}
}  // namespace

SFB_API int sfb_set_source_time_function(sfb_context *ctx, int isource, const float *host, size_t count) {
  if (!ctx || !host) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    Problem &P = ctx->P;
    if (isource < 0 || isource >= static_cast<int>(P.v_src_ispec.size())) throw std::invalid_argument("source index out of range");
    const size_t n = static_cast<size_t>(P.nstep) * 2;
    if (count < n) throw std::invalid_argument("source time function buffer too small");
    std::copy(host, host + n, P.v_src_stf.begin() + static_cast<size_t>(isource) * n);
    if (ctx->on_device) {
      if constexpr (std::is_same<real, float>::value) {
        ck(cudaMemcpyAsync(ctx->src_stf.p + static_cast<size_t>(isource) * n, host, n * sizeof(float),
                           cudaMemcpyHostToDevice, ctx->stream), "stf h2d");
      } else {
        ck(cudaStreamSynchronize(ctx->stream), "sync");
        copy_h2d(ctx->src_stf.p + static_cast<size_t>(isource) * n, host, n, "stf h2d");
      }
    }
    return SFB_OK;
  });
}

SFB_API int sfb_get_stream(const sfb_context *cctx, void **stream) {
  sfb_context *ctx = const_cast<sfb_context *>(cctx);
  if (!ctx || !stream) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    ensure_device(ctx);
    *stream = static_cast<void *>(ctx->stream);
    return SFB_OK;
  });
}

SFB_API int sfb_time_stiffness(sfb_context *ctx, int medium, int reps, double *mean_ms) {
  if (!ctx || !mean_ms || reps < 1) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    if (!medium_index_ok(medium)) throw std::invalid_argument("unsupported medium tag");
    WavefieldSet &W = ensure_wavefield(ctx, SFB_WAVEFIELD_FORWARD);
    const int n = ctx->P.asmb.ngll;
    dev::StaceyStore ss{};
    cudaEvent_t e0, e1;
    ck(cudaEventCreate(&e0), "event");
    ck(cudaEventCreate(&e1), "event");
    ck(cudaEventRecord(e0, ctx->stream), "event record");
    for (int r = 0; r < reps; ++r)
      dev::launch_stiffness(medium, n, ctx->st, W.f[medium], ctx->P.nshots, ss, &W.ctrl.p->istep, ctx->stream,
                            nullptr, nullptr, ctx->shots_variant[medium]);
    ck(cudaEventRecord(e1, ctx->stream), "event record");
    ck(cudaEventSynchronize(e1), "event sync");
    float ms = 0.f;
    ck(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ctx->launches += reps;
    *mean_ms = ms / reps;
    // the repeated launches accumulated into the force array: clear it
    const dev::MediumFields &f = W.f[medium];
    const size_t ld = static_cast<size_t>(f.nglob + (f.nglob & 1)) * f.nc;
    if (ld) ck(cudaMemsetAsync(f.a, 0, ld * ctx->P.nshots * sizeof(real), ctx->stream), "clear force");
    ck(cudaStreamSynchronize(ctx->stream), "sync");
    return SFB_OK;
  });
}


SFB_API int sfb_run_combined(sfb_context *ctx, int nstep, int use_graph) {
  if (!ctx) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    if (nstep != ctx->P.nstep) throw std::invalid_argument("the combined run covers the whole forward run (nstep)");
    run_combined_fused(ctx, use_graph);
    enqueue_nonfinite(ctx, ctx->wf[SFB_WAVEFIELD_ADJOINT]);
    enqueue_nonfinite(ctx, ctx->wf[SFB_WAVEFIELD_BACKWARD]);
    dev::launch_nonfinite_check(ctx->kern.p, ctx->kern.n, ctx->dflag.p, ctx->stream);
    ck(cudaStreamSynchronize(ctx->stream), "combined run");
    check_device_flag(ctx);
    return SFB_OK;
  });
}

SFB_API int sfb_frechet_compute_derivatives(sfb_context *ctx, double dt) {
  if (!ctx) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    WavefieldSet &A = ensure_wavefield(ctx, SFB_WAVEFIELD_ADJOINT);
    WavefieldSet &B = ensure_wavefield(ctx, SFB_WAVEFIELD_BACKWARD);
    const size_t nk = ctx->P.asmb.nloc() * 3;
    if (!ctx->kern.p) {
      ctx->kern.alloc(nk, &ctx->device_bytes);
    }
    poll_device_flag(ctx);
    for (int m : {dev::MED_PSV, dev::MED_AC})
      dev::launch_frechet(m, ctx->P.asmb.ngll, ctx->st, A.f[m], B.f[m], ctx->P.nshots, static_cast<real>(dt),
                          ctx->kern.p, 0, ctx->stream);
    if (ctx->stacey_kernels) {
      if (!ctx->kern_b.p) ctx->kern_b.alloc(ctx->P.asmb.nloc() * 2, &ctx->device_bytes);
      dev::launch_stacey_frechet(ctx->P.asmb.ngll, ctx->st, A.f[dev::MED_PSV], B.f[dev::MED_PSV], ctx->P.nshots,
                                 static_cast<real>(dt), real(0), ctx->kern_b.p, ctx->stream);
    }
    ck(cudaGetLastError(), "frechet");
    note_device_flag(ctx);
    return SFB_OK;
  });
}

SFB_API int sfb_set_adjoint_sources(sfb_context *ctx, int shot, const float *host, size_t count) {
  if (!ctx || !host) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    const Problem &P = ctx->P;
    if (shot < 0 || shot >= P.nshots) throw std::invalid_argument("shot out of range");
    const int nrec = static_cast<int>(P.receivers.size());
    const size_t n = static_cast<size_t>(P.nstep) * nrec * 2;
    if (count < n) throw std::invalid_argument("adjoint source buffer too small ([nstep][nreceivers][2])");
    if (!P.located_adjoint.empty()) throw StateError("the adjoint sources come from the sources file");
    ensure_adjoint_sources(ctx);
    // device layout [source = shot * nrec + r][nstep][2]
    std::vector<float> tmp(n);
    for (int t = 0; t < P.nstep; ++t)
      for (int r = 0; r < nrec; ++r)
        for (int cc = 0; cc < 2; ++cc)
          tmp[(static_cast<size_t>(r) * P.nstep + t) * 2 + cc] = host[(static_cast<size_t>(t) * nrec + r) * 2 + cc];
    ck(cudaStreamSynchronize(ctx->stream), "sync");
    copy_h2d(ctx->adj_stf.p + static_cast<size_t>(shot) * n, tmp.data(), n, "adjoint stf h2d");
    return SFB_OK;
  });
}

SFB_API int sfb_get_kernels(const sfb_context *cctx, int which, double *host, size_t count) {
  sfb_context *ctx = const_cast<sfb_context *>(cctx);
  if (!ctx || !host) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    if (which < 0 || which > 7) throw std::invalid_argument("kernel selector must be in [0, 7]");
    if (which >= 6) {
      // Stacey-traction derivatives, dchi/d(rho vp) and dchi/d(rho vs)
      if (!ctx->kern_b.p) throw StateError("no Stacey-traction kernels have been accumulated (sfb_set_stacey_kernels)");
      const Assembly &a = ctx->P.asmb;
      const size_t nloc = a.nloc();
      const int nn = a.ngll * a.ngll;
      if (count < nloc) throw std::invalid_argument("kernel buffer too small ([nspec][ngll][ngll])");
      std::vector<double> k(nloc * 2);
      ck(cudaStreamSynchronize(ctx->stream), "sync");
      ck(cudaMemcpy(k.data(), ctx->kern_b.p, k.size() * sizeof(double), cudaMemcpyDeviceToHost), "kernels d2h");
      for (int e = 0; e < a.nspec; ++e)
        for (int q = 0; q < nn; ++q)
          host[static_cast<size_t>(e) * nn + q] = k[(static_cast<size_t>(ctx->inv[e]) * nn + q) * 2 + (which - 6)];
      return SFB_OK;
    }
    const Assembly &a = ctx->P.asmb;
    const size_t nloc = a.nloc();
    const int nn = a.ngll * a.ngll;
    if (count < nloc) throw std::invalid_argument("kernel buffer too small ([nspec][ngll][ngll])");
    if (!ctx->kern.p) throw StateError("no kernels have been accumulated");
    std::vector<double> k(nloc * 3);
    ck(cudaStreamSynchronize(ctx->stream), "sync");
    ck(cudaMemcpy(k.data(), ctx->kern.p, k.size() * sizeof(double), cudaMemcpyDeviceToHost), "kernels d2h");
    for (int e = 0; e < a.nspec; ++e) {
      const int d = ctx->inv[e];
      for (int q = 0; q < nn; ++q) {
        const size_t p = static_cast<size_t>(e) * nn + q, pd = static_cast<size_t>(d) * nn + q;
        const double k0 = k[pd * 3], k1 = k[pd * 3 + 1], k2 = k[pd * 3 + 2];
        double v = 0.0;
        if (a.medium[e] == MEDIUM_ACOUSTIC) {
          // rho, kappa; rhop = sum over steps of rho_kl * kappa_kl, alpha =
          // 2 kappa (point/kernels.hpp:189-192)
          v = which == 0 ? k0 : which == 2 ? k1 : which == 3 ? k2 : which == 4 ? 2.0 * k1 : 0.0;
        } else {
          // derived kernels (frechet_derivative.hpp:117-135), linear in the
          // primaries at fixed model: kappa' = lambda + 2 mu - mu
          const float mu = a.mu[p];
          const float kap = a.kappa[p] + static_cast<float>(4.0 / 3.0) * mu - mu;
          const double r = static_cast<double>(mu) / kap;
          switch (which) {
          case 0: v = k0; break;
          case 1: v = k1; break;
          case 2: v = k2; break;
          case 3: v = k0 + k2 + k1; break;
          case 4: v = 2.0 * (1.0 + 4.0 / 3.0 * r) * k2; break;
          case 5: v = 2.0 * (k1 - 4.0 / 3.0 * r * k2); break;
          }
        }
        host[p] = v;
      }
    }
    return SFB_OK;
  });
}

SFB_API int sfb_load_backward_from_forward(sfb_context *ctx) {
  if (!ctx) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    WavefieldSet &F = ensure_wavefield(ctx, SFB_WAVEFIELD_FORWARD);
    WavefieldSet &B = ensure_wavefield(ctx, SFB_WAVEFIELD_BACKWARD);
    copy_fields(ctx, B, F);
    ck(cudaStreamSynchronize(ctx->stream), "copy");
    return SFB_OK;
  });
}

SFB_API int sfb_copy_forward_to_backward(const sfb_context *csrc, sfb_context *dst) {
  sfb_context *src = const_cast<sfb_context *>(csrc);
  if (!src || !dst) return SFB_E_INVALID;
  return guarded(dst, [&]() {
    if (src->P.asmb.nloc() != dst->P.asmb.nloc() || src->P.nstep != dst->P.nstep || src->P.nshots != dst->P.nshots)
      throw std::invalid_argument("the two contexts do not describe the same problem");
    WavefieldSet &S = ensure_wavefield(src, SFB_WAVEFIELD_FORWARD);
    WavefieldSet &D = ensure_wavefield(dst, SFB_WAVEFIELD_FORWARD);
    ck(cudaStreamSynchronize(src->stream), "sync src");
    copy_fields(dst, D, S);
    if (src->stacey_data.p) {
      ensure_store(dst);
      ck(cudaMemcpyAsync(dst->stacey_data.p, src->stacey_data.p, src->stacey_data.n * sizeof(real),
                         cudaMemcpyDeviceToDevice, dst->stream),
         "copy store");
    }
    ck(cudaStreamSynchronize(dst->stream), "sync dst");
    D.step = S.step;
    return SFB_OK;
  });
}

// After the assembly's model changed on the host: refresh the material words
// of the device's static blocks and per-point arrays; the mass matrix is
// rebuilt on the next run.
void refresh_model(sfb_context *ctx) {
  Assembly &a = ctx->P.asmb;
  const size_t nloc = a.nloc();
  const int nn = a.ngll * a.ngll;
  if (ctx->on_device) {
    // the copies below run on the legacy stream, which does not wait for
    // the context's stream: let launches that read the model finish first
    ck(cudaStreamSynchronize(ctx->stream), "sync");
    // refresh the material words of the packed and SoA device arrays
    std::vector<float> m0(nloc), m1(nloc), m2(nloc);
    std::vector<real> pack(nloc * dev::kPackFields);
    ck(cudaMemcpy(pack.data(), ctx->pack.p, pack.size() * sizeof(real), cudaMemcpyDeviceToHost), "pack d2h");
    for (int d = 0; d < a.nspec; ++d) {
      const int e = ctx->perm[d];
      const int m = a.medium[e];
      for (int k = 0; k < nn; ++k) {
        const size_t p = static_cast<size_t>(e) * nn + k, q = static_cast<size_t>(d) * nn + k;
        if (m == MEDIUM_ELASTIC_PSV) { m0[q] = a.kappa[p]; m1[q] = a.mu[p]; m2[q] = a.rho[p]; }
        else if (m == MEDIUM_ELASTIC_SH) { m0[q] = a.mu[p]; m1[q] = a.rho[p]; m2[q] = 0.f; }
        else { m0[q] = a.rho_inverse[p]; m1[q] = a.kappa[p]; m2[q] = 0.f; }
        real *blk = &pack[static_cast<size_t>(d) * dev::kPackFields * nn];
        blk[6 * nn + k] = m0[q];
        blk[7 * nn + k] = m1[q];
      }
    }
    ck(cudaMemcpy(ctx->pack.p, pack.data(), pack.size() * sizeof(real), cudaMemcpyHostToDevice), "pack h2d");
    if (ctx->pack_aff.p) {
      // the material words of the compact block
      const int words = dev::affine_chunk_words(ctx->P.asmb.ngll);
      const int E = dev::kAffineChunk;
      std::vector<float> aff(ctx->pack_aff.n);
      ck(cudaMemcpy(aff.data(), ctx->pack_aff.p, aff.size() * sizeof(float), cudaMemcpyDeviceToHost), "aff d2h");
      for (int m : kMedia) {
        if (!ctx->st.affine[m]) continue;
        for (int i = 0; i < ctx->med_count[m]; ++i) {
          const int d = ctx->med_begin[m] + i;
          float *chunk = &aff[static_cast<size_t>(ctx->st.aff_chunk0[m] + i / E) * words];
          const int el = i % E;
          for (int k = 0; k < nn; ++k) {
            const size_t q = static_cast<size_t>(d) * nn + k;
            chunk[E * nn + el * nn + k] = m0[q];
            chunk[2 * E * nn + el * nn + k] = m1[q];
          }
        }
      }
      ck(cudaMemcpy(ctx->pack_aff.p, aff.data(), aff.size() * sizeof(float), cudaMemcpyHostToDevice), "aff h2d");
    }
    copy_h2d(ctx->mat0_all.p, m0.data(), nloc, "mat0");
    copy_h2d(ctx->mat1_all.p, m1.data(), nloc, "mat1");
    copy_h2d(ctx->mat2_all.p, m2.data(), nloc, "mat2");
    ctx->taps_ready = false;  // pressure taps carry the material
    // captured graphs hold the old tap buffers
    ctx->drop_forward_graphs();
    ctx->drop_combined_graphs();
  }
  ctx->mass_ready = false;
}

SFB_API int sfb_set_model(sfb_context *ctx, const float *rho, const float *vp, const float *vs, size_t count) {
  if (!ctx || !rho || !vp || !vs) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    Assembly &a = ctx->P.asmb;
    const size_t nloc = a.nloc();
    const int nn = a.ngll * a.ngll;
    if (count < nloc) throw std::invalid_argument("model arrays too small ([nspec][ngll][ngll])");
    for (size_t p = 0; p < nloc; ++p) {
      const int e = static_cast<int>(p / nn);
      const double r = rho[p], cp = vp[p], cs = vs[p];
      if (a.medium[e] == MEDIUM_ACOUSTIC) {
        a.kappa[p] = static_cast<float>(r * cp * cp);
        a.rho_inverse[p] = 1.0f / static_cast<float>(r);
        a.rho[p] = static_cast<float>(r);
      } else {
        a.kappa[p] = static_cast<float>(r * (cp * cp - (4.0 / 3.0) * cs * cs));
        a.mu[p] = static_cast<float>(r * cs * cs);
        a.rho[p] = static_cast<float>(r);
        a.rho_inverse[p] = 1.0f / static_cast<float>(r);
      }
    }
    refresh_model(ctx);
    return SFB_OK;
  });
}

SFB_API int sfb_reset(sfb_context *ctx) {
  if (!ctx) return SFB_E_INVALID;
  return guarded(ctx, [&]() {
    if (!ctx->on_device) return SFB_OK;
    for (int w = 0; w < 3; ++w) {
      WavefieldSet &W = ctx->wf[w];
      if (!W.allocated) continue;
      zero_fields(ctx, W);
      for (int m : kMedia) {
        if (W.cu[m].p) ck(cudaMemsetAsync(W.cu[m].p, 0, W.cu[m].n * sizeof(real), ctx->stream), "zero cu");
        if (W.cv[m].p) ck(cudaMemsetAsync(W.cv[m].p, 0, W.cv[m].n * sizeof(real), ctx->stream), "zero cv");
      }
      W.step = 0;
    }
    if (ctx->stacey_data.p) ck(cudaMemsetAsync(ctx->stacey_data.p, 0, ctx->stacey_data.n * sizeof(real), ctx->stream), "zero store");
    if (ctx->kern.p) ck(cudaMemsetAsync(ctx->kern.p, 0, ctx->kern.n * sizeof(double), ctx->stream), "zero kernels");
    ck(cudaStreamSynchronize(ctx->stream), "reset");
    return SFB_OK;
  });
}

