// Host side of libbtam.so: the C ABI declared in include/btam.h.
//
// Owns device memory per system (state, periodic images, neighbour lists,
// moments, results) and one CUDA stream per system.  No torch, no host
// fallback: every evaluation runs the kernels of adp_kernels.cu and
// topo_kernels.cu on the current device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/btam.h"
#include "adp_core.cuh"
#include "linalg.hpp"
#include "adp_kernels.cuh"
#include "solvers.cuh"
#include "tables_io.hpp"
#include "topo_kernels.cuh"
#include "internal.cuh"

using namespace btam;

namespace {

constexpr double kKB = 8.617332478E-5;  // k_B [eV/K] (Macros.hpp:849)

// Packs row-major q, sigma and x of real sites into the device layout.
__global__ void pack_state_kernel(int n, const double *q, const double *sigma,
                                  const double *x, double4 *pos, double2 *xb,
                                  const int *reject = nullptr) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || (reject && *reject)) return;  // a rejected update leaves the state
  double4 p = pos[i];
  double2 b = xb[i];
  if (q) {
    p.x = q[3 * i];
    p.y = q[3 * i + 1];
    p.z = q[3 * i + 2];
  }
  if (sigma) p.w = sigma[i];
  if (x) b.x = x[i];
  pos[i] = p;
  xb[i] = b;
}

// Validation of a staged state update (the checks of validate_state, on the
// device): bit 0 a non-finite or non-positive value, bit 1 a non-H site with
// 0 < x < min_occupancy, bit 2 a site outside the cell along a periodic axis.
__global__ void validate_stage_kernel(int n, const double *q, const double *sigma,
                                      const double *x, const int *code, GhostBox b,
                                      int *flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int f = 0;
  if (q) {
    const double q0 = q[3 * i], q1 = q[3 * i + 1], q2 = q[3 * i + 2];
    if (!(isfinite(q0) && isfinite(q1) && isfinite(q2))) f |= 1;
    else
      for (int a = 0; a < 3; ++a) {
        if (!b.periodic[a]) continue;
        if (b.ortho) {
          const double v = a == 0 ? q0 : (a == 1 ? q1 : q2);
          if (!(v >= b.lo[a] && v < b.hi[a])) f |= 4;
        } else {
          const double d0 = q0 - b.origin[0], d1 = q1 - b.origin[1], d2 = q2 - b.origin[2];
          const double sa = d0 * b.B[a][0] + d1 * b.B[a][1] + d2 * b.B[a][2];
          if (!(sa >= -1e-9 && sa < 1.0 + 1e-9)) f |= 4;
        }
      }
  }
  if (sigma && !(isfinite(sigma[i]) && sigma[i] > 0.0)) f |= 1;
  if (x) {
    const double v = x[i];
    if (!isfinite(v) || v < 0.0) f |= 1;
    else if (code[i] == 0 && v > 0.0 && v < BTAM_MIN_OCCUPANCY) f |= 2;
  }
  if (f) atomicOr(flags, f);
}

// FMA throughput probe: kProbeChains independent dependency chains per
// thread keep the FMA pipe full; the result is stored so nothing is elided.
constexpr int kProbeChains = 8;
template <class T> __global__ void fma_probe_kernel(long long iters, T *sink) {
  T v[kProbeChains];
  const T a = (T)0.999999, b = (T)1e-7;
  for (int c = 0; c < kProbeChains; ++c) v[c] = (T)(threadIdx.x + c);
  for (long long it = 0; it < iters; ++it)
#pragma unroll
    for (int c = 0; c < kProbeChains; ++c) v[c] = fma(v[c], a, b);
  T s = 0;
  for (int c = 0; c < kProbeChains; ++c) s += v[c];
  sink[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// Random-gather throughput probe: every thread draws segment indices with a
// xorshift generator and loads whole 32-byte spline records (u and w of a
// pair kind at a segment) from the FP32 radial tables, the access pattern of
// the evaluation kernels' quadrature points.
__global__ void gather_probe_kernel(const float *rec, int n_rec, long long iters, float *sink) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned st = 0x9E3779B9u * (unsigned)(tid + 1);
  float acc = 0.f;
  for (long long it = 0; it < iters; ++it) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      st ^= st << 13;
      st ^= st >> 17;
      st ^= st << 5;
      const int m = (int)(((unsigned long long)st * (unsigned)n_rec) >> 32);
      float v[8];
      ld8(rec + 8 * (size_t)m, v);
      acc += v[0] + v[7];
    }
  }
  sink[tid] = acc;
}

__global__ void spline_eval_kernel(SplineView<double> s, int n, const double *r, double *v,
                                   double *dv) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double a, b;
  spline_vd(s, r[i], a, b);
  v[i] = a;
  dv[i] = b;
}

}  // namespace

static int build_list(btam_system *s, int n_all, int n_query, double rc, int maxn, int filter,
                      int allow_empty, int *&offs, int &q_cap, int *&idx, long long &idx_cap,
                      int &total);

namespace {

// Reciprocal rows and rc-shell widths of a cell (rows = lattice vectors).
// Same arithmetic as the oracle's image rule (oracle/btam_oracle.cpp).
int make_box(const double *origin, const double *cell, const int *periodic, double rc,
             GhostBox &b) {
  memset(&b, 0, sizeof(b));
  double A[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) A[r][c] = cell[3 * r + c];
  b.ortho = (cell[1] == 0 && cell[2] == 0 && cell[3] == 0 && cell[5] == 0 &&
             cell[6] == 0 && cell[7] == 0) ? 1 : 0;
  double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
               A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
               A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
  bool any = periodic[0] || periodic[1] || periodic[2];
  if (det == 0.0 && any) return BTAM_ERR_BOX_TOO_SMALL;
  for (int a = 0; a < 3; ++a) {
    const double *p = A[(a + 1) % 3], *s = A[(a + 2) % 3];
    if (det != 0.0) {
      b.B[a][0] = (p[1] * s[2] - p[2] * s[1]) / det;
      b.B[a][1] = (p[2] * s[0] - p[0] * s[2]) / det;
      b.B[a][2] = (p[0] * s[1] - p[1] * s[0]) / det;
    }
  }
  for (int a = 0; a < 3; ++a) {
    for (int c = 0; c < 3; ++c) b.A[a][c] = A[a][c];
    double bn = std::sqrt(b.B[a][0] * b.B[a][0] + b.B[a][1] * b.B[a][1] + b.B[a][2] * b.B[a][2]);
    if (periodic[a]) {
      if (!(bn > 0.0) || 1.0 / bn < 2.0 * rc) return BTAM_ERR_BOX_TOO_SMALL;
    }
    b.w[a] = rc * bn;
    b.lo[a] = origin[a];
    b.hi[a] = origin[a] + A[a][a];
    b.origin[a] = origin[a];
    b.periodic[a] = periodic[a] ? 1 : 0;
  }
  b.rc = rc;
  return BTAM_OK;
}

int validate_state(const btam_system *s, int n, const double *q, const double *sigma,
                   const double *x, const int *code) {
  for (int i = 0; i < n; ++i) {
    if (q)
      for (int a = 0; a < 3; ++a)
        if (!std::isfinite(q[3 * i + a])) return BTAM_ERR_NONFINITE;
    if (sigma && !(std::isfinite(sigma[i]) && sigma[i] > 0.0)) return BTAM_ERR_NONFINITE;
    if (x) {
      if (!std::isfinite(x[i]) || x[i] < 0.0) return BTAM_ERR_NONFINITE;
      if (code && code[i] == 0 && x[i] > 0.0 && x[i] < BTAM_MIN_OCCUPANCY)
        return BTAM_ERR_OCCUPANCY;
    }
    if (q && s->any_periodic) {
      const GhostBox &b = s->box;
      for (int a = 0; a < 3; ++a) {
        if (!b.periodic[a]) continue;
        if (b.ortho) {
          double v = q[3 * i + a];
          if (!(v >= b.lo[a] && v < b.hi[a])) return BTAM_ERR_OUT_OF_BOX;
        } else {
          double d0 = q[3 * i] - b.origin[0], d1 = q[3 * i + 1] - b.origin[1],
                 d2 = q[3 * i + 2] - b.origin[2];
          double sa = d0 * b.B[a][0] + d1 * b.B[a][1] + d2 * b.B[a][2];
          if (!(sa >= -1e-9 && sa < 1.0 + 1e-9)) return BTAM_ERR_OUT_OF_BOX;
        }
      }
    }
  }
  return BTAM_OK;
}

int ensure_sites(btam_system *s, int n_all) {
  if (n_all <= s->cap_all) return BTAM_OK;
  int cap = n_all + n_all / 4 + 64;
  double4 *pos = nullptr;
  double2 *xb = nullptr;
  int *code = nullptr, *owner = nullptr;
  BTAM_TRY(dalloc(pos, s->st, cap));
  BTAM_TRY(dalloc(xb, s->st, cap));
  BTAM_TRY(dalloc(code, s->st, cap));
  BTAM_TRY(dalloc(owner, s->st, cap));
  if (s->pos) {
    BTAM_TRY(cudaMemcpyAsync(pos, s->pos, (size_t)s->n_real * sizeof(double4),
                             cudaMemcpyDeviceToDevice, s->st));
    BTAM_TRY(cudaMemcpyAsync(xb, s->xb, (size_t)s->n_real * sizeof(double2),
                             cudaMemcpyDeviceToDevice, s->st));
    BTAM_TRY(cudaMemcpyAsync(code, s->code, (size_t)s->n_real * sizeof(int),
                             cudaMemcpyDeviceToDevice, s->st));
    BTAM_TRY(cudaMemcpyAsync(owner, s->owner, (size_t)s->n_real * sizeof(int),
                             cudaMemcpyDeviceToDevice, s->st));
    BTAM_TRY(cudaStreamSynchronize(s->st));
  }
  dfree(s->pos, s->st);
  dfree(s->xb, s->st);
  dfree(s->code, s->st);
  dfree(s->owner, s->st);
  s->pos = pos;
  s->xb = xb;
  s->code = code;
  s->owner = owner;
  // packed neighbour rows of the FP32C kernels (rewritten by every pass 1)
  BTAM_TRY(dalloc(s->s32, s->st, cap));
  BTAM_TRY(dalloc(s->sb, s->st, cap));
  BTAM_TRY(dalloc(s->s64, s->st, cap));
  s->cap_all = cap;
  return BTAM_OK;
}

template <class R> EvalArgs<R> eval_args(btam_system *s, R *mom, const RadialView<R> &T) {
  EvalArgs<R> a;
  a.n_real = s->n_real;
  a.n_all = s->n_real + s->n_ghost;
  if (sizeof(R) == 4) {
    a.s32 = s->s32;
    a.sb = s->sb;
  } else {
    a.s64 = s->s64;
  }
  a.pos = s->pos;
  a.xb = s->xb;
  a.code = s->code;
  a.owner = s->owner;
  a.gamma = s->gamma;
  a.offs = s->offs;
  a.idx = s->idx;
  a.T = T;
  a.emb[0] = s->T->v64.t[T_F_MG];
  a.emb[1] = s->T->v64.t[T_F_H];
  a.mass[0] = s->T->host.mass_mg;
  a.mass[1] = s->T->host.mass_h;
  a.mom = mom;
  a.rho = s->rho;
  a.V0 = s->V0;
  a.S0 = s->S0;
  a.selfx = s->selfx;
  a.Rq = s->Rq;
  a.Rs = s->Rs;
  a.Rx = s->Rx;
  a.err = s->err;
  a.rev = s->rev;
  a.own_p = s->own_p;
  a.own_u = s->own_u;
  a.n_own = s->n_own;
  a.pbuf = reinterpret_cast<R *>(s->pbuf);
  a.slot_own = s->slot_own;
  if (s->pbuf) {
    a.pgx = a.pbuf + pbuf_gx_offset(s->n_pairs);
    a.prec1 = a.pbuf + pbuf_prec1_offset(s->n_pairs);
    a.prec2 = a.prec1 + prec2_offset(s->n_own);
  }
  return a;
}

// Buffer of the undirected kernels, allocated only when an undirected variant
// is in use: the pass-2 slot records of the real sites' lists (5 values of R
// per slot), then the pair-rule records of the owned pairs (prec1, prec2);
// layout in pbuf_values and its helpers.
int ensure_pbuf(btam_system *s, size_t elem) {
  if (elem < s->pbuf_elem) elem = s->pbuf_elem;
  const size_t need =
      pbuf_values(s->n_pairs > 0 ? s->n_pairs : 1, s->n_own) * elem;
  s->pbuf_elem = elem;
  if (need <= s->pbuf_bytes) return BTAM_OK;
  BTAM_TRY(dalloc(s->pbuf, s->st, need));
  s->pbuf_bytes = need;
  return BTAM_OK;
}

// the pipelined state evaluations' buffers, events and copy streams
// (defined beside btam_mf_eval_state_async)
void release_state_slots(btam_system *s);

}  // namespace

// One evaluation enqueued on the system's stream.  x_only: the occupancy
// gradients alone with the undirected variants (EvalArgs::x_only); recs_ready:
// the pair-rule kernel's four pass-1 sums are still those of the current
// positions and widths (an earlier x_only evaluation in the same run of
// master-equation steps made them), so pass 1 skips that kernel.  A served
// job's evaluation goes to the server's batcher in full.
static int enqueue_eval(btam_system *s, int precision, bool x_only, bool recs_ready) {
  if (!s) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  if (precision != BTAM_FP64 && precision != BTAM_FP32C) return BTAM_ERR_ARG;
  if (s->batcher) return batcher_eval(s, precision);  // a served job: one shared launch
  const size_t nm = (size_t)s->n_real * kMomStride;
  if (precision == BTAM_FP64) {
    if (!s->mom64) BTAM_TRY(dalloc(s->mom64, s->st, nm));
    EvalArgs<double> a = eval_args<double>(s, s->mom64, s->T->r64);
    a.x_only = x_only;
    a.recs_ready = x_only && recs_ready;
    BTAM_TRY(launch_pass1(a, s->st, s->variant1[0], s->variant2[0]));
    BTAM_TRY(launch_pass2(a, s->st, s->variant2[0]));
  } else {
    if (!s->mom32) BTAM_TRY(dalloc(s->mom32, s->st, nm));
    EvalArgs<float> a = eval_args<float>(s, s->mom32, s->T->r32);
    a.x_only = x_only;
    a.recs_ready = x_only && recs_ready;
    BTAM_TRY(launch_pass1(a, s->st, s->variant1[1], s->variant2[1]));
    BTAM_TRY(launch_pass2(a, s->st, s->variant2[1]));
  }
  BTAM_TRY(launch_totals(s->n_real, s->V0, s->S0, s->Rq, s->Rs, s->Rx, s->totals, s->totals + 4,
                          s->st));
  return BTAM_OK;
}

// Table views for the allocation-free entry point (noalloc.cu).
namespace btam {
// One pool per device, created on first use and kept for the life of the
// process; its release threshold keeps freed blocks cached, so a stream of
// systems of similar sizes reuses memory without returning it to the driver.
cudaMemPool_t device_pool() {
  static std::mutex mu;
  static std::vector<cudaMemPool_t> pools;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if ((int)pools.size() <= dev) pools.resize(dev + 1, nullptr);
  if (!pools[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
    unsigned long long keep = ~0ull;
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[dev] = p;
  }
  return pools[dev];
}

const TablesView<double> &tables_view64(const btam_tables *t) { return t->v64; }
const TablesView<float> &tables_view32(const btam_tables *t) { return t->v32; }
const RadialView<double> &radial_view64(const btam_tables *t) { return t->r64; }
const RadialView<float> &radial_view32(const btam_tables *t) { return t->r32; }
double tables_mass(const btam_tables *t, int code) {
  return code == 1 ? t->host.mass_h : t->host.mass_mg;
}
}  // namespace btam

int make_box_for(const double *origin, const double *cell, const int *periodic, GhostBox &b) {
  return make_box(origin, cell, periodic, BTAM_R_CUTOFF, b);
}

extern "C" {

const char *btam_status_string(int st) {
  switch (st) {
  case BTAM_OK: return "ok";
  case BTAM_ERR_ARG: return "bad argument";
  case BTAM_ERR_IO: return "table file missing or malformed";
  case BTAM_ERR_NEIGHBOR_OVERFLOW: return "more than maxneigh neighbours";
  case BTAM_ERR_NO_NEIGHBORS: return "site without neighbours";
  case BTAM_ERR_BOX_TOO_SMALL: return "periodic cell thinner than 2 rc";
  case BTAM_ERR_NONFINITE: return "non-finite value";
  case BTAM_ERR_OOM: return "device out of memory";
  case BTAM_ERR_CUDA: return "CUDA error";
  case BTAM_ERR_GHOST_OVERFLOW: return "periodic images exceed capacity";
  case BTAM_ERR_OCCUPANCY: return "non-H site with 0 < x < min_occupancy";
  case BTAM_ERR_SPECIES: return "species other than H or Mg";
  case BTAM_ERR_TIMEOUT: return "bounded device wait gave up";
  case BTAM_ERR_NOT_BUILT: return "neighbour lists not built";
  case BTAM_ERR_OUT_OF_BOX: return "site outside the periodic cell";
  case BTAM_ERR_TOO_LARGE: return "more sites or pairs than the entry point holds";
  }
  return "unknown status";
}

int btam_version(void) { return 100; }

const char *btam_last_cuda_error(void) {
  const cudaError_t e = last_cuda_error();
  return e == cudaSuccess ? "" : cudaGetErrorName(e);
}

int btam_pool_usage(long long *used, long long *reserved) {
  if (!used || !reserved) return BTAM_ERR_ARG;
  cudaMemPool_t pool = btam::device_pool();
  if (!pool) return BTAM_ERR_CUDA;
  unsigned long long u = 0, r = 0;
  BTAM_TRY(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &u));
  BTAM_TRY(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &r));
  *used = (long long)u;
  *reserved = (long long)r;
  return BTAM_OK;
}

int btam_tables_load(const char *dir, btam_tables **out) {
  if (!dir || !out) return BTAM_ERR_ARG;
  *out = nullptr;
  btam_tables *t = new btam_tables();
  if (load_host_tables(dir, t->host)) {
    delete t;
    return BTAM_ERR_IO;
  }
  cudaGetDevice(&t->device);
  size_t total = 0;
  for (int k = 0; k < T_COUNT; ++k) total += t->host.t[k].n;
  std::vector<Coef4<double>> h64(total);
  std::vector<Coef4<float>> h32(total);
  size_t off[T_COUNT];
  size_t o = 0;
  for (int k = 0; k < T_COUNT; ++k) {
    off[k] = o;
    const HostSpline &hs = t->host.t[k];
    for (int m = 0; m < hs.n; ++m) {
      const double *c = &hs.abcd[4 * (size_t)m];
      h64[o + m] = Coef4<double>{c[0], c[1], c[2], c[3]};
      h32[o + m] = Coef4<float>{(float)c[0], (float)c[1], (float)c[2], (float)c[3]};
    }
    o += hs.n;
  }
  cudaError_t e = cudaMalloc(&t->d64, total * sizeof(Coef4<double>));
  if (e == cudaSuccess) e = cudaMalloc(&t->d32, total * sizeof(Coef4<float>));
  if (e == cudaSuccess)
    e = cudaMemcpy(t->d64, h64.data(), total * sizeof(Coef4<double>), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(t->d32, h32.data(), total * sizeof(Coef4<float>), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    btam_tables_destroy(t);
    return cuda_status(e);
  }
  for (int k = 0; k < T_COUNT; ++k) {
    const HostSpline &hs = t->host.t[k];
    t->v64.t[k] = SplineView<double>{t->d64 + off[k], hs.dx, 1.0 / hs.dx, hs.n};
    t->v32.t[k] = SplineView<float>{t->d32 + off[k], (float)hs.dx, (float)(1.0 / hs.dx), hs.n};
  }
  // the kernels' per-segment records (every radial table on one knot grid)
  std::vector<double> r64;
  std::vector<float> r32;
  size_t uw64[3], pr64[3], uw32[3], pr32[3];
  double rdx = 0.0;
  int rn = 0;
  if (!pack_radial(t->host, r64, uw64, pr64, rdx, rn) ||
      !pack_radial(t->host, r32, uw32, pr32, rdx, rn)) {
    btam_tables_destroy(t);
    return BTAM_ERR_IO;
  }
  e = cudaMalloc(&t->rad64, r64.size() * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&t->rad32, r32.size() * sizeof(float));
  if (e == cudaSuccess)
    e = cudaMemcpy(t->rad64, r64.data(), r64.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(t->rad32, r32.data(), r32.size() * sizeof(float), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    btam_tables_destroy(t);
    return cuda_status(e);
  }
  t->r64.uw = t->rad64 + uw64[0];
  t->r64.pr = t->rad64 + pr64[0];
  t->r32.uw = t->rad32 + uw32[0];
  t->r32.pr = t->rad32 + pr32[0];
  t->r64.dx = rdx;
  t->r64.inv_dx = 1.0 / rdx;
  t->r64.n = rn;
  t->r32.dx = (float)rdx;
  t->r32.inv_dx = (float)(1.0 / rdx);
  t->r32.n = rn;
  {  // the FP32 uw block with its 16-byte halves placed as the shared-memory
     // kernels read them, so a block stages it with one bulk copy
    const size_t nuw = (size_t)3 * kUWStride * rn;  // floats, a multiple of 8
    std::vector<float> sw(nuw);
    const float *src = r32.data() + uw32[0];
    for (size_t c = 0; c < nuw / 4; ++c) {
      const size_t dst = uw_swapped((int)(c >> 1)) ? (c ^ 1) : c;
      for (int k = 0; k < 4; ++k) sw[4 * dst + k] = src[4 * c + k];
    }
    e = cudaMalloc(&t->uws32, nuw * sizeof(float));
    if (e == cudaSuccess)
      e = cudaMemcpy(t->uws32, sw.data(), nuw * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      btam_tables_destroy(t);
      return cuda_status(e);
    }
    t->r32.uws = t->uws32;
  }
  {  // the FP64 uw block with its 16-byte quarters placed as the
     // shared-memory kernels read them (uw_xor64)
    const size_t nrec = (size_t)3 * rn;
    std::vector<double> sw(nrec * kUWStride);
    const double *src = r64.data() + uw64[0];
    for (size_t r = 0; r < nrec; ++r)
      for (int k = 0; k < 4; ++k) {
        const int pk = k ^ uw_xor64((int)r);
        sw[kUWStride * r + 2 * pk] = src[kUWStride * r + 2 * k];
        sw[kUWStride * r + 2 * pk + 1] = src[kUWStride * r + 2 * k + 1];
      }
    e = cudaMalloc(&t->uws64, sw.size() * sizeof(double));
    if (e == cudaSuccess)
      e = cudaMemcpy(t->uws64, sw.data(), sw.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      btam_tables_destroy(t);
      return cuda_status(e);
    }
    t->r64.uws = t->uws64;
  }
  *out = t;
  return BTAM_OK;
}

void btam_tables_destroy(btam_tables *t) {
  if (!t) return;
  if (t->d64) cudaFree(t->d64);
  if (t->d32) cudaFree(t->d32);
  if (t->rad64) cudaFree(t->rad64);
  if (t->rad32) cudaFree(t->rad32);
  if (t->uws32) cudaFree(t->uws32);
  if (t->uws64) cudaFree(t->uws64);
  delete t;
}

double btam_tables_mass(const btam_tables *t, int species) {
  if (!t) return 0.0;
  if (species == 12) return t->host.mass_mg;
  if (species == 1) return t->host.mass_h;
  return 0.0;
}

int btam_tables_spline(const btam_tables *t, int table, int n, const double *r,
                       double *value, double *deriv) {
  if (!t || table < 0 || table >= T_COUNT || n < 0 || (n > 0 && (!r || !value || !deriv)))
    return BTAM_ERR_ARG;
  if (n == 0) return BTAM_OK;
  double *d = nullptr;
  BTAM_TRY(cudaMalloc(&d, 3 * (size_t)n * sizeof(double)));
  cudaError_t e = cudaMemcpy(d, r, n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    spline_eval_kernel<<<(n + 127) / 128, 128>>>(t->v64.t[table], n, d, d + n, d + 2 * (size_t)n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(value, d + n, n * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess)
    e = cudaMemcpy(deriv, d + 2 * (size_t)n, n * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(d);
  return cuda_status(e);
}

int btam_system_create(const btam_tables *t, int n, const double *q, const double *sigma,
                       const double *x, const int *species, const double *beta,
                       const double *gamma, const double origin[3], const double cell[9],
                       const int periodic[3], btam_system **out) {
  if (!t || !out || n <= 0 || !q || !sigma || !x || !species || !origin || !cell || !periodic)
    return BTAM_ERR_ARG;
  *out = nullptr;
  std::vector<int> code(n);
  for (int i = 0; i < n; ++i) {
    if (species[i] == 12) code[i] = 0;
    else if (species[i] == 1) code[i] = 1;
    else return BTAM_ERR_SPECIES;
  }
  btam_system *s = new btam_system();
  s->T = t;
  cudaGetDevice(&s->device);
  s->n_real = n;
  int st = make_box(origin, cell, periodic, BTAM_R_CUTOFF, s->box);
  if (st != BTAM_OK) {
    delete s;
    return st;
  }
  s->any_periodic = periodic[0] || periodic[1] || periodic[2];
  st = validate_state(s, n, q, sigma, x, code.data());
  if (st == BTAM_OK && beta)
    for (int i = 0; i < n; ++i)
      if (!(std::isfinite(beta[i]) && beta[i] > 0.0)) st = BTAM_ERR_NONFINITE;
  if (st != BTAM_OK) {
    delete s;
    return st;
  }
  cudaError_t e = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete s;
    return cuda_status(e);
  }
  st = ensure_sites(s, n);
  std::vector<double4> hp(n);
  std::vector<double2> hx(n);
  std::vector<int> ho(n);
  for (int i = 0; i < n; ++i) {
    hp[i] = make_double4(q[3 * i], q[3 * i + 1], q[3 * i + 2], sigma[i]);
    hx[i] = make_double2(x[i], beta ? beta[i] : 1.0 / (kKB * 300.0));
    ho[i] = i;
  }
  if (st == BTAM_OK) {
    e = copy_sync(s->pos, hp.data(), n * sizeof(double4), cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess) e = copy_sync(s->xb, hx.data(), n * sizeof(double2), cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess) e = copy_sync(s->code, code.data(), n * sizeof(int), cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess) e = copy_sync(s->owner, ho.data(), n * sizeof(int), cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess) e = dalloc(s->gamma, s->st, n);
    if (e == cudaSuccess) {
      if (gamma) e = copy_sync(s->gamma, gamma, n * sizeof(double), cudaMemcpyHostToDevice, s->st);
      else e = cudaMemsetAsync(s->gamma, 0, n * sizeof(double), s->st);
    }
    if (e == cudaSuccess) e = dalloc(s->stage, s->st, 5 * (size_t)n);
    // err[0]: error bits of the kernels; err[1]: state-validation flags
    if (e == cudaSuccess) e = dalloc(s->err, s->st, 2);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->err, 0, sizeof(int), s->st);
    for (double **p : {&s->rho, &s->V0, &s->S0, &s->selfx, &s->Rs, &s->Rx})
      if (e == cudaSuccess) e = dalloc(*p, s->st, n);
    if (e == cudaSuccess) e = dalloc(s->Rq, s->st, 3 * (size_t)n);
    // totals, then the partial sums of the two-stage totals reduction
    if (e == cudaSuccess) e = dalloc(s->totals, s->st, 4 + 4 * kTotParts);
    if (e == cudaSuccess) e = dalloc(s->bbox, s->st, 6);
    if (e == cudaSuccess) e = dalloc(s->grid, s->st, 1);
    st = cuda_status(e);
  }
  if (st != BTAM_OK) {
    btam_system_destroy(s);
    return st;
  }
  *out = s;
  return BTAM_OK;
}

void btam_system_destroy(btam_system *s) {
  if (!s) return;
  if (s->st) cudaStreamSynchronize(s->st);
  release_state_slots(s);
  dfree(s->pos, s->st); dfree(s->xb, s->st); dfree(s->code, s->st); dfree(s->owner, s->st); dfree(s->image, s->st);
  dfree(s->pt, s->st);
  dfree(s->s32, s->st); dfree(s->sb, s->st); dfree(s->s64, s->st);
  dfree(s->gamma, s->st); dfree(s->stage, s->st); dfree(s->offs, s->st); dfree(s->idx, s->st); dfree(s->cnt, s->st);
  dfree(s->tmp, s->st); dfree(s->bbox, s->st); dfree(s->grid, s->st); dfree(s->cell_of, s->st); dfree(s->cell_cnt, s->st);
  dfree(s->cell_start, s->st); dfree(s->cursor, s->st); dfree(s->cell_sites, s->st); dfree(s->rho, s->st); dfree(s->V0, s->st);
  dfree(s->S0, s->st); dfree(s->selfx, s->st); dfree(s->Rq, s->st); dfree(s->Rs, s->st); dfree(s->Rx, s->st); dfree(s->totals, s->st);
  dfree(s->mom64, s->st); dfree(s->mom32, s->st); dfree(s->err, s->st);
  dfree(s->doffs, s->st); dfree(s->didx, s->st); dfree(s->X, s->st); dfree(s->X0, s->st); dfree(s->dtot, s->st); dfree(s->mu, s->st);
  dfree(s->dctl, s->st);
  dfree(s->dact, s->st); dfree(s->ddeg, s->st); dfree(s->rv, s->st);
  dfree(s->rev, s->st); dfree(s->slot_own, s->st); dfree(s->own_off, s->st); dfree(s->own_p, s->st); dfree(s->own_u, s->st);
  dfree(s->pbuf, s->st);
  s->scratch.release(s->st);
  if (s->st) cudaStreamSynchronize(s->st);
  if (s->st) cudaStreamDestroy(s->st);
  delete s;
}

int btam_system_set_state(btam_system *s, const double *q, const double *sigma,
                          const double *x) {
  if (!s) return BTAM_ERR_ARG;
  // the update is staged on the device and validated there (the checks of
  // validate_state); the device keeps the old state if it is rejected
  const int n = s->n_real;
  double *dq = s->stage, *ds = s->stage + 3 * (size_t)n, *dx = s->stage + 4 * (size_t)n;
  if (q) BTAM_TRY(cudaMemcpyAsync(dq, q, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s->st));
  if (sigma) BTAM_TRY(cudaMemcpyAsync(ds, sigma, n * sizeof(double), cudaMemcpyHostToDevice, s->st));
  if (x) BTAM_TRY(cudaMemcpyAsync(dx, x, n * sizeof(double), cudaMemcpyHostToDevice, s->st));
  if (!q && !sigma && !x) return BTAM_OK;
  BTAM_TRY(cudaMemsetAsync(s->err + 1, 0, sizeof(int), s->st));
  validate_stage_kernel<<<(n + 255) / 256, 256, 0, s->st>>>(
      n, q ? dq : nullptr, sigma ? ds : nullptr, x ? dx : nullptr, s->code, s->box, s->err + 1);
  BTAM_TRY(cudaGetLastError());
  int flags = 0;
  BTAM_TRY(cudaMemcpyAsync(&flags, s->err + 1, sizeof(int), cudaMemcpyDeviceToHost, s->st));
  BTAM_TRY(cudaStreamSynchronize(s->st));
  if (flags & 1) return BTAM_ERR_NONFINITE;
  if (flags & 2) return BTAM_ERR_OCCUPANCY;
  if (flags & 4) return BTAM_ERR_OUT_OF_BOX;
  pack_state_kernel<<<(n + 127) / 128, 128, 0, s->st>>>(n, q ? dq : nullptr, sigma ? ds : nullptr,
                                                        x ? dx : nullptr, s->pos, s->xb);
  BTAM_TRY(cudaGetLastError());
  if (s->n_ghost > 0)
    BTAM_TRY(launch_ghost_refresh(n, s->n_ghost, s->pos, s->xb, s->code, s->owner, s->image,
                                  s->box, s->st));
  return BTAM_OK;
}

int btam_system_info(const btam_system *s, int *n_real, int *n_ghost, long long *n_pairs) {
  if (!s) return BTAM_ERR_ARG;
  if (n_real) *n_real = s->n_real;
  if (n_ghost) *n_ghost = s->n_ghost;
  if (n_pairs) *n_pairs = s->n_pairs;
  return BTAM_OK;
}

void *btam_system_stream(const btam_system *s) { return s ? (void *)s->st : nullptr; }

int btam_neighbors_build(btam_system *s, int all_sites) {
  if (!s) return BTAM_ERR_ARG;
  s->built = false;
  const int n = s->n_real;
  BTAM_TRY(cudaMemsetAsync(s->err, 0, sizeof(int), s->st));
  // ---- periodic images
  s->n_ghost = 0;
  if (s->any_periodic) {
    int *cnt = nullptr, *off = nullptr;
    BTAM_TRY(dalloc(cnt, s->st, n + 1));
    cudaError_t e = dalloc(off, s->st, n + 1);
    if (e == cudaSuccess) e = cudaMemsetAsync(cnt + n, 0, sizeof(int), s->st);
    if (e == cudaSuccess) e = launch_ghost_count(n, s->pos, s->box, cnt, s->st);
    if (e == cudaSuccess) e = exclusive_scan(cnt, off, n + 1, s->scratch, s->st);
    int ng = 0;
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(&ng, off + n, sizeof(int), cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    int st = cuda_status(e);
    if (st == BTAM_OK) st = ensure_sites(s, n + ng);
    if (st == BTAM_OK && ng > 0) {
      e = dalloc(s->image, s->st, ng);
      if (e == cudaSuccess)
        e = launch_ghost_emit(n, s->pos, s->xb, s->code, s->owner, s->image, s->box, off, ng,
                              s->err, s->st);
      st = cuda_status(e);
    }
    dfree(cnt, s->st);
    dfree(off, s->st);
    if (st != BTAM_OK) return st;
    s->n_ghost = ng;
  }
  const int n_all = n + s->n_ghost;
  const int n_query = all_sites ? n_all : n;
  // ---- cells and neighbour buffers
  int max_cells = 4 * n_all + 1024;
  if (max_cells > s->cell_cap) {
    BTAM_TRY(dalloc(s->cell_cnt, s->st, max_cells + 1));
    BTAM_TRY(dalloc(s->cell_start, s->st, max_cells + 1));
    BTAM_TRY(dalloc(s->cursor, s->st, max_cells));
    s->cell_cap = max_cells;
  }
  if (n_all > s->site_cap) {
    BTAM_TRY(dalloc(s->cell_of, s->st, n_all));
    BTAM_TRY(dalloc(s->cell_sites, s->st, n_all));
    s->site_cap = n_all;
  }
  int total = 0;
  int st = build_list(s, n_all, n_query, BTAM_R_CUTOFF, BTAM_MAXNEIGH, -1, 0, s->offs, s->q_cap,
                      s->idx, s->idx_cap, total);
  if (st != BTAM_OK) return st;
  s->n_list = n_query;
  s->n_pairs = total;
  // reverse slots and owned pairs for the undirected pass 2
  if (total > s->rev_cap) {
    BTAM_TRY(dalloc(s->rev, s->st, total));
    BTAM_TRY(dalloc(s->slot_own, s->st, total));
    s->rev_cap = total;
  }
  if (n + 1 > s->own_off_cap) {
    BTAM_TRY(dalloc(s->own_off, s->st, n + 1));
    s->own_off_cap = n + 1;
  }
  BTAM_TRY(launch_pair_links(n, s->offs, s->idx, s->owner, s->rev, s->slot_own, s->cnt,
                             s->own_off, s->own_p, s->own_u, s->own_cap, &s->n_own, s->scratch,
                             s->st));
  if (s->pbuf_elem > 0) {  // a rebuilt list may be longer than the slot buffer
    int st2 = ensure_pbuf(s, s->pbuf_elem);
    if (st2 != BTAM_OK) return st2;
  }
  s->built = true;
  return BTAM_OK;
}

}  // extern "C"

// One CSR neighbour list over the current sites: cell binning, per-site
// search (optionally restricted to one species code), scan and compaction.
static int build_list(btam_system *s, int n_all, int n_query, double rc, int maxn, int filter,
                      int allow_empty, int *&offs, int &q_cap, int *&idx, long long &idx_cap,
                      int &total) {
  if (n_query + 1 > s->cnt_cap) {
    BTAM_TRY(dalloc(s->cnt, s->st, n_query + 1));
    s->cnt_cap = n_query + 1;
  }
  if (n_query + 1 > q_cap) {
    BTAM_TRY(dalloc(offs, s->st, n_query + 1));
    q_cap = n_query + 1;
  }
  if ((long long)n_query * kNbrBuf > s->tmp_cap) {
    BTAM_TRY(dalloc(s->tmp, s->st, (size_t)n_query * kNbrBuf));
    s->tmp_cap = (long long)n_query * kNbrBuf;
  }
  NbrArgs a;
  a.n_all = n_all;
  a.n_query = n_query;
  a.maxn = maxn;
  a.max_cells = s->cell_cap;
  a.rc = rc;
  a.cell_edge = rc * (1.0 + 1e-9) + 1e-9;
  a.code = s->code;
  a.filter_code = filter;
  a.allow_empty = allow_empty;
  a.pos = s->pos;
  a.bbox = s->bbox;
  a.grid = s->grid;
  a.cell_of = s->cell_of;
  a.cell_cnt = s->cell_cnt;
  a.cell_start = s->cell_start;
  a.cursor = s->cursor;
  a.cell_sites = s->cell_sites;
  a.cnt = s->cnt;
  a.tmp = s->tmp;
  a.offs = offs;
  a.err = s->err;
  a.scratch = &s->scratch;
  BTAM_TRY(launch_neighbors(a, s->st));
  total = 0;
  BTAM_TRY(cudaMemcpyAsync(&total, offs + n_query, sizeof(int), cudaMemcpyDeviceToHost, s->st));
  int st = read_err(s);
  if (st != BTAM_OK) return st;
  if (total > idx_cap) {
    BTAM_TRY(dalloc(idx, s->st, total));
    idx_cap = total;
  }
  BTAM_TRY(launch_compact(n_query, s->tmp, offs, idx, s->st));
  BTAM_TRY(cudaStreamSynchronize(s->st));
  return BTAM_OK;
}

extern "C" {

int btam_neighbors_copy(const btam_system *s, int *offs, int *idx, long long idx_cap) {
  if (!s || !offs) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  BTAM_TRY(copy_sync(offs, s->offs, (s->n_list + 1) * sizeof(int), cudaMemcpyDeviceToHost, s->st));
  if (idx) {
    if (idx_cap < s->n_pairs) return BTAM_ERR_ARG;
    BTAM_TRY(copy_sync(idx, s->idx, s->n_pairs * sizeof(int), cudaMemcpyDeviceToHost, s->st));
  }
  return BTAM_OK;
}

int btam_ghosts_copy(const btam_system *s, double *q, int *owner, int *image) {
  if (!s) return BTAM_ERR_ARG;
  const int n = s->n_real, ng = s->n_ghost;
  if (ng == 0) return BTAM_OK;
  std::vector<double4> hp(ng);
  std::vector<char4> hi(ng);
  BTAM_TRY(copy_sync(hp.data(), s->pos + n, ng * sizeof(double4), cudaMemcpyDeviceToHost, s->st));
  BTAM_TRY(copy_sync(hi.data(), s->image, ng * sizeof(char4), cudaMemcpyDeviceToHost, s->st));
  if (owner)
    BTAM_TRY(copy_sync(owner, s->owner + n, ng * sizeof(int), cudaMemcpyDeviceToHost, s->st));
  for (int k = 0; k < ng; ++k) {
    if (q) {
      q[3 * k] = hp[k].x;
      q[3 * k + 1] = hp[k].y;
      q[3 * k + 2] = hp[k].z;
    }
    if (image) {
      image[3 * k] = hi[k].x;
      image[3 * k + 1] = hi[k].y;
      image[3 * k + 2] = hi[k].z;
    }
  }
  return BTAM_OK;
}

int btam_mf_eval_async(btam_system *s, int precision) {
  return enqueue_eval(s, precision, false, false);
}

int btam_mf_eval_x(btam_system *s, int precision) {
  return enqueue_eval(s, precision, true, false);
}

}  // extern "C"

// Keeps the fastest pass-1 and pass-2 launch variants for this system and
// arithmetic form (timed by autotune_passes).
template <class R>
static int autotune_form(btam_system *s, EvalArgs<R> a, int form, int reps) {
  int b1 = 0, b2 = 0;
  cudaError_t e = autotune_passes(a, s->st, reps, &b1, &b2);
  if (e != cudaSuccess) return cuda_status(e);
  s->variant1[form] = b1;
  s->variant2[form] = b2;
  return read_err(s);
}

extern "C" {

int btam_autotune(btam_system *s, int precision, int *pass1_variant, int *pass2_variant) {
  if (!s) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  const size_t nm = (size_t)s->n_real * kMomStride;
  int st;
  if (precision == BTAM_FP64) {
    if (!s->mom64) BTAM_TRY(dalloc(s->mom64, s->st, nm));
    if ((st = ensure_pbuf(s, sizeof(double))) != BTAM_OK) return st;
    st = autotune_form(s, eval_args<double>(s, s->mom64, s->T->r64), 0, 3);
  } else if (precision == BTAM_FP32C) {
    if (!s->mom32) BTAM_TRY(dalloc(s->mom32, s->st, nm));
    if ((st = ensure_pbuf(s, sizeof(float))) != BTAM_OK) return st;
    st = autotune_form(s, eval_args<float>(s, s->mom32, s->T->r32), 1, 3);
  } else {
    return BTAM_ERR_ARG;
  }
  if (st != BTAM_OK) return st;
  // the slot buffer stays only while an undirected variant is selected
  if (!((s->variant1[0] | s->variant1[1] | s->variant2[0] | s->variant2[1]) & kUndirected)) {
    dfree(s->pbuf, s->st);
    s->pbuf_bytes = s->pbuf_elem = 0;
  }
  const int f = precision == BTAM_FP64 ? 0 : 1;
  if (pass1_variant) *pass1_variant = s->variant1[f];
  if (pass2_variant) *pass2_variant = s->variant2[f];
  return BTAM_OK;
}

int btam_set_variants(btam_system *s, int precision, int pass1_variant, int pass2_variant) {
  if (!s || (precision != BTAM_FP64 && precision != BTAM_FP32C)) return BTAM_ERR_ARG;
  if (!valid_variants(pass1_variant, pass2_variant)) return BTAM_ERR_ARG;
  if ((pass1_variant | pass2_variant) & kUndirected) {
    if (!s->built) return BTAM_ERR_NOT_BUILT;
    int st = ensure_pbuf(s, precision == BTAM_FP64 ? sizeof(double) : sizeof(float));
    if (st != BTAM_OK) return st;
  }
  const int f = precision == BTAM_FP64 ? 0 : 1;
  s->variant1[f] = pass1_variant;
  s->variant2[f] = pass2_variant;
  return BTAM_OK;
}

int btam_system_sync(btam_system *s) {
  if (!s) return BTAM_ERR_ARG;
  return read_err(s);
}

int btam_results_copy(btam_system *s, double *rho, double *V0, double *S0, double *Rq,
                      double *Rs, double *Rx, double *totals) {
  if (!s) return BTAM_ERR_ARG;
  const size_t n = (size_t)s->n_real * sizeof(double);
  struct {
    double *dst;
    const double *src;
    size_t bytes;
  } cp[7] = {{rho, s->rho, n}, {V0, s->V0, n}, {S0, s->S0, n}, {Rq, s->Rq, 3 * n},
             {Rs, s->Rs, n},   {Rx, s->Rx, n}, {totals, s->totals, 4 * sizeof(double)}};
  for (auto &c : cp)
    if (c.dst) BTAM_TRY(cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToHost, s->st));
  return read_err(s);
}

int btam_mf_eval(btam_system *s, int precision, double *rho, double *V0, double *S0,
                 double *Rq, double *Rs, double *Rx, double *totals) {
  if (!s) return BTAM_ERR_ARG;
  BTAM_TRY(cudaMemsetAsync(s->err, 0, sizeof(int), s->st));
  int st = btam_mf_eval_async(s, precision);
  if (st != BTAM_OK) return st;
  return btam_results_copy(s, rho, V0, S0, Rq, Rs, Rx, totals);
}

int btam_mf_eval_state(btam_system *s, int precision, const double *q, const double *sigma,
                       const double *x, double *rho, double *V0, double *S0, double *Rq,
                       double *Rs, double *Rx, double *totals) {
  if (!s) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  if (precision != BTAM_FP64 && precision != BTAM_FP32C) return BTAM_ERR_ARG;
  // as btam_system_set_state, but the validation flags are read with the
  // results: the update is applied on the device only if it passes, and
  // the host waits once
  const int n = s->n_real;
  double *dq = s->stage, *ds = s->stage + 3 * (size_t)n, *dx = s->stage + 4 * (size_t)n;
  if (q) BTAM_TRY(cudaMemcpyAsync(dq, q, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s->st));
  if (sigma) BTAM_TRY(cudaMemcpyAsync(ds, sigma, n * sizeof(double), cudaMemcpyHostToDevice, s->st));
  if (x) BTAM_TRY(cudaMemcpyAsync(dx, x, n * sizeof(double), cudaMemcpyHostToDevice, s->st));
  BTAM_TRY(cudaMemsetAsync(s->err, 0, 2 * sizeof(int), s->st));
  if (q || sigma || x) {
    validate_stage_kernel<<<(n + 255) / 256, 256, 0, s->st>>>(
        n, q ? dq : nullptr, sigma ? ds : nullptr, x ? dx : nullptr, s->code, s->box, s->err + 1);
    BTAM_TRY(cudaGetLastError());
    pack_state_kernel<<<(n + 127) / 128, 128, 0, s->st>>>(
        n, q ? dq : nullptr, sigma ? ds : nullptr, x ? dx : nullptr, s->pos, s->xb, s->err + 1);
    BTAM_TRY(cudaGetLastError());
    if (s->n_ghost > 0)
      BTAM_TRY(launch_ghost_refresh(n, s->n_ghost, s->pos, s->xb, s->code, s->owner, s->image,
                                    s->box, s->st));
  }
  int st = btam_mf_eval_async(s, precision);
  if (st != BTAM_OK) return st;
  // the result copies, then the validation flags and error bits behind
  // them, and one wait for all of it
  const size_t nb = (size_t)n * sizeof(double);
  const struct {
    double *dst;
    const double *src;
    size_t bytes;
  } cp[7] = {{rho, s->rho, nb}, {V0, s->V0, nb}, {S0, s->S0, nb}, {Rq, s->Rq, 3 * nb},
             {Rs, s->Rs, nb},   {Rx, s->Rx, nb}, {totals, s->totals, 4 * sizeof(double)}};
  for (const auto &c : cp)
    if (c.dst) BTAM_TRY(cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToHost, s->st));
  int bits[2] = {0, 0};
  BTAM_TRY(cudaMemcpyAsync(bits, s->err, 2 * sizeof(int), cudaMemcpyDeviceToHost, s->st));
  BTAM_TRY(cudaMemsetAsync(s->err, 0, sizeof(int), s->st));
  BTAM_TRY(cudaStreamSynchronize(s->st));
  const int flags = bits[1];
  st = status_from_bits(bits[0]);
  if (flags & 1) return BTAM_ERR_NONFINITE;
  if (flags & 2) return BTAM_ERR_OCCUPANCY;
  if (flags & 4) return BTAM_ERR_OUT_OF_BOX;
  return st;
}

}  // extern "C"

namespace {

// Status of a completed pipelined call from its flags (error bits, then the
// validation flags of its update), with btam_mf_eval_state's precedence.
int state_status(const int *f) {
  if (f[1] & 1) return BTAM_ERR_NONFINITE;
  if (f[1] & 2) return BTAM_ERR_OCCUPANCY;
  if (f[1] & 4) return BTAM_ERR_OUT_OF_BOX;
  return status_from_bits(f[0]);
}

// Waits until the call in slot b has delivered its results, frees the slot
// and returns the call's status.
int retire_state_slot(btam_system *s, int b) {
  auto &sl = s->slot[b];
  const cudaError_t e = cudaEventSynchronize(sl.out);
  sl.ticket = 0;
  return e == cudaSuccess ? state_status(sl.hflags) : cuda_status(e);
}

// The two slots' buffers, events and the copy streams, made on first use.
int ensure_state_slots(btam_system *s) {
  if (s->cp_in && s->cp_out) return BTAM_OK;
  const size_t n = (size_t)s->n_real;
  for (auto &sl : s->slot) {
    BTAM_TRY(dalloc(sl.stage, s->st, 5 * n));
    BTAM_TRY(dalloc(sl.res, s->st, 8 * n + 4));
    BTAM_TRY(dalloc(sl.flags, s->st, 2));
    if (!sl.hflags) BTAM_TRY(cudaMallocHost((void **)&sl.hflags, 2 * sizeof(int)));
    sl.hflags[0] = sl.hflags[1] = 0;
    for (cudaEvent_t *ev : {&sl.in, &sl.used, &sl.done, &sl.out})
      if (!*ev) BTAM_TRY(cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
    sl.ticket = 0;
  }
  if (!s->cp_in) BTAM_TRY(cudaStreamCreateWithFlags(&s->cp_in, cudaStreamNonBlocking));
  if (!s->cp_out) BTAM_TRY(cudaStreamCreateWithFlags(&s->cp_out, cudaStreamNonBlocking));
  // the slot buffers come from the pool in the order of `st`: the copy
  // streams use them only after that
  cudaEvent_t ev = nullptr;
  BTAM_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  cudaError_t e = cudaEventRecord(ev, s->st);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s->cp_in, ev, 0);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s->cp_out, ev, 0);
  cudaEventDestroy(ev);
  return cuda_status(e);
}

void release_state_slots(btam_system *s) {
  if (s->cp_in) cudaStreamSynchronize(s->cp_in);
  if (s->cp_out) cudaStreamSynchronize(s->cp_out);
  for (auto &sl : s->slot) {
    dfree(sl.stage, s->st);
    dfree(sl.res, s->st);
    dfree(sl.flags, s->st);
    if (sl.hflags) cudaFreeHost(sl.hflags);
    sl.hflags = nullptr;
    for (cudaEvent_t *ev : {&sl.in, &sl.used, &sl.done, &sl.out})
      if (*ev) cudaEventDestroy(*ev);
    sl.in = sl.used = sl.done = sl.out = nullptr;
  }
  if (s->cp_in) cudaStreamDestroy(s->cp_in);
  if (s->cp_out) cudaStreamDestroy(s->cp_out);
  s->cp_in = s->cp_out = nullptr;
}

}  // namespace

extern "C" {

int btam_mf_eval_state_async(btam_system *s, int precision, const double *q,
                             const double *sigma, const double *x, double *rho, double *V0,
                             double *S0, double *Rq, double *Rs, double *Rx, double *totals,
                             long long *ticket) {
  if (!s || !ticket) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  if (precision != BTAM_FP64 && precision != BTAM_FP32C) return BTAM_ERR_ARG;
  if (s->batcher) return BTAM_ERR_ARG;  // a served system evaluates in the server's rounds
  int st = ensure_state_slots(s);
  if (st != BTAM_OK) return st;
  const long long tk = s->next_ticket;
  const int b = (int)(tk & 1);
  auto &sl = s->slot[b];
  if (sl.ticket) {  // the call two back still holds this slot: let it finish
    const long long old = sl.ticket;
    s->finished.emplace_back(old, retire_state_slot(s, b));
  }
  const int n = s->n_real;
  const size_t nb = (size_t)n * sizeof(double);
  double *dq = sl.stage, *ds = sl.stage + 3 * (size_t)n, *dx = sl.stage + 4 * (size_t)n;
  // copies in on their own stream, once the slot's staging was last read
  BTAM_TRY(cudaStreamWaitEvent(s->cp_in, sl.used, 0));
  if (q) BTAM_TRY(cudaMemcpyAsync(dq, q, 3 * nb, cudaMemcpyHostToDevice, s->cp_in));
  if (sigma) BTAM_TRY(cudaMemcpyAsync(ds, sigma, nb, cudaMemcpyHostToDevice, s->cp_in));
  if (x) BTAM_TRY(cudaMemcpyAsync(dx, x, nb, cudaMemcpyHostToDevice, s->cp_in));
  BTAM_TRY(cudaEventRecord(sl.in, s->cp_in));
  // validation, the update and the evaluation on the system's stream
  BTAM_TRY(cudaStreamWaitEvent(s->st, sl.in, 0));
  BTAM_TRY(cudaMemsetAsync(s->err, 0, 2 * sizeof(int), s->st));
  if (q || sigma || x) {
    validate_stage_kernel<<<(n + 255) / 256, 256, 0, s->st>>>(
        n, q ? dq : nullptr, sigma ? ds : nullptr, x ? dx : nullptr, s->code, s->box, s->err + 1);
    BTAM_TRY(cudaGetLastError());
    pack_state_kernel<<<(n + 127) / 128, 128, 0, s->st>>>(
        n, q ? dq : nullptr, sigma ? ds : nullptr, x ? dx : nullptr, s->pos, s->xb, s->err + 1);
    BTAM_TRY(cudaGetLastError());
    if (s->n_ghost > 0)
      BTAM_TRY(launch_ghost_refresh(n, s->n_ghost, s->pos, s->xb, s->code, s->owner, s->image,
                                    s->box, s->st));
  }
  BTAM_TRY(cudaEventRecord(sl.used, s->st));
  if ((st = btam_mf_eval_async(s, precision)) != BTAM_OK) return st;
  // the requested results and the flags into the slot (device copies), so
  // that the next call may overwrite the system's result arrays while
  // these go to the host on the copy-out stream
  const struct {
    double *dst;
    const double *src;
    size_t off, bytes;
  } cp[7] = {{rho, s->rho, 0, nb},          {V0, s->V0, (size_t)n, nb},
             {S0, s->S0, 2 * (size_t)n, nb}, {Rq, s->Rq, 3 * (size_t)n, 3 * nb},
             {Rs, s->Rs, 6 * (size_t)n, nb}, {Rx, s->Rx, 7 * (size_t)n, nb},
             {totals, s->totals, 8 * (size_t)n, 4 * sizeof(double)}};
  for (const auto &c : cp)
    if (c.dst)
      BTAM_TRY(cudaMemcpyAsync(sl.res + c.off, c.src, c.bytes, cudaMemcpyDeviceToDevice, s->st));
  BTAM_TRY(cudaMemcpyAsync(sl.flags, s->err, 2 * sizeof(int), cudaMemcpyDeviceToDevice, s->st));
  BTAM_TRY(cudaMemsetAsync(s->err, 0, sizeof(int), s->st));
  BTAM_TRY(cudaEventRecord(sl.done, s->st));
  BTAM_TRY(cudaStreamWaitEvent(s->cp_out, sl.done, 0));
  for (const auto &c : cp)
    if (c.dst)
      BTAM_TRY(cudaMemcpyAsync(c.dst, sl.res + c.off, c.bytes, cudaMemcpyDeviceToHost, s->cp_out));
  BTAM_TRY(cudaMemcpyAsync(sl.hflags, sl.flags, 2 * sizeof(int), cudaMemcpyDeviceToHost,
                           s->cp_out));
  BTAM_TRY(cudaEventRecord(sl.out, s->cp_out));
  sl.ticket = tk;
  s->next_ticket = tk + 1;
  *ticket = tk;
  return BTAM_OK;
}

int btam_mf_eval_state_wait(btam_system *s, long long ticket) {
  if (!s || ticket <= 0) return BTAM_ERR_ARG;
  for (int b = 0; b < 2; ++b)
    if (s->slot[b].ticket == ticket) return retire_state_slot(s, b);
  for (size_t k = 0; k < s->finished.size(); ++k)
    if (s->finished[k].first == ticket) {
      const int st = s->finished[k].second;
      s->finished.erase(s->finished.begin() + (long)k);
      return st;
    }
  return BTAM_ERR_ARG;  // unknown, or already waited for
}

int btam_mf_rho(btam_system *s, int precision, double *rho) {
  if (!s || !rho) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  BTAM_TRY(cudaMemsetAsync(s->err, 0, sizeof(int), s->st));
  const size_t nm = (size_t)s->n_real * kMomStride;
  if (precision == BTAM_FP64) {
    if (!s->mom64) BTAM_TRY(dalloc(s->mom64, s->st, nm));
    BTAM_TRY(launch_pass1(eval_args<double>(s, s->mom64, s->T->r64), s->st));
  } else if (precision == BTAM_FP32C) {
    if (!s->mom32) BTAM_TRY(dalloc(s->mom32, s->st, nm));
    BTAM_TRY(launch_pass1(eval_args<float>(s, s->mom32, s->T->r32), s->st));
  } else {
    return BTAM_ERR_ARG;
  }
  BTAM_TRY(cudaMemcpyAsync(rho, s->rho, s->n_real * sizeof(double), cudaMemcpyDeviceToHost, s->st));
  return read_err(s);
}

int btam_mf_eval_profile(btam_system *s, int precision, double ms[5]) {
  if (!s || !ms) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  if (precision != BTAM_FP64 && precision != BTAM_FP32C) return BTAM_ERR_ARG;
  cudaEvent_t ev[6];
  for (auto &e : ev) BTAM_TRY(cudaEventCreate(&e));
  const size_t nm = (size_t)s->n_real * kMomStride;
  cudaError_t e = cudaEventRecord(ev[0], s->st);
  const int f = precision == BTAM_FP64 ? 0 : 1;
  if (precision == BTAM_FP64) {
    if (!s->mom64 && e == cudaSuccess) e = dalloc(s->mom64, s->st, nm);
    EvalArgs<double> a = eval_args<double>(s, s->mom64, s->T->r64);
    if (e == cudaSuccess) e = launch_pass1(a, s->st, s->variant1[f], s->variant2[f], ev[1]);
    if (e == cudaSuccess) e = cudaEventRecord(ev[2], s->st);
    if (e == cudaSuccess) e = launch_pass2(a, s->st, s->variant2[f], ev[3]);
  } else {
    if (!s->mom32 && e == cudaSuccess) e = dalloc(s->mom32, s->st, nm);
    EvalArgs<float> a = eval_args<float>(s, s->mom32, s->T->r32);
    if (e == cudaSuccess) e = launch_pass1(a, s->st, s->variant1[f], s->variant2[f], ev[1]);
    if (e == cudaSuccess) e = cudaEventRecord(ev[2], s->st);
    if (e == cudaSuccess) e = launch_pass2(a, s->st, s->variant2[f], ev[3]);
  }
  if (e == cudaSuccess) e = cudaEventRecord(ev[4], s->st);
  if (e == cudaSuccess)
    e = launch_totals(s->n_real, s->V0, s->S0, s->Rq, s->Rs, s->Rx, s->totals, s->totals + 4,
                      s->st);
  if (e == cudaSuccess) e = cudaEventRecord(ev[5], s->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  for (int k = 0; k < 5 && e == cudaSuccess; ++k) {
    float t = 0.f;
    e = cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
    ms[k] = t;
  }
  for (auto &x : ev) cudaEventDestroy(x);
  if (e != cudaSuccess) return cuda_status(e);
  return read_err(s);
}

int btam_probe_fma_peak(int fp64, double seconds, double *tflops) {
  if (!tflops || !(seconds > 0.0)) return BTAM_ERR_ARG;
  int dev = 0, sms = 0;
  BTAM_TRY(cudaGetDevice(&dev));
  BTAM_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int threads = 256, blocks = sms * 8;
  float *sink = nullptr;
  BTAM_TRY(cudaMalloc(&sink, (size_t)blocks * threads * sizeof(double)));
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  // calibrate the iteration count on a short run, then time one long launch
  long long iters = 1 << 12;
  double best = 0.0;
  cudaError_t e = cudaSuccess;
  for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {
    cudaEventRecord(a);
    if (fp64) fma_probe_kernel<double><<<blocks, threads>>>(iters, (double *)sink);
    else fma_probe_kernel<float><<<blocks, threads>>>(iters, sink);
    cudaEventRecord(b);
    e = cudaEventSynchronize(b);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
    double flops = 2.0 * kProbeChains * (double)iters * blocks * threads;
    if (ms > 0) best = flops / (ms * 1e-3) / 1e12;
    if (ms > 0 && rep < 3) {
      double scale = seconds * 1e3 / ms;
      if (scale > 1.0) iters = (long long)(iters * (scale > 1e4 ? 1e4 : scale));
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(sink);
  if (e != cudaSuccess) return cuda_status(e);
  *tflops = best;
  return BTAM_OK;
}

int btam_probe_gather_peak(const btam_tables *t, double seconds, double *gbs) {
  if (!t || !gbs || !(seconds > 0.0)) return BTAM_ERR_ARG;
  int dev = 0, sms = 0;
  BTAM_TRY(cudaGetDevice(&dev));
  BTAM_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int threads = 256, blocks = sms * 8;
  const int n_rec = 3 * t->r32.n;  // the u, w records of the three pair kinds
  float *sink = nullptr;
  BTAM_TRY(cudaMalloc(&sink, (size_t)blocks * threads * sizeof(float)));
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  long long iters = 1 << 8;
  double best = 0.0;
  cudaError_t e = cudaSuccess;
  for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {
    cudaEventRecord(a);
    gather_probe_kernel<<<blocks, threads>>>(t->r32.uw, n_rec, iters, sink);
    cudaEventRecord(b);
    e = cudaEventSynchronize(b);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
    const double bytes = 32.0 * 4.0 * (double)iters * blocks * threads;
    if (ms > 0) best = bytes / (ms * 1e-3) / 1e9;
    if (ms > 0 && rep < 3) {
      double scale = seconds * 1e3 / ms;
      if (scale > 1.0) iters = (long long)(iters * (scale > 1e4 ? 1e4 : scale));
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(sink);
  if (e != cudaSuccess) return cuda_status(e);
  *gbs = best;
  return BTAM_OK;
}

}  // extern "C"

int mf_rho64_enqueue(btam_system *s) {
  if (!s->mom64) BTAM_TRY(dalloc(s->mom64, s->st, (size_t)s->n_real * kMomStride));
  BTAM_TRY(launch_pass1(eval_args<double>(s, s->mom64, s->T->r64), s->st, 0, 0));
  return BTAM_OK;
}

int mf_stress_enqueue(btam_system *s, int precision, double **W_out, double **tot_out) {
  double *W = nullptr, *part = nullptr, *tot = nullptr;
  int st = pt_stress_buffers(s, &W, &part, &tot);
  if (st != BTAM_OK) return st;
  const size_t nm = (size_t)s->n_real * kMomStride;
  // the directed pass 1 writes the moment records the stress kernel reads
  if (precision == BTAM_FP64) {
    if (!s->mom64) BTAM_TRY(dalloc(s->mom64, s->st, nm));
    EvalArgs<double> a = eval_args<double>(s, s->mom64, s->T->r64);
    BTAM_TRY(launch_pass1(a, s->st, 0, 0));
    BTAM_TRY(launch_mf_stress(a, W, s->st));
  } else {
    if (!s->mom32) BTAM_TRY(dalloc(s->mom32, s->st, nm));
    EvalArgs<float> a = eval_args<float>(s, s->mom32, s->T->r32);
    BTAM_TRY(launch_pass1(a, s->st, 0, 0));
    BTAM_TRY(launch_mf_stress(a, W, s->st));
  }
  BTAM_TRY(launch_pt_totals(s->n_real, nullptr, nullptr, W, part, tot, s->st));
  *W_out = W;
  *tot_out = tot;
  return BTAM_OK;
}

extern "C" {

int btam_mf_stress(btam_system *s, int precision, double *W0, double *total) {
  if (!s) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  if (precision != BTAM_FP64 && precision != BTAM_FP32C) return BTAM_ERR_ARG;
  double *W = nullptr, *tot = nullptr;
  int st = mf_stress_enqueue(s, precision, &W, &tot);
  if (st != BTAM_OK) return st;
  if (W0)
    BTAM_TRY(cudaMemcpyAsync(W0, W, 9 * (size_t)s->n_real * sizeof(double),
                             cudaMemcpyDeviceToHost, s->st));
  if (total)
    BTAM_TRY(cudaMemcpyAsync(total, tot + 2, 9 * sizeof(double), cudaMemcpyDeviceToHost, s->st));
  return read_err(s);
}

int btam_mf_pair_terms(btam_system *s, int precision, double *self, double *slot,
                       long long slot_cap) {
  if (!s) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  if (precision != BTAM_FP64 && precision != BTAM_FP32C) return BTAM_ERR_ARG;
  int n_slots = 0;
  BTAM_TRY(copy_sync(&n_slots, s->offs + s->n_real, sizeof(int), cudaMemcpyDeviceToHost, s->st));
  if (slot && slot_cap < n_slots) return BTAM_ERR_ARG;
  double *d_self = nullptr, *d_slot = nullptr;
  BTAM_TRY(dalloc(d_self, s->st, 5 * (size_t)s->n_real));
  cudaError_t e = dalloc(d_slot, s->st, 5 * (size_t)n_slots);
  const size_t nm = (size_t)s->n_real * kMomStride;
  // the directed pass 1 writes the moment records and dV0_u/dx_u
  if (e == cudaSuccess) {
    if (precision == BTAM_FP64) {
      if (!s->mom64) e = dalloc(s->mom64, s->st, nm);
      EvalArgs<double> a = eval_args<double>(s, s->mom64, s->T->r64);
      if (e == cudaSuccess) e = launch_pass1(a, s->st, 0, 0);
      if (e == cudaSuccess) e = launch_mf_pair_terms(a, d_self, d_slot, s->st);
    } else {
      if (!s->mom32) e = dalloc(s->mom32, s->st, nm);
      EvalArgs<float> a = eval_args<float>(s, s->mom32, s->T->r32);
      if (e == cudaSuccess) e = launch_pass1(a, s->st, 0, 0);
      if (e == cudaSuccess) e = launch_mf_pair_terms(a, d_self, d_slot, s->st);
    }
  }
  if (e == cudaSuccess && self)
    e = cudaMemcpyAsync(self, d_self, 5 * (size_t)s->n_real * sizeof(double),
                        cudaMemcpyDeviceToHost, s->st);
  if (e == cudaSuccess && slot)
    e = cudaMemcpyAsync(slot, d_slot, 5 * (size_t)n_slots * sizeof(double),
                        cudaMemcpyDeviceToHost, s->st);
  dfree(d_self, s->st);
  dfree(d_slot, s->st);
  if (e != cudaSuccess) return cuda_status(e);
  return read_err(s);
}

int btam_rho_nmf(btam_system *s, double *rho) {
  if (!s || !rho) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  BTAM_TRY(launch_rho_nmf(s->n_real, s->pos, s->xb, s->code, s->offs, s->idx,
                          s->T->v64.t[T_RHO_MG], s->T->v64.t[T_RHO_H], s->rho, s->st));
  BTAM_TRY(cudaMemcpyAsync(rho, s->rho, s->n_real * sizeof(double), cudaMemcpyDeviceToHost, s->st));
  return read_err(s);
}

}  // extern "C"

// ===========================================================================
// Relaxation of (q, sigma) and the hydrogen master equation (solvers.cu).

namespace {

// Evaluation followed by the relaxation view of it: z, g, F and |R|^2.
struct RelaxVecs {
  double *z, *g, *p, *z0, *g0, *work, *tmp, *fterm, *rterm, *ones, *scal, *rho, *alpha;
  double *S[16], *Y[16];
  RelaxBounds bd;
};

int relax_eval(btam_system *s, int prec, RelaxVecs &v, double &f, double &r2) {
  int st = btam_mf_eval_async(s, prec);
  if (st != BTAM_OK) return st;
  BTAM_TRY(relax_gather(s->n_real, s->pos, s->xb, s->V0, s->Rq, s->Rs, v.bd, v.z, v.g, v.fterm,
                        v.rterm, v.scal, v.scal + 1, v.ones, s->st));
  double h[2];
  BTAM_TRY(cudaMemcpyAsync(h, v.scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->st));
  st = read_err(s);
  f = h[0];
  r2 = h[1];
  return st;
}

double dev_dot(btam_system *s, RelaxVecs &v, int n, const double *a, const double *b) {
  vec_dot(n, a, b, v.tmp + 7, s->st);
  double h = 0.0;
  cudaMemcpyAsync(&h, v.tmp + 7, sizeof(double), cudaMemcpyDeviceToHost, s->st);
  cudaStreamSynchronize(s->st);
  return h;
}

__global__ void fill_kernel(int n, double v, double *a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

// g / beta per site: the N-GMRES residual in energy units
__global__ void unbeta_kernel(int n4, const double2 *xb, double *g) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n4) g[i] /= xb[i >> 2].y;
}

// max over sites and components of |p| in unscaled units (p / sqrt(max(x, 1e-3)))
__global__ void absmax_kernel(int n4, const double2 *xb, const double *a, double *out) {
  __shared__ double sh[256];
  double v = 0.0;
  for (int i = threadIdx.x; i < n4; i += 256)
    v = fmax(v, fabs(a[i]) / sqrt(fmax(xb[i >> 2].x, 1e-3)));
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int k = 128; k > 0; k >>= 1) {
    if ((int)threadIdx.x < k) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + k]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

// The relaxation with the reference's option set for its SNES (main-BT-AM.cpp:
// 64-67: -snes_type ngmres, -snes_ngmres_m 3, -snes_linesearch_type cp):
// N-GMRES(m) on the variables z = (q, log sigma) scaled by the occupancies
// (the same z and bounds as the L-BFGS schedule) with the residual
// g(z) = (R_q, sigma R_sigma) / sqrt(x), the gradient of F in energy units
// (the L-BFGS gradient over beta), FP64, every vector on the device.  The
// energy units make the line search's first trial (lambda = 1) move a site
// by its force over its occupancy in A per eV/A instead of beta times that.
// As PETSc's SNESNGMRES with its defaults forms it: each iteration takes
// z^M = z - lambda g(z), lambda from the critical-point line search (one
// secant step on g(z - lambda g) . g from lambda = 0 and the first trial,
// lambda = 1 damped to a 0.05 move), then the
// combination z^A of z^M and the last m
// iterates minimising the linearised |g|; z^A is kept when |g(z^A)| < 2
// min|g| and either 0.1 |z^A - z^M| < min_i |z^A - z_i| or sqrt|g(z)| < 0.9
// sqrt(min|g|), else z^M; the subspace restarts after two consecutive
// iterations with (0.1 |z^A - z^M| > min_i |z^A - z_i| and sqrt|g(z^A)| >
// 0.9 sqrt(min|g|)) or |g(z^A)| > 2 min|g|.  Three evaluations per
// iteration; converged on the projected residual norm as btam_relax.
int relax_ngmres(btam_system *s, double tol, int max_iter, int m, const double *bounds,
                 double *info) {
  constexpr double gammaA = 2.0, gammaC = 2.0, epsilonB = 0.1, deltaB = 0.9;
  constexpr double kTrialMove = 0.05, kMaxMove = 0.5;
  constexpr int restart_it = 2;
  const double sig_lo = bounds ? bounds[0] : 0.001, sig_hi = bounds ? bounds[1] : 0.4,
               x_min = bounds ? bounds[2] : 0.01;
  if (!(sig_lo > 0.0 && sig_hi > sig_lo && x_min >= 0.0)) return BTAM_ERR_ARG;
  const int n = s->n_real, n4 = 4 * n;
  // X F XM FM XA FA D, Xd[m] Fd[m] (n4 each), fterm rterm ones (n), scalars
  double *buf = nullptr;
  BTAM_TRY(dalloc(buf, s->st, (size_t)(7 + 2 * m) * n4 + 3 * (size_t)n + 64));
  double *X = buf, *F = buf + n4, *XM = buf + 2 * (size_t)n4, *FM = buf + 3 * (size_t)n4,
         *XA = buf + 4 * (size_t)n4, *FA = buf + 5 * (size_t)n4, *D = buf + 6 * (size_t)n4;
  std::vector<double *> Xd(m), Fd(m);
  for (int k = 0; k < m; ++k) {
    Xd[k] = buf + (size_t)(7 + k) * n4;
    Fd[k] = buf + (size_t)(7 + m + k) * n4;
  }
  RelaxVecs v;
  v.fterm = buf + (size_t)(7 + 2 * m) * n4;
  v.rterm = v.fterm + n;
  v.ones = v.rterm + n;
  v.scal = v.ones + n;
  v.tmp = v.scal + 2;  // 8 scratch scalars
  double *dots = v.tmp + 8;  // up to 40 dot products
  v.bd.ls_lo = std::log(sig_lo);
  v.bd.ls_hi = std::log(sig_hi);
  v.bd.x_min = x_min;
  fill_kernel<<<(n + 255) / 256, 256, 0, s->st>>>(n, 1.0, v.ones);
  int st = cuda_status(cudaGetLastError());
  if (st == BTAM_OK) st = cuda_status(cudaMemsetAsync(s->err, 0, sizeof(int), s->st));
  // state at z (with the bounds), then its evaluation into (Z, G)
  auto eval_at = [&](const double *z, double *Z, double *G, double &r2) -> int {
    if (z) {
      BTAM_TRY(relax_apply(n, s->xb, z, z, 0.0, v.bd, s->pos, s->st));
      if (s->n_ghost > 0)
        BTAM_TRY(launch_ghost_refresh(n, s->n_ghost, s->pos, s->xb, s->code, s->owner, s->image,
                                      s->box, s->st));
    }
    v.z = Z;
    v.g = G;
    double f = 0.0;
    const int r = relax_eval(s, BTAM_FP64, v, f, r2);
    if (r != BTAM_OK) return r;
    unbeta_kernel<<<(n4 + 255) / 256, 256, 0, s->st>>>(n4, s->xb, G);
    return cuda_status(cudaGetLastError());
  };
  // dot products of a with each b[k], in one wait
  auto mdot = [&](const double *a, const std::vector<const double *> &bs, double *out) -> int {
    for (size_t k = 0; k < bs.size(); ++k) BTAM_TRY(vec_dot(n4, a, bs[k], dots + k, s->st));
    BTAM_TRY(cudaMemcpyAsync(out, dots, bs.size() * sizeof(double), cudaMemcpyDeviceToHost,
                             s->st));
    return cuda_status(cudaStreamSynchronize(s->st));
  };
  auto nrm = [&](const double *a, double &out) -> int {
    double d2 = 0.0;
    const int r = mdot(a, {a}, &d2);
    out = std::sqrt(d2);
    return r;
  };
  int evals = 0, it = 0, status = 0;
  double r2 = 0.0, fnorm = 0.0;
  if (st == BTAM_OK) st = eval_at(nullptr, X, F, r2);
  ++evals;
  if (st == BTAM_OK) st = nrm(F, fnorm);
  std::vector<double> Q((size_t)m * m, 0.0), xi(m), beta(m), H((size_t)m * m);
  double fminnorm = fnorm;
  int k_restart = 1, l = 1, ivec = 0, restart_count = 0;
  auto put = [&](int iv, const double *x, const double *f) -> int {
    BTAM_TRY(cudaMemcpyAsync(Xd[iv], x, n4 * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
    BTAM_TRY(cudaMemcpyAsync(Fd[iv], f, n4 * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
    return BTAM_OK;
  };
  if (st == BTAM_OK) st = put(0, X, F);
  if (st == BTAM_OK && std::sqrt(r2) <= tol) status = 1;
  for (int k = 1; st == BTAM_OK && status == 0 && k <= max_iter; ++k) {
    // z^M: the critical-point line search along -g from z.  Its first trial
    // is lambda = 1 damped so that no q moves by more than 0.05 A nor log
    // sigma by more than 0.05, and its result moves neither by more than
    // 0.5 (the reference's maxstep bound of 1e8 on lambda, in displacement)
    double pmax = 0.0;
    absmax_kernel<<<1, 256, 0, s->st>>>(n4, s->xb, F, v.tmp + 6);
    st = cuda_status(cudaMemcpyAsync(&pmax, v.tmp + 6, sizeof(double), cudaMemcpyDeviceToHost,
                                     s->st));
    if (st == BTAM_OK) st = cuda_status(cudaStreamSynchronize(s->st));
    if (st != BTAM_OK) break;
    const double lam_max = pmax > 0.0 ? std::min(1e8, kMaxMove / pmax) : 1e8;
    double lambda = pmax > kTrialMove ? kTrialMove / pmax : 1.0, r2M = 0.0, fty = 0.0;
    const double fty0 = fnorm * fnorm;
    if (fty0 >= 1e-15 * fnorm) {
      if ((st = cuda_status(vec_axpby(n4, 1.0, X, -lambda, F, D, s->st))) != BTAM_OK) break;
      if ((st = eval_at(D, XM, FM, r2M)) != BTAM_OK) break;
      ++evals;
      if ((st = mdot(FM, {F}, &fty)) != BTAM_OK) break;
      double sl = (fty - fty0) / lambda;  // secant slope from lambda_old = 0
      if (sl > 0.0) sl = -sl;
      if (sl != 0.0 && !(std::fabs(fty) / std::fabs(fty0) < 1e-8)) {
        double lu = lambda - fty / sl;
        if (lu < 1e-12) lu = lambda + fty / sl;
        if (std::isfinite(lu)) lambda = std::min(lu, lam_max);
      }
    }
    if ((st = cuda_status(vec_axpby(n4, 1.0, X, -lambda, F, D, s->st))) != BTAM_OK) break;
    if ((st = eval_at(D, XM, FM, r2M)) != BTAM_OK) break;
    ++evals;
    double fMnorm = 0.0;
    if ((st = nrm(FM, fMnorm)) != BTAM_OK) break;
    // z^A: the combination minimising |(1 - sum beta) g^M + sum beta g_i|
    {
      std::vector<const double *> fs(l);
      for (int i = 0; i < l; ++i) fs[i] = Fd[i];
      std::vector<double> col(l);
      if ((st = mdot(FM, fs, xi.data())) != BTAM_OK) break;
      if ((st = mdot(Fd[ivec], fs, col.data())) != BTAM_OK) break;
      for (int i = 0; i < l; ++i) Q[(size_t)i * m + ivec] = Q[(size_t)ivec * m + i] = col[i];
    }
    const double nu = fMnorm * fMnorm;
    for (int i = 0; i < l; ++i) beta[i] = nu - xi[i];
    for (int j = 0; j < l; ++j)
      for (int i = 0; i < l; ++i)
        H[(size_t)i * l + j] = Q[(size_t)i * m + j] - xi[i] - xi[j] + nu;
    if (l == 1) beta[0] = H[0] != 0.0 ? beta[0] / H[0] : 0.0;
    else lsq_sym(l, H.data(), beta.data());
    double alph = 0.0;
    for (int i = 0; i < l; ++i) alph += beta[i];
    if ((st = cuda_status(vec_axpby(n4, 1.0 - alph, XM, 0.0, XM, D, s->st))) != BTAM_OK) break;
    for (int i = 0; i < l && st == BTAM_OK; ++i)
      st = cuda_status(vec_axpby(n4, 1.0, D, beta[i], Xd[i], D, s->st));
    if (st != BTAM_OK) break;
    double r2A = 0.0;
    if ((st = eval_at(D, XA, FA, r2A)) != BTAM_OK) break;
    ++evals;
    if (fminnorm > fMnorm) fminnorm = fMnorm;
    double fAnorm = 0.0, dnorm = 0.0, dminnorm = -1.0;
    if ((st = nrm(FA, fAnorm)) != BTAM_OK) break;
    if ((st = cuda_status(vec_axpby(n4, 1.0, XA, -1.0, XM, D, s->st))) != BTAM_OK) break;
    if ((st = nrm(D, dnorm)) != BTAM_OK) break;
    for (int i = 0; i < l && st == BTAM_OK; ++i) {
      double dc = 0.0;
      st = cuda_status(vec_axpby(n4, 1.0, Xd[i], -1.0, XA, D, s->st));
      if (st == BTAM_OK) st = nrm(D, dc);
      if (dc < dminnorm || dminnorm < 0.0) dminnorm = dc;
    }
    if (st != BTAM_OK) break;
    // selection
    bool selA = fAnorm < gammaA * fminnorm;
    if (!(epsilonB * dnorm < dminnorm || std::sqrt(fnorm) < deltaB * std::sqrt(fminnorm)))
      selA = false;
    const double *xs = selA ? XA : XM, *fsel = selA ? FA : FM;
    st = cuda_status(cudaMemcpyAsync(X, xs, n4 * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
    if (st == BTAM_OK)
      st = cuda_status(
          cudaMemcpyAsync(F, fsel, n4 * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
    if (st != BTAM_OK) break;
    fnorm = selA ? fAnorm : fMnorm;
    r2 = selA ? r2A : r2M;
    // restart
    bool rs = false;
    if (epsilonB * dnorm > dminnorm && std::sqrt(fAnorm) > deltaB * std::sqrt(fminnorm)) rs = true;
    if (fAnorm > gammaC * fminnorm) rs = true;
    restart_count = rs ? restart_count + 1 : 0;
    ivec = k_restart % m;
    if (restart_count >= restart_it) {
      restart_count = 0;
      k_restart = 1;
      l = 1;
      ivec = 0;
      st = put(0, XM, FM);
    } else {
      if (l < m) ++l;
      ++k_restart;
      if (fminnorm > fnorm) fminnorm = fnorm;
      st = put(ivec, X, F);
    }
    it = k;
    if (!std::isfinite(fnorm)) st = BTAM_ERR_NONFINITE;
    if (std::sqrt(r2) <= tol) status = 1;
  }
  // leave the system at the selected iterate, evaluated; relax_eval has
  // read its objective and residual norm before the scratch is released
  double r2f = r2, ff = 0.0;
  if (st == BTAM_OK) {
    v.z = XM;
    v.g = FM;
    st = cuda_status(relax_apply(n, s->xb, X, X, 0.0, v.bd, s->pos, s->st));
    if (st == BTAM_OK && s->n_ghost > 0)
      st = cuda_status(launch_ghost_refresh(n, s->n_ghost, s->pos, s->xb, s->code, s->owner,
                                            s->image, s->box, s->st));
    if (st == BTAM_OK) st = relax_eval(s, BTAM_FP64, v, ff, r2f);
  }
  dfree(buf, s->st);
  if (info) {
    info[0] = std::sqrt(r2f);
    info[1] = it;
    info[2] = evals;
    info[3] = ff;
    info[4] = status;
  }
  return st;
}

}  // namespace

extern "C" {

int btam_relax(btam_system *s, int mode, double tol, int max_iter, int m, const double *bounds,
               double *info) {
  if (!s || !(tol > 0.0) || max_iter < 0 || m < 1 || m > 16) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  if (mode < 0 || mode > 4) return BTAM_ERR_ARG;
  if (mode == BTAM_RELAX_NGMRES) return relax_ngmres(s, tol, max_iter, m, bounds, info);
  if (mode == BTAM_RELAX_NEWTON) {  // max_iter Newton steps, m unused
    double inf6[6];
    const int st = btam_relax_newton(s, tol, max_iter, 300, bounds, inf6);
    if (info)
      for (int c = 0; c < 5; ++c) info[c] = inf6[c];
    return st;
  }
  const double sig_lo = bounds ? bounds[0] : 0.001, sig_hi = bounds ? bounds[1] : 0.4,
               x_min = bounds ? bounds[2] : 0.01;
  if (!(sig_lo > 0.0 && sig_hi > sig_lo && x_min >= 0.0)) return BTAM_ERR_ARG;
  const int n = s->n_real, n4 = 4 * n;
  // layout: z g p z0 g0 work (n4 each), S[m] Y[m] (n4 each), fterm rterm ones (n), small
  const size_t need = (size_t)(6 + 2 * m) * n4 + 3 * (size_t)n + 64;
  if (!s->rv || s->relax_m < m) {
    BTAM_TRY(dalloc(s->rv, s->st, need));
    s->relax_m = m;
  }
  RelaxVecs v;
  double *b = s->rv;
  v.z = b; v.g = b + n4; v.p = b + 2 * n4; v.z0 = b + 3 * n4; v.g0 = b + 4 * n4;
  v.work = b + 5 * n4;
  for (int k = 0; k < m; ++k) {
    v.S[k] = b + (size_t)(6 + k) * n4;
    v.Y[k] = b + (size_t)(6 + m + k) * n4;
  }
  v.fterm = b + (size_t)(6 + 2 * m) * n4;
  v.rterm = v.fterm + n;
  v.ones = v.rterm + n;
  v.scal = v.ones + n;
  v.tmp = v.scal + 2;       // 8 scratch scalars
  v.rho = v.tmp + 8;        // m
  v.alpha = v.rho + 16;     // m
  v.bd.ls_lo = std::log(sig_lo);
  v.bd.ls_hi = std::log(sig_hi);
  v.bd.x_min = x_min;
  fill_kernel<<<(n + 255) / 256, 256, 0, s->st>>>(n, 1.0, v.ones);
  BTAM_TRY(cudaGetLastError());
  BTAM_TRY(cudaMemsetAsync(s->err, 0, sizeof(int), s->st));

  int prec = (mode == 0) ? BTAM_FP64 : BTAM_FP32C;
  const double switch_tol = 1e-5;  // FP32C noise floor is ~1e-6
  double f, r2;
  int evals = 0, it = 0, st;
  if ((st = relax_eval(s, prec, v, f, r2)) != BTAM_OK) return st;
  ++evals;
  std::vector<int> order;
  std::vector<double> rho_h(16, 0.0);
  bool stalled = false;
  for (; it < max_iter; ++it) {
    if (mode == 1 && prec == BTAM_FP32C && std::sqrt(r2) < switch_tol) {
      prec = BTAM_FP64;
      order.clear();
      if ((st = relax_eval(s, prec, v, f, r2)) != BTAM_OK) return st;
      ++evals;
    }
    if (std::sqrt(r2) <= tol) break;
    BTAM_TRY(lbfgs_direction(n4, v.g, v.S, v.Y, v.rho, order.data(), (int)order.size(), v.p,
                             v.work, v.alpha, v.tmp, s->st));
    double gp = dev_dot(s, v, n4, v.g, v.p);
    if (!(gp < 0.0)) {  // not a descent direction: restart from steepest descent
      order.clear();
      BTAM_TRY(lbfgs_direction(n4, v.g, v.S, v.Y, v.rho, nullptr, 0, v.p, v.work, v.alpha, v.tmp,
                               s->st));
      gp = dev_dot(s, v, n4, v.g, v.p);
    }
    // first step of a history: move no q (A) or log sigma by more than 0.05;
    // this step also seeds the curvature scale of the history
    double alpha = 1.0;
    if (order.empty()) {
      absmax_kernel<<<1, 256, 0, s->st>>>(n4, s->xb, v.p, v.tmp + 6);
      double pmax = 0.0;
      BTAM_TRY(cudaMemcpyAsync(&pmax, v.tmp + 6, sizeof(double), cudaMemcpyDeviceToHost, s->st));
      BTAM_TRY(cudaStreamSynchronize(s->st));
      if (pmax > 0.05) alpha = 0.05 / pmax;
    }
    BTAM_TRY(cudaMemcpyAsync(v.z0, v.z, n4 * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
    BTAM_TRY(cudaMemcpyAsync(v.g0, v.g, n4 * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
    const double f0 = f, r20 = r2;
    bool ok = false;
    for (int ls = 0; ls < 30; ++ls) {
      BTAM_TRY(relax_apply(n, s->xb, v.z0, v.p, alpha, v.bd, s->pos, s->st));
      if (s->n_ghost > 0)
        BTAM_TRY(launch_ghost_refresh(n, s->n_ghost, s->pos, s->xb, s->code, s->owner, s->image,
                                      s->box, s->st));
      if ((st = relax_eval(s, prec, v, f, r2)) != BTAM_OK) return st;
      ++evals;
      // Armijo decrease of F; once F's changes are below its rounding (about
      // 1e-7 relative in the FP32C form, 1e-13 in FP64), a step that lowers
      // the residual is accepted instead
      const double noise = (prec == BTAM_FP32C ? 1e-7 : 1e-13) * std::fabs(f0);
      if (f <= f0 + 1e-4 * alpha * gp || (std::fabs(f - f0) <= noise && r2 < r20)) {
        ok = true;
        break;
      }
      alpha *= 0.5;
    }
    if (!ok) {  // no decrease resolvable at this precision: restore and stop
      BTAM_TRY(relax_apply(n, s->xb, v.z0, v.p, 0.0, v.bd, s->pos, s->st));
      if (s->n_ghost > 0)
        BTAM_TRY(launch_ghost_refresh(n, s->n_ghost, s->pos, s->xb, s->code, s->owner, s->image,
                                      s->box, s->st));
      if (mode == 1 && prec == BTAM_FP32C) prec = BTAM_FP64;  // finish in FP64
      if ((st = relax_eval(s, prec, v, f, r2)) != BTAM_OK) return st;
      ++evals;
      if (!order.empty()) {  // restart from steepest descent before giving up
        order.clear();
        continue;
      }
      stalled = true;
      (void)r20;
      break;
    }
    // history pair (newest last, oldest dropped)
    int slot = (int)order.size() < m ? (int)order.size() : order.front();
    if ((int)order.size() == m) order.erase(order.begin());
    BTAM_TRY(lbfgs_push(n4, v.z, v.z0, v.g, v.g0, v.S[slot], v.Y[slot], v.tmp, s->st));
    double sy = 0.0;
    BTAM_TRY(cudaMemcpyAsync(&sy, v.tmp, sizeof(double), cudaMemcpyDeviceToHost, s->st));
    BTAM_TRY(cudaStreamSynchronize(s->st));
    if (sy > 1e-300) {
      rho_h[slot] = 1.0 / sy;
      BTAM_TRY(cudaMemcpyAsync(v.rho + slot, &rho_h[slot], sizeof(double), cudaMemcpyHostToDevice,
                               s->st));
      order.push_back(slot);
    }
  }
  if (info) {
    info[0] = std::sqrt(r2);
    info[1] = it;
    info[2] = evals;
    info[3] = f;
    info[4] = (std::sqrt(r2) <= tol) ? 1.0 : (stalled ? -1.0 : 0.0);
  }
  BTAM_TRY(cudaStreamSynchronize(s->st));
  return BTAM_OK;
}

int btam_relax_newton(btam_system *s, double tol, int max_newton, int max_cg,
                      const double *bounds, double *info) {
  if (!s || !(tol > 0.0) || max_newton < 0 || max_cg < 1) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  const double sig_lo = bounds ? bounds[0] : 0.001, sig_hi = bounds ? bounds[1] : 0.4,
               x_min = bounds ? bounds[2] : 0.01;
  if (!(sig_lo > 0.0 && sig_hi > sig_lo && x_min >= 0.0)) return BTAM_ERR_ARG;
  const int n = s->n_real, n4 = 4 * n;
  // layout: z g p z0 g0 r d hd (n4 each), fterm rterm ones (n), small; the
  // block of btam_relax with m = 1 has exactly this size
  const size_t need = (size_t)8 * n4 + 3 * (size_t)n + 64;
  if (!s->rv) {
    BTAM_TRY(dalloc(s->rv, s->st, need));
    s->relax_m = 1;
  }
  RelaxVecs v;
  double *b = s->rv;
  v.z = b; v.g = b + n4; v.p = b + 2 * n4; v.z0 = b + 3 * n4; v.g0 = b + 4 * n4;
  double *r = b + 5 * n4, *d = b + 6 * n4, *hd = b + 7 * n4;
  v.work = nullptr;
  v.fterm = b + (size_t)8 * n4;
  v.rterm = v.fterm + n;
  v.ones = v.rterm + n;
  v.scal = v.ones + n;
  v.tmp = v.scal + 2;
  v.bd.ls_lo = std::log(sig_lo);
  v.bd.ls_hi = std::log(sig_hi);
  v.bd.x_min = x_min;
  fill_kernel<<<(n + 255) / 256, 256, 0, s->st>>>(n, 1.0, v.ones);
  BTAM_TRY(cudaGetLastError());
  BTAM_TRY(cudaMemsetAsync(s->err, 0, sizeof(int), s->st));
  auto move = [&](const double *z0, const double *p, double alpha) -> int {
    BTAM_TRY(relax_apply(n, s->xb, z0, p, alpha, v.bd, s->pos, s->st));
    if (s->n_ghost > 0)
      BTAM_TRY(launch_ghost_refresh(n, s->n_ghost, s->pos, s->xb, s->code, s->owner, s->image,
                                    s->box, s->st));
    return BTAM_OK;
  };
  double f, r2;
  int evals = 0, it = 0, cg_total = 0, st;
  if ((st = relax_eval(s, BTAM_FP64, v, f, r2)) != BTAM_OK) return st;
  ++evals;
  bool stalled = false;
  double lam = 0.0;  // damping of the Newton system
  for (; it < max_newton; ++it) {
    if (std::sqrt(r2) <= tol) break;
    BTAM_TRY(cudaMemcpyAsync(v.z0, v.z, n4 * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
    BTAM_TRY(cudaMemcpyAsync(v.g0, v.g, n4 * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
    const double f0 = f, r20 = r2;
    const double gg = dev_dot(s, v, n4, v.g0, v.g0), gnorm = std::sqrt(gg);
    const double zz = dev_dot(s, v, n4, v.z0, v.z0);
    // conjugate gradients on (H + lam I) p = -g, H d by a forward
    // difference of the gradient (one evaluation per iteration), forcing
    // term min(0.5, sqrt|g|).  Negative curvature raises lam past it and
    // restarts (at most 4 times); lam shrinks after full steps.
    const double eta = std::min(0.5, std::sqrt(gnorm));
    for (int restart = 0; restart < 5; ++restart) {
      BTAM_TRY(cudaMemsetAsync(v.p, 0, n4 * sizeof(double), s->st));
      BTAM_TRY(vec_axpby(n4, -1.0, v.g0, 0.0, v.g0, r, s->st));
      BTAM_TRY(cudaMemcpyAsync(d, r, n4 * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
      double rr = gg;
      bool negative = false;
      for (int k = 0; k < max_cg; ++k) {
        const double dd = dev_dot(s, v, n4, d, d);
        if (!(dd > 0.0)) break;
        const double eps = 1.4901161193847656e-08 * (1.0 + std::sqrt(zz)) / std::sqrt(dd);
        if ((st = move(v.z0, d, eps)) != BTAM_OK) return st;
        if ((st = relax_eval(s, BTAM_FP64, v, f, r2)) != BTAM_OK) return st;
        ++evals;
        ++cg_total;
        BTAM_TRY(vec_axpby(n4, 1.0 / eps, v.g, -1.0 / eps, v.g0, hd, s->st));
        if (lam > 0.0) BTAM_TRY(vec_axpby(n4, 1.0, hd, lam, d, hd, s->st));
        const double dhd = dev_dot(s, v, n4, d, hd);
        if (!(dhd > 0.0)) {
          if (restart < 4) {
            lam = std::max(4.0 * lam, 2.0 * (lam - dhd / dd));
            negative = true;
          } else if (k == 0) {
            BTAM_TRY(cudaMemcpyAsync(v.p, d, n4 * sizeof(double), cudaMemcpyDeviceToDevice,
                                     s->st));
          }
          break;
        }
        const double a = rr / dhd;
        BTAM_TRY(vec_axpby(n4, 1.0, v.p, a, d, v.p, s->st));
        BTAM_TRY(vec_axpby(n4, 1.0, r, -a, hd, r, s->st));
        const double rr1 = dev_dot(s, v, n4, r, r);
        if (std::sqrt(rr1) <= eta * gnorm) break;
        BTAM_TRY(vec_axpby(n4, 1.0, r, rr1 / rr, d, d, s->st));
        rr = rr1;
      }
      if (!negative) break;
    }
    double gp = dev_dot(s, v, n4, v.g0, v.p);
    if (!(gp < 0.0)) {  // no descent: steepest descent
      BTAM_TRY(vec_axpby(n4, -1.0, v.g0, 0.0, v.g0, v.p, s->st));
      gp = -gg;
    }
    // no q (A) or log sigma moves by more than 0.2 in one step
    double alpha = 1.0;
    absmax_kernel<<<1, 256, 0, s->st>>>(n4, s->xb, v.p, v.tmp + 6);
    double pmax = 0.0;
    BTAM_TRY(cudaMemcpyAsync(&pmax, v.tmp + 6, sizeof(double), cudaMemcpyDeviceToHost, s->st));
    BTAM_TRY(cudaStreamSynchronize(s->st));
    if (pmax > 0.2) alpha = 0.2 / pmax;
    const double alpha0 = alpha;
    bool ok = false;
    for (int ls = 0; ls < 30; ++ls) {
      if ((st = move(v.z0, v.p, alpha)) != BTAM_OK) return st;
      if ((st = relax_eval(s, BTAM_FP64, v, f, r2)) != BTAM_OK) return st;
      ++evals;
      const double noise = 1e-13 * std::fabs(f0);
      if (f <= f0 + 1e-4 * alpha * gp || (std::fabs(f - f0) <= noise && r2 < r20)) {
        ok = true;
        break;
      }
      alpha *= 0.5;
    }
    if (ok && alpha == alpha0) lam *= 0.25;
    else if (ok) lam = std::max(2.0 * lam, 1e-3);
    if (!ok) {  // restore the last point and stop
      if ((st = move(v.z0, v.p, 0.0)) != BTAM_OK) return st;
      if ((st = relax_eval(s, BTAM_FP64, v, f, r2)) != BTAM_OK) return st;
      ++evals;
      stalled = true;
      break;
    }
  }
  if (info) {
    info[0] = std::sqrt(r2);
    info[1] = it;
    info[2] = evals;
    info[3] = f;
    info[4] = (std::sqrt(r2) <= tol) ? 1.0 : (stalled ? -1.0 : 0.0);
    info[5] = cg_total;
  }
  BTAM_TRY(cudaStreamSynchronize(s->st));
  return BTAM_OK;
}

int btam_dmd_setup(btam_system *s) {
  if (!s) return BTAM_ERR_ARG;
  if (!s->built) return BTAM_ERR_NOT_BUILT;
  const int n = s->n_real;
  int total = 0;
  BTAM_TRY(cudaMemsetAsync(s->err, 0, sizeof(int), s->st));
  int st = build_list(s, n + s->n_ghost, n, BTAM_R_CUTOFF_EB, BTAM_MAX_CHEMICAL_NEIGHS, 1, 1,
                      s->doffs, s->dq_cap, s->didx, s->didx_cap, total);
  if (st != BTAM_OK) return st;
  s->d_pairs = total;
  for (long long **p : {&s->X, &s->X0})
    BTAM_TRY(dalloc(*p, s->st, n));
  BTAM_TRY(dalloc(s->dtot, s->st, 2));
  BTAM_TRY(dalloc(s->dctl, s->st, 3));
  BTAM_TRY(cudaMemsetAsync(s->dctl, 0, 3 * sizeof(unsigned long long), s->st));
  BTAM_TRY(dalloc(s->mu, s->st, n));
  BTAM_TRY(dalloc(s->dact, s->st, n));
  BTAM_TRY(dalloc(s->ddeg, s->st, n));
  BTAM_TRY(dmd_init(n, s->xb, s->code, s->X, s->st));
  BTAM_TRY(dmd_commit_all(n, s->code, s->X, s->xb, s->st));
  if (s->n_ghost > 0)
    BTAM_TRY(launch_ghost_refresh(n, s->n_ghost, s->pos, s->xb, s->code, s->owner, s->image,
                                  s->box, s->st));
  BTAM_TRY(cudaStreamSynchronize(s->st));
  s->dmd_ready = true;
  return BTAM_OK;
}

}  // extern "C"

namespace {

// The reference's diffusion parameters (Variables.hpp:68-92) unless given.
int dmd_params(const double *params, DmdParams &prm) {
  prm.dt = params ? params[0] : 4e-4;
  prm.Df = params ? params[1] : 0.045;
  prm.dr = params ? params[2] : 3.2;
  prm.min_dx = params ? params[3] : 1e-8;
  prm.max_x = params ? params[4] : 0.9;
  return (prm.dt >= 0.0 && prm.Df >= 0.0 && prm.dr > 0.0 && prm.max_x > 0.0) ? BTAM_OK
                                                                              : BTAM_ERR_ARG;
}

DmdArgs dmd_args(btam_system *s) {
  DmdArgs a;
  a.n = s->n_real;
  a.xb = s->xb;
  a.code = s->code;
  a.owner = s->owner;
  a.Rx = s->Rx;
  a.gamma = s->gamma;
  a.moffs = s->offs;
  a.midx = s->idx;
  a.doffs = s->doffs;
  a.didx = s->didx;
  a.X = s->X;
  a.X0 = s->X0;
  a.mu = s->mu;
  a.active = s->dact;
  a.deg = s->ddeg;
  a.ctl = s->dctl;
  return a;
}

// Images follow their owners' new occupancies.
int dmd_refresh_images(btam_system *s) {
  if (s->n_ghost > 0)
    BTAM_TRY(launch_ghost_refresh(s->n_real, s->n_ghost, s->pos, s->xb, s->code, s->owner,
                                  s->image, s->box, s->st));
  return BTAM_OK;
}

int dmd_finish(btam_system *s, long long *total_quanta) {
  if (total_quanta) {
    BTAM_TRY(dmd_total(s->n_real, s->code, s->X, s->dtot, s->st));
    BTAM_TRY(cudaMemcpyAsync(total_quanta, s->dtot, 2 * sizeof(long long), cudaMemcpyDeviceToHost,
                             s->st));
  }
  return read_err(s);
}

}  // namespace

extern "C" {

int btam_dmd_step(btam_system *s, int precision, int nsteps, const double *params,
                  long long *total_quanta) {
  if (!s || nsteps < 0) return BTAM_ERR_ARG;
  if (!s->dmd_ready) return BTAM_ERR_NOT_BUILT;
  DmdParams prm;
  if (dmd_params(params, prm) != BTAM_OK) return BTAM_ERR_ARG;
  BTAM_TRY(cudaMemsetAsync(s->err, 0, sizeof(int), s->st));
  const DmdArgs a = dmd_args(s);
  for (int k = 0; k < nsteps; ++k) {
    // chemical potentials at the current x; positions and widths do not
    // move during the steps, so the pair-rule sums of the first are kept
    int st = enqueue_eval(s, precision, true, k > 0);
    if (st != BTAM_OK) return st;
    BTAM_TRY(dmd_step(a, prm, s->st));
    if ((st = dmd_refresh_images(s)) != BTAM_OK) return st;
  }
  return dmd_finish(s, total_quanta);
}

int btam_dmd_step_ctl(btam_system *s, int precision, int nsteps, const double *params,
                      long long *total_quanta, double *stats) {
  if (!s || nsteps < 0) return BTAM_ERR_ARG;
  if (!s->dmd_ready) return BTAM_ERR_NOT_BUILT;
  DmdParams prm;
  if (dmd_params(params, prm) != BTAM_OK) return BTAM_ERR_ARG;
  const double max_dx = params ? params[5] : 0.05;
  const double max_sub_d = params ? params[6] : 64.0;
  if (!(max_dx > 0.0) || !(max_sub_d >= 1.0 && max_sub_d <= 1e6)) return BTAM_ERR_ARG;
  const long long max_sub = (long long)max_sub_d;
  BTAM_TRY(cudaMemsetAsync(s->err, 0, sizeof(int), s->st));
  const DmdArgs a = dmd_args(s);
  unsigned long long clip0 = 0;
  BTAM_TRY(copy_sync(&clip0, s->dctl + 2, sizeof(clip0), cudaMemcpyDeviceToHost, s->st));
  long long subs = 0, split = 0;
  double worst = 0.0;
  bool recs = false;  // the pair-rule sums of this call's positions are made
  for (int k = 0; k < nsteps; ++k) {
    int st = enqueue_eval(s, precision, true, recs);
    if (st != BTAM_OK) return st;
    recs = true;
    BTAM_TRY(dmd_prepare(a, s->st));
    BTAM_TRY(dmd_control(a, prm, max_dx, s->st));
    unsigned long long bits[2] = {0, 0};
    BTAM_TRY(copy_sync(bits, s->dctl, sizeof(bits), cudaMemcpyDeviceToHost, s->st));
    double r[2];
    std::memcpy(r, bits, sizeof(r));
    const double need = std::max(r[0], r[1]);
    if (!std::isfinite(need)) return BTAM_ERR_NONFINITE;
    worst = std::max(worst, need);
    const long long m = std::min(max_sub, std::max(1ll, (long long)std::ceil(need)));
    DmdParams sub = prm;
    sub.dt = prm.dt / (double)m;
    for (long long j = 0; j < m; ++j) {
      if (j > 0) {  // fresh chemical potentials for every later sub-step
        if ((st = enqueue_eval(s, precision, true, true)) != BTAM_OK) return st;
        BTAM_TRY(dmd_prepare(a, s->st));
      }
      BTAM_TRY(dmd_apply(a, sub, s->st));
      if ((st = dmd_refresh_images(s)) != BTAM_OK) return st;
    }
    subs += m;
    split += m > 1;
  }
  int st = dmd_finish(s, total_quanta);
  if (stats) {
    unsigned long long clip1 = 0;
    BTAM_TRY(copy_sync(&clip1, s->dctl + 2, sizeof(clip1), cudaMemcpyDeviceToHost, s->st));
    stats[0] = (double)subs;
    stats[1] = (double)split;
    stats[2] = (double)(clip1 - clip0);
    stats[3] = worst;
  }
  return st;
}

int btam_dmd_run(btam_system *s, int precision, int nsteps, const double *params,
                 int relax_every, int relax_mode, double relax_tol, int relax_max_iter,
                 long long *total_quanta, double *stats) {
  if (!s || nsteps < 0 || relax_every < 0) return BTAM_ERR_ARG;
  if (!s->dmd_ready) return BTAM_ERR_NOT_BUILT;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  int done = 0;
  while (done < nsteps) {
    const int k = relax_every > 0 ? std::min(relax_every, nsteps - done) : nsteps - done;
    double st4[4] = {0, 0, 0, 0};
    int st = btam_dmd_step_ctl(s, precision, k, params, nullptr, st4);
    if (st != BTAM_OK) return st;
    for (int c = 0; c < 3; ++c) acc[c] += st4[c];
    acc[3] = std::max(acc[3], st4[3]);
    done += k;
    if (relax_every > 0 && done % relax_every == 0) {
      // the mechanical state follows the new occupancies
      double info[5] = {0, 0, 0, 0, 0};
      st = btam_relax(s, relax_mode, relax_tol, relax_max_iter,
                      relax_mode == BTAM_RELAX_NGMRES ? 3 : 8, nullptr, info);
      if (st != BTAM_OK) return st;
      acc[4] += 1.0;
      acc[5] += info[2];
    }
  }
  if (stats)
    for (int c = 0; c < 6; ++c) stats[c] = acc[c];
  BTAM_TRY(cudaMemsetAsync(s->err, 0, sizeof(int), s->st));
  return dmd_finish(s, total_quanta);
}

int btam_dmd_clip_count(btam_system *s, long long *clipped) {
  if (!s || !clipped) return BTAM_ERR_ARG;
  if (!s->dmd_ready) return BTAM_ERR_NOT_BUILT;
  unsigned long long c = 0;
  BTAM_TRY(copy_sync(&c, s->dctl + 2, sizeof(c), cudaMemcpyDeviceToHost, s->st));
  *clipped = (long long)c;
  return BTAM_OK;
}

int btam_dmd_occupancy(btam_system *s, double *x, long long *quanta, double *mu) {
  if (!s) return BTAM_ERR_ARG;
  if (!s->dmd_ready) return BTAM_ERR_NOT_BUILT;
  const int n = s->n_real;
  if (quanta)
    BTAM_TRY(cudaMemcpyAsync(quanta, s->X, n * sizeof(long long), cudaMemcpyDeviceToHost, s->st));
  if (mu) BTAM_TRY(cudaMemcpyAsync(mu, s->mu, n * sizeof(double), cudaMemcpyDeviceToHost, s->st));
  if (x) {
    std::vector<double2> h(n);
    BTAM_TRY(cudaMemcpyAsync(h.data(), s->xb, n * sizeof(double2), cudaMemcpyDeviceToHost, s->st));
    BTAM_TRY(cudaStreamSynchronize(s->st));
    for (int i = 0; i < n; ++i) x[i] = h[i].x;
  }
  return read_err(s);
}

int btam_dmd_graph_copy(const btam_system *s, int *offs, int *idx, long long idx_cap) {
  if (!s || !offs) return BTAM_ERR_ARG;
  if (!s->dmd_ready) return BTAM_ERR_NOT_BUILT;
  BTAM_TRY(copy_sync(offs, s->doffs, (s->n_real + 1) * sizeof(int), cudaMemcpyDeviceToHost, s->st));
  if (idx) {
    if (idx_cap < s->d_pairs) return BTAM_ERR_ARG;
    BTAM_TRY(copy_sync(idx, s->didx, s->d_pairs * sizeof(int), cudaMemcpyDeviceToHost, s->st));
  }
  return BTAM_OK;
}

int btam_system_get_state(btam_system *s, double *q, double *sigma, double *x) {
  if (!s) return BTAM_ERR_ARG;
  const int n = s->n_real;
  std::vector<double4> hp(n);
  std::vector<double2> hx(n);
  BTAM_TRY(cudaMemcpyAsync(hp.data(), s->pos, n * sizeof(double4), cudaMemcpyDeviceToHost, s->st));
  BTAM_TRY(cudaMemcpyAsync(hx.data(), s->xb, n * sizeof(double2), cudaMemcpyDeviceToHost, s->st));
  BTAM_TRY(cudaStreamSynchronize(s->st));
  for (int i = 0; i < n; ++i) {
    if (q) {
      q[3 * i] = hp[i].x;
      q[3 * i + 1] = hp[i].y;
      q[3 * i + 2] = hp[i].z;
    }
    if (sigma) sigma[i] = hp[i].w;
    if (x) x[i] = hx[i].x;
  }
  return BTAM_OK;
}

}  // extern "C"
