// Batched evaluation: many independent systems (cells or clusters of uneven
// size) evaluated by the same kernels as one system (pass 1 with its
// pair-rule kernel, pass 2 with its pair and site kernels, per-system
// totals), on persistent grids, replayed as a single CUDA graph.
//
// Layout in HBM: the real sites of every system first (system k owns rows
// [R_k, R_k + n_k)), then the periodic images of every system (system k owns
// rows [N + G_k, N + G_k + g_k), N = total real sites).  Neighbour indices,
// owners and CSR offsets are renumbered into this layout once, on the device,
// when the batch is made; the kernels of adp_kernels.cu then see one large
// system whose sites happen to belong to different cells, which is exactly
// what they already handle: a warp per site, each site reading only its own
// neighbours, and per-site beta / gamma.  Because every per-site result is
// computed by the same instructions in the same order as for the system on
// its own, batch results equal the single-system results bitwise; the
// per-system totals use the same reduction tree as a single system.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "../../include/btam.h"
#include "adp_kernels.cuh"
#include "internal.cuh"

namespace {

// Renumbers system k's rows into the batch layout: rows below n_real go to
// base_real + row, image rows to base_img + (row - n_real).
__device__ __forceinline__ int batch_row(int j, int n_real, int base_real, int base_img) {
  return j < n_real ? base_real + j : base_img + (j - n_real);
}

__global__ void remap_idx_kernel(long long n, const int *src, int *dst, int n_real,
                                 int base_real, int base_img) {
  long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) dst[p] = batch_row(src[p], n_real, base_real, base_img);
}

__global__ void remap_owner_kernel(int n_all, const int *src, int *dst_real, int *dst_img,
                                   int n_real, int base_real) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_all) return;
  int o = base_real + src[i];
  if (i < n_real)
    dst_real[i] = o;
  else
    dst_img[i - n_real] = o;
}

__global__ void shift_offs_kernel(int n, const int *src, int *dst, int base) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = base + src[i];
}

// Reverse slots keep -1 (no reverse pair) and move by the pair base otherwise.
__global__ void shift_rev_kernel(long long n, const int *src, int *dst, int base) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[i] < 0 ? -1 : base + src[i];
}

// Slot-to-owned-pair links (2 t + direction) move by twice the owned-pair base.
__global__ void shift_slot_own_kernel(long long n, const int *src, int *dst, int own_base) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[i] < 0 ? -1 : 2 * own_base + src[i];
}

inline int blocks_of(long long n, int per) { return (int)((n + per - 1) / per); }

// Copies the site rows (real, then images) of the systems in the table into
// their batch rows: blockIdx.y picks the system, the x dimension strides rows.
__global__ void batch_gather_kernel(BatchXfer t, double4 *pos, double2 *xb,
                                    unsigned char *site_on) {
  const BatchXfer::Sys &d = t.sys[blockIdx.y];
  const int rows = d.n + d.g;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
    const int dst = r < d.n ? d.R + r : d.G + (r - d.n);
    pos[dst] = d.pos[r];
    xb[dst] = d.xb[r];
    if (r < d.n) site_on[dst] = 1;  // this system is evaluated in the round
  }
}

// Copies the results of the systems in the table from their batch rows into
// their own buffers, with their totals (4 each) and the batch's error bits.
__global__ void batch_scatter_kernel(BatchXfer t, const double *rho, const double *V0,
                                     const double *S0, const double *Rq, const double *Rs,
                                     const double *Rx, const double *totals, const int *err) {
  const BatchXfer::Sys &d = t.sys[blockIdx.y];
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  for (int r = tid; r < d.n; r += gridDim.x * blockDim.x) {
    const int src = d.R + r;
    d.rho[r] = rho[src];
    d.V0[r] = V0[src];
    d.S0[r] = S0[src];
    d.Rq[3 * (size_t)r] = Rq[3 * (size_t)src];
    d.Rq[3 * (size_t)r + 1] = Rq[3 * (size_t)src + 1];
    d.Rq[3 * (size_t)r + 2] = Rq[3 * (size_t)src + 2];
    d.Rs[r] = Rs[src];
    d.Rx[r] = Rx[src];
  }
  if (tid < 4) d.totals[tid] = totals[4 * (size_t)d.k + tid];
  if (tid == 0 && *err) atomicOr(d.err, *err);
}

}  // namespace

struct btam_batch {
  const btam_tables *T = nullptr;
  int device = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t ev = nullptr;
  std::vector<btam_system *> sys;
  std::vector<int> base_real, base_img;  // per system
  std::vector<long long> base_pair;
  int n_sys = 0, n_real = 0, n_all = 0;
  long long n_pairs = 0;
  int *seg = nullptr;  // n_sys + 1 real-site offsets
  double4 *pos = nullptr;
  double2 *xb = nullptr;
  int *code = nullptr, *owner = nullptr;
  double *gamma = nullptr;
  int *offs = nullptr, *idx = nullptr;
  // undirected pass 2: reverse slots, owned slots and their sites, slot buffer
  Site32 *s32 = nullptr;  // packed neighbour rows of the FP32C kernels [all]
  SiteB *sb = nullptr;
  Site64 *s64 = nullptr;  // packed neighbour rows of the FP64 kernels [all]
  // the systems a served round evaluates (1 per real site), used while masked
  unsigned char *site_on = nullptr;
  bool masked = false;
  int *rev = nullptr, *slot_own = nullptr, *own_p = nullptr, *own_u = nullptr;
  int n_own = 0;
  char *pbuf = nullptr;
  size_t pbuf_bytes = 0, pbuf_elem = 0;
  double *rho = nullptr, *V0 = nullptr, *S0 = nullptr, *selfx = nullptr, *Rq = nullptr,
         *Rs = nullptr, *Rx = nullptr, *totals = nullptr;
  double *mom64 = nullptr;
  float *mom32 = nullptr;
  int *err = nullptr;
  // launch variants per arithmetic form (0 FP64, 1 FP32C); persistent grids
  // unless btam_batch_autotune finds a full grid faster
  int variant1[2] = {kPersistent, kPersistent}, variant2[2] = {kPersistent, kPersistent};
  // instantiated graph per form and the variants it was captured with
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  int exec_v1[2] = {-1, -1}, exec_v2[2] = {-1, -1};
  const char *exec_pbuf[2] = {nullptr, nullptr};  // slot buffer the graph writes
};

namespace {

template <class R> EvalArgs<R> batch_args(btam_batch *b, R *mom, const RadialView<R> &T) {
  EvalArgs<R> a;
  a.n_real = b->n_real;
  a.n_all = b->n_all;
  if (sizeof(R) == 4) {
    a.s32 = b->s32;
    a.sb = b->sb;
  } else {
    a.s64 = b->s64;
  }
  if (b->masked) a.site_on = b->site_on;
  a.pos = b->pos;
  a.xb = b->xb;
  a.code = b->code;
  a.owner = b->owner;
  a.gamma = b->gamma;
  a.offs = b->offs;
  a.idx = b->idx;
  a.T = T;
  a.emb[0] = b->T->v64.t[T_F_MG];
  a.emb[1] = b->T->v64.t[T_F_H];
  a.mass[0] = b->T->host.mass_mg;
  a.mass[1] = b->T->host.mass_h;
  a.mom = mom;
  a.rho = b->rho;
  a.V0 = b->V0;
  a.S0 = b->S0;
  a.selfx = b->selfx;
  a.Rq = b->Rq;
  a.Rs = b->Rs;
  a.Rx = b->Rx;
  a.err = b->err;
  a.rev = b->rev;
  a.own_p = b->own_p;
  a.own_u = b->own_u;
  a.n_own = b->n_own;
  a.pbuf = reinterpret_cast<R *>(b->pbuf);
  a.slot_own = b->slot_own;
  if (b->pbuf) {
    a.pgx = a.pbuf + pbuf_gx_offset(b->n_pairs);
    a.prec1 = a.pbuf + pbuf_prec1_offset(b->n_pairs);
    a.prec2 = a.prec1 + prec2_offset(b->n_own);
  }
  return a;
}

// Slot records (5 R per slot) then the pair-rule records (prec1, prec2);
// layout in pbuf_values and its helpers.
int batch_pbuf(btam_batch *b, size_t elem) {
  if (elem < b->pbuf_elem) elem = b->pbuf_elem;
  const size_t need =
      pbuf_values(b->n_pairs > 0 ? b->n_pairs : 1, b->n_own) * elem;
  b->pbuf_elem = elem;
  if (need <= b->pbuf_bytes) return BTAM_OK;
  BTAM_TRY(dalloc(b->pbuf, b->st, need));
  b->pbuf_bytes = need;
  return BTAM_OK;
}

int batch_read_err(btam_batch *b) {
  int bits = 0;
  cudaError_t e = cudaMemcpyAsync(&bits, b->err, sizeof(int), cudaMemcpyDeviceToHost, b->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->err, 0, sizeof(int), b->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->st);
  if (e != cudaSuccess) return cuda_status(e);
  return status_from_bits(bits);
}

// Copies system k's site rows (real and images) into the batch, ordered
// after everything already enqueued on the system's stream.
int copy_sites(btam_batch *b, int k) {
  btam_system *s = b->sys[k];
  BTAM_TRY(cudaEventRecord(b->ev, s->st));
  BTAM_TRY(cudaStreamWaitEvent(b->st, b->ev, 0));
  const int n = s->n_real, g = s->n_ghost;
  BTAM_TRY(cudaMemcpyAsync(b->pos + b->base_real[k], s->pos, n * sizeof(double4),
                           cudaMemcpyDeviceToDevice, b->st));
  BTAM_TRY(cudaMemcpyAsync(b->xb + b->base_real[k], s->xb, n * sizeof(double2),
                           cudaMemcpyDeviceToDevice, b->st));
  if (g > 0) {
    BTAM_TRY(cudaMemcpyAsync(b->pos + b->base_img[k], s->pos + n, g * sizeof(double4),
                             cudaMemcpyDeviceToDevice, b->st));
    BTAM_TRY(cudaMemcpyAsync(b->xb + b->base_img[k], s->xb + n, g * sizeof(double2),
                             cudaMemcpyDeviceToDevice, b->st));
  }
  return BTAM_OK;
}

void free_batch(btam_batch *b) {
  for (int f = 0; f < 2; ++f)
    if (b->exec[f]) cudaGraphExecDestroy(b->exec[f]);
  dfree(b->seg, b->st);
  dfree(b->pos, b->st);
  dfree(b->xb, b->st);
  dfree(b->code, b->st);
  dfree(b->owner, b->st);
  dfree(b->gamma, b->st);
  dfree(b->offs, b->st);
  dfree(b->idx, b->st);
  dfree(b->rho, b->st);
  dfree(b->V0, b->st);
  dfree(b->S0, b->st);
  dfree(b->selfx, b->st);
  dfree(b->Rq, b->st);
  dfree(b->Rs, b->st);
  dfree(b->Rx, b->st);
  dfree(b->totals, b->st);
  dfree(b->mom64, b->st);
  dfree(b->mom32, b->st);
  dfree(b->err, b->st);
  dfree(b->rev, b->st);
  dfree(b->s32, b->st);
  dfree(b->sb, b->st);
  dfree(b->s64, b->st);
  dfree(b->site_on, b->st);
  dfree(b->slot_own, b->st);
  dfree(b->own_p, b->st);
  dfree(b->own_u, b->st);
  dfree(b->pbuf, b->st);
  if (b->ev) cudaEventDestroy(b->ev);
  if (b->st) cudaStreamDestroy(b->st);
  delete b;
}

int batch_build(btam_batch *b) {
  const int ns = b->n_sys;
  // sizes and bases
  std::vector<int> n_list_pairs(ns);
  long long n_real = 0, n_img = 0, n_pairs = 0;
  b->base_real.resize(ns);
  b->base_img.resize(ns);
  b->base_pair.resize(ns);
  std::vector<int> seg(ns + 1);
  for (int k = 0; k < ns; ++k) {
    btam_system *s = b->sys[k];
    // real sites' pairs: offs[n_real]; when the lists cover the real sites
    // only that is every entry, known on the host (no wait on the system's
    // stream); when they also cover the images it is read back
    int last = (int)s->n_pairs;
    if (s->n_list != s->n_real)
      BTAM_TRY(copy_sync(&last, s->offs + s->n_real, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    n_list_pairs[k] = last;
    if (n_real + n_img + s->n_real + s->n_ghost > 0x7fffffffLL || n_pairs + last > 0x7fffffffLL)
      return BTAM_ERR_TOO_LARGE;
    b->base_real[k] = (int)n_real;
    b->base_pair[k] = n_pairs;
    seg[k] = (int)n_real;
    n_real += s->n_real;
    n_img += s->n_ghost;
    n_pairs += last;
  }
  seg[ns] = (int)n_real;
  long long own_total = 0;
  for (int k = 0; k < ns; ++k) own_total += b->sys[k]->n_own;
  long long gacc = 0;
  for (int k = 0; k < ns; ++k) {
    b->base_img[k] = (int)(n_real + gacc);
    gacc += b->sys[k]->n_ghost;
  }
  b->n_real = (int)n_real;
  b->n_all = (int)(n_real + n_img);
  b->n_pairs = n_pairs;
  const size_t nr = n_real, na = b->n_all;
  BTAM_TRY(dalloc(b->seg, b->st, ns + 1));
  BTAM_TRY(dalloc(b->pos, b->st, na));
  BTAM_TRY(dalloc(b->xb, b->st, na));
  BTAM_TRY(dalloc(b->code, b->st, na));
  BTAM_TRY(dalloc(b->owner, b->st, na));
  BTAM_TRY(dalloc(b->s32, b->st, na));
  BTAM_TRY(dalloc(b->sb, b->st, na));
  BTAM_TRY(dalloc(b->s64, b->st, na));
  BTAM_TRY(dalloc(b->site_on, b->st, nr));
  BTAM_TRY(dalloc(b->gamma, b->st, nr));
  BTAM_TRY(dalloc(b->offs, b->st, nr + 1));
  BTAM_TRY(dalloc(b->idx, b->st, (size_t)n_pairs));
  BTAM_TRY(dalloc(b->rho, b->st, nr));
  BTAM_TRY(dalloc(b->V0, b->st, nr));
  BTAM_TRY(dalloc(b->S0, b->st, nr));
  BTAM_TRY(dalloc(b->selfx, b->st, nr));
  BTAM_TRY(dalloc(b->Rq, b->st, 3 * nr));
  BTAM_TRY(dalloc(b->Rs, b->st, nr));
  BTAM_TRY(dalloc(b->Rx, b->st, nr));
  // totals (4 per system), then the partial sums of the totals reduction
  BTAM_TRY(dalloc(b->totals, b->st, 4 * (size_t)ns * (1 + kTotParts)));
  BTAM_TRY(dalloc(b->err, b->st, 1));
  BTAM_TRY(dalloc(b->rev, b->st, (size_t)n_pairs));
  BTAM_TRY(dalloc(b->slot_own, b->st, (size_t)n_pairs));
  BTAM_TRY(dalloc(b->own_p, b->st, (size_t)own_total));
  BTAM_TRY(dalloc(b->own_u, b->st, (size_t)own_total));
  b->n_own = (int)own_total;
  BTAM_TRY(cudaMemsetAsync(b->err, 0, sizeof(int), b->st));
  BTAM_TRY(cudaMemcpyAsync(b->seg, seg.data(), (ns + 1) * sizeof(int), cudaMemcpyHostToDevice,
                           b->st));
  long long own_base = 0;
  for (int k = 0; k < ns; ++k) {
    btam_system *s = b->sys[k];
    const int n = s->n_real, g = s->n_ghost, R = b->base_real[k], G = b->base_img[k];
    int st = copy_sites(b, k);
    if (st != BTAM_OK) return st;
    BTAM_TRY(cudaMemcpyAsync(b->code + R, s->code, n * sizeof(int), cudaMemcpyDeviceToDevice,
                             b->st));
    if (g > 0)
      BTAM_TRY(cudaMemcpyAsync(b->code + G, s->code + n, g * sizeof(int),
                               cudaMemcpyDeviceToDevice, b->st));
    BTAM_TRY(cudaMemcpyAsync(b->gamma + R, s->gamma, n * sizeof(double),
                             cudaMemcpyDeviceToDevice, b->st));
    remap_owner_kernel<<<blocks_of(n + g, 256), 256, 0, b->st>>>(n + g, s->owner, b->owner + R,
                                                                  b->owner + G, n, R);
    shift_offs_kernel<<<blocks_of(n, 256), 256, 0, b->st>>>(n, s->offs, b->offs + R,
                                                             (int)b->base_pair[k]);
    if (n_list_pairs[k] > 0) {
      remap_idx_kernel<<<blocks_of(n_list_pairs[k], 256), 256, 0, b->st>>>(
          n_list_pairs[k], s->idx, b->idx + b->base_pair[k], n, R, G);
      shift_rev_kernel<<<blocks_of(n_list_pairs[k], 256), 256, 0, b->st>>>(
          n_list_pairs[k], s->rev, b->rev + b->base_pair[k], (int)b->base_pair[k]);
      shift_slot_own_kernel<<<blocks_of(n_list_pairs[k], 256), 256, 0, b->st>>>(
          n_list_pairs[k], s->slot_own, b->slot_own + b->base_pair[k], (int)own_base);
    }
    if (s->n_own > 0) {
      shift_offs_kernel<<<blocks_of(s->n_own, 256), 256, 0, b->st>>>(
          s->n_own, s->own_p, b->own_p + own_base, (int)b->base_pair[k]);
      shift_offs_kernel<<<blocks_of(s->n_own, 256), 256, 0, b->st>>>(
          s->n_own, s->own_u, b->own_u + own_base, R);
      own_base += s->n_own;
    }
    BTAM_TRY(cudaGetLastError());
  }
  const int tail = (int)n_pairs;
  BTAM_TRY(cudaMemcpyAsync(b->offs + b->n_real, &tail, sizeof(int), cudaMemcpyHostToDevice, b->st));
  BTAM_TRY(cudaStreamSynchronize(b->st));
  return BTAM_OK;
}

// Enqueues one evaluation of every system: pass 1, pass 2, per-system totals.
template <class R> cudaError_t enqueue_eval(btam_batch *b, int form, R *mom, const RadialView<R> &T) {
  EvalArgs<R> a = batch_args<R>(b, mom, T);
  cudaError_t e = launch_pass1(a, b->st, b->variant1[form], b->variant2[form]);
  if (e == cudaSuccess) e = launch_pass2(a, b->st, b->variant2[form]);
  if (e == cudaSuccess)
    e = launch_seg_totals(b->n_sys, b->seg, b->V0, b->S0, b->Rq, b->Rs, b->Rx, b->totals,
                          b->totals + 4 * (size_t)b->n_sys, b->st);
  return e;
}

int ensure_moments(btam_batch *b, int precision) {
  const size_t nm = (size_t)b->n_real * kMomStride;
  if (precision == BTAM_FP64 && !b->mom64) BTAM_TRY(dalloc(b->mom64, b->st, nm));
  if (precision == BTAM_FP32C && !b->mom32) BTAM_TRY(dalloc(b->mom32, b->st, nm));
  return BTAM_OK;
}

// Captures the evaluation of one arithmetic form into a graph (again only
// when the launch variants changed since the last capture).
int ensure_graph(btam_batch *b, int precision) {
  const int f = precision == BTAM_FP64 ? 0 : 1;
  if (b->exec[f] && b->exec_v1[f] == b->variant1[f] && b->exec_v2[f] == b->variant2[f] &&
      b->exec_pbuf[f] == b->pbuf)
    return BTAM_OK;
  if (b->exec[f]) {
    cudaGraphExecDestroy(b->exec[f]);
    b->exec[f] = nullptr;
  }
  cudaGraph_t g = nullptr;
  BTAM_TRY(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeRelaxed));
  cudaError_t e = f == 0 ? enqueue_eval<double>(b, 0, b->mom64, b->T->r64)
                         : enqueue_eval<float>(b, 1, b->mom32, b->T->r32);
  cudaError_t e2 = cudaStreamEndCapture(b->st, &g);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec[f], g, 0);
  if (g) cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    b->exec[f] = nullptr;
    return cuda_status(e);
  }
  b->exec_v1[f] = b->variant1[f];
  b->exec_v2[f] = b->variant2[f];
  b->exec_pbuf[f] = b->pbuf;
  return BTAM_OK;
}

}  // namespace

extern "C" {

int btam_batch_create(btam_system *const *systems, int n_sys, btam_batch **out) {
  if (!out || !systems || n_sys <= 0) return BTAM_ERR_ARG;
  *out = nullptr;
  int cur = -1;
  if (cudaGetDevice(&cur) != cudaSuccess) return BTAM_ERR_CUDA;
  const btam_tables *T = systems[0] ? systems[0]->T : nullptr;
  for (int k = 0; k < n_sys; ++k) {
    const btam_system *s = systems[k];
    if (!s || s->T != T) return BTAM_ERR_ARG;
    if (!s->built) return BTAM_ERR_NOT_BUILT;
    if (s->device != cur) return BTAM_ERR_ARG;
  }
  btam_batch *b = new btam_batch;
  b->T = T;
  b->device = systems[0]->device;
  b->n_sys = n_sys;
  b->sys.assign(systems, systems + n_sys);
  int st = cuda_status(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking));
  if (st == BTAM_OK) st = cuda_status(cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming));
  if (st == BTAM_OK) st = batch_build(b);
  if (st != BTAM_OK) {
    free_batch(b);
    return st;
  }
  *out = b;
  return BTAM_OK;
}

int btam_batch_destroy(btam_batch *b) {
  if (!b) return BTAM_ERR_ARG;
  if (b->st) cudaStreamSynchronize(b->st);
  free_batch(b);
  return BTAM_OK;
}

int btam_batch_info(const btam_batch *b, int *n_sys, int *n_real, int *n_all,
                    long long *n_pairs) {
  if (!b) return BTAM_ERR_ARG;
  if (n_sys) *n_sys = b->n_sys;
  if (n_real) *n_real = b->n_real;
  if (n_all) *n_all = b->n_all;
  if (n_pairs) *n_pairs = b->n_pairs;
  return BTAM_OK;
}

void *btam_batch_stream(const btam_batch *b) { return b ? (void *)b->st : nullptr; }

int btam_batch_set_state(btam_batch *b, int k, const double *q, const double *sigma,
                         const double *x) {
  if (!b || k < 0 || k >= b->n_sys) return BTAM_ERR_ARG;
  int st = btam_system_set_state(b->sys[k], q, sigma, x);
  if (st != BTAM_OK) return st;
  return copy_sites(b, k);
}

int btam_batch_autotune(btam_batch *b, int precision, int *pass1_variant, int *pass2_variant) {
  if (!b || (precision != BTAM_FP64 && precision != BTAM_FP32C)) return BTAM_ERR_ARG;
  int st = ensure_moments(b, precision);
  if (st != BTAM_OK) return st;
  const int f = precision == BTAM_FP64 ? 0 : 1;
  st = batch_pbuf(b, f == 0 ? sizeof(double) : sizeof(float));
  if (st != BTAM_OK) return st;
  int v1 = 0, v2 = 0;
  cudaError_t e = f == 0 ? autotune_passes(batch_args<double>(b, b->mom64, b->T->r64), b->st, 3,
                                           &v1, &v2)
                         : autotune_passes(batch_args<float>(b, b->mom32, b->T->r32), b->st, 3,
                                           &v1, &v2);
  if (e != cudaSuccess) return cuda_status(e);
  b->variant1[f] = v1;
  b->variant2[f] = v2;
  if (!((b->variant1[0] | b->variant1[1] | b->variant2[0] | b->variant2[1]) & kUndirected)) {
    dfree(b->pbuf, b->st);
    b->pbuf_bytes = b->pbuf_elem = 0;
  }
  if (pass1_variant) *pass1_variant = v1;
  if (pass2_variant) *pass2_variant = v2;
  return batch_read_err(b);
}

int btam_batch_set_variants(btam_batch *b, int precision, int pass1_variant, int pass2_variant) {
  if (!b || (precision != BTAM_FP64 && precision != BTAM_FP32C)) return BTAM_ERR_ARG;
  if (!valid_variants(pass1_variant, pass2_variant)) return BTAM_ERR_ARG;
  if ((pass1_variant | pass2_variant) & kUndirected) {
    int st = batch_pbuf(b, precision == BTAM_FP64 ? sizeof(double) : sizeof(float));
    if (st != BTAM_OK) return st;
  }
  const int f = precision == BTAM_FP64 ? 0 : 1;
  b->variant1[f] = pass1_variant;
  b->variant2[f] = pass2_variant;
  return BTAM_OK;
}

int btam_batch_eval_async(btam_batch *b, int precision) {
  if (!b || (precision != BTAM_FP64 && precision != BTAM_FP32C)) return BTAM_ERR_ARG;
  int st = ensure_moments(b, precision);
  if (st == BTAM_OK) st = ensure_graph(b, precision);
  if (st != BTAM_OK) return st;
  return cuda_status(cudaGraphLaunch(b->exec[precision == BTAM_FP64 ? 0 : 1], b->st));
}

}  // extern "C"

// ---- evaluation rounds of the job server (server.cu) -----------------------
// The systems in a round's table: their site rows are copied in after
// everything already enqueued on their streams (ready events), the batch is
// evaluated, and their results are copied back into their own buffers.
int batch_round(btam_batch *b, const BatchXfer &t, const cudaEvent_t *ready, int precision) {
  if (t.n <= 0) return BTAM_OK;
  for (int k = 0; k < t.n; ++k) BTAM_TRY(cudaStreamWaitEvent(b->st, ready[k], 0));
  int rows = 0;
  for (int k = 0; k < t.n; ++k) rows = std::max(rows, t.sys[k].n + t.sys[k].g);
  const dim3 grid(std::max(1, std::min(64, blocks_of(rows, 256))), t.n);
  // only the systems in the table are evaluated: the others' rows keep
  // their last results, which nobody reads
  BTAM_TRY(cudaMemsetAsync(b->site_on, 0, (size_t)b->n_real, b->st));
  batch_gather_kernel<<<grid, 256, 0, b->st>>>(t, b->pos, b->xb, b->site_on);
  BTAM_TRY(cudaGetLastError());
  BTAM_TRY(cudaMemsetAsync(b->err, 0, sizeof(int), b->st));
  // the kernels are launched directly, not replayed from a captured graph:
  // the other jobs' threads keep making CUDA calls meanwhile (their
  // neighbour builds free scratch memory with cudaFree, which synchronises
  // implicitly and must never meet a stream in capture)
  int st = ensure_moments(b, precision);
  if (st != BTAM_OK) return st;
  b->masked = true;
  const cudaError_t ev = precision == BTAM_FP64 ? enqueue_eval<double>(b, 0, b->mom64, b->T->r64)
                                                : enqueue_eval<float>(b, 1, b->mom32, b->T->r32);
  b->masked = false;
  BTAM_TRY(ev);
  batch_scatter_kernel<<<grid, 256, 0, b->st>>>(t, b->rho, b->V0, b->S0, b->Rq, b->Rs, b->Rx,
                                                 b->totals, b->err);
  return cuda_status(cudaGetLastError());
}

// Row bases of system k in the batch layout.
void batch_bases(const btam_batch *b, int k, int *R, int *G) {
  *R = b->base_real[k];
  *G = b->base_img[k];
}

cudaStream_t batch_stream_of(const btam_batch *b) { return b->st; }

extern "C" {

int btam_batch_sync(btam_batch *b) {
  if (!b) return BTAM_ERR_ARG;
  return batch_read_err(b);
}

int btam_batch_results_copy(btam_batch *b, int k, double *rho, double *V0, double *S0,
                            double *Rq, double *Rs, double *Rx, double *totals) {
  if (!b || k < 0 || k >= b->n_sys) return BTAM_ERR_ARG;
  const int n = b->sys[k]->n_real;
  const size_t o = b->base_real[k];
  auto get = [&](double *dst, const double *src, size_t count) -> cudaError_t {
    if (!dst || count == 0) return cudaSuccess;
    return cudaMemcpyAsync(dst, src, count * sizeof(double), cudaMemcpyDeviceToHost, b->st);
  };
  BTAM_TRY(get(rho, b->rho + o, n));
  BTAM_TRY(get(V0, b->V0 + o, n));
  BTAM_TRY(get(S0, b->S0 + o, n));
  BTAM_TRY(get(Rq, b->Rq + 3 * o, 3 * (size_t)n));
  BTAM_TRY(get(Rs, b->Rs + o, n));
  BTAM_TRY(get(Rx, b->Rx + o, n));
  BTAM_TRY(get(totals, b->totals + 4 * (size_t)k, 4));
  return batch_read_err(b);
}

int btam_batch_totals_copy(btam_batch *b, double *totals) {
  if (!b || !totals) return BTAM_ERR_ARG;
  BTAM_TRY(cudaMemcpyAsync(totals, b->totals, 4 * (size_t)b->n_sys * sizeof(double),
                           cudaMemcpyDeviceToHost, b->st));
  return batch_read_err(b);
}

}  // extern "C"
