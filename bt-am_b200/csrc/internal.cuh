// Internal layout of the library's opaque handles (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <utility>
#include <vector>

#include "../../include/btam.h"

#include "adp_core.cuh"
#include "tables_io.hpp"
#include "adp_kernels.cuh"
#include "topo_kernels.cuh"

using namespace btam;

// The job server's evaluation batcher (server.cu).
struct EvalBatcher;

struct btam_tables {
  HostTables host;
  int device = 0;
  Coef4<double> *d64 = nullptr;
  Coef4<float> *d32 = nullptr;
  TablesView<double> v64;
  TablesView<float> v32;
  // the radial tables as the kernels' per-segment records
  double *rad64 = nullptr;
  float *rad32 = nullptr;
  float *uws32 = nullptr;  // the FP32 uw block in its shared-memory layout
  double *uws64 = nullptr;  // the FP64 uw block in its shared-memory layout
  RadialView<double> r64;
  RadialView<float> r32;
};

struct btam_system {
  const btam_tables *T = nullptr;
  int device = 0;
  cudaStream_t st = nullptr;
  int n_real = 0, n_ghost = 0, cap_all = 0;
  GhostBox box;
  bool any_periodic = false;
  // site arrays (real then images)
  double4 *pos = nullptr;
  double2 *xb = nullptr;
  int *code = nullptr, *owner = nullptr;
  char4 *image = nullptr;
  double *gamma = nullptr;
  Site32 *s32 = nullptr;  // packed neighbour rows of the FP32C kernels [all]
  SiteB *sb = nullptr;
  Site64 *s64 = nullptr;  // packed neighbour rows of the FP64 kernels [all]
  // staging for host updates
  double *stage = nullptr;  // 5 n_real doubles: q (3n), sigma, x
  // neighbour lists
  bool built = false;
  int n_list = 0;
  long long n_pairs = 0, idx_cap = 0;
  int *offs = nullptr, *idx = nullptr, *cnt = nullptr, *tmp = nullptr;
  long long tmp_cap = 0;
  int q_cap = 0;
  // cells
  int cell_cap = 0, site_cap = 0;
  unsigned long long *bbox = nullptr;
  CellGrid *grid = nullptr;
  int *cell_of = nullptr, *cell_cnt = nullptr, *cell_start = nullptr, *cursor = nullptr,
      *cell_sites = nullptr;
  // results
  double *rho = nullptr, *V0 = nullptr, *S0 = nullptr, *selfx = nullptr, *Rq = nullptr,
         *Rs = nullptr, *Rx = nullptr, *totals = nullptr;
  double *mom64 = nullptr;
  float *mom32 = nullptr;
  int *err = nullptr;
  DeviceScratch scratch;
  // kernel block shapes per arithmetic form (index 0 FP64, 1 FP32C), chosen
  // by btam_autotune
  int variant1[2] = {0, 0}, variant2[2] = {0, 0};
  int cnt_cap = 0;
  // diffusive graph and master-equation state
  bool dmd_ready = false;
  int *doffs = nullptr, *didx = nullptr, dq_cap = 0;
  long long didx_cap = 0, d_pairs = 0;
  long long *X = nullptr, *X0 = nullptr, *dtot = nullptr;
  unsigned long long *dctl = nullptr;  // step-control maxima and clip count (DmdArgs::ctl)
  double *mu = nullptr;
  int *dact = nullptr, *ddeg = nullptr;
  // relaxation work vectors
  int relax_m = 0;
  double *rv = nullptr;  // one block holding every relaxation vector
  // pair links and slot buffer of the undirected pass 2
  int *rev = nullptr, *slot_own = nullptr, *own_off = nullptr, *own_p = nullptr,
      *own_u = nullptr;
  long long rev_cap = 0, own_cap = 0;
  int own_off_cap = 0, n_own = 0;
  char *pbuf = nullptr;
  size_t pbuf_bytes = 0, pbuf_elem = 0;  // bytes; bytes per value (0: none yet)
  // non-mean-field forms: site records, outputs and totals (point.cu)
  double *pt = nullptr;
  size_t pt_cap = 0;
  // the job server's evaluation batcher this system's evaluations go to
  // (null: its own kernels), and the events that order them
  EvalBatcher *batcher = nullptr;
  cudaEvent_t batch_ready = nullptr, batch_done = nullptr;
  // pipelined state evaluations (btam_mf_eval_state_async): two slots, each
  // with its own staging and result buffers, so that one call's host copies
  // run on the copy streams while the next call evaluates on `st`
  struct StateSlot {
    double *stage = nullptr;  // q (3n), sigma (n), x (n)
    double *res = nullptr;    // rho, V0, S0, Rq (3n), Rs, Rx (8n), totals (4)
    int *flags = nullptr;     // error bits, validation flags (device)
    int *hflags = nullptr;    // their host copy (pinned)
    cudaEvent_t in = nullptr, used = nullptr, done = nullptr, out = nullptr;
    long long ticket = 0;     // the call in the slot (0: free)
  } slot[2];
  cudaStream_t cp_in = nullptr, cp_out = nullptr;  // host-to-device, device-to-host
  long long next_ticket = 1;
  std::vector<std::pair<long long, int>> finished;  // calls retired before their wait
};

// ---- evaluation rounds of the job server ----------------------------------
// A table of systems whose evaluations one batch launch serves: each
// system's device buffers and its rows in the batch layout (batch.cu).
struct BatchXfer {
  static constexpr int kMax = 96;  // systems per round (kernel-argument table)
  struct Sys {
    const double4 *pos;
    const double2 *xb;
    double *rho, *V0, *S0, *Rq, *Rs, *Rx, *totals;
    int *err;
    int n, g;  // real sites, images
    int R, G;  // their first rows in the batch
    int k;     // the system's index in the batch
  } sys[kMax];
  int n = 0;
};
// Enqueues on the batch's stream: after each system's ready event, its site
// rows into the batch; one evaluation of the batch; the results back.
int batch_round(btam_batch *b, const BatchXfer &t, const cudaEvent_t *ready, int precision);
void batch_bases(const btam_batch *b, int k, int *R, int *G);
cudaStream_t batch_stream_of(const btam_batch *b);

// btam_mf_eval_async of a system attached to the job server's batcher
// hands the evaluation to it (server.cu).
int batcher_eval(btam_system *s, int precision);

// Point-form buffers reused by the mean-field stress, and the fixed-order
// totals over per-site V, Fq, W (V, Fq may be NULL) into tot[12]
// (point.cu).
int pt_stress_buffers(btam_system *s, double **W, double **part, double **tot);
cudaError_t launch_pt_totals(int n, const double *V, const double *Fq, const double *W,
                             double *part, double *tot, cudaStream_t st);

// Enqueues the FP64 directed pass 1: the mean-field rho-bar, V0 and S0 of
// the current state into the system's buffers (btam_capi.cu).
int mf_rho64_enqueue(btam_system *s);

// Enqueues the mean-field Hessian blocks of the current state into Hd (9
// per real site); with Hslot (9 per entry of the real sites' lists), Hd
// holds the i = u blocks and Hslot the per-neighbour ones (mf_hessian.cu).
int mf_hessian_enqueue(btam_system *s, double *Hd, double *Hslot);
// The same blocks on a given rho-bar and, if gmp is set, per-list-entry
// rho gradients (3 per entry of a real site) instead of the degree-3 ones.
int mf_hessian_enqueue_with(btam_system *s, const double *rho, const double *gmp, double *Hd,
                            double *Hslot);

// Enqueues the directed pass 1 and the mean-field stress of the current
// state; *W: per-site stress (9 n), *tot: totals whose [2..10] hold the sum
// (btam_capi.cu).
int mf_stress_enqueue(btam_system *s, int precision, double **W, double **tot);

// Box of a cell (rows = lattice vectors) and origin at the potential's
// cutoff, with the checks of btam_system_create (btam_capi.cu).
int make_box_for(const double *origin, const double *cell, const int *periodic, GhostBox &b);


// ---- host helpers shared by the library sources

inline int status_from_bits(int bits) {
  if (bits & (1 << kErrBitOverflow)) return BTAM_ERR_NEIGHBOR_OVERFLOW;
  if (bits & (1 << kErrBitEmpty)) return BTAM_ERR_NO_NEIGHBORS;
  if (bits & (1 << kErrBitGhostOverflow)) return BTAM_ERR_GHOST_OVERFLOW;
  if (bits & (1 << kErrBitCells)) return BTAM_ERR_OOM;
  if (bits & (1 << kErrBitNonFinite)) return BTAM_ERR_NONFINITE;
  if (bits & (1 << kErrBitTimeout)) return BTAM_ERR_TIMEOUT;
  return BTAM_OK;
}

// The CUDA runtime error that this thread last turned into a status
// (btam_last_cuda_error reports it).
inline cudaError_t &last_cuda_error() {
  static thread_local cudaError_t e = cudaSuccess;
  return e;
}

inline int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return BTAM_OK;
  last_cuda_error() = e;
  if (e == cudaErrorMemoryAllocation) return BTAM_ERR_OOM;
  return BTAM_ERR_CUDA;
}

#define BTAM_TRY(expr)                         \
  do {                                         \
    cudaError_t _e = (expr);                   \
    if (_e != cudaSuccess) return cuda_status(_e); \
  } while (0)

// Device memory of systems and batches comes from the library's
// stream-ordered pool of the current device (cudaMallocFromPoolAsync on the
// owner's stream), so creating and destroying systems never synchronises the
// device and never stalls other systems' work in flight; freed blocks stay
// in the pool for the next system.
template <class T> inline cudaError_t dalloc(T *&p, cudaStream_t st, size_t count) {
  if (p) cudaFreeAsync(p, st);
  p = nullptr;
  if (count == 0) count = 1;
  cudaMemPool_t pool = btam::device_pool();
  if (!pool) return cudaErrorMemoryAllocation;
  return cudaMallocFromPoolAsync((void **)&p, count * sizeof(T), pool, st);
}

template <class T> inline void dfree(T *&p, cudaStream_t st) {
  if (p) cudaFreeAsync(p, st);
  p = nullptr;
}

// Synchronous copies ordered on a stream (the memory may come from the
// stream-ordered pool, so the copy must follow the allocation on `st`).
inline cudaError_t copy_sync(void *dst, const void *src, size_t bytes, cudaMemcpyKind kind,
                             cudaStream_t st) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e;
}

// Waits for the stream, returns the error bits raised since the last read
// (as a status) and clears them.
inline int read_err(btam_system *s) {
  int bits = 0;
  cudaError_t e = cudaMemcpyAsync(&bits, s->err, sizeof(int), cudaMemcpyDeviceToHost, s->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->err, 0, sizeof(int), s->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  if (e != cudaSuccess) return cuda_status(e);
  return status_from_bits(bits);
}

