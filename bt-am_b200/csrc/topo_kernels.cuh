// Device topology: periodic images, cell binning, neighbour lists.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace btam {

constexpr int kNbrBuf = 256;  // per-site candidate buffer (>= maxneigh = 250)

// Error bits raised by kernels (mapped to btam_status codes by the host).
enum ErrBit : int {
  kErrBitOverflow = 0,       // more than maxneigh neighbours
  kErrBitEmpty = 1,          // a site without neighbours
  kErrBitGhostOverflow = 2,  // more images than allocated
  kErrBitCells = 3,          // cell grid did not fit
  kErrBitNonFinite = 4,      // NaN/Inf in an output
  kErrBitTimeout = 5,        // a bounded wait gave up
};

// Box description shared by the image kernels.  A[b] = lattice vector b;
// B[a] = reciprocal row a (fractional s_a = (q - origin) . B[a]);
// w[a] = rc |B[a]| (fractional width of the rc shell across faces a).
struct GhostBox {
  double A[3][3], B[3][3], w[3], lo[3], hi[3], origin[3], rc;
  int periodic[3];
  int ortho;
};

struct CellGrid {
  double lo[3];
  double edge, inv_edge;
  int n[3];
};

// The library's stream-ordered memory pool of the current device (defined
// in btam_capi.cu).
cudaMemPool_t device_pool();

// Growable device scratch for library temporaries (CUB scans), allocated in
// stream order from the library pool.
struct DeviceScratch {
  void *ptr = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t need, cudaStream_t st) {
    if (need <= bytes) return cudaSuccess;
    release(st);
    cudaMemPool_t pool = device_pool();
    if (!pool) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMallocFromPoolAsync(&ptr, need, pool, st);
    if (e == cudaSuccess) bytes = need;
    else ptr = nullptr;
    return e;
  }
  void release(cudaStream_t st) {
    if (ptr) cudaFreeAsync(ptr, st);
    ptr = nullptr;
    bytes = 0;
  }
  ~DeviceScratch() {
    if (ptr) cudaFree(ptr);
  }
};

struct NbrArgs {
  int n_all, n_query, maxn, max_cells;
  double rc, cell_edge;
  const double4 *pos;
  unsigned long long *bbox;  // 6
  CellGrid *grid;
  int *cell_of, *cell_cnt, *cell_start, *cursor, *cell_sites;
  int *cnt;   // n_query + 1
  int *tmp;   // n_query * kNbrBuf
  int *offs;  // n_query + 1
  int *err;
  DeviceScratch *scratch;
  // optional restriction to one species code (-1: all sites), e.g. the H-H
  // diffusive graph; allow_empty = 1 accepts sites with no neighbour
  const int *code = nullptr;
  int filter_code = -1;
  int allow_empty = 0;
};

cudaError_t exclusive_scan(const int *in, int *out, int n, DeviceScratch &s,
                           cudaStream_t st);
cudaError_t launch_ghost_count(int n, const double4 *pos, const GhostBox &b, int *cnt,
                               cudaStream_t st);
cudaError_t launch_ghost_emit(int n, double4 *pos, double2 *xb, int *code, int *owner,
                              char4 *image, const GhostBox &b, const int *off,
                              int max_ghosts, int *err, cudaStream_t st);
cudaError_t launch_ghost_refresh(int n_real, int n_ghost, double4 *pos, double2 *xb,
                                 int *code, const int *owner, const char4 *image,
                                 const GhostBox &b, cudaStream_t st);
cudaError_t launch_neighbors(const NbrArgs &a, cudaStream_t st);
// Pair links of the real sites' neighbour lists for the undirected pass 2:
// rev[p] = the slot of the reverse pair (o, copy of u) in the list of o =
// owner of idx[p], or -1 if o's list lacks it (rounding at exactly rc for an
// image pair); slot p is owned by its site u when u < o or rev[p] < 0, and the
// owned slots are listed as (own_p, own_u) in site-then-slot order.
// own_cnt / own_off: n_real + 1 ints of scratch; *n_own returned after a
// stream synchronisation.
cudaError_t launch_pair_links(int n_real, const int *offs, const int *idx, const int *owner,
                              int *rev, int *slot_own, int *own_cnt, int *own_off, int *&own_p,
                              int *&own_u, long long &own_cap, int *n_own,
                              DeviceScratch &scratch, cudaStream_t st);

cudaError_t launch_compact(int n_query, const int *tmp, const int *offs, int *idx,
                           cudaStream_t st);

}  // namespace btam
