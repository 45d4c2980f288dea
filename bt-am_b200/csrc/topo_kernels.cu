// Topology on the device: periodic images ("ghosts"), cell binning and
// neighbour lists in the reference's order.
//
// Reference behaviour reproduced:
//  * images: DMSwarmCreateGhostAtoms (Ghosts.cpp:123-648) marks, per local
//    site in index order and per direction n0..n26 (x fastest, n13 skipped),
//    the sites inside the rc-wide buffer slab; each copy is then shifted to
//    the far side of the box (the shift its single-rank search at
//    Ghosts.cpp:768-794 intends).  Triclinic cells (no reference counterpart)
//    keep every image inside the cell widened by rc.
//  * neighbours: `neighbors` (Neighbors.cpp:39-134) lists, for every site,
//    all other sites with sqrt((dx^2 + dy^2) + dz^2) <= rc in IEEE double, in
//    ascending index order; more than maxneigh = 250 is an error, and so is
//    an empty list.
// The brute-force O(N^2) scan becomes: bin sites into cells of edge >= rc
// (counting sort), one warp per query site scanning the 27 surrounding cells
// with a ballot-compacted candidate buffer in shared memory, a warp bitonic
// sort to restore ascending order, and an exclusive scan into CSR.
#include "topo_kernels.cuh"

#include <cub/device/device_scan.cuh>

namespace btam {

namespace {

__device__ __forceinline__ bool ghost_in(const GhostBox &b, const double *qi,
                                         int dir, double *p) {
  if (dir == 13) return false;
  int d[3] = {dir % 3 - 1, (dir / 3) % 3 - 1, dir / 9 - 1};
  for (int a = 0; a < 3; ++a)
    if (d[a] != 0 && !b.periodic[a]) return false;
  for (int a = 0; a < 3; ++a) {
    double s = qi[a];
    for (int c = 0; c < 3; ++c)
      if (d[c] != 0) s = __dadd_rn(s, (double)(-d[c]) * b.A[c][a]);
    p[a] = s;
  }
  if (b.ortho) {
    for (int a = 0; a < 3; ++a) {
      double lw, up;
      if (d[a] == -1) {
        lw = b.lo[a];
        up = __dadd_rn(b.lo[a], b.rc);
      } else if (d[a] == 1) {
        lw = __dadd_rn(b.hi[a], -b.rc);
        up = b.hi[a];
      } else {
        lw = b.lo[a];
        up = b.hi[a];
      }
      if (!(qi[a] >= lw && qi[a] < up)) return false;
    }
    return true;
  }
  double dq0 = __dadd_rn(p[0], -b.origin[0]), dq1 = __dadd_rn(p[1], -b.origin[1]),
         dq2 = __dadd_rn(p[2], -b.origin[2]);
  for (int a = 0; a < 3; ++a) {
    double sa = __dadd_rn(__dadd_rn(__dmul_rn(dq0, b.B[a][0]), __dmul_rn(dq1, b.B[a][1])),
                          __dmul_rn(dq2, b.B[a][2]));
    if (!(sa >= -b.w[a] && sa < __dadd_rn(1.0, b.w[a]))) return false;
  }
  return true;
}

__global__ void ghost_count_kernel(int n, const double4 *pos, GhostBox b, int *cnt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 q = pos[i];
  double qi[3] = {q.x, q.y, q.z}, p[3];
  int c = 0;
  for (int dir = 0; dir < 27; ++dir) c += ghost_in(b, qi, dir, p) ? 1 : 0;
  cnt[i] = c;
}

__global__ void ghost_emit_kernel(int n, int n_real_base, double4 *pos, double2 *xb,
                                  int *code, int *owner, char4 *image, GhostBox b,
                                  const int *off, int max_ghosts, int *err) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 q = pos[i];
  double qi[3] = {q.x, q.y, q.z}, p[3];
  int k = off[i];
  for (int dir = 0; dir < 27; ++dir) {
    if (!ghost_in(b, qi, dir, p)) continue;
    if (k >= max_ghosts) {
      atomicOr(err, 1 << kErrBitGhostOverflow);
      return;
    }
    int g = n_real_base + k;
    pos[g] = make_double4(p[0], p[1], p[2], q.w);
    xb[g] = xb[i];
    code[g] = code[i];
    owner[g] = i;
    image[k] = make_char4((char)(1 - dir % 3), (char)(1 - (dir / 3) % 3),
                          (char)(1 - dir / 9), 0);
    ++k;
  }
}

// Ghost rows follow their owners: position = owner position + image shift.
__global__ void ghost_refresh_kernel(int n_real, int n_ghost, double4 *pos,
                                     double2 *xb, int *code, const int *owner,
                                     const char4 *image, GhostBox b) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_ghost) return;
  int g = n_real + k, o = owner[g];
  double4 q = pos[o];
  char4 t = image[k];
  int d[3] = {-(int)t.x, -(int)t.y, -(int)t.z};
  double qi[3] = {q.x, q.y, q.z}, p[3];
  for (int a = 0; a < 3; ++a) {
    double s = qi[a];
    for (int c = 0; c < 3; ++c)
      if (d[c] != 0) s = __dadd_rn(s, (double)(-d[c]) * b.A[c][a]);
    p[a] = s;
  }
  pos[g] = make_double4(p[0], p[1], p[2], q.w);
  xb[g] = xb[o];
  code[g] = code[o];
}

// ---- cell binning --------------------------------------------------------
__device__ __forceinline__ unsigned long long ord_encode(double v) {
  unsigned long long u = __double_as_longlong(v);
  return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double ord_decode(unsigned long long u) {
  u = (u & 0x8000000000000000ull) ? (u & 0x7fffffffffffffffull) : ~u;
  return __longlong_as_double(u);
}

__global__ void bbox_init_kernel(unsigned long long *mm) {
  // lo slots start at the largest encoding, hi slots at the smallest
  if (threadIdx.x < 6) mm[threadIdx.x] = threadIdx.x < 3 ? ~0ull : 0ull;
}

__global__ void bbox_kernel(int n, const double4 *pos, unsigned long long *mm) {
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double4 q = pos[i];
    lo[0] = fmin(lo[0], q.x); lo[1] = fmin(lo[1], q.y); lo[2] = fmin(lo[2], q.z);
    hi[0] = fmax(hi[0], q.x); hi[1] = fmax(hi[1], q.y); hi[2] = fmax(hi[2], q.z);
  }
  for (int a = 0; a < 3; ++a) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[a] = fmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
      hi[a] = fmax(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
    }
  }
  if ((threadIdx.x & 31) == 0)
    for (int a = 0; a < 3; ++a) {
      atomicMin(&mm[a], ord_encode(lo[a]));
      atomicMax(&mm[3 + a], ord_encode(hi[a]));
    }
}

__global__ void cell_setup_kernel(const unsigned long long *mm, double cell_edge,
                                  CellGrid *g, int max_cells, int *err) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  // Cells of edge >= rc; a sparse system in a large box widens the edge
  // until the grid fits the allocated cell arrays.
  for (int attempt = 0; attempt < 64; ++attempt) {
    long long total = 1;
    for (int a = 0; a < 3; ++a) {
      double lo = ord_decode(mm[a]), hi = ord_decode(mm[3 + a]);
      g->lo[a] = lo;
      int nc = (int)floor((hi - lo) / cell_edge) + 1;
      if (nc < 1) nc = 1;
      g->n[a] = nc;
      total *= nc;
    }
    g->edge = cell_edge;
    g->inv_edge = 1.0 / cell_edge;
    if (total <= max_cells) return;
    cell_edge *= 1.25;
  }
  atomicOr(err, 1 << kErrBitCells);
  g->n[0] = g->n[1] = g->n[2] = 0;
}

__device__ __forceinline__ int cell_coord(const CellGrid &g, double v, int a) {
  int c = (int)((v - g.lo[a]) * g.inv_edge);
  return c < 0 ? 0 : (c >= g.n[a] ? g.n[a] - 1 : c);
}

__global__ void cell_count_kernel(int n, const double4 *pos, const CellGrid *gp,
                                  int *cell_of, int *cell_cnt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  CellGrid g = *gp;
  if (i >= n || g.n[0] == 0) return;
  double4 q = pos[i];
  int c = (cell_coord(g, q.z, 2) * g.n[1] + cell_coord(g, q.y, 1)) * g.n[0] +
          cell_coord(g, q.x, 0);
  cell_of[i] = c;
  atomicAdd(&cell_cnt[c], 1);
}

__global__ void cell_fill_kernel(int n, const CellGrid *gp, const int *cell_of,
                                 const int *cell_start, int *cursor, int *cell_sites) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || gp->n[0] == 0) return;
  int c = cell_of[i];
  int k = atomicAdd(&cursor[c], 1);
  cell_sites[cell_start[c] + k] = i;
}

// One warp per query site.
template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32)
neighbor_kernel(int n_query, const double4 *pos, const CellGrid *gp,
                const int *cell_start, const int *cell_sites, double rc,
                int maxn, int *cnt, int *tmp, int *err, const int *code, int filter,
                int allow_empty) {
  __shared__ int buf[WARPS][kNbrBuf];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * WARPS + warp;
  if (i >= n_query) return;
  if (filter >= 0 && code[i] != filter) {  // not a site of this graph
    if (lane == 0) cnt[i] = 0;
    return;
  }
  CellGrid g = *gp;
  double4 qi = pos[i];
  int cx = cell_coord(g, qi.x, 0), cy = cell_coord(g, qi.y, 1), cz = cell_coord(g, qi.z, 2);
  int count = 0;
  int *b = buf[warp];
  for (int dz = -1; dz <= 1; ++dz) {
    int z = cz + dz;
    if (z < 0 || z >= g.n[2]) continue;
    for (int dy = -1; dy <= 1; ++dy) {
      int y = cy + dy;
      if (y < 0 || y >= g.n[1]) continue;
      for (int dx = -1; dx <= 1; ++dx) {
        int x = cx + dx;
        if (x < 0 || x >= g.n[0]) continue;
        int c = (z * g.n[1] + y) * g.n[0] + x;
        int s0 = cell_start[c], s1 = cell_start[c + 1];
        for (int base = s0; base < s1; base += 32) {
          int t = base + lane;
          bool ok = false;
          int j = -1;
          if (t < s1) {
            j = cell_sites[t];
            if (j != i && (filter < 0 || code[j] == filter)) {
              double4 qj = pos[j];
              double ex = __dadd_rn(qi.x, -qj.x), ey = __dadd_rn(qi.y, -qj.y),
                     ez = __dadd_rn(qi.z, -qj.z);
              double r2 = __dadd_rn(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)),
                                    __dmul_rn(ez, ez));
              ok = __dsqrt_rn(r2) <= rc;
            }
          }
          unsigned m = __ballot_sync(0xffffffffu, ok);
          int slot = count + __popc(m & ((1u << lane) - 1u));
          if (ok && slot < kNbrBuf) b[slot] = j;
          count += __popc(m);
        }
      }
    }
  }
  __syncwarp();
  int kept = count < kNbrBuf ? count : kNbrBuf;
  for (int t = kept + lane; t < kNbrBuf; t += 32) b[t] = 0x7fffffff;
  __syncwarp();
  // bitonic sort, ascending
  for (int k = 2; k <= kNbrBuf; k <<= 1)
    for (int jj = k >> 1; jj > 0; jj >>= 1) {
      for (int t = lane; t < kNbrBuf; t += 32) {
        int p = t ^ jj;
        if (p > t) {
          int a = b[t], c = b[p];
          bool up = (t & k) == 0;
          if ((a > c) == up) {
            b[t] = c;
            b[p] = a;
          }
        }
      }
      __syncwarp();
    }
  if (count > maxn) {
    if (lane == 0) atomicOr(err, 1 << kErrBitOverflow);
    count = maxn;
  }
  if (count == 0 && lane == 0 && !allow_empty) atomicOr(err, 1 << kErrBitEmpty);
  for (int t = lane; t < count; t += 32) tmp[(size_t)i * kNbrBuf + t] = b[t];
  if (lane == 0) cnt[i] = count;
}

__global__ void compact_kernel(int n_query, const int *tmp, const int *offs, int *idx) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= n_query) return;
  int o = offs[warp], c = offs[warp + 1] - o;
  for (int t = lane; t < c; t += 32) idx[o + t] = tmp[(size_t)warp * kNbrBuf + t];
}

inline int blocks(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

// ---------------------------------------------------------------------------
cudaError_t exclusive_scan(const int *in, int *out, int n, DeviceScratch &s,
                           cudaStream_t st) {
  size_t need = 0;
  cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, need, in, out, n, st);
  if (e != cudaSuccess) return e;
  if ((e = s.ensure(need, st)) != cudaSuccess) return e;
  size_t have = s.bytes;
  return cub::DeviceScan::ExclusiveSum(s.ptr, have, in, out, n, st);
}

cudaError_t launch_ghost_count(int n, const double4 *pos, const GhostBox &b, int *cnt,
                               cudaStream_t st) {
  if (n > 0) ghost_count_kernel<<<blocks(n, 128), 128, 0, st>>>(n, pos, b, cnt);
  return cudaGetLastError();
}

cudaError_t launch_ghost_emit(int n, double4 *pos, double2 *xb, int *code, int *owner,
                              char4 *image, const GhostBox &b, const int *off,
                              int max_ghosts, int *err, cudaStream_t st) {
  if (n > 0)
    ghost_emit_kernel<<<blocks(n, 128), 128, 0, st>>>(n, n, pos, xb, code, owner, image,
                                                      b, off, max_ghosts, err);
  return cudaGetLastError();
}

cudaError_t launch_ghost_refresh(int n_real, int n_ghost, double4 *pos, double2 *xb,
                                 int *code, const int *owner, const char4 *image,
                                 const GhostBox &b, cudaStream_t st) {
  if (n_ghost > 0)
    ghost_refresh_kernel<<<blocks(n_ghost, 128), 128, 0, st>>>(n_real, n_ghost, pos, xb,
                                                               code, owner, image, b);
  return cudaGetLastError();
}

cudaError_t launch_neighbors(const NbrArgs &a, cudaStream_t st) {
  cudaError_t e;
  // bounding box of all sites, cell grid
  bbox_init_kernel<<<1, 32, 0, st>>>(a.bbox);
  bbox_kernel<<<148, 256, 0, st>>>(a.n_all, a.pos, a.bbox);
  cell_setup_kernel<<<1, 32, 0, st>>>(a.bbox, a.cell_edge, a.grid, a.max_cells, a.err);
  cudaMemsetAsync(a.cell_cnt, 0, (size_t)(a.max_cells + 1) * sizeof(int), st);
  cell_count_kernel<<<blocks(a.n_all, 256), 256, 0, st>>>(a.n_all, a.pos, a.grid, a.cell_of,
                                                          a.cell_cnt);
  if ((e = exclusive_scan(a.cell_cnt, a.cell_start, a.max_cells + 1, *a.scratch, st)) !=
      cudaSuccess)
    return e;
  cudaMemsetAsync(a.cursor, 0, (size_t)a.max_cells * sizeof(int), st);
  cell_fill_kernel<<<blocks(a.n_all, 256), 256, 0, st>>>(a.n_all, a.grid, a.cell_of, a.cell_start,
                                                         a.cursor, a.cell_sites);
  constexpr int W = 4;
  neighbor_kernel<W><<<blocks(a.n_query, W), W * 32, 0, st>>>(
      a.n_query, a.pos, a.grid, a.cell_start, a.cell_sites, a.rc, a.maxn, a.cnt, a.tmp,
      a.err, a.code, a.filter_code, a.allow_empty);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  // offsets: exclusive scan of counts with one extra zero slot at the end
  cudaMemsetAsync(a.cnt + a.n_query, 0, sizeof(int), st);
  if ((e = exclusive_scan(a.cnt, a.offs, a.n_query + 1, *a.scratch, st)) != cudaSuccess)
    return e;
  return cudaGetLastError();
}

// ---- pair links --------------------------------------------------------
// Slot of the entry of o's (ascending) list whose owner is u: a binary search
// for u itself when the pair is between real sites, else a scan of o's image
// entries (indices >= n_real, at the end of the list).
__device__ int reverse_slot(int u, bool real_pair, int o, int n_real, const int *offs,
                            const int *idx, const int *owner) {
  int lo = offs[o], hi = offs[o + 1];
  int a = lo, b = hi;  // first entry >= (real_pair ? u : n_real)
  const int key = real_pair ? u : n_real;
  while (a < b) {
    int m = (a + b) >> 1;
    if (idx[m] < key) a = m + 1;
    else b = m;
  }
  if (real_pair) return (a < hi && idx[a] == u) ? a : -1;
  for (int t = a; t < hi; ++t)
    if (owner[idx[t]] == u) return t;
  return -1;
}

__global__ void pair_rev_kernel(int n_real, const int *offs, const int *idx, const int *owner,
                                int *rev, int *own_cnt) {
  const int u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (u >= n_real) return;
  int cnt = 0;
  for (int base = offs[u]; base < offs[u + 1]; base += 32) {
    int p = base + lane;
    bool own = false;
    if (p < offs[u + 1]) {
      int j = idx[p], o = owner[j];
      int r = reverse_slot(u, j < n_real, o, n_real, offs, idx, owner);
      rev[p] = r;
      own = (u < o) || r < 0;
    }
    cnt += __popc(__ballot_sync(0xffffffffu, own));
  }
  if (lane == 0) own_cnt[u] = cnt;
}

// Owned pairs in site order, and every slot's owned pair and direction:
// slot_own = 2 t for the owned slot of pair t, 2 t + 1 for its reverse slot.
__global__ void pair_own_kernel(int n_real, const int *offs, const int *idx, const int *owner,
                                const int *rev, const int *own_off, int *own_p, int *own_u,
                                int *slot_own) {
  const int u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (u >= n_real) return;
  int at = own_off[u];
  for (int base = offs[u]; base < offs[u + 1]; base += 32) {
    int p = base + lane;
    bool own = false;
    if (p < offs[u + 1]) own = (u < owner[idx[p]]) || rev[p] < 0;
    unsigned m = __ballot_sync(0xffffffffu, own);
    if (own) {
      int k = at + __popc(m & ((1u << lane) - 1u));
      own_p[k] = p;
      own_u[k] = u;
      slot_own[p] = 2 * k;
      if (rev[p] >= 0) slot_own[rev[p]] = 2 * k + 1;
    }
    at += __popc(m);
  }
}

cudaError_t launch_pair_links(int n_real, const int *offs, const int *idx, const int *owner,
                              int *rev, int *slot_own, int *own_cnt, int *own_off, int *&own_p,
                              int *&own_u, long long &own_cap, int *n_own,
                              DeviceScratch &scratch, cudaStream_t st) {
  cudaError_t e;
  *n_own = 0;
  if (n_real <= 0) return cudaSuccess;
  const int blocks = (int)(((long long)n_real * 32 + 127) / 128);
  pair_rev_kernel<<<blocks, 128, 0, st>>>(n_real, offs, idx, owner, rev, own_cnt);
  if ((e = cudaMemsetAsync(own_cnt + n_real, 0, sizeof(int), st)) != cudaSuccess) return e;
  if ((e = exclusive_scan(own_cnt, own_off, n_real + 1, scratch, st)) != cudaSuccess) return e;
  int total = 0;
  if ((e = cudaMemcpyAsync(&total, own_off + n_real, sizeof(int), cudaMemcpyDeviceToHost, st)) !=
      cudaSuccess)
    return e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  if (total > own_cap) {
    cudaMemPool_t pool = device_pool();
    if (!pool) return cudaErrorMemoryAllocation;
    if (own_p) cudaFreeAsync(own_p, st);
    if (own_u) cudaFreeAsync(own_u, st);
    own_p = own_u = nullptr;
    own_cap = 0;
    if ((e = cudaMallocFromPoolAsync((void **)&own_p, (size_t)total * sizeof(int), pool, st)) !=
        cudaSuccess)
      return e;
    if ((e = cudaMallocFromPoolAsync((void **)&own_u, (size_t)total * sizeof(int), pool, st)) !=
        cudaSuccess)
      return e;
    own_cap = total;
  }
  int n_slots = 0;
  if ((e = cudaMemcpyAsync(&n_slots, offs + n_real, sizeof(int), cudaMemcpyDeviceToHost, st)) !=
      cudaSuccess)
    return e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  if (n_slots > 0 &&
      (e = cudaMemsetAsync(slot_own, 0xff, (size_t)n_slots * sizeof(int), st)) != cudaSuccess)
    return e;
  pair_own_kernel<<<blocks, 128, 0, st>>>(n_real, offs, idx, owner, rev, own_off, own_p, own_u,
                                          slot_own);
  *n_own = total;
  return cudaGetLastError();
}

cudaError_t launch_compact(int n_query, const int *tmp, const int *offs, int *idx,
                           cudaStream_t st) {
  if (n_query > 0)
    compact_kernel<<<blocks((long long)n_query * 32, 256), 256, 0, st>>>(n_query, tmp, offs,
                                                                         idx);
  return cudaGetLastError();
}

}  // namespace btam
