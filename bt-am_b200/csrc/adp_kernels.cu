// Two-pass mean-field ADP kernels for sm_100a.
//
// Work decomposition (one warp per site, no atomics, fixed summation order,
// so every result is bitwise reproducible and independent of what else runs
// on the device):
//  pass 1, phase A: lanes stride over the site's neighbours; each lane
//          evaluates a pair's 12 pair-rule points, its centre point and its
//          6 neighbour-displaced triplet points (19 geometries, u/w/phi/rho
//          splines) and accumulates 22 moment sums;
//  pass 1, phase B: lane = (centre displacement d, neighbour group g),
//          d in 0..5, g in 0..4 (30 lanes): each lane accumulates the 9
//          components of G(d) plus B(g,g) over every 5th neighbour;
//  pass 1 epilogue (lane 0, FP64): energy, free entropy, dV0/dx_i and the
//          76-value moment record;
//  pass 2: lanes stride over the neighbours of u; each lane evaluates the 25
//          geometries of its pair with value+derivative splines and contracts
//          them with u's moments (staged in shared memory) and the
//          neighbour's moments (read-only cache), accumulating 5 residual
//          components.
// There is no tensor-core work: every term is a gather plus spline
// evaluation plus a handful of FMAs.  FP32 form: per-pair arithmetic in
// float, per-lane accumulation with two-sum compensation, lane/warp
// reductions and the per-site epilogue in double.
#include "adp_kernels.cuh"
#include "topo_kernels.cuh"

namespace btam {

namespace {


// Per-lane accumulator: plain double for the FP64 form, a two-sum
// compensated float pair for the FP32 form.
template <class R> struct Acc;
template <> struct Acc<double> {
  double v = 0.0;
  __device__ __forceinline__ void add(double t) { v += t; }
  __device__ __forceinline__ double get() const { return v; }
};
template <> struct Acc<float> {
  float hi = 0.0f, lo = 0.0f;
  __device__ __forceinline__ void add(float t) {
    float s = hi + t;
    float bp = s - hi;
    float e = (hi - (s - bp)) + (t - bp);
    hi = s;
    lo += e;
  }
  __device__ __forceinline__ double get() const { return (double)hi + (double)lo; }
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <class R>
__device__ __forceinline__ V3<R> pair_vec(const double4 &a, const double4 &b) {
  // the difference is taken in double so the FP32 form loses nothing to the
  // absolute coordinate magnitude
  return mk3<R>((R)(a.x - b.x), (R)(a.y - b.y), (R)(a.z - b.z));
}

__device__ __forceinline__ bool finite(double v) { return isfinite(v); }

// What the pair kernels read about a neighbour: one 32-byte load from the
// packed Site32 rows in the FP32C form, two 32-byte loads from the Site64 rows
// in the FP64 form, the separate arrays otherwise.  BO: also beta and owner
// (the pass-2 pair kernel), from the same FP64 row.
template <class R> __device__ __forceinline__ bool site_off(const EvalArgs<R> &a, int i) {
  return a.site_on && !a.site_on[i];
}

template <class R> struct NbSite {
  double x, y, z;
  R sigma, occ;
  int code;
  bool active;
  double beta;
  int owner;
};
template <class R, bool BO = false>
__device__ __forceinline__ NbSite<R> nb_site(const EvalArgs<R> &a, int j) {
  NbSite<R> n;
  if (sizeof(R) == 4 && a.s32) {
    double4 h;
    asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
        : "=d"(h.x), "=d"(h.y), "=d"(h.z), "=d"(h.w)
        : "l"(a.s32 + j));
    const long long w = __double_as_longlong(h.w);  // (sig_code, occ), low word first
    const float sig_code = __int_as_float((int)(w & 0xffffffffll));
    const float occ = __int_as_float((int)(w >> 32));
    n.x = h.x;
    n.y = h.y;
    n.z = h.z;
    n.sigma = (R)fabsf(sig_code);
    n.code = sig_code < 0.0f ? 1 : 0;
    n.occ = (R)occ;
    n.active = occ >= 0.0f;
    if (BO) {
      const SiteB e = a.sb[j];
      n.beta = e.beta;
      n.owner = e.owner;
    }
  } else if (sizeof(R) == 8 && a.s64) {
    double4 h, t;
    const double *row = reinterpret_cast<const double *>(a.s64 + j);
    asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
        : "=d"(h.x), "=d"(h.y), "=d"(h.z), "=d"(h.w)
        : "l"(row));
    asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
        : "=d"(t.x), "=d"(t.y), "=d"(t.z), "=d"(t.w)
        : "l"(row + 4));
    const long long co = __double_as_longlong(t.y);  // (code, owner), low word first
    n.x = h.x;
    n.y = h.y;
    n.z = h.z;
    n.sigma = (R)h.w;
    n.occ = (R)t.x;
    n.code = (int)(co & 0xffffffffll);
    n.active = !(t.x < kMinOcc);
    n.beta = t.z;
    n.owner = (int)(co >> 32);
  } else {
    const double4 q = a.pos[j];
    const double2 xb = a.xb[j];
    n.x = q.x;
    n.y = q.y;
    n.z = q.z;
    n.sigma = (R)q.w;
    n.occ = (R)xb.x;
    n.code = a.code[j];
    n.active = !(xb.x < kMinOcc);
    if (BO) {
      n.beta = xb.y;
      n.owner = a.owner[j];
    }
  }
  return n;
}
template <class R> __device__ __forceinline__ V3<R> pair_vec(const double4 &a, const NbSite<R> &b) {
  return mk3<R>((R)(a.x - b.x), (R)(a.y - b.y), (R)(a.z - b.z));
}
template <class R>
__device__ __forceinline__ V3<R> pair_vec(const NbSite<R> &a, const NbSite<R> &b) {
  return mk3<R>((R)(a.x - b.x), (R)(a.y - b.y), (R)(a.z - b.z));
}

// Packs the FP32C neighbour rows (Site32, SiteB) of all sites.
__global__ void pack_sites_kernel(int n, const double4 *pos, const double2 *xb, const int *code,
                                  const int *owner, Site32 *s32, SiteB *sb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 q = pos[i];
  const double2 b = xb[i];
  Site32 r;
  r.x = q.x;
  r.y = q.y;
  r.z = q.z;
  r.sig_code = code[i] == 1 ? -(float)q.w : (float)q.w;
  r.occ = b.x < kMinOcc ? -1.0f : (float)b.x;
  s32[i] = r;
  SiteB e;
  e.beta = b.y;
  e.owner = owner[i];
  e.pad = 0;
  sb[i] = e;
}

// Packs the FP64 neighbour rows (Site64) of all sites.
__global__ void pack_sites64_kernel(int n, const double4 *pos, const double2 *xb,
                                    const int *code, const int *owner, Site64 *s64) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 q = pos[i];
  const double2 b = xb[i];
  Site64 r;
  r.x = q.x;
  r.y = q.y;
  r.z = q.z;
  r.sigma = q.w;
  r.occ = b.x;
  r.code = code[i];
  r.owner = owner[i];
  r.beta = b.y;
  r.pad = 0.0;
  s64[i] = r;
}

// ---- record stores of the undirected kernels -------------------------------
// 256-bit store of 8 R.
__device__ __forceinline__ void st_rec(float *p, const float (&v)[8]) {
  asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "f"(v[0]),
               "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7])
               : "memory");
}
__device__ __forceinline__ void st_rec(double *p, const double (&v)[8]) {
  asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(v[0]), "d"(v[1]),
               "d"(v[2]), "d"(v[3])
               : "memory");
  asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p + 4), "d"(v[4]), "d"(v[5]),
               "d"(v[6]), "d"(v[7])
               : "memory");
}
// 16-byte (FP32) / 32-byte (FP64) store of the first four values of a record.
template <class R> __device__ __forceinline__ void st_rec4(R *p, const R *v);
template <> __device__ __forceinline__ void st_rec4<float>(float *p, const float *v) {
  *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
template <> __device__ __forceinline__ void st_rec4<double>(double *p, const double *v) {
  asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(v[0]), "d"(v[1]),
               "d"(v[2]), "d"(v[3])
               : "memory");
}


// One thread per owned pair t = (u, j): the pair's 12-point pair-rule record
// (pair_rule_record), shared by pass 1 of both sites and by pass 2.  Pairs
// with an empty site get a zero record.
// The tables as a kernel reads them.  SM (FP32 only): the uw block is first
// copied into the block's dynamic shared memory by all its threads, so the
// call must come before any thread leaves; the pr block stays in global
// memory.
template <class R, bool SM> struct KView { using type = RadialView<R>; };
template <> struct KView<float, true> { using type = RadialViewS<float>; };
template <> struct KView<double, true> { using type = RadialViewS<double>; };
constexpr int kUWSharedMax = 3 * kUWStride * 1200;  // values: up to 1200 segments
// Dynamic shared memory of a staging kernel: the table and its mbarrier.
template <class R> constexpr size_t uw_shared_bytes(int n) {
  return (size_t)3 * kUWStride * (size_t)n * sizeof(R) + 16;
}
// Bounded wait on phase 0 of a shared-memory mbarrier (true: completed).
__device__ __forceinline__ bool mbar_wait0(unsigned bar) {
  for (int it = 0; it < (1 << 22); ++it) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// `ok` is false (the same in every thread of the block) when the staging copy
// did not complete within two bounded waits: the timeout bit is then set and
// the block must return without touching the table; nothing recovers the
// evaluation, whose call reports BTAM_ERR_TIMEOUT.
template <class R, bool SM>
__device__ __forceinline__ typename KView<R, SM>::type kernel_view(const EvalArgs<R> &a,
                                                                   bool &ok) {
  ok = true;
  if constexpr (SM) {
    // dynamic shared memory: the table (a multiple of 32 bytes), then an
    // 8-byte mbarrier; the kernels that stage it hold no static shared memory
    extern __shared__ __align__(128) unsigned char uw_raw[];
    R *uw_dyn = reinterpret_cast<R *>(uw_raw);
    const int nuw = 3 * kUWStride * a.T.n;  // a multiple of 8 values
    bool staged = false;
    if (a.T.uws) {
      // one bulk copy of the pre-laid-out table (the tile is regular: one
      // contiguous, 16-byte aligned block), completion on the mbarrier
      const unsigned dst = (unsigned)__cvta_generic_to_shared(uw_dyn);
      const unsigned bytes = (unsigned)sizeof(R) * (unsigned)nuw;
      const unsigned bar = dst + bytes;
      if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        unsigned long long state;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 %0, [%1], %2;"
                     : "=l"(state)
                     : "r"(bar), "r"(bytes)
                     : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
            "[%3];" ::"r"(dst),
            "l"(a.T.uws), "r"(bytes), "r"(bar)
            : "memory");
        (void)state;
      }
      staged = __syncthreads_and(mbar_wait0(bar)) != 0;
      if (!staged) {  // the copy did not complete in time: flag it and wait
                      // once more; the threads never write over a copy that
                      // may still be in flight
        if (threadIdx.x == 0) atomicOr(a.err, 1 << kErrBitTimeout);
        staged = __syncthreads_and(mbar_wait0(bar)) != 0;
        if (!staged) ok = false;
      }
    }
    if (!staged && ok) {
      // 16-byte pieces c of the table, placed as ld_uw reads them: FP32
      // halves c of record c / 2, swapped where uw_swapped says; FP64
      // quarters c of record c / 4, permuted by uw_xor64
      const int npieces = nuw * (int)sizeof(R) / 16;
      for (int c = threadIdx.x; c < npieces; c += blockDim.x) {
        const int dst = sizeof(R) == 4 ? (uw_swapped(c >> 1) ? (c ^ 1) : c)
                                       : ((c & ~3) | ((c & 3) ^ uw_xor64(c >> 2)));
        reinterpret_cast<float4 *>(uw_dyn)[dst] =
            __ldg(reinterpret_cast<const float4 *>(a.T.uw) + c);
      }
      __syncthreads();
    }
    RadialViewS<R> T;
    T.uw = uw_dyn;
    T.pr = a.T.pr;
    T.dx = a.T.dx;
    T.inv_dx = a.T.inv_dx;
    T.n = a.T.n;
    return T;
  } else {
    return a.T;
  }
}

template <class R, int TPB>
__global__ void __launch_bounds__(TPB)
pass1u_pair_kernel(const EvalArgs<R> a) {
  const RadialView<R> &T = a.T;
#pragma unroll 1
  for (int t = blockIdx.x * TPB + threadIdx.x; t < a.n_own; t += gridDim.x * TPB) {
    const int p = a.own_p[t], u = a.own_u[t];
    if (site_off(a, u)) continue;
    const int j = a.idx[p];
    const NbSite<R> su = nb_site(a, u), sj = nb_site(a, j);
    if (a.x_only) {  // the four pass-1 sums, occupied or not
      R s4[kPr1];
      pair_rule_sums<R>(T, pair_vec<R>(su, sj), su.sigma, sj.sigma, su.code, sj.code, s4);
      st_rec4(a.prec1 + (size_t)kPr1 * t, s4);
      continue;
    }
    R rec[kPrRec];
    if (su.active && sj.active) {
      pair_rule_record<R>(T, pair_vec<R>(su, sj), su.sigma, sj.sigma, su.occ, sj.occ, su.code,
                          sj.code, rec);
    } else {
#pragma unroll
      for (int c = 0; c < kPrRec; ++c) rec[c] = (R)0;
    }
    st_rec4(a.prec1 + (size_t)kPr1 * t, rec);
    R *dst = a.prec2 + (size_t)kPr2 * t;
#pragma unroll
    for (int h = 0; h < kPr2 / 8; ++h) {
      R v[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) v[c] = rec[kPr1 + 8 * h + c];
      st_rec(dst + 8 * h, v);
    }
  }
}

// Sum over a group of G lanes of each lane's N partials (N a multiple of G),
// by recursive halving: at each level a lane keeps half of its current index
// range and adds its partner's values for that half (partner lane ^ G/2, ...,
// ^ 1).  In the FP32 form every addition is a two-sum and the rounding
// errors ride along as a second FP32 word (lo), so the per-site totals are
// compensated sums of the lanes' partials.  Lane L of a group ends with the
// totals of values tree_base<N, G>(L) + [0, N/G), in v[0..N/G) (+ lo).
template <int N, int M, bool FIRST, class R, int CAP>
__device__ __forceinline__ void halve_level(R (&v)[CAP], R (&lo)[CAP], int lane) {
  const bool up = (lane & M) != 0;
#pragma unroll
  for (int k = 0; k < N / 2; ++k) {
    const R keep = up ? v[N / 2 + k] : v[k];
    const R give = up ? v[k] : v[N / 2 + k];
    const R got = __shfl_xor_sync(0xffffffffu, give, M);
    if (sizeof(R) == 4) {
      R keep_lo = (R)0, got_lo = (R)0;
      if (!FIRST) {
        keep_lo = up ? lo[N / 2 + k] : lo[k];
        const R give_lo = up ? lo[k] : lo[N / 2 + k];
        got_lo = __shfl_xor_sync(0xffffffffu, give_lo, M);
      }
      const R s = keep + got;
      const R bp = s - keep;
      const R e = (keep - (s - bp)) + (got - bp);
      v[k] = s;
      lo[k] = (keep_lo + got_lo) + e;
    } else {
      v[k] = keep + got;
    }
  }
}

// The levels of a tree over groups of G lanes (G = 32, 16 or 8; masks G/2 ... 1):
// afterwards lane L of a group holds the totals of its group's values
// tree_base<N, G>(L) + [0, N/G).
template <int N, int M, class R, int CAP>
__device__ __forceinline__ void tree_levels(R (&v)[CAP], R (&lo)[CAP], int lane) {
  halve_level<N, M, N == CAP>(v, lo, lane);
  if constexpr (M > 1) tree_levels<N / 2, M / 2>(v, lo, lane);
}
template <int G, int N, class R> __device__ __forceinline__ void lane_tree(R (&v)[N], R (&lo)[N], int lane) {
  if (sizeof(R) != 4) {  // FP64: no compensation word
#pragma unroll
    for (int k = 0; k < N; ++k) lo[k] = (R)0;
  }
  tree_levels<N, G / 2>(v, lo, lane);
}
template <int N, int G> __device__ __forceinline__ int tree_base(int lane) {
  int b = 0, n = N;
#pragma unroll
  for (int m = G / 2; m >= 1; m >>= 1) {
    n >>= 1;
    if (lane & m) b += n;
  }
  return b;
}
// The total of a lane_tree value: hi + lo in the FP32 form; the FP64 form
// carries no lo word (its lo array is never written).
template <class R> __device__ __forceinline__ double tree_total(R hi, R lo) {
  return sizeof(R) == 4 ? (double)hi + (double)lo : (double)hi;
}

// Kernels are instantiated for several (warps per block, minimum resident
// blocks) shapes; the second number caps the registers per thread and so
// trades instruction-level parallelism for occupancy.  btam_autotune times
// the shapes on the actual system and keeps the fastest.
// Pass 1: one group of G lanes per site (G = 32, 16 or 8: one, two or four
// sites per warp), one lane per neighbour, in two parts (pass1_pair_part1
// and _part2, so that few accumulators are live at once): each lane
// evaluates its pairs' 13 triplet geometries (and, unless UND, their 12
// pair-rule points) and adds them to its own FP32 partials (at most
// ceil(250 / G) pairs per lane); the group then forms the per-site
// compensated totals (lane_tree) and runs the FP64 epilogue (eight lanes form
// the record's duals, one the rest).
// UND: the pair-rule sums (rho, phi, B(f, f) over the 12 pair points) come
// from the pair-rule records written by pass1u_pair_kernel instead of being
// evaluated here.
// FP64: the first pass over a site's slots keeps each active slot's pair
// vector and weight X (and its pair kind) in shared memory, up to kCap slots
// per site, for the three axis sweeps of part II, which then skip the
// neighbour's row and the vector; the cache holds a whole neighbour list
// (136 slots) where the block's static shared memory stays under 47 KB.
template <int NSITES> __host__ __device__ constexpr int p1_cache_cap() {
  constexpr int room = (47000 - NSITES * (int)sizeof(SiteSums)) / (NSITES * 33);
  return room > 136 ? 136 : (room < 0 ? 0 : room);
}

template <class R, int W, int MB, int G, bool UND>
__global__ void __launch_bounds__(W * 32, MB)
pass1_kernel(const EvalArgs<R> a) {
  constexpr int SPW = 32 / G;  // sites per warp
  __shared__ SiteSums ss[W * SPW];
  constexpr int kCap = sizeof(R) == 8 ? p1_cache_cap<W * SPW>() : 0;
  __shared__ double4 rx_s[kCap > 0 ? W * SPW * kCap : 1];  // (r0, X) per cached slot
  __shared__ signed char pk_s[kCap > 0 ? W * SPW * kCap : 1];  // pair kind, -1: inactive
  const RadialView<R> &T = a.T;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int half = lane / G, sl = lane % G, gbase = half * G;
  // grid-stride over groups of SPW sites: one group per warp per trip (a full
  // grid makes one trip; a persistent grid of a few blocks per SM makes
  // several); one copy of the body for every trip: a site gives the same
  // bits whichever trip of whichever grid computes it
#pragma unroll 1
  for (int wi = blockIdx.x * W + warp; wi * SPW < a.n_real; wi += gridDim.x * W) {
  const int i = wi * SPW + half;
  const bool live = i < a.n_real && !site_off(a, i);
  const double2 xbi = live ? a.xb[i] : make_double2(0.0, 1.0);
  const double xi = xbi.x;
  const bool act = live && !(xi < kMinOcc);
  R *mom = a.mom + (size_t)(live ? i : 0) * kMomStride;
  const double4 qi = act ? a.pos[i] : make_double4(0.0, 0.0, 0.0, 0.0);
  const int ci = act ? a.code[i] : 0;
  const int nb0 = act ? a.offs[i] : 0, nb1 = act ? a.offs[i + 1] : 0;
  double *site = reinterpret_cast<double *>(&ss[warp * SPW + half]);
  {  // part I: pair rule, centre and neighbour-displaced points
    R acc[kP1PartI], lo[kP1PartI];
#pragma unroll
    for (int c = 0; c < kP1PartI; ++c) acc[c] = (R)0;
#pragma unroll 1
    for (int p = nb0 + sl; p < nb1; p += G) {
      const NbSite<R> sj = nb_site(a, a.idx[p]);
      const int c = (warp * SPW + half) * kCap + (p - nb0);  // cache entry
      if (kCap > 0 && p - nb0 < kCap)
        pk_s[c] = sj.active ? (signed char)pair_kind(ci, sj.code) : (signed char)-1;
      if (!sj.active) continue;
      const int cj = sj.code;
      const V3<R> r0 = pair_vec<R>(qi, sj);
      if (kCap > 0 && p - nb0 < kCap)
        rx_s[c] = make_double4(r0.x, r0.y, r0.z, (double)((R)xi * sj.occ));
      if (UND) {
        const int so = a.slot_own[p];
        R rec[4];
        ld4(a.prec1 + (size_t)kPr1 * (so >> 1), rec);
        const R xj = sj.occ, X = (R)xi * xj;
        acc[kP1Rho] += xj * rec[(so & 1) ? 0 : 1];
        acc[kP1Epair] += (R)0.5 * X * rec[2];
        acc[kP1Ediag] += X * X * rec[3];
      } else {
        R rj, ep, ed;
        pass1_pair_rule<R>(T, r0, (R)qi.w, sj.sigma, (R)xi, sj.occ, ci, cj, rj, nullptr, ep,
                           ed);
        acc[kP1Rho] += rj;
        acc[kP1Epair] += ep;
        acc[kP1Ediag] += ed;
      }
      pass1_pair_part1<R>(T, r0, sj.sigma, (R)xi * sj.occ, pair_kind(ci, cj), acc);
    }
    lane_tree<G>(acc, lo, lane);
    const int v0 = tree_base<kP1PartI, G>(sl);
#pragma unroll
    for (int k = 0; k < kP1PartI / G; ++k)
      if (act && v0 + k < kP1Gd && v0 + k != kP1Sself)
        site[p1_site_slot(v0 + k)] = tree_total(acc[k], lo[k]);
  }
  if constexpr (sizeof(R) == 4) {  // part II: centre-displaced points
    R acc[kP1PartII], lo[kP1PartII];
#pragma unroll
    for (int c = 0; c < kP1PartII; ++c) acc[c] = (R)0;
#pragma unroll 1
    for (int p = nb0 + sl; p < nb1; p += G) {
      const NbSite<R> sj = nb_site(a, a.idx[p]);
      if (!sj.active) continue;
      pass1_pair_part2<R>(T, pair_vec<R>(qi, sj), (R)qi.w, (R)xi * sj.occ,
                          pair_kind(ci, sj.code), acc);
    }
    lane_tree<G>(acc, lo, lane);
    const int t0 = tree_base<kP1PartII, G>(sl);
#pragma unroll
    for (int k = 0; k < kP1PartII / G; ++k)
      if (act && t0 + k < 1 + 54)
        site[p1_site_slot(p1_part2_value(t0 + k))] = tree_total(acc[k], lo[k]);
  } else {
    // FP64: part II one axis at a time (19 live accumulators instead of 55;
    // each displaced point is still evaluated once), sself summed over the
    // three axes in axis order
    double sself = 0.0;
#pragma unroll 1
    for (int ax = 0; ax < 3; ++ax) {
      R acc[kP1PartI], lo[kP1PartI];
#pragma unroll
      for (int c = 0; c < kP1PartI; ++c) acc[c] = (R)0;
#pragma unroll 1
      for (int p = nb0 + sl; p < nb1; p += G) {
        if (kCap > 0 && p - nb0 < kCap) {
          const int c = (warp * SPW + half) * kCap + (p - nb0);
          const int pk = pk_s[c];
          if (pk < 0) continue;
          const double4 rx = rx_s[c];
          pass1_pair_part2_axis<R>(T, mk3<R>((R)rx.x, (R)rx.y, (R)rx.z), (R)qi.w, (R)rx.w, pk,
                                   ax, acc);
          continue;
        }
        const NbSite<R> sj = nb_site(a, a.idx[p]);
        if (!sj.active) continue;
        pass1_pair_part2_axis<R>(T, pair_vec<R>(qi, sj), (R)qi.w, (R)xi * sj.occ,
                                 pair_kind(ci, sj.code), ax, acc);
      }
      lane_tree<G>(acc, lo, lane);
      const int t0 = tree_base<kP1PartI, G>(sl);
#pragma unroll
      for (int k = 0; k < kP1PartI / G; ++k) {
        const int t = t0 + k;
        if (t == 0) sself += tree_total(acc[k], lo[k]);
        else if (act && t < 1 + 18)
          site[p1_site_slot(p1_part2_value(1 + 18 * ax + (t - 1)))] = tree_total(acc[k], lo[k]);
      }
    }
    // lane 0 of the group held part index 0 in every axis
    if (act && sl == 0) site[p1_site_slot(kP1Sself)] = sself;
  }
  __syncwarp();
  // epilogue: lanes 0..7 of the group form the record's eight duals, lane 0
  // the rest
  double b = 0.0;
  if (act && sl < 8) b = site_dual(ss[warp * SPW + half], sl, mom);
  double bgd = 0.0;
#pragma unroll
  for (int d = 0; d < 6; ++d) bgd += __shfl_sync(0xffffffffu, b, gbase + 2 + d);
  if (act && sl == 0) {
    SiteResult res;
    site_scalars(ss[warp * SPW + half], bgd, a.emb[ci], xi, ci, xbi.y, a.gamma[i], qi.w,
                 a.mass[ci], res, mom);
    a.rho[i] = res.rho;
    a.V0[i] = res.V0;
    a.S0[i] = res.S0;
    a.selfx[i] = res.selfx;
    if (!(finite(res.V0) && finite(res.S0) && finite(res.selfx)))
      atomicOr(a.err, 1 << kErrBitNonFinite);
  }
  if (live && !act) {  // empty site: no energy, no moments
    for (int c = sl; c < kMomStride; c += G) mom[c] = (R)0;
    if (sl == 0) a.rho[i] = a.V0[i] = a.S0[i] = a.selfx[i] = 0.0;
  }
  __syncwarp();  // the warp's shared buffers are reused by its next sites
  }
}

template <class R, int W, int MB>
__global__ void __launch_bounds__(W * 32, MB)
pass2_kernel(const EvalArgs<R> a) {
  __shared__ R mu_s[W][kMomStride];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // one copy of the body for every trip: a site or pair gives the same bits
  // whichever trip of whichever grid computes it
#pragma unroll 1
  for (int u = blockIdx.x * W + warp; u < a.n_real; u += gridDim.x * W) {
  if (site_off(a, u)) continue;
  const double2 xbu = a.xb[u];
  const double xu = xbu.x;
  if (xu < kMinOcc) {
    if (lane == 0) {
      a.Rq[3 * u] = a.Rq[3 * u + 1] = a.Rq[3 * u + 2] = 0.0;
      a.Rs[u] = a.Rx[u] = 0.0;
    }
    continue;
  }
  const R *mu_g = a.mom + (size_t)u * kMomStride;
  for (int c = lane; c < kMomStride; c += 32) mu_s[warp][c] = mu_g[c];
  __syncwarp();
  const MomRec<R, false> mu(mu_s[warp]);
  const double4 qu = a.pos[u];
  const int cu = a.code[u];
  const int nb0 = a.offs[u], nb1 = a.offs[u + 1];
  Acc<R> acc[5];
  for (int p = nb0 + lane; p < nb1; p += 32) {
    const int j = a.idx[p];
    const double2 xbj = a.xb[j];
    if (xbj.x < kMinOcc) continue;
    const int o = a.owner[j];
    const double4 qj = a.pos[j];
    const MomRec<R, true> mj(a.mom + (size_t)o * kMomStride);
    Pass2Out<R> out;
    out.gq[0] = out.gq[1] = out.gq[2] = out.gs = out.gx = (R)0;
    pass2_pair<R>(a.T, pair_vec<R>(qu, qj), (R)qu.w, (R)qj.w, (R)xu, (R)xbj.x, cu,
                  a.code[j], mu.scalar(0), mj.scalar(0), mj.scalar(1), (R)(xbj.y / xbu.y), mu,
                  mj, out);
    acc[0].add(out.gq[0]);
    acc[1].add(out.gq[1]);
    acc[2].add(out.gq[2]);
    acc[3].add(out.gs);
    acc[4].add(out.gx);
  }
  double t[5];
#pragma unroll
  for (int c = 0; c < 5; ++c) t[c] = warp_sum(acc[c].get());
  if (lane == 0) {
    double gs = t[3], gx = t[4];
    residual_epilogue(qu.w, xu, cu, xbu.y, a.gamma[u], a.selfx[u], gs, gx);
    a.Rq[3 * u] = t[0];
    a.Rq[3 * u + 1] = t[1];
    a.Rq[3 * u + 2] = t[2];
    a.Rs[u] = gs;
    a.Rx[u] = gx;
    if (!(finite(t[0]) && finite(t[1]) && finite(t[2]) && finite(gs) && finite(gx)))
      atomicOr(a.err, 1 << kErrBitNonFinite);
  }
  __syncwarp();  // mu_s is reloaded for the warp's next site
  }
}

// Mean-field stress of every real site, W0_u = sum_j dV0_u/dq_j (x) (q_j - q_u)
// at fixed sigma and x: evaluate_DV0_i_dF_bulk_MgHx (MgHx-mf-V-bulk.cpp:
// 2329-2552) at reference positions q0 = q (by translation invariance of
// V0_u, the reference's sum over the term sites a of d<term>/dq_a (x) q0_a).
// pass2_pair with omega = 0 returns the self part of pair j, the terms of
// dV0_u/dq_u that pair j carries, which is -dV0_u/dq_j; with r0 = q_u - q_j
// the pair adds self (x) r0.  Directed form, a warp per site.
template <class R, int W>
__global__ void __launch_bounds__(W * 32)
mf_stress_kernel(const EvalArgs<R> a, double *W0) {
  __shared__ R mu_s[W][kMomStride];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll 1
  for (int u = blockIdx.x * W + warp; u < a.n_real; u += gridDim.x * W) {
  const double2 xbu = a.xb[u];
  const double xu = xbu.x;
  if (xu < kMinOcc) {
    if (lane < 9) W0[9 * (size_t)u + lane] = 0.0;
    continue;
  }
  const R *mu_g = a.mom + (size_t)u * kMomStride;
  for (int c = lane; c < kMomStride; c += 32) mu_s[warp][c] = mu_g[c];
  __syncwarp();
  const MomRec<R, false> mu(mu_s[warp]);
  const double4 qu = a.pos[u];
  const int cu = a.code[u];
  Acc<R> acc[9];
  for (int p = a.offs[u] + lane; p < a.offs[u + 1]; p += 32) {
    const int j = a.idx[p];
    const double2 xbj = a.xb[j];
    if (xbj.x < kMinOcc) continue;
    const int o = a.owner[j];
    const double4 qj = a.pos[j];
    const MomRec<R, true> mj(a.mom + (size_t)o * kMomStride);
    Pass2Out<R> out;
    out.gq[0] = out.gq[1] = out.gq[2] = out.gs = out.gx = (R)0;
    const V3<R> r0 = pair_vec<R>(qu, qj);
    pass2_pair<R>(a.T, r0, (R)qu.w, (R)qj.w, (R)xu, (R)xbj.x, cu, a.code[j], mu.scalar(0),
                  mj.scalar(0), mj.scalar(1), (R)0, mu, mj, out);
    const R rv[3] = {r0.x, r0.y, r0.z};
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int d = 0; d < 3; ++d) acc[3 * c + d].add(out.gq[c] * rv[d]);
  }
  double t[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) t[c] = warp_sum(acc[c].get());
  if (lane == 0) {
    bool ok = true;
    for (int c = 0; c < 9; ++c) {
      W0[9 * (size_t)u + c] = t[c];
      ok = ok && finite(t[c]);
    }
    if (!ok) atomicOr(a.err, 1 << kErrBitNonFinite);
  }
  __syncwarp();  // mu_s is reloaded for the warp's next site
  }
}

// Per-pair terms of the residual assembly, unweighted (the reference's
// per-pair functions): a warp per real site u, a lane per slot p of u's
// list (neighbour j).  self[5u..5u+4] = dV0_u/d(q_u, sigma_u, x_u): the sum
// over u's pairs of their self parts, and dV0_u/dx_u from pass 1;
// slot[5p..5p+4] = dV0_j/d(q_u, sigma_u, x_u), the pair's cross part.  Zero
// for an empty u or j.  Reads the moment records of a directed pass 1.
template <class R, int W>
__global__ void __launch_bounds__(W * 32)
mf_pair_terms_kernel(const EvalArgs<R> a, double *self, double *slot) {
  __shared__ R mu_s[W][kMomStride];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll 1
  for (int u = blockIdx.x * W + warp; u < a.n_real; u += gridDim.x * W) {
  const double2 xbu = a.xb[u];
  const double xu = xbu.x;
  const int nb0 = a.offs[u], nb1 = a.offs[u + 1];
  if (xu < kMinOcc) {
    for (int p = nb0 + lane; p < nb1; p += 32)
      for (int c = 0; c < 5; ++c) slot[5 * (size_t)p + c] = 0.0;
    if (lane < 5) self[5 * (size_t)u + lane] = 0.0;
    continue;
  }
  const R *mu_g = a.mom + (size_t)u * kMomStride;
  for (int c = lane; c < kMomStride; c += 32) mu_s[warp][c] = mu_g[c];
  __syncwarp();
  const MomRec<R, false> mu(mu_s[warp]);
  const double4 qu = a.pos[u];
  const int cu = a.code[u];
  Acc<R> acc[4];
  bool ok = true;
  for (int p = nb0 + lane; p < nb1; p += 32) {
    const int j = a.idx[p];
    const double2 xbj = a.xb[j];
    double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (!(xbj.x < kMinOcc)) {
      const int o = a.owner[j];
      const double4 qj = a.pos[j];
      const MomRec<R, true> mj(a.mom + (size_t)o * kMomStride);
      Pass2Parts<R> P;
      pass2_pair_parts<R>(a.T, pair_vec<R>(qu, qj), (R)qu.w, (R)qj.w, (R)xu, (R)xbj.x, cu,
                          a.code[j], mu.scalar(0), mj.scalar(0), mj.scalar(1), mu, mj, P);
      acc[0].add(P.self_q[0]);
      acc[1].add(P.self_q[1]);
      acc[2].add(P.self_q[2]);
      acc[3].add(P.self_s);
      v[0] = P.cros_q[0];
      v[1] = P.cros_q[1];
      v[2] = P.cros_q[2];
      v[3] = P.cros_s;
      v[4] = P.cros_x;
    }
    for (int c = 0; c < 5; ++c) {
      slot[5 * (size_t)p + c] = v[c];
      ok = ok && finite(v[c]);
    }
  }
  double t[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) t[c] = warp_sum(acc[c].get());
  if (lane == 0) {
    for (int c = 0; c < 4; ++c) {
      self[5 * (size_t)u + c] = t[c];
      ok = ok && finite(t[c]);
    }
    self[5 * (size_t)u + 4] = a.selfx[u];
  }
  if (__any_sync(0xffffffffu, !ok) && lane == 0) atomicOr(a.err, 1 << kErrBitNonFinite);
  __syncwarp();  // mu_s is reloaded for the warp's next site
  }
}

// One owned slot p = (u, j): both directions of the pair from its 25
// geometries (pass2_pair_sym); u's part into slot p, j's part into the
// reverse slot.  Pairs with an empty site give zero records, so every slot
// of the real sites' lists is written exactly once per evaluation.
// XO: the occupancy gradients alone (EvalArgs::x_only): only prec1 is read
// and only the gx slot values are written.
template <class R, class TV, bool XO = false>
__device__ __forceinline__ void pass2u_one(const EvalArgs<R> &a, const TV &T, int t) {
  const int p = a.own_p[t], u = a.own_u[t];
  if (site_off(a, u)) return;
  const int j = a.idx[p], r = a.rev[p];
  const NbSite<R> su = nb_site<R, true>(a, u), sj = nb_site<R, true>(a, j);
  R vu[8], vj[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) vu[c] = vj[c] = (R)0;
  if (su.active && sj.active) {
    const int o = sj.owner;
    const double bu = su.beta, bj = sj.beta;
    const MomRec<R, true> mu(a.mom + (size_t)u * kMomStride);
    const MomRec<R, true> mj(a.mom + (size_t)o * kMomStride);
    Pass2Out<R> ou, oj;
    ou.gq[0] = ou.gq[1] = ou.gq[2] = ou.gs = ou.gx = (R)0;
    oj.gq[0] = oj.gq[1] = oj.gq[2] = oj.gs = oj.gx = (R)0;
    R pr[kPrRec];
    {
      R v4[4];
      ld4(a.prec1 + (size_t)kPr1 * t, v4);
#pragma unroll
      for (int c = 0; c < kPr1; ++c) pr[c] = v4[c];
    }
    if constexpr (XO) {
#pragma unroll
      for (int c = kPr1; c < kPrRec; ++c) pr[c] = (R)0;
    } else {
      const R *src = a.prec2 + (size_t)kPr2 * t;
#pragma unroll
      for (int h = 0; h < kPr2 / 8; ++h) {
        R v[8];
        ld8(src + 8 * h, v);
#pragma unroll
        for (int c = 0; c < 8; ++c) pr[kPr1 + 8 * h + c] = v[c];
      }
    }
    pass2_pair_sym<R, MomRec<R, true>, MomRec<R, true>, TV, XO>(
        T, pair_vec<R>(su, sj), su.sigma, sj.sigma, su.occ, sj.occ, su.code, sj.code,
        mu.scalar(0), mu.scalar(1), mj.scalar(0), mj.scalar(1), (R)(bj / bu), (R)(bu / bj), mu,
        mj, pr, ou, oj);
    vu[0] = ou.gq[0]; vu[1] = ou.gq[1]; vu[2] = ou.gq[2]; vu[3] = ou.gs; vu[4] = ou.gx;
    vj[0] = oj.gq[0]; vj[1] = oj.gq[1]; vj[2] = oj.gq[2]; vj[3] = oj.gs; vj[4] = oj.gx;
  }
  // slot records: (gq, gs) as one 4-vector, gx in its own array
  if (!XO) st_rec4(a.pbuf + 4 * (size_t)p, vu);
  a.pgx[p] = vu[4];
  if (r >= 0) {
    if (!XO) st_rec4(a.pbuf + 4 * (size_t)r, vj);
    a.pgx[r] = vj[4];
  }
}

// One thread per owned slot (pass2u_one).
template <class R, int TPB, int MB>
__global__ void __launch_bounds__(TPB, MB)
pass2u_pair_kernel(const EvalArgs<R> a) {
  // one copy of the body for every trip: a site or pair gives the same bits
  // whichever trip of whichever grid computes it
  if (a.x_only) {
#pragma unroll 1
    for (int t = blockIdx.x * TPB + threadIdx.x; t < a.n_own; t += gridDim.x * TPB)
      pass2u_one<R, RadialView<R>, true>(a, a.T, t);
    return;
  }
#pragma unroll 1
  for (int t = blockIdx.x * TPB + threadIdx.x; t < a.n_own; t += gridDim.x * TPB)
    pass2u_one(a, a.T, t);
}

// The same with the uw block of the tables staged in shared memory (115 KB
// in FP32, 229 KB in FP64; one block of TPB threads per SM): the triplet
// geometries of a pair then gather their spline records from shared memory
// instead of L1.
template <class R, int TPB>
__global__ void __launch_bounds__(TPB, 1)
pass2u_pair_smem_kernel(const EvalArgs<R> a) {
  bool ok;
  const auto T = kernel_view<R, true>(a, ok);
  if (!ok) return;  // the staging copy timed out (flagged)
  if (a.x_only) {
#pragma unroll 1
    for (int t = blockIdx.x * TPB + threadIdx.x; t < a.n_own; t += gridDim.x * TPB)
      pass2u_one<R, decltype(T), true>(a, T, t);
    return;
  }
#pragma unroll 1
  for (int t = blockIdx.x * TPB + threadIdx.x; t < a.n_own; t += gridDim.x * TPB)
    pass2u_one(a, T, t);
}

// One warp per site: compensated sum of its slot records in slot order,
// then the same epilogue as the directed kernel.
template <class R, int W>
__global__ void __launch_bounds__(W * 32)
pass2u_site_kernel(const EvalArgs<R> a) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // one copy of the body for every trip: a site or pair gives the same bits
  // whichever trip of whichever grid computes it
#pragma unroll 1
  for (int u = blockIdx.x * W + warp; u < a.n_real; u += gridDim.x * W) {
    if (site_off(a, u)) continue;
    const double2 xbu = a.xb[u];
    const double xu = xbu.x;
    if (xu < kMinOcc) {
      if (lane == 0) {
        a.Rq[3 * u] = a.Rq[3 * u + 1] = a.Rq[3 * u + 2] = 0.0;
        a.Rs[u] = a.Rx[u] = 0.0;
      }
      continue;
    }
    Acc<R> acc[5];
    if (a.x_only) {  // the occupancy gradients alone; R_q and R_sigma are 0
      for (int p = a.offs[u] + lane; p < a.offs[u + 1]; p += 32) acc[4].add(ld_ro(a.pgx + p));
      const double tx = warp_sum(acc[4].get());
      if (lane == 0) {
        double gs = 0.0, gx = tx;
        residual_epilogue(a.pos[u].w, xu, a.code[u], xbu.y, a.gamma[u], a.selfx[u], gs, gx);
        a.Rq[3 * u] = a.Rq[3 * u + 1] = a.Rq[3 * u + 2] = 0.0;
        a.Rs[u] = 0.0;
        a.Rx[u] = gx;
        if (!finite(gx)) atomicOr(a.err, 1 << kErrBitNonFinite);
      }
      continue;
    }
    for (int p = a.offs[u] + lane; p < a.offs[u + 1]; p += 32) {
      R v[4];
      ld4(a.pbuf + 4 * (size_t)p, v);
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[c].add(v[c]);
      acc[4].add(ld_ro(a.pgx + p));
    }
    double t[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) t[c] = warp_sum(acc[c].get());
    if (lane == 0) {
      double gs = t[3], gx = t[4];
      residual_epilogue(a.pos[u].w, xu, a.code[u], xbu.y, a.gamma[u], a.selfx[u], gs, gx);
      a.Rq[3 * u] = t[0];
      a.Rq[3 * u + 1] = t[1];
      a.Rq[3 * u + 2] = t[2];
      a.Rs[u] = gs;
      a.Rx[u] = gx;
      if (!(finite(t[0]) && finite(t[1]) && finite(t[2]) && finite(gs) && finite(gx)))
        atomicOr(a.err, 1 << kErrBitNonFinite);
    }
  }
}

// Deterministic FP64 totals in two stages.  Stage 1: block (b, k) sums the
// sites [lo + len b / P, lo + len (b + 1) / P) of system k (lo = seg[k],
// len = seg[k + 1] - lo; one system [0, n) when seg is null) with fixed
// per-thread strides and a fixed tree into part[k][b]; stage 2: one warp per
// system sums its P partials (lane-strided, then a fixed shuffle tree).  The order depends only
// on the system's own sites, so a system's totals in a batch equal its own
// totals bitwise.
__global__ void __launch_bounds__(kTotThreads)
totals_part_kernel(const int *seg, int n, const double *V0, const double *S0, const double *Rq,
                   const double *Rs, const double *Rx, double *part) {
  __shared__ double sh[4][kTotThreads];
  const int k = blockIdx.y, b = blockIdx.x, t = threadIdx.x;
  const long long lo = seg ? seg[k] : 0, len = (seg ? seg[k + 1] : n) - lo;
  const long long i0 = lo + len * b / kTotParts, i1 = lo + len * (b + 1) / kTotParts;
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  for (long long i = i0 + t; i < i1; i += kTotThreads) {
    v[0] += V0[i];
    v[1] += S0[i];
    v[2] += Rq[3 * i] * Rq[3 * i] + Rq[3 * i + 1] * Rq[3 * i + 1] +
            Rq[3 * i + 2] * Rq[3 * i + 2] + Rs[i] * Rs[i];
    v[3] += Rx[i] * Rx[i];
  }
  for (int c = 0; c < 4; ++c) sh[c][t] = v[c];
  __syncthreads();
  for (int h = kTotThreads / 2; h > 0; h >>= 1) {
    if (t < h)
      for (int c = 0; c < 4; ++c) sh[c][t] += sh[c][t + h];
    __syncthreads();
  }
  if (t < 4) part[((size_t)k * kTotParts + b) * 4 + t] = sh[t][0];
}

__global__ void __launch_bounds__(32) totals_final_kernel(const double *part, double *out) {
  const int k = blockIdx.x, lane = threadIdx.x;
  for (int c = 0; c < 4; ++c) {
    double v = 0.0;
    for (int b = lane; b < kTotParts; b += 32) v += part[((size_t)k * kTotParts + b) * 4 + c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) out[4 * k + c] = v;
  }
}

__global__ void rho_nmf_kernel(int n, const double4 *pos, const double2 *xb, const int *code,
                               const int *offs, const int *idx, SplineView<double> rmg,
                               SplineView<double> rh, double *out) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int i = warp;
  double acc = 0.0;
  if (!(xb[i].x < kMinOcc)) {
    const double4 qi = pos[i];
    for (int p = offs[i] + lane; p < offs[i + 1]; p += 32) {
      int j = idx[p];
      double xj = xb[j].x;
      if (xj < kMinOcc) continue;
      double4 qj = pos[j];
      double dx = qi.x - qj.x, dy = qi.y - qj.y, dz = qi.z - qj.z;
      double r = sqrt(dx * dx + dy * dy + dz * dz);
      acc += xj * spline_v(code[j] == 0 ? rmg : rh, r);
    }
  }
  acc = warp_sum(acc);
  if (lane == 0) out[i] = acc;
}

inline int nblocks(long long n, int per) { return (int)((n + per - 1) / per); }

}  // namespace

// Grid of a launch: one warp per site, or (persistent, variant >= 8) as many
// blocks as fit on the device at once, each warp looping over sites.
template <class K> int grid_of(K kernel, int n, int W, bool persistent) {
  int full = nblocks(n, W);
  if (!persistent) return full;
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, W * 32, 0);
  int g = sms * (per > 0 ? per : 1);
  return g < full ? g : full;
}
template <class R, int W, int MB, int G>
void go1(const EvalArgs<R> &a, cudaStream_t st, bool pers, bool und, cudaEvent_t mid) {
  const int n_groups = (a.n_real + 32 / G - 1) / (32 / G);
  if (und) {
    auto kp = pass1u_pair_kernel<R, 128>;
    int g = a.recs_ready ? 0 : nblocks(a.n_own, 128);  // kept sums: no pair-rule kernel
    if (pers && g > 0) {
      int dev = 0, sms = 0, per = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kp, 128, 0);
      int gp = sms * (per > 0 ? per : 1);
      g = gp < g ? gp : g;
    }
    if (g > 0) kp<<<g, 128, 0, st>>>(a);
    if (mid) cudaEventRecord(mid, st);
    auto k = pass1_kernel<R, W, MB, G, true>;
    k<<<grid_of(k, n_groups, W, pers), W * 32, 0, st>>>(a);
  } else {
    if (mid) cudaEventRecord(mid, st);
    auto k = pass1_kernel<R, W, MB, G, false>;
    k<<<grid_of(k, n_groups, W, pers), W * 32, 0, st>>>(a);
  }
}
// Persistent grid of a kernel that holds `smem` bytes of dynamic shared
// memory (the uw tables): as many blocks as fit on the device at once, at
// most `full`.
template <class K> int smem_grid(K kernel, int threads, size_t smem, int full) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem);
  const int g = sms * (per > 0 ? per : 1);
  return g < full ? g : full;
}

template <class R, int W, int MB> void go2(const EvalArgs<R> &a, cudaStream_t st, bool pers) {
  auto k = pass2_kernel<R, W, MB>;
  k<<<grid_of(k, a.n_real, W, pers), W * 32, 0, st>>>(a);
}

template <class R>
cudaError_t launch_pass1(const EvalArgs<R> &a, cudaStream_t st, int v, int v2, cudaEvent_t mid) {
  if (a.n_real <= 0) return cudaSuccess;
  const bool pers = (v & kPersistent) != 0;
  // the pair-rule records are made (and then also used by pass 1) whenever
  // either pass runs undirected: the undirected pass 2 reads them
  const bool und = ((v | v2) & kUndirected) != 0 && has_undirected(a);
  if (a.s32 && a.n_all > 0)
    pack_sites_kernel<<<nblocks(a.n_all, 256), 256, 0, st>>>(a.n_all, a.pos, a.xb, a.code,
                                                             a.owner, a.s32, a.sb);
  if (a.s64 && a.n_all > 0)
    pack_sites64_kernel<<<nblocks(a.n_all, 256), 256, 0, st>>>(a.n_all, a.pos, a.xb, a.code,
                                                               a.owner, a.s64);
  switch (v & (kPersistent - 1)) {
  case 1: go1<R, 4, 5, 8>(a, st, pers, und, mid); break;
  case 2: go1<R, 4, 4, 16>(a, st, pers, und, mid); break;
  case 3: go1<R, 8, 2, 16>(a, st, pers, und, mid); break;
  case 4: go1<R, 4, 5, 16>(a, st, pers, und, mid); break;
  case 5: go1<R, 4, 3, 16>(a, st, pers, und, mid); break;
  default: go1<R, 4, 1, 32>(a, st, pers, und, mid); break;
  }
  return cudaGetLastError();
}
template <class R, int TPB, int MB>
void go2u(const EvalArgs<R> &a, cudaStream_t st, bool pers, cudaEvent_t mid) {
  auto k = pass2u_pair_kernel<R, TPB, MB>;
  int g = nblocks(a.n_own, TPB);
  if (pers) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, TPB, 0);
    int gp = sms * (per > 0 ? per : 1);
    g = gp < g ? gp : g;
  }
  if (g > 0) k<<<g, TPB, 0, st>>>(a);
  if (mid) cudaEventRecord(mid, st);
  auto ks = pass2u_site_kernel<R, 4>;
  ks<<<grid_of(ks, a.n_real, 4, pers), 128, 0, st>>>(a);
}

// Shared-memory variant of the undirected pass-2 pair kernel: tables of up
// to 1200 segments (115 KB in FP32, 230 KB in FP64, within the 227 KB a
// block may hold), one block of TPB threads per SM (always a persistent
// grid); larger tables take the default shape.
template <class R, int TPB>
void go2u_smem(const EvalArgs<R> &a, cudaStream_t st, cudaEvent_t mid) {
  if (a.T.n > kUWSharedMax / (3 * kUWStride)) {
    go2u<R, 128, 1>(a, st, false, mid);
    return;
  }
  const size_t bytes = uw_shared_bytes<R>(a.T.n);
  auto k = pass2u_pair_smem_kernel<R, TPB>;
  const int g = smem_grid(k, TPB, bytes, nblocks(a.n_own, TPB));
  if (g > 0) k<<<g, TPB, bytes, st>>>(a);
  if (mid) cudaEventRecord(mid, st);
  auto ks = pass2u_site_kernel<R, 4>;
  ks<<<grid_of(ks, a.n_real, 4, true), 128, 0, st>>>(a);
}

template <class R>
cudaError_t launch_pass2(const EvalArgs<R> &a, cudaStream_t st, int v, cudaEvent_t mid) {
  if (a.n_real <= 0) return cudaSuccess;
  const bool pers = (v & kPersistent) != 0;
  if ((v & kUndirected) && has_undirected(a)) {
    switch (v & (kPersistent - 1)) {
    case 1: go2u<R, 128, 5>(a, st, pers, mid); break;
    case 2: go2u<R, 128, 4>(a, st, pers, mid); break;
    case 3: go2u<R, 256, 2>(a, st, pers, mid); break;
    case 4: go2u_smem<R, 512>(a, st, mid); break;
    case 5: go2u_smem<R, 384>(a, st, mid); break;
    case 6: go2u<R, 128, 3>(a, st, pers, mid); break;
    default: go2u<R, 128, 1>(a, st, pers, mid); break;
    }
    return cudaGetLastError();
  }
  if (mid) cudaEventRecord(mid, st);
  if (v & kUndirected) {  // links absent: the directed default
    go2<R, 4, 1>(a, st, false);
    return cudaGetLastError();
  }
  switch (v & (kPersistent - 1)) {
  case 1: go2<R, 4, 3>(a, st, pers); break;
  case 2: go2<R, 4, 4>(a, st, pers); break;
  case 3: go2<R, 4, 5>(a, st, pers); break;
  case 4: go2<R, 8, 2>(a, st, pers); break;
  case 5: go2<R, 2, 8>(a, st, pers); break;
  default: go2<R, 4, 1>(a, st, pers); break;
  }
  return cudaGetLastError();
}
template <class R>
cudaError_t launch_mf_stress(const EvalArgs<R> &a, double *W0, cudaStream_t st) {
  if (a.n_real > 0)
    mf_stress_kernel<R, 4><<<nblocks(a.n_real, 4), 128, 0, st>>>(a, W0);
  return cudaGetLastError();
}
template <class R>
cudaError_t launch_mf_pair_terms(const EvalArgs<R> &a, double *self, double *slot,
                                 cudaStream_t st) {
  if (a.n_real > 0)
    mf_pair_terms_kernel<R, 4><<<nblocks(a.n_real, 4), 128, 0, st>>>(a, self, slot);
  return cudaGetLastError();
}
template cudaError_t launch_mf_pair_terms<double>(const EvalArgs<double> &, double *, double *,
                                                  cudaStream_t);
template cudaError_t launch_mf_pair_terms<float>(const EvalArgs<float> &, double *, double *,
                                                 cudaStream_t);
template cudaError_t launch_mf_stress<double>(const EvalArgs<double> &, double *, cudaStream_t);
template cudaError_t launch_mf_stress<float>(const EvalArgs<float> &, double *, cudaStream_t);

template cudaError_t launch_pass1<double>(const EvalArgs<double> &, cudaStream_t, int, int,
                                          cudaEvent_t);
template cudaError_t launch_pass1<float>(const EvalArgs<float> &, cudaStream_t, int, int,
                                         cudaEvent_t);
template cudaError_t launch_pass2<double>(const EvalArgs<double> &, cudaStream_t, int,
                                          cudaEvent_t);
template cudaError_t launch_pass2<float>(const EvalArgs<float> &, cudaStream_t, int, cudaEvent_t);

// Times every launch variant: for each form (directed; undirected when the
// pair links exist) every pass-1 shape with a full and a persistent grid,
// then every pass-2 shape of that form after the form's best pass 1 has
// written the moments (and records) pass 2 reads; best of reps launches
// each.  The form with the smaller pass-1 + pass-2 time wins.
template <class R>
cudaError_t autotune_passes(const EvalArgs<R> &a, cudaStream_t st, int reps, int *best1,
                            int *best2) {
  cudaEvent_t e0, e1;
  cudaError_t e = cudaEventCreate(&e0);
  if (e != cudaSuccess) return e;
  e = cudaEventCreate(&e1);
  if (e != cudaSuccess) {
    cudaEventDestroy(e0);
    return e;
  }
  auto time_one = [&](bool second, int v, int v2) -> float {
    float best = 1e30f;
    for (int r = 0; r < reps && e == cudaSuccess; ++r) {
      e = cudaEventRecord(e0, st);
      if (e == cudaSuccess) e = second ? launch_pass2(a, st, v) : launch_pass1(a, st, v, v2);
      if (e == cudaSuccess) e = cudaEventRecord(e1, st);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best) best = ms;
    }
    return best;
  };
  int b1 = 0, b2 = 0;
  float best_total = 1e30f;
  const int n_forms = has_undirected(a) ? 2 : 1;
  for (int u = 0; u < n_forms && e == cudaSuccess; ++u) {
    const int form = u ? kUndirected : 0;
    int f1 = form, f2 = form;
    float t1 = 1e30f, t2 = 1e30f;
    for (int p = 0; p < 2; ++p)
      for (int v = 0; v < kPass1Variants && e == cudaSuccess; ++v) {
        const int var = v | (p ? kPersistent : 0) | form;
        float t = time_one(false, var, form);
        if (t < t1) { t1 = t; f1 = var; }
      }
    if (e == cudaSuccess) e = launch_pass1(a, st, f1, form);
    const int n2 = u ? kPass2UVariants : kPass2Variants;
    for (int p = 0; p < 2; ++p)
      for (int v = 0; v < n2 && e == cudaSuccess; ++v) {
        const int var = v | (p ? kPersistent : 0) | form;
        float t = time_one(true, var, 0);
        if (t < t2) { t2 = t; f2 = var; }
      }
    if (t1 + t2 < best_total) {
      best_total = t1 + t2;
      b1 = f1;
      b2 = f2;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e == cudaSuccess) {
    *best1 = b1;
    *best2 = b2;
  }
  return e;
}
template cudaError_t autotune_passes<double>(const EvalArgs<double> &, cudaStream_t, int, int *,
                                             int *);
template cudaError_t autotune_passes<float>(const EvalArgs<float> &, cudaStream_t, int, int *,
                                            int *);

cudaError_t launch_totals(int n_real, const double *V0, const double *S0, const double *Rq,
                          const double *Rs, const double *Rx, double *out, double *part,
                          cudaStream_t st) {
  totals_part_kernel<<<dim3(kTotParts, 1), kTotThreads, 0, st>>>(nullptr, n_real, V0, S0, Rq,
                                                                 Rs, Rx, part);
  totals_final_kernel<<<1, 32, 0, st>>>(part, out);
  return cudaGetLastError();
}

cudaError_t launch_seg_totals(int n_sys, const int *seg, const double *V0, const double *S0,
                              const double *Rq, const double *Rs, const double *Rx, double *out,
                              double *part, cudaStream_t st) {
  if (n_sys > 0) {
    totals_part_kernel<<<dim3(kTotParts, n_sys), kTotThreads, 0, st>>>(seg, 0, V0, S0, Rq, Rs,
                                                                      Rx, part);
    totals_final_kernel<<<n_sys, 32, 0, st>>>(part, out);
  }
  return cudaGetLastError();
}

cudaError_t launch_rho_nmf(int n_real, const double4 *pos, const double2 *xb, const int *code,
                           const int *offs, const int *idx, SplineView<double> rho_mg,
                           SplineView<double> rho_h, double *out, cudaStream_t st) {
  if (n_real > 0)
    rho_nmf_kernel<<<nblocks((long long)n_real * 32, 128), 128, 0, st>>>(
        n_real, pos, xb, code, offs, idx, rho_mg, rho_h, out);
  return cudaGetLastError();
}

}  // namespace btam
