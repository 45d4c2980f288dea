// Residual evaluation that allocates no device memory.
//
// Who needs this: callers whose device memory is owned by someone else and
// who must not (or cannot) call cudaMalloc/cudaFree themselves, for example
// a host framework whose caching allocator owns the whole device, a
// real-time loop where cudaMalloc's implicit device synchronisation is not
// acceptable, or an embedding that hands this library only pre-allocated
// buffers.  They pass their own device buffers for the inputs and outputs;
// the per-site moment records and per-site intermediates that the two
// kernels exchange live in the file-scope array below instead of a
// per-system cudaMalloc.
//
// Limits and sharing rules:
//  * at most kNoAllocMaxSites real sites per call (larger requests return
//    BTAM_ERR_TOO_LARGE before touching the device);
//  * the array is created when the library is loaded on a device and stays
//    allocated until the process exits (about 10.9 MB per device);
//  * every call on a device uses the same array and leaves its contents
//    behind: calls whose work overlaps on the GPU (different streams or
//    host threads at the same time) race on it and give wrong results;
//    serialise them;
//  * the first call on each device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current; make that first call
//    before any stream capture begins;
//  * a call reads the kernels' error flag back to the host and waits for
//    its stream before returning, so the host blocks until the evaluation
//    has finished.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/btam.h"
#include "adp_core.cuh"
#include "adp_kernels.cuh"
#include "topo_kernels.cuh"

using namespace btam;

namespace {

constexpr int kNoAllocMaxSites = 16384;
constexpr int kNoAllocMaxDevices = 64;
// moment records (kMomStride doubles per site; the FP32 form uses the same
// bytes as floats), then rho, S0, dV0/dx per site, then the error flag (32
// doubles' room), then the partial sums of the totals reduction
constexpr size_t kNoAllocDoubles =
    (size_t)kNoAllocMaxSites * kMomStride + 3 * (size_t)kNoAllocMaxSites + 32 + 4 * kTotParts;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

std::mutex g_noalloc_mu;
double *g_noalloc_addr[kNoAllocMaxDevices] = {nullptr};

// Device address of the scratch array on the current device (looked up once
// per device; the host-side symbol is only a handle, not a device pointer).
cudaError_t noalloc_scratch(double **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_addr[dev] = (double *)p;
  }
  *out = g_noalloc_addr[dev];
  return cudaSuccess;
}

int noalloc_status(cudaError_t e) {
  if (e == cudaSuccess) return BTAM_OK;
  if (e == cudaErrorMemoryAllocation) return BTAM_ERR_OOM;
  return BTAM_ERR_CUDA;
}

}  // namespace

// Defined in btam_capi.cu: the device table views of a loaded btam_tables.
namespace btam {
const TablesView<double> &tables_view64(const btam_tables *t);
const RadialView<double> &radial_view64(const btam_tables *t);
const RadialView<float> &radial_view32(const btam_tables *t);
double tables_mass(const btam_tables *t, int code);
}  // namespace btam

extern "C" int btam_mf_eval_noalloc(const btam_tables *t, int precision, int n_real,
                                    const double *pos4, const double *xb,
                                    const int *code, const int *owner,
                                    const double *gamma, const int *offs,
                                    const int *idx, double *V0, double *Rq,
                                    double *Rs, double *Rx, double *totals,
                                    void *stream) {
  if (!t || n_real <= 0 || !pos4 || !xb || !code || !owner || !gamma || !offs || !idx ||
      !V0 || !Rq || !Rs || !Rx || !totals)
    return BTAM_ERR_ARG;
  if (precision != BTAM_FP64 && precision != BTAM_FP32C) return BTAM_ERR_ARG;
  if (n_real > kNoAllocMaxSites) return BTAM_ERR_TOO_LARGE;
  double *scratch = nullptr;
  cudaError_t e = noalloc_scratch(&scratch);
  if (e != cudaSuccess) return noalloc_status(e);
  cudaStream_t st = (cudaStream_t)stream;
  double *mom = scratch;
  double *rho = scratch + (size_t)kNoAllocMaxSites * kMomStride;
  double *S0 = rho + kNoAllocMaxSites;
  double *selfx = S0 + kNoAllocMaxSites;
  int *err = (int *)(selfx + kNoAllocMaxSites);
  double *part = selfx + kNoAllocMaxSites + 32;
  // the only state that must start at zero: the error flag (the kernels
  // overwrite every moment record and per-site value they later read)
  e = cudaMemsetAsync(err, 0, sizeof(int), st);
  if (e != cudaSuccess) return noalloc_status(e);
  auto fill = [&](auto &a) {
    a.n_real = n_real;
    a.pos = (const double4 *)pos4;
    a.xb = (const double2 *)xb;
    a.code = code;
    a.owner = owner;
    a.gamma = gamma;
    a.offs = offs;
    a.idx = idx;
    a.emb[0] = tables_view64(t).t[T_F_MG];
    a.emb[1] = tables_view64(t).t[T_F_H];
    a.mass[0] = tables_mass(t, 0);
    a.mass[1] = tables_mass(t, 1);
    a.rho = rho;
    a.V0 = V0;
    a.S0 = S0;
    a.selfx = selfx;
    a.Rq = Rq;
    a.Rs = Rs;
    a.Rx = Rx;
    a.err = err;
  };
  if (precision == BTAM_FP64) {
    EvalArgs<double> a;
    fill(a);
    a.T = radial_view64(t);
    a.mom = mom;
    e = launch_pass1(a, st);
    if (e == cudaSuccess) e = launch_pass2(a, st);
  } else {
    EvalArgs<float> a;
    fill(a);
    a.T = radial_view32(t);
    a.mom = (float *)mom;
    e = launch_pass1(a, st);
    if (e == cudaSuccess) e = launch_pass2(a, st);
  }
  if (e == cudaSuccess) e = launch_totals(n_real, V0, S0, Rq, Rs, Rx, totals, part, st);
  int bits = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&bits, err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return noalloc_status(e);
  if (bits & (1 << kErrBitNonFinite)) return BTAM_ERR_NONFINITE;
  if (bits & (1 << kErrBitTimeout)) return BTAM_ERR_TIMEOUT;
  return bits ? BTAM_ERR_CUDA : BTAM_OK;
}
