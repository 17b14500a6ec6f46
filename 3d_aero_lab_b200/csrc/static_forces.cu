// static_forces.cu - the pressure-force integral (cfdForces) for callers that cannot allocate
// device memory.
//
// a3d_solver_forces keeps its partial sums in scratch that the solver allocated with
// cudaMalloc when it was created.  Some callers have no solver object and may not call
// cudaMalloc at all: an N-API addon running inside a host application that hands it a
// fixed, pre-sized pool of device memory, or code that must not change the device's
// allocation state while another component is capturing or replaying work.  They own the
// state and force-list arrays already and need only the integral.  This entry point uses
// a file-scope __device__ array as its scratch instead: the array is part of the loaded
// module, so every GPU that loads the library holds it (about 96 KiB) until the process
// exits, and no call allocates or frees anything.
#include "solver.cuh"

namespace a3d {

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 4096;                                  // partials the scratch can hold
constexpr long kMaxEntries = (long)kMaxBlocks * kThreads;         // 1,048,576 force-list cells
constexpr int kScratchDoubles = 3 * kMaxBlocks + 3;               // partials, then the 3 totals

// Shared by every call on a device; it keeps the previous call's contents.  Each call writes
// every partial it reads before reading it, so nothing has to start at zero.
__device__ __align__(256) double g_force_scratch[kScratchDoubles];

// Device address of the scratch in the current context.  In host code `g_force_scratch` names a
// host-side shadow, not device memory, so it is never passed to a kernel directly.  The address
// is looked up on every call (a query that allocates nothing): a cached one would go stale if
// the device were reset and the library's module loaded again at another address.  The first
// call on a device may load the module, so it belongs before any stream capture.
int scratch_for_current_device(double** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_force_scratch);
  if (e != cudaSuccess || !p) {
    set_error("cudaGetSymbolAddress(force scratch) failed: %s", cudaGetErrorString(e));
    return A3D_ERR_CUDA;
  }
  *out = (double*)p;
  return A3D_OK;
}

// One CTA per 256 list cells: FP64 Fx, Fz, My partials (src/air_cfd.js:445-449).
__global__ void k_force_partials(const float* __restrict__ r, const float* __restrict__ ru,
                                 const float* __restrict__ rv, const float* __restrict__ rw,
                                 const float* __restrict__ E, long n, const int64_t* __restrict__ fq,
                                 const double* __restrict__ fcx, const double* __restrict__ fcz,
                                 const double* __restrict__ fx, const double* __restrict__ fz, double xcg,
                                 double zcg, double* scratch) {
  __shared__ double sh[3][kThreads / 32];
  double v[3] = {0, 0, 0};
  const long e = (long)blockIdx.x * kThreads + threadIdx.x;
  if (e < n) {
    const long q = fq[e];
    const double rr = r[q], u = (double)ru[q] / rr, vv = (double)rv[q] / rr, w = (double)rw[q] / rr;
    const double dp = (kGamma - 1) * ((double)E[q] - 0.5 * rr * (u * u + vv * vv + w * w)) - 1 / kGamma;
    const double Fx = -dp * fcx[e], Fz = -dp * fcz[e];
    v[0] = Fx; v[1] = Fz; v[2] = (fz[e] - zcg) * Fx - (fx[e] - xcg) * Fz;
  }
  for (int c = 0; c < 3; c++)
    for (int o = 16; o; o >>= 1) v[c] += __shfl_down_sync(0xffffffffu, v[c], o);
  if ((threadIdx.x & 31) == 0)
    for (int c = 0; c < 3; c++) sh[c][threadIdx.x >> 5] = v[c];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int c = 0; c < 3; c++) {
      double s = 0;
      for (int w2 = 0; w2 < kThreads / 32; w2++) s += sh[c][w2];
      scratch[3 * blockIdx.x + c] = s;
    }
}

// Sums the partials of this call in a fixed order into the three totals at the scratch tail.
__global__ void k_force_total(int nb, double* scratch) {
  __shared__ double sh[3][kThreads / 32];
  double v[3] = {0, 0, 0};
  for (int b = threadIdx.x; b < nb; b += kThreads)
    for (int c = 0; c < 3; c++) v[c] += scratch[3 * b + c];
  for (int c = 0; c < 3; c++)
    for (int o = 16; o; o >>= 1) v[c] += __shfl_down_sync(0xffffffffu, v[c], o);
  if ((threadIdx.x & 31) == 0)
    for (int c = 0; c < 3; c++) sh[c][threadIdx.x >> 5] = v[c];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int c = 0; c < 3; c++) {
      double s = 0;
      for (int w2 = 0; w2 < kThreads / 32; w2++) s += sh[c][w2];
      scratch[3 * kMaxBlocks + c] = s;
    }
}

}  // namespace

}  // namespace a3d

using namespace a3d;

extern "C" int a3d_forces_noalloc(const float* r, const float* ru, const float* rv, const float* rw, const float* E,
                                  int64_t n, const int64_t* q, const double* cx, const double* cz, const double* x,
                                  const double* z, double alpha_deg, double M, double S, double xcg, double zcg,
                                  double cref, void* stream, double out[3]) {
  clear_error();
  A3D_ARG(out, "null output");
  A3D_ARG(n >= 0, "negative force-list length");
  if (n > kMaxEntries) {
    set_error("force list of %lld cells exceeds the static scratch limit of %ld cells", (long long)n, kMaxEntries);
    return A3D_ERR_ARG;
  }
  A3D_ARG(n == 0 || (r && ru && rv && rw && E && q && cx && cz && x && z), "null device array");
  A3D_TRY(use_device(-1));
  double* scratch = nullptr;
  A3D_TRY(scratch_for_current_device(&scratch));
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = (int)((n + kThreads - 1) / kThreads);
  if (nb > 0)
    k_force_partials<<<nb, kThreads, 0, st>>>(r, ru, rv, rw, E, n, q, cx, cz, x, z, xcg, zcg, scratch);
  k_force_total<<<1, kThreads, 0, st>>>(nb, scratch);
  A3D_CUDA(cudaGetLastError());
  double tot[3];
  A3D_CUDA(cudaMemcpyAsync(tot, scratch + 3 * kMaxBlocks, sizeof tot, cudaMemcpyDeviceToHost, st));
  A3D_CUDA(cudaStreamSynchronize(st));
  const double a = alpha_deg * kDeg, qd = 0.5 * M * M, k = 2 / (qd * S);  // src/air_cfd.js:450-451
  out[0] = k * (tot[1] * std::cos(a) - tot[0] * std::sin(a));
  out[1] = k * (tot[0] * std::cos(a) + tot[1] * std::sin(a));
  out[2] = k * tot[2] / cref;
  return A3D_OK;
}
