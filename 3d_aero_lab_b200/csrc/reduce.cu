// reduce.cu - force list and the FP64 post-processing reductions of a solver case:
//   cfdForceList (src/air_cfd.js:143-152)    deterministic stream compaction in cell order
//   cfdForces    (src/air_cfd.js:443-452)    C_L, C_D, C_m over the force list
//   Trefftz CD_i (src/air_cfd.js:560-570)    transverse kinetic energy on a cross plane
//   residual     (src/air_cfd.js:552-555)    RMS density change, with a non-finite flag
//   Mach max     (src/air_cfd.js:571-572)
// Every reduction runs a fixed grid of kRedBlocks CTAs that write per-CTA partials, then a
// single CTA sums the partials in a fixed order: results do not depend on scheduling.
#include <cub/block/block_reduce.cuh>
#include <cub/block/block_scan.cuh>
#include <algorithm>
#include <cmath>
#include <vector>
#include "solver.cuh"

namespace a3d {

namespace {

constexpr int kRedBlocks = 256, kRedThreads = 256;
constexpr int kFlThreads = 256, kFlPerThread = 4, kFlPerBlock = kFlThreads * kFlPerThread;
constexpr double kCG = 1.4;

struct FlArgs {
  int NX, NY, NZ;
  int k0, k1;  // owned planes
  const uint8_t* t;
  const float *ap0, *ap2, *Xd, *Yd, *Zd, *Xc, *Zc;
};

// Fluid cell whose x or z aperture jumps: projected areas cx, cz (src/air_cfd.js:146-149).
__device__ __forceinline__ bool force_entry(const FlArgs& f, long q, double& cx, double& cz) {
  if (f.t[q] != T_FLUID) return false;
  const long NX = f.NX, NXY = NX * f.NY;
  const int i = (int)(q % NX), j = (int)((q / NX) % f.NY), k = (int)(q / NXY);
  if (k < f.k0 || k >= f.k1) return false;
  const double axm = i > 0 ? (double)f.ap0[q - 1] : 1.0, azm = k > 0 ? (double)f.ap2[q - NXY] : 1.0;
  cx = ((double)f.ap0[q] - axm) * (double)f.Yd[j] * (double)f.Zd[k];
  cz = ((double)f.ap2[q] - azm) * (double)f.Xd[i] * (double)f.Yd[j];
  return cx != 0 || cz != 0;
}

__global__ void k_fl_count(FlArgs f, long N, int* counts) {
  const long base = (long)blockIdx.x * kFlPerBlock + (long)threadIdx.x * kFlPerThread;
  int n = 0;
  for (int e = 0; e < kFlPerThread; e++) {
    double cx, cz;
    if (base + e < N && force_entry(f, base + e, cx, cz)) n++;
  }
  typedef cub::BlockReduce<int, kFlThreads> BR;
  __shared__ typename BR::TempStorage tmp;
  const int tot = BR(tmp).Sum(n);
  if (threadIdx.x == 0) counts[blockIdx.x] = tot;
}

__global__ void k_fl_write(FlArgs f, long N, const long* offsets, int64_t* oq, double* ocx, double* ocz,
                           double* ox, double* oz) {
  const long base = (long)blockIdx.x * kFlPerBlock + (long)threadIdx.x * kFlPerThread;
  int n = 0;
  bool hit[kFlPerThread];
  double cx[kFlPerThread], cz[kFlPerThread];
  for (int e = 0; e < kFlPerThread; e++) {
    hit[e] = base + e < N && force_entry(f, base + e, cx[e], cz[e]);
    n += hit[e];
  }
  typedef cub::BlockScan<int, kFlThreads> BS;
  __shared__ typename BS::TempStorage tmp;
  int pre;
  BS(tmp).ExclusiveSum(n, pre);
  long o = offsets[blockIdx.x] + pre;
  const long NX = f.NX, NXY = NX * f.NY;
  for (int e = 0; e < kFlPerThread; e++) {
    if (!hit[e]) continue;
    const long q = base + e;
    oq[o] = q; ocx[o] = cx[e]; ocz[o] = cz[e];
    ox[o] = f.Xc[q % NX]; oz[o] = f.Zc[q / NXY];
    o++;
  }
}

// ---- deterministic block reduction of K doubles ----
template <int K>
__device__ __forceinline__ void block_sum_store(double v[K], double* out) {
  __shared__ double sh[K][kRedThreads / 32];
  for (int c = 0; c < K; c++)
    for (int o = 16; o; o >>= 1) v[c] += __shfl_down_sync(0xffffffffu, v[c], o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0)
    for (int c = 0; c < K; c++) sh[c][w] = v[c];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int c = 0; c < K; c++) {
      double s = 0;
      for (int x = 0; x < kRedThreads / 32; x++) s += sh[c][x];
      out[c] = s;
    }
}

template <int K>
__global__ void k_finalize(const double* partials, double* out) {
  double v[K];
  for (int c = 0; c < K; c++) v[c] = partials[threadIdx.x * K + c];  // kRedBlocks == kRedThreads
  block_sum_store<K>(v, out);
}

struct PostArgs {
  const float* Q;  // current state, component stride Np, row pitch NXp
  long Np, N;
  long q0, q1;     // owned cells in the reference layout: [q0, q1)
  int NX, NXp;
  const uint8_t* t;  // cell types in the reference layout
  __device__ __forceinline__ long pad(long q) const { return (q / NX) * NXp + q % NX; }
};

__global__ void k_forces(PostArgs p, long n, const int64_t* fq, const double* fcx, const double* fcz,
                         const double* fx, const double* fz, double xcg, double zcg, double* partials) {
  double v[3] = {0, 0, 0};
  const double pinf = 1 / kCG;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const long q = p.pad(fq[e]);
    const double r = p.Q[q], u = (double)p.Q[p.Np + q] / r, vv = (double)p.Q[2 * p.Np + q] / r,
                 w = (double)p.Q[3 * p.Np + q] / r;
    const double dp = (kCG - 1) * ((double)p.Q[4 * p.Np + q] - 0.5 * r * (u * u + vv * vv + w * w)) - pinf;
    const double Fx = -dp * fcx[e], Fz = -dp * fcz[e];
    v[0] += Fx; v[1] += Fz; v[2] += (fz[e] - zcg) * Fx - (fx[e] - xcg) * Fz;
  }
  block_sum_store<3>(v, partials + blockIdx.x * 3);
}

__global__ void k_trefftz(PostArgs p, int NX, int NY, int k0, int k1, int i0, double tx, double ca, double sa,
                          const float* Yd, const float* Zd, double* partials) {
  double v[1] = {0};
  const long M = (long)NY * (k1 - k0);
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < M; e += (long)gridDim.x * blockDim.x) {
    const int j = (int)(e % NY), k = k0 + (int)(e / NY);
    double u = 0, vv = 0, w = 0, ws = 0;
    for (int di = 0; di < 2; di++) {
      const long qr = ((long)k * NY + j) * NX + i0 + di, q = ((long)k * NY + j) * p.NXp + i0 + di;
      if (p.t[qr] != T_FLUID) continue;
      const double ww = di ? tx : 1 - tx, r = p.Q[q];
      u += ww * (double)p.Q[p.Np + q] / r;
      vv += ww * (double)p.Q[2 * p.Np + q] / r;
      w += ww * (double)p.Q[3 * p.Np + q] / r;
      ws += ww;
    }
    if (ws < 1e-6) continue;
    u /= ws; vv /= ws; w /= ws;
    const double vn = w * ca - u * sa;
    v[0] += (vv * vv + vn * vn) * (double)Yd[j] * (double)Zd[k];
  }
  block_sum_store<1>(v, partials + blockIdx.x);
}

__global__ void k_residual(PostArgs p, const float* prevR, int stride, double* partials, int* flag) {
  double v[2] = {0, 0};
  const long M = (p.N + stride - 1) / stride;
  bool bad = false;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < M; e += (long)gridDim.x * blockDim.x) {
    const long qr = e * stride, q = p.pad(qr);
    if (qr < p.q0 || qr >= p.q1 || p.t[qr] != T_FLUID) continue;
    const float r = p.Q[q];
    if (!isfinite(r)) bad = true;
    const double d = (double)r - (double)prevR[q];
    v[0] += d * d;
    v[1] += 1;
  }
  if (bad) atomicOr(flag, 1);
  block_sum_store<2>(v, partials + blockIdx.x * 2);
}

__global__ void k_mach(PostArgs p, int stride, double* partials) {
  __shared__ double sh[kRedThreads / 32];
  double m2max = 0;
  const long M = (p.N + stride - 1) / stride;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < M; e += (long)gridDim.x * blockDim.x) {
    const long qr = e * stride, q = p.pad(qr);
    if (qr < p.q0 || qr >= p.q1 || p.t[qr] != T_FLUID) continue;
    const double r = p.Q[q], u = (double)p.Q[p.Np + q] / r, v = (double)p.Q[2 * p.Np + q] / r,
                 w = (double)p.Q[3 * p.Np + q] / r;
    const double pr = (kCG - 1) * ((double)p.Q[4 * p.Np + q] - 0.5 * r * (u * u + v * v + w * w));
    const double m2 = (u * u + v * v + w * w) / (kCG * pr / r);
    if (m2 > m2max) m2max = m2;
  }
  for (int o = 16; o; o >>= 1) m2max = fmax(m2max, __shfl_down_sync(0xffffffffu, m2max, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m2max;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0;
    for (int x = 0; x < kRedThreads / 32; x++) m = fmax(m, sh[x]);
    partials[blockIdx.x] = m;
  }
}

__global__ void k_max_finalize(const double* partials, double* out) {
  __shared__ double sh[kRedThreads / 32];
  double m = partials[threadIdx.x];
  for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0;
    for (int x = 0; x < kRedThreads / 32; x++) r = fmax(r, sh[x]);
    out[0] = r;
  }
}

PostArgs post_args(a3d_solver* s) {
  PostArgs p;
  p.Q = s->buf[s->iQ];
  p.Np = s->Np;
  p.N = s->N;
  p.NX = s->grid.NX;
  p.NXp = s->NXp;
  p.t = s->geo.t;
  const long NXY = (long)s->grid.NX * s->grid.NY;
  p.q0 = s->own_k0 * NXY;
  p.q1 = s->own_k1 * NXY;
  return p;
}

FlArgs fl_args(a3d_solver* s) {
  FlArgs f;
  f.NX = s->grid.NX; f.NY = s->grid.NY; f.NZ = s->grid.NZ;
  f.k0 = s->own_k0; f.k1 = s->own_k1;
  f.t = s->geo.t; f.ap0 = s->geo.ap0; f.ap2 = s->geo.ap2;
  f.Xd = s->grid.Xd; f.Yd = s->grid.Yd; f.Zd = s->grid.Zd; f.Xc = s->grid.Xc; f.Zc = s->grid.Zc;
  return f;
}

// cfdLocate (src/air_cfd.js:453): bracketing index and weight on the float32 centres.
void locate(const std::vector<float>& c, double v, int& i, double& tx) {
  const int n = (int)c.size();
  if (v <= c[0]) { i = 0; tx = 0; return; }
  if (v >= c[n - 1]) { i = n - 2; tx = 1; return; }
  int lo = 0, hi = n - 1;
  while (hi - lo > 1) { const int m = (lo + hi) >> 1; if (c[m] <= v) lo = m; else hi = m; }
  i = lo;
  tx = (v - (double)c[lo]) / ((double)c[hi] - (double)c[lo]);
}

}  // namespace

int build_force_list(a3d_solver* s) {
  const long N = s->N;
  const long nb = (N + kFlPerBlock - 1) / kFlPerBlock;
  FlArgs f = fl_args(s);
  int* d_counts = nullptr;
  long* d_off = nullptr;
  A3D_CUDA(cudaMalloc(&d_counts, nb * sizeof(int)));
  std::vector<int> counts(nb);
  k_fl_count<<<(unsigned)nb, kFlThreads, 0, s->st>>>(f, N, d_counts);
  cudaError_t e = cudaMemcpyAsync(counts.data(), d_counts, nb * sizeof(int), cudaMemcpyDeviceToHost, s->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  if (e != cudaSuccess) { cudaFree(d_counts); set_error("force list count: %s", cudaGetErrorString(e)); return A3D_ERR_CUDA; }
  std::vector<long> off(nb);
  long tot = 0;
  for (long b = 0; b < nb; b++) { off[b] = tot; tot += counts[b]; }
  s->fl.n = tot;
  const size_t n1 = (size_t)std::max(tot, 1L);
  char* blk = nullptr;
  e = cudaMalloc(&blk, n1 * (8 + 4 * 8) + 256);
  if (e == cudaSuccess) e = cudaMalloc(&d_off, nb * sizeof(long));
  if (e != cudaSuccess) { cudaFree(d_counts); cudaFree(blk); set_error("force list alloc: %s", cudaGetErrorString(e)); return A3D_ERR_NOMEM; }
  s->fl.block = blk;
  s->fl.q = (int64_t*)blk;
  s->fl.cx = (double*)(blk + n1 * 8);
  s->fl.cz = s->fl.cx + n1;
  s->fl.x = s->fl.cz + n1;
  s->fl.z = s->fl.x + n1;
  e = cudaMemcpyAsync(d_off, off.data(), nb * sizeof(long), cudaMemcpyHostToDevice, s->st);
  if (e == cudaSuccess) {
    k_fl_write<<<(unsigned)nb, kFlThreads, 0, s->st>>>(f, N, d_off, s->fl.q, s->fl.cx, s->fl.cz, s->fl.x, s->fl.z);
    e = cudaStreamSynchronize(s->st);
  }
  cudaFree(d_counts);
  cudaFree(d_off);
  if (e != cudaSuccess) { set_error("force list write: %s", cudaGetErrorString(e)); return A3D_ERR_CUDA; }
  return A3D_OK;
}

}  // namespace a3d

using namespace a3d;

extern "C" int a3d_solver_force_list(a3d_solver* s, int64_t* n_out, int64_t cap, int64_t* q, double* cx, double* cz,
                                     double* x, double* z) {
  clear_error();
  A3D_ARG(s && n_out, "null pointer");
  A3D_CUDA(cudaSetDevice(s->device));
  *n_out = s->fl.n;
  const long n = std::min<long>(cap, s->fl.n);
  if (n > 0) {
    if (q) A3D_CUDA(cudaMemcpy(q, s->fl.q, n * 8, cudaMemcpyDeviceToHost));
    if (cx) A3D_CUDA(cudaMemcpy(cx, s->fl.cx, n * 8, cudaMemcpyDeviceToHost));
    if (cz) A3D_CUDA(cudaMemcpy(cz, s->fl.cz, n * 8, cudaMemcpyDeviceToHost));
    if (x) A3D_CUDA(cudaMemcpy(x, s->fl.x, n * 8, cudaMemcpyDeviceToHost));
    if (z) A3D_CUDA(cudaMemcpy(z, s->fl.z, n * 8, cudaMemcpyDeviceToHost));
  }
  return A3D_OK;
}

extern "C" int a3d_solver_forces(a3d_solver* s, double alpha_deg, double M, double S, double xcg, double zcg,
                                 double cref, double out[3]) {
  clear_error();
  A3D_ARG(s && out, "null pointer");
  A3D_CUDA(cudaSetDevice(s->device));
  double* part = s->d_red;
  double* res = s->d_red + 4096 * 4;
  k_forces<<<kRedBlocks, kRedThreads, 0, s->st>>>(post_args(s), s->fl.n, s->fl.q, s->fl.cx, s->fl.cz, s->fl.x,
                                                  s->fl.z, xcg, zcg, part);
  k_finalize<3><<<1, kRedThreads, 0, s->st>>>(part, res);
  A3D_CUDA(cudaGetLastError());
  A3D_CUDA(cudaMemcpyAsync(s->h_red, res, 3 * sizeof(double), cudaMemcpyDeviceToHost, s->st));
  A3D_CUDA(cudaStreamSynchronize(s->st));
  const double Fx = s->h_red[0], Fz = s->h_red[1], My = s->h_red[2];
  const double a = alpha_deg * kDeg, qd = 0.5 * M * M, k = 2 / (qd * S);  // src/air_cfd.js:450-451
  out[0] = k * (Fz * std::cos(a) - Fx * std::sin(a));
  out[1] = k * (Fx * std::cos(a) + Fz * std::sin(a));
  out[2] = k * My / cref;
  return A3D_OK;
}

extern "C" int a3d_solver_trefftz(a3d_solver* s, double xT, double alpha_deg, double M, double S, double* cdi) {
  clear_error();
  A3D_ARG(s && cdi, "null pointer");
  A3D_ARG(s->grid.NX >= 2, "Trefftz plane needs NX >= 2");
  A3D_CUDA(cudaSetDevice(s->device));
  int i0;
  double tx;
  locate(s->grid.hXc, xT, i0, tx);
  const double a = alpha_deg * kDeg, Mn = std::max(M, 0.05);
  double* part = s->d_red;
  double* res = s->d_red + 4096 * 4;
  k_trefftz<<<kRedBlocks, kRedThreads, 0, s->st>>>(post_args(s), s->grid.NX, s->grid.NY, s->own_k0, s->own_k1, i0, tx,
                                                   std::cos(a), std::sin(a), s->grid.Yd, s->grid.Zd, part);
  k_finalize<1><<<1, kRedThreads, 0, s->st>>>(part, res);
  A3D_CUDA(cudaGetLastError());
  A3D_CUDA(cudaMemcpyAsync(s->h_red, res, sizeof(double), cudaMemcpyDeviceToHost, s->st));
  A3D_CUDA(cudaStreamSynchronize(s->st));
  *cdi = 2 * s->h_red[0] / (Mn * Mn * S);
  return A3D_OK;
}

extern "C" int a3d_solver_residual(a3d_solver* s, int32_t stride, double* res_out) {
  clear_error();
  A3D_ARG(s && res_out, "null pointer");
  A3D_ARG(stride >= 1, "stride");
  A3D_CUDA(cudaSetDevice(s->device));
  const long nIt = s->it - s->prevIt;
  double res = -1;
  int rc = A3D_OK;
  if (s->havePrev && nIt > 0) {
    double* part = s->d_red;
    double* out = s->d_red + 4096 * 4;
    A3D_CUDA(cudaMemsetAsync(s->d_flag, 0, sizeof(int), s->st));
    k_residual<<<kRedBlocks, kRedThreads, 0, s->st>>>(post_args(s), s->prevR, stride, part, s->d_flag);
    k_finalize<2><<<1, kRedThreads, 0, s->st>>>(part, out);
    A3D_CUDA(cudaGetLastError());
    A3D_CUDA(cudaMemcpyAsync(s->h_red, out, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    A3D_CUDA(cudaMemcpyAsync(s->h_red + 2, s->d_flag, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    A3D_CUDA(cudaStreamSynchronize(s->st));
    int flag;
    memcpy(&flag, s->h_red + 2, sizeof(int));
    res = std::sqrt(s->h_red[0] / std::max(1.0, s->h_red[1])) / (double)nIt;
    s->res_parts[0] = s->h_red[0];
    s->res_parts[1] = s->h_red[1];
    if (flag) { set_error("non-finite density in the state"); rc = A3D_ERR_NONFINITE; }
  }
  A3D_CUDA(cudaMemcpyAsync(s->prevR, s->buf[s->iQ], s->Np * sizeof(float), cudaMemcpyDeviceToDevice, s->st));
  A3D_CUDA(cudaStreamSynchronize(s->st));
  s->prevIt = s->it;
  s->havePrev = true;
  *res_out = res;
  return rc;
}

extern "C" int a3d_solver_mach_max(a3d_solver* s, int32_t stride, double* mmax) {
  clear_error();
  A3D_ARG(s && mmax, "null pointer");
  A3D_ARG(stride >= 1, "stride");
  A3D_CUDA(cudaSetDevice(s->device));
  double* part = s->d_red;
  double* out = s->d_red + 4096 * 4;
  k_mach<<<kRedBlocks, kRedThreads, 0, s->st>>>(post_args(s), stride, part);
  k_max_finalize<<<1, kRedThreads, 0, s->st>>>(part, out);
  A3D_CUDA(cudaGetLastError());
  A3D_CUDA(cudaMemcpyAsync(s->h_red, out, sizeof(double), cudaMemcpyDeviceToHost, s->st));
  A3D_CUDA(cudaStreamSynchronize(s->st));
  *mmax = std::sqrt(s->h_red[0]);
  return A3D_OK;
}

// Planes [k0, k1) that the force list, the Trefftz plane, the residual and the Mach maximum
// cover: a z slab's own planes, without the halo planes it shares with its neighbours.
extern "C" int a3d_solver_set_owned(a3d_solver* s, int32_t k0, int32_t k1) {
  clear_error();
  A3D_ARG(s, "null solver");
  A3D_ARG(0 <= k0 && k0 < k1 && k1 <= s->grid.NZ, "owned planes must satisfy 0 <= k0 < k1 <= NZ");
  A3D_CUDA(cudaSetDevice(s->device));
  A3D_CUDA(cudaStreamSynchronize(s->st));
  s->own_k0 = k0;
  s->own_k1 = k1;
  if (s->fl.block) cudaFree(s->fl.block);
  s->fl = ForceList();
  return build_force_list(s);
}

extern "C" int a3d_solver_residual_parts(a3d_solver* s, double out[2]) {
  clear_error();
  A3D_ARG(s && out, "null pointer");
  out[0] = s->res_parts[0];
  out[1] = s->res_parts[1];
  return A3D_OK;
}
