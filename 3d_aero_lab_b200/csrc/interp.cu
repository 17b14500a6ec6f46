// interp.cu - grid sequencing: a converged coarse case's state interpolated onto a finer case
// of the same geometry (interpState, src/app_cfd.js:322-357; used by setupCFD,
// src/app_cfd.js:271-278, to pre-converge on a coarse grid before the target grid).
//
// The reference's 2-D rule in 3-D: per target cell, trilinear weights over the eight coarse
// centres around it (x fastest, then y, then z; weight (wx*wy)*wz), corners that are not fluid
// skipped and the weights renormalised; the nearest fluid coarse cell within +-3 cells (squared
// index distance, first found) when every corner is excluded; the free stream when there is
// none.  Target cells that are not fluid take the free stream, as reset() gives them.
//
// The fractional indices are separable, so the host forms them once per axis (fracIdx,
// src/app_cfd.js:322-327) in FP64; the device accumulates in FP64 with explicitly rounded
// products and sums (no contraction), so the result is bit-identical to a host evaluation.
#include <cmath>
#include <vector>
#include "solver.cuh"

namespace a3d {
namespace {

struct AxisMaps {
  const int* i0[3];
  const double* t[3];
};

struct InterpArgs {
  AxisMaps m;
  const float* QA;        // coarse state, padded layout
  const uint8_t* tA;      // coarse cell types, reference layout
  long NpA;
  int NXA, NYA, NZA, NXpA;
  float* QB;              // target state, padded layout
  const uint8_t* tB;
  long NpB;
  int NXB, NYB, NZB, NXpB;
  float F[5];             // target free stream as stored by reset()
};

__global__ void k_interp_state(InterpArgs a) {
  const long pB = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long nrow = (long)a.NYB * a.NZB * a.NXpB;
  if (pB >= nrow) return;
  const int i = (int)(pB % a.NXpB);
  const long row = pB / a.NXpB;
  const int j = (int)(row % a.NYB), k = (int)(row / a.NYB);
  float out[5] = {a.F[0], a.F[1], a.F[2], a.F[3], a.F[4]};
  if (i < a.NXB && a.tB[((long)k * a.NYB + j) * a.NXB + i] == T_FLUID) {
    const int i0 = a.m.i0[0][i], j0 = a.m.i0[1][j], k0 = a.m.i0[2][k];
    const double tx = a.m.t[0][i], ty = a.m.t[1][j], tz = a.m.t[2][k];
    double acc[5] = {0, 0, 0, 0, 0}, wsum = 0;
    for (int dk = 0; dk < 2; dk++)
      for (int dj = 0; dj < 2; dj++)
        for (int di = 0; di < 2; di++) {
          const double w = __dmul_rn(__dmul_rn(di ? tx : 1.0 - tx, dj ? ty : 1.0 - ty), dk ? tz : 1.0 - tz);
          const int ia = min(i0 + di, a.NXA - 1), ja = min(j0 + dj, a.NYA - 1), ka = min(k0 + dk, a.NZA - 1);
          if (a.tA[((long)ka * a.NYA + ja) * a.NXA + ia] != T_FLUID || w <= 0) continue;
          const long p = ((long)ka * a.NYA + ja) * a.NXpA + ia;
#pragma unroll
          for (int v = 0; v < 5; v++) acc[v] = __dadd_rn(acc[v], __dmul_rn(w, (double)a.QA[v * a.NpA + p]));
          wsum = __dadd_rn(wsum, w);
        }
    if (wsum > 0) {
#pragma unroll
      for (int v = 0; v < 5; v++) out[v] = (float)__ddiv_rn(acc[v], wsum);
    } else {
      long best = -1;
      int bd = 1 << 30;
      for (int dk = -3; dk <= 3; dk++)
        for (int dj = -3; dj <= 3; dj++)
          for (int di = -3; di <= 3; di++) {
            const int ia = min(max(i0 + di, 0), a.NXA - 1), ja = min(max(j0 + dj, 0), a.NYA - 1),
                      ka = min(max(k0 + dk, 0), a.NZA - 1);
            const int d2 = di * di + dj * dj + dk * dk;
            if (a.tA[((long)ka * a.NYA + ja) * a.NXA + ia] == T_FLUID && d2 < bd) {
              bd = d2;
              best = ((long)ka * a.NYA + ja) * a.NXpA + ia;
            }
          }
      if (best >= 0) {
#pragma unroll
        for (int v = 0; v < 5; v++) out[v] = a.QA[v * a.NpA + best];
      }
    }
  }
#pragma unroll
  for (int v = 0; v < 5; v++) a.QB[v * a.NpB + pB] = out[v];
}

// fracIdx (src/app_cfd.js:322-327): fractional index of v among the ascending centres c.
double frac_idx(const std::vector<float>& c, double v) {
  const int n = (int)c.size();
  if (v <= c[0]) return (v - c[0]) / ((double)c[1] - c[0]);
  if (v >= c[n - 1]) return n - 1 + (v - c[n - 1]) / ((double)c[n - 1] - c[n - 2]);
  int lo = 0, hi = n - 1;
  while (hi - lo > 1) {
    const int m = (lo + hi) >> 1;
    if (c[m] <= v) lo = m;
    else hi = m;
  }
  return lo + (v - c[lo]) / ((double)c[hi] - c[lo]);
}

}  // namespace
}  // namespace a3d

using namespace a3d;

extern "C" int a3d_solver_interp_state(a3d_solver* fine, const a3d_solver* coarse) {
  clear_error();
  A3D_ARG(fine && coarse, "null solver");
  A3D_ARG(fine != coarse, "target and source are the same solver");
  A3D_ARG(fine->device == coarse->device, "solvers on different devices");
  const GridDev &gA = coarse->grid, &gB = fine->grid;
  A3D_ARG(gA.NX >= 2 && gA.NY >= 2 && gA.NZ >= 2, "source grid needs two cells per axis");
  A3D_CUDA(cudaSetDevice(fine->device));
  // per-axis maps on the host: coarse base index and weight of every target centre
  const std::vector<float>* cA[3] = {&gA.hXc, &gA.hYc, &gA.hZc};
  const std::vector<float>* cB[3] = {&gB.hXc, &gB.hYc, &gB.hZc};
  const int nB[3] = {gB.NX, gB.NY, gB.NZ}, nA[3] = {gA.NX, gA.NY, gA.NZ};
  const size_t tot = (size_t)nB[0] + nB[1] + nB[2];
  std::vector<double> ht(tot);
  std::vector<int> hi(tot);
  size_t off = 0;
  for (int d = 0; d < 3; d++) {
    for (int b = 0; b < nB[d]; b++) {
      const double f = frac_idx(*cA[d], (*cB[d])[b]);
      const int i0 = std::min(std::max((int)std::floor(f), 0), nA[d] - 1);
      hi[off + b] = i0;
      ht[off + b] = std::min(std::max(f - i0, 0.0), 1.0);
    }
    off += nB[d];
  }
  void* dmap = nullptr;
  const size_t bytes = tot * (sizeof(double) + sizeof(int));
  A3D_CUDA(cudaMallocAsync(&dmap, bytes, fine->st));
  double* dt = (double*)dmap;
  int* di = (int*)(dt + tot);
  int rc = A3D_OK;
  cudaEvent_t ev = nullptr;
  auto cu = [&](cudaError_t e) {
    if (e != cudaSuccess && rc == A3D_OK) { set_error("CUDA: %s", cudaGetErrorString(e)); rc = A3D_ERR_CUDA; }
  };
  cu(cudaMemcpyAsync(dt, ht.data(), tot * sizeof(double), cudaMemcpyHostToDevice, fine->st));
  cu(cudaMemcpyAsync(di, hi.data(), tot * sizeof(int), cudaMemcpyHostToDevice, fine->st));
  // the coarse state as of this call: the target stream waits for the source stream
  cu(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  if (rc == A3D_OK) cu(cudaEventRecord(ev, coarse->st));
  if (rc == A3D_OK) cu(cudaStreamWaitEvent(fine->st, ev, 0));
  if (rc == A3D_OK) {
    InterpArgs a;
    off = 0;
    for (int d = 0; d < 3; d++) { a.m.i0[d] = di + off; a.m.t[d] = dt + off; off += nB[d]; }
    a.QA = coarse->buf[coarse->iQ]; a.tA = coarse->geo.t; a.NpA = coarse->Np;
    a.NXA = gA.NX; a.NYA = gA.NY; a.NZA = gA.NZ; a.NXpA = coarse->NXp;
    a.QB = fine->buf[fine->iQ]; a.tB = fine->geo.t; a.NpB = fine->Np;
    a.NXB = gB.NX; a.NYB = gB.NY; a.NZB = gB.NZ; a.NXpB = fine->NXp;
    for (int c = 0; c < 5; c++) a.F[c] = (float)fine->F[c];
    const long n = (long)gB.NZ * gB.NY * fine->NXp;
    k_interp_state<<<(unsigned)((n + 255) / 256), 256, 0, fine->st>>>(a);
    cu(cudaGetLastError());
    // later work on the source waits for this read of its state
    if (rc == A3D_OK) cu(cudaEventRecord(ev, fine->st));
    if (rc == A3D_OK) cu(cudaStreamWaitEvent(coarse->st, ev, 0));
  }
  cu(cudaFreeAsync(dmap, fine->st));
  if (ev) cudaEventDestroy(ev);
  if (rc != A3D_OK) return rc;
  fine->it = 0;
  fine->havePrev = false;
  fine->prevIt = 0;
  return A3D_OK;
}
