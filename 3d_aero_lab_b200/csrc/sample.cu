// sample.cu - display sampling on the device (cfdStencil + cfdSample, src/air_cfd.js:453-482).
//
// The reference reads the whole state back (5N floats) every readback to paint surfaces,
// slices and probes.  Here the host asks for primitive states at a list of points and only
// those come back: trilinear weights over fluid and fixed-state cells around the point
// (|y| for the mirrored half), renormalised; if they vanish, the nearest fluid cell of the
// 4 x 4 x 4 neighbourhood; v negated for y < 0.  FP64 arithmetic, one thread per point.
#include <cmath>
#include "solver.cuh"

namespace a3d {

namespace {

__device__ void locate(const float* c, int n, double v, int& i, double& t) {  // cfdLocate
  if (v <= c[0]) { i = 0; t = 0; return; }
  if (v >= c[n - 1]) { i = n - 2; t = 1; return; }
  int lo = 0, hi = n - 1;
  while (hi - lo > 1) {
    const int m = (lo + hi) >> 1;
    if ((double)c[m] <= v) lo = m; else hi = m;
  }
  i = lo;
  t = (v - (double)c[lo]) / ((double)c[hi] - (double)c[lo]);
}

struct SampleArgs {
  const float* Q;
  long Np;
  int NX, NY, NZ, NXp;
  const uint8_t* t;
  const float *Xc, *Yc, *Zc;
};

__global__ void k_sample(SampleArgs a, int n, const double* __restrict__ xyz, double* __restrict__ out,
                         int* __restrict__ ok) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double x = xyz[3 * p], y = xyz[3 * p + 1], z = xyz[3 * p + 2], ay = fabs(y);
  int i, j, k;
  double tx, ty, tz;
  locate(a.Xc, a.NX, x, i, tx);
  locate(a.Yc, a.NY, ay, j, ty);
  locate(a.Zc, a.NZ, z, k, tz);
  long idx[8];
  double w[8], ws = 0;
  for (int c = 0; c < 8; c++) {
    const int di = c & 1, dj = (c >> 1) & 1, dk = c >> 2;
    const long q = ((long)(k + dk) * a.NY + (j + dj)) * a.NX + (i + di);
    const double ww = (di ? tx : 1 - tx) * (dj ? ty : 1 - ty) * (dk ? tz : 1 - tz);
    const uint8_t tt = a.t[q];
    const bool use = tt == T_FLUID || tt >= T_SINK;
    idx[c] = q;
    w[c] = use ? ww : 0;
    ws += use ? ww : 0;
  }
  if (ws > 1e-6) {
    for (int c = 0; c < 8; c++) w[c] /= ws;
  } else {  // nearest fluid cell
    long best = -1;
    double bd = INFINITY;
    for (int dk = -1; dk <= 2; dk++)
      for (int dj = -1; dj <= 2; dj++)
        for (int di = -1; di <= 2; di++) {
          const int ia = i + di, jb = j + dj, kc = k + dk;
          if (ia < 0 || jb < 0 || kc < 0 || ia >= a.NX || jb >= a.NY || kc >= a.NZ) continue;
          const long q = ((long)kc * a.NY + jb) * a.NX + ia;
          if (a.t[q] != T_FLUID) continue;
          const double ex = (double)a.Xc[ia] - x, ey = (double)a.Yc[jb] - ay, ez = (double)a.Zc[kc] - z;
          const double d2 = ex * ex + ey * ey + ez * ez;
          if (d2 < bd) { bd = d2; best = q; }
        }
    for (int c = 0; c < 8; c++) { idx[c] = best < 0 ? 0 : best; w[c] = best < 0 ? 0 : (c == 0 ? 1 : 0); }
  }
  double r = 0, ru = 0, rv = 0, rw = 0, E = 0, wsum = 0;
  for (int c = 0; c < 8; c++) {
    const double ww = w[c];
    if (!(ww != 0)) continue;
    const long q = idx[c], qp = (q / a.NX) * a.NXp + q % a.NX;
    r += ww * (double)a.Q[qp];
    ru += ww * (double)a.Q[a.Np + qp];
    rv += ww * (double)a.Q[2 * a.Np + qp];
    rw += ww * (double)a.Q[3 * a.Np + qp];
    E += ww * (double)a.Q[4 * a.Np + qp];
    wsum += ww;
  }
  double* o = out + 5 * p;
  if (wsum == 0) {
    ok[p] = 0;
    for (int c = 0; c < 5; c++) o[c] = 0;
    return;
  }
  const double ysgn = y < 0 ? -1 : 1;
  r = fmax(r, 1e-6);
  const double u = ru / r, v = rv / r * ysgn, wv = rw / r;
  o[0] = r; o[1] = u; o[2] = v; o[3] = wv;
  o[4] = fmax((kGamma - 1) * (E - 0.5 * r * (u * u + v * v + wv * wv)), 1e-7);
  ok[p] = 1;
}

}  // namespace

}  // namespace a3d

using namespace a3d;

extern "C" int a3d_solver_sample(a3d_solver* s, int32_t n, const double* xyz, double* out5, int32_t* ok) {
  clear_error();
  A3D_ARG(s && n >= 0 && (n == 0 || (xyz && out5 && ok)), "sample arguments");
  A3D_ARG(s->grid.NX >= 2 && s->grid.NY >= 2 && s->grid.NZ >= 2, "sampling needs two cells per axis");
  if (n == 0) return A3D_OK;
  A3D_CUDA(cudaSetDevice(s->device));
  char* buf = nullptr;
  const size_t bx = (size_t)n * 3 * 8, bo = (size_t)n * 5 * 8, bk = (size_t)n * 4;
  A3D_CUDA(cudaMallocAsync(&buf, bx + bo + bk, s->st));
  double* dxyz = (double*)buf;
  double* dout = (double*)(buf + bx);
  int* dok = (int*)(buf + bx + bo);
  SampleArgs a;
  a.Q = s->buf[s->iQ]; a.Np = s->Np; a.NX = s->grid.NX; a.NY = s->grid.NY; a.NZ = s->grid.NZ; a.NXp = s->NXp;
  a.t = s->geo.t; a.Xc = s->grid.Xc; a.Yc = s->grid.Yc; a.Zc = s->grid.Zc;
  cudaError_t e = cudaMemcpyAsync(dxyz, xyz, bx, cudaMemcpyHostToDevice, s->st);
  if (e == cudaSuccess) {
    k_sample<<<(n + 127) / 128, 128, 0, s->st>>>(a, n, dxyz, dout, dok);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out5, dout, bo, cudaMemcpyDeviceToHost, s->st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ok, dok, bk, cudaMemcpyDeviceToHost, s->st);
  cudaFreeAsync(buf, s->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  if (e != cudaSuccess) { set_error("sample: %s", cudaGetErrorString(e)); return A3D_ERR_CUDA; }
  return A3D_OK;
}
