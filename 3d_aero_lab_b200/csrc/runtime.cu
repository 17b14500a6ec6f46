// runtime.cu - library-wide plumbing: error strings, device selection, grid/geometry buffers.
#include <cstdarg>
#include <cstring>
#include <string>
#include "geom.cuh"

namespace a3d {

namespace {
thread_local std::string g_last_error;
}

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

void clear_error() { g_last_error.clear(); }

int use_device(int device) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    set_error("no CUDA device visible (%s)", e == cudaSuccess ? "0 devices" : cudaGetErrorString(e));
    return A3D_ERR_NODEVICE;
  }
  if (device >= 0) {
    if (device >= n) { set_error("device %d out of range (%d visible)", device, n); return A3D_ERR_ARG; }
    A3D_CUDA(cudaSetDevice(device));
  }
  return A3D_OK;
}

int grid_upload(const int32_t dims[3], const double* xf, const double* yf, const double* zf, cudaStream_t st,
                GridDev& gd) {
  gd.NX = dims[0]; gd.NY = dims[1]; gd.NZ = dims[2];
  const int n[3] = {gd.NX, gd.NY, gd.NZ};
  const double* f[3] = {xf, yf, zf};
  std::vector<double>* hf[3] = {&gd.hXf, &gd.hYf, &gd.hZf};
  std::vector<float>* hd[3] = {&gd.hXd, &gd.hYd, &gd.hZd};
  std::vector<float>* hc[3] = {&gd.hXc, &gd.hYc, &gd.hZc};
  for (int a = 0; a < 3; a++) {
    hf[a]->assign(f[a], f[a] + n[a] + 1);
    hd[a]->resize(n[a]);
    hc[a]->resize(n[a]);
    for (int i = 0; i < n[a]; i++) {  // centres and sizes stored in float32 (src/air_cfd.js:36)
      (*hc[a])[i] = (float)(0.5 * (f[a][i] + f[a][i + 1]));
      (*hd[a])[i] = (float)(f[a][i + 1] - f[a][i]);
    }
  }
  gd.hYd0 = gd.hYd[0];
  gd.hZd0 = gd.hZd[0];
  // one block: 3 face arrays (f64) then 9 float arrays, each padded to 256 bytes
  size_t off = 0, offs[12];
  for (int a = 0; a < 3; a++) { offs[a] = off; off += round_up((n[a] + 1) * 8, 256); }
  for (int k = 0; k < 9; k++) { offs[3 + k] = off; off += round_up(n[k % 3] * 4 + 4, 256); }
  char* base = nullptr;
  A3D_CUDA(cudaMalloc(&base, off));
  gd.block = base;
  double** df[3] = {&gd.Xf, &gd.Yf, &gd.Zf};
  float** dd[3] = {&gd.Xd, &gd.Yd, &gd.Zd};
  float** dc[3] = {&gd.Xc, &gd.Yc, &gd.Zc};
  float** dr[3] = {&gd.rXd, &gd.rYd, &gd.rZd};
  for (int a = 0; a < 3; a++) {
    *df[a] = (double*)(base + offs[a]);
    *dd[a] = (float*)(base + offs[3 + a]);
    *dc[a] = (float*)(base + offs[6 + a]);
    *dr[a] = (float*)(base + offs[9 + a]);
  }
  std::vector<float> rec;
  for (int a = 0; a < 3; a++) {
    A3D_CUDA(cudaMemcpy(*df[a], hf[a]->data(), (n[a] + 1) * 8, cudaMemcpyHostToDevice));
    A3D_CUDA(cudaMemcpy(*dd[a], hd[a]->data(), n[a] * 4, cudaMemcpyHostToDevice));
    A3D_CUDA(cudaMemcpy(*dc[a], hc[a]->data(), n[a] * 4, cudaMemcpyHostToDevice));
    rec.resize(n[a]);
    for (int i = 0; i < n[a]; i++) rec[i] = 1.0f / (*hd[a])[i];
    A3D_CUDA(cudaMemcpy(*dr[a], rec.data(), n[a] * 4, cudaMemcpyHostToDevice));
  }
  (void)st;
  return A3D_OK;
}

void grid_free(GridDev& gd) {
  if (gd.block) cudaFree(gd.block);
  gd.block = nullptr;
}

int geom_alloc(long N, GeomDev& g) {
  const size_t fb = round_up(N * 4, 256), tb = round_up(N, 256);
  char* base = nullptr;
  A3D_CUDA(cudaMalloc(&base, tb + 5 * fb));
  g.block = base;
  g.t = (uint8_t*)base;
  g.phi = (float*)(base + tb);
  g.ap0 = (float*)(base + tb + fb);
  g.ap1 = (float*)(base + tb + 2 * fb);
  g.ap2 = (float*)(base + tb + 3 * fb);
  g.ap3 = (float*)(base + tb + 4 * fb);
  return A3D_OK;
}

void geom_free(GeomDev& g) {
  if (g.block) cudaFree(g.block);
  g.block = nullptr;
}

}  // namespace a3d

extern "C" const char* a3d_last_error(void) { return a3d::g_last_error.c_str(); }
extern "C" int a3d_abi_version(void) { return 1; }
