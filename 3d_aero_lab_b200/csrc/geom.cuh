// geom.cuh - device-resident grid and cut-cell geometry of one case.
#pragma once
#include <vector>
#include "common.cuh"

namespace a3d {

// Grid axes on the device: faces in FP64 (inside tests), centres and sizes in FP32 exactly
// as the reference keeps them (src/air_cfd.js:36), plus FP32 reciprocals of the sizes.
struct GridDev {
  int NX = 0, NY = 0, NZ = 0;
  double *Xf = nullptr, *Yf = nullptr, *Zf = nullptr;
  float *Xd = nullptr, *Yd = nullptr, *Zd = nullptr;
  float *Xc = nullptr, *Yc = nullptr, *Zc = nullptr;
  float *rXd = nullptr, *rYd = nullptr, *rZd = nullptr;
  std::vector<double> hXf, hYf, hZf;
  std::vector<float> hXd, hYd, hZd, hXc, hYc, hZc;
  float hYd0 = 0, hZd0 = 0;
  void* block = nullptr;  // single allocation backing all device arrays
};

// The reference's per-cell geometry arrays (src/air_cfd.js:71): t u8, phi and ap0..ap3 f32.
struct GeomDev {
  uint8_t* t = nullptr;
  float *phi = nullptr, *ap0 = nullptr, *ap1 = nullptr, *ap2 = nullptr, *ap3 = nullptr;
  void* block = nullptr;
};

// Inside-test context shared by the geometry kernels.
struct GeoDev {
  const a3d_shape* a;
  const double *Xf, *Yf, *Zf;
  const float *Xd, *Yd, *Zd, *Yc, *Zc;
  int NX, NY, NZ;
  bool volW, volH, volV;
  double hp0, hp1, cR, sR, tdR;
};

__device__ bool solid_at(const GeoDev& g, double x, double y, double z);

int grid_upload(const int32_t dims[3], const double* xf, const double* yf, const double* zf, cudaStream_t st,
                GridDev& gd);
void grid_free(GridDev& gd);
int geom_alloc(long N, GeomDev& g);
void geom_free(GeomDev& g);
int geom_build_device(const a3d_shape& shape, const GridDev& gd, double h, double delta_deg, const GeomDev& out,
                      cudaStream_t st, int64_t counts[2], int32_t vol[3]);

}  // namespace a3d
