// geom.cu - cut-cell geometry on the GPU (cfdGeom, src/air_cfd.js:50-141).
//
// Every node of the grid and every sub-sample point of a cut cell runs the inside
// tests of the aircraft (fuselage, volume wing/tail when they are thicker than 1.5
// cells, fin, podded-nacelle envelope; src/air_cfd.js:60-67 and src/air_field.js:115-134)
// in FP64 on the device.  The kernels follow the reference's sequence:
//   node inside flags -> phi (27 samples) and +face apertures (9 samples) -> thin-wing
//   baffles (wing, then the deflected tail) -> solid test phi < 0.2 -> fixed-state jet
//   and intake layers -> face clean-up next to solids -> forced-open fixed-cell faces.
// Results are bit-identical to the reference's arithmetic wherever the device's double
// transcendentals round like the host's; the tests compare every cell.
#include <cmath>
#include <vector>
#include "geom.cuh"

namespace a3d {

namespace {

__device__ __forceinline__ double naca_t(double t, double x) {  // src/aircraft.js:58
  x = fmax(0.0, fmin(1.0, x));
  return 5 * t * (0.2969 * sqrt(x) - 0.126 * x - 0.3516 * x * x + 0.2843 * pow(x, 3.0) - 0.1036 * pow(x, 4.0));
}
__device__ __forceinline__ double naca_c(double m, double x) {  // src/aircraft.js:59, p = 0.4
  const double p = 0.4;
  if (m == 0) return 0;
  return x < p ? m / (p * p) * (2 * p * x - x * x) : m / pow(1 - p, 2.0) * ((1 - 2 * p) + 2 * p * x - x * x);
}
__device__ __forceinline__ double s_chord(const a3d_surface& S, double s) { return S.cr + (S.ct - S.cr) * s / S.semi; }
__device__ __forceinline__ double s_xle(const a3d_surface& S, double s) { return S.x0 + s * S.tanL; }
__device__ __forceinline__ double s_tc(const a3d_surface& S, double s) { return S.tcR + (S.tcT - S.tcR) * s / S.semi; }

__device__ double fus_radius(const a3d_shape& a, double x) {  // src/aircraft.js:66-72
  if (x <= 0) return 0;
  if (x < a.fus_Ln) { const double s = 1 - x / a.fus_Ln; return a.fus_R0 * pow(fmax(0.0, 1 - s * s), a.fus_noseP); }
  if (x <= a.fus_xt0) return a.fus_R0;
  if (x >= a.fus_L) return a.fus_Re;
  const double t = (x - a.fus_xt0) / a.fus_Lt;
  return a.fus_Re + (a.fus_R0 - a.fus_Re) * 0.5 * (1 + cos(kPi * t));
}
__device__ __forceinline__ double fus_center(const a3d_shape& a, double x) {  // src/aircraft.js:73
  return x <= a.fus_xt0 ? 0 : a.fus_tailUp * a.fus_R0 * pow((x - a.fus_xt0) / a.fus_Lt, 2.0);
}

// Point inside the thickness envelope of a lifting surface (AirGeom.inLift).
__device__ bool in_lift(const a3d_surface& S, double x, double ay, double z) {
  if (x < S.bb[0] || x > S.bb[1] || z < S.bb[2] || z > S.bb[3] || ay > S.semi) return false;
  const double c = s_chord(S, ay), xc = (x - s_xle(S, ay)) / c;
  if (xc < 0 || xc > 1) return false;
  const double th = naca_t(s_tc(S, ay), xc) * c * (ay >= S.semi - 1e-6 ? 0 : 1);
  const double zm = S.z0 + (ay - S.sA) * S.tanD_deg + naca_c(S.camber, xc) * c + (-(xc - 0.25) * c * S.tanI_deg);
  return z >= zm - th && z <= zm + th;
}
// Point inside the fin on the symmetry plane (AirGeom.inVt).
__device__ bool in_fin(const a3d_surface& V, double x, double ay, double z) {
  const double s = z - V.z0;
  if (s < -0.5 || s > V.semi) return false;
  const double ss = fmax(0.0, s), c = s_chord(V, ss), xc = (x - s_xle(V, ss)) / c;
  if (xc < 0 || xc > 1) return false;
  return ay <= naca_t(s_tc(V, ss), xc) * c;
}

}  // namespace

__device__ bool solid_at(const GeoDev& g, double x, double y, double z) {
  const a3d_shape& a = *g.a;
  const double ay = fabs(y);
  for (int e = 0; e < a.n_engines; e++) {  // podded nacelle envelope (float32 radius table)
    const a3d_engine& v = a.engines[e];
    if (v.internal || v.env_n == 0) continue;
    const double xe = x - v.x0;
    if (xe < 0 || xe > v.env_xmax) continue;
    const double f = xe / v.env_xmax * v.env_n;
    const int k = min(v.env_n - 1, (int)floor(f));
    const double r = (double)v.env_R[k] + ((double)v.env_R[k + 1] - (double)v.env_R[k]) * (f - k);
    if (hypot(ay - v.y, z - v.z) < r) return true;
  }
  if (x >= 0 && x <= a.fus_L) {  // fuselage (AirGeom.inFus)
    const double R = fus_radius(a, x), dz = z - fus_center(a, x);
    if (ay * ay + dz * dz <= R * R) return true;
  }
  if (g.volW && ay >= a.wing.sA * 0.9 && in_lift(a.wing, x, ay, z)) return true;
  if (g.volH && ay >= a.htail.sA * 0.9) {  // tail deflected by delta about its quarter root chord
    const double dx = x - g.hp0, dz = z - g.hp1;
    if (in_lift(a.htail, g.hp0 + dx * g.cR - dz * g.sR, ay, g.hp1 + dx * g.sR + dz * g.cR)) return true;
  }
  return g.volV && in_fin(a.vtail, x, ay, z);
}

namespace {

__constant__ double kSub[3] = {1.0 / 6, 0.5, 5.0 / 6};  // sub-sample offsets (src/air_cfd.js:72)

__global__ void k_nodes(GeoDev g, uint8_t* cin) {
  const long NX1 = g.NX + 1, NY1 = g.NY + 1, total = NX1 * NY1 * (g.NZ + 1);
  for (long n = blockIdx.x * (long)blockDim.x + threadIdx.x; n < total; n += (long)gridDim.x * blockDim.x) {
    const int i = (int)(n % NX1), j = (int)((n / NX1) % NY1), k = (int)(n / (NX1 * NY1));
    cin[n] = solid_at(g, g.Xf[i], g.Yf[j], g.Zf[k]) ? 1 : 0;
  }
}

// phi by 27 sub-samples and the three +face apertures by 9 sub-samples (src/air_cfd.js:73-90).
__global__ void k_cells(GeoDev g, const uint8_t* cin, float* phi, float* ap0, float* ap1, float* ap2, float* ap3) {
  const long NX = g.NX, NY = g.NY, N = NX * NY * g.NZ;
  const long NX1 = NX + 1, NXY1 = NX1 * (NY + 1);
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < N; q += (long)gridDim.x * blockDim.x) {
    const int i = (int)(q % NX), j = (int)((q / NX) % NY), k = (int)(q / (NX * NY));
    auto cn = [&](int a, int b, int c) { return (int)cin[c * NXY1 + b * NX1 + a]; };
    const double xf = g.Xf[i], yf = g.Yf[j], zf = g.Zf[k];
    const double xd = g.Xd[i], yd = g.Yd[j], zd = g.Zd[k];
    int s = 0;
    for (int c = 0; c < 8; c++) s += cn(i + (c & 1), j + ((c >> 1) & 1), k + (c >> 2));
    float ph;
    if (s == 0) ph = 1.f;
    else if (s == 8) ph = 0.f;
    else {
      int n = 0;
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
          for (int c = 0; c < 3; c++)
            if (!solid_at(g, xf + kSub[a] * xd, yf + kSub[b] * yd, zf + kSub[c] * zd)) n++;
      ph = (float)(n / 27.0);
    }
    phi[q] = ph;
    float apv[3];
    for (int d = 0; d < 3; d++) {
      int m;
      if (d == 0) m = cn(i + 1, j, k) + cn(i + 1, j + 1, k) + cn(i + 1, j, k + 1) + cn(i + 1, j + 1, k + 1);
      else if (d == 1) m = cn(i, j + 1, k) + cn(i + 1, j + 1, k) + cn(i, j + 1, k + 1) + cn(i + 1, j + 1, k + 1);
      else m = cn(i, j, k + 1) + cn(i + 1, j, k + 1) + cn(i, j + 1, k + 1) + cn(i + 1, j + 1, k + 1);
      if (m == 0) { apv[d] = 1.f; continue; }
      if (m == 4) { apv[d] = 0.f; continue; }
      int n = 0;
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
          const double x = d == 0 ? g.Xf[i + 1] : xf + kSub[a] * xd;
          const double y = d == 1 ? g.Yf[j + 1] : yf + (d == 0 ? kSub[a] : kSub[b]) * yd;
          const double z = d == 2 ? g.Zf[k + 1] : zf + kSub[b] * zd;
          if (!solid_at(g, x, y, z)) n++;
        }
      apv[d] = (float)(n / 9.0);
    }
    ap0[q] = apv[0]; ap1[q] = apv[1]; ap2[q] = apv[2]; ap3[q] = 0.f;
  }
}

// Camber-surface height of a thin surface at (x, |y|), or false outside its planform
// (zMean, src/air_cfd.js:92).
__device__ bool camber_z(const a3d_surface& S, double sA, double x, double ay, double& z) {
  if (ay > S.semi || ay < sA) return false;
  const double c = s_chord(S, ay), xc = (x - s_xle(S, ay)) / c;
  if (xc < 0 || xc > 1) return false;
  z = S.z0 + (ay - sA) * S.tanD_deg + naca_c(S.camber, xc) * c - (xc - 0.25) * c * S.tanI_deg;
  return true;
}

// Baffle on the z face nearest the mean camber surface of column (i, j): the face aperture
// is reduced by the planform coverage and the local slope dz/dx is stored in ap3
// (src/air_cfd.js:94-111).  One thread per column; columns never share a cell.
__global__ void k_baffle(GeoDev g, int which, float* ap2, float* ap3) {
  const a3d_surface& S = which == 0 ? g.a->wing : g.a->htail;
  const double sA = S.sA;
  const bool rot = which == 1;
  const long NX = g.NX, NY = g.NY;
  for (long n = blockIdx.x * (long)blockDim.x + threadIdx.x; n < NX * NY; n += (long)gridDim.x * blockDim.x) {
    const int i = (int)(n % NX), j = (int)(n / NX);
    if (g.Yf[j] > S.semi || g.Yf[j + 1] < sA) continue;
    int cov = 0;
    double zs = 0, ss = 0;
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) {
        const double x = g.Xf[i] + kSub[a] * (double)g.Xd[i], y = g.Yf[j] + kSub[b] * (double)g.Yd[j];
        double zm, z1, z0;
        if (!camber_z(S, sA, x, y, zm)) continue;
        const double e = 0.02 * s_chord(S, fmin(y, S.semi));
        const bool ok1 = camber_z(S, sA, x + e, y, z1), ok0 = camber_z(S, sA, x - e, y, z0);
        double sl = (ok1 && ok0) ? (z1 - z0) / (2 * e) : ok1 ? (z1 - zm) / e : ok0 ? (zm - z0) / e : 0;
        if (rot) { zm -= (x - g.hp0) * g.tdR; sl -= g.tdR; }
        cov++; zs += zm; ss += sl;
      }
    if (!cov) continue;
    const double zm = zs / cov;
    int k = 0;
    while (k < g.NZ - 2 && (double)g.Zc[k + 1] <= zm) k++;
    const long q = ((long)k * NY + j) * NX + i;
    ap2[q] = (float)fmin((double)ap2[q], 1 - cov / 9.0);
    ap3[q] = (float)(ss / cov);
  }
}

__global__ void k_solid(long N, const float* phi, uint8_t* t) {  // src/air_cfd.js:114
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < N; q += (long)gridDim.x * blockDim.x)
    t[q] = phi[q] < 0.2 ? T_SOLID : T_FLUID;
}

// One fixed-state layer at x index i: cells whose centre lies in the ring [rin - pad, rout + pad]
// around the engine axis become type `ty` with phi = 1 (src/air_cfd.js:123, 128).
__global__ void k_mark(GeoDev g, int i, double ey, double ez, double rin, double rout, int ty, uint8_t bit,
                       uint8_t* t, float* phi, uint8_t* mark, unsigned long long* count) {
  const long NY = g.NY, NZ = g.NZ;
  for (long n = blockIdx.x * (long)blockDim.x + threadIdx.x; n < NY * NZ; n += (long)gridDim.x * blockDim.x) {
    const int j = (int)(n % NY), k = (int)(n / NY);
    const double r = hypot((double)g.Yc[j] - ey, (double)g.Zc[k] - ez);
    if (r <= rout && r >= rin) {
      const long q = ((long)k * NY + j) * g.NX + i;
      t[q] = (uint8_t)ty; phi[q] = 1.f; mark[q] |= bit;
      atomicAdd(count, 1ULL);
    }
  }
}

// Apertures of faces touching a solid closed; baffle slope dropped on domain-top faces,
// on closed faces and around fixed cells (src/air_cfd.js:132-136).
__global__ void k_cleanup(int NX, int NY, int NZ, const uint8_t* t, float* ap0, float* ap1, float* ap2, float* ap3) {
  const long NXY = (long)NX * NY, N = NXY * NZ;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < N; q += (long)gridDim.x * blockDim.x) {
    const int i = (int)(q % NX), j = (int)((q / NX) % NY), k = (int)(q / NXY);
    const bool tq = t[q] == T_SOLID;
    if (i + 1 < NX && (tq || t[q + 1] == T_SOLID)) ap0[q] = 0.f;
    if (j + 1 < NY && (tq || t[q + NX] == T_SOLID)) ap1[q] = 0.f;
    if (k + 1 >= NZ) ap3[q] = 0.f;
    else if (tq || t[q + NXY] == T_SOLID) { ap2[q] = 0.f; ap3[q] = 0.f; }
    if (t[q] >= T_SINK || (k + 1 < NZ && t[q + NXY] >= T_SINK)) ap3[q] = 0.f;
  }
}

// Jet cells open their +x face toward fluid; intake cells open the -x neighbour's +x face
// (src/air_cfd.js:138).  The flat index q +- 1 is used as the reference does.
__global__ void k_force_open(long N, const uint8_t* t, const uint8_t* mark, float* ap0) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < N; q += (long)gridDim.x * blockDim.x) {
    const uint8_t m = mark[q];
    if (!m) continue;
    if ((m & 1) && q + 1 < N && t[q + 1] == T_FLUID) ap0[q] = 1.f;
    if ((m & 2) && q >= 1 && t[q - 1] == T_FLUID) ap0[q - 1] = 1.f;
  }
}

__global__ void k_counts(long N, const uint8_t* t, const float* phi, const float* ap0, const float* ap1,
                         const float* ap2, unsigned long long* out) {  // src/air_cfd.js:139
  unsigned long long ns = 0, nc = 0;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < N; q += (long)gridDim.x * blockDim.x) {
    if (t[q] == T_SOLID) ns++;
    else if (t[q] == T_FLUID && (phi[q] < 1.f || ap0[q] < 1.f || ap1[q] < 1.f || ap2[q] < 1.f)) nc++;
  }
  for (int o = 16; o; o >>= 1) { ns += __shfl_down_sync(0xffffffffu, ns, o); nc += __shfl_down_sync(0xffffffffu, nc, o); }
  if ((threadIdx.x & 31) == 0) { atomicAdd(out, ns); atomicAdd(out + 1, nc); }
}

int grid_blocks(long work, int threads = 256) {
  long b = (work + threads - 1) / threads;
  return (int)std::max(1L, std::min(b, 148L * 32));
}

}  // namespace

int geom_build_device(const a3d_shape& shape, const GridDev& gd, double h, double delta_deg, const GeomDev& out,
                      cudaStream_t st, int64_t counts[2], int32_t vol[3]) {
  const int NX = gd.NX, NY = gd.NY, NZ = gd.NZ;
  const long N = (long)NX * NY * NZ;
  a3d_shape* d_shape = nullptr;
  uint8_t *cin = nullptr, *mark = nullptr;
  unsigned long long* d_cnt = nullptr;
  const long nodes = (long)(NX + 1) * (NY + 1) * (NZ + 1);
  int rc = A3D_OK;
  auto fail = [&](cudaError_t e, const char* what) {
    set_error("%s: %s", what, cudaGetErrorString(e));
    rc = e == cudaErrorMemoryAllocation ? A3D_ERR_NOMEM : A3D_ERR_CUDA;
  };
  cudaError_t e;
  if ((e = cudaMallocAsync(&d_shape, sizeof(a3d_shape), st)) != cudaSuccess) { fail(e, "cudaMallocAsync(shape)"); return rc; }
  if ((e = cudaMallocAsync(&cin, nodes, st)) != cudaSuccess) fail(e, "cudaMallocAsync(node flags)");
  if (rc == A3D_OK && (e = cudaMallocAsync(&mark, N, st)) != cudaSuccess) fail(e, "cudaMallocAsync(marks)");
  if (rc == A3D_OK && (e = cudaMallocAsync(&d_cnt, 2 * sizeof(unsigned long long), st)) != cudaSuccess) fail(e, "cudaMallocAsync(counts)");
  if (rc == A3D_OK) {
    GeoDev g;
    g.a = d_shape;
    g.Xf = gd.Xf; g.Yf = gd.Yf; g.Zf = gd.Zf; g.Xd = gd.Xd; g.Yd = gd.Yd; g.Zd = gd.Zd; g.Yc = gd.Yc; g.Zc = gd.Zc;
    g.NX = NX; g.NY = NY; g.NZ = NZ;
    const a3d_surface& ht = shape.htail;
    const double dR = delta_deg * kDeg;
    g.hp0 = ht.x0 + 0 * ht.tanL + 0.25 * ht.cr;  // htail.xLE(0) + 0.25 * cr
    g.hp1 = ht.z0;
    g.cR = std::cos(dR); g.sR = std::sin(dR); g.tdR = std::tan(dR);
    auto thick = [&](const a3d_surface& S) { return 0.5 * (S.tcR * S.cr + S.tcT * S.ct) >= 1.5 * h; };
    g.volW = thick(shape.wing); g.volH = thick(ht); g.volV = thick(shape.vtail);
    if (vol) { vol[0] = g.volW; vol[1] = g.volH; vol[2] = g.volV; }
    cudaMemcpyAsync(d_shape, &shape, sizeof(a3d_shape), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(mark, 0, N, st);
    k_nodes<<<grid_blocks(nodes), 256, 0, st>>>(g, cin);
    k_cells<<<grid_blocks(N), 256, 0, st>>>(g, cin, out.phi, out.ap0, out.ap1, out.ap2, out.ap3);
    k_baffle<<<grid_blocks((long)NX * NY), 256, 0, st>>>(g, 0, out.ap2, out.ap3);
    k_baffle<<<grid_blocks((long)NX * NY), 256, 0, st>>>(g, 1, out.ap2, out.ap3);
    k_solid<<<grid_blocks(N), 256, 0, st>>>(N, out.phi, out.t);
    // fixed-state layers, in the reference's engine/exit order; a layer that catches no cell
    // centre is marked again with a padded ring (src/air_cfd.js:124, 129)
    auto layer_at = [&](double xv) { int i = 0; while (i < NX - 1 && gd.hXf[i + 1] <= xv) i++; return i; };
    auto mark_ring = [&](int i, const a3d_engine& E, double rin, double rout, int ty, uint8_t bit, unsigned long long& n) {
      cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long), st);
      k_mark<<<grid_blocks((long)NY * NZ), 256, 0, st>>>(g, i, E.y, E.z, rin, rout, ty, bit, out.t, out.phi, mark, d_cnt);
      cudaMemcpyAsync(&n, d_cnt, sizeof(n), cudaMemcpyDeviceToHost, st);
      return cudaStreamSynchronize(st);
    };
    for (int en = 0; en < shape.n_engines && rc == A3D_OK; en++) {
      const a3d_engine& E = shape.engines[en];
      for (int x = 0; x < shape.n_exits && rc == A3D_OK; x++) {
        const a3d_exit& ex = shape.exits[x];
        const int i = layer_at(E.x0 + ex.x - 1e-3);
        unsigned long long n = 0;
        if ((e = mark_ring(i, E, ex.Rin, ex.R, ex.type, 1, n)) != cudaSuccess) { fail(e, "exit layer"); break; }
        if (!n) {
          const double pad = 0.55 * std::max(std::max((double)gd.hYd0, (double)gd.hZd0), h);
          if ((e = mark_ring(i, E, ex.Rin - pad, ex.R + pad, ex.type, 1, n)) != cudaSuccess) fail(e, "exit layer");
        }
      }
      if (!E.internal && rc == A3D_OK) {
        const int i = layer_at(E.x0 + shape.lip_x + 1e-3);
        unsigned long long n = 0;
        // ring test r <= 0.9 lip_r + pad with no inner bound
        if ((e = mark_ring(i, E, -1e300, 0.9 * shape.lip_r, T_SINK, 2, n)) != cudaSuccess) { fail(e, "intake layer"); break; }
        if (!n && (e = mark_ring(i, E, -1e300, 0.9 * shape.lip_r + 0.55 * h, T_SINK, 2, n)) != cudaSuccess) fail(e, "intake layer");
      }
    }
    if (rc == A3D_OK) {
      k_cleanup<<<grid_blocks(N), 256, 0, st>>>(NX, NY, NZ, out.t, out.ap0, out.ap1, out.ap2, out.ap3);
      k_force_open<<<grid_blocks(N), 256, 0, st>>>(N, out.t, mark, out.ap0);
      cudaMemsetAsync(d_cnt, 0, 2 * sizeof(unsigned long long), st);
      k_counts<<<grid_blocks(N), 256, 0, st>>>(N, out.t, out.phi, out.ap0, out.ap1, out.ap2, d_cnt);
      unsigned long long hc[2] = {0, 0};
      cudaMemcpyAsync(hc, d_cnt, sizeof(hc), cudaMemcpyDeviceToHost, st);
      if ((e = cudaStreamSynchronize(st)) != cudaSuccess) fail(e, "geometry kernels");
      else if ((e = cudaGetLastError()) != cudaSuccess) fail(e, "geometry launch");
      if (counts) { counts[0] = (int64_t)hc[0]; counts[1] = (int64_t)hc[1]; }
    }
  }
  cudaFreeAsync(d_cnt, st);
  cudaFreeAsync(mark, st);
  cudaFreeAsync(cin, st);
  cudaFreeAsync(d_shape, st);
  cudaStreamSynchronize(st);
  return rc;
}

}  // namespace a3d

extern "C" int a3d_geom_build(const a3d_shape* shape, const int32_t dims[3], const double* xf, const double* yf,
                              const double* zf, double h, double delta_deg, uint8_t* t, float* phi, float* ap0,
                              float* ap1, float* ap2, float* ap3, int64_t counts[2], int32_t vol[3]) {
  using namespace a3d;
  clear_error();
  A3D_ARG(shape && dims && xf && yf && zf, "null pointer");
  A3D_ARG(dims[0] >= 1 && dims[1] >= 2 && dims[2] >= 1, "grid dims (NY >= 2 for the symmetry mirror)");
  A3D_TRY(use_device(-1));
  GridDev gd;
  A3D_TRY(grid_upload(dims, xf, yf, zf, nullptr, gd));
  const long N = (long)dims[0] * dims[1] * dims[2];
  GeomDev g{};
  int rc = A3D_OK;
  cudaStream_t st = nullptr;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) { grid_free(gd); set_error("cudaStreamCreate failed"); return A3D_ERR_CUDA; }
  rc = geom_alloc(N, g);
  if (rc == A3D_OK) rc = geom_build_device(*shape, gd, h, delta_deg, g, st, counts, vol);
  if (rc == A3D_OK) {
    cudaError_t e = cudaSuccess;
    if (t && e == cudaSuccess) e = cudaMemcpy(t, g.t, N, cudaMemcpyDeviceToHost);
    if (phi && e == cudaSuccess) e = cudaMemcpy(phi, g.phi, N * 4, cudaMemcpyDeviceToHost);
    if (ap0 && e == cudaSuccess) e = cudaMemcpy(ap0, g.ap0, N * 4, cudaMemcpyDeviceToHost);
    if (ap1 && e == cudaSuccess) e = cudaMemcpy(ap1, g.ap1, N * 4, cudaMemcpyDeviceToHost);
    if (ap2 && e == cudaSuccess) e = cudaMemcpy(ap2, g.ap2, N * 4, cudaMemcpyDeviceToHost);
    if (ap3 && e == cudaSuccess) e = cudaMemcpy(ap3, g.ap3, N * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { set_error("geometry copy-out: %s", cudaGetErrorString(e)); rc = A3D_ERR_CUDA; }
  }
  geom_free(g);
  grid_free(gd);
  cudaStreamDestroy(st);
  return rc;
}
