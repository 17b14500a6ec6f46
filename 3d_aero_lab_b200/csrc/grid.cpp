// grid.cpp - stretched Cartesian half-domain grid (cfdAxis / cfdGrid, src/air_cfd.js:14-44).
//
// Host code: the grid is a few hundred face coordinates per axis.  The core box around
// the aircraft is uniform with spacing h; outside it the faces grow geometrically by
// r = 1.14 out to the far-field limits, and h is iterated (at most six times) until the
// cell count is within 4 % of the target.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <vector>
#include "common.cuh"

namespace a3d {

namespace {

double js_round(double x) {  // JavaScript Math.round (halves go up)
  double r = std::floor(x);
  return (x - r >= 0.5) ? r + 1 : r;
}

double naca_camber(double m, double x) {  // src/aircraft.js:59, p = 0.4
  const double p = 0.4;
  if (m == 0) return 0;
  return x < p ? m / (p * p) * (2 * p * x - x * x) : m / std::pow(1 - p, 2) * ((1 - 2 * p) + 2 * p * x - x * x);
}

double chord(const a3d_surface& S, double s) { return S.cr + (S.ct - S.cr) * s / S.semi; }
double x_le(const a3d_surface& S, double s) { return S.x0 + s * S.tanL; }

// One axis: uniform faces on [c0, c1] (spacing close to h) then geometric growth toward
// lo and hi; the outermost stretched cell is merged into its neighbour when it would be
// less than half the neighbour's size.
std::vector<double> axis_faces(double c0, double c1, double h, double lo, double hi, double r) {
  const int n = (int)std::max(1.0, js_round((c1 - c0) / h));
  const double hh = (c1 - c0) / n;
  std::vector<double> left, right, core;
  core.reserve(n + 1);
  for (int i = 0; i <= n; i++) core.push_back(c0 + i * hh);
  if (lo < c0 - 1e-9) {
    double d = hh, x = c0;
    while (x > lo + 1e-9) { d *= r; x -= d; left.push_back(x); }
    left.back() = lo;
    const size_t m = left.size();
    if (m > 1 && (left[m - 2] - lo) < 0.5 * (m > 2 ? left[m - 3] - left[m - 2] : hh)) left.erase(left.begin() + (m - 2));
  }
  if (hi > c1 + 1e-9) {
    double d = hh, x = c1;
    while (x < hi - 1e-9) { d *= r; x += d; right.push_back(x); }
    right.back() = hi;
    const size_t m = right.size();
    if (m > 1 && (hi - right[m - 2]) < 0.5 * (m > 2 ? right[m - 2] - right[m - 3] : hh)) right.erase(right.begin() + (m - 2));
  }
  std::vector<double> f(left.rbegin(), left.rend());
  f.insert(f.end(), core.begin(), core.end());
  f.insert(f.end(), right.begin(), right.end());
  return f;
}

}  // namespace
}  // namespace a3d

extern "C" int a3d_grid_build(const a3d_shape* shape, double target_cells, int32_t cap, double* xf, double* yf,
                              double* zf, int32_t dims[3], double* h_out, double core_out[5]) {
  using namespace a3d;
  clear_error();
  A3D_ARG(shape && xf && yf && zf && dims && h_out && core_out, "null pointer");
  A3D_ARG(target_cells >= 8 && target_cells < 4e9, "target_cells out of range");
  const a3d_shape& a = *shape;
  A3D_ARG(a.n_engines >= 0 && a.n_engines <= A3D_MAX_ENGINES && a.n_exits >= 0 && a.n_exits <= A3D_MAX_EXITS,
          "engine/exit count");
  const a3d_surface &w = a.wing, &ht = a.htail, &vt = a.vtail;
  // core box around the aircraft (src/air_cfd.js:22-26)
  const double L = a.fus_L, Lc = std::max(L, a.ref_b);
  double x0 = -0.02 * L;
  double x1 = std::max(std::max(L, x_le(ht, ht.semi) + ht.ct), x_le(vt, vt.semi) + vt.ct) + 0.03 * L;
  double y1 = std::max(w.semi, ht.semi) + 0.03 * Lc, z0 = -a.fus_R0 - 0.03 * L, z1 = vt.z0 + vt.semi + 0.02 * L;
  for (int e = 0; e < a.n_engines; e++) {
    const a3d_engine& E = a.engines[e];
    x0 = std::min(x0, E.x0 - 0.02 * L);
    if (a.n_exits > 0) x1 = std::max(x1, E.x0 + a.exits[a.n_exits - 1].x + 0.05 * L);
    if (!E.internal) {
      y1 = std::max(y1, E.y + a.view_Rmax + 0.03 * Lc);
      z0 = std::min(z0, E.z - a.view_Rmax - 0.03 * L);
    }
  }
  {  // wing tip mid-chord height, surface point (semi, 0.5, side 0) of src/aircraft.js:90-97
    const double s = w.semi, c = chord(w, s);
    const double cam = naca_camber(w.camber, 0.5) * c, shear = -(0.5 - 0.25) * c * w.tanI_pt;
    const double zt = w.z0 + (s - 0) * w.tanD_pt + cam + shear;
    z0 = std::min(std::min(z0, zt - 0.05 * L), ht.z0 - 0.05 * L);
  }
  // far-field limits (src/air_cfd.js:27)
  const double lx0 = x0 - 0.55 * Lc, lx1 = x1 + 0.9 * Lc, ly1 = y1 + 0.6 * Lc, lz0 = z0 - 0.6 * Lc, lz1 = z1 + 0.6 * Lc;
  const double r = 1.14;
  double h = std::cbrt((x1 - x0) * y1 * (z1 - z0) / (target_cells * 0.6));
  std::vector<double> ax, ay, az;
  for (int it = 0; it < 6; it++) {  // src/air_cfd.js:30-34
    ax = axis_faces(x0, x1, h, lx0, lx1, r);
    ay = axis_faces(0, y1, h, 0, ly1, r);
    az = axis_faces(z0, z1, h, lz0, lz1, r);
    const double n = (double)(ax.size() - 1) * (double)(ay.size() - 1) * (double)(az.size() - 1);
    h *= std::cbrt(n / target_cells);
    if (std::fabs(n / target_cells - 1) < 0.04) break;
  }
  ax = axis_faces(x0, x1, h, lx0, lx1, r);  // the final axes use the last update of h (src/air_cfd.js:35)
  ay = axis_faces(0, y1, h, 0, ly1, r);
  az = axis_faces(z0, z1, h, lz0, lz1, r);
  if ((int64_t)ax.size() > cap || (int64_t)ay.size() > cap || (int64_t)az.size() > cap) {
    set_error("grid needs %zu/%zu/%zu faces, capacity %d", ax.size(), ay.size(), az.size(), cap);
    return A3D_ERR_ARG;
  }
  std::copy(ax.begin(), ax.end(), xf);
  std::copy(ay.begin(), ay.end(), yf);
  std::copy(az.begin(), az.end(), zf);
  dims[0] = (int32_t)ax.size() - 1;
  dims[1] = (int32_t)ay.size() - 1;
  dims[2] = (int32_t)az.size() - 1;
  *h_out = h;
  core_out[0] = x0; core_out[1] = x1; core_out[2] = y1; core_out[3] = z0; core_out[4] = z1;
  return A3D_OK;
}
