// stage_march.cu - the z-marching RK-stage kernel (KERNEL_MARCH).
//
// A CTA owns a tile of 32 (x) by 8 (y) cell columns and walks a run of z planes.  Per plane:
//   1. every thread shifts its column's 4-plane register window (k-1 .. k+2) and loads
//      plane k+2 (coalesced rows of 32 cells per component);
//   2. plane k's primitives and codes go to shared memory with a 2-cell halo in x and y
//      (halo cells are loaded by the first 160 threads, with the reference's ghost rules);
//   3. every face is evaluated exactly once per tile: the x face i-1/2 and y face j-1/2 of
//      each column from shared memory, the z face k+1/2 from the register window, plus the
//      40 faces on the tile's +x/+y edges.  Fluxes are stored premultiplied by the face
//      aperture, so a closed face costs nothing;
//   4. each cell sums its six faces, adds the wall-pressure and baffle terms, divides by phi,
//      takes its local dt and applies the RK update with the positivity clamps.
// The reference evaluates each face twice (once from each side); the fluxes are the same
// numbers because the face state depends only on the four cells around the face.
#include "flux.cuh"
#include "solver.cuh"

namespace a3d {

namespace {

constexpr int TX = 32, TY = 8, HX = TX + 4, HY = TY + 4;

struct MarchSmem {
  float P[5][HY][HX];     // plane k primitives (rho, u, v, w, p) with a 2-cell halo
  uint8_t C[HY][HX];      // plane k codes
  float Fx[5][TY][TX + 1];  // a * flux of x face i-1/2 (index i - i0), unrotated components
  float Fy[5][TY + 1][TX];  // a * flux of y face j-1/2 (index j - j0)
  float Ax[TY][TX + 1];     // x face apertures
  float Ay[TY + 1][TX];     // y face apertures
};

// Primitive state and code of cell (i, j, k) with ghost handling (src/air_cfd.js:205-210).
__device__ __forceinline__ uint8_t load_cell(const StageArgs& a, int i, int j, int k, float P[5]) {
  if (i < 0 || i >= a.NX || k < 0 || k >= a.NZ || j >= a.NY) {
#pragma unroll
    for (int v = 0; v < 5; v++) P[v] = a.Pff[v];
    return T_GHOST;
  }
  const bool mirror = j < 0;
  const int jj = mirror ? -1 - j : j;
  const long q = ((long)k * a.NY + jj) * a.NXp + i;
  const uint8_t c = a.code[q];
  const int t = c & 7;
  if (t >= T_SINK) {
#pragma unroll
    for (int v = 0; v < 5; v++) P[v] = a.Pfix[t - T_SINK][v];
  } else {
    cons_to_prim(__ldg(a.Qin + q), __ldg(a.Qin + a.Np + q), __ldg(a.Qin + 2 * a.Np + q), __ldg(a.Qin + 3 * a.Np + q),
                 __ldg(a.Qin + 4 * a.Np + q), P);
  }
  if (mirror) { P[2] = -P[2]; return T_MIRROR; }
  return c;
}

__device__ __forceinline__ Prim sprim(const MarchSmem& S, int y, int x, int d) {
  float P[5] = {S.P[0][y][x], S.P[1][y][x], S.P[2][y][x], S.P[3][y][x], S.P[4][y][x]};
  return rot(P, d);
}

// x face between smem columns x-1 and x (cells i-1 and i) in smem row y; returns a * flux.
__device__ __forceinline__ float face_x(const StageArgs& a, const MarchSmem& S, int y, int x, int i, int j, int k,
                                        float G[5]) {
  const uint8_t cl = S.C[y][x - 1], cr = S.C[y][x];
  float A = 1.f;
  if (i - 1 >= 0 && (cl & C_IRR)) A = a.ap0[((long)k * a.NY + j) * a.NX + (i - 1)];
  if (A > 0.f) {
    float F[5];
    face_flux(sprim(S, y, x - 2, 0), sprim(S, y, x - 1, 0), sprim(S, y, x, 0), sprim(S, y, x + 1, 0),
              a.order2 && (cl & C_OKX), a.order2 && (cr & C_OKX), F);
    G[0] = A * F[0]; G[1] = A * F[1]; G[2] = A * F[2]; G[3] = A * F[3]; G[4] = A * F[4];
  } else {
    G[0] = G[1] = G[2] = G[3] = G[4] = 0.f;
  }
  return A;
}

// y face between smem rows y-1 and y (cells j-1 and j) in smem column x.
__device__ __forceinline__ float face_y(const StageArgs& a, const MarchSmem& S, int y, int x, int i, int j, int k,
                                        float G[5]) {
  const uint8_t cl = S.C[y - 1][x], cr = S.C[y][x];
  float A = 1.f;
  if (j - 1 >= 0 && (cl & C_IRR)) A = a.ap1[((long)k * a.NY + (j - 1)) * a.NX + i];
  if (A > 0.f) {
    float F[5];
    face_flux(sprim(S, y - 2, x, 1), sprim(S, y - 1, x, 1), sprim(S, y, x, 1), sprim(S, y + 1, x, 1),
              a.order2 && (cl & C_OKY), a.order2 && (cr & C_OKY), F);
    G[0] = A * F[0]; G[1] = A * F[2]; G[2] = A * F[1]; G[3] = A * F[3]; G[4] = A * F[4];
  } else {
    G[0] = G[1] = G[2] = G[3] = G[4] = 0.f;
  }
  return A;
}

// z face between register planes b (k) and c (k+1) of the column.
__device__ __forceinline__ float face_z(const StageArgs& a, const float Pa[5], const float Pb[5], const float Pc[5],
                                        const float Pe[5], uint8_t cb, uint8_t cc, bool in_dom_b, long qb, float G[5]) {
  float A = 1.f;
  if (in_dom_b && (cb & C_IRR)) A = a.ap2[qb];
  if (A > 0.f) {
    float F[5];
    face_flux(rot(Pa, 2), rot(Pb, 2), rot(Pc, 2), rot(Pe, 2), a.order2 && (cb & C_OKZ), a.order2 && (cc & C_OKZ), F);
    G[0] = A * F[0]; G[1] = A * F[2]; G[2] = A * F[3]; G[3] = A * F[1]; G[4] = A * F[4];
  } else {
    G[0] = G[1] = G[2] = G[3] = G[4] = 0.f;
  }
  return A;
}

__global__ void __launch_bounds__(TX * TY, 2) k_stage_march(StageArgs a, int kz) {
  __shared__ MarchSmem S;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int i = i0 + tx, j = j0 + ty;
  const int k0 = blockIdx.z * kz, k1 = min(a.NZ, k0 + kz);
  const bool in_dom = i < a.NX && j < a.NY;
  const long NXY = (long)a.NX * a.NY, Np = a.Np;
  const float rx = in_dom ? a.rXd[i] : 0.f, ry = in_dom ? a.rYd[j] : 0.f;

  // register window of this column: planes k-1, k, k+1, k+2
  float Wm[5], W0[5], W1[5], W2[5];
  uint8_t cm, c0, c1, c2;
  float Gz[5], Az;  // flux of z face k-1/2
  {
    float Wa[5];
    const uint8_t ca = load_cell(a, i, j, k0 - 2, Wa);
    cm = load_cell(a, i, j, k0 - 1, Wm);
    c0 = load_cell(a, i, j, k0, W0);
    c1 = load_cell(a, i, j, k0 + 1, W1);
    (void)ca;
    Az = 1.f;
#pragma unroll
    for (int c = 0; c < 5; c++) Gz[c] = 0.f;
    if (in_dom) Az = face_z(a, Wa, Wm, W0, W1, cm, c0, k0 - 1 >= 0, ((long)(k0 - 1) * a.NY + j) * a.NX + i, Gz);
  }

  for (int k = k0; k < k1; k++) {
    c2 = load_cell(a, i, j, k + 2, W2);
    // ---- plane k to shared memory (interior + halo) ----
#pragma unroll
    for (int v = 0; v < 5; v++) S.P[v][ty + 2][tx + 2] = W0[v];
    S.C[ty + 2][tx + 2] = c0;
    if (threadIdx.x < 160) {
      int hx, hy;
      const int h = threadIdx.x;
      if (h < 32) { hy = 2 + (h >> 2); const int c = h & 3; hx = c < 2 ? c : TX + c; }
      else { const int g = h - 32; const int r = g >> 5; hy = r < 2 ? r : TY + r; hx = 2 + (g & 31); }
      float P[5];
      const uint8_t c = load_cell(a, i0 + hx - 2, j0 + hy - 2, k, P);
#pragma unroll
      for (int v = 0; v < 5; v++) S.P[v][hy][hx] = P[v];
      S.C[hy][hx] = c;
    }
    __syncthreads();
    // ---- face fluxes ----
    if (j < a.NY && i <= a.NX) {
      float G[5];
      const float A = face_x(a, S, ty + 2, tx + 2, i, j, k, G);
#pragma unroll
      for (int v = 0; v < 5; v++) S.Fx[v][ty][tx] = G[v];
      S.Ax[ty][tx] = A;
    }
    if (i < a.NX && j <= a.NY) {
      float G[5];
      const float A = face_y(a, S, ty + 2, tx + 2, i, j, k, G);
#pragma unroll
      for (int v = 0; v < 5; v++) S.Fy[v][ty][tx] = G[v];
      S.Ay[ty][tx] = A;
    }
    if (ty == TY - 1) {  // +y edge faces of the tile (face j0+8-1/2)
      const int jj = j0 + TY;
      if (i < a.NX && jj - 1 < a.NY) {
        float G[5];
        const float A = face_y(a, S, TY + 2, tx + 2, i, jj, k, G);
#pragma unroll
        for (int v = 0; v < 5; v++) S.Fy[v][TY][tx] = G[v];
        S.Ay[TY][tx] = A;
      }
    } else if (ty == TY - 2 && tx < TY) {  // +x edge faces (face i0+32-1/2), one per row
      const int row = tx, ii = i0 + TX, jr = j0 + row;
      if (jr < a.NY && ii - 1 < a.NX) {
        float G[5];
        const float A = face_x(a, S, row + 2, TX + 2, ii, jr, k, G);
#pragma unroll
        for (int v = 0; v < 5; v++) S.Fx[v][row][TX] = G[v];
        S.Ax[row][TX] = A;
      }
    }
    float Gn[5], An = 1.f;
    if (in_dom) An = face_z(a, Wm, W0, W1, W2, c0, c1, true, ((long)k * a.NY + j) * a.NX + i, Gn);
    __syncthreads();
    // ---- residual and RK update ----
    if (in_dom) {
      const long q = ((long)k * a.NY + j) * a.NX + i;    // reference (geometry) index
      const long qp = ((long)k * a.NY + j) * a.NXp + i;  // padded state index
      const int t = c0 & 7;
      float o[5];
      if (t != T_FLUID) {
        if (t >= T_SINK) {
#pragma unroll
          for (int c = 0; c < 5; c++) o[c] = a.Ufix[t - T_SINK][c];
        } else {
#pragma unroll
          for (int c = 0; c < 5; c++) o[c] = __ldg(a.B + c * Np + qp);
        }
      } else {
        const float rz = a.rZd[k];
        const float pC = W0[4];
        float R[5];
#pragma unroll
        for (int c = 0; c < 5; c++)
          R[c] = (S.Fx[c][ty][tx] - S.Fx[c][ty][tx + 1]) * rx + (S.Fy[c][ty][tx] - S.Fy[c][ty + 1][tx]) * ry +
                 (Gz[c] - Gn[c]) * rz;
        R[1] += pC * (S.Ax[ty][tx + 1] - S.Ax[ty][tx]) * rx;  // wall-pressure source
        R[2] += pC * (S.Ay[ty + 1][tx] - S.Ay[ty][tx]) * ry;
        R[3] += pC * (An - Az) * rz;
        if (c0 & C_BAF) {  // baffle transpiration w = u dz/dx (src/air_cfd.js:226-233)
          const float sUp = a.ap3[q], sDn = k > 0 ? a.ap3[q - NXY] : 0.f;
          if (sUp != 0.f || sDn != 0.f) {
            const float r = W0[0], u = W0[1], v = W0[2], w = W0[3];
            const float Hh = (pC / kGm + 0.5f * r * (u * u + v * v + w * w) + pC) / r;
            const float m = (sDn != 0.f ? (1.f - Az) * r * u * sDn : 0.f) - (sUp != 0.f ? (1.f - An) * r * u * sUp : 0.f);
            const float mh = m * rz;
            R[0] += mh; R[1] += mh * u; R[2] += mh * v; R[3] += mh * w; R[4] += mh * Hh;
          }
        }
        const float ph = (c0 & C_IRR) ? a.phi[q] : 1.f;
        if (ph != 1.f) {
          const float iph = 1.f / ph;
#pragma unroll
          for (int c = 0; c < 5; c++) R[c] *= iph;
        }
        float qin[5];
#pragma unroll
        for (int c = 0; c < 5; c++) qin[c] = __ldg(a.Qin + c * Np + qp);
        float Pb[5], bq[5];
        if (a.wa == 0.f) {
#pragma unroll
          for (int c = 0; c < 5; c++) { Pb[c] = W0[c]; bq[c] = 0.f; }
        } else {
#pragma unroll
          for (int c = 0; c < 5; c++) bq[c] = __ldg(a.B + c * Np + qp);
          cons_to_prim(bq[0], bq[1], bq[2], bq[3], bq[4], Pb);
        }
        const float as = sqrtf(kG * Pb[4] / Pb[0]);
        const float dt = a.cfl * fmaxf(ph, 0.25f) /
                         ((fabsf(Pb[1]) + as) * rx + (fabsf(Pb[2]) + as) * ry + (fabsf(Pb[3]) + as) * rz);
#pragma unroll
        for (int c = 0; c < 5; c++) o[c] = (a.wa == 0.f) ? (qin[c] + dt * R[c]) : (a.wa * bq[c] + a.wb * (qin[c] + dt * R[c]));
        o[0] = fmaxf(o[0], 1e-4f);  // positivity clamps (src/air_cfd.js:247-249)
        const float ke = 0.5f * (o[1] * o[1] + o[2] * o[2] + o[3] * o[3]) / o[0];
        if (kGm * (o[4] - ke) < 1e-5f) o[4] = 1e-5f / kGm + ke;
      }
#pragma unroll
      for (int c = 0; c < 5; c++) a.Out[c * Np + qp] = o[c];
    }
    // ---- shift the window ----
#pragma unroll
    for (int c = 0; c < 5; c++) { Gz[c] = Gn[c]; Wm[c] = W0[c]; W0[c] = W1[c]; W1[c] = W2[c]; }
    Az = An;
    cm = c0; c0 = c1; c1 = c2;
    (void)cm;
  }
}

}  // namespace

int launch_march(a3d_solver* s, const StageArgs& a) {
  const int kz = s->march_kz;
  dim3 grid((a.NX + TX - 1) / TX, (a.NY + TY - 1) / TY, (a.NZ + kz - 1) / kz);
  k_stage_march<<<grid, TX * TY, 0, s->st>>>(a, kz);
  A3D_CUDA(cudaGetLastError());
  return A3D_OK;
}

}  // namespace a3d
