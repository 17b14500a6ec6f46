// stage_fused.cuh - the RK-stage tile with per-cell face states (KERNEL_FUSED, stage kernel 3).
//
// Tiling and plane ring as stage_tma.cu (32 x 8 columns per CTA, z march, TMA ring of 4
// planes).  What changes is how a face is evaluated:
//   * every cell forms its MUSCL face states once per direction (lo = P - s/2, hi = P + s/2)
//     instead of once per face side; x neighbours trade states through warp shuffles, y
//     neighbours through shared memory, z neighbours through the register window;
//   * the x face i-1/2 and the z face k+1/2 of a column are evaluated together in packed f32x2
//     arithmetic (flux2.cuh); the y face j-1/2 alone with the same arithmetic;
//   * the first-order fallback for a non-positive reconstructed density or pressure
//     (src/air_cfd.js:221) is left out: it cannot fire for these floored states (flux.cuh).
// Per plane: [A] column primitives of plane k+2 and the plane-k tile to shared memory;
// [B] face states, x/z fluxes; [C] y fluxes and the tile-edge faces; [D] residual and update.
// Three CTA barriers separate A|B, B|C and C|D.
#pragma once
#include "flux2.cuh"
#include "solver.cuh"
#include "tma.cuh"
#include "tma_ring.cuh"

namespace a3d {
namespace fused {

using namespace ring;

struct FusedSmem {
  Slot slot[NSLOT];
  float P[5][HY][HX];        // plane-k primitives with a 2-cell halo
  uint8_t C[HY][HX];         // plane-k codes (ghosts marked)
  float YH[5][TY + 1][TX];   // + y face state of cell row r-1 (row 0: halo row j0-1)
  float XE[2][5][TY];        // + x face state of column i0+31 and - x face state of column i0+32
  float FY[5][TY + 1][TX];   // a * y flux of face j-1/2 (row TY: the tile's + y edge face)
  float AY[TY + 1][TX];
  float FXE[5][TY];          // a * x flux of the tile's + x edge face, per row
  float AXE[TY];
  uint64_t bar[NSLOT];
  int abort;
};

__device__ __forceinline__ void load_p(const FusedSmem& S, int y, int x, float P[5]) {
#pragma unroll
  for (int v = 0; v < 5; v++) P[v] = S.P[v][y][x];
}

// Face states along x or y of the tile cell at shared-memory (y, x).
__device__ __forceinline__ void tile_states(const FusedSmem& S, int y, int x, int d, bool order2, float lo[5],
                                            float hi[5]) {
  float Pm[5], P[5], Pp[5];
  load_p(S, y, x, P);
  if (d == 0) { load_p(S, y, x - 1, Pm); load_p(S, y, x + 1, Pp); }
  else { load_p(S, y - 1, x, Pm); load_p(S, y + 1, x, Pp); }
  const uint8_t c = S.C[y][x];
  v::face_states(Pm, P, Pp, order2 && (c & (d == 0 ? C_OKX : C_OKY)), lo, hi);
}

// Single face along direction d: left + state L, right - state R, centres Pl, Pr for the
// first-order fallback; returns the flux premultiplied by the aperture A (0 if closed).
// x and z faces are evaluated in packed f32x2 form (lane x for x faces, lane y for z faces,
// as in the paired x/z evaluation of the plane loop), so that a face at a tile boundary
// gets exactly the numbers it would get inside a tile: results do not depend on the tiling.
__device__ __forceinline__ void single_face(float L[5], float R[5], const float Pl[5], const float Pr[5], int d,
                                            float A, float G[5]) {
  (void)Pl;  // the first-order fallback cannot fire (flux.cuh, face_flux_lr, says why)
  (void)Pr;
  float F[5], Fu[5];
  if (d == 1) {
    v::hllc(v::rotv(L, d), v::rotv(R, d), F);
  } else {
    const v::PrimV<float> l = v::rotv(L, d), r = v::rotv(R, d);
    float2 F2[5];
    v::hllc(v::pack(l, l), v::pack(r, r), F2);
#pragma unroll
    for (int c = 0; c < 5; c++) F[c] = d == 0 ? F2[c].x : F2[c].y;
  }
  v::unrotv(F, d, Fu);
#pragma unroll
  for (int c = 0; c < 5; c++) G[c] = A > 0.f ? A * Fu[c] : 0.f;
}

// One tile: columns [bx*32, +32) x [by*8, +8), planes [bz*kz, +kz) of the case described by
// `a`; tmQ maps the stage's input state, B and Out are the stage's base and output states.
// Used by the single-case kernel below and by the batched persistent kernel (batch.cu).
// Returns false if a bounded wait ran out (the error is flagged in *a.err).
template <bool STAGE2>
__device__ __forceinline__ bool stage_tile(FusedSmem& S, const CUtensorMap* tmQp, const CUtensorMap* tmCp,
                                           const StageArgs& a, const float* __restrict__ Bp,
                                           float* __restrict__ Outp, int bx, int by, int bz, int kz) {
  const CUtensorMap& tmQ = *tmQp;
  const CUtensorMap& tmC = *tmCp;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int i0 = bx * TX, j0 = by * TY;
  const int i = i0 + tx, j = j0 + ty;
  const int k0 = bz * kz, k1 = min(a.NZ, k0 + kz);
  const bool in_dom = i < a.NX && j < a.NY;
  const bool order2 = a.order2 != 0;
  const long NXY = (long)a.NX * a.NY, Np = a.Np;
  const float rx = in_dom ? a.rXd[i] : 0.f, ry = in_dom ? a.rYd[j] : 0.f;

  __syncthreads();  // a previous tile of this CTA is completely done with the shared memory
  if (threadIdx.x == 0) {
    for (int s = 0; s < NSLOT; s++) mbar_init(&S.bar[s], 1);
    S.abort = 0;
    fence_barrier_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    fence_proxy_async_smem();  // earlier tiles' generic reads of the slots before these copies
    for (int p = k0 - 2; p <= k0 + 1; p++) issue_plane(S, &tmQ, &tmC, a, p, k0, i0, j0);
  }

  // Column window: primitives of planes k, k+1 (W0, W1), the + z face state of plane k (Zh0)
  // and the flux of face k-1/2 (Gz, Az).
  bool ok = true;
  float W0[5], W1[5], Zh0[5], Gz[5], Az = 1.f;
  uint8_t c0, c1;
  {
    float Wa[5], Wm[5], lo[5], him[5], hi0[5];
    ok &= mbar_wait(&S.bar[slot_of(k0 - 2, k0)], parity_of(k0 - 2, k0));
    slot_cell(a, S.slot[slot_of(k0 - 2, k0)], i, j, k0 - 2, i0, j0, Wa);
    ok &= mbar_wait(&S.bar[slot_of(k0 - 1, k0)], parity_of(k0 - 1, k0));
    const uint8_t cm = slot_cell(a, S.slot[slot_of(k0 - 1, k0)], i, j, k0 - 1, i0, j0, Wm);
    ok &= mbar_wait(&S.bar[slot_of(k0, k0)], parity_of(k0, k0));
    c0 = slot_cell(a, S.slot[slot_of(k0, k0)], i, j, k0, i0, j0, W0);
    ok &= mbar_wait(&S.bar[slot_of(k0 + 1, k0)], parity_of(k0 + 1, k0));
    c1 = slot_cell(a, S.slot[slot_of(k0 + 1, k0)], i, j, k0 + 1, i0, j0, W1);
    v::face_states(Wa, Wm, W0, order2 && (cm & C_OKZ), lo, him);  // cell k0-1
    v::face_states(Wm, W0, W1, order2 && (c0 & C_OKZ), lo, hi0);  // cell k0
#pragma unroll
    for (int c = 0; c < 5; c++) Zh0[c] = hi0[c];
    // face k0-1/2 between cells k0-1 and k0
    Az = (k0 - 1 >= 0 && (cm & C_IRR) && in_dom) ? __ldg(a.ap2 + ((long)(k0 - 1) * a.NY + j) * a.NX + i) : 1.f;
    single_face(him, lo, Wm, W0, 2, Az, Gz);
  }
  if (!ok) S.abort = 1;
  __syncthreads();
  int last_issued = k0 + 1, first_pending = k0 - 2;
  if (S.abort) {
    drain(S, a, k0, first_pending, last_issued);
    return false;
  }
  if (threadIdx.x == 0) issue_plane(S, &tmQ, &tmC, a, k0 + 2, k0, i0, j0);
  last_issued = k0 + 2;

  for (int k = k0; k < k1; k++) {
    const long q = ((long)k * a.NY + j) * a.NX + i;
    const long qp = ((long)k * a.NY + j) * a.NXp + i;
    float bq[5];
    if (STAGE2 && in_dom) {
#pragma unroll
      for (int c = 0; c < 5; c++) bq[c] = __ldg(Bp + c * Np + qp);
    }
    // ---------------- [A] plane k+2 column, plane-k tile ----------------
    const int sk = slot_of(k, k0), sk2 = slot_of(k + 2, k0);
    ok = mbar_wait(&S.bar[sk2], parity_of(k + 2, k0));
    float W2[5];
    const uint8_t c2 = slot_cell(a, S.slot[sk2], i, j, k + 2, i0, j0, W2);
#pragma unroll
    for (int v = 0; v < 5; v++) S.P[v][ty + 2][tx + 2] = W0[v];
    S.C[ty + 2][tx + 2] = c0;
    if (threadIdx.x < 160) {
      int hx, hy;
      const int h = threadIdx.x;
      if (h < 32) { hy = 2 + (h >> 2); const int c = h & 3; hx = c < 2 ? c : TX + c; }
      else { const int g = h - 32; const int r = g >> 5; hy = r < 2 ? r : TY + r; hx = 2 + (g & 31); }
      float P[5];
      const uint8_t c = slot_cell(a, S.slot[sk], i0 + hx - 2, j0 + hy - 2, k, i0, j0, P);
#pragma unroll
      for (int v = 0; v < 5; v++) S.P[v][hy][hx] = P[v];
      S.C[hy][hx] = c;
    }
    if (!ok) S.abort = 1;
    __syncthreads();
    if (S.abort) { first_pending = k + 2; break; }
    if (k + 3 <= k1 + 1) {
      if (threadIdx.x == 0) {
        fence_proxy_async_smem();
        issue_plane(S, &tmQ, &tmC, a, k + 3, k0, i0, j0);
      }
      last_issued = k + 3;
    }
    // ---------------- [B] face states; x face i-1/2 and z face k+1/2 ----------------
    float xlo[5], xhi[5], ylo[5], yhi[5], z1lo[5], z1hi[5];
    tile_states(S, ty + 2, tx + 2, 0, order2, xlo, xhi);
    tile_states(S, ty + 2, tx + 2, 1, order2, ylo, yhi);
    v::face_states(W0, W1, W2, order2 && (c1 & C_OKZ), z1lo, z1hi);  // cell k+1
#pragma unroll
    for (int c = 0; c < 5; c++) S.YH[c][ty + 1][tx] = yhi[c];
    if (ty == 0) {  // + y state of the halo row below the tile
      float lo[5], hi[5];
      tile_states(S, 1, tx + 2, 1, order2, lo, hi);
#pragma unroll
      for (int c = 0; c < 5; c++) S.YH[c][0][tx] = hi[c];
    }
    // + x state of the left neighbour: from the next lane down, or the halo column for lane 0
    float xl[5];
#pragma unroll
    for (int c = 0; c < 5; c++) xl[c] = __shfl_up_sync(0xffffffffu, xhi[c], 1);
    if (tx == 0) {
      float lo[5];
      tile_states(S, ty + 2, 1, 0, order2, lo, xl);
    }
    if (tx == TX - 1) {  // states around the tile's + x edge face, for [C]
      float lo[5], hi[5];
      tile_states(S, ty + 2, TX + 2, 0, order2, lo, hi);
#pragma unroll
      for (int c = 0; c < 5; c++) { S.XE[0][c][ty] = xhi[c]; S.XE[1][c][ty] = lo[c]; }
    }
    // apertures: x face from the left cell's +x aperture, z face from this cell's +z aperture
    const uint8_t cl = S.C[ty + 2][tx + 1];
    const float Ax = (i - 1 >= 0 && (cl & C_IRR) && j < a.NY && i <= a.NX)
                         ? __ldg(a.ap0 + ((long)k * a.NY + j) * a.NX + (i - 1)) : 1.f;
    const float An = ((c0 & C_IRR) && in_dom) ? __ldg(a.ap2 + q) : 1.f;
    float Gx[5], Gn[5];
    {
      float xL[5], xR[5], zL[5], zR[5];
#pragma unroll
      for (int c = 0; c < 5; c++) { xL[c] = xl[c]; xR[c] = xlo[c]; zL[c] = Zh0[c]; zR[c] = z1lo[c]; }
      // (no first-order fallback: it cannot fire for these floored states, see flux.cuh)
      float2 F2[5];
      v::hllc(v::pack(v::rotv(xL, 0), v::rotv(zL, 2)), v::pack(v::rotv(xR, 0), v::rotv(zR, 2)), F2);
      float Fx[5] = {F2[0].x, F2[1].x, F2[2].x, F2[3].x, F2[4].x};
      float Fz[5] = {F2[0].y, F2[1].y, F2[2].y, F2[3].y, F2[4].y};
      float Ux[5], Uz[5];
      v::unrotv(Fx, 0, Ux);
      v::unrotv(Fz, 2, Uz);
#pragma unroll
      for (int c = 0; c < 5; c++) {
        Gx[c] = Ax > 0.f ? Ax * Ux[c] : 0.f;
        Gn[c] = An > 0.f ? An * Uz[c] : 0.f;
      }
    }
    __syncthreads();
    // ---------------- [C] y face j-1/2; tile-edge faces ----------------
    if (i < a.NX && j <= a.NY) {
      float L[5], R[5], Pl[5];
#pragma unroll
      for (int c = 0; c < 5; c++) { L[c] = S.YH[c][ty][tx]; R[c] = ylo[c]; }
      load_p(S, ty + 1, tx + 2, Pl);
      const uint8_t cb = S.C[ty + 1][tx + 2];
      const float A = (j - 1 >= 0 && (cb & C_IRR)) ? __ldg(a.ap1 + ((long)k * a.NY + (j - 1)) * a.NX + i) : 1.f;
      float G[5];
      single_face(L, R, Pl, W0, 1, A, G);
#pragma unroll
      for (int c = 0; c < 5; c++) S.FY[c][ty][tx] = G[c];
      S.AY[ty][tx] = A;
    }
    if (ty == TY - 1) {  // + y edge face j0+8-1/2, between this row and the halo row above
      const int jj = j0 + TY;
      if (i < a.NX && jj - 1 < a.NY) {
        float L[5], R[5], hi[5], Pr[5];
        tile_states(S, TY + 2, tx + 2, 1, order2, R, hi);
#pragma unroll
        for (int c = 0; c < 5; c++) L[c] = yhi[c];
        load_p(S, TY + 2, tx + 2, Pr);
        const float A = (c0 & C_IRR) ? __ldg(a.ap1 + q) : 1.f;
        float G[5];
        single_face(L, R, W0, Pr, 1, A, G);
#pragma unroll
        for (int c = 0; c < 5; c++) S.FY[c][TY][tx] = G[c];
        S.AY[TY][tx] = A;
      }
    } else if (ty == TY - 2 && tx < TY) {  // + x edge faces i0+32-1/2, one per row
      const int row = tx, jr = j0 + row, ii = i0 + TX;
      if (jr < a.NY && ii - 1 < a.NX) {
        float L[5], R[5], Pl[5], Pr[5];
#pragma unroll
        for (int c = 0; c < 5; c++) { L[c] = S.XE[0][c][row]; R[c] = S.XE[1][c][row]; }
        load_p(S, row + 2, TX + 1, Pl);
        load_p(S, row + 2, TX + 2, Pr);
        const uint8_t cb = S.C[row + 2][TX + 1];
        const float A = (cb & C_IRR) ? __ldg(a.ap0 + ((long)k * a.NY + jr) * a.NX + (ii - 1)) : 1.f;
        float G[5];
        single_face(L, R, Pl, Pr, 0, A, G);
#pragma unroll
        for (int c = 0; c < 5; c++) S.FXE[c][row] = G[c];
        S.AXE[row] = A;
      }
    }
    __syncthreads();
    // ---------------- [D] residual and RK update ----------------
    float Gxn[5];
#pragma unroll
    for (int c = 0; c < 5; c++) Gxn[c] = __shfl_down_sync(0xffffffffu, Gx[c], 1);
    float Axn = __shfl_down_sync(0xffffffffu, Ax, 1);
    if (tx == TX - 1) {
#pragma unroll
      for (int c = 0; c < 5; c++) Gxn[c] = S.FXE[c][ty];
      Axn = S.AXE[ty];
    }
    if (in_dom) {
      const int t = c0 & 7;
      float o[5];
      const Slot& sl = S.slot[sk];
      if (t != T_FLUID) {
        if (t >= T_SINK) {
#pragma unroll
          for (int c = 0; c < 5; c++) o[c] = a.Ufix[t - T_SINK][c];
        } else if (STAGE2) {
#pragma unroll
          for (int c = 0; c < 5; c++) o[c] = bq[c];
        } else {
#pragma unroll
          for (int c = 0; c < 5; c++) o[c] = sl.Q[c][ty + 2][tx + 4];
        }
      } else {
        const float rz = a.rZd[k];
        const float pC = W0[4];
        float R[5];
#pragma unroll
        for (int c = 0; c < 5; c++)
          R[c] = (Gx[c] - Gxn[c]) * rx + (S.FY[c][ty][tx] - S.FY[c][ty + 1][tx]) * ry + (Gz[c] - Gn[c]) * rz;
        R[1] += pC * (Axn - Ax) * rx;  // wall-pressure source
        R[2] += pC * (S.AY[ty + 1][tx] - S.AY[ty][tx]) * ry;
        R[3] += pC * (An - Az) * rz;
        if (c0 & C_BAF) {  // baffle transpiration w = u dz/dx (src/air_cfd.js:226-233)
          const float sUp = __ldg(a.ap3 + q), sDn = k > 0 ? __ldg(a.ap3 + q - NXY) : 0.f;
          if (sUp != 0.f || sDn != 0.f) {
            const float r = W0[0], u = W0[1], v = W0[2], w = W0[3];
            const float Hh = (pC / kGm + 0.5f * r * (u * u + v * v + w * w) + pC) / r;
            const float m = (sDn != 0.f ? (1.f - Az) * r * u * sDn : 0.f) - (sUp != 0.f ? (1.f - An) * r * u * sUp : 0.f);
            const float mh = m * rz;
            R[0] += mh; R[1] += mh * u; R[2] += mh * v; R[3] += mh * w; R[4] += mh * Hh;
          }
        }
        const float ph = (c0 & C_IRR) ? __ldg(a.phi + q) : 1.f;
        if (ph != 1.f) {
          const float iph = 1.f / ph;
#pragma unroll
          for (int c = 0; c < 5; c++) R[c] *= iph;
        }
        float Pb[5];
        if (STAGE2) cons_to_prim(bq[0], bq[1], bq[2], bq[3], bq[4], Pb);
        else {
#pragma unroll
          for (int c = 0; c < 5; c++) Pb[c] = W0[c];
        }
        const float as = sqrtf(kG * Pb[4] / Pb[0]);
        const float dt = a.cfl * fmaxf(ph, 0.25f) /
                         ((fabsf(Pb[1]) + as) * rx + (fabsf(Pb[2]) + as) * ry + (fabsf(Pb[3]) + as) * rz);
#pragma unroll
        for (int c = 0; c < 5; c++) {
          const float qin = sl.Q[c][ty + 2][tx + 4];
          o[c] = STAGE2 ? (a.wa * bq[c] + a.wb * (qin + dt * R[c])) : (qin + dt * R[c]);
        }
        o[0] = fmaxf(o[0], 1e-4f);  // positivity clamps (src/air_cfd.js:247-249)
        const float ke = 0.5f * (o[1] * o[1] + o[2] * o[2] + o[3] * o[3]) / o[0];
        if (kGm * (o[4] - ke) < 1e-5f) o[4] = 1e-5f / kGm + ke;
      }
#pragma unroll
      for (int c = 0; c < 5; c++) Outp[c * Np + qp] = o[c];
    }
    // ---------------- shift the column window ----------------
#pragma unroll
    for (int c = 0; c < 5; c++) { Gz[c] = Gn[c]; W0[c] = W1[c]; W1[c] = W2[c]; Zh0[c] = z1hi[c]; }
    Az = An;
    c0 = c1;
    c1 = c2;
  }
  if (S.abort) {
    drain(S, a, k0, first_pending, last_issued);
    return false;
  }
  // every issued plane has been waited for: retire the ring barriers so that a persistent CTA
  // can initialise them again for its next tile
  __syncthreads();
  if (threadIdx.x == 0)
    for (int s = 0; s < NSLOT; s++) mbar_inval(&S.bar[s]);
  return true;
}

}  // namespace fused
}  // namespace a3d
