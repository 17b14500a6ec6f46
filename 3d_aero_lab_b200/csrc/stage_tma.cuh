// stage_tma.cuh - the TMA-fed z-marching RK-stage tile (KERNEL_TMA, the default), shared by the
// single-case kernel (stage_tma.cu) and the persistent batch kernel (batch.cu).
//
// A CTA owns 32 x 8 cell columns and walks a run of z planes, evaluating every face once.
// The planes arrive through a 4-deep ring of shared-memory slots filled by
// `cp.async.bulk.tensor` (one 40 x 12 x 5-component state box and one 64 x 12 code box per
// plane, completing on the slot's mbarrier).  While the CTA computes plane k, planes k+1 .. k+3
// are already resident or in flight, so no global load latency sits on the critical path
// except the stage-2 base state, which is loaded at the top of the plane's iteration.
//
// A prologue loads planes k0-2 .. k0+1 and forms the z face k0-1/2.  Per plane k:
//   wait for plane k+2; column primitives of k+2 into the register window;
//   plane-k primitives (interior from registers, halo from the slot) to shared memory;
//   barrier; issue the TMA of plane k+3 into the slot plane k-1 has left;
//   x and y face fluxes from shared memory, z face k+1/2 from the register window;
//   barrier; residual, local dt, RK update, clamps, store.
#pragma once
#include <cudaTypedefs.h>
#include "flux.cuh"
#include "solver.cuh"
#include "store.cuh"
#include "tma.cuh"
#include "tma_ring.cuh"

namespace a3d {
namespace tma {

using namespace ring;

struct TmaSmem {
  Slot slot[NSLOT];
  float P[5][HY][HX];       // plane-k primitives with a 2-cell halo
  uint8_t C[HY][HX];        // plane-k codes (ghosts marked)
  float Fx[5][TY][TX + 1];  // a * flux of x face i-1/2
  float Fy[5][TY + 1][TX];  // a * flux of y face j-1/2
  float Ax[TY][TX + 1];
  float Ay[TY + 1][TX];
  uint64_t bar[NSLOT];
  int abort;
};

__device__ __forceinline__ Prim sprim(const TmaSmem& S, int y, int x, int d) {
  float P[5] = {S.P[0][y][x], S.P[1][y][x], S.P[2][y][x], S.P[3][y][x], S.P[4][y][x]};
  return rot(P, d);
}

// x face between columns x-1 and x of shared-memory row y; `own`, when given, is the
// primitive state of cell x already in registers (saves its five shared-memory loads).
__device__ __forceinline__ float face_x(const StageArgs& a, const TmaSmem& S, int y, int x, int i, int j, int k,
                                        float G[5], const float* own = nullptr) {
  const uint8_t cl = S.C[y][x - 1], cr = S.C[y][x];
  float A = 1.f;
  if (i - 1 >= 0 && (cl & C_IRR)) A = __ldg(a.ap0 + ((long)k * a.NY + j) * a.NX + (i - 1));
  if (A > 0.f) {
    float F[5];
    face_flux(sprim(S, y, x - 2, 0), sprim(S, y, x - 1, 0), own ? rot(own, 0) : sprim(S, y, x, 0),
              sprim(S, y, x + 1, 0), a.order2 && (cl & C_OKX), a.order2 && (cr & C_OKX), F);
    G[0] = A * F[0]; G[1] = A * F[1]; G[2] = A * F[2]; G[3] = A * F[3]; G[4] = A * F[4];
  } else {
    G[0] = G[1] = G[2] = G[3] = G[4] = 0.f;
  }
  return A;
}

__device__ __forceinline__ float face_y(const StageArgs& a, const TmaSmem& S, int y, int x, int i, int j, int k,
                                        float G[5], const float* own = nullptr) {
  const uint8_t cl = S.C[y - 1][x], cr = S.C[y][x];
  float A = 1.f;
  if (j - 1 >= 0 && (cl & C_IRR)) A = __ldg(a.ap1 + ((long)k * a.NY + (j - 1)) * a.NX + i);
  if (A > 0.f) {
    float F[5];
    face_flux(sprim(S, y - 2, x, 1), sprim(S, y - 1, x, 1), own ? rot(own, 1) : sprim(S, y, x, 1),
              sprim(S, y + 1, x, 1), a.order2 && (cl & C_OKY), a.order2 && (cr & C_OKY), F);
    G[0] = A * F[0]; G[1] = A * F[2]; G[2] = A * F[1]; G[3] = A * F[3]; G[4] = A * F[4];
  } else {
    G[0] = G[1] = G[2] = G[3] = G[4] = 0.f;
  }
  return A;
}

// z face between cell b (plane k) and cell c (plane k+1) of the column.  Lb is b's +z face
// state, carried from the face below; c's slope gives this face's right state and, in Lc, the
// left state of the face above: each z slope is formed once.  Same numbers as face_flux.
__device__ __forceinline__ float face_z_carry(const StageArgs& a, const float Lb[5], const float Pb[5],
                                              const float Pc[5], const float Pe[5], uint8_t cb, uint8_t cc,
                                              bool in_dom_b, long qb, float G[5], float Lc[5]) {
  const float h = (a.order2 && (cc & C_OKZ)) ? 0.5f : 0.f;
  float Rc[5];
#pragma unroll
  for (int v = 0; v < 5; v++) {
    const float sl = minmod(Pc[v] - Pb[v], Pe[v] - Pc[v]);
    Rc[v] = fmaf(-h, sl, Pc[v]);
    Lc[v] = fmaf(h, sl, Pc[v]);
  }
  float A = 1.f;
  if (in_dom_b && (cb & C_IRR)) A = __ldg(a.ap2 + qb);
  if (A > 0.f) {
    float F[5];
    face_flux_lr(rot(Lb, 2), rot(Rc, 2), rot(Pb, 2), rot(Pc, 2), F);
    G[0] = A * F[0]; G[1] = A * F[2]; G[2] = A * F[3]; G[3] = A * F[1]; G[4] = A * F[4];
  } else {
    G[0] = G[1] = G[2] = G[3] = G[4] = 0.f;
  }
  return A;
}

// One tile: columns (bx, by), planes [bz*kz, bz*kz + kz).  Stage 1 reads the state through
// tmQ; stage 2 also reads the base state Bp; the result goes to Outp.  Returns false if a
// bounded wait ran out (flagged in *a.err); the CTA's copies in flight are then drained.
// PERSISTENT: the CTA runs further tiles after this one (batch kernel), so the tile starts with
// a barrier and retires its ring barriers at the end.
// RANGE: the z runs cover planes [a.kb, a.ke) only (a z slab's own planes, or one z chunk of a
// pipelined step).  PUSH: a cell store also goes to a neighbour slab that keeps the plane as a
// halo plane (store_out).
template <bool STAGE2, bool PERSISTENT, bool RANGE = false, bool PUSH = false>
__device__ __forceinline__ bool stage_tile(TmaSmem& S, const CUtensorMap* tmQ, const CUtensorMap* tmC,
                                           const StageArgs& a, const float* __restrict__ Bp,
                                           float* __restrict__ Outp, int bx, int by, int bz, int kz) {
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int i0 = bx * TX, j0 = by * TY;
  const int i = i0 + tx, j = j0 + ty;
  const int k0 = RANGE ? a.kb + bz * kz : bz * kz, k1 = RANGE ? min(a.ke, k0 + kz) : min(a.NZ, k0 + kz);
  const bool in_dom = i < a.NX && j < a.NY;
  const long NXY = (long)a.NX * a.NY, Np = a.Np;
  const float rx = in_dom ? a.rXd[i] : 0.f, ry = in_dom ? a.rYd[j] : 0.f;

  if (PERSISTENT) __syncthreads();  // a previous tile of this CTA is completely done with the shared memory
  if (threadIdx.x == 0) {
    for (int s = 0; s < NSLOT; s++) mbar_init(&S.bar[s], 1);
    S.abort = 0;
    fence_barrier_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    fence_proxy_async_smem();  // earlier tiles' generic reads of the slots before these copies
    for (int p = k0 - 2; p <= k0 + 1; p++) issue_plane(S, tmQ, tmC, a, p, k0, i0, j0);
  }

  bool ok = true;
  float Lz[5], W0[5], W1[5], W2[5];  // Lz: +z face state of the plane-k cell (carried)
  uint8_t cm, c0, c1, c2;
  float Gz[5], Az = 1.f;
  {
    float Wa[5], Wm[5], Lm[5];
    ok &= mbar_wait(&S.bar[slot_of(k0 - 2, k0)], parity_of(k0 - 2, k0), a.wait_limit);
    slot_cell(a, S.slot[slot_of(k0 - 2, k0)], i, j, k0 - 2, i0, j0, Wa);
    ok &= mbar_wait(&S.bar[slot_of(k0 - 1, k0)], parity_of(k0 - 1, k0), a.wait_limit);
    cm = slot_cell(a, S.slot[slot_of(k0 - 1, k0)], i, j, k0 - 1, i0, j0, Wm);
    ok &= mbar_wait(&S.bar[slot_of(k0, k0)], parity_of(k0, k0), a.wait_limit);
    c0 = slot_cell(a, S.slot[slot_of(k0, k0)], i, j, k0, i0, j0, W0);
    ok &= mbar_wait(&S.bar[slot_of(k0 + 1, k0)], parity_of(k0 + 1, k0), a.wait_limit);
    c1 = slot_cell(a, S.slot[slot_of(k0 + 1, k0)], i, j, k0 + 1, i0, j0, W1);
#pragma unroll
    for (int c = 0; c < 5; c++) Gz[c] = 0.f;
    {
      const float hm = (a.order2 && (cm & C_OKZ)) ? 0.5f : 0.f;
#pragma unroll
      for (int v = 0; v < 5; v++) Lm[v] = fmaf(hm, minmod(Wm[v] - Wa[v], W0[v] - Wm[v]), Wm[v]);
    }
    if (in_dom) Az = face_z_carry(a, Lm, Wm, W0, W1, cm, c0, k0 - 1 >= 0, ((long)(k0 - 1) * a.NY + j) * a.NX + i, Gz, Lz);
  }
  if (!ok) S.abort = 1;
  __syncthreads();  // slots of planes k0-2 and k0-1 are free again
  int last_issued = k0 + 1;  // meaningful in thread 0, which issues every copy
  int first_pending = k0 - 2;
  if (S.abort) {
    drain(S, a, k0, first_pending, last_issued);
    return false;
  }
  if (threadIdx.x == 0) issue_plane(S, tmQ, tmC, a, k0 + 2, k0, i0, j0);
  last_issued = k0 + 2;

  for (int k = k0; k < k1; k++) {
    const long q = ((long)k * a.NY + j) * a.NX + i;    // geometry (reference) index
    const long qp = ((long)k * a.NY + j) * a.NXp + i;  // padded state index
    // ---- plane k+2 into the column window; plane k to shared memory ----
    const int sk = slot_of(k, k0), sk2 = slot_of(k + 2, k0);
    ok = mbar_wait(&S.bar[sk2], parity_of(k + 2, k0), a.wait_limit);
    c2 = slot_cell(a, S.slot[sk2], i, j, k + 2, i0, j0, W2);
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
        issue_plane(S, tmQ, tmC, a, k + 3, k0, i0, j0);
      }
      last_issued = k + 3;
    }
    // ---- face fluxes ----
    if (j < a.NY && i <= a.NX) {
      float G[5];
      const float A = face_x(a, S, ty + 2, tx + 2, i, j, k, G, W0);
#pragma unroll
      for (int v = 0; v < 5; v++) S.Fx[v][ty][tx] = G[v];
      S.Ax[ty][tx] = A;
    }
    if (i < a.NX && j <= a.NY) {
      float G[5];
      const float A = face_y(a, S, ty + 2, tx + 2, i, j, k, G, W0);
#pragma unroll
      for (int v = 0; v < 5; v++) S.Fy[v][ty][tx] = G[v];
      S.Ay[ty][tx] = A;
    }
    if (ty == TY - 1) {  // +y edge faces of the tile
      const int jj = j0 + TY;
      if (i < a.NX && jj - 1 < a.NY) {
        float G[5];
        const float A = face_y(a, S, TY + 2, tx + 2, i, jj, k, G);
#pragma unroll
        for (int v = 0; v < 5; v++) S.Fy[v][TY][tx] = G[v];
        S.Ay[TY][tx] = A;
      }
    } else if (ty == TY - 2 && tx < TY) {  // +x edge faces, one per row
      const int row = tx, ii = i0 + TX, jr = j0 + row;
      if (jr < a.NY && ii - 1 < a.NX) {
        float G[5];
        const float A = face_x(a, S, row + 2, TX + 2, ii, jr, k, G);
#pragma unroll
        for (int v = 0; v < 5; v++) S.Fx[v][row][TX] = G[v];
        S.Ax[row][TX] = A;
      }
    }
    float bq[5];
    if (STAGE2 && in_dom) {
#pragma unroll
      for (int c = 0; c < 5; c++) bq[c] = __ldg(Bp + c * Np + qp);
    }
    float Gn[5], An = 1.f;
    float Ln[5];
    if (in_dom) An = face_z_carry(a, Lz, W0, W1, W2, c0, c1, true, q, Gn, Ln);
    __syncthreads();
    // ---- residual and RK update ----
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
          R[c] = (S.Fx[c][ty][tx] - S.Fx[c][ty][tx + 1]) * rx + (S.Fy[c][ty][tx] - S.Fy[c][ty + 1][tx]) * ry +
                 (Gz[c] - Gn[c]) * rz;
        R[1] += pC * (S.Ax[ty][tx + 1] - S.Ax[ty][tx]) * rx;  // wall-pressure source
        R[2] += pC * (S.Ay[ty + 1][tx] - S.Ay[ty][tx]) * ry;
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
        const float gp = kG * Pb[4], as = gp * rsqrtf(gp * Pb[0]);
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
      if (PUSH) {
        store_out(a, Outp, qp, k, o);
      } else {
#pragma unroll
        for (int c = 0; c < 5; c++) Outp[c * Np + qp] = o[c];
      }
    }
#pragma unroll
    for (int c = 0; c < 5; c++) { Gz[c] = Gn[c]; Lz[c] = Ln[c]; W0[c] = W1[c]; W1[c] = W2[c]; }
    Az = An;
    cm = c0; c0 = c1; c1 = c2;
    (void)cm;
  }
  if (S.abort) {
    drain(S, a, k0, first_pending, last_issued);
    return false;
  }
  if (PERSISTENT) {
    // every issued plane has been waited for: retire the ring barriers so that the CTA can
    // initialise them again for its next tile
    __syncthreads();
    if (threadIdx.x == 0)
      for (int s = 0; s < NSLOT; s++) mbar_inval(&S.bar[s]);
  }
  return true;
}

}  // namespace tma
}  // namespace a3d
