// stage_pair.cuh - the paired-cell, TMA-fed z-marching RK-stage tile (KERNEL_PAIR).
//
// A CTA owns 32 x 16 cell columns and walks a run of z planes; each of its 256 threads owns
// the two x-adjacent cells (x0, x0+1) of one row, so that the arithmetic of the pair runs in
// packed f32x2 instructions (pair.cuh):
//   * y faces j-1/2 and z faces k+1/2 of the two cells: one packed evaluation each;
//   * the x faces x0-1/2 and x0+1/2: one packed evaluation, the three x slopes of the pair
//     (cells x0-1, x0, x0+1) formed once;
//   * residual, local time step, RK update and clamps of the two cells: packed.
// Every face is evaluated once per tile; the tile's +x and +y edge faces by two warps.
//
// The planes arrive through a 4-deep ring of shared-memory slots filled by
// `cp.async.bulk.tensor` (one 40 x 20 x 5-component state box and one 64 x 20 code box per
// plane, completing on the slot's mbarrier; no cluster multicast).  Per plane k:
//   [A] plane-k primitives to shared memory (own pair from the column registers, the 2-cell
//       halo - no corners, which no face reads - by warps 0-2 from the slot); barrier;
//       thread 0 queues plane k+3 into the slot plane k-1 has left;
//   [B] x and y face fluxes to shared memory, edge faces; stage 2 loads its base state;
//       wait for plane k+2, its column primitives into the registers, z face k+1/2;
//       barrier;
//   [C] residual, local dt, RK update, clamps, store.
#pragma once
#include <cudaTypedefs.h>
#include "flux.cuh"
#include "pair.cuh"
#include "solver.cuh"
#include "tma.cuh"

namespace a3d {
namespace pair {

using namespace pk;

constexpr int TX = 32, TY = 16;
constexpr int NT = (TX / 2) * TY;  // 256 threads, one x-pair of cells each
constexpr int HY = TY + 4;         // rows with the 2-row halo
constexpr int NP = TX / 2 + 3;     // pairs per row of the plane arrays: columns i0-2 .. i0+TX+3
constexpr int QBX = 40;            // state box width: x from i0-4 (16-byte aligned start)
constexpr int CBX = 64;            // code box width: x from i0-16
constexpr int NSLOT = 4;
constexpr uint32_t kQBytes = 5 * HY * QBX * 4, kCBytes = HY * CBX;
// A tiled TMA copy needs its innermost coordinate times the element size to be a multiple of
// 16 bytes: the state box starts at x = i0 - 4 (float) and the code box at x = i0 - 16 (u8),
// both aligned when TX is a multiple of 16.
static_assert(TX % 16 == 0, "TMA box x origins must stay 16-byte aligned");
static_assert((QBX * 4) % 16 == 0 && CBX % 16 == 0, "TMA box rows must be whole 16-byte units");
static_assert(kQBytes % 16 == 0 && kCBytes % 16 == 0, "TMA transaction sizes must be 16-byte multiples");
static_assert(QBX >= TX + 8 && CBX >= TX + 18, "the boxes must cover the tile and its 2-cell x halo");

struct __align__(128) Slot {
  float Q[5][HY][QBX];  // conservative state of one plane
  uint8_t C[HY][CBX];   // codes of that plane
};
static_assert(sizeof(Slot) % 128 == 0, "slots must keep the 128-byte TMA destination alignment");

struct PairSmem {
  Slot slot[NSLOT];
  float2 P[5][HY][NP];          // plane-k primitives; pair p holds cells (i0-2+2p, i0-1+2p)
  uint16_t C[HY][NP];           // their codes, first cell in the low byte
  float2 Fx[5][TY][TX / 2 + 1]; // a * flux of x faces (x0-1/2, x0+1/2) of each pair; [16].x: the +x edge face
  float2 Ax[TY][TX / 2 + 1];
  float2 Fy[5][TY + 1][TX / 2]; // a * flux of the y faces j-1/2 of each pair; row TY: the +y edge faces
  float2 Ay[TY + 1][TX / 2];
  uint64_t bar[NSLOT];
  int abort;
};

// Slot of plane p for a CTA whose run starts at k0 (the ring starts with plane k0-2), and the
// mbarrier phase parity of that use of the slot.
__device__ __forceinline__ int slot_of(int p, int k0) { return (p - k0 + 2) & (NSLOT - 1); }
__device__ __forceinline__ uint32_t parity_of(int p, int k0) { return ((p - k0 + 2) / NSLOT) & 1; }

// Thread 0 queues plane p into its slot: one state box and one code box, or a bare arrive
// when the plane lies outside the domain (its cells are then all far-field ghosts).
__device__ __forceinline__ void issue_plane(PairSmem& S, const CUtensorMap* tmQ, const CUtensorMap* tmC,
                                            const StageArgs& a, int p, int k0, int i0, int j0) {
  const int s = slot_of(p, k0);
  if (p < 0 || p >= a.NZ) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&S.bar[s])) : "memory");
    return;
  }
  mbar_expect_tx(&S.bar[s], kQBytes + kCBytes);
  tma_load_4d(&S.slot[s].Q[0][0][0], tmQ, &S.bar[s], i0 - 4, j0 - 2, p, 0);
  tma_load_3d(&S.slot[s].C[0][0], tmC, &S.bar[s], i0 - 16, j0 - 2, p);
}

// A wait ran out: flag the error for the host and wait (bounded, full limit) for the copies
// this CTA still has in flight, so that none lands in shared memory after the CTA has left.
__device__ __forceinline__ void drain(PairSmem& S, const StageArgs& a, int k0, int first_pending, int last_issued) {
  if (threadIdx.x != 0) return;
  atomicOr(a.err, 1);
  for (int p = first_pending; p <= last_issued; p++) mbar_wait(&S.bar[slot_of(p, k0)], parity_of(p, k0));
}

// Primitive states and codes of cells (x, x+1) of row j in the resident plane k (slot s), x
// even, with the ghost rules of src/air_cfd.js:205-210: far field outside x, z and +y, the
// symmetry mirror with v negated below y = 0, the fixed state in fixed-state cells (type >= 3).
// INSIDE: the caller knows both cells lie inside the domain (no ghost tests).  Codes: first
// cell in the low byte; ghosts T_GHOST, mirror cells T_MIRROR (no slope or aperture bits).
template <bool INSIDE>
__device__ __forceinline__ uint32_t slot_pair(const StageArgs& a, const Slot& s, int x, int j, int k, int i0, int j0,
                                              f2 P[5]) {
  const bool mirror = !INSIDE && j < 0;
  // for every pair a tile reads these slot positions stay inside the slot; whatever a ghost's
  // position holds (another plane, or nothing loaded) is replaced below
  const int ys = (mirror ? -1 - j : j) - j0 + 2, xs = x - i0 + 4;
  const uint32_t c = *reinterpret_cast<const uint16_t*>(&s.C[ys][x - i0 + 16]);
  f2 q[5];
#pragma unroll
  for (int v = 0; v < 5; v++) q[v] = *reinterpret_cast<const float2*>(&s.Q[v][ys][xs]);
  prim2(q, P);
  const uint32_t t0 = c & 7, t1 = (c >> 8) & 7;
  if (INSIDE) {
    if (t0 >= T_SINK || t1 >= T_SINK) {  // fixed-state cells (rare)
#pragma unroll
      for (int v = 0; v < 5; v++) {
        if (t0 >= T_SINK) P[v].x = a.Pfix[t0 - T_SINK][v];
        if (t1 >= T_SINK) P[v].y = a.Pfix[t1 - T_SINK][v];
      }
    }
    return c;
  }
  const bool kg = k < 0 || k >= a.NZ || j >= a.NY;
  const bool g0 = kg || x < 0 || x >= a.NX, g1 = kg || x + 1 < 0 || x + 1 >= a.NX;
  if ((!g0 && t0 >= T_SINK) || (!g1 && t1 >= T_SINK)) {
#pragma unroll
    for (int v = 0; v < 5; v++) {
      if (!g0 && t0 >= T_SINK) P[v].x = a.Pfix[t0 - T_SINK][v];
      if (!g1 && t1 >= T_SINK) P[v].y = a.Pfix[t1 - T_SINK][v];
    }
  }
#pragma unroll
  for (int v = 0; v < 5; v++) {
    P[v].x = g0 ? a.Pff[v] : P[v].x;
    P[v].y = g1 ? a.Pff[v] : P[v].y;
  }
  P[2].x = (mirror && !g0) ? -P[2].x : P[2].x;
  P[2].y = (mirror && !g1) ? -P[2].y : P[2].y;
  const uint32_t e0 = g0 ? (uint32_t)T_GHOST : mirror ? (uint32_t)T_MIRROR : (c & 0xFF);
  const uint32_t e1 = g1 ? (uint32_t)T_GHOST : mirror ? (uint32_t)T_MIRROR : (c >> 8);
  return e0 | (e1 << 8);
}

// x faces x0-1/2 (lane x) and x0+1/2 (lane y) of the cell pair at plane-array pair p, row y
// (cells x0, x0+1 of row jj, plane k).  c: the pair's primitives; cl, cc: codes of the pair to
// the left and of this pair.  The slopes of cells x0-1, x0, x0+1 are each formed once.
// G: aperture-weighted fluxes (mass, x-, y-, z-momentum, energy); returns the apertures.
__device__ __forceinline__ f2 xfaces(const StageArgs& a, const PairSmem& S, int y, int p, const f2 c[5], uint32_t cl,
                                     uint32_t cc, int q, uint32_t okm, f2 G[5]) {
  const float h1 = half_if((cl >> 8) & okm, C_OKX), h2 = half_if(cc & okm, C_OKX);
  const float h3 = half_if((cc >> 8) & okm, C_OKX);
  f2 Ls[5], Rs[5];
#pragma unroll
  for (int v = 0; v < 5; v++) {
    const f2 ab = S.P[v][y][p - 1];   // cells x0-2, x0-1
    const float e = S.P[v][y][p + 1].x;  // cell x0+2
    const float p0 = ab.x, p1 = ab.y, p2 = c[v].x, p3 = c[v].y;
    const float s1 = minmod(p1 - p0, p2 - p1), s2 = minmod(p2 - p1, p3 - p2), s3 = minmod(p3 - p2, e - p3);
    Ls[v] = make_float2(fmaf(h1, s1, p1), fmaf(h2, s2, p2));
    Rs[v] = make_float2(fmaf(-h2, s2, p2), fmaf(-h3, s3, p3));
  }
  // face x0-1/2 is cell x0-1's +x face, face x0+1/2 cell x0's (src/air_cfd.js:211, 223-224)
  // q: geometry index of cell x0; a cell outside the domain carries a ghost code, never C_IRR
  f2 A = f2s(1.f);
  if ((cl >> 8) & C_IRR) A.x = __ldg(a.ap0 + q - 1);
  if (cc & C_IRR) A.y = __ldg(a.ap0 + q);
  // a closed face (A = 0) contributes A * F = 0: the flux of its finite states is formed
  // anyway, without a branch (src/air_cfd.js:223-224 skips it)
  f2 F[5];
  hllc2(PP{Ls[0], Ls[1], Ls[2], Ls[3], Ls[4]}, PP{Rs[0], Rs[1], Rs[2], Rs[3], Rs[4]}, F);
#pragma unroll
  for (int v = 0; v < 5; v++) G[v] = mul(A, F[v]);
  return A;
}

// y faces j-1/2 of the two cells (x0, x0+1) at plane-array pair p, row y (cell row jj, plane
// k).  c: their primitives; cb, cc: codes of the pair in row y-1 and of this pair.
__device__ __forceinline__ f2 yfaces(const StageArgs& a, const PairSmem& S, int y, int p, const f2 c[5], uint32_t cb,
                                     uint32_t cc, int qb, uint32_t okm, f2 G[5]) {
  const f2 hL = make_float2(half_if(cb & okm, C_OKY), half_if(cb & okm, C_OKY << 8));
  const f2 hR = make_float2(-half_if(cc & okm, C_OKY), -half_if(cc & okm, C_OKY << 8));
  f2 Ls[5], Rs[5];
#pragma unroll
  for (int v = 0; v < 5; v++) {
    const f2 pa = S.P[v][y - 2][p], pb = S.P[v][y - 1][p], pe = S.P[v][y + 1][p];
    const f2 d1 = sub(pb, pa), d2 = sub(c[v], pb), d3 = sub(pe, c[v]);
    const f2 sL = make_float2(minmod(d1.x, d2.x), minmod(d1.y, d2.y));
    const f2 sR = make_float2(minmod(d2.x, d3.x), minmod(d2.y, d3.y));
    Ls[v] = fma(hL, sL, pb);
    Rs[v] = fma(hR, sR, c[v]);
  }
  // face j-1/2 is cell (x, j-1)'s +y face; below y = 0 lies the symmetry mirror (open)
  // qb: geometry index of cell (x0, jj-1); ghost and mirror codes never carry C_IRR
  f2 A = f2s(1.f);
  if (cb & C_IRR) A.x = __ldg(a.ap1 + qb);
  if (cb & (C_IRR << 8)) A.y = __ldg(a.ap1 + qb + 1);
  f2 F[5];  // closed faces: A * F = 0, no branch
  hllc2(PP{Ls[0], Ls[2], Ls[1], Ls[3], Ls[4]}, PP{Rs[0], Rs[2], Rs[1], Rs[3], Rs[4]}, F);
  G[0] = mul(A, F[0]); G[1] = mul(A, F[2]); G[2] = mul(A, F[1]); G[3] = mul(A, F[3]); G[4] = mul(A, F[4]);
  return A;
}

// z faces k+1/2 of the pair: cells b (plane k, primitives Pb, codes cb) and c (plane k+1, Pc,
// cc), with e (plane k+2, Pe) above.  Lb is b's +z face state, carried from the face below;
// c's slope gives this face's right state and, in Lc, the left state of the face above: each
// z slope is formed once.  qb: geometry index of b's first cell.
__device__ __forceinline__ f2 zfaces(const StageArgs& a, const f2 Lb[5], const f2 Pb[5], const f2 Pc[5],
                                     const f2 Pe[5], uint32_t cb, uint32_t cc, int qb, uint32_t okm, f2 G[5],
                                     f2 Lc[5]) {
  const f2 h = make_float2(half_if(cc & okm, C_OKZ), half_if(cc & okm, C_OKZ << 8));
  const f2 hn = make_float2(-h.x, -h.y);
  f2 Rc[5];
#pragma unroll
  for (int v = 0; v < 5; v++) {
    const f2 d1 = sub(Pc[v], Pb[v]), d2 = sub(Pe[v], Pc[v]);
    const f2 s = make_float2(minmod(d1.x, d2.x), minmod(d1.y, d2.y));
    Rc[v] = fma(hn, s, Pc[v]);
    Lc[v] = fma(h, s, Pc[v]);
  }
  // cells outside the domain carry ghost codes, never C_IRR
  f2 A = f2s(1.f);
  if (cb & C_IRR) A.x = __ldg(a.ap2 + qb);
  if (cb & (C_IRR << 8)) A.y = __ldg(a.ap2 + qb + 1);
  f2 F[5];  // closed faces: A * F = 0, no branch
  hllc2(PP{Lb[0], Lb[3], Lb[1], Lb[2], Lb[4]}, PP{Rc[0], Rc[3], Rc[1], Rc[2], Rc[4]}, F);
  G[0] = mul(A, F[0]); G[1] = mul(A, F[2]); G[2] = mul(A, F[3]); G[3] = mul(A, F[1]); G[4] = mul(A, F[4]);
  return A;
}

// Baffle transpiration of one cell (src/air_cfd.js:226-233): w = u dz/dx through the +z face
// (slope sUp = ap3 of the cell) and the -z face (sDn = ap3 of the cell below), with the cell's
// own state; Am, Ap: the cell's -z and +z apertures.
__device__ __forceinline__ void baffle(const StageArgs& a, int q, int k, int NXY, float r, float u, float v, float w,
                                       float pC, float Am, float Ap, float rz, float R[5]) {
  const float sUp = __ldg(a.ap3 + q), sDn = k > 0 ? __ldg(a.ap3 + q - NXY) : 0.f;
  if (sUp != 0.f || sDn != 0.f) {
    const float Hh = (pC / kGm + 0.5f * r * (u * u + v * v + w * w) + pC) / r;
    const float m = (sDn != 0.f ? (1.f - Am) * r * u * sDn : 0.f) - (sUp != 0.f ? (1.f - Ap) * r * u * sUp : 0.f);
    const float mh = m * rz;
    R[0] += mh; R[1] += mh * u; R[2] += mh * v; R[3] += mh * w; R[4] += mh * Hh;
  }
}

// Output store of a pair: the cell's own buffer and, on a z slab whose neighbour keeps this
// plane as a halo plane, the neighbour's buffer of the same role (peer stores across GPUs).
template <bool PUSH>
__device__ __forceinline__ void store_pair(const StageArgs& a, float* __restrict__ Out, long qp, int k, bool in1,
                                           const f2 o[5]) {
#pragma unroll
  for (int c = 0; c < 5; c++) {
    if (in1) *reinterpret_cast<float2*>(Out + c * a.Np + qp) = o[c];
    else Out[c * a.Np + qp] = o[c].x;
  }
  if (PUSH) {
#pragma unroll
    for (int sd = 0; sd < 2; sd++) {
      if (a.peer[sd] && k >= a.peer_k0[sd] && k < a.peer_k1[sd]) {
        float* P = a.peer[sd] + qp + (long)a.peer_dk[sd] * a.NY * a.NXp;
#pragma unroll
        for (int c = 0; c < 5; c++) {
          if (in1) *reinterpret_cast<float2*>(P + c * a.peer_np[sd]) = o[c];
          else P[c * a.peer_np[sd]] = o[c].x;
        }
      }
    }
  }
}

// One tile: columns (bx, by), planes [bz*kz, bz*kz + kz).  Stage 1 reads the state through
// tmQ; stage 2 also reads the base state Bp; the result goes to Outp.  Returns false if a
// bounded wait ran out (flagged in *a.err); the CTA's copies in flight are then drained.
// PERSISTENT: the CTA runs further tiles after this one, so the tile starts with a barrier and
// retires its ring barriers at the end.  RANGE: the z runs cover planes [a.kb, a.ke) only (a z
// slab's own planes, or one z chunk of a pipelined step).  PUSH: stores also go to the
// neighbour slab that keeps the plane as a halo plane.
template <bool STAGE2, bool PERSISTENT, bool RANGE = false, bool PUSH = false>
__device__ __forceinline__ bool stage_tile(PairSmem& S, const CUtensorMap* tmQ, const CUtensorMap* tmC,
                                           const StageArgs& a, const float* __restrict__ Bp,
                                           float* __restrict__ Outp, int bx, int by, int bz, int kz) {
  const int t = threadIdx.x, tx2 = t & 15, ty = t >> 4;
  const int i0 = bx * TX, j0 = by * TY;
  const int x0 = i0 + 2 * tx2, j = j0 + ty;
  const int pp = tx2 + 1, hy = ty + 2;  // this thread's pair and row in the plane arrays
  const int k0 = RANGE ? a.kb + bz * kz : bz * kz, k1 = RANGE ? min(a.ke, k0 + kz) : min(a.NZ, k0 + kz);
  const bool jin = j < a.NY;
  const bool in0 = jin && x0 < a.NX, in1 = jin && x0 + 1 < a.NX;
  // the halo (and so every cell the tile reads) inside the domain in x and y; own cells inside
  const bool tile_in = i0 >= 2 && i0 + TX + 2 <= a.NX && j0 >= 2 && j0 + TY + 2 <= a.NY;
  const bool own_in = i0 + TX <= a.NX && j0 + TY <= a.NY;
  const int NXY = a.NX * a.NY, PL = a.NY * a.NXp;  // plane strides of the geometry and state arrays
  const int q0 = j * a.NX + x0, qp0 = j * a.NXp + x0;  // this pair's indices in plane 0
  const long Np = a.Np;
  const uint32_t okm = a.order2 ? 0xFFFFu : 0u;  // slope flags count only at second order
  const f2 rx = make_float2(in0 ? a.rXd[x0] : 0.f, in1 ? a.rXd[x0 + 1] : 0.f);
  const f2 ry = f2s(jin ? a.rYd[j] : 0.f);
  // halo pair converted by threads 0..95: rows j0-2, j0-1 (warp 0), j0+TY, j0+TY+1 (warp 1),
  // the two columns either side of rows j0 .. j0+TY-1 (warp 2)
  int hp_y = 0, hp_p = 0;
  if (t < 32) { hp_y = t >> 4; hp_p = 1 + (t & 15); }
  else if (t < 64) { hp_y = HY - 2 + ((t - 32) >> 4); hp_p = 1 + (t & 15); }
  else if (t < 96) { hp_y = 2 + (t & 15); hp_p = (t & 16) ? TX / 2 + 1 : 0; }
  const int hp_x = i0 - 2 + 2 * hp_p, hp_j = j0 + hp_y - 2;

  if (PERSISTENT) __syncthreads();  // a previous tile of this CTA is completely done with the shared memory
  if (t == 0) {
    for (int s = 0; s < NSLOT; s++) mbar_init(&S.bar[s], 1);
    S.abort = 0;
    fence_barrier_init();
  }
  __syncthreads();
  if (t == 0) {
    fence_proxy_async_smem();  // earlier tiles' generic reads of the slots before these copies
    for (int p = k0 - 2; p <= k0 + 1; p++) issue_plane(S, tmQ, tmC, a, p, k0, i0, j0);
  }
  auto own = [&](int kk, f2 P[5]) -> uint32_t {
    const Slot& s = S.slot[slot_of(kk, k0)];
    if (own_in && kk >= 0 && kk < a.NZ) return slot_pair<true>(a, s, x0, j, kk, i0, j0, P);
    return slot_pair<false>(a, s, x0, j, kk, i0, j0, P);
  };

  bool ok = true;
  f2 W0[5], W1[5], Lz[5], Gz[5];  // column window (planes k, k+1), carried +z state, flux of face k-1/2
  f2 Az;
  uint32_t c0, c1;
  {
    f2 Wa[5], Wm[5], Lm[5];
    ok &= mbar_wait(&S.bar[slot_of(k0 - 2, k0)], parity_of(k0 - 2, k0), a.wait_limit);
    own(k0 - 2, Wa);
    ok &= mbar_wait(&S.bar[slot_of(k0 - 1, k0)], parity_of(k0 - 1, k0), a.wait_limit);
    const uint32_t cm = own(k0 - 1, Wm);
    ok &= mbar_wait(&S.bar[slot_of(k0, k0)], parity_of(k0, k0), a.wait_limit);
    c0 = own(k0, W0);
    ok &= mbar_wait(&S.bar[slot_of(k0 + 1, k0)], parity_of(k0 + 1, k0), a.wait_limit);
    c1 = own(k0 + 1, W1);
    const f2 hm = make_float2(half_if(cm & okm, C_OKZ), half_if(cm & okm, C_OKZ << 8));
#pragma unroll
    for (int v = 0; v < 5; v++) {
      const f2 d1 = sub(Wm[v], Wa[v]), d2 = sub(W0[v], Wm[v]);
      Lm[v] = fma(hm, make_float2(minmod(d1.x, d2.x), minmod(d1.y, d2.y)), Wm[v]);
    }
    Az = zfaces(a, Lm, Wm, W0, W1, cm, c0, (k0 - 1) * NXY + q0, okm, Gz, Lz);
  }
  if (!ok) S.abort = 1;
  __syncthreads();  // slots of planes k0-2 and k0-1 are free again
  int last_issued = k0 + 1;  // meaningful in thread 0, which issues every copy
  int first_pending = k0 - 2;
  if (S.abort) {
    drain(S, a, k0, first_pending, last_issued);
    return false;
  }
  if (t == 0) issue_plane(S, tmQ, tmC, a, k0 + 2, k0, i0, j0);
  last_issued = k0 + 2;

  for (int k = k0; k < k1; k++) {
    const int sk = slot_of(k, k0), sk2 = slot_of(k + 2, k0);
    const int q = k * NXY + q0;    // geometry index of the pair's first cell
    const int qp = k * PL + qp0;   // padded state index of the pair
    // ---- [A] plane k to shared memory ----
#pragma unroll
    for (int v = 0; v < 5; v++) S.P[v][hy][pp] = W0[v];
    S.C[hy][pp] = (uint16_t)c0;
    if (t < 96) {
      f2 P[5];
      const bool inside = tile_in && k >= 0 && k < a.NZ;
      const uint32_t c = inside ? slot_pair<true>(a, S.slot[sk], hp_x, hp_j, k, i0, j0, P)
                                : slot_pair<false>(a, S.slot[sk], hp_x, hp_j, k, i0, j0, P);
#pragma unroll
      for (int v = 0; v < 5; v++) S.P[v][hp_y][hp_p] = P[v];
      S.C[hp_y][hp_p] = (uint16_t)c;
    }
    __syncthreads();
    if (k + 3 <= k1 + 1) {
      if (t == 0) {
        fence_proxy_async_smem();
        issue_plane(S, tmQ, tmC, a, k + 3, k0, i0, j0);
      }
      last_issued = k + 3;
    }
    // ---- [B] x and y face fluxes ----
    {
      f2 G[5];
      const f2 A = xfaces(a, S, hy, pp, W0, S.C[hy][pp - 1], c0, q, okm, G);
#pragma unroll
      for (int v = 0; v < 5; v++) S.Fx[v][ty][tx2] = G[v];
      S.Ax[ty][tx2] = A;
    }
    {
      f2 G[5];
      const f2 A = yfaces(a, S, hy, pp, W0, S.C[hy - 1][pp], c0, q - a.NX, okm, G);
#pragma unroll
      for (int v = 0; v < 5; v++) S.Fy[v][ty][tx2] = G[v];
      S.Ay[ty][tx2] = A;
    }
    if (t >= 192 && t < 192 + TX / 2) {  // warp 6: the +y edge faces j0+TY-1/2
      const int e = t - 192;
      f2 c[5], G[5];
#pragma unroll
      for (int v = 0; v < 5; v++) c[v] = S.P[v][TY + 2][e + 1];
      const f2 A = yfaces(a, S, TY + 2, e + 1, c, S.C[TY + 1][e + 1], S.C[TY + 2][e + 1],
                          k * NXY + (j0 + TY - 1) * a.NX + i0 + 2 * e, okm, G);
#pragma unroll
      for (int v = 0; v < 5; v++) S.Fy[v][TY][e] = G[v];
      S.Ay[TY][e] = A;
    } else if (t >= 224 && t < 224 + TY) {  // warp 7: the +x edge faces i0+TX-1/2, one per row (lane x)
      const int r = t - 224;
      f2 c[5], G[5];
#pragma unroll
      for (int v = 0; v < 5; v++) c[v] = S.P[v][r + 2][TX / 2 + 1];
      const f2 A = xfaces(a, S, r + 2, TX / 2 + 1, c, S.C[r + 2][TX / 2], S.C[r + 2][TX / 2 + 1],
                          k * NXY + (j0 + r) * a.NX + i0 + TX, okm, G);
#pragma unroll
      for (int v = 0; v < 5; v++) S.Fx[v][r][TX / 2] = G[v];
      S.Ax[r][TX / 2] = A;
    }
    f2 bq[5];
    if (STAGE2 && in0) {
#pragma unroll
      for (int c = 0; c < 5; c++) bq[c] = __ldg(reinterpret_cast<const float2*>(Bp + c * Np + qp));
    }
    // ---- plane k+2 into the column window; z face k+1/2 ----
    ok = mbar_wait(&S.bar[sk2], parity_of(k + 2, k0), a.wait_limit);
    // S.abort is written only here, between the two barriers of a plane, and read only after
    // the second: every thread sees the same value
    if (!ok) S.abort = 1;
    f2 W2[5], Gn[5], Ln[5];
    const uint32_t c2 = own(k + 2, W2);
    const f2 An = zfaces(a, Lz, W0, W1, W2, c0, c1, q, okm, Gn, Ln);
    __syncthreads();
    if (S.abort) { first_pending = k + 2; break; }  // the wait for plane k+2 ran out
    // ---- [C] residual and RK update ----
    if (in0) {
      const Slot& sl = S.slot[sk];
      const int xs = 4 + 2 * tx2;
      const f2 rz = f2s(a.rZd[k]);
      f2 R[5];
#pragma unroll
      for (int c = 0; c < 5; c++) {
        const f2 fxm = S.Fx[c][ty][tx2];
        const f2 fxp = make_float2(fxm.y, S.Fx[c][ty][tx2 + 1].x);
        const f2 fym = S.Fy[c][ty][tx2], fyp = S.Fy[c][ty + 1][tx2];
        R[c] = fma(sub(Gz[c], Gn[c]), rz, fma(sub(fym, fyp), ry, mul(sub(fxm, fxp), rx)));
      }
      {  // wall-pressure source (src/air_cfd.js:225)
        const f2 axm = S.Ax[ty][tx2];
        const f2 axp = make_float2(axm.y, S.Ax[ty][tx2 + 1].x);
        const f2 aym = S.Ay[ty][tx2], ayp = S.Ay[ty + 1][tx2];
        const f2 pC = W0[4];
        R[1] = fma(mul(pC, sub(axp, axm)), rx, R[1]);
        R[2] = fma(mul(pC, sub(ayp, aym)), ry, R[2]);
        R[3] = fma(mul(pC, sub(An, Az)), rz, R[3]);
      }
      if (c0 & (C_BAF | (C_BAF << 8))) {  // baffle transpiration (rare)
        float Rx[5] = {R[0].x, R[1].x, R[2].x, R[3].x, R[4].x}, Ry[5] = {R[0].y, R[1].y, R[2].y, R[3].y, R[4].y};
        if (c0 & C_BAF)
          baffle(a, q, k, NXY, W0[0].x, W0[1].x, W0[2].x, W0[3].x, W0[4].x, Az.x, An.x, rz.x, Rx);
        if (in1 && (c0 & (C_BAF << 8)))
          baffle(a, q + 1, k, NXY, W0[0].y, W0[1].y, W0[2].y, W0[3].y, W0[4].y, Az.y, An.y, rz.y, Ry);
#pragma unroll
        for (int c = 0; c < 5; c++) R[c] = make_float2(Rx[c], Ry[c]);
      }
      f2 ph = f2s(1.f);
      if (c0 & C_IRR) ph.x = __ldg(a.phi + q);
      if (in1 && (c0 & (C_IRR << 8))) ph.y = __ldg(a.phi + q + 1);
      if (ph.x != 1.f || ph.y != 1.f) {
        const f2 iph = make_float2(1.f / ph.x, 1.f / ph.y);
#pragma unroll
        for (int c = 0; c < 5; c++) R[c] = mul(R[c], iph);
      }
      // local time step from the base state (src/air_cfd.js:243; stage 2 recomputes it from B = Q)
      f2 Pb[5];
      if (STAGE2) prim2(bq, Pb);
      else {
#pragma unroll
        for (int c = 0; c < 5; c++) Pb[c] = W0[c];
      }
      const f2 gp = mul(kPkG, Pb[4]);
      const f2 as = mul(gp, rsq(mul(gp, Pb[0])));
      const f2 su = make_float2(fabsf(Pb[1].x) + as.x, fabsf(Pb[1].y) + as.y);
      const f2 sv = make_float2(fabsf(Pb[2].x) + as.x, fabsf(Pb[2].y) + as.y);
      const f2 sw = make_float2(fabsf(Pb[3].x) + as.x, fabsf(Pb[3].y) + as.y);
      const f2 den = fma(sw, rz, fma(sv, ry, mul(su, rx)));
      const f2 num = mul(f2s(a.cfl), mx(ph, f2s(0.25f)));
      const f2 dt = make_float2(num.x / den.x, num.y / den.y);
      f2 o[5];
#pragma unroll
      for (int c = 0; c < 5; c++) {
        const f2 qin = *reinterpret_cast<const float2*>(&sl.Q[c][hy][xs]);
        const f2 s1 = fma(dt, R[c], qin);
        o[c] = STAGE2 ? fma(f2s(a.wa), bq[c], mul(f2s(a.wb), s1)) : s1;
      }
      // positivity clamps (src/air_cfd.js:247-249)
      o[0] = mx(o[0], f2s(1e-4f));
      const f2 k2 = mul(kPkHalf, fma(o[1], o[1], fma(o[2], o[2], mul(o[3], o[3]))));
      const f2 ke = make_float2(k2.x / o[0].x, k2.y / o[0].y);
      const f2 pe = mul(kPkGm, sub(o[4], ke));
      if (pe.x < 1e-5f) o[4].x = 1e-5f / kGm + ke.x;
      if (pe.y < 1e-5f) o[4].y = 1e-5f / kGm + ke.y;
      // solid and fixed-state cells (src/air_cfd.js:242): the base state, or the fixed state
      const uint32_t t0 = c0 & 7, t1 = (c0 >> 8) & 7;
      if (t0 != T_FLUID || t1 != T_FLUID) {
#pragma unroll
        for (int c = 0; c < 5; c++) {
          const f2 base = STAGE2 ? bq[c] : *reinterpret_cast<const f2*>(&sl.Q[c][hy][xs]);
          if (t0 != T_FLUID) o[c].x = t0 >= T_SINK ? a.Ufix[t0 - T_SINK][c] : base.x;
          if (t1 != T_FLUID && in1) o[c].y = t1 >= T_SINK ? a.Ufix[t1 - T_SINK][c] : base.y;
        }
      }
      store_pair<PUSH>(a, Outp, qp, k, in1, o);
    }
#pragma unroll
    for (int c = 0; c < 5; c++) { Gz[c] = Gn[c]; Lz[c] = Ln[c]; W0[c] = W1[c]; W1[c] = W2[c]; }
    Az = An;
    c0 = c1;
    c1 = c2;
  }
  if (S.abort) {  // read after the barrier that ended the loop: the same value in every thread
    drain(S, a, k0, first_pending, last_issued);
    return false;
  }
  if (PERSISTENT) {
    // every issued plane has been waited for: retire the ring barriers so that the CTA can
    // initialise them again for its next tile
    __syncthreads();
    if (t == 0)
      for (int s = 0; s < NSLOT; s++) mbar_inval(&S.bar[s]);
  }
  return true;
}

}  // namespace pair
}  // namespace a3d
