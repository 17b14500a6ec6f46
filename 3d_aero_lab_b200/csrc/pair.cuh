// pair.cuh - packed two-lane arithmetic of the paired-cell stage tile (stage_pair.cuh).
//
// A thread of that tile owns two x-adjacent cells, so nearly every value it forms comes in
// pairs: two cells' primitives, two faces' reconstructed states, two fluxes.  sm_100a adds and
// multiplies such pairs in one instruction (FADD2 / FMUL2 / FFMA2, PTX `*.f32x2`), with the
// rounding of the scalar instruction in each lane.  Minimum, maximum, reciprocal, rsqrt and
// selects have no packed form and are written per lane.
//
// The arithmetic is the scheme of src/air_cfd.js:169-251 (cfdPrim5, mmod, cfdHLLC and the
// stage update) in the same rearranged float32 form as flux.cuh.
#pragma once
#include <cuda_runtime.h>
#include "flux.cuh"

namespace a3d {
namespace pk {

typedef float2 f2;

__device__ __forceinline__ f2 f2s(float s) { return make_float2(s, s); }
// Packed constants read from the constant bank (gamma, 1/(gamma-1), 1/2, -1/2, gamma-1): a
// packed operand must be a register pair or a constant-bank pair; pairs of immediates would
// be rebuilt in registers at every use (measured: 1.5 % faster than in-register constants).
__constant__ f2 kPkG = {kG, kG}, kPkIgm = {1.0f / kGm, 1.0f / kGm}, kPkHalf = {0.5f, 0.5f}, kPkMHalf = {-0.5f, -0.5f},
                kPkGm = {kGm, kGm};

__device__ __forceinline__ f2 add(f2 a, f2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ f2 mul(f2 a, f2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ f2 fma(f2 a, f2 b, f2 c) { return __ffma2_rn(a, b, c); }
// a - b: the packed subtraction (FADD2 with a negated operand), no constant operand to stage
__device__ __forceinline__ f2 sub(f2 a, f2 b) {
  f2 r;
  asm("{\n .reg .b64 ra, rb, rd;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n"
      " sub.rn.f32x2 rd, ra, rb;\n mov.b64 {%0, %1}, rd;\n}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}

__device__ __forceinline__ f2 mn(f2 a, f2 b) { return make_float2(fminf(a.x, b.x), fminf(a.y, b.y)); }
__device__ __forceinline__ f2 mx(f2 a, f2 b) { return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
__device__ __forceinline__ f2 rcp(f2 a) { return make_float2(__fdividef(1.0f, a.x), __fdividef(1.0f, a.y)); }
__device__ __forceinline__ f2 rsq(f2 a) { return make_float2(rsqrtf(a.x), rsqrtf(a.y)); }
__device__ __forceinline__ f2 sel(bool lx, bool ly, f2 a, f2 b) { return make_float2(lx ? a.x : b.x, ly ? a.y : b.y); }

// Rotated primitive states of two faces (un normal to the face, u1 and u2 tangential).
struct PP {
  f2 r, un, u1, u2, p;
};

// Conservative -> primitive for two cells, with the floors rho >= 1e-6, p >= 1e-7 (cfdPrim5,
// src/air_cfd.js:169).  Output order (rho, u, v, w, p).
__device__ __forceinline__ void prim2(const f2 q[5], f2 P[5]) {
  const f2 r = mx(q[0], f2s(1e-6f));
  const f2 ir = make_float2(1.0f / r.x, 1.0f / r.y);
  const f2 u = mul(q[1], ir), v = mul(q[2], ir), w = mul(q[3], ir);
  const f2 k2 = fma(u, u, fma(v, v, mul(w, w)));
  const f2 e = fma(mul(kPkMHalf, r), k2, q[4]);  // E - rho |u|^2 / 2
  P[0] = r; P[1] = u; P[2] = v; P[3] = w;
  P[4] = mx(mul(kPkGm, e), f2s(1e-7f));
}

// HLLC flux of two faces (cfdHLLC, src/air_cfd.js:179-195), the rearranged form of flux.cuh's
// hllc: d = S - u_K, q = rho_K d, g = 1/(S - S_M); rho* = q g; tangential fluxes v_t F_mass;
// E* = g (d E + (S_M - u)(q S_M + p)); the total energy on the upwind side only; no
// supersonic branch (the clipped wave speed S' = min(S_L, 0) / max(S_R, 0) makes the star
// formula the upwind state flux where the fan is supersonic).
__device__ __forceinline__ void hllc2(const PP& L, const PP& R, f2 F[5]) {
  const f2 gL = mul(kPkG, L.p), gR = mul(kPkG, R.p);
  const f2 aL = mul(gL, rsq(mul(gL, L.r))), aR = mul(gR, rsq(mul(gR, R.r)));
  const f2 SL = mn(sub(L.un, aL), sub(R.un, aR)), SR = mx(add(L.un, aL), add(R.un, aR));
  const f2 dL = sub(SL, L.un), dR = sub(SR, R.un);
  const f2 qL = mul(L.r, dL), qR = mul(R.r, dR);
  const f2 SM = mul(sub(fma(qL, L.un, sub(R.p, L.p)), mul(qR, R.un)), rcp(sub(qL, qR)));
  const bool lx = SM.x >= 0.f, ly = SM.y >= 0.f;
  const f2 rK = sel(lx, ly, L.r, R.r), uK = sel(lx, ly, L.un, R.un);
  const f2 v1 = sel(lx, ly, L.u1, R.u1), v2 = sel(lx, ly, L.u2, R.u2), pK = sel(lx, ly, L.p, R.p);
  const f2 kK = fma(uK, uK, fma(v1, v1, mul(v2, v2)));
  const f2 EK = fma(pK, kPkIgm, mul(mul(kPkHalf, rK), kK));
  const f2 S = make_float2(lx ? fminf(SL.x, 0.f) : fmaxf(SR.x, 0.f), ly ? fminf(SL.y, 0.f) : fmaxf(SR.y, 0.f));
  const f2 d = sel(lx, ly, dL, dR), q = sel(lx, ly, qL, qR);
  const f2 den = sub(sel(lx, ly, SL, SR), SM);
  // where S' = 0 the star terms are multiplied away; keep their divisor finite there
  const f2 g = make_float2(__fdividef(1.0f, S.x != 0.f ? den.x : 1.f), __fdividef(1.0f, S.y != 0.f ? den.y : 1.f));
  const f2 m = mul(rK, uK), qg = mul(q, g);
  F[0] = fma(S, sub(qg, rK), m);
  F[1] = fma(S, sub(mul(qg, SM), m), fma(m, uK, pK));
  F[2] = mul(v1, F[0]);
  F[3] = mul(v2, F[0]);
  const f2 Es = mul(g, fma(sub(SM, uK), fma(q, SM, pK), mul(d, EK)));
  F[4] = fma(S, sub(Es, EK), mul(uK, add(EK, pK)));
}

// The half-slope factor of a cell: 1/2 when the MUSCL slope test passed (flag bit set), else 0
// (the state is then the cell value, src/air_cfd.js:213-216).
__device__ __forceinline__ float half_if(uint32_t code, uint32_t bit) { return (code & bit) ? 0.5f : 0.f; }

}  // namespace pk
}  // namespace a3d
