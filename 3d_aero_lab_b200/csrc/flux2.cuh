// flux2.cuh - HLLC written once for `float` (one face) and `float2` (two faces at once in
// sm_100a packed f32x2 arithmetic: FADD2 / FMUL2 / FFMA2), so that a face evaluated alone
// and a face evaluated in a pair produce the same numbers.
//
// Same flux as cfdHLLC (src/air_cfd.js:179-195): Davis wave speeds, contact speed SM, star
// state on the upwind side of the contact, upwind state flux when the fan is supersonic.
// Branch-free: the star and the upwind fluxes are both formed and selected per face.
#pragma once
#include <cuda_runtime.h>
#include "flux.cuh"

namespace a3d {
namespace v {

// Scalar forms round every operation like the packed ones (no mul+add contraction), so a face
// gives bit-identical fluxes whether it is evaluated alone or in a pair - and the result of a
// case does not depend on how its planes are split into tiles.
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float rcp(float a) { return __fdividef(1.0f, a); }
__device__ __forceinline__ float rsqrt(float a) { return rsqrtf(a); }
__device__ __forceinline__ float min(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ float max(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ float splat(float s, float) { return s; }
__device__ __forceinline__ float neg(float a) { return -a; }

__device__ __forceinline__ float2 add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 rcp(float2 a) { return make_float2(__fdividef(1.0f, a.x), __fdividef(1.0f, a.y)); }
__device__ __forceinline__ float2 rsqrt(float2 a) { return make_float2(rsqrtf(a.x), rsqrtf(a.y)); }
__device__ __forceinline__ float2 min(float2 a, float2 b) { return make_float2(fminf(a.x, b.x), fminf(a.y, b.y)); }
__device__ __forceinline__ float2 max(float2 a, float2 b) { return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
__device__ __forceinline__ float2 splat(float s, float2) { return make_float2(s, s); }
__device__ __forceinline__ float2 neg(float2 a) { return make_float2(-a.x, -a.y); }

// Per-face predicates and selects.
struct M1 { bool x; };
struct M2 { bool x, y; };
__device__ __forceinline__ M1 ge0(float a) { return {a >= 0.f}; }
__device__ __forceinline__ M2 ge0(float2 a) { return {a.x >= 0.f, a.y >= 0.f}; }
__device__ __forceinline__ M1 le0(float a) { return {a <= 0.f}; }
__device__ __forceinline__ M2 le0(float2 a) { return {a.x <= 0.f, a.y <= 0.f}; }
__device__ __forceinline__ M1 ne0(float a) { return {a != 0.f}; }
__device__ __forceinline__ M2 ne0(float2 a) { return {a.x != 0.f, a.y != 0.f}; }
__device__ __forceinline__ M1 lor(M1 a, M1 b) { return {a.x || b.x}; }
__device__ __forceinline__ M2 lor(M2 a, M2 b) { return {a.x || b.x, a.y || b.y}; }
__device__ __forceinline__ float sel(M1 m, float a, float b) { return m.x ? a : b; }
__device__ __forceinline__ float2 sel(M2 m, float2 a, float2 b) { return make_float2(m.x ? a.x : b.x, m.y ? a.y : b.y); }

template <class T>
struct PrimV {
  T r, un, u1, u2, p;  // rotated frame: un normal to the face
};

template <class T, class M>
__device__ __forceinline__ PrimV<T> sel(M m, const PrimV<T>& a, const PrimV<T>& b) {
  return {sel(m, a.r, b.r), sel(m, a.un, b.un), sel(m, a.u1, b.u1), sel(m, a.u2, b.u2), sel(m, a.p, b.p)};
}

// HLLC flux through faces with left/right states L, R (already reconstructed).
// F = {mass, normal momentum, tangential momenta, energy}.
// Same rearrangement as flux.cuh: d = S - u_K, q = rho_K d, g = 1/(S - S_M); rho* = q g,
// tangential fluxes v_t F_mass, E* = g (d E + (S_M - u)(q S_M + p)); the total energy on the
// upwind side K only; sound speeds g p rsqrt(g p rho); and no supersonic branch: with the wave
// speed clipped to S' = min(S_L, 0) left of the contact and max(S_R, 0) right of it, the star
// formula gives the upwind state flux where the fan is supersonic (S' = 0).
template <class T>
__device__ __forceinline__ void hllc(const PrimV<T>& L, const PrimV<T>& R, T F[5]) {
  const T g = splat(kG, L.r), igm = splat(1.0f / kGm, L.r), half = splat(0.5f, L.r), zero = splat(0.f, L.r);
  const T one = splat(1.f, L.r);
  const T gL = mul(g, L.p), gR = mul(g, R.p);
  const T aL = mul(gL, rsqrt(mul(gL, L.r))), aR = mul(gR, rsqrt(mul(gR, R.r)));
  const T SL = min(sub(L.un, aL), sub(R.un, aR)), SR = max(add(L.un, aL), add(R.un, aR));
  const T dL = sub(SL, L.un), dR = sub(SR, R.un);
  const T qL = mul(L.r, dL), qR = mul(R.r, dR);
  // contact speed SM = (pR - pL + qL uL - qR uR) / (qL - qR)
  const T SM = mul(sub(fma(qL, L.un, sub(R.p, L.p)), mul(qR, R.un)), rcp(sub(qL, qR)));
  const auto left = ge0(SM);
  const PrimV<T> K = sel(left, L, R);
  const T kK = fma(K.un, K.un, fma(K.u1, K.u1, mul(K.u2, K.u2)));
  const T EK = fma(K.p, igm, mul(mul(half, K.r), kK));
  const T mK = mul(K.r, K.un);
  const T SK = sel(left, SL, SR), S = sel(left, min(SL, zero), max(SR, zero));
  const T dK = sel(left, dL, dR), qK = sel(left, qL, qR);
  const T gK = rcp(sel(ne0(S), sub(SK, SM), one));  // S' = 0: star terms vanish, keep this finite
  F[0] = fma(S, sub(mul(qK, gK), K.r), mK);
  F[1] = fma(S, fma(mul(qK, gK), SM, neg(mK)), fma(mK, K.un, K.p));
  F[2] = mul(K.u1, F[0]);
  F[3] = mul(K.u2, F[0]);
  const T Es = mul(gK, fma(sub(SM, K.un), fma(qK, SM, K.p), mul(dK, EK)));
  F[4] = fma(S, sub(Es, EK), mul(K.un, add(EK, K.p)));
}

// MUSCL face states of one cell along one direction: lo = P - s/2 (state on its - face),
// hi = P + s/2 (state on its + face), with the minmod slope s of (P - Pm, Pp - P) when the
// slope test passed, s = 0 otherwise (src/air_cfd.js:213-220).  Unrotated order.
__device__ __forceinline__ void face_states(const float Pm[5], const float P[5], const float Pp[5], bool ok,
                                            float lo[5], float hi[5]) {
#pragma unroll
  for (int c = 0; c < 5; c++) {
    const float a = P[c] - Pm[c], b = Pp[c] - P[c];
    const float s = ok ? minmod(a, b) : 0.f;
    lo[c] = fmaf(-0.5f, s, P[c]);
    hi[c] = fmaf(0.5f, s, P[c]);
  }
}

__device__ __forceinline__ PrimV<float> rotv(const float P[5], int d) {
  if (d == 0) return {P[0], P[1], P[2], P[3], P[4]};
  if (d == 1) return {P[0], P[2], P[1], P[3], P[4]};
  return {P[0], P[3], P[1], P[2], P[4]};
}

__device__ __forceinline__ PrimV<float2> pack(const PrimV<float>& a, const PrimV<float>& b) {
  return {make_float2(a.r, b.r), make_float2(a.un, b.un), make_float2(a.u1, b.u1), make_float2(a.u2, b.u2),
          make_float2(a.p, b.p)};
}

__device__ __forceinline__ bool nonpositive(const float L[5], const float R[5]) {
  return L[0] <= 0.f || L[4] <= 0.f || R[0] <= 0.f || R[4] <= 0.f;
}

// Rotated-frame flux back to (mass, x-, y-, z-momentum, energy).
__device__ __forceinline__ void unrotv(const float F[5], int d, float o[5]) {
  o[0] = F[0]; o[4] = F[4];
  if (d == 0) { o[1] = F[1]; o[2] = F[2]; o[3] = F[3]; }
  else if (d == 1) { o[1] = F[2]; o[2] = F[1]; o[3] = F[3]; }
  else { o[1] = F[2]; o[2] = F[3]; o[3] = F[1]; }
}

}  // namespace v
}  // namespace a3d
