// flux.cuh - FP32 device arithmetic of the Euler step: primitives, minmod MUSCL
// reconstruction and the HLLC flux (src/air_cfd.js:169-196, CFD3_FS 276-295).
//
// Faces are evaluated in a rotated frame: `un` is the velocity component normal to the
// face, `u1`, `u2` the two tangential ones.  The HLLC formulas of the reference are
// symmetric in the tangential components, so the rotation changes no arithmetic.
#pragma once
#include <cuda_runtime.h>

namespace a3d {

constexpr float kG = 1.4f;
constexpr float kGm = 1.4f - 1.0f;  // gamma - 1 as the float32 shader forms it

struct Prim {
  float r, un, u1, u2, p;
};

// Conservative -> primitive with the reference's floors rho >= 1e-6, p >= 1e-7
// (cfdPrim5, src/air_cfd.js:169); output in the unrotated order (rho, u, v, w, p).
__device__ __forceinline__ void cons_to_prim(float a0, float a1, float a2, float a3, float a4, float o[5]) {
  const float r = fmaxf(a0, 1e-6f), ir = 1.0f / r;
  const float u = a1 * ir, v = a2 * ir, w = a3 * ir;
  o[0] = r; o[1] = u; o[2] = v; o[3] = w;
  o[4] = fmaxf(kGm * (a4 - 0.5f * r * (u * u + v * v + w * w)), 1e-7f);
}

// mmod (src/air_cfd.js:196): 0 when a and b differ in sign, else the one nearer zero.
// `min.xorsign.abs` gives min(|a|, |b|) with the sign bit of a XOR b: negative exactly when the
// signs differ, so max(., 0) zeroes that case and copysign restores a's sign otherwise.  Three
// instructions, the same value as the reference's branch form.
__device__ __forceinline__ float minmod(float a, float b) {
  float m;
  asm("min.xorsign.abs.f32 %0, %1, %2;" : "=f"(m) : "f"(a), "f"(b));
  return copysignf(fmaxf(m, 0.f), a);
}

// Rotate (rho, u, v, w, p) so that component d of the velocity becomes `un`.
__device__ __forceinline__ Prim rot(const float P[5], int d) {
  Prim o;
  o.r = P[0]; o.p = P[4];
  if (d == 0) { o.un = P[1]; o.u1 = P[2]; o.u2 = P[3]; }
  else if (d == 1) { o.un = P[2]; o.u1 = P[1]; o.u2 = P[3]; }
  else { o.un = P[3]; o.u1 = P[1]; o.u2 = P[2]; }
  return o;
}

// HLLC flux with Davis wave-speed estimates (cfdHLLC, src/air_cfd.js:179-195).
// Output: mass, normal momentum, tangential momenta, energy.
// The star-region flux is the reference's, rearranged to need two divisions instead of four:
// with d = S - u_K, q = rho_K d (both already formed for S_M) and g = 1/(S - S_M),
//   rho* = q g,   F_t = v_t F_mass   (m v + S (rho* v - rho v) = v (m + S (rho* - rho))),
//   E*   = rho* (E/rho + (S_M - u)(S_M + p/q)) = g (d E + (S_M - u)(q S_M + p)).
// The supersonic cases need no branch: F = F_K + S' (U*_K - U_K) with S' = min(S_L, 0) on the
// left of the contact and max(S_R, 0) on its right is the upwind state flux F_K exactly when
// the fan is supersonic (S' = 0 makes every star term 0 * finite) and the star flux otherwise.
// Sound speeds as g p rsqrt(g p rho).  Same values up to float32 rounding.
__device__ __forceinline__ void hllc(const Prim& L, const Prim& R, float F[5]) {
  const float gL = kG * L.p, gR = kG * R.p;
  const float aL = gL * rsqrtf(gL * L.r), aR = gR * rsqrtf(gR * R.r);
  const float SL = fminf(L.un - aL, R.un - aR), SR = fmaxf(L.un + aL, R.un + aR);
  const float dL = SL - L.un, dR = SR - R.un;
  const float qL = L.r * dL, qR = R.r * dR;
  const float SM = __fdividef(R.p - L.p + qL * L.un - qR * R.un, qL - qR);
  const bool left = SM >= 0.f;
  const float rK = left ? L.r : R.r, uK = left ? L.un : R.un, v1 = left ? L.u1 : R.u1, v2 = left ? L.u2 : R.u2;
  const float pK = left ? L.p : R.p;
  const float EK = pK * (1.0f / kGm) + 0.5f * rK * (uK * uK + v1 * v1 + v2 * v2);  // total energy, side K only
  const float S = left ? fminf(SL, 0.f) : fmaxf(SR, 0.f);
  const float d = left ? dL : dR, q = left ? qL : qR;
  // where S' = 0 the star terms are multiplied away; keep their divisor finite there
  const float g = __fdividef(1.0f, S != 0.f ? (left ? SL : SR) - SM : 1.f);
  const float m = rK * uK;
  F[0] = m + S * (q * g - rK);
  F[1] = m * uK + pK + S * (q * g * SM - m);
  F[2] = v1 * F[0];
  F[3] = v2 * F[0];
  F[4] = uK * (EK + pK) + S * (g * (d * EK + (SM - uK) * (q * SM + pK)) - EK);
}

// Flux from reconstructed face states L, R of the cells b (left) and c (right).
//
// The reference falls back to first order (L = b, R = c) when a reconstructed density or
// pressure is not positive (src/air_cfd.js:221).  Here that can never happen, so the test is
// left out and the fluxes are the same bit for bit:
//   * every primitive state a face reads has density >= 1e-6 and pressure >= 1e-7: cell values
//     through cons_to_prim's floors, far-field and fixed states through the same floors on the
//     host (prim_of in solver.cu), mirror ghosts are cell values with v negated;
//   * a minmod-limited state is b + s/2 with s = 0, or s of the sign of both differences and no
//     larger than |c - b|; it therefore lies between b and (b + c) / 2 > 0, and its float32
//     value, rounded from at least (b + c) / 2 - b * 2^-25, stays positive;
//   * with NaN inputs the reference's comparisons are false as well.
__device__ __forceinline__ void face_flux_lr(const Prim& L, const Prim& R, const Prim&, const Prim&, float F[5]) {
  hllc(L, R, F);
}

// Flux through the face between cells b (left) and c (right) along one direction, with the
// neighbours a (left of b) and e (right of c).  okL/okR: the slope test at b and c passed
// (three fluid cells and both faces fully open, src/air_cfd.js:213-216).  The reference's
// first-order fallback (src/air_cfd.js:221) cannot fire here (face_flux_lr says why).
__device__ __forceinline__ void face_flux(const Prim& a, const Prim& b, const Prim& c, const Prim& e, bool okL,
                                          bool okR, float F[5]) {
  // Branch-free: the half-slope factor is 0 where the slope test failed, so the state is the
  // cell value itself (b + 0 * s); the slopes of neighbouring finite states are finite.
  const float hL = okL ? 0.5f : 0.f, hR = okR ? -0.5f : 0.f;
  Prim L, R;
  L.r = fmaf(hL, minmod(b.r - a.r, c.r - b.r), b.r);
  L.un = fmaf(hL, minmod(b.un - a.un, c.un - b.un), b.un);
  L.u1 = fmaf(hL, minmod(b.u1 - a.u1, c.u1 - b.u1), b.u1);
  L.u2 = fmaf(hL, minmod(b.u2 - a.u2, c.u2 - b.u2), b.u2);
  L.p = fmaf(hL, minmod(b.p - a.p, c.p - b.p), b.p);
  R.r = fmaf(hR, minmod(c.r - b.r, e.r - c.r), c.r);
  R.un = fmaf(hR, minmod(c.un - b.un, e.un - c.un), c.un);
  R.u1 = fmaf(hR, minmod(c.u1 - b.u1, e.u1 - c.u1), c.u1);
  R.u2 = fmaf(hR, minmod(c.u2 - b.u2, e.u2 - c.u2), c.u2);
  R.p = fmaf(hR, minmod(c.p - b.p, e.p - c.p), c.p);
  face_flux_lr(L, R, b, c, F);
}

// Scatter a rotated-frame flux back to (mass, x-, y-, z-momentum, energy).
__device__ __forceinline__ void unrot(const float F[5], int d, float o[5]) {
  o[0] = F[0]; o[4] = F[4];
  if (d == 0) { o[1] = F[1]; o[2] = F[2]; o[3] = F[3]; }
  else if (d == 1) { o[1] = F[2]; o[2] = F[1]; o[3] = F[3]; }
  else { o[1] = F[2]; o[2] = F[3]; o[3] = F[1]; }
}

}  // namespace a3d
