// tma_ring.cuh - the plane ring shared by the TMA-fed stage kernels.
//
// A CTA owning a 32 x 8 column tile keeps NSLOT shared-memory slots; plane p of its z run
// [k0, k1) lives in slot (p - k0 + 2) mod NSLOT.  Each slot holds one 40 x 12 x 5-component
// state box (x from i0-4, y from j0-2) and one 64 x 12 code box (x from i0-16), both loaded
// by `cp.async.bulk.tensor` completing on the slot's mbarrier.
#pragma once
#include "flux.cuh"
#include "solver.cuh"
#include "tma.cuh"

namespace a3d {
namespace ring {

constexpr int TX = 32, TY = 8, HX = TX + 4, HY = TY + 4;
constexpr int QBX = 40;  // state box width: x from i0-4 (16-byte aligned start)
constexpr int CBX = 64;  // code box width: x from i0-16
constexpr int NSLOT = 4;
constexpr uint32_t kQBytes = 5 * HY * QBX * 4, kCBytes = HY * CBX;
// A tiled TMA copy needs its innermost coordinate times the element size to be a multiple of
// 16 bytes.  Tiles start at i0 = bx * TX, so the state box at x = i0 - 4 (float) and the code
// box at x = i0 - 16 (u8) are aligned whenever TX is a multiple of 16.
static_assert(TX % 16 == 0, "TMA box x origins must stay 16-byte aligned");
static_assert((QBX * 4) % 16 == 0 && CBX % 16 == 0, "TMA box rows must be whole 16-byte units");
static_assert(kQBytes % 16 == 0 && kCBytes % 16 == 0, "TMA transaction sizes must be 16-byte multiples");

struct __align__(128) Slot {
  float Q[5][HY][QBX];  // conservative state of one plane
  uint8_t C[HY][CBX];   // codes of that plane
};



// Primitive state and code of cell (i, j) of a resident plane k, with the ghost rules of
// src/air_cfd.js:205-210 (far field outside x, z and +y; mirror with v negated below y = 0).
__device__ __forceinline__ uint8_t slot_cell(const StageArgs& a, const Slot& s, int i, int j, int k, int i0, int j0,
                                             float P[5]) {
  // Converted without branches, then overridden by selects: for every cell a tile reads (its
  // columns and the 2-cell halo) the slot indices below stay inside the slot, and whatever a
  // ghost's slot position holds (another plane, or nothing loaded) is replaced.
  const bool ghost = i < 0 || i >= a.NX || k < 0 || k >= a.NZ || j >= a.NY;
  const bool mirror = j < 0;
  const int y = (mirror ? -1 - j : j) - j0 + 2, xq = i - i0 + 4;
  const uint8_t c = s.C[y][i - i0 + 16];
  const int t = c & 7;
  cons_to_prim(s.Q[0][y][xq], s.Q[1][y][xq], s.Q[2][y][xq], s.Q[3][y][xq], s.Q[4][y][xq], P);
  if (!ghost && t >= T_SINK) {  // fixed-state cell (rare)
#pragma unroll
    for (int v = 0; v < 5; v++) P[v] = a.Pfix[t - T_SINK][v];
  }
#pragma unroll
  for (int v = 0; v < 5; v++) P[v] = ghost ? a.Pff[v] : P[v];
  P[2] = (mirror && !ghost) ? -P[2] : P[2];
  return ghost ? (uint8_t)T_GHOST : mirror ? (uint8_t)T_MIRROR : c;
}

// Slot of plane p for a CTA whose run starts at k0 (the ring starts with plane k0-2), and the
// mbarrier phase parity of that use of the slot.
__device__ __forceinline__ int slot_of(int p, int k0) { return (p - k0 + 2) & (NSLOT - 1); }
__device__ __forceinline__ uint32_t parity_of(int p, int k0) { return ((p - k0 + 2) / NSLOT) & 1; }

// Thread 0 queues plane p into its slot: one state box and one code box, or a bare arrive
// when the plane lies outside the domain (its cells are then all far-field ghosts).
template <class Smem>
__device__ __forceinline__ void issue_plane(Smem& S, const CUtensorMap* tmQ, const CUtensorMap* tmC,
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

// A wait ran out: flag the error for the host and wait (bounded) for the copies this CTA
// still has in flight, so that none lands in shared memory after the CTA has left.
template <class Smem>
__device__ void drain(Smem& S, const StageArgs& a, int k0, int first_pending, int last_issued) {
  if (threadIdx.x != 0) return;
  atomicOr(a.err, 1);
  for (int p = first_pending; p <= last_issued; p++) mbar_wait(&S.bar[slot_of(p, k0)], parity_of(p, k0));
}


}  // namespace ring
}  // namespace a3d
