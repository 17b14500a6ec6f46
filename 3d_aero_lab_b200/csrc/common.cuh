// common.cuh - shared definitions of libaero3d: status handling, device constants.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include "../../include/aero3d.h"

namespace a3d {

// Per-thread message of the last failure (returned by a3d_last_error()).
void set_error(const char* fmt, ...);
void clear_error();

// CUDA call wrapper: on failure record "<call> @ file:line: <cuda message>" and return.
#define A3D_CUDA(call)                                                                      \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) {                                                                \
      ::a3d::set_error("%s @ %s:%d: %s", #call, __FILE__, __LINE__, cudaGetErrorString(e_)); \
      return (e_ == cudaErrorMemoryAllocation) ? A3D_ERR_NOMEM : A3D_ERR_CUDA;              \
    }                                                                                       \
  } while (0)

#define A3D_TRY(expr)           \
  do {                          \
    int rc_ = (expr);           \
    if (rc_ != A3D_OK) return rc_; \
  } while (0)

#define A3D_ARG(cond, msg)                                          \
  do {                                                              \
    if (!(cond)) { ::a3d::set_error("bad argument: %s", msg); return A3D_ERR_ARG; } \
  } while (0)

// Makes `device` current; A3D_ERR_NODEVICE if no CUDA device is visible.
int use_device(int device);

constexpr double kGamma = 1.4;                       // src/air_cfd.js:11
constexpr double kPi = 3.141592653589793;
constexpr double kDeg = kPi / 180;                   // src/field.js:7

// Cell type codes (src/air_cfd.js:48): 0 fluid, 1 solid, 3 inlet sink, 4 bypass jet, 5 core jet.
// Inside the solver the low 3 bits of the per-cell code byte hold the type; 6 and 7 mark
// far-field and symmetry-mirror ghost cells of a tile.
enum : uint8_t { T_FLUID = 0, T_SOLID = 1, T_SINK = 3, T_JETB = 4, T_JETC = 5, T_GHOST = 6, T_MIRROR = 7 };
// Code byte: bits 0-2 type, bit 3/4/5 MUSCL slope allowed in x/y/z (static part of the
// test at src/air_cfd.js:214), bit 6 "irregular" (phi != 1 or a +face aperture != 1),
// bit 7 "baffle" (this cell's or the lower cell's +z face carries a baffle slope).
enum : uint8_t { C_OKX = 8, C_OKY = 16, C_OKZ = 32, C_IRR = 64, C_BAF = 128 };

inline long round_up(long v, long m) { return (v + m - 1) / m * m; }

}  // namespace a3d
