// solver.cu - the SSP-RK2 cut-cell Euler solver object (CfdCPU / CfdGPU, src/air_cfd.js:157-438).
//
// State: three structure-of-arrays float32 buffers Q, S1, B (rho, rho*u, rho*v, rho*w, E),
// each component a [NZ][NY][NXp] array with the row pitch NXp = NX rounded up to 16 (the
// alignment TMA tiles need).  One iteration is two stage launches:
//   S1 = Q + dt R(Q)                         (stage 1, dt from Q)
//   B  = 0.5 Q + 0.5 (S1 + dt R(S1))         (stage 2, dt again from Q)
// followed by a buffer rotation Q <-> B (src/air_cfd.js:252-258).  dt is recomputed from
// the base state Q in both stages, as the reference's shader does (CFD3_FS :357-359); it is
// the value CfdCPU stores in stage 1 and reuses.
//
// Three stage kernels are built:
//   KERNEL_CELL - one thread per cell, six faces per cell, the reference's structure (here);
//   KERNEL_TMA  - CTA tile of 32 x 8 columns marching in z, every face flux computed once per
//                 tile, planes staged by a TMA ring (stage_tma.cuh);
//   KERNEL_PAIR - the same marching over 32 x 16 columns, each thread two x-adjacent cells in
//                 packed f32x2 arithmetic (stage_pair.cuh), the default.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include "flux.cuh"
#include "solver.cuh"
#include "store.cuh"

namespace a3d {

namespace {

// ----------------------------------------------------------------------------------------
// per-cell codes: type, static slope-test bits, irregular and baffle flags
// ----------------------------------------------------------------------------------------
__global__ void k_codes(int NX, int NY, int NZ, int NXp, const uint8_t* t, const float* phi, const float* ap0,
                        const float* ap1, const float* ap2, const float* ap3, uint8_t* code) {
  const long NXY = (long)NX * NY, N = NXY * NZ;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < N; q += (long)gridDim.x * blockDim.x) {
    const int i = (int)(q % NX), j = (int)((q / NX) % NY), k = (int)(q / NXY);
    uint8_t c = t[q] & 7;
    auto fluid = [&](long qq) { return t[qq] == T_FLUID; };
    // slope allowed at this cell along d: both neighbours in the domain and fluid, this cell
    // fluid, both faces fully open (src/air_cfd.js:214; out-of-domain ghosts are never fluid)
    if (t[q] == T_FLUID) {
      if (i > 0 && i + 1 < NX && fluid(q - 1) && fluid(q + 1) && ap0[q - 1] == 1.f && ap0[q] == 1.f) c |= C_OKX;
      if (j > 0 && j + 1 < NY && fluid(q - NX) && fluid(q + NX) && ap1[q - NX] == 1.f && ap1[q] == 1.f) c |= C_OKY;
      if (k > 0 && k + 1 < NZ && fluid(q - NXY) && fluid(q + NXY) && ap2[q - NXY] == 1.f && ap2[q] == 1.f) c |= C_OKZ;
    }
    if (phi[q] != 1.f || ap0[q] != 1.f || ap1[q] != 1.f || ap2[q] != 1.f) c |= C_IRR;
    if (ap3[q] != 0.f || (k > 0 && ap3[q - NXY] != 0.f)) c |= C_BAF;
    code[((long)k * NY + j) * NXp + i] = c;
  }
}

// Local time step of every fluid cell from a state (the stage kernels' arithmetic: rsqrt sound
// speed, reciprocal sizes); 0 for the other cells, as the reference's shader leaves them.
__global__ void k_local_dt(StageArgs a, const float* __restrict__ Q, float* __restrict__ dt) {
  const long NXY = (long)a.NX * a.NY, N = NXY * a.NZ;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < N; q += (long)gridDim.x * blockDim.x) {
    const int i = (int)(q % a.NX), j = (int)((q / a.NX) % a.NY), k = (int)(q / NXY);
    const long qp = ((long)k * a.NY + j) * a.NXp + i;
    float v = 0.f;
    if ((a.code[qp] & 7) == T_FLUID) {
      float P[5];
      cons_to_prim(Q[qp], Q[a.Np + qp], Q[2 * a.Np + qp], Q[3 * a.Np + qp], Q[4 * a.Np + qp], P);
      const float ph = (a.code[qp] & C_IRR) ? a.phi[q] : 1.f;
      const float gp = kG * P[4], as = gp * rsqrtf(gp * P[0]);
      v = a.cfl * fmaxf(ph, 0.25f) /
          ((fabsf(P[1]) + as) * a.rXd[i] + (fabsf(P[2]) + as) * a.rYd[j] + (fabsf(P[3]) + as) * a.rZd[k]);
    }
    dt[q] = v;
  }
}

__global__ void k_fill(float* Q, long Np, float f0, float f1, float f2, float f3, float f4) {
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < Np; q += (long)gridDim.x * blockDim.x) {
    Q[q] = f0; Q[Np + q] = f1; Q[2 * Np + q] = f2; Q[3 * Np + q] = f3; Q[4 * Np + q] = f4;
  }
}

// ----------------------------------------------------------------------------------------
// KERNEL_CELL: one thread per cell, the reference's per-cell structure.
// ----------------------------------------------------------------------------------------

// Primitive state of the stencil cell at (i, j, k) with the reference's ghost rules
// (src/air_cfd.js:205-210): far field beyond the domain in x, z and +y, symmetry mirror
// (v negated) below y = 0, fixed-state substitution for types 3-5.  Returns the type.
__device__ __forceinline__ int stencil_prim(const StageArgs& a, int i, int j, int k, float P[5]) {
  if (i < 0 || i >= a.NX || k < 0 || k >= a.NZ || j >= a.NY) {
    for (int v = 0; v < 5; v++) P[v] = a.Pff[v];
    return T_GHOST;
  }
  const bool mirror = j < 0;
  const int jj = mirror ? -1 - j : j;
  const long q = ((long)k * a.NY + jj) * a.NXp + i;
  const int t = a.code[q] & 7;
  if (t >= T_SINK) { for (int v = 0; v < 5; v++) P[v] = a.Pfix[t - T_SINK][v]; }
  else cons_to_prim(a.Qin[q], a.Qin[a.Np + q], a.Qin[2 * a.Np + q], a.Qin[3 * a.Np + q], a.Qin[4 * a.Np + q], P);
  if (mirror) { P[2] = -P[2]; return T_MIRROR; }
  return t;
}

__global__ void __launch_bounds__(256) k_stage_cell(StageArgs a) {
  const long NXY = (long)a.NX * a.NY, N = NXY * a.NZ;
  const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (q >= N) return;
  const int i = (int)(q % a.NX), j = (int)((q / a.NX) % a.NY), k = (int)(q / NXY);
  if (k < a.kb || k >= a.ke) return;  // not one of this solver's own planes
  const long qp = ((long)k * a.NY + j) * a.NXp + i;  // padded state/code index
  const uint8_t cq = a.code[qp];
  const int t = cq & 7;
  const long Np = a.Np;
  if (t != T_FLUID) {  // src/air_cfd.js:242
    float o[5];
    if (t >= T_SINK) for (int c = 0; c < 5; c++) o[c] = a.Ufix[t - T_SINK][c];
    else for (int c = 0; c < 5; c++) o[c] = a.B[c * Np + qp];
    store_out(a, a.Out, qp, k, o);
    return;
  }
  float Pc[5];
  cons_to_prim(a.Qin[qp], a.Qin[Np + qp], a.Qin[2 * Np + qp], a.Qin[3 * Np + qp], a.Qin[4 * Np + qp], Pc);
  const float pC = Pc[4];
  float R[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  const float* apd[3] = {a.ap0, a.ap1, a.ap2};
  const long st[3] = {1, a.NX, NXY};
  const int ic[3] = {i, j, k}, nd[3] = {a.NX, a.NY, a.NZ};
  const float rh[3] = {a.rXd[i], a.rYd[j], a.rZd[k]};
  float Aface[3][2];
  for (int d = 0; d < 3; d++) {
    Prim P[5];
    bool fl[5];
    for (int m = -2; m <= 2; m++) {
      float W[5];
      const int ii = i + (d == 0 ? m : 0), jj = j + (d == 1 ? m : 0), kk = k + (d == 2 ? m : 0);
      const int tt = (m == 0) ? T_FLUID : stencil_prim(a, ii, jj, kk, W);
      if (m == 0) for (int v = 0; v < 5; v++) W[v] = Pc[v];
      P[m + 2] = rot(W, d);
      fl[m + 2] = tt == T_FLUID;
    }
    float A[4];
    for (int m = -2; m <= 1; m++) {
      const int c = ic[d] + m;
      A[m + 2] = (c < 0 || c >= nd[d]) ? 1.f : apd[d][q + m * st[d]];
    }
    bool ok[3];
    for (int x = 0; x < 3; x++)
      ok[x] = a.order2 && fl[x] && fl[x + 1] && fl[x + 2] && A[x] == 1.f && A[x + 1] == 1.f;
    float F[5], G[5];
    if (A[2] > 0.f) {  // + face
      face_flux(P[1], P[2], P[3], P[4], ok[1], ok[2], F);
      unrot(F, d, G);
      for (int c = 0; c < 5; c++) R[c] -= A[2] * G[c] * rh[d];
    }
    if (A[1] > 0.f) {  // - face
      face_flux(P[0], P[1], P[2], P[3], ok[0], ok[1], F);
      unrot(F, d, G);
      for (int c = 0; c < 5; c++) R[c] += A[1] * G[c] * rh[d];
    }
    R[1 + d] += pC * (A[2] - A[1]) * rh[d];  // wall-pressure source
    Aface[d][0] = A[1];
    Aface[d][1] = A[2];
  }
  if (cq & C_BAF) {  // baffle transpiration w = u dz/dx (src/air_cfd.js:226-233)
    const float sUp = a.ap3[q], sDn = k > 0 ? a.ap3[q - NXY] : 0.f;
    if (sUp != 0.f || sDn != 0.f) {
      const float r = Pc[0], u = Pc[1], v = Pc[2], w = Pc[3];
      const float Hh = (pC / kGm + 0.5f * r * (u * u + v * v + w * w) + pC) / r;
      const float m = (sDn != 0.f ? (1.f - Aface[2][0]) * r * u * sDn : 0.f) - (sUp != 0.f ? (1.f - Aface[2][1]) * r * u * sUp : 0.f);
      const float mh = m * rh[2];
      R[0] += mh; R[1] += mh * u; R[2] += mh * v; R[3] += mh * w; R[4] += mh * Hh;
    }
  }
  const float ph = (cq & C_IRR) ? a.phi[q] : 1.f;
  if (ph != 1.f) { const float iph = 1.f / ph; for (int c = 0; c < 5; c++) R[c] *= iph; }
  // local time step from the base state (src/air_cfd.js:243, CFD3_FS :357-359)
  float Pb[5];
  if (a.wa == 0.f) { for (int v = 0; v < 5; v++) Pb[v] = Pc[v]; }
  else cons_to_prim(a.B[qp], a.B[Np + qp], a.B[2 * Np + qp], a.B[3 * Np + qp], a.B[4 * Np + qp], Pb);
  const float as = sqrtf(kG * Pb[4] / Pb[0]);
  const float dt = a.cfl * fmaxf(ph, 0.25f) / ((fabsf(Pb[1]) + as) * rh[0] + (fabsf(Pb[2]) + as) * rh[1] + (fabsf(Pb[3]) + as) * rh[2]);
  float o[5];
  for (int c = 0; c < 5; c++) {
    const float qin = a.Qin[c * Np + qp];
    o[c] = (a.wa == 0.f) ? (qin + dt * R[c]) : (a.wa * a.B[c * Np + qp] + a.wb * (qin + dt * R[c]));
  }
  o[0] = fmaxf(o[0], 1e-4f);  // positivity clamps (src/air_cfd.js:247-249)
  const float ke = 0.5f * (o[1] * o[1] + o[2] * o[2] + o[3] * o[3]) / o[0];
  if (kGm * (o[4] - ke) < 1e-5f) o[4] = 1e-5f / kGm + ke;
  store_out(a, a.Out, qp, k, o);
}

int blocks_for(long work, int threads = 256) {
  return (int)std::max(1L, std::min((work + threads - 1) / threads, 148L * 64));
}

void prim_of(const double U[5], float P[5]) {  // cfdPrim5 in float64, rounded to float32
  const double r = std::max(U[0], 1e-6), u = U[1] / r, v = U[2] / r, w = U[3] / r;
  P[0] = (float)r; P[1] = (float)u; P[2] = (float)v; P[3] = (float)w;
  P[4] = (float)std::max((kGamma - 1) * (U[4] - 0.5 * r * (u * u + v * v + w * w)), 1e-7);
}

}  // namespace


void fill_stage_args(a3d_solver* s, StageArgs& a, const float* Qin, const float* B, float* Out, float wa, float wb) {
  a.Qin = Qin; a.B = B; a.Out = Out; a.Np = s->Np; a.NXp = s->NXp;
  a.code = s->code; a.phi = s->geo.phi; a.ap0 = s->geo.ap0; a.ap1 = s->geo.ap1; a.ap2 = s->geo.ap2; a.ap3 = s->geo.ap3;
  a.rXd = s->grid.rXd; a.rYd = s->grid.rYd; a.rZd = s->grid.rZd;
  a.NX = s->grid.NX; a.NY = s->grid.NY; a.NZ = s->grid.NZ;
  a.wa = wa; a.wb = wb; a.cfl = (float)s->cfl; a.order2 = s->order == 2;
  a.err = s->d_flag + 1;
  a.wait_limit = s->wait_limit;
  a.kb = s->own_k0;
  a.ke = s->own_k1;
  for (int sd = 0; sd < 2; sd++) {
    a.peer[sd] = nullptr;
    a.peer_np[sd] = 0;
    a.peer_k0[sd] = a.peer_k1[sd] = a.peer_dk[sd] = 0;
    a3d_solver* n = s->nbr[sd];
    if (!n || !Out) continue;
    // the neighbour's buffer of the role Out plays here; a neighbour that already finished
    // this iteration's stage 2 has swapped its B into its current state
    float* dst = Out == s->buf[s->iS1] ? n->buf[n->iS1]
               : Out == s->buf[s->iB] ? (n->it > s->it ? n->buf[n->iQ] : n->buf[n->iB]) : nullptr;
    if (!dst) continue;
    // own planes that the neighbour stores as halo planes: its planes outside its own range
    const int g0 = s->z_lo + s->own_k0, g1 = s->z_lo + s->own_k1;
    const int h0 = sd == 0 ? n->z_lo + n->own_k1 : n->z_lo, h1 = sd == 0 ? n->z_lo + n->grid.NZ : n->z_lo + n->own_k0;
    const int k0 = std::max(g0, h0), k1 = std::min(g1, h1);
    if (k0 >= k1) continue;
    a.peer[sd] = dst;
    a.peer_np[sd] = n->Np;
    a.peer_k0[sd] = k0 - s->z_lo;
    a.peer_k1[sd] = k1 - s->z_lo;
    a.peer_dk[sd] = s->z_lo - n->z_lo;
  }
  prim_of(s->F, a.Pff);
  for (int f = 0; f < 3; f++) {
    prim_of(s->fix[f], a.Pfix[f]);
    for (int c = 0; c < 5; c++) a.Ufix[f][c] = (float)s->fix[f][c];
  }
}

int launch_stage(a3d_solver* s, const StageArgs& a) {
  if (s->kernel == KERNEL_TMA || s->kernel == KERNEL_PAIR) {
    const int qin_buf = a.Qin == s->buf[0] ? 0 : a.Qin == s->buf[1] ? 1 : 2;
    if (s->kernel == KERNEL_PAIR) return launch_pair(s, a, qin_buf, a.wa != 0.f);
    return launch_tma(s, a, qin_buf, a.wa != 0.f);
  }
  k_stage_cell<<<(unsigned)((s->N + 255) / 256), 256, 0, s->st>>>(a);
  A3D_CUDA(cudaGetLastError());
  return A3D_OK;
}

int solver_finish_setup(a3d_solver* s) {
  const long N = s->N;
  s->NXp = (int)round_up(s->grid.NX, 16);
  s->Np = round_up((long)s->NXp * s->grid.NY * s->grid.NZ, 64);
  // the tiled stage kernels index cells and padded cells of one component in 32-bit integers
  A3D_ARG(s->Np < (1L << 31), "grid too large: more than 2^31 padded cells per component");
  A3D_CUDA(cudaMalloc(&s->state, 3 * 5 * s->Np * sizeof(float)));
  for (int b = 0; b < 3; b++) s->buf[b] = s->state + (long)b * 5 * s->Np;
  A3D_CUDA(cudaMemsetAsync(s->state, 0, 3 * 5 * s->Np * sizeof(float), s->st));
  A3D_CUDA(cudaMalloc(&s->code, round_up(s->Np, 256)));
  A3D_CUDA(cudaMemsetAsync(s->code, T_GHOST, round_up(s->Np, 256), s->st));
  k_codes<<<blocks_for(N), 256, 0, s->st>>>(s->grid.NX, s->grid.NY, s->grid.NZ, s->NXp, s->geo.t, s->geo.phi,
                                            s->geo.ap0, s->geo.ap1, s->geo.ap2, s->geo.ap3, s->code);
  A3D_CUDA(cudaGetLastError());
  A3D_CUDA(cudaMalloc(&s->d_red, 4096 * 8 * sizeof(double)));
  A3D_CUDA(cudaMallocHost(&s->h_red, 64 * sizeof(double)));
  A3D_CUDA(cudaMalloc(&s->d_flag, 16));
  A3D_CUDA(cudaMemsetAsync(s->d_flag, 0, 16, s->st));
  A3D_CUDA(cudaMalloc(&s->prevR, s->Np * sizeof(float)));
  s->own_k0 = 0;
  s->own_k1 = s->grid.NZ;
  A3D_CUDA(cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming));
  for (int c = 0; c < kMaxChunks; c++) {
    A3D_CUDA(cudaStreamCreateWithFlags(&s->cst[c], cudaStreamNonBlocking));
    for (int t = 0; t < 2; t++) A3D_CUDA(cudaEventCreateWithFlags(&s->cev[c][t], cudaEventDisableTiming));
  }
  A3D_TRY(build_force_list(s));
  A3D_TRY(make_tensor_maps(s));
  A3D_TRY(a3d_solver_set_kernel(s, s->kernel, 0));  // the automatic z run
  const double F0[5] = {1, 0, 0, 0, 1 / (kGamma * (kGamma - 1))};  // src/air_cfd.js:162
  for (int c = 0; c < 5; c++) { s->F[c] = F0[c]; s->fix[0][c] = s->fix[1][c] = s->fix[2][c] = F0[c]; }
  A3D_CUDA(cudaStreamSynchronize(s->st));
  return A3D_OK;
}

}  // namespace a3d

using namespace a3d;

namespace {

int new_solver(int device, const int32_t dims[3], const double* xf, const double* yf, const double* zf,
               a3d_solver** out) {
  A3D_ARG(out && dims && xf && yf && zf, "null pointer");
  A3D_ARG(dims[0] >= 1 && dims[1] >= 2 && dims[2] >= 1, "grid dims (NY >= 2 for the symmetry mirror)");
  A3D_ARG((double)dims[0] * dims[1] * dims[2] < 2.0e9, "grid too large");
  A3D_TRY(use_device(device));
  a3d_solver* s = new a3d_solver();
  cudaGetDevice(&s->device);
  if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete s;
    set_error("cudaStreamCreate failed");
    return A3D_ERR_CUDA;
  }
  if (cudaEventCreateWithFlags(&s->ev, cudaEventDisableTiming) != cudaSuccess) {
    cudaStreamDestroy(s->st);
    delete s;
    set_error("cudaEventCreate failed");
    return A3D_ERR_CUDA;
  }
  s->N = (long)dims[0] * dims[1] * dims[2];
  int rc = grid_upload(dims, xf, yf, zf, s->st, s->grid);
  if (rc == A3D_OK) rc = geom_alloc(s->N, s->geo);
  if (rc != A3D_OK) { a3d_solver_destroy(s); return rc; }
  *out = s;
  return A3D_OK;
}

}  // namespace

extern "C" int a3d_solver_create(const int32_t dims[3], const double* xf, const double* yf, const double* zf,
                                 const uint8_t* t, const float* phi, const float* ap0, const float* ap1,
                                 const float* ap2, const float* ap3, int device, a3d_solver** out) {
  clear_error();
  A3D_ARG(t && phi && ap0 && ap1 && ap2 && ap3, "null geometry array");
  a3d_solver* s = nullptr;
  A3D_TRY(new_solver(device, dims, xf, yf, zf, &s));
  const long N = s->N;
  int rc = A3D_OK;
  cudaError_t e = cudaMemcpy(s->geo.t, t, N, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(s->geo.phi, phi, N * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(s->geo.ap0, ap0, N * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(s->geo.ap1, ap1, N * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(s->geo.ap2, ap2, N * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(s->geo.ap3, ap3, N * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) { set_error("geometry upload: %s", cudaGetErrorString(e)); rc = A3D_ERR_CUDA; }
  if (rc == A3D_OK) rc = solver_finish_setup(s);
  if (rc != A3D_OK) { a3d_solver_destroy(s); return rc; }
  *out = s;
  return A3D_OK;
}

extern "C" int a3d_solver_create_shape(const a3d_shape* shape, const int32_t dims[3], const double* xf,
                                       const double* yf, const double* zf, double h, double delta_deg, int device,
                                       a3d_solver** out) {
  clear_error();
  A3D_ARG(shape, "null shape");
  a3d_solver* s = nullptr;
  A3D_TRY(new_solver(device, dims, xf, yf, zf, &s));
  int rc = geom_build_device(*shape, s->grid, h, delta_deg, s->geo, s->st, nullptr, nullptr);
  if (rc == A3D_OK) rc = solver_finish_setup(s);
  if (rc != A3D_OK) { a3d_solver_destroy(s); return rc; }
  *out = s;
  return A3D_OK;
}

// Planes [z_lo, z_hi) of the case that a3d_solver_create_shape would build on the full grid
// `dims`: the geometry is built for the full grid in temporary device memory, and the slab
// solver keeps its planes' geometry, the z faces zf[z_lo .. z_hi] and cells of its own.  Every
// slab array is the full one's, cut: a slab holding two halo planes beyond the planes it owns
// reproduces the full case's face fluxes on its owned planes once the halos are exchanged.
extern "C" int a3d_solver_create_shape_slab(const a3d_shape* shape, const int32_t dims[3], const double* xf,
                                            const double* yf, const double* zf, double h, double delta_deg,
                                            int32_t z_lo, int32_t z_hi, int device, a3d_solver** out) {
  clear_error();
  A3D_ARG(shape && dims && zf, "null pointer");
  A3D_ARG(0 <= z_lo && z_lo < z_hi && z_hi <= dims[2], "slab planes must satisfy 0 <= z_lo < z_hi <= NZ");
  const int32_t sd[3] = {dims[0], dims[1], z_hi - z_lo};
  a3d_solver* s = nullptr;
  A3D_TRY(new_solver(device, sd, xf, yf, zf + z_lo, &s));
  s->z_lo = z_lo;
  GridDev gfull;
  GeomDev full;
  const long NXY = (long)dims[0] * dims[1], Nfull = NXY * dims[2];
  int rc = grid_upload(dims, xf, yf, zf, s->st, gfull);
  if (rc == A3D_OK) rc = geom_alloc(Nfull, full);
  if (rc == A3D_OK) rc = geom_build_device(*shape, gfull, h, delta_deg, full, s->st, nullptr, nullptr);
  if (rc == A3D_OK) {
    const long o = (long)z_lo * NXY, n = s->N;
    cudaError_t e = cudaMemcpyAsync(s->geo.t, full.t + o, n, cudaMemcpyDeviceToDevice, s->st);
    const float* src[5] = {full.phi, full.ap0, full.ap1, full.ap2, full.ap3};
    float* dst[5] = {s->geo.phi, s->geo.ap0, s->geo.ap1, s->geo.ap2, s->geo.ap3};
    for (int a = 0; a < 5 && e == cudaSuccess; a++)
      e = cudaMemcpyAsync(dst[a], src[a] + o, n * sizeof(float), cudaMemcpyDeviceToDevice, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    if (e != cudaSuccess) { set_error("slab geometry: %s", cudaGetErrorString(e)); rc = A3D_ERR_CUDA; }
  }
  geom_free(full);
  grid_free(gfull);
  if (rc == A3D_OK) rc = solver_finish_setup(s);
  if (rc != A3D_OK) { a3d_solver_destroy(s); return rc; }
  *out = s;
  return A3D_OK;
}

extern "C" int a3d_solver_destroy(a3d_solver* s) {
  if (!s) return A3D_OK;
  cudaSetDevice(s->device);
  if (s->st) cudaStreamSynchronize(s->st);
  cudaFree(s->state);
  cudaFree(s->code);
  cudaFree(s->d_red);
  if (s->h_red) cudaFreeHost(s->h_red);
  cudaFree(s->d_flag);
  cudaFree(s->prevR);
  if (s->fl.block) cudaFree(s->fl.block);
  geom_free(s->geo);
  grid_free(s->grid);
  if (s->ev) cudaEventDestroy(s->ev);
  if (s->ev_fork) cudaEventDestroy(s->ev_fork);
  for (int c = 0; c < kMaxChunks; c++) {
    if (s->cst[c]) cudaStreamDestroy(s->cst[c]);
    for (int t = 0; t < 2; t++)
      if (s->cev[c][t]) cudaEventDestroy(s->cev[c][t]);
  }
  if (s->st) cudaStreamDestroy(s->st);
  delete s;
  return A3D_OK;
}

extern "C" int a3d_solver_dims(a3d_solver* s, int32_t dims[3], int64_t* n_cells) {
  clear_error();
  A3D_ARG(s, "null solver");
  if (dims) { dims[0] = s->grid.NX; dims[1] = s->grid.NY; dims[2] = s->grid.NZ; }
  if (n_cells) *n_cells = s->N;
  return A3D_OK;
}

extern "C" int a3d_solver_set_opt(a3d_solver* s, double cfl, int32_t order) {
  clear_error();
  A3D_ARG(s, "null solver");
  A3D_ARG(cfl > 0 && cfl < 10, "cfl");
  A3D_ARG(order == 1 || order == 2, "order must be 1 or 2");
  s->cfl = cfl;
  s->order = order;
  return A3D_OK;
}

extern "C" int a3d_solver_set_free(a3d_solver* s, const double F[5]) {
  clear_error();
  A3D_ARG(s && F, "null pointer");
  for (int c = 0; c < 5; c++) s->F[c] = F[c];
  return A3D_OK;
}

extern "C" int a3d_solver_set_fix(a3d_solver* s, const double fix[15]) {
  clear_error();
  A3D_ARG(s && fix, "null pointer");
  for (int c = 0; c < 15; c++) s->fix[c / 5][c % 5] = fix[c];
  return A3D_OK;
}

extern "C" int a3d_solver_reset(a3d_solver* s) {
  clear_error();
  A3D_ARG(s, "null solver");
  A3D_CUDA(cudaSetDevice(s->device));
  k_fill<<<blocks_for(s->Np), 256, 0, s->st>>>(s->buf[s->iQ], s->Np, (float)s->F[0], (float)s->F[1],
                                                (float)s->F[2], (float)s->F[3], (float)s->F[4]);
  A3D_CUDA(cudaGetLastError());
  s->it = 0;
  s->havePrev = false;
  s->prevIt = 0;
  return A3D_OK;
}

namespace {

// Number of pipelined z chunks a3d_solver_step uses: kernels 2 and 4 on a whole case only.  Automatic:
// four chunks from 0.8M cells up, where a stage takes long enough to hide the extra stream and
// event calls (measured: 4.1M-cell fighter 13.5 -> 15.1 G cell-updates/s, 1.0M-cell airliner
// 10.1 -> 11.2), none below (0.6M-cell interceptor 8.4 -> 8.1 with four).
int chunk_count(const a3d_solver* s) {
  if ((s->kernel != KERNEL_TMA && s->kernel != KERNEL_PAIR) || s->nbr[0] || s->nbr[1] || s->own_k0 != 0 ||
      s->own_k1 != s->grid.NZ)
    return 1;
  const int runs = (s->grid.NZ + s->march_kz - 1) / s->march_kz;
  const int K = s->chunks_req > 0 ? s->chunks_req : (s->N >= 800000 ? 4 : 1);
  return std::max(1, std::min(K, std::min(runs, kMaxChunks)));
}

// n iterations with the case cut into K z chunks of whole z runs (so every cell sees the same
// arithmetic as in one launch).  Chunk c's stage waits for the previous stage of chunks c-1 and
// c+1 only: a stage reads two planes beyond its chunk and writes inside it, so those are its
// only producers (read after write) and its only remaining readers (write after read).
int step_chunked(a3d_solver* s, int n, int K) {
  const int kz = s->march_kz, NZ = s->grid.NZ, runs = (NZ + kz - 1) / kz;
  int kb[kMaxChunks], ke[kMaxChunks];
  for (int c = 0; c < K; c++) {
    kb[c] = (c * runs / K) * kz;
    ke[c] = std::min(NZ, ((c + 1) * runs / K) * kz);
  }
  A3D_CUDA(cudaEventRecord(s->ev_fork, s->st));
  for (int c = 0; c < K; c++) A3D_CUDA(cudaStreamWaitEvent(s->cst[c], s->ev_fork, 0));
  bool first = true;
  for (int i = 0; i < n; i++) {
    float *Q = s->buf[s->iQ], *S1 = s->buf[s->iS1], *B = s->buf[s->iB];
    for (int stage = 0; stage < 2; stage++) {
      StageArgs a;
      if (stage == 0) fill_stage_args(s, a, Q, Q, S1, 0.f, 1.f);
      else fill_stage_args(s, a, S1, Q, B, 0.5f, 0.5f);
      const int qin_buf = a.Qin == s->buf[0] ? 0 : a.Qin == s->buf[1] ? 1 : 2;
      const int prev = stage ^ 1;
      for (int c = 0; c < K; c++) {
        if (!first) {
          if (c > 0) A3D_CUDA(cudaStreamWaitEvent(s->cst[c], s->cev[c - 1][prev], 0));
          if (c + 1 < K) A3D_CUDA(cudaStreamWaitEvent(s->cst[c], s->cev[c + 1][prev], 0));
        }
        a.kb = kb[c];
        a.ke = ke[c];
        if (s->kernel == KERNEL_PAIR) A3D_TRY(launch_pair(s, a, qin_buf, stage == 1, s->cst[c]));
        else A3D_TRY(launch_tma(s, a, qin_buf, stage == 1, s->cst[c]));
        A3D_CUDA(cudaEventRecord(s->cev[c][stage], s->cst[c]));
      }
      first = false;
    }
    std::swap(s->iQ, s->iB);
    s->it++;
  }
  for (int c = 0; c < K; c++) A3D_CUDA(cudaStreamWaitEvent(s->st, s->cev[c][1], 0));
  return A3D_OK;
}

}  // namespace

// Pipelined z chunks of a3d_solver_step (kernel 2): 0 = automatic (4 from 0.8M cells up, else 1),
// 1 = one launch per stage, 2..4 = that many chunks.  Results do not depend on it.
extern "C" int a3d_solver_set_chunks(a3d_solver* s, int32_t chunks) {
  clear_error();
  A3D_ARG(s, "null solver");
  A3D_ARG(chunks >= 0 && chunks <= kMaxChunks, "chunks must be 0 (automatic) or 1..4");
  s->chunks_req = chunks;
  return A3D_OK;
}

// The number of z chunks a3d_solver_step would use now (stage launches per stage).
extern "C" int a3d_solver_get_chunks(a3d_solver* s, int32_t* chunks) {
  clear_error();
  A3D_ARG(s && chunks, "null pointer");
  *chunks = chunk_count(s);
  return A3D_OK;
}

extern "C" int a3d_solver_step(a3d_solver* s, int32_t n) {
  clear_error();
  A3D_ARG(s, "null solver");
  A3D_ARG(n >= 0, "negative iteration count");
  A3D_ARG(s->phase == 0, "a lone stage 1 (a3d_solver_stage) is waiting for its stage 2");
  A3D_ARG(!s->nbr[0] && !s->nbr[1], "a slab with neighbours advances by a3d_solver_stage");
  A3D_CUDA(cudaSetDevice(s->device));
  const int K = chunk_count(s);
  if (K > 1 && n > 0) return step_chunked(s, n, K);
  StageArgs a1, a2;
  for (int i = 0; i < n; i++) {
    float *Q = s->buf[s->iQ], *S1 = s->buf[s->iS1], *B = s->buf[s->iB];
    fill_stage_args(s, a1, Q, Q, S1, 0.f, 1.f);
    A3D_TRY(launch_stage(s, a1));
    fill_stage_args(s, a2, S1, Q, B, 0.5f, 0.5f);
    A3D_TRY(launch_stage(s, a2));
    std::swap(s->iQ, s->iB);
    s->it++;
  }
  return A3D_OK;
}

// One RK stage of an iteration, for callers that exchange halo planes between the stages:
// which = 1 forms S1 = Q + dt R(Q); which = 2 forms B = Q/2 + (S1 + dt R(S1))/2, makes it the
// current state and counts the iteration.  The pair is the same work as a3d_solver_step(s, 1).
extern "C" int a3d_solver_stage(a3d_solver* s, int32_t which) {
  clear_error();
  A3D_ARG(s, "null solver");
  A3D_ARG(which == 1 || which == 2, "stage must be 1 or 2");
  A3D_ARG(which == s->phase + 1, which == 1 ? "stage 1 again before stage 2" : "stage 2 before stage 1");
  for (a3d_solver* n : s->nbr) {
    if (!n) continue;
    // the neighbour is at the same stage of the same iteration, before or after its own launch
    const bool ok = which == 1 ? n->it == s->it
                               : ((n->it == s->it && n->phase == 1) || (n->it == s->it + 1 && n->phase == 0));
    A3D_ARG(ok, "neighbour slabs out of step");
    A3D_ARG(s->kernel == KERNEL_CELL || s->kernel == KERNEL_TMA || s->kernel == KERNEL_PAIR,
            "halo push needs stage kernel 0, 2 or 4");
  }
  A3D_CUDA(cudaSetDevice(s->device));
  float *Q = s->buf[s->iQ], *S1 = s->buf[s->iS1], *B = s->buf[s->iB];
  StageArgs a;
  if (which == 1) {
    fill_stage_args(s, a, Q, Q, S1, 0.f, 1.f);
    A3D_TRY(launch_stage(s, a));
    s->phase = 1;
  } else {
    fill_stage_args(s, a, S1, Q, B, 0.5f, 0.5f);
    A3D_TRY(launch_stage(s, a));
    std::swap(s->iQ, s->iB);
    s->it++;
    s->phase = 0;
  }
  if (s->nbr[0] || s->nbr[1]) A3D_CUDA(cudaEventRecord(s->ev, s->st));
  return A3D_OK;
}

// Makes s's stage kernels also store the planes that its neighbours keep as halo planes
// straight into the neighbours' buffers (peer stores when they live on other devices), so
// that no copy is needed between stages.  lo / hi: the slabs below and above (either may be
// null).  Every slab of the split must be given its neighbours; afterwards a slab advances
// by a3d_solver_stage, with a3d_solver_sync_neighbors between the stages of all slabs.
// Kernels 0, 2 and 4 store only own planes and push; others are refused.
extern "C" int a3d_solver_set_neighbors(a3d_solver* s, a3d_solver* lo, a3d_solver* hi) {
  clear_error();
  A3D_ARG(s && s != lo && s != hi, "null or self neighbour");
  A3D_ARG(s->kernel == KERNEL_CELL || s->kernel == KERNEL_TMA || s->kernel == KERNEL_PAIR,
          "halo push needs stage kernel 0, 2 or 4");
  for (a3d_solver* n : {lo, hi}) {
    if (!n) continue;
    A3D_ARG(n->grid.NX == s->grid.NX && n->grid.NY == s->grid.NY, "neighbour differs in NX or NY");
    A3D_ARG(n->it == s->it && n->phase == 0 && s->phase == 0, "neighbours must be at the same iteration");
    if (n->device != s->device) {
      int can = 0;
      A3D_CUDA(cudaDeviceCanAccessPeer(&can, s->device, n->device));
      A3D_ARG(can, "no peer access between the slabs' devices");
      A3D_CUDA(cudaSetDevice(s->device));
      const cudaError_t e = cudaDeviceEnablePeerAccess(n->device, 0);
      if (e == cudaErrorPeerAccessAlreadyEnabled) cudaGetLastError();
      else A3D_CUDA(e);
    }
  }
  if (lo) A3D_ARG(lo->z_lo < s->z_lo, "lower neighbour must start below");
  if (hi) A3D_ARG(hi->z_lo > s->z_lo, "upper neighbour must start above");
  s->nbr[0] = lo;
  s->nbr[1] = hi;
  return A3D_OK;
}

// s's next stage waits until its neighbours' last stages (and their pushes into s) are done.
extern "C" int a3d_solver_sync_neighbors(a3d_solver* s) {
  clear_error();
  A3D_ARG(s, "null solver");
  A3D_CUDA(cudaSetDevice(s->device));
  for (a3d_solver* n : s->nbr)
    if (n) A3D_CUDA(cudaStreamWaitEvent(s->st, n->ev, 0));
  return A3D_OK;
}

namespace {
float* state_buffer(a3d_solver* s, int which) { return s->buf[which == 1 ? s->iS1 : s->iQ]; }
}  // namespace

// Copies planes [src_k0, src_k0 + nk) of src's current state (which = 0) or stage-1 state
// (which = 1) into planes [dst_k0, dst_k0 + nk) of dst's buffer of the same role: the halo
// exchange of a z-slab decomposition.  The two solvers must share NX and NY; they may live
// on different devices (peer copy).  Stream-ordered both ways: the copy runs on dst's stream
// after src's work so far, and src's later work waits for the copy.
extern "C" int a3d_solver_copy_planes(a3d_solver* dst, int32_t dst_k0, a3d_solver* src, int32_t src_k0, int32_t nk,
                                      int32_t which) {
  clear_error();
  A3D_ARG(dst && src && dst != src, "two distinct solvers");
  A3D_ARG(which == 0 || which == 1, "which: 0 current state, 1 stage-1 state");
  A3D_ARG(dst->grid.NX == src->grid.NX && dst->grid.NY == src->grid.NY, "solvers differ in NX or NY");
  A3D_ARG(nk >= 1 && src_k0 >= 0 && src_k0 + nk <= src->grid.NZ && dst_k0 >= 0 && dst_k0 + nk <= dst->grid.NZ,
          "plane range");
  const long plane = (long)src->grid.NY * src->NXp;
  const size_t bytes = (size_t)nk * plane * sizeof(float);
  const float* sp = state_buffer(src, which) + src_k0 * plane;
  float* dp = state_buffer(dst, which) + dst_k0 * plane;
  A3D_CUDA(cudaSetDevice(src->device));
  A3D_CUDA(cudaEventRecord(src->ev, src->st));
  A3D_CUDA(cudaSetDevice(dst->device));
  A3D_CUDA(cudaStreamWaitEvent(dst->st, src->ev, 0));
  for (int c = 0; c < 5; c++) {
    if (src->device == dst->device)
      A3D_CUDA(cudaMemcpyAsync(dp + c * dst->Np, sp + c * src->Np, bytes, cudaMemcpyDeviceToDevice, dst->st));
    else
      A3D_CUDA(cudaMemcpyPeerAsync(dp + c * dst->Np, dst->device, sp + c * src->Np, src->device, bytes, dst->st));
  }
  A3D_CUDA(cudaEventRecord(dst->ev, dst->st));
  A3D_CUDA(cudaSetDevice(src->device));
  A3D_CUDA(cudaStreamWaitEvent(src->st, dst->ev, 0));
  return A3D_OK;
}

// Device address of plane k of component c of the current (which = 0) or stage-1 (which = 1)
// state; planes of one component are contiguous, `plane_floats` apart.  For exchanges that a
// caller runs itself on the solver's stream (NCCL send/recv between ranks).
extern "C" int a3d_solver_plane_ptr(a3d_solver* s, int32_t which, int32_t c, int32_t k, void** ptr,
                                    int64_t* plane_floats) {
  clear_error();
  A3D_ARG(s && ptr && plane_floats, "null pointer");
  A3D_ARG((which == 0 || which == 1) && c >= 0 && c < 5 && k >= 0 && k < s->grid.NZ, "which, component or plane");
  const long plane = (long)s->grid.NY * s->NXp;
  *ptr = state_buffer(s, which) + c * s->Np + k * plane;
  *plane_floats = plane;
  return A3D_OK;
}

// The `dt` field of CfdGPU.read() (src/air_cfd.js:435): the local time step of each fluid cell
// in the solver's last iteration, formed from that iteration's base state, which stays in the
// B buffer after the swap; 0 for the other cells and before the first iteration.  Cell order
// as a3d_solver_read; synchronises.
extern "C" int a3d_solver_read_dt(a3d_solver* s, float* dt) {
  clear_error();
  A3D_ARG(s && dt, "null pointer");
  A3D_ARG(s->phase == 0, "between the two stages of an iteration");
  A3D_CUDA(cudaSetDevice(s->device));
  float* d = nullptr;
  A3D_CUDA(cudaMallocAsync(&d, s->N * sizeof(float), s->st));
  if (s->it == 0) {
    A3D_CUDA(cudaMemsetAsync(d, 0, s->N * sizeof(float), s->st));
  } else {
    StageArgs a;
    fill_stage_args(s, a, nullptr, nullptr, nullptr, 0.f, 1.f);
    k_local_dt<<<blocks_for(s->N), 256, 0, s->st>>>(a, s->buf[s->iB], d);
  }
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(dt, d, s->N * sizeof(float), cudaMemcpyDeviceToHost, s->st);
  cudaFreeAsync(d, s->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  if (e != cudaSuccess) { set_error("read_dt: %s", cudaGetErrorString(e)); return A3D_ERR_CUDA; }
  return A3D_OK;
}

extern "C" int a3d_solver_iterations(a3d_solver* s, int64_t* it) {
  clear_error();
  A3D_ARG(s && it, "null pointer");
  *it = s->it;
  return A3D_OK;
}

extern "C" int a3d_solver_read(a3d_solver* s, float* r, float* ru, float* rv, float* rw, float* E) {
  clear_error();
  A3D_ARG(s && r && ru && rv && rw && E, "null pointer");
  A3D_CUDA(cudaSetDevice(s->device));
  float* dst[5] = {r, ru, rv, rw, E};
  const float* Q = s->buf[s->iQ];
  const size_t row = s->grid.NX * sizeof(float), pitch = s->NXp * sizeof(float);
  for (int c = 0; c < 5; c++)
    A3D_CUDA(cudaMemcpy2DAsync(dst[c], row, Q + c * s->Np, pitch, row, (size_t)s->grid.NY * s->grid.NZ,
                               cudaMemcpyDeviceToHost, s->st));
  A3D_CUDA(cudaStreamSynchronize(s->st));
  return check_kernel_error(s);
}

extern "C" int a3d_solver_write(a3d_solver* s, const float* r, const float* ru, const float* rv, const float* rw,
                                const float* E) {
  clear_error();
  A3D_ARG(s && r && ru && rv && rw && E, "null pointer");
  A3D_CUDA(cudaSetDevice(s->device));
  const float* src[5] = {r, ru, rv, rw, E};
  float* Q = s->buf[s->iQ];
  const size_t row = s->grid.NX * sizeof(float), pitch = s->NXp * sizeof(float);
  for (int c = 0; c < 5; c++)
    A3D_CUDA(cudaMemcpy2DAsync(Q + c * s->Np, pitch, src[c], row, row, (size_t)s->grid.NY * s->grid.NZ,
                               cudaMemcpyHostToDevice, s->st));
  A3D_CUDA(cudaStreamSynchronize(s->st));
  return A3D_OK;
}

// Selects the stage kernel (0: per-cell, 2: TMA tile, 4: paired-cell TMA tile) and the z planes
// per CTA of the tiled kernels.  march_kz = 0 picks it for the TMA tiles: 32 planes where that still
// launches four waves of CTAs (column tiles x z runs >= 4 x resident CTAs), else the longest run
// of 16, 8 or 4 planes that launches two waves, else 2.  Shorter runs cost more ring prologue
// per plane but keep the SMs busy and the z chunks of a3d_solver_step overlapping.  Measured
// (G cell-updates/s, fighter): 15.8M cells 32 planes 16.0 (16: 15.7); 4.1M 16 planes 15.1 (32:
// 13.8); 2.0M 8 planes 13.5 (16: 12.2); 1.0M 4 planes 12.6 (8: 11.8); 0.3M 2 planes 7.3 (8:
// 5.6); 31k 2 planes 1.5 (8: 0.7).  Not part of the reference surface.
extern "C" int a3d_solver_set_kernel(a3d_solver* s, int32_t kernel, int32_t march_kz) {
  clear_error();
  A3D_ARG(s, "null solver");
  A3D_ARG(kernel == KERNEL_CELL || kernel == KERNEL_TMA || kernel == KERNEL_PAIR, "kernel must be 0, 2 or 4");
  A3D_ARG(march_kz >= 0 && march_kz <= 1024, "march_kz");
  if (march_kz == 0) {
    march_kz = 16;
    if (kernel == KERNEL_TMA || kernel == KERNEL_PAIR) {
      const int ty = kernel == KERNEL_PAIR ? 16 : 8;  // tile rows
      const long columns = (long)((s->grid.NX + 31) / 32) * ((s->grid.NY + ty - 1) / ty);
      int resident = 0;
      A3D_CUDA(cudaSetDevice(s->device));
      if (kernel == KERNEL_PAIR) A3D_TRY(pair_resident_ctas(&resident));
      else A3D_TRY(tma_resident_ctas(&resident));
      auto ctas = [&](int kz) { return columns * ((s->grid.NZ + kz - 1) / kz); };
      march_kz = 2;
      if (ctas(32) >= 4L * resident) march_kz = 32;
      else
        for (int kz : {16, 8, 4})
          if (ctas(kz) >= 2L * resident) { march_kz = kz; break; }
    }
  }
  s->kernel = kernel;
  s->march_kz = march_kz;
  return A3D_OK;
}

// Try_waits a stage kernel spends on one TMA copy before it gives up, flags the solver and
// leaves (A3D_WAIT_LIMIT_DEFAULT unless set; 0: at once).  A stage kernel that gives up makes
// the next a3d_solver_sync, a3d_solver_read or reduction return A3D_ERR_TIMEOUT.  Not part of
// the reference surface: it lets a test make a wait run out without anything faulting.
extern "C" int a3d_solver_set_wait_limit(a3d_solver* s, uint32_t limit) {
  clear_error();
  A3D_ARG(s, "null solver");
  s->wait_limit = limit;
  return A3D_OK;
}

extern "C" int a3d_solver_get_kernel(a3d_solver* s, int32_t* kernel, int32_t* march_kz) {
  clear_error();
  A3D_ARG(s && kernel && march_kz, "null pointer");
  *kernel = s->kernel;
  *march_kz = s->march_kz;
  return A3D_OK;
}

extern "C" int a3d_solver_stream(a3d_solver* s, void** stream) {
  clear_error();
  A3D_ARG(s && stream, "null pointer");
  *stream = (void*)s->st;
  return A3D_OK;
}

extern "C" int a3d_solver_sync(a3d_solver* s) {
  clear_error();
  A3D_ARG(s, "null solver");
  A3D_CUDA(cudaSetDevice(s->device));
  A3D_CUDA(cudaStreamSynchronize(s->st));
  return check_kernel_error(s);
}

namespace a3d {
int check_kernel_error(a3d_solver* s) {
  int f = 0;
  A3D_CUDA(cudaMemcpyAsync(&f, s->d_flag + 1, sizeof(int), cudaMemcpyDeviceToHost, s->st));
  A3D_CUDA(cudaStreamSynchronize(s->st));
  if (f) {
    // reported once: the flag is cleared, so that the solver can step again (the state of the
    // failed stage is not meaningful; a caller resets it or loads a state)
    A3D_CUDA(cudaMemsetAsync(s->d_flag + 1, 0, sizeof(int), s->st));
    A3D_CUDA(cudaStreamSynchronize(s->st));
    set_error("a stage kernel gave up waiting for a TMA copy (bounded wait ran out)");
    return A3D_ERR_TIMEOUT;
  }
  return A3D_OK;
}
}  // namespace a3d
