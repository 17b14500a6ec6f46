// solver.cuh - one solver case: device state, geometry codes, force list, reduction scratch.
#pragma once
#include <cuda.h>
#include "geom.cuh"

namespace a3d {

// Arguments of one RK stage (src/air_cfd.js:237-251): Out = wa*B + wb*(Qin + dt*R(Qin)).
struct StageArgs {
  const float* __restrict__ Qin;
  const float* __restrict__ B;
  float* __restrict__ Out;
  long Np;                       // component stride of the SoA state (5 components)
  int NXp;                        // row pitch of the state and code arrays (NX rounded up to 16)
  const uint8_t* __restrict__ code;  // per-cell codes, same padded layout as the state
  const float* __restrict__ phi;
  const float* __restrict__ ap0;
  const float* __restrict__ ap1;
  const float* __restrict__ ap2;
  const float* __restrict__ ap3;
  const float* __restrict__ rXd;  // 1/dx, 1/dy, 1/dz (float32)
  const float* __restrict__ rYd;
  const float* __restrict__ rZd;
  int NX, NY, NZ;
  float wa, wb, cfl;
  int order2;                     // 1: MUSCL-minmod, 0: first order (opt.order)
  float Pff[5];                   // primitive far-field state (rho, u, v, w, p)
  float Pfix[3][5];               // primitive fixed states of types 3, 4, 5
  float Ufix[3][5];               // conservative fixed states written to fixed cells
  int* err;                       // set when a bounded wait inside a stage kernel ran out
  uint32_t wait_limit;            // try_waits a stage kernel spends on one TMA copy before giving up
  // z slabs (kernels 0 and 2): planes this launch computes and stores, and the halo push
  int kb, ke;                     // [kb, ke): the solver's own planes (all planes unless split)
  float* peer[2];                 // lower/upper neighbour slab's buffer of the output role, or null
  long peer_np[2];                // its component stride
  int peer_k0[2], peer_k1[2];     // own planes [k0, k1) that are the neighbour's halo planes
  int peer_dk[2];                 // the neighbour's plane index = own plane index + peer_dk
};

// Device-side force-list entry arrays (cfdForceList).
struct ForceList {
  long n = 0;
  int64_t* q = nullptr;
  double *cx = nullptr, *cz = nullptr, *x = nullptr, *z = nullptr;
  void* block = nullptr;
};

// Stage kernels by number (the numbers 1 and 3 belonged to two tiles since retired: slower
// than the TMA tiles on every measured case).
enum StageKernel { KERNEL_CELL = 0, KERNEL_TMA = 2, KERNEL_PAIR = 4 };
constexpr int kMaxChunks = 4;  // z chunks of a pipelined step (6 or 8 measured no faster)

}  // namespace a3d

struct a3d_solver {
  int device = 0;
  cudaStream_t st = nullptr;
  a3d::GridDev grid;
  a3d::GeomDev geo;
  long N = 0, Np = 0;             // cells; component stride (padded layout)
  int NXp = 0;                    // row pitch: state[c*Np + (k*NY + j)*NXp + i]
  float* state = nullptr;         // 3 buffers x 5 components x Np floats
  float* buf[3] = {nullptr, nullptr, nullptr};
  int iQ = 0, iS1 = 1, iB = 2;
  uint8_t* code = nullptr;
  a3d::ForceList fl;
  double F[5];
  double fix[3][5];
  double cfl = 0.7;
  int order = 2;
  long it = 0;
  int kernel = a3d::KERNEL_PAIR;     // the fastest single-case stage kernel measured on B200
  CUtensorMap tmQ[3];             // TMA maps over the three state buffers
  CUtensorMap tmC;                // TMA map over the code array
  CUtensorMap tmQp[3];            // the same maps with the paired tile's boxes (32 x 16 columns + halo)
  CUtensorMap tmCp;
  uint32_t wait_limit = A3D_WAIT_LIMIT_DEFAULT;  // try_waits a stage kernel spends on one TMA copy
  int march_kz = 16;              // z planes per CTA of the marching kernels
  // reductions
  double* d_red = nullptr;        // device partials + results
  double* h_red = nullptr;        // pinned host mirror of the results
  int* d_flag = nullptr;          // [0] non-finite flag, [1] stage-kernel wait timeout
  float* prevR = nullptr;         // density snapshot for the residual
  long prevIt = 0;
  bool havePrev = false;
  double res_parts[2] = {0, 0};   // sum of squares and cell count of the last residual
  // z-slab decomposition of one case (a3d_solver_create_shape_slab)
  int phase = 0;                  // 1 between a lone stage 1 and its stage 2 (a3d_solver_stage)
  int own_k0 = 0, own_k1 = 0;     // own planes: the ones stage kernels store and reductions cover
  int z_lo = 0;                   // global index of the slab's plane 0
  a3d_solver* nbr[2] = {nullptr, nullptr};  // lower/upper neighbour slab the stage kernels push to
  cudaEvent_t ev = nullptr;       // orders plane copies and pushes between solvers
  // pipelined z chunks of a3d_solver_step (kernel 2): chunk c's stages run on stream cst[c] and
  // wait only for chunks c-1 and c+1, so one stage's tail overlaps the next stage's start
  int chunks_req = 0;             // 0: automatic
  cudaStream_t cst[a3d::kMaxChunks] = {};
  cudaEvent_t cev[a3d::kMaxChunks][2] = {};
  cudaEvent_t ev_fork = nullptr;
};

namespace a3d {
int solver_finish_setup(a3d_solver* s);           // codes + force list + state buffers
int launch_stage(a3d_solver* s, const StageArgs& a);
void fill_stage_args(a3d_solver* s, StageArgs& a, const float* Qin, const float* B, float* Out, float wa, float wb);
int build_force_list(a3d_solver* s);
int make_tensor_maps(a3d_solver* s);
int launch_tma(a3d_solver* s, const StageArgs& a, int qin_buf, bool stage2, cudaStream_t st = nullptr);
int launch_pair(a3d_solver* s, const StageArgs& a, int qin_buf, bool stage2, cudaStream_t st = nullptr);
int make_pair_tensor_maps(a3d_solver* s);
size_t pair_smem_bytes();
int pair_resident_ctas(int* n);         // CTAs of the paired-tile stage kernel resident on the current device
size_t tma_smem_bytes();
int tma_resident_ctas(int* n);          // CTAs of the TMA stage kernel resident on the current device
int check_kernel_error(a3d_solver* s);  // A3D_ERR_TIMEOUT if a stage kernel flagged a timeout
}  // namespace a3d
