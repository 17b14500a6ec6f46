// stage_pair.cu - the single-case RK-stage kernel over the paired-cell tile (stage_pair.cuh):
// one CTA per 32 x 16-column tile and z run, two CTAs per SM; plus its tensor maps.
#include "stage_pair.cuh"

namespace a3d {

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();  // stage_tma.cu

namespace {

using namespace pair;

// At most 128 registers: two CTAs (16 warps) per SM.  MODE 0: all planes of the case; 1: planes
// [a.kb, a.ke) (a z chunk or a slab's own planes); 2: the same with the halo push of a z slab.
template <bool STAGE2, int MODE>
__global__ void __launch_bounds__(NT, 2)
    k_stage_pair(const __grid_constant__ CUtensorMap tmQ, const __grid_constant__ CUtensorMap tmC, StageArgs a,
                 int kz) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  PairSmem& S = *reinterpret_cast<PairSmem*>(smem_raw);
  stage_tile<STAGE2, false, MODE >= 1, MODE == 2>(S, &tmQ, &tmC, a, a.B, a.Out, blockIdx.x, blockIdx.y, blockIdx.z,
                                                  kz);
}

template <bool STAGE2, int MODE>
int set_attributes() {
  A3D_CUDA(cudaFuncSetAttribute(k_stage_pair<STAGE2, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)pair_smem_bytes()));
  A3D_CUDA(cudaFuncSetAttribute(k_stage_pair<STAGE2, MODE>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  return A3D_OK;
}

template <int MODE>
void launch_mode(const a3d_solver* s, const StageArgs& a, int qin_buf, bool stage2, dim3 grid, cudaStream_t st) {
  const size_t sm = pair_smem_bytes();
  if (stage2) k_stage_pair<true, MODE><<<grid, NT, sm, st>>>(s->tmQp[qin_buf], s->tmCp, a, s->march_kz);
  else k_stage_pair<false, MODE><<<grid, NT, sm, st>>>(s->tmQp[qin_buf], s->tmCp, a, s->march_kz);
}

}  // namespace

// Two CTAs per SM need two tiles' shared memory (plus the 1 KB the hardware reserves per CTA)
// within the SM's 228 KB.
static_assert(2 * (sizeof(PairSmem) + 128 + 1024) <= 228 * 1024, "the paired tile no longer fits two CTAs per SM");

size_t pair_smem_bytes() { return sizeof(PairSmem) + 128; }

int pair_resident_ctas(int* n) {
  int dev = 0, sms = 0, per_sm = 0;
  A3D_CUDA(cudaGetDevice(&dev));
  A3D_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  A3D_TRY((set_attributes<false, 1>()));
  A3D_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_stage_pair<false, 1>, NT, pair_smem_bytes()));
  *n = sms * std::max(1, per_sm);
  return A3D_OK;
}

// Tensor maps of the paired tile: boxes 40 x 20 x 1 x 5 over the padded state buffers and
// 64 x 20 x 1 over the code array.
int make_pair_tensor_maps(a3d_solver* s) {
  auto enc = tensor_map_encoder();
  if (!enc) { set_error("cuTensorMapEncodeTiled is not available from the driver"); return A3D_ERR_CUDA; }
  const cuuint64_t NX = s->grid.NX, NY = s->grid.NY, NZ = s->grid.NZ, NXp = s->NXp;
  for (int b = 0; b < 3; b++) {
    const cuuint64_t dims[4] = {NX, NY, NZ, 5};
    const cuuint64_t strides[3] = {NXp * 4, NXp * NY * 4, (cuuint64_t)s->Np * 4};
    const cuuint32_t box[4] = {QBX, HY, 1, 5}, es[4] = {1, 1, 1, 1};
    CUresult r = enc(&s->tmQp[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, s->buf[b], dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) { set_error("cuTensorMapEncodeTiled(pair state) failed: %d", (int)r); return A3D_ERR_CUDA; }
  }
  const cuuint64_t cd[3] = {NX, NY, NZ}, cs[2] = {NXp, NXp * NY};
  const cuuint32_t cb[3] = {CBX, HY, 1}, ce[3] = {1, 1, 1};
  CUresult r = enc(&s->tmCp, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, s->code, cd, cs, cb, ce, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) { set_error("cuTensorMapEncodeTiled(pair codes) failed: %d", (int)r); return A3D_ERR_CUDA; }
  A3D_TRY((set_attributes<false, 0>()));
  A3D_TRY((set_attributes<true, 0>()));
  A3D_TRY((set_attributes<false, 1>()));
  A3D_TRY((set_attributes<true, 1>()));
  A3D_TRY((set_attributes<false, 2>()));
  A3D_TRY((set_attributes<true, 2>()));
  return A3D_OK;
}

// The paired-tile stage kernel over planes [a.kb, a.ke) on stream st (the solver's by default).
int launch_pair(a3d_solver* s, const StageArgs& a, int qin_buf, bool stage2, cudaStream_t st) {
  const int kz = s->march_kz;
  dim3 grid((a.NX + TX - 1) / TX, (a.NY + TY - 1) / TY, (a.ke - a.kb + kz - 1) / kz);
  if (!st) st = s->st;
  if (a.peer[0] || a.peer[1]) launch_mode<2>(s, a, qin_buf, stage2, grid, st);
  else if (a.kb != 0 || a.ke != a.NZ) launch_mode<1>(s, a, qin_buf, stage2, grid, st);
  else launch_mode<0>(s, a, qin_buf, stage2, grid, st);
  A3D_CUDA(cudaGetLastError());
  return A3D_OK;
}

}  // namespace a3d
