// stage_tma.cu - the single-case RK-stage kernel over the TMA tile (stage_tma.cuh): one CTA per
// 32 x 8-column tile and z run, three CTAs per SM; plus the tensor maps every TMA-fed kernel
// of a solver uses.
#include "stage_tma.cuh"

namespace a3d {

namespace {

using namespace tma;

// 80 registers without spills: three CTAs (24 warps) per SM.  MODE 0: all planes of the case;
// 1: planes [a.kb, a.ke) (a z chunk or a slab's own planes); 2: the same with the halo push of
// a z slab.  Separate instances, so that the whole-case kernel carries none of it.
template <bool STAGE2, int MODE>
__global__ void __launch_bounds__(TX * TY, 3)
    k_stage_tma(const __grid_constant__ CUtensorMap tmQ, const __grid_constant__ CUtensorMap tmC, StageArgs a,
                int kz) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  TmaSmem& S = *reinterpret_cast<TmaSmem*>(smem_raw);
  stage_tile<STAGE2, false, MODE >= 1, MODE == 2>(S, &tmQ, &tmC, a, a.B, a.Out, blockIdx.x, blockIdx.y, blockIdx.z,
                                                  kz);
}

template <bool STAGE2, int MODE>
int set_tma_attributes() {
  A3D_CUDA(cudaFuncSetAttribute(k_stage_tma<STAGE2, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)tma_smem_bytes()));
  A3D_CUDA(cudaFuncSetAttribute(k_stage_tma<STAGE2, MODE>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  return A3D_OK;
}

template <int MODE>
void launch_mode(const a3d_solver* s, const StageArgs& a, int qin_buf, bool stage2, dim3 grid, cudaStream_t st) {
  const size_t sm = tma_smem_bytes();
  if (stage2) k_stage_tma<true, MODE><<<grid, TX * TY, sm, st>>>(s->tmQ[qin_buf], s->tmC, a, s->march_kz);
  else k_stage_tma<false, MODE><<<grid, TX * TY, sm, st>>>(s->tmQ[qin_buf], s->tmC, a, s->march_kz);
}

}  // namespace

// The driver's tensor-map encoder, looked up once.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

// Three CTAs per SM need three tiles' shared memory (plus the 1 KB the hardware reserves per
// CTA) within the SM's 228 KB.
static_assert(3 * (sizeof(TmaSmem) + 128 + 1024) <= 228 * 1024, "the TMA tile no longer fits three CTAs per SM");

size_t tma_smem_bytes() { return sizeof(TmaSmem) + 128; }

int tma_resident_ctas(int* n) {
  int dev = 0, sms = 0, per_sm = 0;
  A3D_CUDA(cudaGetDevice(&dev));
  A3D_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  A3D_TRY((set_tma_attributes<false, 1>()));
  A3D_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_stage_tma<false, 1>, TX * TY, tma_smem_bytes()));
  *n = sms * std::max(1, per_sm);
  return A3D_OK;
}

// Tensor maps over the padded state buffers (x, y, z, component) and the code array (x, y, z).
int make_tensor_maps(a3d_solver* s) {
  auto enc = tensor_map_encoder();
  if (!enc) { set_error("cuTensorMapEncodeTiled is not available from the driver"); return A3D_ERR_CUDA; }
  const cuuint64_t NX = s->grid.NX, NY = s->grid.NY, NZ = s->grid.NZ, NXp = s->NXp;
  for (int b = 0; b < 3; b++) {
    const cuuint64_t dims[4] = {NX, NY, NZ, 5};
    const cuuint64_t strides[3] = {NXp * 4, NXp * NY * 4, (cuuint64_t)s->Np * 4};
    const cuuint32_t box[4] = {QBX, HY, 1, 5}, es[4] = {1, 1, 1, 1};
    CUresult r = enc(&s->tmQ[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, s->buf[b], dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) { set_error("cuTensorMapEncodeTiled(state) failed: %d", (int)r); return A3D_ERR_CUDA; }
  }
  const cuuint64_t cd[3] = {NX, NY, NZ}, cs[2] = {NXp, NXp * NY};
  const cuuint32_t cb[3] = {CBX, HY, 1}, ce[3] = {1, 1, 1};
  CUresult r = enc(&s->tmC, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, s->code, cd, cs, cb, ce, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) { set_error("cuTensorMapEncodeTiled(codes) failed: %d", (int)r); return A3D_ERR_CUDA; }
  // kernel attributes are per device: set them on every solver's device
  A3D_TRY((set_tma_attributes<false, 0>()));
  A3D_TRY((set_tma_attributes<true, 0>()));
  A3D_TRY((set_tma_attributes<false, 1>()));
  A3D_TRY((set_tma_attributes<true, 1>()));
  A3D_TRY((set_tma_attributes<false, 2>()));
  A3D_TRY((set_tma_attributes<true, 2>()));
  return make_pair_tensor_maps(s);
}

// The stage kernel over planes [a.kb, a.ke) on stream st (the solver's stream by default).
int launch_tma(a3d_solver* s, const StageArgs& a, int qin_buf, bool stage2, cudaStream_t st) {
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
