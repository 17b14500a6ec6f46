// stage_fused.cu - single-case launch of the fused RK-stage tile (KERNEL_FUSED, stage kernel 3).
// One CTA per tile: grid (ceil(NX/32), ceil(NY/8), ceil(NZ/kz)).  See stage_fused.cuh.
#include "stage_fused.cuh"

namespace a3d {

namespace {

using namespace fused;

template <bool STAGE2>
__global__ void __launch_bounds__(TX * TY, 2)
    k_stage_fused(const __grid_constant__ CUtensorMap tmQ, const __grid_constant__ CUtensorMap tmC, StageArgs a,
                  int kz) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  FusedSmem& S = *reinterpret_cast<FusedSmem*>(smem_raw);
  stage_tile<STAGE2>(S, &tmQ, &tmC, a, a.B, a.Out, blockIdx.x, blockIdx.y, blockIdx.z, kz);
}

}  // namespace

size_t fused_smem_bytes() { return sizeof(fused::FusedSmem) + 128; }

int fused_set_attributes() {
  A3D_CUDA(cudaFuncSetAttribute(k_stage_fused<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)fused_smem_bytes()));
  A3D_CUDA(cudaFuncSetAttribute(k_stage_fused<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)fused_smem_bytes()));
  A3D_CUDA(cudaFuncSetAttribute(k_stage_fused<false>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  A3D_CUDA(cudaFuncSetAttribute(k_stage_fused<true>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  return A3D_OK;
}

int launch_fused(a3d_solver* s, const StageArgs& a, int qin_buf, bool stage2) {
  const int kz = s->march_kz;
  dim3 grid((a.NX + TX - 1) / TX, (a.NY + TY - 1) / TY, (a.NZ + kz - 1) / kz);
  if (stage2)
    k_stage_fused<true><<<grid, TX * TY, fused_smem_bytes(), s->st>>>(s->tmQ[qin_buf], s->tmC, a, kz);
  else
    k_stage_fused<false><<<grid, TX * TY, fused_smem_bytes(), s->st>>>(s->tmQ[qin_buf], s->tmC, a, kz);
  A3D_CUDA(cudaGetLastError());
  return A3D_OK;
}

}  // namespace a3d
