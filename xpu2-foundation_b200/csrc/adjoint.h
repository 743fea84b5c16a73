// The adjoint kernel (adjoint.cu; internal to libx2).
#pragma once
#include "integrator.cuh"

namespace x2 {

// Fills adjoint.cu's copy of the Sobol direction table (every translation unit with sampling kernels has one).
cudaError_t uploadSobolAdjoint(const uint32_t directions[17][32]);

// Each sample of the chunks (64 x count items a chunk) replayed, its contributions credited: gradients (FP64: 3 a
// material's albedo, then 1 a material's roughness, then 3 a light's radiance) += dL/dI of its pixel / samples a pixel
// x d(radiance)/d(parameter); texGrad (FP32, 3 a texel; null: not wanted) += dL/dtexel. Dynamic shared memory: 4 x
// materials + 3 x lights floats.
__global__ void adjointKernel(SceneView s, const x2_chunk* chunks, uint32_t chunkCount, uint32_t count, const float* dLossdImage,
                              double* gradients, uint32_t materials, uint32_t lights, float* texGrad);

}  // namespace x2
