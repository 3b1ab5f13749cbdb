// Link-time stand-ins used when the YMRT reference sources are built for the
// host as the oracle. Test infrastructure only; never linked into ymrt_b200.
//
// * CUDA runtime: the reference's scene module "uploads" meshes and scene
//   arrays with cudaMalloc/cudaMemcpy. In the oracle every buffer stays in host
//   memory (the reference's Get*Device() accessors return host pointers when
//   compiled without __CUDA_ARCH__), so these map to malloc/memcpy/free.
//   Kernel launches are refused: the oracle harness calls the stage kernels
//   as host functions itself.
// * assimp: model import is outside the hot path; the importer entry points
//   the scene module references fail cleanly.
// The device build of the reference (oracle/ref_gpu_harness.cu) compiles this
// file with YMRT_ORACLE_REAL_CUDA defined: it keeps only the assimp stand-ins
// and links the real CUDA runtime.
#include <cstdlib>
#include <cstring>
#include <cuda_runtime_api.h>
#include <assimp/Importer.hpp>
#include <assimp/material.h>

extern "C" {

#ifndef YMRT_ORACLE_REAL_CUDA
cudaError_t CUDARTAPI cudaMalloc(void** ptr, size_t size) {
  *ptr = std::malloc(size ? size : 1);
  return *ptr ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t CUDARTAPI cudaMallocAsync(void** ptr, size_t size, cudaStream_t) {
  return cudaMalloc(ptr, size);
}
cudaError_t CUDARTAPI cudaFree(void* ptr) {
  std::free(ptr);
  return cudaSuccess;
}
cudaError_t CUDARTAPI cudaMemcpy(void* dst, const void* src, size_t count, enum cudaMemcpyKind) {
  std::memmove(dst, src, count);
  return cudaSuccess;
}
cudaError_t CUDARTAPI cudaMemcpyAsync(void* dst, const void* src, size_t count, enum cudaMemcpyKind,
                                      cudaStream_t) {
  std::memmove(dst, src, count);
  return cudaSuccess;
}
cudaError_t CUDARTAPI cudaStreamSynchronize(cudaStream_t) { return cudaSuccess; }
cudaError_t CUDARTAPI cudaLaunchKernel(const void*, dim3, dim3, void**, size_t, cudaStream_t) {
  return cudaErrorNotSupported;
}
const char* CUDARTAPI cudaGetErrorString(cudaError_t error) {
  return error == cudaSuccess ? "no error" : "oracle host stand-in: operation not supported";
}
#endif  // YMRT_ORACLE_REAL_CUDA

aiReturn aiGetMaterialFloatArray(const aiMaterial*, const char*, unsigned int, unsigned int, ai_real*,
                                 unsigned int*) {
  return aiReturn_FAILURE;
}
aiReturn aiGetMaterialColor(const aiMaterial*, const char*, unsigned int, unsigned int, aiColor4D*) {
  return aiReturn_FAILURE;
}
unsigned int aiGetMaterialTextureCount(const aiMaterial*, aiTextureType) { return 0; }
aiReturn aiGetMaterialTexture(const aiMaterial*, aiTextureType, unsigned int, aiString*, aiTextureMapping*,
                              unsigned int*, ai_real*, aiTextureOp*, aiTextureMapMode*, unsigned int*) {
  return aiReturn_FAILURE;
}
}  // extern "C"

namespace Assimp {
Importer::Importer() : pimpl(nullptr) {}
Importer::~Importer() {}
void Importer::FreeScene() {}
const aiScene* Importer::ReadFile(const char*, unsigned int) { return nullptr; }
}  // namespace Assimp
