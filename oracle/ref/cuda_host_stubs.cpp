// TEST INFRASTRUCTURE ONLY (oracle/_ref build).
//
// S3DPrinterInfo.cpp (cfms_tomo/Tomo_Shell_vc_src/cpu_src/S3DPrinterInfo.cpp:88-90,208,311-312,368-369)
// allocates its CUDA-path staging buffers with pinned host memory.  Those
// buffers are only touched by the reference CUDA engine and by the
// TOMO_CPU_FLAT_TRI debug switch, never by the INT3 path this oracle runs, so
// the CPU-only oracle library satisfies the three runtime symbols with plain
// heap memory instead of linking libcudart.
#include <cstdlib>
#include <cuda_runtime_api.h>

extern "C" {

cudaError_t CUDARTAPI cudaHostAlloc(void** ptr, size_t size, unsigned int /*flags*/)
{
  *ptr = std::malloc(size == 0 ? 1 : size);
  return (*ptr == nullptr) ? cudaErrorMemoryAllocation : cudaSuccess;
}

cudaError_t CUDARTAPI cudaMallocHost(void** ptr, size_t size)
{
  return cudaHostAlloc(ptr, size, 0);
}

cudaError_t CUDARTAPI cudaFreeHost(void* ptr)
{
  std::free(ptr);
  return cudaSuccess;
}

}  // extern "C"
