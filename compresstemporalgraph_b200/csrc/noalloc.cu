// Device scratch of tga_pagerank_noalloc: a file-scope __device__ array, so that entry point
// needs no cudaMalloc.  It sits in its own translation unit (its own CUDA module): under the
// runtime's default lazy module loading the ~20 MiB are reserved on a device only once the
// no-allocation entry point has looked the array up there, so the other entry points do not
// carry it.  Under eager module loading (CUDA_MODULE_LOADING=EAGER) every module is loaded when
// the context is created, so the array is reserved then, for every user of the library.
//
// The address looked up per device is cached for the life of the process.  It belongs to the
// device's primary context: after cudaDeviceReset (or anything else that destroys and recreates
// the primary context) the module is loaded again at a new address, so the cache is checked on
// every call and refreshed when the runtime no longer knows the cached pointer.
#include <mutex>
#include <string>

#include "engine.hpp"

namespace tga {

static __device__ __align__(256) unsigned char g_pr_noalloc_scratch[kPrNoAllocScratchBytes];

int pr_noalloc_scratch(int device, unsigned char** out) {
  constexpr int kMaxDevices = 64;
  static std::mutex mu;
  static unsigned char* addr[kMaxDevices] = {};
  if (device < 0 || device >= kMaxDevices) return fail(TGA_E_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (addr[device]) {
    // A pointer of a destroyed context is unknown to the runtime (or no longer device memory).
    cudaPointerAttributes pa{};
    const cudaError_t e = cudaPointerGetAttributes(&pa, addr[device]);
    if (e != cudaSuccess || pa.type != cudaMemoryTypeDevice || pa.device != device) {
      cudaGetLastError();
      addr[device] = nullptr;
    }
  }
  if (!addr[device]) {
    int cur = -1;
    TGA_CUDA_TRY(cudaGetDevice(&cur));
    if (cur != device) TGA_CUDA_TRY(cudaSetDevice(device));
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_pr_noalloc_scratch);
    if (cur != device) cudaSetDevice(cur);
    if (e != cudaSuccess)
      return fail(TGA_E_CUDA, std::string("cudaGetSymbolAddress of the no-allocation scratch failed: ") +
                                  cudaGetErrorString(e));
    addr[device] = static_cast<unsigned char*>(p);
  }
  *out = addr[device];
  return TGA_OK;
}

}  // namespace tga
