// Harness main of the reference GPU programs (see harness_pre.h).  TEST INFRASTRUCTURE ONLY.
//
// Runs the reference program's main unchanged, then writes every device buffer it allocated to
// the file named by $TGA_REF_DUMP: buffers it freed as they were just before cudaFree, buffers it
// kept as they are after its main returned.  Record layout (little-endian): int32 source line of
// the allocation, uint64 size in bytes, uint8 1 if freed by the program, uint64 bytes that follow,
// then those bytes.  Buffers larger than 256 MiB are recorded without their bytes.
//
// With $TGA_REF_TIMES set it also records the device time of every kernel the program launches
// (its own kernels and the Thrust kernels it calls): the harness defines cudaLaunchKernel, which
// every `<<<...>>>` launch of the program calls, so the programs are linked against the shared CUDA
// runtime and the definition brackets the runtime's own cudaLaunchKernel (found with
// dlsym(RTLD_NEXT)) with two events on the launch's stream.  The file gets one line per kernel
// name: launches, total milliseconds.  The programs synchronise after their launches, so the
// events add no overlap that was not there.
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <string>
#include <vector>

int tga_ref_main();

namespace {
constexpr size_t kSnapMax = 256u << 20;
struct Rec {
  int line;
  size_t n;
  void* p;
  bool live;
  std::vector<unsigned char> bytes;
};
std::vector<Rec>& recs() {
  static std::vector<Rec> r;
  return r;
}
void snap(Rec& r) {
  if (r.n > kSnapMax) return;
  r.bytes.resize(r.n);
  if (cudaMemcpy(r.bytes.data(), r.p, r.n, cudaMemcpyDeviceToHost) != cudaSuccess) r.bytes.clear();
}
struct Launch {
  const void* func;
  cudaEvent_t a, b;
};
std::vector<Launch>& launches() {
  static std::vector<Launch> l;
  return l;
}
bool timing() {
  static const bool on = std::getenv("TGA_REF_TIMES") != nullptr;
  return on;
}
void write_times(const char* path) {
  std::map<std::string, std::pair<long, double>> by;
  for (const Launch& l : launches()) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, l.a, l.b) != cudaSuccess) continue;
    const char* name = nullptr;
    if (cudaFuncGetName(&name, l.func) != cudaSuccess || !name) name = "?";
    auto& e = by[name];
    e.first += 1;
    e.second += ms;
  }
  FILE* f = std::fopen(path, "w");
  if (!f) return;
  for (const auto& kv : by) std::fprintf(f, "%ld %.6f %s\n", kv.second.first, kv.second.second, kv.first.c_str());
  std::fclose(f);
}
}  // namespace

extern "C" cudaError_t CUDARTAPI cudaLaunchKernel(const void* func, dim3 grid, dim3 block, void** args, size_t shmem,
                                                 cudaStream_t stream) {
  using Fn = cudaError_t(CUDARTAPI*)(const void*, dim3, dim3, void**, size_t, cudaStream_t);
  static Fn real = reinterpret_cast<Fn>(dlsym(RTLD_NEXT, "cudaLaunchKernel"));
  if (!real) return cudaErrorUnknown;
  if (!timing()) return real(func, grid, block, args, shmem, stream);
  Launch l{func, nullptr, nullptr};
  cudaEventCreate(&l.a);
  cudaEventCreate(&l.b);
  cudaEventRecord(l.a, stream);
  const cudaError_t e = real(func, grid, block, args, shmem, stream);
  cudaEventRecord(l.b, stream);
  launches().push_back(l);
  return e;
}

cudaError_t tga_ref_malloc(void** p, size_t n, int line) {
  const cudaError_t e = cudaMalloc(p, n);
  if (e == cudaSuccess) recs().push_back(Rec{line, n, *p, true, {}});
  return e;
}

cudaError_t tga_ref_free(void* p, int line) {
  (void)line;
  for (auto it = recs().rbegin(); it != recs().rend(); ++it) {
    if (it->live && it->p == p) {
      cudaDeviceSynchronize();
      snap(*it);
      it->live = false;
      break;
    }
  }
  return cudaFree(p);
}

int main() {
  const char* out = std::getenv("TGA_REF_DUMP");
  if (!out) {
    std::fprintf(stderr, "TGA_REF_DUMP is not set\n");
    return 2;
  }
  const int rc = tga_ref_main();
  const cudaError_t sync = cudaDeviceSynchronize();
  if (sync != cudaSuccess) {
    std::fprintf(stderr, "reference program ended with a CUDA error: %s\n", cudaGetErrorString(sync));
    return 3;
  }
  FILE* f = std::fopen(out, "wb");
  if (!f) return 4;
  for (Rec& r : recs()) {
    if (r.live) snap(r);
    const int32_t line = r.line;
    const uint64_t n = r.n;
    const uint8_t freed = r.live ? 0 : 1;
    const uint64_t have = r.bytes.size();
    std::fwrite(&line, 4, 1, f);
    std::fwrite(&n, 8, 1, f);
    std::fwrite(&freed, 1, 1, f);
    std::fwrite(&have, 8, 1, f);
    if (have) std::fwrite(r.bytes.data(), 1, have, f);
  }
  std::fclose(f);
  if (const char* times = std::getenv("TGA_REF_TIMES")) write_times(times);
  // The reference's neighbour-access main ends with `return;` in an int function, so its value is
  // indeterminate; its failures exit(1) from inside (CHECK), so reaching here means it completed.
  std::printf("harness: reference main returned %d\n", rc);
  return 0;
}
