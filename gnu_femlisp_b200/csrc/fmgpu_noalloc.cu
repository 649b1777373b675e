// fmgpu_noalloc.cu -- a dot product that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host whose device memory is already
// handed to its own pool allocator (a framework's caching allocator, or a Lisp
// image that reserves device memory up front), and a caller inside a
// latency-critical loop that must not take the implicit device
// synchronisation of cudaMalloc/cudaFree.  fmg_dot_noalloc serves them: the
// caller passes device pointers to the inputs and to the output, and the
// reduction partials and the completion counter live in a fixed array that is
// part of the loaded library, not in memory allocated per call.
//
// Limits and rules:
//   * n <= FMG_NOALLOC_MAX_N (134,217,728 doubles, 32,768 chunks of 4096); the
//     scratch array is 32,800 doubles (about 256 KB) and every GPU that loads
//     the library holds it until the process exits;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture begins;
//   * every call makes the context's device current for its own duration and
//     gives the calling thread back the device that was current before, so a
//     host that works on several devices keeps its own current device;
//   * every call shares the one array, so calls that overlap on the GPU (on
//     different streams, or from different host threads) race and must not be
//     issued; the completion counter is cleared at the start of every call.
#include <mutex>

#include "fmgpu_kernels.cuh"

using namespace fmg;

namespace {

constexpr long long kNoAllocMaxChunks = 32768;
constexpr long long kNoAllocMaxN = kNoAllocMaxChunks * kChunk;
// partials of the chunk sums, then 32 doubles whose first word is the counter
constexpr long long kNoAllocScratch = kNoAllocMaxChunks + 32;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratch];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_addr[kMaxDevices] = {nullptr};

// Makes a device current and, on leaving the scope, restores the device that
// was current before (only when it differs).
struct DeviceScope {
  int prev = -1;
  bool switched = false;
  cudaError_t enter(int dev) {
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return e;
    if (prev == dev) return cudaSuccess;
    e = cudaSetDevice(dev);
    switched = e == cudaSuccess;
    return e;
  }
  ~DeviceScope() {
    if (switched) cudaSetDevice(prev);
  }
};

}  // namespace

namespace fmg {  // context accessors, defined in fmgpu.cu
int ctx_device(const fmg_ctx* c);
cudaStream_t ctx_stream(const fmg_ctx* c);
int ctx_error(fmg_ctx* c, int code, const char* msg);
}  // namespace fmg

extern "C" int fmg_dot_noalloc(fmg_ctx* ctx, const double* x, const double* y, long n, double* out) {
  if (!ctx) return FMG_ERR_ARG;
  if (!x || !y || !out || n < 0)
    return ctx_error(ctx, FMG_ERR_ARG, "fmg_dot_noalloc: null pointer or negative length");
  if (n > kNoAllocMaxN)
    return ctx_error(ctx, FMG_ERR_ARG,
                             "fmg_dot_noalloc: n exceeds FMG_NOALLOC_MAX_N (134217728); use fmg_dot");
  const int dev = ctx_device(ctx);
  cudaStream_t st = ctx_stream(ctx);
  if (dev < 0 || dev >= kMaxDevices) return ctx_error(ctx, FMG_ERR_ARG, "fmg_dot_noalloc: device id");
  // the context's device is current for the call; the caller's is restored
  DeviceScope scope;
  if (cudaError_t e = scope.enter(dev); e != cudaSuccess) return ctx_error(ctx, FMG_ERR_CUDA, cudaGetErrorString(e));
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {  // set-up, once per device, with that device current
      cudaError_t e = cudaGetSymbolAddress((void**)&g_noalloc_addr[dev], g_noalloc_scratch);
      if (e != cudaSuccess) {
        g_noalloc_addr[dev] = nullptr;
        return ctx_error(ctx, FMG_ERR_CUDA, cudaGetErrorString(e));
      }
    }
    scratch = g_noalloc_addr[dev];
  }
  if (n == 0) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double), st);
    return e == cudaSuccess ? FMG_OK : ctx_error(ctx, FMG_ERR_CUDA, cudaGetErrorString(e));
  }
  unsigned* counter = reinterpret_cast<unsigned*>(scratch + kNoAllocMaxChunks);
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned), st);
  if (e != cudaSuccess) return ctx_error(ctx, FMG_ERR_CUDA, cudaGetErrorString(e));
  Reduce R;
  R.part = scratch;
  R.counter = counter;
  R.scal = out;
  R.epi = EPI_STORE;
  R.slot = 0;
  launch_dot(x, y, (long long)n, R, st);
  e = cudaGetLastError();
  return e == cudaSuccess ? FMG_OK : ctx_error(ctx, FMG_ERR_CUDA, cudaGetErrorString(e));
}
