// Scratch-free variant of the adjoint two-electron gradient.
//
// Some callers cannot allocate device memory once they are running: a driver that
// has handed the whole device to its own pool allocator (a further cudaMalloc
// fails or fragments it), a geometry-optimisation or molecular-dynamics loop
// that forbids allocation after start-up so that its memory footprint and
// latency stay fixed, or code running where cudaMalloc's implicit device
// synchronisation is not allowed.  hfgpu_grad2e_device_noalloc serves them: it
// takes the scratch of the large gradient classes from one fixed array compiled
// into this library instead of allocating it.
//
// The array is file-scope device memory of HFGPU_NOALLOC_SCRATCH_BYTES; every
// GPU that loads the library holds it until the process exits.  Host code cannot
// use the array's name as a device address, so the first call on each device
// looks the address up with cudaGetSymbolAddress (with that device current) and
// caches it; make that first call before any stream capture.  All calls share
// the array: calls that overlap on the GPU race on it.  Nothing in the array has
// to start at zero -- each quartet initialises the slots it reads.
#include <mutex>
#include <string>

#include "../../include/hfgpu.h"
#include "hfgpu_common.cuh"

#define HFGPU_NOALLOC_SCRATCH_BYTES (32u << 20)

static __device__ __align__(256) double g_noalloc_scratch[HFGPU_NOALLOC_SCRATCH_BYTES / sizeof(double)];

int hfgpu_grad_fixed_scratch(hfgpu_handle* h, const double* DJ, double cJ, int nK, const double* DK, double cK,
                             double* grad, int precision, void* scratch, size_t scratch_bytes);
int hfgpu_device_of(const hfgpu_handle* h);
int hfgpu_cuda_error(hfgpu_handle* h, int cuda_code, const char* where);

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

// Device address of the scratch array on device `dev`, looked up once per device with that
// device current; the caller's current device is restored before returning.
int scratch_address(hfgpu_handle* h, int dev, void** out) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    cudaError_t e = cudaSetDevice(dev);
    void* a = nullptr;
    if (e == cudaSuccess) e = cudaGetSymbolAddress(&a, g_noalloc_scratch);
    if (prev >= 0 && prev != dev) cudaSetDevice(prev);
    if (e != cudaSuccess) return hfgpu_cuda_error(h, (int)e, "cudaGetSymbolAddress of the fixed gradient scratch");
    if (a == nullptr) return hfgpu_cuda_error(h, (int)cudaErrorInvalidSymbol, "fixed gradient scratch has no address");
    g_addr[dev] = a;
  }
  *out = g_addr[dev];
  return HFGPU_OK;
}
}  // namespace

extern "C" long long hfgpu_noalloc_scratch_bytes(void) { return (long long)HFGPU_NOALLOC_SCRATCH_BYTES; }

extern "C" int hfgpu_grad2e_device_noalloc(hfgpu_handle* h, const double* DJ, double cJ, int nK, const double* DK,
                                           double cK, double* grad, int precision) {
  if (!h || !grad) return HFGPU_ERR_INVALID;
  const int dev = hfgpu_device_of(h);
  if (dev < 0 || dev >= kMaxDevices) return HFGPU_ERR_INVALID;
  void* p = nullptr;
  const int rc = scratch_address(h, dev, &p);
  if (rc) return rc;
  return hfgpu_grad_fixed_scratch(h, DJ, cJ, nK, DK, cK, grad, precision, p, HFGPU_NOALLOC_SCRATCH_BYTES);
}
