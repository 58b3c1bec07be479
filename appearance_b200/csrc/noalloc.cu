// ap_trace_rays_static: the batch closest-hit / any-hit query of ap_trace_rays
// for callers that must not allocate device memory.
//
// Some hosts cannot let a plug-in call cudaMalloc: an engine or a serving
// process that owns the whole device-memory budget and hands out no more, or a
// latency-critical thread for which cudaMalloc's implicit device-wide
// synchronisation is not acceptable.  This entry point allocates nothing: its
// device staging (the rays in, the hit records out and the work cursor) lives
// in a file-scope static __device__ array of fixed size, so it holds at most
// kStaticMaxRays rays per call.  Every GPU that loads the library keeps that
// array (about 3 MiB) until the process exits.
//
// The array is shared by every call on a device, from every handle and stream:
// calls whose work overlaps on the GPU race on it, so a caller must serialise
// them (this entry point itself returns only after its copies are done).  The
// array keeps the last call's contents; the work cursor, the only part that
// must start at zero, is cleared on every call.
//
// Set-up: the first call on a device, with that device current, looks up the
// array's device address with cudaGetSymbolAddress (the array's name is only a
// host-side stand-in, not a device address) and caches it; that first call
// should therefore come before any stream capture.  The cached address belongs
// to the device's context of that moment: after cudaDeviceReset (or any
// teardown of the primary context) in the same process it is stale, so this
// entry point must not be used across a device reset.
//
// The call makes the handle's device current for its duration and gives the
// calling thread its previous current device back before it returns; on every
// path that returns after the first copy was queued it waits for the stream,
// so no copy or kernel on the shared array outlives the call.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/appearance_cuda.h"
#include "device_scope.h"
#include "frame.cuh"

namespace ap {
int handle_trace_context(void* hp, const DevScene** scene, const TwoLevel** two_level, cudaStream_t* stream,
                         int* num_sms, int* device, std::string** err);
}

namespace {

constexpr uint32_t kStaticMaxRays = 65536;
// 16 B origin+tmax, 16 B direction, 16 B hit record per ray, then the cursor
constexpr size_t kOriginOff = 0;
constexpr size_t kDirOff = (size_t)kStaticMaxRays * 16;
constexpr size_t kHitOff = (size_t)kStaticMaxRays * 32;
constexpr size_t kCursorOff = (size_t)kStaticMaxRays * 48;
constexpr size_t kScratchBytes = kCursorOff + 256;

static __device__ __align__(256) unsigned char g_trace_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of g_trace_scratch on the current device `dev`.
cudaError_t scratch_address(int dev, char** out) {
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_trace_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[dev] = p;
  }
  *out = static_cast<char*>(g_scratch_addr[dev]);
  return cudaSuccess;
}

int cuda_fail(std::string* err, cudaError_t e, const char* what) {
  *err = std::string(what) + ": " + cudaGetErrorString(e);
  return AP_E_CUDA;
}

}  // namespace

extern "C" int ap_trace_rays_static(void* handle, const float* origins_tmax, const float* dirs, uint32_t n,
                                    int any_hit, uint32_t* out4) {
  const ap::DevScene* scene = nullptr;
  const ap::TwoLevel* two_level = nullptr;
  cudaStream_t stream = nullptr;
  int num_sms = 0, device = 0;
  std::string* err = nullptr;
  int rc = ap::handle_trace_context(handle, &scene, &two_level, &stream, &num_sms, &device, &err);
  if (rc != AP_OK) return rc;
  if (!origins_tmax || !dirs || !out4) {
    *err = "null buffer";
    return AP_E_INVALID;
  }
  if (n > kStaticMaxRays) {
    *err = "ap_trace_rays_static: " + std::to_string(n) + " rays exceed the static scratch limit of " +
           std::to_string(kStaticMaxRays) + " rays per call";
    return AP_E_INVALID;
  }
  if (n == 0) return AP_OK;
  if (device < 0 || device >= kMaxDevices) {
    *err = "device index out of range";
    return AP_E_INVALID;
  }
  ap::DeviceScope device_scope(device);
  cudaError_t e = device_scope.status();
  if (e != cudaSuccess) return cuda_fail(err, e, "cudaSetDevice");
  char* base = nullptr;
  e = scratch_address(device, &base);
  if (e != cudaSuccess) return cuda_fail(err, e, "cudaGetSymbolAddress");
  float4* o = reinterpret_cast<float4*>(base + kOriginOff);
  float4* d = reinterpret_cast<float4*>(base + kDirOff);
  uint4* hits = reinterpret_cast<uint4*>(base + kHitOff);
  uint32_t* cursor = reinterpret_cast<uint32_t*>(base + kCursorOff);
  // From the first queued copy on, every return waits for the stream first.
  auto fail_after_queue = [&](cudaError_t code, const char* what) {
    cudaStreamSynchronize(stream);
    cudaGetLastError();
    return cuda_fail(err, code, what);
  };
  if ((e = cudaMemcpyAsync(o, origins_tmax, (size_t)n * 16, cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(d, dirs, (size_t)n * 16, cudaMemcpyHostToDevice, stream)) != cudaSuccess)
    return fail_after_queue(e, "ray upload");
  ap::launch_trace_batch(*scene, o, d, n, any_hit, hits, cursor, num_sms, stream,
                         two_level);  // zeroes the cursor first
  if ((e = cudaGetLastError()) != cudaSuccess) return fail_after_queue(e, "trace launch");
  if ((e = cudaMemcpyAsync(out4, hits, (size_t)n * 16, cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
    return fail_after_queue(e, "hit readback");
  if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return cuda_fail(err, e, "trace");
  return AP_OK;
}
