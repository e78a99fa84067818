// Closest-hit replay that allocates nothing (rtb_trace_replay_static, include/rtb200.h).
//
// rtb_trace_replay stages the caller's rays and the hit records in a device buffer the
// context grows with cudaMalloc.  Some callers cannot allocate device memory at the time
// they query: code running where the allocator is owned by someone else (a host framework
// with a fixed device-memory budget, a real-time frame loop that forbids allocation after
// start-up, or an embedding that only hands out pre-reserved pools).  For them this entry
// point stages rays and hits in a fixed device array defined in this file and calls no
// cudaMalloc, cudaFree or allocating library routine.
//
// The array is a file-scope __device__ variable: every GPU that loads the library holds it
// (RTB_STATIC_REPLAY_MAX_RAYS x 52 bytes) until the process exits.  Host code cannot use the
// array's name as a device address, so the first call on each device (with that device
// current) looks the address up with cudaGetSymbolAddress and caches it; that first call
// should come before any stream capture.  The cached address belongs to the device's
// primary context: after cudaDeviceReset (or anything else that destroys that context and
// reloads the module) it no longer names the array, so a process that resets a device must
// not call this entry point on it again.  Every call on a device shares the one array and
// the last call's contents stay in it; that is harmless here because the trace kernel
// writes every output record of every ray of the call (flag, distance, order, material and
// normal, misses included), so no slot of an earlier call is read back.  Calls that overlap
// on the GPU race on the array: issue them from one thread, or serialise them.
#include <cstring>
#include <mutex>

#include "rtb_internal.h"

namespace rtb {
namespace {

constexpr int kMaxRays = RTB_STATIC_REPLAY_MAX_RAYS;
// Per ray: origin.xyz + direction.xyz (24 B), flag, distance, order, material (16 B),
// normal (12 B); each section starts on a 256-byte boundary.
constexpr size_t kRaysBytes = (size_t)kMaxRays * 24;
constexpr size_t kWordBytes = (size_t)kMaxRays * 4;
constexpr size_t kNormalBytes = (size_t)kMaxRays * 12;
constexpr size_t kScratchBytes = kRaysBytes + 4 * kWordBytes + kNormalBytes;
static_assert(kRaysBytes % 256 == 0 && kWordBytes % 256 == 0, "sections stay 256-byte aligned");

static __device__ __align__(256) unsigned char g_replay_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned char* g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of this device's copy of g_replay_scratch (set up once per device; the
// device must be current).
cudaError_t scratch_address(int device, unsigned char** out) {
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_replay_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[device] = (unsigned char*)p;
  }
  *out = g_scratch_ptr[device];
  return cudaSuccess;
}

}  // namespace
}  // namespace rtb

using namespace rtb;

extern "C" rtb_status rtb_trace_replay_static(const rtb_scene* scene, const float* rays, int ray_count,
                                              int use_bvh, int* hit_flags, float* hit_distances,
                                              int* hit_orders, int* hit_materials,
                                              float* hit_normals) {
  if (!scene || !rays || !hit_flags || !hit_distances || !hit_orders || !hit_materials ||
      !hit_normals || ray_count <= 0)
    return RTB_ERR_INVALID_ARGUMENT;
  if (ray_count > kMaxRays) return RTB_ERR_LIMIT;  // more rays than the fixed scratch holds
  if (scene->device < 0 || scene->device >= kMaxDevices) return RTB_ERR_INVALID_ARGUMENT;
  int previous = 0;
  if (cudaGetDevice(&previous) != cudaSuccess) return RTB_ERR_CUDA;
  if (cudaSetDevice(scene->device) != cudaSuccess) return RTB_ERR_CUDA;
  rtb_status status = RTB_OK;
  unsigned char* base = nullptr;
  cudaError_t e = scratch_address(scene->device, &base);
  if (e == cudaSuccess) {
    const size_t n = (size_t)ray_count;
    float* d_rays = (float*)base;
    int* d_flags = (int*)(base + kRaysBytes);
    float* d_t = (float*)(base + kRaysBytes + kWordBytes);
    int* d_order = (int*)(base + kRaysBytes + 2 * kWordBytes);
    int* d_mat = (int*)(base + kRaysBytes + 3 * kWordBytes);
    float* d_normal = (float*)(base + kRaysBytes + 4 * kWordBytes);
    cudaStream_t sm = cudaStreamPerThread;
    e = cudaMemcpyAsync(d_rays, rays, n * 24, cudaMemcpyHostToDevice, sm);
    if (e == cudaSuccess)
      e = launch_trace(scene->dev, use_bvh, d_rays, ray_count, d_flags, d_t, d_order, d_mat, d_normal, sm);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hit_flags, d_flags, n * 4, cudaMemcpyDeviceToHost, sm);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hit_distances, d_t, n * 4, cudaMemcpyDeviceToHost, sm);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hit_orders, d_order, n * 4, cudaMemcpyDeviceToHost, sm);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hit_materials, d_mat, n * 4, cudaMemcpyDeviceToHost, sm);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hit_normals, d_normal, n * 12, cudaMemcpyDeviceToHost, sm);
    cudaError_t se = cudaStreamSynchronize(sm);
    if (e == cudaSuccess) e = se;
  }
  if (e != cudaSuccess) status = RTB_ERR_CUDA;
  cudaSetDevice(previous);
  return status;
}
