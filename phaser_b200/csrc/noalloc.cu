// S^2 sampling without any device allocation (phgpu_sample_s2_noalloc).
//
// Who needs it: a caller that must not allocate device memory once it is
// running -- a registration node with a fixed memory budget reserved at
// start-up, or a latency-bound loop where cudaMalloc / cudaFree would
// synchronise the device and stall the other streams.  Such a caller owns its
// cloud and output buffers on the device and cannot create a phgpu_ctx per
// request (a context allocates its buffers).
//
// How: the sampler's scratch (projected points, bin keys, bin-sorted points,
// bin and row counts, bin starts, row tables, occupancy maps) and the grid directions live
// in one file-scope __device__ array of fixed size.  The first call on each device, with that
// device current, looks the array's address up with cudaGetSymbolAddress
// (this may load the module on that device); it should therefore come before
// any stream capture.  Later calls reuse the cached address.  Every call runs
// the same kernels as phgpu_sample_s2 (launch_sample), which clears the
// parts that must start at zero -- bin and row counts, cursors, the
// direction-bin maps -- with cudaMemsetAsync on the caller's stream and
// rebuilds everything else from the points; nothing relies on the array's
// load-time contents or on an earlier call's.
//
// One array per device: calls that overlap in time on the same device (two
// host threads, or two streams with work in flight) race on it.  Serialise
// them (one stream, or an event between calls).
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "../../include/phaser_gpu.h"
#include "kernels.h"

namespace phgpu {

constexpr size_t kNoAllocScratchBytes = 16u << 20;  // 16 MiB: grid directions, then the sampler scratch
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

constexpr int kMaxPoints = PHGPU_NOALLOC_MAX_POINTS;
constexpr int kMaxBw = PHGPU_NOALLOC_MAX_BANDWIDTH;
constexpr size_t kGridBytes = sizeof(float4) * 4 * (size_t)kMaxBw * kMaxBw;  // 1 MiB
constexpr size_t kScratchBytes = kNoAllocScratchBytes;

constexpr int kMaxDevices = 64;
struct DeviceSlot {
  char* scratch = nullptr;  // device address of g_noalloc_scratch
  int grid_bw = 0;          // bandwidth whose grid is resident
};
std::mutex g_mu;
DeviceSlot g_slots[kMaxDevices];
float4 g_host_grid[4 * kMaxBw * kMaxBw];  // staging for the grid upload (guarded by g_mu)

// The context's grid (capi.cu): float sin/cos of float DH angles.
void dh_grid(int bw, float4* out) {
  const int n = 2 * bw;
  for (int i = 0; i < n; ++i) {
    const float th = (float)((M_PI * (double)(2 * i + 1)) / (double)(4 * bw));
    for (int j = 0; j < n; ++j) {
      const float ph = (float)((2.0 * M_PI * (double)j) / (double)(2 * bw));
      out[(size_t)i * n + j] = make_float4(sinf(th) * cosf(ph), sinf(th) * sinf(ph), cosf(th), 0.0f);
    }
  }
}

}  // namespace
}  // namespace phgpu

using namespace phgpu;

int phgpu_sample_s2_noalloc(const phgpu_params* params, const phgpu_cloud* cloud, float* values_dev,
                            int32_t* nn_index_dev, void* stream) {
  if (!params || !cloud || !values_dev || !cloud->on_device || (cloud->n_points > 0 && !cloud->xyzi))
    return PHGPU_ERR_INVALID;
  const int bw = (int)params->spherical_bandwidth;
  if (bw < 1 || params->spatial_n_voxels < 1) return PHGPU_ERR_INVALID;
  if (bw > kMaxBw || cloud->n_points > (uint64_t)kMaxPoints) return PHGPU_ERR_LIMIT;
  if (sampler_scratch_bytes(kMaxPoints, 4 * kMaxBw * kMaxBw) + kGridBytes > kScratchBytes) return PHGPU_ERR_LIMIT;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return PHGPU_ERR_CUDA;
  cudaStream_t st = (cudaStream_t)stream;
  char* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    DeviceSlot& slot = g_slots[dev];
    if (!slot.scratch) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return PHGPU_ERR_CUDA;
      slot.scratch = (char*)p;
    }
    if (slot.grid_bw != bw) {
      // a pageable host-to-device copy cannot be captured: refuse instead of
      // invalidating the caller's capture
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) return PHGPU_ERR_CUDA;
      if (cs != cudaStreamCaptureStatusNone) return PHGPU_ERR_INVALID;
      dh_grid(bw, g_host_grid);
      // pageable source: the call returns once the source has been staged
      if (cudaMemcpyAsync(slot.scratch, g_host_grid, sizeof(float4) * 4 * (size_t)bw * bw, cudaMemcpyHostToDevice,
                          st) != cudaSuccess) {
        slot.grid_bw = 0;
        return PHGPU_ERR_CUDA;
      }
      slot.grid_bw = bw;
    }
    scratch = slot.scratch;
  }
  SampleArgs a;
  a.xyzi = reinterpret_cast<const float4*>(cloud->xyzi);
  a.refl = cloud->reflectivity;
  a.amb = cloud->ambient;
  a.n_points = (int)cloud->n_points;
  a.max_points = kMaxPoints;
  a.grid = reinterpret_cast<const float4*>(scratch);
  a.n_queries = 4 * bw * bw;
  a.n2b = 2 * bw;
  // squared voxel size of the rejection, as the context computes it
  const float vs = (fabsf(params->spatial_low_pass_lower) + fabsf(params->spatial_low_pass_upper)) /
                   (float)params->spatial_n_voxels;
  a.max_sq = vs * vs;
  a.n_out_ch = 4;
  a.out = values_dev;
  a.nn_idx = nn_index_dev;
  a.scratch = scratch + kGridBytes;
  return launch_sample(a, st) == cudaSuccess ? PHGPU_OK : PHGPU_ERR_CUDA;
}
