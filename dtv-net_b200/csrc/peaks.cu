// Roofline denominators measured on the device the library runs on.
//
// The projectors are not bound by HBM: the volume and the sinogram stay in
// L2, and what limits them is the texture unit's bilinear-fetch rate (one
// fetch per forward-projector sample and per backprojected voxel-view). The
// exact adjoint's cell-record scatter is bound by the L2's rate of 16-byte
// vector reductions. These two entry points time each rate with a kernel that
// does nothing else, so the projector kernels' fractions of them can be
// reported beside their HBM fractions. They allocate, synchronise and are
// meant for benchmarks, not for the projection path.
#include <algorithm>
#include <cuda_fp16.h>

#include "common.cuh"

namespace dtv {
namespace {

constexpr int kTexW = 384, kTexH = 384, kTexL = 64, kTexFetch = 64;

template <class R>
__device__ __forceinline__ float fold(R r);
template <>
__device__ __forceinline__ float fold<float2>(float2 r) { return r.x + r.y; }
template <>
__device__ __forceinline__ float fold<float4>(float4 r) { return r.x + r.y + r.z + r.w; }

// Every thread takes kTexFetch bilinear fetches from a 16 x 16-pixel patch of
// its block's tile, one layer per fetch, all coordinates inside the texture
// (u, v in [20, 384 - 20)).
template <class R>
__global__ void texture_rate_kernel(cudaTextureObject_t t, float* out) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const float u0 = 20.f + (threadIdx.x & 15) * 1.3f + (blockIdx.x % 16) * 20.f;
  const float v0 = 10.f + (threadIdx.x >> 4) * 1.3f + ((blockIdx.x / 16) % 16) * 20.f;
  float acc = 0.f;
  for (int n = 0; n < kTexFetch; ++n) {
    const float u = u0 + n * 0.37f, v = v0 + 0.11f * n;
    acc += fold<R>(tex2DLayered<R>(t, u, v, n % kTexL));
  }
  out[tid] = acc;
}

// The same access pattern on a 2-D array holding the 64 planes as an 8 x 8
// grid of 384 x 384 tiles (texture gather works on 2-D arrays only): either a
// bilinear fetch of a half2 texel or a gather (tld4) of the four 32-bit texels
// of the same footprint, unfiltered.
constexpr int kTileGrid = 8;
template <bool Gather>
__global__ void texture_tiled_rate_kernel(cudaTextureObject_t t, float* out) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const float u0 = 20.f + (threadIdx.x & 15) * 1.3f + (blockIdx.x % 16) * 20.f;
  const float v0 = 10.f + (threadIdx.x >> 4) * 1.3f + ((blockIdx.x / 16) % 16) * 20.f;
  float acc = 0.f;
  unsigned int bits = 0u;
  for (int n = 0; n < kTexFetch; ++n) {
    const int tile = n % kTexL;
    const float u = u0 + n * 0.37f + (tile % kTileGrid) * kTexW;
    const float v = v0 + 0.11f * n + (tile / kTileGrid) * kTexH;
    if (Gather) {
      const uint4 g = tex2Dgather<uint4>(t, u, v, 0);
      bits ^= g.x + g.y + g.z + g.w;
    } else {
      const float2 r = tex2D<float2>(t, u, v);
      acc += r.x + r.y;
    }
  }
  out[tid] = acc + (float)(bits & 0xFFu);
}

// Each warp adds one float4 per lane into 32 consecutive records (512
// contiguous bytes) per step, walking the records with a stride that keeps
// all warps on distinct lines; pattern 1 scatters the lanes over the buffer.
__global__ void atomic_v4_rate_kernel(float4* rec, int64_t n_rec, int steps, int pattern) {
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const float4 one = make_float4(1.f, 2.f, 3.f, 4.f);
  uint64_t h = (uint64_t)(warp * 32 + lane) * 0x9E3779B97F4A7C15ull;
  for (int s = 0; s < steps; ++s) {
    int64_t r;
    if (pattern == 0) {
      r = ((warp + (int64_t)s * 7919) * 32) % n_rec + lane;
      if (r >= n_rec) r -= n_rec;
    } else {
      h ^= h >> 29;
      h *= 0xBF58476D1CE4E5B9ull;
      r = (int64_t)(h % (uint64_t)n_rec);
    }
    atomicAdd(rec + r, one);
  }
}

template <class R>
int time_texture(cudaChannelFormatDesc cd, int esz, double* out) {
  cudaArray_t arr = nullptr;
  unsigned char* fill = nullptr;
  float* sink = nullptr;
  cudaTextureObject_t tex = 0;
  cudaEvent_t a = nullptr, b = nullptr;
  int rc = DTV_OK;
  const int blocks = 148 * 64, threads = 256, reps = 10;
  auto run = [&]() -> int {
    DTV_CUDA_TRY(cudaMalloc3DArray(&arr, &cd, make_cudaExtent(kTexW, kTexH, kTexL),
                                   cudaArrayLayered));
    const size_t bytes = (size_t)kTexW * kTexH * kTexL * esz;
    DTV_CUDA_TRY(cudaMalloc(&fill, bytes));
    DTV_CUDA_TRY(cudaMemset(fill, 0x3c, bytes));
    cudaMemcpy3DParms cp = {};
    cp.srcPtr = make_cudaPitchedPtr(fill, (size_t)kTexW * esz, kTexW, kTexH);
    cp.dstArray = arr;
    cp.extent = make_cudaExtent(kTexW, kTexH, kTexL);
    cp.kind = cudaMemcpyDeviceToDevice;
    DTV_CUDA_TRY(cudaMemcpy3D(&cp));
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td = {};
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    DTV_CUDA_TRY(cudaCreateTextureObject(&tex, &rd, &td, nullptr));
    DTV_CUDA_TRY(cudaMalloc(&sink, sizeof(float) * blocks * threads));
    for (int i = 0; i < 3; ++i) {
      texture_rate_kernel<R><<<blocks, threads>>>(tex, sink); note_launch();
    }
    DTV_LAUNCH_CHECK();
    DTV_CUDA_TRY(cudaEventCreate(&a));
    DTV_CUDA_TRY(cudaEventCreate(&b));
    DTV_CUDA_TRY(cudaEventRecord(a));
    for (int i = 0; i < reps; ++i) {
      texture_rate_kernel<R><<<blocks, threads>>>(tex, sink); note_launch();
    }
    DTV_CUDA_TRY(cudaEventRecord(b));
    DTV_CUDA_TRY(cudaEventSynchronize(b));
    DTV_LAUNCH_CHECK();
    float ms = 0.f;
    DTV_CUDA_TRY(cudaEventElapsedTime(&ms, a, b));
    *out = (double)blocks * threads * kTexFetch * reps / (ms * 1e-3);
    return DTV_OK;
  };
  rc = run();
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  if (tex) cudaDestroyTextureObject(tex);
  if (sink) cudaFree(sink);
  if (fill) cudaFree(fill);
  if (arr) cudaFreeArray(arr);
  return rc;
}

template <bool Gather>
int time_texture_tiled(double* out) {
  cudaArray_t arr = nullptr;
  unsigned char* fill = nullptr;
  float* sink = nullptr;
  cudaTextureObject_t tex = 0;
  cudaEvent_t a = nullptr, b = nullptr;
  const int blocks = 148 * 64, threads = 256, reps = 10;
  const int W = kTexW * kTileGrid, H = kTexH * kTileGrid;
  auto run = [&]() -> int {
    const cudaChannelFormatDesc cd = Gather ? cudaCreateChannelDesc<unsigned int>()
                                            : cudaCreateChannelDescHalf2();
    DTV_CUDA_TRY(cudaMallocArray(&arr, &cd, W, H, Gather ? cudaArrayTextureGather : 0));
    const size_t bytes = (size_t)W * H * 4;
    DTV_CUDA_TRY(cudaMalloc(&fill, bytes));
    DTV_CUDA_TRY(cudaMemset(fill, 0x3c, bytes));
    DTV_CUDA_TRY(cudaMemcpy2DToArray(arr, 0, 0, fill, (size_t)W * 4, (size_t)W * 4, H,
                                     cudaMemcpyDeviceToDevice));
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td = {};
    td.addressMode[0] = td.addressMode[1] = cudaAddressModeBorder;
    td.filterMode = Gather ? cudaFilterModePoint : cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    DTV_CUDA_TRY(cudaCreateTextureObject(&tex, &rd, &td, nullptr));
    DTV_CUDA_TRY(cudaMalloc(&sink, sizeof(float) * blocks * threads));
    for (int i = 0; i < 3; ++i) {
      texture_tiled_rate_kernel<Gather><<<blocks, threads>>>(tex, sink); note_launch();
    }
    DTV_LAUNCH_CHECK();
    DTV_CUDA_TRY(cudaEventCreate(&a));
    DTV_CUDA_TRY(cudaEventCreate(&b));
    DTV_CUDA_TRY(cudaEventRecord(a));
    for (int i = 0; i < reps; ++i) {
      texture_tiled_rate_kernel<Gather><<<blocks, threads>>>(tex, sink); note_launch();
    }
    DTV_CUDA_TRY(cudaEventRecord(b));
    DTV_CUDA_TRY(cudaEventSynchronize(b));
    DTV_LAUNCH_CHECK();
    float ms = 0.f;
    DTV_CUDA_TRY(cudaEventElapsedTime(&ms, a, b));
    *out = (double)blocks * threads * kTexFetch * reps / (ms * 1e-3);
    return DTV_OK;
  };
  const int rc = run();
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  if (tex) cudaDestroyTextureObject(tex);
  if (sink) cudaFree(sink);
  if (fill) cudaFree(fill);
  if (arr) cudaFreeArray(arr);
  return rc;
}

}  // namespace
}  // namespace dtv

extern "C" {

int dtv_measure_texture_fetch_rate(int32_t texel_bits, double* fetches_per_second) {
  using namespace dtv;
  DTV_CHECK(fetches_per_second, "NULL argument");
  DTV_CHECK(texel_bits == 32 || texel_bits == 64, "texel_bits must be 32 or 64");
  if (texel_bits == 32) return time_texture<float2>(cudaCreateChannelDescHalf2(), 4,
                                                    fetches_per_second);
  return time_texture<float4>(cudaCreateChannelDescHalf4(), 8, fetches_per_second);
}

int dtv_measure_texture_gather_rate(int32_t gather, double* fetches_per_second) {
  using namespace dtv;
  DTV_CHECK(fetches_per_second, "NULL argument");
  DTV_CHECK(gather == 0 || gather == 1, "gather must be 0 (bilinear half2) or 1 (gather u32)");
  return gather ? time_texture_tiled<true>(fetches_per_second)
                : time_texture_tiled<false>(fetches_per_second);
}

int dtv_measure_atomic_v4_rate(int64_t records, int32_t pattern, double* atomics_per_second) {
  using namespace dtv;
  DTV_CHECK(atomics_per_second, "NULL argument");
  DTV_CHECK(records >= 1024 && records <= (int64_t)1 << 26,
            "records must lie in [1024, 2^26] (16-byte records)");
  DTV_CHECK(pattern == 0 || pattern == 1, "pattern must be 0 (contiguous) or 1 (scattered)");
  float4* rec = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  const int blocks = 148 * 16, threads = 256, steps = 256, reps = 5;
  auto run = [&]() -> int {
    DTV_CUDA_TRY(cudaMalloc(&rec, records * sizeof(float4)));
    DTV_CUDA_TRY(cudaMemset(rec, 0, records * sizeof(float4)));
    atomic_v4_rate_kernel<<<blocks, threads>>>(rec, records, steps, pattern); note_launch();
    DTV_LAUNCH_CHECK();
    DTV_CUDA_TRY(cudaEventCreate(&a));
    DTV_CUDA_TRY(cudaEventCreate(&b));
    DTV_CUDA_TRY(cudaEventRecord(a));
    for (int i = 0; i < reps; ++i) {
      atomic_v4_rate_kernel<<<blocks, threads>>>(rec, records, steps, pattern); note_launch();
    }
    DTV_CUDA_TRY(cudaEventRecord(b));
    DTV_CUDA_TRY(cudaEventSynchronize(b));
    DTV_LAUNCH_CHECK();
    float ms = 0.f;
    DTV_CUDA_TRY(cudaEventElapsedTime(&ms, a, b));
    *atomics_per_second = (double)blocks * threads * steps * reps / (ms * 1e-3);
    return DTV_OK;
  };
  const int rc = run();
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  if (rec) cudaFree(rec);
  return rc;
}

}  // extern "C"
