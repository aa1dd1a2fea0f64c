// Texture-fetch rate of the B200: bilinear fetches per second from a layered
// 2-D texture (384 x 384 x 64) for 32-, 64- and 128-bit texel formats. The
// projectors are bound by this unit, so their roofline fraction is reported
// against the 32-bit rate measured here (one fetch per forward-projector
// sample and per backprojected voxel-view).
//
// Build and run (one GPU):
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 \
//        -o /tmp/texture_fetch_rate dtv-net_b200/probes/texture_fetch_rate.cu
//   /tmp/texture_fetch_rate
// Every fetch coordinate lies inside the texture.
#include <cstdio>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#define CK(x) do { cudaError_t e = (x); if (e != cudaSuccess) { printf("%s: %s\n", #x, cudaGetErrorString(e)); return 1; } } while (0)
constexpr int W = 384, H = 384, L = 64, FETCH = 64;

template <class R>
__device__ __forceinline__ float red(R r);
template <> __device__ __forceinline__ float red<float>(float r) { return r; }
template <> __device__ __forceinline__ float red<float2>(float2 r) { return r.x + r.y; }
template <> __device__ __forceinline__ float red<float4>(float4 r) { return r.x + r.y + r.z + r.w; }

template <class R>
__global__ void fetch(cudaTextureObject_t t, float* out) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const float u0 = 20.f + (threadIdx.x & 15) * 1.3f + (blockIdx.x % 16) * 20.f;
  const float v0 = 10.f + (threadIdx.x >> 4) * 1.3f + ((blockIdx.x / 16) % 16) * 20.f;
  float acc = 0.f;
  for (int n = 0; n < FETCH; ++n) {
    const float u = u0 + n * 0.37f, v = v0 + 0.11f * n;
    acc += red<R>(tex2DLayered<R>(t, u, v, n % L));
  }
  out[tid] = acc;
}

template <class R>
int run(cudaChannelFormatDesc cd, int esz, const char* name) {
  cudaArray_t arr;
  CK(cudaMalloc3DArray(&arr, &cd, make_cudaExtent(W, H, L), cudaArrayLayered));
  // fill with a pattern: copy from a device buffer of bytes
  size_t bytes = (size_t)W * H * L * esz;
  unsigned char* d;
  CK(cudaMalloc(&d, bytes));
  CK(cudaMemset(d, 0x3c, bytes));  // half 1.0-ish / small floats
  cudaMemcpy3DParms cp = {};
  cp.srcPtr = make_cudaPitchedPtr(d, W * esz, W, H);
  cp.dstArray = arr;
  cp.extent = make_cudaExtent(W, H, L);
  cp.kind = cudaMemcpyDeviceToDevice;
  CK(cudaMemcpy3D(&cp));
  cudaResourceDesc rd = {};
  rd.resType = cudaResourceTypeArray;
  rd.res.array.array = arr;
  cudaTextureDesc td = {};
  td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
  td.filterMode = cudaFilterModeLinear;
  td.readMode = cudaReadModeElementType;
  cudaTextureObject_t t;
  CK(cudaCreateTextureObject(&t, &rd, &td, nullptr));
  const int blocks = 148 * 64, threads = 256;
  float* out;
  CK(cudaMalloc(&out, sizeof(float) * blocks * threads));
  for (int i = 0; i < 3; ++i) fetch<R><<<blocks, threads>>>(t, out);
  CK(cudaDeviceSynchronize());
  cudaEvent_t a, b;
  cudaEventCreate(&a); cudaEventCreate(&b);
  cudaEventRecord(a);
  const int reps = 10;
  for (int i = 0; i < reps; ++i) fetch<R><<<blocks, threads>>>(t, out);
  cudaEventRecord(b);
  CK(cudaEventSynchronize(b));
  float ms; cudaEventElapsedTime(&ms, a, b);
  double fetches = (double)blocks * threads * FETCH * reps;
  printf("%-8s %8.3f ms  %7.1f Gfetch/s  %.2f fetch/clk/SM@1.965GHz\n", name, ms / reps,
         fetches / (ms * 1e-3) / 1e9, fetches / (ms * 1e-3) / (148 * 1.965e9));
  cudaDestroyTextureObject(t); cudaFreeArray(arr); cudaFree(d); cudaFree(out);
  return 0;
}

int main() {
  int r = 0;
  r |= run<float>(cudaCreateChannelDesc<float>(), 4, "float");
  r |= run<float2>(cudaCreateChannelDescHalf2(), 4, "half2");
  r |= run<float4>(cudaCreateChannelDescHalf4(), 8, "half4");
  r |= run<float2>(cudaCreateChannelDesc<float2>(), 8, "float2");
  r |= run<float4>(cudaCreateChannelDesc<float4>(), 16, "float4");
  return r;
}
