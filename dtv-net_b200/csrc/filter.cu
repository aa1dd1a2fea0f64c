// FBP detector-row filter: cosine weighting followed by the spatial Ram-Lak
// ramp, one fused pass over the sinogram.
//
// Follows model/ConeBeamLayers/Standard/StandardGeometry.py:51-93 (and the
// Beijing variant BeijingGeometry.py:57-84): the residual is multiplied by
//   cos(i, j) = SDD / sqrt(SDD^2 + (i - mid_i)^2 + (j - mid_j)^2)
// over each view's rows i and columns j, then every detector row of length W
// is cross-correlated with the W+1-tap kernel k[t], t = 0..W, centred at
// m = floor(W/2): k[m] = 1/8, k[t] = 0 for even t - m != 0, and
// k[t] = -1/(2 pi^2 (t-m)^2) for odd t - m, with W/2 zero columns of padding on
// each side (torch conv2d, padding (0, W/2)). W must be even (for odd W the
// reference's output row is one column short and its reshape fails).
//
// Design: one block per detector row; the weighted row sits in shared memory
// with its zero padding, the odd-offset taps (the even ones are zero) are
// built once per block in FP64 and rounded to FP32 as the reference's
// float32 kernel array holds them, and each output sums tap pairs
// k_d * (x[u-d] + x[u+d]) in FP32. The transpose (for autograd) applies the
// same symmetric correlation first and the cosine weight after.
#include <atomic>

#include "common.cuh"

namespace dtv {

constexpr int kFiltThreads = 256;
constexpr int kFiltMaxWidth = 8192;

__global__ void __launch_bounds__(kFiltThreads) fbp_filter_kernel(const float* __restrict__ in,
                                                                  float* __restrict__ out, int rows_per_view,
                                                                  int width, float sdd, float mid_i,
                                                                  float mid_j, int adjoint) {
  extern __shared__ float sm[];
  const int half = width / 2;
  float* xs = sm;                   // [half zeros | row | half zeros]
  float* taps = sm + 2 * width;     // taps[d] for odd d = 1, 3, ..., stored at d >> 1
  const int64_t r = blockIdx.x;
  const float fi = (float)(r % rows_per_view) - mid_i;
  const float* src = in + r * width;
  for (int j = threadIdx.x; j < 2 * width; j += blockDim.x) {
    const int c = j - half;
    float x = 0.f;
    if (c >= 0 && c < width) {
      x = __ldg(src + c);
      if (!adjoint) {
        const float fj = (float)c - mid_j;
        x *= sdd / sqrtf(sdd * sdd + fi * fi + fj * fj);
      }
    }
    xs[j] = x;
  }
  for (int e = threadIdx.x; e < (half + 1) / 2; e += blockDim.x) {
    const double d = 2.0 * e + 1.0;
    taps[e] = (float)(-0.5 / (3.141592653589793 * 3.141592653589793 * d * d));
  }
  __syncthreads();
  for (int u = threadIdx.x; u < width; u += blockDim.x) {
    const float* x = xs + half + u;
    float acc = 0.125f * x[0];
    float acc2 = 0.f;
    int e = 0;
    for (; e + 1 < (half + 1) / 2; e += 2) {
      const int d0 = 2 * e + 1, d1 = d0 + 2;
      acc = fmaf(taps[e], x[-d0] + x[d0], acc);
      acc2 = fmaf(taps[e + 1], x[-d1] + x[d1], acc2);
    }
    for (; e < (half + 1) / 2; ++e) {
      const int d = 2 * e + 1;
      acc = fmaf(taps[e], x[-d] + x[d], acc);
    }
    float y = acc + acc2;
    if (adjoint) {
      const float fj = (float)u - mid_j;
      y *= sdd / sqrtf(sdd * sdd + fi * fi + fj * fj);
    }
    out[r * width + u] = y;
  }
}

}  // namespace dtv

using namespace dtv;

extern "C" int dtv_fbp_filter(const float* in, float* out, int64_t rows, int32_t rows_per_view,
                              int32_t width, float sdd, float mid_i, float mid_j, int32_t adjoint,
                              void* stream) {
  DTV_CHECK(in && out, "NULL argument");
  DTV_CHECK(in != out, "the filter cannot run in place");
  DTV_CHECK(rows > 0 && rows_per_view > 0 && rows % rows_per_view == 0,
            "rows must be a positive multiple of rows_per_view");
  DTV_CHECK(rows <= 2147483647LL, "too many rows");
  DTV_CHECK(width >= 2 && width % 2 == 0 && width <= kFiltMaxWidth,
            "row width must be even and in [2, %d]", kFiltMaxWidth);
  DTV_CHECK(sdd > 0.f, "sdd must be positive");
  const size_t smem = sizeof(float) * (2 * (size_t)width + width / 4 + 1);
  if (smem > 48 * 1024) {
    // per-device function attribute, raised once to the widest row's need
    static std::atomic<unsigned long long> raised{0};
    int dev = 0;
    DTV_CUDA_TRY(cudaGetDevice(&dev));
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(raised.load() & bit)) {
      const int most = (int)(sizeof(float) * (2 * kFiltMaxWidth + kFiltMaxWidth / 4 + 1));
      DTV_CUDA_TRY(cudaFuncSetAttribute(fbp_filter_kernel,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, most));
      raised |= bit;
    }
  }
  fbp_filter_kernel<<<(unsigned)rows, kFiltThreads, smem, as_stream(stream)>>>(
      in, out, rows_per_view, width, sdd, mid_i, mid_j, adjoint ? 1 : 0);
  note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}
