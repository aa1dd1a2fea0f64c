// Ray set-up shared by the forward projectors: the phase rules of the
// reference's ray marchers restated on the unified per-view geometry, the
// projector output epilogues and the per-ray sample loop.
#pragma once

#include "common.cuh"

namespace dtv {

struct RayParams {
  int nx, ny, nz, nu, nv, n_views;
  int phase;
  double voxel[3];
  double step;
  float scale;
  // ray tile of a block (tu x tv pixels) and of a warp (wu x wv = 32), log2
  int ltu, ltv, lwu;
  int band;  // tile rows per band of the band-major block order; 0: view-major
};

inline RayParams make_ray_params(const GeomParams& gp) {
  RayParams r;
  r.nx = gp.nx; r.ny = gp.ny; r.nz = gp.nz;
  r.nu = gp.nu; r.nv = gp.nv; r.n_views = gp.n_views;
  r.phase = gp.phase;
  for (int c = 0; c < 3; ++c) r.voxel[c] = gp.voxel[c];
  r.step = gp.step;
  r.scale = (float)gp.scale;
  r.ltu = 4; r.ltv = 4; r.lwu = 3;
  r.band = 0;
  return r;
}

// Per-ray set-up: the first sample position and step (index space) and the
// number of samples that can be non-zero.
struct RaySetup {
  float p0[3];
  float dp[3];
  int count;
};

// `sxy` / `sz` are added to the start position's x,y / z (1/2 where the
// sampler takes texture coordinates, whose texel centres sit at i + 1/2).
__device__ __forceinline__ RaySetup setup_ray(const RayParams& rp, const FPView& f, int u, int v,
                                              float sxy = 0.f, float sz = 0.f) {
  RaySetup rs;
  double r[3], rw[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    r[c] = f.d0ms[c] + u * f.u[c] + v * f.v[c];
    rw[c] = r[c] * rp.voxel[c];
  }
  const double inv = rsqrt(rw[0] * rw[0] + rw[1] * rw[1] + rw[2] * rw[2]);
  double d[3], dw[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    d[c] = r[c] * inv;    // index units per world unit of alpha
    dw[c] = rw[c] * inv;  // unit world direction
  }
  const int n3[3] = {rp.nx, rp.ny, rp.nz};
  double a0;
  double ktot;
  if (rp.phase == DTV_PHASE_BOX) {
    double lo = -1e300, hi = 1e300;
    bool miss = false;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (d[c] == 0.0) {
        if (f.s[c] < -0.5 || f.s[c] > n3[c] - 0.5) miss = true;
      } else {
        double t0 = (-0.5 - f.s[c]) / d[c], t1 = (n3[c] - 0.5 - f.s[c]) / d[c];
        lo = fmax(lo, fmin(t0, t1));
        hi = fmin(hi, fmax(t0, t1));
      }
    }
    if (miss || !(hi > lo)) {
      rs.count = 0;
      return rs;
    }
    ktot = ceil((hi - lo) / rp.step);
    a0 = lo + 0.5 * rp.step;
  } else {
    int ax;
    if (rp.phase == DTV_PHASE_STANDARD) {
      ax = fabs(dw[0]) >= fabs(dw[1]) ? 0 : 1;  // Standard forwardKernel.cu:45
    } else {                                    // Beijing forwardKernel.cu:40-58
      const double dom = fmax(fabs(dw[0]), fmax(fabs(dw[2]), fabs(dw[1])));
      ax = fabs(dw[0]) == dom ? 0 : (fabs(dw[1]) == dom ? 1 : 2);
    }
    // bounds +-n/2 in WORLD units against the world source (the reference's
    // alpha range, forwardKernel.cu:46-58)
    const double e = n3[ax] * 0.5;
    const double t0 = (-e - f.sw[ax]) / dw[ax], t1 = (e - f.sw[ax]) / dw[ax];
    const double lo = fmin(t0, t1) - 3.0, hi = fmax(t0, t1) + 3.0;
    a0 = lo;
    ktot = ceil((hi - lo) / rp.step);
  }
  // clip k to samples whose position lies in (-1, n) on every axis
  double klo = 0.0, khi = ktot;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double base = f.s[c] + a0 * d[c];
    const double dc = d[c] * rp.step;
    if (fabs(dc) < 1e-12) {
      if (base <= -1.0 || base >= n3[c]) khi = -1.0;
    } else {
      const double ka = (-1.0 - base) / dc, kb = (n3[c] - base) / dc;
      klo = fmax(klo, fmin(ka, kb));
      khi = fmin(khi, fmax(ka, kb));
    }
  }
  const double kb = fmax(floor(klo), 0.0);
  const double ke = fmin(ceil(khi) + 1.0, ktot);
  if (!(ke > kb)) {
    rs.count = 0;
    return rs;
  }
  rs.count = (int)(ke - kb);
  const double ab = a0 + kb * rp.step;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    rs.p0[c] = (float)(f.s[c] + ab * d[c] + (c < 2 ? sxy : sz));
    rs.dp[c] = (float)(d[c] * rp.step);
  }
  return rs;
}

struct FPOut {
  float* out;
  const float* g;
  float sigma;
  double* abs_sum;
  int epilogue;
};

constexpr int kFPThreads = 256;

__device__ __forceinline__ void block_add_double(double val, double* dst) {
  __shared__ double red[kFPThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = val;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < kFPThreads / 32; ++i) s += red[i];
    if (s != 0.0) atomicAdd(dst, s);
  }
}

template <class Sampler>
__device__ __forceinline__ float ray_sum(const Sampler& smp, const RaySetup& rs) {
  float a0 = 0.f, a1 = 0.f;
  int k = 0;
  float kb = 0.f;  // (float)k, advanced by exact integer additions
  for (; k + 3 < rs.count; k += 4, kb += 4.f) {
    float s[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float kf = kb + (float)j;
      s[j] = smp(fmaf(kf, rs.dp[0], rs.p0[0]), fmaf(kf, rs.dp[1], rs.p0[1]),
                 fmaf(kf, rs.dp[2], rs.p0[2]));
    }
    a0 += s[0];
    a1 += s[1];
    a0 += s[2];
    a1 += s[3];
  }
  for (; k < rs.count; ++k) {
    const float kf = (float)k;
    a0 += smp(fmaf(kf, rs.dp[0], rs.p0[0]), fmaf(kf, rs.dp[1], rs.p0[1]),
              fmaf(kf, rs.dp[2], rs.p0[2]));
  }
  return a0 + a1;
}

// Two samplers along the same ray in one loop (their set-ups differ only in
// the coordinate offsets, so the counts agree). Each sum is accumulated in
// exactly the order of ray_sum, so it has ray_sum's bits.
template <class SA, class SB>
__device__ __forceinline__ void ray_sum2(const SA& sa, const RaySetup& ra, const SB& sb,
                                         const RaySetup& rb, float& sum_a, float& sum_b) {
  float a0 = 0.f, a1 = 0.f, b0 = 0.f, b1 = 0.f;
  int k = 0;
  float kb = 0.f;
  for (; k + 3 < ra.count; k += 4, kb += 4.f) {
    float s[4], t[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float kf = kb + (float)j;
      s[j] = sa(fmaf(kf, ra.dp[0], ra.p0[0]), fmaf(kf, ra.dp[1], ra.p0[1]),
                fmaf(kf, ra.dp[2], ra.p0[2]));
      t[j] = sb(fmaf(kf, rb.dp[0], rb.p0[0]), fmaf(kf, rb.dp[1], rb.p0[1]),
                fmaf(kf, rb.dp[2], rb.p0[2]));
    }
    a0 += s[0];
    a1 += s[1];
    a0 += s[2];
    a1 += s[3];
    b0 += t[0];
    b1 += t[1];
    b0 += t[2];
    b1 += t[3];
  }
  for (; k < ra.count; ++k) {
    const float kf = (float)k;
    a0 += sa(fmaf(kf, ra.dp[0], ra.p0[0]), fmaf(kf, ra.dp[1], ra.p0[1]),
             fmaf(kf, ra.dp[2], ra.p0[2]));
    b0 += sb(fmaf(kf, rb.dp[0], rb.p0[0]), fmaf(kf, rb.dp[1], rb.p0[1]),
             fmaf(kf, rb.dp[2], rb.p0[2]));
  }
  sum_a = a0 + a1;
  sum_b = b0 + b1;
}

// z-pair sampler through the texture unit: layer L of the half2 layered
// texture holds (f[L-2], f[L-1]). x, y arrive as texture coordinates (shifted
// by 1/2), z as a voxel index.
struct PairSampler {
  cudaTextureObject_t tex;
  float lmax;  // nz + 2, the last layer
  __device__ __forceinline__ float operator()(float x, float y, float z) const {
    const float fz = floorf(z);
    const float w = z - fz;
    const float L = fminf(fmaxf(fz + 2.f, 0.f), lmax);
    const float2 a = tex2DLayered<float2>(tex, x, y, (int)L);
    return fmaf(w, a.y - a.x, a.x);
  }
};

__device__ __forceinline__ void fp_store(const RayParams& rp, const FPOut& o, int n, int b, int u,
                                         int v, float val, float& res) {
  const int64_t idx = ((int64_t)b * rp.n_views + n) * rp.nu * rp.nv + (int64_t)v * rp.nu + u;
  if (o.epilogue == DTV_EPI_STORE) {
    o.out[idx] = val;
    res = val;
  } else {
    res = val - o.g[idx];
    if (o.epilogue == DTV_EPI_RESIDUAL) o.out[idx] = res;
    else o.out[idx] = (o.out[idx] + o.sigma * res) / (1.f + o.sigma);
  }
}

// Shared-memory staged z-pair forward projector (forward_tma.cu).
int fp_tma_launch(Plan* p, const RayParams& rp, const FPOut& o, int batch, cudaStream_t st);

}  // namespace dtv
