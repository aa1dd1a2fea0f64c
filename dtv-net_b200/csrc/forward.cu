// Ray-driven cone-beam forward projector (all views and batch items in one
// launch) and its exact transpose.
//
// Follows Standard/plug/kernel/forwardKernel.cu:22-86 and
// Beijing/plug/kernel/forwardKernel.cu:17-76: a thread per detector pixel sums
// trilinear samples (border value 0) of the volume at a uniform spacing along
// the source-to-pixel ray and scales the sum. Differences of design:
//   - one launch covers every view and batch item (the reference launched per
//     view after a host sync, forwardKernel.cu:134-136);
//   - the per-ray set-up (ray direction, phase rule, sample range) runs in FP64
//     and the sample loop visits only samples that can touch the volume (the
//     reference marched the whole +-n/2 +-3 world interval, :45-80; skipped
//     samples contribute exactly 0);
//   - the volume is sampled either from a zero-padded staged copy with
//     software trilinear weights in FP32 (exact adjoint available), or through
//     a texture object (hardware filtering, as the reference).
#include <algorithm>
#include <vector>
#include <string.h>

#include "ray.cuh"

namespace dtv {

// ---- samplers --------------------------------------------------------------------------
template <class T>
struct SoftSampler {
  const T* vol;  // padded volume of this batch item
  int px, pxy;   // padded pitches
  float mx, my, mz;  // clamp maxima (n along each axis)
  __device__ __forceinline__ float operator()(float x, float y, float z) const {
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    const float ax = x - fx, ay = y - fy, az = z - fz;
    const int ix = (int)fminf(fmaxf(fx, -2.f), mx) + kPad;
    const int iy = (int)fminf(fmaxf(fy, -2.f), my) + kPad;
    const int iz = (int)fminf(fmaxf(fz, -2.f), mz) + kPad;
    const T* b = vol + (iz * pxy + iy * px + ix);
    const float v000 = load_as_float(b, 0), v001 = load_as_float(b, 1);
    const float v010 = load_as_float(b, px), v011 = load_as_float(b, px + 1);
    const float v100 = load_as_float(b, pxy), v101 = load_as_float(b, pxy + 1);
    const float v110 = load_as_float(b, pxy + px), v111 = load_as_float(b, pxy + px + 1);
    const float c00 = fmaf(ax, v001 - v000, v000), c01 = fmaf(ax, v011 - v010, v010);
    const float c10 = fmaf(ax, v101 - v100, v100), c11 = fmaf(ax, v111 - v110, v110);
    const float c0 = fmaf(ay, c01 - c00, c00), c1 = fmaf(ay, c11 - c10, c10);
    return fmaf(az, c1 - c0, c0);
  }
};

// The same trilinear interpolation from the quad copy of the padded volume:
// record (x, y, z) = (f(x,y,z), f(x+1,y,z), f(x,y+1,z), f(x+1,y+1,z)), so a
// sample makes two 16-byte loads (planes z and z+1) instead of eight 4-byte
// ones, and the lerps run in the order of SoftSampler (same result bits).
struct QuadSampler {
  const float4* q;  // quad records of this batch item (padded indexing)
  int px, pxy;
  float mx, my, mz;
  __device__ __forceinline__ float operator()(float x, float y, float z) const {
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    const float ax = x - fx, ay = y - fy, az = z - fz;
    const int ix = (int)fminf(fmaxf(fx, -2.f), mx) + kPad;
    const int iy = (int)fminf(fmaxf(fy, -2.f), my) + kPad;
    const int iz = (int)fminf(fmaxf(fz, -2.f), mz) + kPad;
    const float4* b = q + (iz * pxy + iy * px + ix);
    const float4 lo = __ldg(b), hi = __ldg(b + pxy);
    const float c00 = fmaf(ax, lo.y - lo.x, lo.x), c01 = fmaf(ax, lo.w - lo.z, lo.z);
    const float c10 = fmaf(ax, hi.y - hi.x, hi.x), c11 = fmaf(ax, hi.w - hi.z, hi.z);
    const float c0 = fmaf(ay, c01 - c00, c00), c1 = fmaf(ay, c11 - c10, c10);
    return fmaf(az, c1 - c0, c0);
  }
};

// Packed FP32 pairs (Blackwell's two-lane FP32 arithmetic): the z-pair
// samplers interpolate both planes of a cell in one instruction.
__device__ __forceinline__ unsigned long long f32x2(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ unsigned long long f32x2_lerp(unsigned long long w,
                                                         unsigned long long a,
                                                         unsigned long long b) {
  unsigned long long d, r;  // a + w (b - a), each lane rounded as fmaf(w, b - a, a)
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(b), "l"(a));
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(w), "l"(d), "l"(a));
  return r;
}
__device__ __forceinline__ unsigned long long half2_to_f32x2(unsigned int w) {
  const float2 f = __half22float2(u32_as_half2(w));
  return f32x2(f.x, f.y);
}

// Exact trilinear sample of the FP16 z pairs (DTV_PLAN_PAIRS_EXACT): one
// 16-byte record [L][Y][X] holds the four x/y corner words of the sample's
// cell, word = (f[fz], f[fz+1]) at layer L = floor(z) + 3, so a sample is one
// 128-bit load through L1 and FP32 x/y/z weights (x, then y, then z, as
// SoftSampler; both planes at once in packed FP32). Positions arrive in voxel
// index coordinates within one step of (-1, n) (the ray set-up), inside the
// kQuadPad border; the record index is clamped into the array all the same,
// so no position can address memory outside it.
struct PairQuadSampler {
  const uint4* rec;  // records of this batch item, shifted to (x, y, z) = (0, 0, 0)
  float px;          // records per row (nx + 6)
  int plane;         // records per layer
  int lo, hi;        // valid record offsets from rec: [lo, hi]
  __device__ __forceinline__ float operator()(float x, float y, float z) const {
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    const float ax = x - fx, ay = y - fy, az = z - fz;
    int q = (int)fz * plane + (int)fmaf(fy, px, fx);
    q = min(max(q, lo), hi);
    const uint4 r = __ldg(rec + q);
    const unsigned long long wx = f32x2(ax, ax), wy = f32x2(ay, ay);
    const unsigned long long a0 = f32x2_lerp(wx, half2_to_f32x2(r.x), half2_to_f32x2(r.y));
    const unsigned long long a1 = f32x2_lerp(wx, half2_to_f32x2(r.z), half2_to_f32x2(r.w));
    float lo0, hi0;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo0), "=f"(hi0) : "l"(f32x2_lerp(wy, a0, a1)));
    return fmaf(az, hi0 - lo0, lo0);
  }
};

// The exact sampler over batch item b's records.
__device__ __forceinline__ PairQuadSampler pair_quad_sampler(const RayParams& rp,
                                                             const uint4* rec, int64_t rec_elems,
                                                             int b) {
  PairQuadSampler smp;
  const int px = rp.nx + 2 * kQuadPad;
  smp.px = (float)px;
  smp.plane = px * (rp.ny + 2 * kQuadPad);
  const int origin = kQuadPad * smp.plane + kQuadPad * px + kQuadPad;
  smp.rec = rec + b * rec_elems + origin;
  smp.lo = -origin;
  smp.hi = (int)rec_elems - 1 - origin;
  return smp;
}

// Texture coordinates: the ray set-up already added the 1/2 texel offset.
struct TexSampler {
  cudaTextureObject_t tex;
  __device__ __forceinline__ float operator()(float x, float y, float z) const {
    return tex3D<float>(tex, x, y, z);
  }
};


// Ray tiles {log2 tu, log2 tv, log2 wu}: a block projects tu x tv detector
// pixels of one view (tu * tv = 256), a warp wu x (32 / wu) of them. The shape
// decides how compact each warp's texture footprint is.
static const int kRayTiles[kNumRayTiles][3] = {{4, 4, 3}, {4, 4, 4}, {5, 3, 5}, {4, 4, 2},
                                               {5, 3, 3}, {3, 5, 3}, {6, 2, 5}, {3, 5, 2}};

// The (ray tile, view) of this block of a (tiles, views) grid. View-major:
// the grid's own order. Band-major (rp.band tile rows per band): blocks in
// launch order take every view of one band of tiles before the next band, so
// the blocks resident at any time sample one slab of the volume.
__device__ __forceinline__ void block_tile_view(const RayParams& rp, int& tile, int& n) {
  if (rp.band <= 0) {
    tile = (int)blockIdx.x;
    n = (int)blockIdx.y;
    return;
  }
  const int tiles = (int)gridDim.x;
  const int tiles_u = (rp.nu + (1 << rp.ltu) - 1) >> rp.ltu;
  const int64_t per_band = (int64_t)tiles_u * rp.band;
  const int64_t lin = (int64_t)blockIdx.y * tiles + blockIdx.x;
  const int64_t band = lin / (per_band * rp.n_views);
  const int64_t r = lin - band * per_band * rp.n_views;
  const int64_t in_band = min(per_band, (int64_t)tiles - band * per_band);  // last band: shorter
  n = (int)(r / in_band);
  tile = (int)(band * per_band + (r - (int64_t)n * in_band));
}

__device__ __forceinline__ void tile_pixel(const RayParams& rp, int& u, int& v, int& n) {
  const int t = threadIdx.x, w = t >> 5, l = t & 31;
  const int tiles_u = (rp.nu + (1 << rp.ltu) - 1) >> rp.ltu;
  int tile;
  block_tile_view(rp, tile, n);
  const int tu = tile % tiles_u, tv = tile / tiles_u;
  const int lwpr = rp.ltu - rp.lwu;  // log2 warps per tile row
  u = (tu << rp.ltu) + ((w & ((1 << lwpr) - 1)) << rp.lwu) + (l & ((1 << rp.lwu) - 1));
  v = (tv << rp.ltv) + ((w >> lwpr) << (5 - rp.lwu)) + (l >> rp.lwu);
}

template <class T>
__global__ void __launch_bounds__(kFPThreads) fp_soft_kernel(RayParams rp, const FPView* __restrict__ views,
                                                             const T* __restrict__ vpad,
                                                             int64_t pad_elems, FPOut o) {
  int u, v, n;
  tile_pixel(rp, u, v, n);
  const int b = blockIdx.z;
  float res = 0.f;
  const bool live = u < rp.nu && v < rp.nv;
  if (live) {
    const RaySetup rs = setup_ray(rp, views[n], u, v);
    SoftSampler<T> smp;
    smp.vol = vpad + b * pad_elems;
    smp.px = rp.nx + 2 * kPad;
    smp.pxy = smp.px * (rp.ny + 2 * kPad);
    smp.mx = (float)rp.nx; smp.my = (float)rp.ny; smp.mz = (float)rp.nz;
    const float val = rs.count > 0 ? ray_sum(smp, rs) * rp.scale : 0.f;
    fp_store(rp, o, n, b, u, v, val, res);
  }
  if (o.abs_sum) block_add_double((double)fabsf(res), o.abs_sum);
}

__global__ void __launch_bounds__(kFPThreads) fp_quad_kernel(RayParams rp, const FPView* __restrict__ views,
                                                             const float4* __restrict__ quads,
                                                             int64_t pad_elems, FPOut o) {
  int u, v, n;
  tile_pixel(rp, u, v, n);
  const int b = blockIdx.z;
  float res = 0.f;
  if (u < rp.nu && v < rp.nv) {
    const RaySetup rs = setup_ray(rp, views[n], u, v);
    QuadSampler smp;
    smp.q = quads + b * pad_elems;
    smp.px = rp.nx + 2 * kPad;
    smp.pxy = smp.px * (rp.ny + 2 * kPad);
    smp.mx = (float)rp.nx; smp.my = (float)rp.ny; smp.mz = (float)rp.nz;
    const float val = rs.count > 0 ? ray_sum(smp, rs) * rp.scale : 0.f;
    fp_store(rp, o, n, b, u, v, val, res);
  }
  if (o.abs_sum) block_add_double((double)fabsf(res), o.abs_sum);
}

__global__ void __launch_bounds__(kFPThreads) fp_tex_kernel(RayParams rp, const FPView* __restrict__ views,
                                                            const cudaTextureObject_t* texs, FPOut o) {
  int u, v, n;
  tile_pixel(rp, u, v, n);
  const int b = blockIdx.z;
  float res = 0.f;
  if (u < rp.nu && v < rp.nv) {
    const RaySetup rs = setup_ray(rp, views[n], u, v, 0.5f, 0.5f);
    TexSampler smp{texs[b]};
    const float val = rs.count > 0 ? ray_sum(smp, rs) * rp.scale : 0.f;
    fp_store(rp, o, n, b, u, v, val, res);
  }
  if (o.abs_sum) block_add_double((double)fabsf(res), o.abs_sum);
}

__global__ void __launch_bounds__(kFPThreads) fp_pair_kernel(RayParams rp, const FPView* __restrict__ views,
                                                             const cudaTextureObject_t* texs,
                                                             FPOut o) {
  int u, v, n;
  tile_pixel(rp, u, v, n);
  const int b = blockIdx.z;
  float res = 0.f;
  if (u < rp.nu && v < rp.nv) {
    const RaySetup rs = setup_ray(rp, views[n], u, v, 0.5f, 0.f);
    PairSampler smp{texs[b], (float)(rp.nz + 2)};
    const float val = rs.count > 0 ? ray_sum(smp, rs) * rp.scale : 0.f;
    fp_store(rp, o, n, b, u, v, val, res);
  }
  if (o.abs_sum) block_add_double((double)fabsf(res), o.abs_sum);
}

__global__ void __launch_bounds__(kFPThreads) fp_pairx_kernel(RayParams rp,
                                                              const FPView* __restrict__ views,
                                                              const uint4* __restrict__ rec,
                                                              int64_t rec_elems, FPOut o) {
  int u, v, n;
  tile_pixel(rp, u, v, n);
  const int b = blockIdx.z;
  float res = 0.f;
  if (u < rp.nu && v < rp.nv) {
    const RaySetup rs = setup_ray(rp, views[n], u, v);
    const PairQuadSampler smp = pair_quad_sampler(rp, rec, rec_elems, b);
    const float val = rs.count > 0 ? ray_sum(smp, rs) * rp.scale : 0.f;
    fp_store(rp, o, n, b, u, v, val, res);
  }
  if (o.abs_sum) block_add_double((double)fabsf(res), o.abs_sum);
}

// The correction pass of a PDHG reconstruction whose texture-filtered z-pair
// operator A (8-bit weights) is corrected by the exact-weight one E: per ray,
// both sums in one march (the texture fetch and the 16-byte record load of a
// sample go to different units), then
//   g_eff = g + (A f - E f),  w = (w + sigma (E f - g)) / (1 + sigma),
//   abs_sum += |E f - g|.
// Each sum has the bits of fp_pair_kernel / fp_pairx_kernel for the ray.
struct RefreshOut {
  const float* g;
  float* w;
  float* g_eff;
  float sigma;
  double* abs_sum;
};

// 4 blocks per SM (64 registers, a 16-byte spill in the ray set-up): 4%
// faster than the 3 blocks its 78 registers would allow.
__global__ void __launch_bounds__(kFPThreads, 4) fp_refresh_kernel(RayParams rp,
                                                                const FPView* __restrict__ views,
                                                                const cudaTextureObject_t* texs,
                                                                const uint4* __restrict__ rec,
                                                                int64_t rec_elems, RefreshOut o) {
  int u, v, n;
  tile_pixel(rp, u, v, n);
  const int b = blockIdx.z;
  float res = 0.f;
  if (u < rp.nu && v < rp.nv) {
    const RaySetup rt = setup_ray(rp, views[n], u, v, 0.5f, 0.f);  // texture coordinates
    const RaySetup rs = setup_ray(rp, views[n], u, v);             // voxel index coordinates
    const PairSampler fast{texs[b], (float)(rp.nz + 2)};
    const PairQuadSampler exact = pair_quad_sampler(rp, rec, rec_elems, b);
    float sf = 0.f, se = 0.f;
    if (rs.count > 0) ray_sum2(fast, rt, exact, rs, sf, se);
    const float a = sf * rp.scale, e = se * rp.scale;
    const int64_t idx = ((int64_t)b * rp.n_views + n) * rp.nu * rp.nv + (int64_t)v * rp.nu + u;
    const float gi = o.g[idx];
    res = e - gi;
    o.g_eff[idx] = gi + (a - e);
    o.w[idx] = (o.w[idx] + o.sigma * res) / (1.f + o.sigma);
  }
  if (o.abs_sum) block_add_double((double)fabsf(res), o.abs_sum);
}

// Writes the exact sampler's records of one volume: record (X, Y, L) =
// words (X, Y), (X+1, Y), (X, Y+1), (X+1, Y+1) of z-pair layer L, word =
// half2(f[L-3], f[L-2]) at padded column (X, Y) = (x + 3, y + 3), zero outside
// the volume. Only records that reach the volume are written (X in [2, nx+2],
// Y in [2, ny+2], L in [2, nz+2]); the others keep the plan's initial zeros.
// A thread owns one record column and kStageLayers layers of it.
template <class Tin>
__global__ void __launch_bounds__(256) stage_pair_quads_kernel(const Tin* __restrict__ in,
                                                               uint4* __restrict__ rec, int nx,
                                                               int ny, int nz);

// Writes the z-pair layers of one volume: layer L = (f[L-2], f[L-1]), zero
// outside [0, nz), to the layered texture and, when `lin` is set, to the
// linear [nz+3][ny][pitch] copy. A thread owns one (x, y) column and a run of
// kStageLayers layers (grid z), so the whole volume is in flight at once.
constexpr int kStageLayers = 16;

template <class Tin>
__global__ void __launch_bounds__(256) stage_pairs_kernel(const Tin* __restrict__ in,
                                                          cudaSurfaceObject_t surf,
                                                          unsigned int* __restrict__ lin, int pitch,
                                                          int64_t lin_plane, int nx, int ny,
                                                          int nz) {
  const int x = blockIdx.x * 32 + (threadIdx.x & 31);
  const int y = blockIdx.y * 8 + (threadIdx.x >> 5);
  if (x >= nx || y >= ny) return;
  const int L0 = blockIdx.z * kStageLayers;
  const int L1 = min(L0 + kStageLayers, nz + 3);
  const int64_t plane = (int64_t)nx * ny;
  const Tin* col = in + (int64_t)y * nx + x;
  auto member = [&](int z) {
    return (z >= 0 && z < nz) ? __float2half_rn(load_as_float(col, z * plane))
                              : __float2half_rn(0.f);
  };
  __half prev = member(L0 - 2);  // f[L-2]
#pragma unroll 4
  for (int L = L0; L < L1; ++L) {
    const __half cur = member(L - 1);  // the new member f[L-1]
    const unsigned int bits = (unsigned int)__half_as_ushort(prev) |
                              ((unsigned int)__half_as_ushort(cur) << 16);
    if (surf) surf2DLayeredwrite(bits, surf, x * 4, y, L);
    if (lin) lin[(int64_t)L * lin_plane + (int64_t)y * pitch + x] = bits;
    prev = cur;
  }
}

template <class Tin>
__global__ void __launch_bounds__(256) stage_pair_quads_kernel(const Tin* __restrict__ in,
                                                               uint4* __restrict__ rec, int nx,
                                                               int ny, int nz) {
  const int X = blockIdx.x * 32 + (threadIdx.x & 31) + kQuadPad - 1;
  const int Y = blockIdx.y * 8 + (threadIdx.x >> 5) + kQuadPad - 1;
  if (X > nx + kQuadPad - 1 || Y > ny + kQuadPad - 1) return;
  const int L0 = kQuadPad - 1 + blockIdx.z * kStageLayers;
  const int L1 = min(L0 + kStageLayers, nz + kQuadPad);
  const int64_t plane = (int64_t)nx * ny;
  const int x = X - kQuadPad, y = Y - kQuadPad;
  // the four columns of the record: (x, y), (x+1, y), (x, y+1), (x+1, y+1)
  const bool in_c[4] = {x >= 0 && y >= 0, x + 1 < nx && y >= 0, x >= 0 && y + 1 < ny,
                        x + 1 < nx && y + 1 < ny};
  const int64_t off[4] = {(int64_t)y * nx + x, (int64_t)y * nx + x + 1,
                          (int64_t)(y + 1) * nx + x, (int64_t)(y + 1) * nx + x + 1};
  auto member = [&](int c, int z) {
    return (in_c[c] && z >= 0 && z < nz) ? __float2half_rn(load_as_float(in + off[c], z * plane))
                                         : __float2half_rn(0.f);
  };
  const int px = nx + 2 * kQuadPad;
  const int64_t rplane = (int64_t)px * (ny + 2 * kQuadPad);
  uint4* col = rec + (int64_t)Y * px + X;
  __half prev[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) prev[c] = member(c, L0 - kQuadPad);
  for (int L = L0; L < L1; ++L) {
    unsigned int wd[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const __half cur = member(c, L - kQuadPad + 1);
      wd[c] = (unsigned int)__half_as_ushort(prev[c]) | ((unsigned int)__half_as_ushort(cur) << 16);
      prev[c] = cur;
    }
    col[L * rplane] = make_uint4(wd[0], wd[1], wd[2], wd[3]);
  }
}

// ---- staging -------------------------------------------------------------------------
template <class Tin, class Tout>
__global__ void stage_pad_kernel(const Tin* __restrict__ in, Tout* __restrict__ out, int nx, int ny,
                                 int nz, int64_t pad_elems) {
  const int64_t vol = (int64_t)nx * ny * nz;
  const int b = blockIdx.y;
  const int px = nx + 2 * kPad, pxy = px * (ny + 2 * kPad);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < vol;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx);
    const int64_t r = i / nx;
    const int y = (int)(r % ny), z = (int)(r / ny);
    const float val = load_as_float(in + b * vol, i);
    store_from_float(out + b * pad_elems, (int64_t)(z + kPad) * pxy + (y + kPad) * px + x + kPad,
                     val);
  }
}

template <class Tin, class Tout>
__global__ void stage_surface_kernel(const Tin* __restrict__ in, cudaSurfaceObject_t surf, int nx,
                                     int ny, int nz) {
  const int64_t vol = (int64_t)nx * ny * nz;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < vol;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx);
    const int64_t r = i / nx;
    const int y = (int)(r % ny), z = (int)(r / ny);
    if constexpr (sizeof(Tout) == 4) {
      surf3Dwrite(load_as_float(in, i), surf, x * 4, y, z);
    } else {  // half texels are written through their bit pattern
      surf3Dwrite(__half_as_ushort(__float2half_rn(load_as_float(in, i))), surf, x * 2, y, z);
    }
  }
}

static int grid_for(int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  return (int)std::min<int64_t>(b, 148 * 16);
}

// Quad records (padded indexing, border kPad) of one volume: only records that
// reach an interior voxel are written; the others stay zero from the plan's
// initial clear. grid: (x, y) tiles of 32 x 8, z planes.
template <class Tin>
__global__ void __launch_bounds__(256) stage_quads_kernel(const Tin* __restrict__ in,
                                                          float4* __restrict__ q, int nx, int ny,
                                                          int nz) {
  const int x = blockIdx.x * 32 + (threadIdx.x & 31) + kPad - 1;  // padded x in [kPad-1, kPad+nx)
  const int y = blockIdx.y * 8 + (threadIdx.x >> 5) + kPad - 1;
  const int z = blockIdx.z + kPad;
  if (x >= kPad + nx || y >= kPad + ny) return;
  const int px = nx + 2 * kPad, py = ny + 2 * kPad;
  const Tin* plane = in + (int64_t)(z - kPad) * nx * ny;
  auto at = [&](int xx, int yy) {
    const int ox = xx - kPad, oy = yy - kPad;
    return (ox >= 0 && ox < nx && oy >= 0 && oy < ny) ? load_as_float(plane, (int64_t)oy * nx + ox)
                                                      : 0.f;
  };
  q[((int64_t)z * py + y) * px + x] = make_float4(at(x, y), at(x + 1, y), at(x, y + 1),
                                                  at(x + 1, y + 1));
}

template <class Tin>
static int stage_volume_soft(Plan* p, const Tin* vol, int batch, cudaStream_t st) {
  const GeomParams& g = p->gp;
  const int64_t vox = (int64_t)g.nx * g.ny * g.nz;
  dim3 grid(grid_for(vox), batch);
  if (p->d_vol_quads) {
    dim3 qg((g.nx + 1 + 31) / 32, (g.ny + 1 + 7) / 8, g.nz);
    for (int b = 0; b < batch; ++b) {
      stage_quads_kernel<Tin><<<qg, 256, 0, st>>>(vol + b * vox, p->d_vol_quads + b * p->pad_elems,
                                                  g.nx, g.ny, g.nz); note_launch();
      DTV_LAUNCH_CHECK();
    }
    return DTV_OK;
  }
  if (p->stage_dtype == DTV_F16) {
    stage_pad_kernel<Tin, __half><<<grid, 256, 0, st>>>(vol, (__half*)p->d_vol_pad, g.nx, g.ny, g.nz,
                                                        p->pad_elems); note_launch();
  }
  else {
    stage_pad_kernel<Tin, float><<<grid, 256, 0, st>>>(vol, (float*)p->d_vol_pad, g.nx, g.ny, g.nz,
                                                       p->pad_elems); note_launch();
  }
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

template <class Tin>
static int stage_volume_tex(Plan* p, const Tin* vol, int batch, cudaStream_t st) {
  const GeomParams& g = p->gp;
  const int64_t vox = (int64_t)g.nx * g.ny * g.nz;
  for (int b = 0; b < batch; ++b) {
    const cudaSurfaceObject_t surf = p->vol_surf[b];
    if (p->stage_dtype == DTV_F16) {
      stage_surface_kernel<Tin, __half><<<grid_for(vox), 256, 0, st>>>(vol + b * vox, surf, g.nx,
                                                                        g.ny, g.nz); note_launch();
    } else {
      stage_surface_kernel<Tin, float><<<grid_for(vox), 256, 0, st>>>(vol + b * vox, surf, g.nx,
                                                                       g.ny, g.nz); note_launch();
    }
    DTV_LAUNCH_CHECK();
  }
  return DTV_OK;
}

template <class Tin>
static int stage_volume_pairs(Plan* p, const Tin* vol, int batch, cudaStream_t st) {
  const GeomParams& g = p->gp;
  const int64_t vox = (int64_t)g.nx * g.ny * g.nz;
  dim3 grid((g.nx + 31) / 32, (g.ny + 7) / 8, (g.nz + 3 + kStageLayers - 1) / kStageLayers);
  for (int b = 0; b < batch; ++b) {
    if (p->d_pair_quad) {  // exact sampler: its records only
      dim3 qg((g.nx + 1 + 31) / 32, (g.ny + 1 + 7) / 8, (g.nz + 1 + kStageLayers - 1) / kStageLayers);
      stage_pair_quads_kernel<Tin><<<qg, 256, 0, st>>>(vol + b * vox,
                                                       p->d_pair_quad + b * p->pair_quad_elems,
                                                       g.nx, g.ny, g.nz); note_launch();
    } else {
      unsigned int* lin =
          p->d_pair_lin ? p->d_pair_lin + (int64_t)b * p->pair_pitch * g.ny * (g.nz + 3) : nullptr;
      stage_pairs_kernel<Tin><<<grid, 256, 0, st>>>(vol + b * vox, p->pair_surf[b], lin,
                                                    p->pair_pitch, (int64_t)p->pair_pitch * g.ny,
                                                    g.nx, g.ny, g.nz); note_launch();
    }
    DTV_LAUNCH_CHECK();
  }
  return DTV_OK;
}

// Writes batch items 0 .. batch-1 of vol into the plan's staged copy.
static int stage_volume(Plan* p, const void* vol, int vol_dtype, int batch, cudaStream_t st) {
  int rc;
  const bool tex = (p->flags & DTV_PLAN_TEX) != 0;
  const bool pairs = (p->flags & (DTV_PLAN_TEX_PAIRS | DTV_PLAN_PAIRS_EXACT)) != 0;
  switch (vol_dtype) {
    case DTV_F32:
      rc = pairs ? stage_volume_pairs(p, (const float*)vol, batch, st)
                 : tex ? stage_volume_tex(p, (const float*)vol, batch, st)
                       : stage_volume_soft(p, (const float*)vol, batch, st);
      break;
    case DTV_F16:
      rc = pairs ? stage_volume_pairs(p, (const __half*)vol, batch, st)
                 : tex ? stage_volume_tex(p, (const __half*)vol, batch, st)
                       : stage_volume_soft(p, (const __half*)vol, batch, st);
      break;
    default:
      rc = pairs ? stage_volume_pairs(p, (const __nv_bfloat16*)vol, batch, st)
                 : tex ? stage_volume_tex(p, (const __nv_bfloat16*)vol, batch, st)
                       : stage_volume_soft(p, (const __nv_bfloat16*)vol, batch, st);
      break;
  }
  return rc;
}

static RayParams plan_ray_params(const Plan* p) {
  RayParams rp = make_ray_params(p->gp);
  rp.ltu = kRayTiles[p->fp_ray_tile][0];
  rp.ltv = kRayTiles[p->fp_ray_tile][1];
  rp.lwu = kRayTiles[p->fp_ray_tile][2];
  rp.band = p->fp_band;
  return rp;
}

int forward_impl(Plan* p, const void* vol, int vol_dtype, int batch, float* out, int epilogue,
                 const float* g, float sigma, double* abs_sum, cudaStream_t st) {
  const GeomParams& gp = p->gp;
  const bool tex = (p->flags & DTV_PLAN_TEX) != 0;
  const bool pairs = (p->flags & (DTV_PLAN_TEX_PAIRS | DTV_PLAN_PAIRS_EXACT)) != 0;
  int rc = stage_volume(p, vol, vol_dtype, batch, st);
  if (rc) return rc;
  const RayParams rp = plan_ray_params(p);
  FPOut o{out, g, sigma, abs_sum, epilogue};
  const int tiles = ((gp.nu + (1 << rp.ltu) - 1) >> rp.ltu) * ((gp.nv + (1 << rp.ltv) - 1) >> rp.ltv);
  dim3 grid(tiles, gp.n_views, batch);
  if (p->flags & DTV_PLAN_TMA) {
    return fp_tma_launch(p, rp, o, batch, st);
  } else if (p->d_pair_quad) {
    fp_pairx_kernel<<<grid, kFPThreads, 0, st>>>(rp, p->d_fpv, p->d_pair_quad, p->pair_quad_elems,
                                                 o); note_launch();
  } else if (pairs) {
    fp_pair_kernel<<<grid, kFPThreads, 0, st>>>(rp, p->d_fpv, p->pair_tex_dev, o); note_launch();
  } else if (tex) {
    fp_tex_kernel<<<grid, kFPThreads, 0, st>>>(rp, p->d_fpv, p->vol_tex_dev, o); note_launch();
  } else if (p->d_vol_quads) {
    fp_quad_kernel<<<grid, kFPThreads, 0, st>>>(rp, p->d_fpv, p->d_vol_quads, p->pad_elems, o); note_launch();
  } else if (p->stage_dtype == DTV_F16) {
    fp_soft_kernel<__half><<<grid, kFPThreads, 0, st>>>(rp, p->d_fpv, (const __half*)p->d_vol_pad,
                                                        p->pad_elems, o); note_launch();
  } else {
    fp_soft_kernel<float><<<grid, kFPThreads, 0, st>>>(rp, p->d_fpv, (const float*)p->d_vol_pad,
                                                       p->pad_elems, o); note_launch();
  }
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

// The correction pass (fp_refresh_kernel) of a DTV_PLAN_TEX_PAIRS plan `fast`
// and a DTV_PLAN_PAIRS_EXACT plan `exact` of the same geometry: each stages
// the volume into its own copy, one launch projects through both.
int forward_refresh_impl(Plan* fast, Plan* exact, const void* vol, int vol_dtype, int batch,
                         const float* g, float sigma, float* w, float* g_eff, double* abs_sum,
                         cudaStream_t st) {
  const GeomParams& gp = fast->gp;
  int rc = stage_volume(fast, vol, vol_dtype, batch, st);
  if (rc) return rc;
  rc = stage_volume(exact, vol, vol_dtype, batch, st);
  if (rc) return rc;
  RayParams rp = plan_ray_params(fast);
  // band-major plans march bands of one tile row here: with the exact
  // sampler's records beside the z-pairs, the narrower slab keeps more of both
  // in L2 (5.66 ms against 5.74 ms with the plan's 4 rows at 256^3 x 64 views)
  if (rp.band > 0) rp.band = 1;
  const int tiles = ((gp.nu + (1 << rp.ltu) - 1) >> rp.ltu) * ((gp.nv + (1 << rp.ltv) - 1) >> rp.ltv);
  dim3 grid(tiles, gp.n_views, batch);
  fp_refresh_kernel<<<grid, kFPThreads, 0, st>>>(rp, fast->d_fpv, fast->pair_tex_dev,
                                                 exact->d_pair_quad, exact->pair_quad_elems,
                                                 RefreshOut{g, w, g_eff, sigma, abs_sum});
  note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

// ---- several plans' forward projections in one launch -----------------------------------
// A flat grid over every plan's (view, 16x16-ray tile) blocks, heaviest plans
// first; a block finds its plan by the blocks' prefix offsets (kernel
// parameters, read uniformly) and runs the z-pair sampler of fp_pair_kernel,
// so each ray's sum is the same computation as a single-plan launch.
struct FPManyItem {
  RayParams rp;
  const FPView* views;
  cudaTextureObject_t tex;
  FPOut o;
  int tiles_u, tiles;
  int block0;
};
struct FPMany {
  FPManyItem it[kManyItems];
  int count;
};
static_assert(sizeof(FPMany) <= 31 * 1024, "kernel parameter space");

__global__ void __launch_bounds__(kFPThreads) fp_pair_many_kernel(const __grid_constant__ FPMany m) {
  int k = 0;
  while (k + 1 < m.count && (int)blockIdx.x >= m.it[k + 1].block0) ++k;
  const FPManyItem& it = m.it[k];
  const int local = (int)blockIdx.x - it.block0;
  const int n = local / it.tiles, tile = local % it.tiles;
  const int t = threadIdx.x, w = t >> 5, l = t & 31;
  const int u = (tile % it.tiles_u) * 16 + (w & 1) * 8 + (l & 7);
  const int v = (tile / it.tiles_u) * 16 + (w >> 1) * 4 + (l >> 3);
  const RayParams& rp = it.rp;
  if (u < rp.nu && v < rp.nv) {
    const RaySetup rs = setup_ray(rp, it.views[n], u, v, 0.5f, 0.f);
    PairSampler smp{it.tex, (float)(rp.nz + 2)};
    const float val = rs.count > 0 ? ray_sum(smp, rs) * rp.scale : 0.f;
    float res;
    fp_store(rp, it.o, n, 0, u, v, val, res);
  }
}

int forward_many_impl(Plan* const* plans, const void* const* vols, int vol_dtype, float* const* outs,
                      int count, int epilogue, const float* const* gs, float sigma,
                      cudaStream_t st) {
  for (int k = 0; k < count; ++k) {
    Plan* p = plans[k];
    int rc;
    switch (vol_dtype) {
      case DTV_F32: rc = stage_volume_pairs(p, (const float*)vols[k], 1, st); break;
      case DTV_F16: rc = stage_volume_pairs(p, (const __half*)vols[k], 1, st); break;
      default: rc = stage_volume_pairs(p, (const __nv_bfloat16*)vols[k], 1, st); break;
    }
    if (rc) return rc;
  }
  // heaviest first (rays x volume edge), so the longest blocks start earliest
  std::vector<int> order(count);
  for (int k = 0; k < count; ++k) order[k] = k;
  auto work = [&](int k) {
    const GeomParams& g = plans[k]->gp;
    return (double)g.n_views * g.nu * g.nv * std::max(g.nx, std::max(g.ny, g.nz));
  };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work(a) > work(b); });
  FPMany m;
  for (int c0 = 0; c0 < count; c0 += kManyItems) {
    const int cnt = std::min(kManyItems, count - c0);
    int64_t blocks = 0;
    for (int j = 0; j < cnt; ++j) {
      const int k = order[c0 + j];
      Plan* p = plans[k];
      const GeomParams& gp = p->gp;
      FPManyItem& it = m.it[j];
      it.rp = make_ray_params(gp);
      it.views = p->d_fpv;
      it.tex = p->pair_tex[0];
      it.o = FPOut{outs[k], gs ? gs[k] : nullptr, sigma, nullptr, epilogue};
      it.tiles_u = (gp.nu + 15) / 16;
      it.tiles = it.tiles_u * ((gp.nv + 15) / 16);
      it.block0 = (int)blocks;
      blocks += (int64_t)it.tiles * gp.n_views;
    }
    DTV_CHECK(blocks < 2147483647LL, "too many blocks for one launch");
    m.count = cnt;
    fp_pair_many_kernel<<<(unsigned)blocks, kFPThreads, 0, st>>>(m);
    note_launch();
    DTV_LAUNCH_CHECK();
  }
  return DTV_OK;
}

// ---- exact transpose of the soft forward projector -------------------------------------
// A^T y scatters every forward sample's value y_r * scale * w_tap onto its 8
// trilinear taps. Instead of 8 global atomics per sample, the volume is cut
// into kAB^3 bricks: one block owns a brick (plus a one-voxel halo) in shared
// memory and, for every view, visits the rays that can reach it -- the
// detector rectangle onto which the brick's box projects, through the view's
// projective map -- rebuilding each ray with the forward projector's own
// set-up and scattering only the samples whose base voxel floor(p) lies in the
// brick (the first brick along an axis also takes base -1, whose upper taps
// are inside). Every contributing sample belongs to exactly one brick, so the
// sum is the exact transpose; each brick then adds its tile to the output once.
// Ray table: rays[2*r] = (p0, count), rays[2*r+1] = (dp, 0) for ray r = (n*nv + v)*nu + u.
__global__ void ray_table_kernel(RayParams rp, const FPView* __restrict__ views,
                                 float4* __restrict__ rays) {
  const int64_t total = (int64_t)rp.n_views * rp.nu * rp.nv;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < total;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int u = (int)(r % rp.nu);
    const int64_t q = r / rp.nu;
    const int v = (int)(q % rp.nv), n = (int)(q / rp.nv);
    const RaySetup rs = setup_ray(rp, views[n], u, v);
    const int c = rs.count > 0 ? rs.count : 0;
    rays[2 * r] = make_float4(c ? rs.p0[0] : 0.f, c ? rs.p0[1] : 0.f, c ? rs.p0[2] : 0.f,
                              __int_as_float(c));
    rays[2 * r + 1] = make_float4(c ? rs.dp[0] : 0.f, c ? rs.dp[1] : 0.f, c ? rs.dp[2] : 0.f, 0.f);
  }
}

int build_ray_table(Plan* p, cudaStream_t st) {
  RayParams rp = make_ray_params(p->gp);
  const int64_t total = (int64_t)rp.n_views * rp.nu * rp.nv;
  ray_table_kernel<<<grid_for(total), 256, 0, st>>>(rp, p->d_fpv, p->d_rays); note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

constexpr int kAB = 16;         // brick edge (voxels)
constexpr int kAT = kAB + 2;    // tile edge: voxels lo-1 .. lo+kAB
constexpr int kAdjThreads = 256;

template <bool kTable>
__global__ void __launch_bounds__(kAdjThreads) adjoint_brick_kernel(
    RayParams rp, const FPView* __restrict__ views, const BPView* __restrict__ pviews,
    const float4* __restrict__ rays, const float* __restrict__ sino, float* __restrict__ out) {
  __shared__ float tile[kAT * kAT * kAT];
  const int nbx = (rp.nx + kAB - 1) / kAB, nby = (rp.ny + kAB - 1) / kAB;
  const int bid = blockIdx.x;
  const int lo[3] = {(bid % nbx) * kAB, ((bid / nbx) % nby) * kAB, (bid / (nbx * nby)) * kAB};
  const int n3[3] = {rp.nx, rp.ny, rp.nz};
  const int b = blockIdx.y;
  for (int i = threadIdx.x; i < kAT * kAT * kAT; i += blockDim.x) tile[i] = 0.f;
  // base voxels owned by this brick: [blo, bhi] per axis
  float blo[3], bhi[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    blo[c] = lo[c] == 0 ? -1.f : (float)lo[c];
    bhi[c] = (float)(min(lo[c] + kAB, n3[c]) - 1);
  }
  __syncthreads();
  const int64_t per_view = (int64_t)rp.nu * rp.nv;
  const float* sb = sino + (int64_t)b * rp.n_views * per_view;
  for (int n = 0; n < rp.n_views; ++n) {
    // detector rectangle of the box [blo, bhi + 1] through view n
    const float* m = pviews[n].m;
    float umin = 3.4e38f, umax = -3.4e38f, vmin = 3.4e38f, vmax = -3.4e38f;
#pragma unroll
    for (int cr = 0; cr < 8; ++cr) {
      const float x = (cr & 1) ? bhi[0] + 1.f : blo[0];
      const float y = (cr & 2) ? bhi[1] + 1.f : blo[1];
      const float z = (cr & 4) ? bhi[2] + 1.f : blo[2];
      const float h = fmaf(m[8], x, fmaf(m[9], y, fmaf(m[10], z, m[11])));
      const float u = fmaf(m[0], x, fmaf(m[1], y, fmaf(m[2], z, m[3]))) / h;
      const float v = fmaf(m[4], x, fmaf(m[5], y, fmaf(m[6], z, m[7]))) / h;
      umin = fminf(umin, u); umax = fmaxf(umax, u);
      vmin = fminf(vmin, v); vmax = fmaxf(vmax, v);
    }
    const int u0 = max(0, (int)fmaxf(floorf(umin) - 1.f, -1.f));
    const int u1 = min(rp.nu - 1, (int)fminf(ceilf(umax) + 1.f, (float)rp.nu));
    const int v0 = max(0, (int)fmaxf(floorf(vmin) - 1.f, -1.f));
    const int v1 = min(rp.nv - 1, (int)fminf(ceilf(vmax) + 1.f, (float)rp.nv));
    if (u0 > u1 || v0 > v1) continue;
    const int w = u1 - u0 + 1;
    const int cnt = w * (v1 - v0 + 1);
    const float* sv = sb + n * per_view;
    for (int r = threadIdx.x; r < cnt; r += blockDim.x) {  // one ray per thread
      const int u = u0 + r % w, v = v0 + r / w;
      const float y = __ldg(sv + (int64_t)v * rp.nu + u) * rp.scale;
      if (y == 0.f) continue;
      RaySetup rs;
      if constexpr (kTable) {
        const int64_t r2 = 2 * (((int64_t)n * rp.nv + v) * rp.nu + u);
        const float4 a = __ldg(rays + r2), d = __ldg(rays + r2 + 1);
        rs.p0[0] = a.x; rs.p0[1] = a.y; rs.p0[2] = a.z;
        rs.count = __float_as_int(a.w);
        rs.dp[0] = d.x; rs.dp[1] = d.y; rs.dp[2] = d.z;
      } else {
        rs = setup_ray(rp, views[n], u, v);
      }
      if (rs.count <= 0) continue;
      // samples that can have their base in this brick (one-sample margin)
      float kl = 0.f, kh = (float)rs.count;
      bool miss = false;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (rs.dp[c] != 0.f) {
          const float ka = (blo[c] - 1.f - rs.p0[c]) / rs.dp[c];
          const float kb = (bhi[c] + 2.f - rs.p0[c]) / rs.dp[c];
          kl = fmaxf(kl, fminf(ka, kb));
          kh = fminf(kh, fmaxf(ka, kb));
        } else if (rs.p0[c] < blo[c] - 1.f || rs.p0[c] >= bhi[c] + 2.f) {
          miss = true;
        }
      }
      if (miss || !(kh >= kl)) continue;
      const int k0 = max(0, (int)floorf(kl) - 1);
      const int k1 = min(rs.count, (int)ceilf(kh) + 1);
      for (int k = k0; k < k1; ++k) {
        const float kf = (float)k;  // positions exactly as the forward projector forms them
        const float x = fmaf(kf, rs.dp[0], rs.p0[0]), yy = fmaf(kf, rs.dp[1], rs.p0[1]),
                    z = fmaf(kf, rs.dp[2], rs.p0[2]);
        const float fx = floorf(x), fy = floorf(yy), fz = floorf(z);
        if (fx < blo[0] || fx > bhi[0] || fy < blo[1] || fy > bhi[1] || fz < blo[2] ||
            fz > bhi[2])
          continue;
        const float ax = x - fx, ay = yy - fy, az = z - fz;
        const int tx = (int)fx - lo[0] + 1, ty = (int)fy - lo[1] + 1, tz = (int)fz - lo[2] + 1;
        float* t = tile + (tz * kAT + ty) * kAT + tx;
        const float wz1 = az * y, wz0 = y - wz1;
        const float w00 = wz0 - ay * wz0, w01 = ay * wz0, w10 = wz1 - ay * wz1, w11 = ay * wz1;
        atomicAdd(t, w00 - ax * w00);
        atomicAdd(t + 1, ax * w00);
        atomicAdd(t + kAT, w01 - ax * w01);
        atomicAdd(t + kAT + 1, ax * w01);
        atomicAdd(t + kAT * kAT, w10 - ax * w10);
        atomicAdd(t + kAT * kAT + 1, ax * w10);
        atomicAdd(t + kAT * kAT + kAT, w11 - ax * w11);
        atomicAdd(t + kAT * kAT + kAT + 1, ax * w11);
      }
    }
  }
  __syncthreads();
  float* ob = out + (int64_t)b * rp.nx * rp.ny * rp.nz;
  for (int i = threadIdx.x; i < kAT * kAT * kAT; i += blockDim.x) {
    const float val = tile[i];
    if (val == 0.f) continue;
    const int tx = i % kAT, ty = (i / kAT) % kAT, tz = i / (kAT * kAT);
    const int gx = lo[0] - 1 + tx, gy = lo[1] - 1 + ty, gz = lo[2] - 1 + tz;
    if (gx < 0 || gy < 0 || gz < 0 || gx >= rp.nx || gy >= rp.ny || gz >= rp.nz) continue;
    atomicAdd(ob + ((int64_t)gz * rp.ny + gy) * rp.nx + gx, val);
  }
}

// ---- the same transpose with vector atomics into cell records ---------------------------
// Record (ix, iy, z) holds the four contributions of a trilinear cell to the
// voxels (ix, iy, z), (ix+1, iy, z), (ix, iy+1, z), (ix+1, iy+1, z); x and y
// run over [-1, n-1] (the cells whose corners reach the volume), z over
// [0, nz-1]. A sample of base cell (ix, iy, iz) adds its bilinear weights
// times (1 - az) to record (ix, iy, iz) and times az to record (ix, iy, iz+1):
// two 16-byte vector reductions into L2 instead of eight scalar atomics. A
// gather pass then sums each voxel's four record entries. Samples whose cell
// lies wholly in the zero border are skipped, as their forward taps read zeros.
__global__ void __launch_bounds__(256) adjoint_cells_kernel(RayParams rp,
                                                            const FPView* __restrict__ views,
                                                            const float4* __restrict__ rays,
                                                            const float* __restrict__ sino,
                                                            float4* __restrict__ cells, int batch,
                                                            int zb0, int zb1) {
  const int64_t per = (int64_t)rp.n_views * rp.nu * rp.nv;
  const int64_t total = per * batch;
  const int cx = rp.nx + 1, cy = rp.ny + 1;
  const int64_t cplane = (int64_t)cx * cy, citem = cplane * rp.nz;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < total;
       r += (int64_t)gridDim.x * blockDim.x) {
    const float val = __ldg(sino + r) * rp.scale;
    if (val == 0.f) continue;
    const int b = (int)(r / per);
    const int64_t ray = r - b * per;
    RaySetup rs;
    if (rays) {
      const float4 a = __ldg(rays + 2 * ray), c = __ldg(rays + 2 * ray + 1);
      rs.p0[0] = a.x; rs.p0[1] = a.y; rs.p0[2] = a.z;
      rs.count = __float_as_int(a.w);
      rs.dp[0] = c.x; rs.dp[1] = c.y; rs.dp[2] = c.z;
    } else {
      const int u = (int)(ray % rp.nu);
      const int64_t q = ray / rp.nu;
      rs = setup_ray(rp, views[(int)(q / rp.nv)], u, (int)(q % rp.nv));
    }
    float4* cb = cells + b * citem;
    // this launch takes the samples whose base z-cell is in [zb0, zb1): their
    // k range from the ray's (monotone) z, widened by one, then tested exactly
    int k0 = 0, k1 = rs.count;
    if (rs.dp[2] != 0.f) {
      const float inv = 1.f / rs.dp[2];
      const float ka = ((float)zb0 - rs.p0[2]) * inv, kb = ((float)zb1 - rs.p0[2]) * inv;
      const float cnt = (float)rs.count;  // clamp in float: the estimates may be huge
      k0 = (int)fminf(fmaxf(floorf(fminf(ka, kb)) - 1.f, 0.f), cnt);
      k1 = (int)fminf(fmaxf(ceilf(fmaxf(ka, kb)) + 1.f, 0.f), cnt);
    }
    for (int k = k0; k < k1; ++k) {
      const float kf = (float)k;
      const float x = fmaf(kf, rs.dp[0], rs.p0[0]), y = fmaf(kf, rs.dp[1], rs.p0[1]),
                  z = fmaf(kf, rs.dp[2], rs.p0[2]);
      const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
      const int ix = (int)fx, iy = (int)fy, iz = (int)fz;
      if (iz < zb0 || iz >= zb1 || ix < -1 || ix > rp.nx - 1 || iy < -1 || iy > rp.ny - 1)
        continue;
      const float ax = x - fx, ay = y - fy, az = z - fz;
      const float bx = 1.f - ax, by = 1.f - ay;
      const int64_t cell = (int64_t)(iy + 1) * cx + (ix + 1);  // within a z-plane
      if (iz >= 0) {
        const float w = val * (1.f - az);
        atomicAdd(cb + iz * cplane + cell,
                  make_float4(w * bx * by, w * ax * by, w * bx * ay, w * ax * ay));
      }
      if (iz + 1 < rp.nz) {
        const float w = val * az;
        atomicAdd(cb + (iz + 1) * cplane + cell,
                  make_float4(w * bx * by, w * ax * by, w * bx * ay, w * ax * ay));
      }
    }
  }
}

__global__ void adjoint_gather_kernel(const float4* __restrict__ cells, float* __restrict__ out,
                                      int nx, int ny, int nz, int batch) {
  const int cx = nx + 1, cy = ny + 1;
  const int64_t vox = (int64_t)nx * ny * nz, total = vox * batch;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int b = (int)(i / vox);
    const int64_t j = i - b * vox;
    const int x = (int)(j % nx);
    const int64_t q = j / nx;
    const int y = (int)(q % ny), z = (int)(q / ny);
    const float4* rz = cells + (int64_t)b * cx * cy * nz + (int64_t)z * cx * cy;
    const float4* r11 = rz + (int64_t)(y + 1) * cx + (x + 1);  // cell (x, y)
    const float4* r01 = r11 - 1;                                // cell (x-1, y)
    const float4* r10 = r11 - cx;                               // cell (x, y-1)
    const float4* r00 = r10 - 1;                                // cell (x-1, y-1)
    out[i] = __ldg(&r11->x) + __ldg(&r01->y) + __ldg(&r10->z) + __ldg(&r00->w);
  }
}

int adjoint_impl(Plan* p, const float* sino, int batch, float* out, cudaStream_t st) {
  const GeomParams& gp = p->gp;
  RayParams rp = make_ray_params(gp);
  const int64_t vox = (int64_t)gp.nx * gp.ny * gp.nz;
  if (p->adjoint_method == 1 && p->d_cells) {
    const int64_t cells = (int64_t)(gp.nx + 1) * (gp.ny + 1) * gp.nz * batch;
    DTV_CUDA_TRY(cudaMemsetAsync(p->d_cells, 0, cells * sizeof(float4), st));
    const int64_t rays = (int64_t)gp.n_views * gp.nu * gp.nv * batch;
    const int grid = (int)std::min<int64_t>((rays + 255) / 256, 148LL * 64);
    // z-slabs of base cells whose records (at most 72 MB over the batch) stay
    // resident in L2 while their samples scatter; base cells run over [-1, nz-1]
    const int64_t plane_bytes = (int64_t)(gp.nx + 1) * (gp.ny + 1) * sizeof(float4) * batch;
    const int slab = (int)std::max<int64_t>(1, (72LL << 20) / plane_bytes);
    for (int zb0 = -1; zb0 < gp.nz; zb0 += slab) {
      const int zb1 = std::min(zb0 + slab, gp.nz);
      adjoint_cells_kernel<<<grid, 256, 0, st>>>(rp, p->d_fpv, p->d_rays, sino, p->d_cells, batch,
                                                 zb0, zb1); note_launch();
      DTV_LAUNCH_CHECK();
    }
    const int ggrid = (int)std::min<int64_t>((vox * batch + 255) / 256, 148LL * 32);
    adjoint_gather_kernel<<<ggrid, 256, 0, st>>>(p->d_cells, out, gp.nx, gp.ny, gp.nz, batch); note_launch();
    DTV_LAUNCH_CHECK();
    return DTV_OK;
  }
  const int bricks = ((gp.nx + kAB - 1) / kAB) * ((gp.ny + kAB - 1) / kAB) *
                     ((gp.nz + kAB - 1) / kAB);
  DTV_CUDA_TRY(cudaMemsetAsync(out, 0, vox * batch * sizeof(float), st));
  if (p->d_rays) {
    adjoint_brick_kernel<true><<<dim3(bricks, batch), kAdjThreads, 0, st>>>(
        rp, p->d_fpv, p->d_bpv, p->d_rays, sino, out); note_launch();
  } else {
    adjoint_brick_kernel<false><<<dim3(bricks, batch), kAdjThreads, 0, st>>>(
        rp, p->d_fpv, p->d_bpv, nullptr, sino, out); note_launch();
  }
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

}  // namespace dtv
