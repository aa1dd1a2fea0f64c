// Voxel-driven FDK-weighted backprojector: every view in one launch, each
// voxel accumulated in registers and written once.
//
// Follows Standard/plug/kernel/backwardKernel.cu:22-53 (+ helper_geometry.h:
// 26-42) and Beijing/plug/kernel/backwardKernel.cu:18-45: per voxel and view,
// the detector coordinate of the voxel's projection is sampled bilinearly
// (border value 0) and weighted by bp_scale * (SDD/L)^power. The reference ran
// one launch per view (or per 21 views), read-modify-writing the whole volume
// each time (backwardKernel.cu:50,101-103). Here the view loop is inside the
// kernel; the projective map of each view (FP64-derived, see geometry.cu)
// gives the detector coordinates with one reciprocal per voxel-view.
#include <algorithm>
#include <type_traits>
#include <vector>
#include <string.h>

#include "common.cuh"

namespace dtv {

struct BPParams {
  int nx, ny, nz, nu, nv, n_views;
  int power;
  int extent;
  float scale;
  int64_t sino_pad_elems;  // one padded view
  int warp;                // columns of a warp and a quad (DTV_TUNE_BP_WARP)
  int vsplit;              // 2: two halves of a block sum the two halves of the views
};

constexpr int kBPTile = 16;  // columns per block edge
// Views whose 3x4 maps travel in one launch's parameters: read through the
// constant cache, they leave the L1/texture pipe to the sinogram fetches.
constexpr int kBPParamViews = 640;
struct BPMaps {
  float m[kBPParamViews][12];
};
static_assert(sizeof(BPMaps) <= 31 * 1024, "kernel parameter space");
// voxels per thread along z: 8, or 4 / 2 where a volume has too few columns
// to fill the GPU (bp_zc); the results do not depend on it
constexpr int kZCMax = 8;
constexpr int64_t kBPWantBlocks = 4 * 148;  // four resident blocks per SM
constexpr int kBPThreads = kBPTile * kBPTile;

struct SoftBil {
  const float* s;  // padded view
  int pu;
  float mu, mv;
  __device__ __forceinline__ float operator()(float u, float v) const {
    const float fu = floorf(u), fv = floorf(v);
    const float au = u - fu, av = v - fv;
    const int iu = (int)fminf(fmaxf(fu, -2.f), mu) + kPad;
    const int iv = (int)fminf(fmaxf(fv, -2.f), mv) + kPad;
    const float* b = s + iv * pu + iu;
    const float v00 = __ldg(b), v01 = __ldg(b + 1), v10 = __ldg(b + pu), v11 = __ldg(b + pu + 1);
    const float c0 = fmaf(au, v01 - v00, v00), c1 = fmaf(au, v11 - v10, v10);
    return fmaf(av, c1 - c0, c0);
  }
};

// The same bilinear sample from 16-byte records of the padded view (exact
// plans): record (U, V) = (s(U, V), s(U+1, V), s(U, V+1), s(U+1, V+1)) at
// padded indices, one 128-bit load per voxel-view.
struct QuadBil {
  const float4* q;  // records of the view
  int pu;
  float mu, mv;
  __device__ __forceinline__ float operator()(float u, float v) const {
    const float fu = floorf(u), fv = floorf(v);
    const float au = u - fu, av = v - fv;
    const int iu = (int)fminf(fmaxf(fu, -2.f), mu) + kPad;
    const int iv = (int)fminf(fmaxf(fv, -2.f), mv) + kPad;
    const float4 r = __ldg(q + iv * pu + iu);
    const float c0 = fmaf(au, r.y - r.x, r.x), c1 = fmaf(au, r.w - r.z, r.z);
    return fmaf(av, c1 - c0, c0);
  }
};

// Where the backprojector's detector values come from. kSrcBoth: the texture
// and the quad records of the same sinogram, two sums per voxel (the
// correction pass of a texture-filtered plan against an exact one).
enum BPSource { kSrcSoft = 0, kSrcTex = 1, kSrcQuad = 2, kSrcBoth = 3 };

// Where a block's sums go: out = base + sum (out = sum when base is NULL; base
// may be out). kSrcBoth: out takes the quad-record sum E, and
// diff = diff_base + (E - T) with T the texture sum.
struct BPOut {
  float* out;
  const float* base;
  float* diff;
  const float* diff_base;
};

// kZAff: every view's u and h are independent of z (a detector parallel to the
// rotation axis, as in the circular orbits), so per column and view the kernel
// computes u, 1/h and the weight once and each voxel costs one FMA for v, one
// fetch and one FMA.
// Where a view's 3x4 map comes from: the launch parameters (one chunk of
// views) or the plan's device table.
struct ParamMaps {
  const BPMaps* m;
  __device__ __forceinline__ const float* row(int jn) const { return m->m[jn]; }
};
struct TableMaps {
  const BPView* v;  // first view of the chunk
  __device__ __forceinline__ const float* row(int jn) const { return v[jn].m; }
};

// One block's columns: tile `tile` of 16x16 (x, y) columns, z-chunk `zc` of ZC
// voxels, views n0 .. n0 + n_chunk - 1. With bp.vsplit == 2 (volumes too small
// to fill the GPU otherwise) the tile is 16x8 columns and the block's two
// halves take the first and the second half of the views; the second half's
// sums are added to the first's through shared memory, in that order, so the
// result is deterministic.
template <int kSrc, bool kZAff, int ZC, bool kSplit, class Maps>
__device__ __forceinline__ void bp_columns(const BPParams& bp, const Maps& maps, int n0, int n_chunk,
                                           const float* __restrict__ spad, cudaTextureObject_t tex,
                                           const BPOut& dst, int tile, int zc) {
  const int tiles_x = (bp.nx + kBPTile - 1) / kBPTile;
  // this thread's column in the 16 x 16 tile; a warp covers 16 x 2, 8 x 4 or
  // 4 x 8 columns (the narrower, the fewer detector rows' cache sectors one
  // fetch instruction touches when a voxel spans several pixels)
  const int t = (int)threadIdx.x;
  constexpr bool split = kSplit;  // bp.vsplit == 2, chosen by the launch
  const int half = split ? t >> 7 : 0;
  int li, lj;
  if constexpr (split) {
    li = t & 15;
    lj = (t & 127) >> 4;
  } else if (bp.warp >= 3) {
    // quads (4 consecutive lanes) of 2 x 2 columns; a warp of 8 quads covers
    // 8 x 4 (warp 3) or 4 x 8 (warp 4) columns
    const int q = (t >> 2) & 7, qi = t & 1, qj = (t >> 1) & 1, w = t >> 5;
    if (bp.warp == 3) {
      li = ((q & 3) << 1 | qi) | ((w & 1) << 3);
      lj = ((q >> 2) << 1 | qj) | ((w >> 1) << 2);
    } else {
      li = ((q & 1) << 1 | qi) | ((w & 3) << 2);
      lj = ((q >> 1) << 1 | qj) | ((w >> 2) << 3);
    }
  } else if (bp.warp == 1) {
    li = (t & 7) | (((t >> 5) & 1) << 3);
    lj = ((t >> 3) & 3) | ((t >> 6) << 2);
  } else if (bp.warp == 2) {
    li = (t & 3) | (((t >> 5) & 3) << 2);
    lj = ((t >> 2) & 7) | ((t >> 7) << 3);
  } else {
    li = t & 15;
    lj = t >> 4;
  }
  const int i = (tile % tiles_x) * kBPTile + li;
  const int j = (tile / tiles_x) * (split ? kBPTile / 2 : kBPTile) + lj;
  const int k0 = zc * ZC;
  const bool valid = i < bp.nx && j < bp.ny;
  if (!valid && !split) return;  // the split halves meet at a barrier below
  // this thread's views: all of the chunk, or one half of it
  const int hv = (n_chunk + 1) / 2;
  const int jn0 = split ? half * hv : 0;
  const int jn1 = !valid ? jn0 : (split && half == 0 ? hv : n_chunk);
  constexpr bool kBoth = kSrc == kSrcBoth;
  float acc[ZC], act[kBoth ? ZC : 1];
#pragma unroll
  for (int z = 0; z < ZC; ++z) acc[z] = 0.f;
#pragma unroll
  for (int z = 0; z < (kBoth ? ZC : 1); ++z) act[z] = 0.f;
  const float fi = (float)i, fj = (float)j;
  const int pu = bp.nu + 2 * kPad;
  const float mu = (float)bp.nu, mv = (float)bp.nv;
  for (int jn = jn0; jn < jn1; ++jn) {
    const int n = n0 + jn;
    const float* w = maps.row(jn);
    const float m0 = w[0], m1 = w[1], m2 = w[2], m3 = w[3];
    const float m4 = w[4], m5 = w[5], m6 = w[6], m7 = w[7];
    const float m8 = w[8], m9 = w[9], m10 = w[10], m11 = w[11];
    const float bu = fmaf(m0, fi, fmaf(m1, fj, m3));
    const float bv = fmaf(m4, fi, fmaf(m5, fj, m7));
    const float bh = fmaf(m8, fi, fmaf(m9, fj, m11));
    using Smp = typename std::conditional<kSrc == kSrcQuad || kBoth, QuadBil, SoftBil>::type;
    Smp smp;
    if constexpr (kSrc == kSrcQuad || kBoth)
      smp = QuadBil{reinterpret_cast<const float4*>(spad) + (int64_t)n * bp.sino_pad_elems, pu,
                    mu, mv};
    else
      smp = SoftBil{spad + (int64_t)n * bp.sino_pad_elems, pu, mu, mv};
    if constexpr (kZAff) {
      const float rh = __frcp_rn(bh);
      // v from the absolute slice index: the same bits for every z-chunking.
      // Coordinates are rounded explicitly (no contraction into FMAs), so
      // every kernel instance samples a voxel-view at the same position.
      const float u = __fmul_rn(bu, rh), vb = __fmul_rn(bv, rh), dv = __fmul_rn(m6, rh);
      const float tu = __fadd_rn(u, 0.5f);  // texture coordinate (texel centres at i + 1/2)
      float wgt = bp.scale;
      if (bp.power == 2) wgt *= rh * rh;
      else if (bp.power == 1) wgt *= rh;
      const bool col_out = bp.extent && (tu < -1.f || tu > bp.nx + 1.f);
      if (col_out) continue;
#pragma unroll
      for (int z = 0; z < ZC; ++z) {
        const float v = fmaf((float)(k0 + z), dv, vb);
        const float tv = __fadd_rn(v, 0.5f);
        float wz = wgt;
        if (bp.extent && (tv < -1.f || tv > bp.ny + 1.f)) wz = 0.f;
        float val;
        if constexpr (kSrc == kSrcTex) val = tex2DLayered<float>(tex, tu, tv, n);
        else val = smp(u, v);
        acc[z] = fmaf(val, wz, acc[z]);
        if constexpr (kBoth) act[z] = fmaf(tex2DLayered<float>(tex, tu, tv, n), wz, act[z]);
      }
    } else {
#pragma unroll
      for (int z = 0; z < ZC; ++z) {
        const float fk = (float)(k0 + z);
        const float h = fmaf(m10, fk, bh);
        const float rh = __frcp_rn(h);
        const float u = __fmul_rn(fmaf(m2, fk, bu), rh);
        const float v = __fmul_rn(fmaf(m6, fk, bv), rh);
        const float tu = __fadd_rn(u, 0.5f), tv = __fadd_rn(v, 0.5f);
        float wgt = bp.scale;
        if (bp.power == 2) wgt *= rh * rh;
        else if (bp.power == 1) wgt *= rh;
        if (bp.extent && (tu < -1.f || tu > bp.nx + 1.f || tv < -1.f || tv > bp.ny + 1.f))
          wgt = 0.f;
        float val;
        if constexpr (kSrc == kSrcTex) val = tex2DLayered<float>(tex, tu, tv, n);
        else val = smp(u, v);
        acc[z] = fmaf(val, wgt, acc[z]);
        if constexpr (kBoth) act[z] = fmaf(tex2DLayered<float>(tex, tu, tv, n), wgt, act[z]);
      }
    }
  }
  if constexpr (split) {
    // the second half hands its sums to the first: acc = first + second
    // (dynamic shared memory, given only to split launches)
    extern __shared__ float red[];
    const int lt = t & 127;
    if (half == 1) {
#pragma unroll
      for (int z = 0; z < ZC; ++z) {
        red[z * 128 + lt] = acc[z];
        if constexpr (kBoth) red[(ZC + z) * 128 + lt] = act[z];
      }
    }
    __syncthreads();
    if (half == 1 || !valid) return;
#pragma unroll
    for (int z = 0; z < ZC; ++z) {
      acc[z] = acc[z] + red[z * 128 + lt];
      if constexpr (kBoth) act[z] = act[z] + red[(ZC + z) * 128 + lt];
    }
  }
  const int64_t plane = (int64_t)bp.nx * bp.ny;
  const int64_t col = (int64_t)j * bp.nx + i;
#pragma unroll
  for (int z = 0; z < ZC; ++z) {
    const int k = k0 + z;
    if (k < bp.nz) {
      const int64_t e = col + k * plane;
      dst.out[e] = dst.base ? dst.base[e] + acc[z] : acc[z];
      if constexpr (kBoth) {
        const float d = acc[z] - act[z];
        dst.diff[e] = dst.diff_base ? dst.diff_base[e] + d : d;
      }
    }
  }
}

template <int kSrc, bool kZAff, int ZC, bool kSplit>
__global__ void __launch_bounds__(kBPThreads) bp_kernel(BPParams bp, const __grid_constant__ BPMaps maps,
                                                        int n0, int n_chunk,
                                                        const float* __restrict__ spad,
                                                        cudaTextureObject_t tex, BPOut dst) {
  bp_columns<kSrc, kZAff, ZC, kSplit>(bp, ParamMaps{&maps}, n0, n_chunk, spad, tex, dst,
                                      (int)blockIdx.x, (int)blockIdx.y);
}

// Records of the exact backprojector: record (U, V) of view n from the four
// detector values (u, v) = (U - 2 .. U - 1, V - 2 .. V - 1), zero outside the
// view. Only records that reach the view (U in [1, nu+1], V in [1, nv+1]) are
// written; the rest keep the plan's initial zeros.
__global__ void stage_sino_quad_kernel(const float* __restrict__ in, float4* __restrict__ out,
                                       int nu, int nv, int n_views) {
  const int U = blockIdx.x * 32 + (threadIdx.x & 31) + 1;
  const int V = blockIdx.y * 8 + (threadIdx.x >> 5) + 1;
  const int n = blockIdx.z;
  if (U > nu + 1 || V > nv + 1 || n >= n_views) return;
  const float* s = in + (int64_t)n * nu * nv;
  const int u = U - kPad, v = V - kPad;
  auto at = [&](int uu, int vv) {
    return (uu >= 0 && uu < nu && vv >= 0 && vv < nv) ? __ldg(s + (int64_t)vv * nu + uu) : 0.f;
  };
  out[(int64_t)n * (nu + 2 * kPad) * (nv + 2 * kPad) + (int64_t)V * (nu + 2 * kPad) + U] =
      make_float4(at(u, v), at(u + 1, v), at(u, v + 1), at(u + 1, v + 1));
}

__global__ void stage_sino_pad_kernel(const float* __restrict__ in, float* __restrict__ out, int nu,
                                      int nv, int64_t n_views_total) {
  const int pu = nu + 2 * kPad;
  const int64_t per = (int64_t)nu * nv, pper = (int64_t)pu * (nv + 2 * kPad);
  const int64_t total = per * n_views_total;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t n = i / per;
    const int r = (int)(i - n * per);
    const int u = r % nu, v = r / nu;
    out[n * pper + (int64_t)(v + kPad) * pu + u + kPad] = __ldg(in + i);
  }
}

// Voxels per thread along z: the largest of 8, 4, 2 whose grid has
// kBPWantBlocks blocks (2 if none has).
template <class BlocksFor>
static int bp_zc(BlocksFor blocks_for) {
  for (int c = kZCMax; c > 2; c /= 2)
    if (blocks_for(c) >= kBPWantBlocks) return c;
  return 2;
}

template <int kSrc, bool kZAff, bool kSplit>
static void launch_bp_split(int zc, dim3 grid, cudaStream_t st, const BPParams& bp,
                            const BPMaps& maps, int n0, int cnt, const float* sp,
                            cudaTextureObject_t tx, const BPOut& dst) {
  // split launches: the second half's sums of each voxel in shared memory
  const size_t sm = kSplit ? (size_t)(kSrc == kSrcBoth ? 2 : 1) * zc * 128 * sizeof(float) : 0;
  if (zc == 8)
    bp_kernel<kSrc, kZAff, 8, kSplit><<<grid, kBPThreads, sm, st>>>(bp, maps, n0, cnt, sp, tx, dst);
  else if (zc == 4)
    bp_kernel<kSrc, kZAff, 4, kSplit><<<grid, kBPThreads, sm, st>>>(bp, maps, n0, cnt, sp, tx, dst);
  else
    bp_kernel<kSrc, kZAff, 2, kSplit><<<grid, kBPThreads, sm, st>>>(bp, maps, n0, cnt, sp, tx, dst);
}

template <int kSrc, bool kZAff>
static void launch_bp_zc(int zc, dim3 grid, cudaStream_t st, const BPParams& bp,
                         const BPMaps& maps, int n0, int cnt, const float* sp,
                         cudaTextureObject_t tx, const BPOut& dst) {
  if (bp.vsplit == 2)
    launch_bp_split<kSrc, kZAff, true>(zc, grid, st, bp, maps, n0, cnt, sp, tx, dst);
  else
    launch_bp_split<kSrc, kZAff, false>(zc, grid, st, bp, maps, n0, cnt, sp, tx, dst);
}

template <int kSrc>
static void launch_bp_src(bool zaff, int zc, dim3 grid, cudaStream_t st, const BPParams& bp,
                          const BPMaps& maps, int n0, int cnt, const float* sp,
                          cudaTextureObject_t tx, const BPOut& dst) {
  if (zaff) launch_bp_zc<kSrc, true>(zc, grid, st, bp, maps, n0, cnt, sp, tx, dst);
  else launch_bp_zc<kSrc, false>(zc, grid, st, bp, maps, n0, cnt, sp, tx, dst);
}

static void launch_bp(int src, bool zaff, int zc, dim3 grid, cudaStream_t st, const BPParams& bp,
                      const BPMaps& maps, int n0, int cnt, const float* sp, cudaTextureObject_t tx,
                      const BPOut& dst) {
  switch (src) {
    case kSrcTex: launch_bp_src<kSrcTex>(zaff, zc, grid, st, bp, maps, n0, cnt, sp, tx, dst); break;
    case kSrcQuad: launch_bp_src<kSrcQuad>(zaff, zc, grid, st, bp, maps, n0, cnt, sp, tx, dst); break;
    case kSrcBoth: launch_bp_src<kSrcBoth>(zaff, zc, grid, st, bp, maps, n0, cnt, sp, tx, dst); break;
    default: launch_bp_src<kSrcSoft>(zaff, zc, grid, st, bp, maps, n0, cnt, sp, tx, dst); break;
  }
}

// Column tiles of 16 x 16, or of 16 x 8 where the plan splits its views.
static int bp_tiles(const GeomParams& gp, int vsplit) {
  const int th = vsplit == 2 ? kBPTile / 2 : kBPTile;
  return ((gp.nx + kBPTile - 1) / kBPTile) * ((gp.ny + th - 1) / th);
}

// A volume whose 16 x 16 column tiles cannot give four blocks per SM even with
// two slices per thread splits its views between two halves of each block
// (twice the blocks, half the views each). A property of the plan's geometry
// alone, so every launch of the plan sums its views in the same order.
static int bp_vsplit(const GeomParams& gp) {
  return gp.n_views >= 2 && (int64_t)bp_tiles(gp, 1) * ((gp.nz + 1) / 2) < kBPWantBlocks ? 2 : 1;
}

static BPParams plan_bp_params(const Plan* p) {
  const GeomParams& gp = p->gp;
  BPParams bp;
  bp.nx = gp.nx; bp.ny = gp.ny; bp.nz = gp.nz;
  bp.nu = gp.nu; bp.nv = gp.nv; bp.n_views = gp.n_views;
  bp.power = gp.bp_power;
  bp.extent = gp.bp_extent;
  bp.scale = (float)gp.bp_scale;
  bp.sino_pad_elems = (int64_t)(gp.nu + 2 * kPad) * (gp.nv + 2 * kPad);
  bp.warp = p->bp_warp;
  bp.vsplit = bp_vsplit(gp);
  return bp;
}

// Copies one batch item's sinogram into the plan's staged form: the layered
// texture (texture plans), the quad records (exact plans) or the padded array.
static int stage_sino(Plan* p, const float* sino, cudaStream_t st) {
  const GeomParams& gp = p->gp;
  if (p->sino_tex != nullptr) {
    cudaMemcpy3DParms cp;
    memset(&cp, 0, sizeof(cp));
    cp.srcPtr = make_cudaPitchedPtr((void*)sino, gp.nu * sizeof(float), gp.nu, gp.nv);
    cp.dstArray = p->sino_arrays[0];
    cp.extent = make_cudaExtent(gp.nu, gp.nv, gp.n_views);
    cp.kind = cudaMemcpyDeviceToDevice;
    DTV_CUDA_TRY(cudaMemcpy3DAsync(&cp, st));
  } else if (p->d_sino_quad != nullptr) {
    dim3 qg((gp.nu + 1 + 31) / 32, (gp.nv + 1 + 7) / 8, gp.n_views);
    stage_sino_quad_kernel<<<qg, 256, 0, st>>>(sino, p->d_sino_quad, gp.nu, gp.nv, gp.n_views);
    note_launch();
    DTV_LAUNCH_CHECK();
  } else {
    const int64_t per_item = (int64_t)gp.nu * gp.nv * gp.n_views;
    stage_sino_pad_kernel<<<(int)std::min<int64_t>((per_item + 255) / 256, 148 * 16), 256, 0,
                            st>>>(sino, p->d_sino_pad, gp.nu, gp.nv, gp.n_views);
    note_launch();
    DTV_LAUNCH_CHECK();
  }
  return DTV_OK;
}

static dim3 bp_grid(const GeomParams& gp, int* zc_out) {
  const int tiles = bp_tiles(gp, bp_vsplit(gp));
  const int zc = bp_zc([&](int c) { return (int64_t)tiles * ((gp.nz + c - 1) / c); });
  *zc_out = zc;
  return dim3(tiles, (gp.nz + zc - 1) / zc);
}

// The views in chunks of kBPParamViews (their maps travel in the launch
// parameters); later chunks add onto the first one's result.
static int bp_view_chunks(const Plan* p, int src, const float* sp, cudaTextureObject_t tx,
                          BPOut dst, cudaStream_t st) {
  const GeomParams& gp = p->gp;
  const BPParams bp = plan_bp_params(p);
  int zc;
  const dim3 grid = bp_grid(gp, &zc);
  BPMaps maps;
  for (int n0 = 0; n0 < gp.n_views; n0 += kBPParamViews) {
    const int cnt = std::min(kBPParamViews, gp.n_views - n0);
    for (int j = 0; j < cnt; ++j) memcpy(maps.m[j], p->h_bpv[n0 + j].m, sizeof(maps.m[j]));
    if (n0 > 0) {
      dst.base = dst.out;
      dst.diff_base = dst.diff;
    }
    launch_bp(src, p->bp_zaffine != 0, zc, grid, st, bp, maps, n0, cnt, sp, tx, dst);
    note_launch();
    DTV_LAUNCH_CHECK();
  }
  return DTV_OK;
}

int backward_impl(Plan* p, const float* sino, int batch, const float* base, float* out,
                  cudaStream_t st) {
  const GeomParams& gp = p->gp;
  const bool tex = p->sino_tex != nullptr;      // allocated for the texture plans
  const bool quad = p->d_sino_quad != nullptr;  // the exact plans
  const int64_t per_item = (int64_t)gp.nu * gp.nv * gp.n_views;
  const int64_t vox = (int64_t)gp.nx * gp.ny * gp.nz;
  for (int b = 0; b < batch; ++b) {
    int rc = stage_sino(p, sino + b * per_item, st);
    if (rc) return rc;
    const cudaTextureObject_t tx = tex ? p->sino_tex[0] : 0;
    const float* sp = tex ? nullptr
                          : quad ? reinterpret_cast<const float*>(p->d_sino_quad) : p->d_sino_pad;
    const int src = tex ? kSrcTex : quad ? kSrcQuad : kSrcSoft;
    rc = bp_view_chunks(p, src, sp, tx, BPOut{out + b * vox, base ? base + b * vox : nullptr,
                                              nullptr, nullptr}, st);
    if (rc) return rc;
  }
  return DTV_OK;
}

// The correction pass of a texture plan `fast` against an exact plan `exact`
// of the same geometry: out = BP_exact(sino), e_b = out - BP_fast(sino), one
// launch reading both plans' staged copies of the sinogram.
int backward_refresh_impl(Plan* fast, Plan* exact, const float* sino, int batch, float* out,
                          float* e_b, cudaStream_t st) {
  const GeomParams& gp = fast->gp;
  const int64_t per_item = (int64_t)gp.nu * gp.nv * gp.n_views;
  const int64_t vox = (int64_t)gp.nx * gp.ny * gp.nz;
  for (int b = 0; b < batch; ++b) {
    int rc = stage_sino(fast, sino + b * per_item, st);
    if (rc) return rc;
    rc = stage_sino(exact, sino + b * per_item, st);
    if (rc) return rc;
    rc = bp_view_chunks(fast, kSrcBoth, reinterpret_cast<const float*>(exact->d_sino_quad),
                        fast->sino_tex[0], BPOut{out + b * vox, nullptr, e_b + b * vox, nullptr},
                        st);
    if (rc) return rc;
  }
  return DTV_OK;
}

// ---- several plans' backprojections in one launch ---------------------------------------
// A flat grid over every plan's (column tile, z-chunk) blocks; a block finds
// its plan by the blocks' prefix offsets (kernel parameters, read uniformly).
// The plans' maps travel in the launch parameters too, up to kBPManyViews
// views per launch, so they are read through the constant cache as in the
// single-plan launch (maps read from device memory go through the same L1
// path as the texture fetches: 14% slower on 16 volumes of 96^3-256^3). A
// plan with more views than that reads its maps from its device table.
// Texture plans only; each item's sinogram is first copied into its plan's
// layered array.
constexpr int kBPManyViews = 560;
struct BPManyItem {
  BPParams bp;
  const BPView* views;  // device table (used when map0 < 0)
  cudaTextureObject_t tex;
  float* out;
  int tiles;
  int block0;
  int zaffine;
  int map0;  // first row of this plan's maps in BPMany::m, or -1
};
struct BPMany {
  BPManyItem it[kManyItems];
  int count;
  float m[kBPManyViews][12];
};
static_assert(sizeof(BPMany) <= 31 * 1024, "kernel parameter space");

// Rows of maps in a launch's parameters.
struct RowMaps {
  const float (*r)[12];
  __device__ __forceinline__ const float* row(int jn) const { return r[jn]; }
};

// Every item of one launch has the same bp.vsplit (kSplit).
template <int ZC, bool kSplit>
__global__ void __launch_bounds__(kBPThreads) bp_many_kernel(const __grid_constant__ BPMany m,
                                                             int accumulate) {
  int k = 0;
  while (k + 1 < m.count && (int)blockIdx.x >= m.it[k + 1].block0) ++k;
  const BPManyItem& it = m.it[k];
  const int local = (int)blockIdx.x - it.block0;
  const int tile = local % it.tiles, zc = local / it.tiles;
  const BPOut dst{it.out, accumulate ? it.out : nullptr, nullptr, nullptr};
  if (it.map0 >= 0) {
    const RowMaps rows{m.m + it.map0};
    if (it.zaffine)
      bp_columns<kSrcTex, true, ZC, kSplit>(it.bp, rows, 0, it.bp.n_views, nullptr, it.tex, dst, tile, zc);
    else
      bp_columns<kSrcTex, false, ZC, kSplit>(it.bp, rows, 0, it.bp.n_views, nullptr, it.tex, dst, tile, zc);
  } else if (it.zaffine) {
    bp_columns<kSrcTex, true, ZC, kSplit>(it.bp, TableMaps{it.views}, 0, it.bp.n_views, nullptr, it.tex,
                                  dst, tile, zc);
  } else {
    bp_columns<kSrcTex, false, ZC, kSplit>(it.bp, TableMaps{it.views}, 0, it.bp.n_views, nullptr, it.tex,
                                   dst, tile, zc);
  }
}

int backward_many_impl(Plan* const* plans, const float* const* sinos, float* const* outs, int count,
                       int accumulate, cudaStream_t st) {
  BPMany m;
  // plans that split their views run in launches of their own
  std::vector<int> ord;
  for (int split = 1; split <= 2; ++split)
    for (int k = 0; k < count; ++k)
      if (bp_vsplit(plans[k]->gp) == split) ord.push_back(k);
  int c0 = 0;
  while (c0 < count) {
    // this launch's plans: up to kManyItems of one split kind, whose maps fit
    // the parameters (a plan with more views than fit at all takes its maps
    // from its table)
    const int kind = bp_vsplit(plans[ord[c0]]->gp);
    int cnt = 0, rows = 0;
    while (c0 + cnt < count && cnt < kManyItems) {
      const GeomParams& g = plans[ord[c0 + cnt]]->gp;
      if (bp_vsplit(g) != kind) break;
      const int nv = g.n_views;
      if (nv <= kBPManyViews && rows + nv > kBPManyViews) break;
      if (nv <= kBPManyViews) rows += nv;
      ++cnt;
    }
    // one z-chunk length for the whole launch, from its total column tiles
    const int zc = bp_zc([&](int c) {
      int64_t b = 0;
      for (int k = 0; k < cnt; ++k) {
        const GeomParams& gp = plans[ord[c0 + k]]->gp;
        b += (int64_t)bp_tiles(gp, bp_vsplit(gp)) * ((gp.nz + c - 1) / c);
      }
      return b;
    });
    int64_t blocks = 0;
    int row = 0;
    for (int k = 0; k < cnt; ++k) {
      Plan* p = plans[ord[c0 + k]];
      const GeomParams& gp = p->gp;
      cudaMemcpy3DParms cp;
      memset(&cp, 0, sizeof(cp));
      cp.srcPtr = make_cudaPitchedPtr((void*)sinos[ord[c0 + k]], gp.nu * sizeof(float), gp.nu, gp.nv);
      cp.dstArray = p->sino_arrays[0];
      cp.extent = make_cudaExtent(gp.nu, gp.nv, gp.n_views);
      cp.kind = cudaMemcpyDeviceToDevice;
      DTV_CUDA_TRY(cudaMemcpy3DAsync(&cp, st));
      BPManyItem& it = m.it[k];
      it.bp = plan_bp_params(p);
      it.bp.sino_pad_elems = 0;
      it.views = p->d_bpv;
      it.tex = p->sino_tex[0];
      it.out = outs[ord[c0 + k]];
      it.tiles = bp_tiles(gp, it.bp.vsplit);
      it.block0 = (int)blocks;
      it.zaffine = p->bp_zaffine;
      it.map0 = -1;
      if (gp.n_views <= kBPManyViews) {
        it.map0 = row;
        for (int j = 0; j < gp.n_views; ++j) memcpy(m.m[row + j], p->h_bpv[j].m, sizeof(m.m[0]));
        row += gp.n_views;
      }
      blocks += (int64_t)it.tiles * ((gp.nz + zc - 1) / zc);
    }
    DTV_CHECK(blocks < 2147483647LL, "too many blocks for one launch");
    m.count = cnt;
    const unsigned nb = (unsigned)blocks;
    if (kind == 2) {
      const size_t sm = (size_t)zc * 128 * sizeof(float);
      if (zc == 8) bp_many_kernel<8, true><<<nb, kBPThreads, sm, st>>>(m, accumulate);
      else if (zc == 4) bp_many_kernel<4, true><<<nb, kBPThreads, sm, st>>>(m, accumulate);
      else bp_many_kernel<2, true><<<nb, kBPThreads, sm, st>>>(m, accumulate);
    } else {
      if (zc == 8) bp_many_kernel<8, false><<<nb, kBPThreads, 0, st>>>(m, accumulate);
      else if (zc == 4) bp_many_kernel<4, false><<<nb, kBPThreads, 0, st>>>(m, accumulate);
      else bp_many_kernel<2, false><<<nb, kBPThreads, 0, st>>>(m, accumulate);
    }
    note_launch();
    DTV_LAUNCH_CHECK();
    c0 += cnt;
  }
  return DTV_OK;
}

}  // namespace dtv
