// Internal definitions shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include <string>

#include "dtv_b200.h"

namespace dtv {

// ---- error reporting -------------------------------------------------------------
// Host-side count of kernel launches issued by the library (dtv_launch_count).
void note_launch();
void set_error(const char* fmt, ...);
int fail(int code, const char* fmt, ...);

#define DTV_CUDA_TRY(expr)                                                             \
  do {                                                                                 \
    cudaError_t _e = (expr);                                                           \
    if (_e != cudaSuccess)                                                             \
      return ::dtv::fail(DTV_ERR_CUDA, "%s failed: %s (%s:%d)", #expr,                 \
                         cudaGetErrorString(_e), __FILE__, __LINE__);                  \
  } while (0)

#define DTV_CHECK(cond, ...)                                                           \
  do {                                                                                 \
    if (!(cond)) return ::dtv::fail(DTV_ERR_INVALID, __VA_ARGS__);                     \
  } while (0)

// Launch-error check right after a kernel launch.
#define DTV_LAUNCH_CHECK()                                                             \
  do {                                                                                 \
    cudaError_t _e = cudaGetLastError();                                               \
    if (_e != cudaSuccess)                                                             \
      return ::dtv::fail(DTV_ERR_CUDA, "kernel launch failed: %s (%s:%d)",             \
                         cudaGetErrorString(_e), __FILE__, __LINE__);                  \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// ---- storage types -------------------------------------------------------------------
__device__ __forceinline__ float load_as_float(const float* p, int64_t i) { return __ldg(p + i); }
__device__ __forceinline__ float load_as_float(const __half* p, int64_t i) {
  return __half2float(p[i]);
}
__device__ __forceinline__ float load_as_float(const __nv_bfloat16* p, int64_t i) {
  return __bfloat162float(p[i]);
}
__device__ __forceinline__ void store_from_float(float* p, int64_t i, float v) { p[i] = v; }
__device__ __forceinline__ void store_from_float(__half* p, int64_t i, float v) {
  p[i] = __float2half_rn(v);
}
__device__ __forceinline__ void store_from_float(__nv_bfloat16* p, int64_t i, float v) {
  p[i] = __float2bfloat16_rn(v);
}

// The half2 held in a 32-bit word (low half first, as surface and linear
// z-pair copies store it).
__device__ __forceinline__ __half2 u32_as_half2(unsigned int w) {
  return __halves2half2(__ushort_as_half((unsigned short)(w & 0xFFFFu)),
                        __ushort_as_half((unsigned short)(w >> 16)));
}

// Zero border of the exact sampler's records (texels on each side in x and y,
// layers in z). The ray set-up keeps every sample within one step of (-1, n)
// on each axis, so its cell corner lies in [-2, n] and a border of 3 leaves a
// whole texel of slack for the FP32 rounding of the sample positions.
constexpr int kQuadPad = 3;

inline int dtype_size(int dt) { return dt == DTV_F32 ? 4 : 2; }
inline bool dtype_ok(int dt) { return dt == DTV_F32 || dt == DTV_F16 || dt == DTV_BF16; }

// ---- per-view tables (built in FP64 on the host) ------------------------------------
// Forward projector, index space (voxel (i,j,k) centred at (i,j,k)):
//   ray to pixel (u,v): r = d0ms + u*U + v*V   (d0ms = pixel(0,0) centre - source)
//   source S (index) and Sw (world) for the phase rule.
struct FPView {
  double s[3];     // source, index coordinates
  double sw[3];    // source, world coordinates
  double d0ms[3];  // pixel (0,0) centre minus source, index coordinates
  double u[3];     // one pixel step along u, index coordinates
  double v[3];     // one pixel step along v, index coordinates
  double pad;
};
static_assert(sizeof(FPView) == 128, "FPView layout");

// Backprojector: projective map from voxel index (i,j,k,1):
//   h = m[8..11].x, u = m[0..3].x / h, v = m[4..7].x / h (pixel-index coordinates),
//   weight = bp_scale * h^-power, with h = L / SDD (distances along the normal).
struct BPView {
  float m[12];
  float pad[4];
};
static_assert(sizeof(BPView) == 64, "BPView layout");

struct GeomParams {
  int nx, ny, nz, nu, nv, n_views;
  int phase;
  int bp_power;
  int bp_extent;
  double voxel[3];
  double vol_offset[3];
  double det_offset[2];
  double step, scale, bp_scale;
};

// Host helpers (geometry.cu)
int build_tables(const dtv_geometry* g, GeomParams* gp, FPView* fpv, BPView* bpv);
int validate_geometry(const dtv_geometry* g);
double count_fp_samples(const GeomParams& gp, const FPView* fpv);

// ---- plans -----------------------------------------------------------------------------
struct Plan {
  int device;
  int flags;
  int max_batch;
  GeomParams gp;
  FPView* d_fpv;  // device
  BPView* d_bpv;  // device
  BPView* h_bpv;  // host copy (the backprojector passes the maps as launch parameters)
  // soft sampler staging: zero-padded volumes (border kPad) of max_batch items
  void* d_vol_pad;
  // FP32 soft plans: quad records (x..x+1, y..y+1 of one plane) over the same
  // padded grid, read by the forward projector instead of d_vol_pad
  float4* d_vol_quads;
  int stage_dtype;    // DTV_F32 or DTV_F16
  int64_t pad_elems;  // elements of one padded volume
  // soft bilinear staging: zero-padded sinogram of one batch item
  float* d_sino_pad;
  // exact plans: 16-byte records (2x2 detector values) of the padded sinogram
  float4* d_sino_quad;
  // texture sampler (DTV_PLAN_TEX): one 3-D array per batch item for the
  // volume, one layered array for a sinogram
  cudaArray_t* vol_arrays;
  cudaTextureObject_t* vol_tex;      // host copy
  cudaTextureObject_t* vol_tex_dev;  // device copy (kernel argument)
  cudaSurfaceObject_t* vol_surf;     // staging writes into vol_arrays
  cudaArray_t* sino_arrays;
  cudaTextureObject_t* sino_tex;
  // z-pair sampler (DTV_PLAN_TEX_PAIRS): one layered half2 array per batch item
  cudaArray_t* pair_arrays;
  cudaTextureObject_t* pair_tex;
  cudaSurfaceObject_t* pair_surf;
  cudaTextureObject_t* pair_tex_dev;
  int fp_ray_tile;           // DTV_TUNE_FP_RAY_TILE
  int fp_band;               // DTV_TUNE_FP_BAND
  int bp_warp;               // DTV_TUNE_BP_WARP
  // shared-memory staged forward projector (DTV_PLAN_TMA): the z pairs as a
  // linear [batch][nz+3][ny][pair_pitch] u32 array and its two tensor maps
  // (boxes for chunks along x and along y)
  unsigned int* d_pair_lin;
  int pair_pitch;
  // exact z-pair sampler (DTV_PLAN_PAIRS_EXACT): per batch item, 16-byte
  // records [L][Y][X] of the four x/y corner words of a z-pair cell, over the
  // grid padded by kQuadPad zero texels on every side (X = x + 3, Y = y + 3,
  // L = floor(z) + 3 holds (f[L-3], f[L-2]))
  uint4* d_pair_quad;
  int64_t pair_quad_elems;  // records per batch item
  int fp_tex_share;          // DTV_TUNE_FP_TEX_SHARE
  alignas(64) unsigned char tmap[2][128];
  int* d_status;             // device error bits
  int bp_zaffine;            // every view's u and h are independent of z
  // adjoint ray table (DTV_PLAN_ADJOINT): per view and pixel, (p0, count) and (dp, 0)
  float4* d_rays;
  // adjoint cell records (DTV_PLAN_ADJOINT): (nx+1)(ny+1)nz float4 per batch item
  float4* d_cells;
  int adjoint_method;  // DTV_TUNE_ADJOINT
  double fp_samples;  // per volume, < 0 until computed
  uint64_t geom_key;  // hash of the geometry and its per-view tables
};

constexpr int kNumRayTiles = 8;  // forward-projector ray tiles (DTV_TUNE_FP_RAY_TILE)
// default forward block order (DTV_TUNE_FP_BAND): bands of kDefaultBand tile
// rows for staged volumes above kBandAboveBytes, view by view below
constexpr int kDefaultBand = 4;
constexpr double kBandAboveBytes = 32.0 * (1 << 20);
constexpr int kPad = 2;  // zero border of the staged volume

// kernels entry points used across units
int forward_impl(Plan* p, const void* vol, int vol_dtype, int batch, float* out, int epilogue,
                 const float* g, float sigma, double* abs_sum, cudaStream_t st);
// out = base + BP(sino); base NULL: out = BP(sino) (base may be out)
int backward_impl(Plan* p, const float* sino, int batch, const float* base, float* out,
                  cudaStream_t st);
// the correction passes of a texture-filtered plan against an exact one
int forward_refresh_impl(Plan* fast, Plan* exact, const void* vol, int vol_dtype, int batch,
                         const float* g, float sigma, float* w, float* g_eff, double* abs_sum,
                         cudaStream_t st);
int backward_refresh_impl(Plan* fast, Plan* exact, const float* sino, int batch, float* out,
                          float* e_b, cudaStream_t st);
int adjoint_impl(Plan* p, const float* sino, int batch, float* out, cudaStream_t st);
int encode_pair_maps(Plan* p);
// several plans' projections in one launch (forward.cu, backward.cu)
constexpr int kManyItems = 24;  // plans per launch; more run in further launches
int forward_many_impl(Plan* const* plans, const void* const* vols, int vol_dtype, float* const* outs,
                      int count, int epilogue, const float* const* gs, float sigma,
                      cudaStream_t st);
int backward_many_impl(Plan* const* plans, const float* const* sinos, float* const* outs, int count,
                       int accumulate, cudaStream_t st);
int build_ray_table(Plan* p, cudaStream_t st);

}  // namespace dtv
