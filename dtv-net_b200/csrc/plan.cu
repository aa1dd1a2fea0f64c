#include <algorithm>
// Plans (device tables + sampler staging) and the projector entry points.
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "common.cuh"

namespace dtv {

namespace {

struct DeviceGuard {
  int prev = -1;
  bool ok = false;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && cudaSetDevice(dev) == cudaSuccess) ok = true;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

void free_plan(Plan* p) {
  if (!p) return;
  if (p->vol_tex) {
    for (int b = 0; b < p->max_batch; ++b)
      if (p->vol_tex[b]) cudaDestroyTextureObject(p->vol_tex[b]);
  }
  if (p->vol_surf) {
    for (int b = 0; b < p->max_batch; ++b)
      if (p->vol_surf[b]) cudaDestroySurfaceObject(p->vol_surf[b]);
  }
  free(p->vol_surf);
  for (int b = 0; p->pair_arrays && b < p->max_batch; ++b) {
    if (p->pair_tex && p->pair_tex[b]) cudaDestroyTextureObject(p->pair_tex[b]);
    if (p->pair_surf && p->pair_surf[b]) cudaDestroySurfaceObject(p->pair_surf[b]);
    if (p->pair_arrays[b]) cudaFreeArray(p->pair_arrays[b]);
  }
  free(p->pair_arrays);
  free(p->pair_tex);
  free(p->pair_surf);
  cudaFree(p->pair_tex_dev);
  if (p->vol_arrays) {
    for (int b = 0; b < p->max_batch; ++b)
      if (p->vol_arrays[b]) cudaFreeArray(p->vol_arrays[b]);
  }
  if (p->sino_tex && p->sino_tex[0]) cudaDestroyTextureObject(p->sino_tex[0]);
  if (p->sino_arrays && p->sino_arrays[0]) cudaFreeArray(p->sino_arrays[0]);
  free(p->vol_tex);
  free(p->vol_arrays);
  free(p->sino_tex);
  free(p->sino_arrays);
  cudaFree(p->vol_tex_dev);
  cudaFree(p->d_rays);
  cudaFree(p->d_cells);
  cudaFree(p->d_pair_lin);
  cudaFree(p->d_pair_quad);
  cudaFree(p->d_status);
  cudaFree(p->d_fpv);
  cudaFree(p->d_bpv);
  free(p->h_bpv);
  cudaFree(p->d_vol_pad);
  cudaFree(p->d_vol_quads);
  cudaFree(p->d_sino_pad);
  cudaFree(p->d_sino_quad);
  delete p;
}

int make_tex3d(cudaArray_t arr, int filter_linear, cudaTextureObject_t* out) {
  cudaResourceDesc rd;
  memset(&rd, 0, sizeof(rd));
  rd.resType = cudaResourceTypeArray;
  rd.res.array.array = arr;
  cudaTextureDesc td;
  memset(&td, 0, sizeof(td));
  // same sampling state as the reference (forwardKernel.cu:102-107)
  td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
  td.filterMode = filter_linear ? cudaFilterModeLinear : cudaFilterModePoint;
  td.readMode = cudaReadModeElementType;
  td.normalizedCoords = 0;
  DTV_CUDA_TRY(cudaCreateTextureObject(out, &rd, &td, nullptr));
  return DTV_OK;
}


// FNV-1a over the plan's geometry: sizes, rules and spacings field by field,
// then the per-view tables (fully initialised, no padding bytes left unset).
static uint64_t fnv1a(const void* data, size_t n, uint64_t h) {
  const unsigned char* b = static_cast<const unsigned char*>(data);
  for (size_t i = 0; i < n; ++i) {
    h ^= b[i];
    h *= 1099511628211ull;
  }
  return h;
}
static uint64_t geometry_key(const GeomParams& gp, const std::vector<FPView>& fpv,
                             const std::vector<BPView>& bpv) {
  const int ints[9] = {gp.nx, gp.ny, gp.nz, gp.nu, gp.nv, gp.n_views, gp.phase, gp.bp_power,
                       gp.bp_extent};
  const double dbl[13] = {gp.voxel[0], gp.voxel[1], gp.voxel[2], gp.vol_offset[0],
                          gp.vol_offset[1], gp.vol_offset[2], gp.det_offset[0],
                          gp.det_offset[1], gp.step, gp.scale, gp.bp_scale, 0.0, 0.0};
  uint64_t h = 14695981039346656037ull;
  h = fnv1a(ints, sizeof(ints), h);
  h = fnv1a(dbl, sizeof(dbl), h);
  h = fnv1a(fpv.data(), sizeof(FPView) * fpv.size(), h);
  return fnv1a(bpv.data(), sizeof(BPView) * bpv.size(), h);
}

int create_plan(const dtv_geometry* g, int max_batch, int flags, int device, Plan** out) {
  DTV_CHECK(out != nullptr, "out is NULL");
  *out = nullptr;
  DTV_CHECK(max_batch > 0, "max_batch must be positive");
  DTV_CHECK(!(flags & DTV_PLAN_TMA) || (flags & DTV_PLAN_TEX_PAIRS),
            "DTV_PLAN_TMA needs DTV_PLAN_TEX_PAIRS");
  DTV_CHECK((flags & ~(DTV_PLAN_TEX | DTV_PLAN_STAGE_F16 | DTV_PLAN_TEX_PAIRS | DTV_PLAN_ADJOINT |
                       DTV_PLAN_TMA | DTV_PLAN_PAIRS_EXACT)) ==
                0,
            "unknown plan flags 0x%x", flags);
  DTV_CHECK(!((flags & DTV_PLAN_PAIRS_EXACT) &&
              (flags & (DTV_PLAN_TEX | DTV_PLAN_TEX_PAIRS | DTV_PLAN_TMA))),
            "DTV_PLAN_PAIRS_EXACT excludes DTV_PLAN_TEX, DTV_PLAN_TEX_PAIRS and DTV_PLAN_TMA");
  DTV_CHECK(!((flags & DTV_PLAN_TEX) && (flags & DTV_PLAN_TEX_PAIRS)),
            "DTV_PLAN_TEX and DTV_PLAN_TEX_PAIRS are exclusive");
  int ndev = 0;
  DTV_CUDA_TRY(cudaGetDeviceCount(&ndev));
  DTV_CHECK(device >= 0 && device < ndev, "device %d out of range (%d devices)", device, ndev);
  DeviceGuard dg(device);
  if (!dg.ok) return fail(DTV_ERR_CUDA, "cannot select device %d", device);

  Plan* p = new Plan();
  memset(p, 0, sizeof(*p));
  p->device = device;
  p->flags = flags;
  p->max_batch = max_batch;
  p->fp_samples = -1.0;
  std::vector<FPView> fpv(g ? g->n_views : 0);
  std::vector<BPView> bpv(g ? g->n_views : 0);
  int rc = validate_geometry(g);
  if (rc) {
    delete p;
    return rc;
  }
  rc = build_tables(g, &p->gp, fpv.data(), bpv.data());
  if (rc) {
    delete p;
    return rc;
  }
  const GeomParams& gp = p->gp;
  p->geom_key = geometry_key(gp, fpv, bpv);
  p->bp_zaffine = 1;
  for (int n = 0; n < gp.n_views; ++n)
    if (bpv[n].m[2] != 0.f || bpv[n].m[10] != 0.f) p->bp_zaffine = 0;
#define PLAN_CUDA(expr)                                                                  \
  do {                                                                                   \
    cudaError_t _e = (expr);                                                             \
    if (_e != cudaSuccess) {                                                             \
      free_plan(p);                                                                      \
      return fail(_e == cudaErrorMemoryAllocation ? DTV_ERR_ALLOC : DTV_ERR_CUDA,        \
                  "%s failed: %s", #expr, cudaGetErrorString(_e));                       \
    }                                                                                    \
  } while (0)
  PLAN_CUDA(cudaMalloc(&p->d_fpv, sizeof(FPView) * gp.n_views));
  PLAN_CUDA(cudaMalloc(&p->d_bpv, sizeof(BPView) * gp.n_views));
  PLAN_CUDA(cudaMemcpy(p->d_fpv, fpv.data(), sizeof(FPView) * gp.n_views, cudaMemcpyHostToDevice));
  PLAN_CUDA(cudaMemcpy(p->d_bpv, bpv.data(), sizeof(BPView) * gp.n_views, cudaMemcpyHostToDevice));
  p->h_bpv = (BPView*)malloc(sizeof(BPView) * gp.n_views);
  if (!p->h_bpv) {
    free_plan(p);
    return fail(DTV_ERR_ALLOC, "host allocation failed");
  }
  memcpy(p->h_bpv, bpv.data(), sizeof(BPView) * gp.n_views);

  p->stage_dtype = (flags & DTV_PLAN_STAGE_F16) ? DTV_F16 : DTV_F32;
  p->pad_elems = (int64_t)(gp.nx + 2 * kPad) * (gp.ny + 2 * kPad) * (gp.nz + 2 * kPad);
  const size_t esz = p->stage_dtype == DTV_F16 ? 2 : 4;
  // Staged volumes of the software sampler (FP32: quad records, FP16: the
  // padded volume): zero border written once here, interiors by each call.
  if (flags & DTV_PLAN_PAIRS_EXACT) {
    p->pair_quad_elems = (int64_t)(gp.nx + 2 * kQuadPad) * (gp.ny + 2 * kQuadPad) *
                         (gp.nz + 2 * kQuadPad - 1);
    if (p->pair_quad_elems >= (1LL << 31)) {
      free_plan(p);
      return fail(DTV_ERR_UNSUPPORTED, "volume too large for DTV_PLAN_PAIRS_EXACT");
    }
    const size_t bytes = sizeof(uint4) * p->pair_quad_elems * max_batch;
    PLAN_CUDA(cudaMalloc(&p->d_pair_quad, bytes));
    PLAN_CUDA(cudaMemset(p->d_pair_quad, 0, bytes));  // records beyond the volume stay zero
  } else if (!(flags & (DTV_PLAN_TEX | DTV_PLAN_TEX_PAIRS))) {
    if (p->stage_dtype == DTV_F32) {
      PLAN_CUDA(cudaMalloc(&p->d_vol_quads, sizeof(float4) * p->pad_elems * max_batch));
      PLAN_CUDA(cudaMemset(p->d_vol_quads, 0, sizeof(float4) * p->pad_elems * max_batch));
    } else {
      PLAN_CUDA(cudaMalloc(&p->d_vol_pad, esz * p->pad_elems * max_batch));
      PLAN_CUDA(cudaMemset(p->d_vol_pad, 0, esz * p->pad_elems * max_batch));
    }
  }
  const int64_t sino_pad = (int64_t)(gp.nu + 2 * kPad) * (gp.nv + 2 * kPad) * gp.n_views;
  PLAN_CUDA(cudaMalloc(&p->d_sino_pad, sizeof(float) * sino_pad));
  PLAN_CUDA(cudaMemset(p->d_sino_pad, 0, sizeof(float) * sino_pad));
  if (flags & DTV_PLAN_PAIRS_EXACT) {
    PLAN_CUDA(cudaMalloc(&p->d_sino_quad, sizeof(float4) * sino_pad));
    PLAN_CUDA(cudaMemset(p->d_sino_quad, 0, sizeof(float4) * sino_pad));
  }

  if (flags & DTV_PLAN_TEX) {
    p->vol_arrays = (cudaArray_t*)calloc(max_batch, sizeof(cudaArray_t));
    p->vol_tex = (cudaTextureObject_t*)calloc(max_batch, sizeof(cudaTextureObject_t));
    p->vol_surf = (cudaSurfaceObject_t*)calloc(max_batch, sizeof(cudaSurfaceObject_t));
    if (!p->vol_arrays || !p->vol_tex || !p->vol_surf) {
      free_plan(p);
      return fail(DTV_ERR_ALLOC, "host allocation failed");
    }
    cudaChannelFormatDesc cd = p->stage_dtype == DTV_F16 ? cudaCreateChannelDescHalf()
                                                         : cudaCreateChannelDesc<float>();
    for (int b = 0; b < max_batch; ++b) {
      PLAN_CUDA(cudaMalloc3DArray(&p->vol_arrays[b], &cd, make_cudaExtent(gp.nx, gp.ny, gp.nz),
                                  cudaArraySurfaceLoadStore));
      rc = make_tex3d(p->vol_arrays[b], 1, &p->vol_tex[b]);
      if (rc) {
        free_plan(p);
        return rc;
      }
      cudaResourceDesc rd;
      memset(&rd, 0, sizeof(rd));
      rd.resType = cudaResourceTypeArray;
      rd.res.array.array = p->vol_arrays[b];
      PLAN_CUDA(cudaCreateSurfaceObject(&p->vol_surf[b], &rd));
    }
    PLAN_CUDA(cudaMalloc(&p->vol_tex_dev, sizeof(cudaTextureObject_t) * max_batch));
    PLAN_CUDA(cudaMemcpy(p->vol_tex_dev, p->vol_tex, sizeof(cudaTextureObject_t) * max_batch,
                         cudaMemcpyHostToDevice));
  }
  int max_layers = 0;
  if (flags & (DTV_PLAN_TEX | DTV_PLAN_TEX_PAIRS))
    PLAN_CUDA(cudaDeviceGetAttribute(&max_layers, cudaDevAttrMaxTexture2DLayeredLayers, device));
  if (flags & DTV_PLAN_TEX_PAIRS) {
    if (gp.nz + 3 > max_layers) {
      free_plan(p);
      return fail(DTV_ERR_UNSUPPORTED, "nz + 3 = %d exceeds the %d texture layers of the device",
                  gp.nz + 3, max_layers);
    }
    p->pair_arrays = (cudaArray_t*)calloc(max_batch, sizeof(cudaArray_t));
    p->pair_tex = (cudaTextureObject_t*)calloc(max_batch, sizeof(cudaTextureObject_t));
    p->pair_surf = (cudaSurfaceObject_t*)calloc(max_batch, sizeof(cudaSurfaceObject_t));
    if (!p->pair_arrays || !p->pair_tex || !p->pair_surf) {
      free_plan(p);
      return fail(DTV_ERR_ALLOC, "host allocation failed");
    }
    cudaChannelFormatDesc cd = cudaCreateChannelDescHalf2();
    for (int b = 0; b < max_batch; ++b) {
      PLAN_CUDA(cudaMalloc3DArray(&p->pair_arrays[b], &cd,
                                  make_cudaExtent(gp.nx, gp.ny, gp.nz + 3),
                                  cudaArrayLayered | cudaArraySurfaceLoadStore));
      rc = make_tex3d(p->pair_arrays[b], 1, &p->pair_tex[b]);
      if (rc) {
        free_plan(p);
        return rc;
      }
      cudaResourceDesc rd;
      memset(&rd, 0, sizeof(rd));
      rd.resType = cudaResourceTypeArray;
      rd.res.array.array = p->pair_arrays[b];
      PLAN_CUDA(cudaCreateSurfaceObject(&p->pair_surf[b], &rd));
    }
    PLAN_CUDA(cudaMalloc(&p->pair_tex_dev, sizeof(cudaTextureObject_t) * max_batch));
    PLAN_CUDA(cudaMemcpy(p->pair_tex_dev, p->pair_tex, sizeof(cudaTextureObject_t) * max_batch,
                         cudaMemcpyHostToDevice));
  }
  PLAN_CUDA(cudaMalloc(&p->d_status, sizeof(int)));
  PLAN_CUDA(cudaMemset(p->d_status, 0, sizeof(int)));
  if (flags & DTV_PLAN_TMA) {
    p->pair_pitch = (gp.nx + 3) & ~3;  // rows of whole 16-byte units
    const size_t words = (size_t)p->pair_pitch * gp.ny * (gp.nz + 3) * max_batch;
    PLAN_CUDA(cudaMalloc(&p->d_pair_lin, words * sizeof(unsigned int)));
    PLAN_CUDA(cudaMemset(p->d_pair_lin, 0, words * sizeof(unsigned int)));
    p->fp_tex_share = 0;
    rc = encode_pair_maps(p);
    if (rc) {
      free_plan(p);
      return rc;
    }
  }
  if ((flags & (DTV_PLAN_TEX | DTV_PLAN_TEX_PAIRS)) && gp.n_views <= max_layers) {
    // backprojector: the sinogram as a layered texture (one layer per view);
    // with more views than layers the backprojector samples in software
    p->sino_arrays = (cudaArray_t*)calloc(1, sizeof(cudaArray_t));
    p->sino_tex = (cudaTextureObject_t*)calloc(1, sizeof(cudaTextureObject_t));
    if (!p->sino_arrays || !p->sino_tex) {
      free_plan(p);
      return fail(DTV_ERR_ALLOC, "host allocation failed");
    }
    cudaChannelFormatDesc sd = cudaCreateChannelDesc<float>();
    PLAN_CUDA(cudaMalloc3DArray(&p->sino_arrays[0], &sd, make_cudaExtent(gp.nu, gp.nv, gp.n_views),
                                cudaArrayLayered));
    rc = make_tex3d(p->sino_arrays[0], 1, &p->sino_tex[0]);
    if (rc) {
      free_plan(p);
      return rc;
    }
  }
  if (flags & DTV_PLAN_ADJOINT) {
    const size_t n = (size_t)gp.n_views * gp.nu * gp.nv * 2;
    PLAN_CUDA(cudaMalloc(&p->d_rays, n * sizeof(float4)));
    const size_t cells = (size_t)(gp.nx + 1) * (gp.ny + 1) * gp.nz * max_batch;
    PLAN_CUDA(cudaMalloc(&p->d_cells, cells * sizeof(float4)));
    p->adjoint_method = 1;
    rc = build_ray_table(p, 0);
    if (!rc) {
      cudaError_t e = cudaStreamSynchronize(0);
      if (e != cudaSuccess) rc = fail(DTV_ERR_CUDA, "ray table: %s", cudaGetErrorString(e));
    }
    if (rc) {
      free_plan(p);
      return rc;
    }
  }
#undef PLAN_CUDA
  p->bp_warp = 4;  // 4 x 8 columns per warp in quads of 2 x 2 (fewest texture wavefronts)
  // forward block order: bands of 4 tile rows across views once the staged
  // volume is too large to stay in L2 from one view to the next
  if (!(flags & DTV_PLAN_TMA)) {
    const double voxels = (double)gp.nx * gp.ny * gp.nz;
    double staged;
    if (flags & DTV_PLAN_TEX_PAIRS) staged = (double)gp.nx * gp.ny * (gp.nz + 3) * 4.0;
    else if (flags & DTV_PLAN_PAIRS_EXACT) staged = (double)p->pair_quad_elems * 16.0;
    else if (flags & DTV_PLAN_TEX) staged = voxels * (p->stage_dtype == DTV_F16 ? 2.0 : 4.0);
    else if (p->d_vol_quads) staged = (double)p->pad_elems * 16.0;
    else staged = (double)p->pad_elems * 2.0;
    p->fp_band = staged > kBandAboveBytes ? kDefaultBand : 0;
  }
  *out = p;
  return DTV_OK;
}

int check_plan_call(const dtv_plan* plan, int batch) {
  DTV_CHECK(plan != nullptr, "plan is NULL");
  const Plan* p = reinterpret_cast<const Plan*>(plan);
  DTV_CHECK(batch > 0 && batch <= p->max_batch, "batch %d outside [1, %d]", batch, p->max_batch);
  return DTV_OK;
}

}  // namespace
}  // namespace dtv

using namespace dtv;

extern "C" {

int dtv_plan_create(const dtv_geometry* g, int32_t max_batch, int32_t flags, int32_t device,
                    dtv_plan** out) {
  Plan* p = nullptr;
  int rc = create_plan(g, max_batch, flags, device, &p);
  if (out) *out = reinterpret_cast<dtv_plan*>(p);
  return rc;
}

int dtv_plan_destroy(dtv_plan* plan) {
  if (!plan) return DTV_OK;
  Plan* p = reinterpret_cast<Plan*>(plan);
  DeviceGuard dg(p->device);
  free_plan(p);
  return DTV_OK;
}

int dtv_plan_set_tuning(dtv_plan* plan, int32_t key, int32_t value) {
  DTV_CHECK(plan != nullptr, "plan is NULL");
  Plan* p = reinterpret_cast<Plan*>(plan);
  switch (key) {
    case DTV_TUNE_ADJOINT:
      DTV_CHECK(value == 0 || value == 1, "DTV_TUNE_ADJOINT must be 0 or 1");
      DTV_CHECK(value == 0 || p->d_cells, "DTV_TUNE_ADJOINT 1 needs a DTV_PLAN_ADJOINT plan");
      p->adjoint_method = value;
      return DTV_OK;
    case DTV_TUNE_FP_TEX_SHARE:
      DTV_CHECK(p->flags & DTV_PLAN_TMA, "DTV_TUNE_FP_TEX_SHARE needs a DTV_PLAN_TMA plan");
      DTV_CHECK(value >= 0 && value <= 8, "DTV_TUNE_FP_TEX_SHARE must be in [0, 8]");
      p->fp_tex_share = value;
      return DTV_OK;
    case DTV_TUNE_FP_RAY_TILE:
      DTV_CHECK(value >= 0 && value < kNumRayTiles, "DTV_TUNE_FP_RAY_TILE must be in [0, %d]",
                kNumRayTiles - 1);
      p->fp_ray_tile = value;
      return DTV_OK;
    case DTV_TUNE_FP_BAND:
      DTV_CHECK(!(p->flags & DTV_PLAN_TMA), "DTV_TUNE_FP_BAND does not apply to DTV_PLAN_TMA plans");
      DTV_CHECK(value >= 0 && value <= 4096, "DTV_TUNE_FP_BAND must be in [0, 4096]");
      p->fp_band = value;
      return DTV_OK;
    case DTV_TUNE_BP_WARP:
      DTV_CHECK(value >= 0 && value <= 4, "DTV_TUNE_BP_WARP must be in [0, 4]");
      p->bp_warp = value;
      return DTV_OK;
    default:
      return fail(DTV_ERR_INVALID, "unknown tuning key %d", key);
  }
}

int dtv_plan_get_tuning(const dtv_plan* plan, int32_t key, int32_t* value) {
  DTV_CHECK(plan && value, "NULL argument");
  const Plan* p = reinterpret_cast<const Plan*>(plan);
  switch (key) {
    case DTV_TUNE_FP_RAY_TILE:
      *value = p->fp_ray_tile;
      return DTV_OK;
    case DTV_TUNE_FP_TEX_SHARE:
      *value = p->fp_tex_share;
      return DTV_OK;
    case DTV_TUNE_ADJOINT:
      *value = p->adjoint_method;
      return DTV_OK;
    case DTV_TUNE_FP_BAND:
      *value = p->fp_band;
      return DTV_OK;
    case DTV_TUNE_BP_WARP:
      *value = p->bp_warp;
      return DTV_OK;
    default:
      return fail(DTV_ERR_INVALID, "unknown tuning key %d", key);
  }
}

int dtv_plan_device_status(dtv_plan* plan, int32_t* status, int32_t reset) {
  DTV_CHECK(plan && status, "NULL argument");
  Plan* p = reinterpret_cast<Plan*>(plan);
  DeviceGuard dg(p->device);
  if (!dg.ok) return fail(DTV_ERR_CUDA, "cannot select device %d", p->device);
  int v = 0;
  DTV_CUDA_TRY(cudaDeviceSynchronize());
  DTV_CUDA_TRY(cudaMemcpy(&v, p->d_status, sizeof(int), cudaMemcpyDeviceToHost));
  if (reset) DTV_CUDA_TRY(cudaMemset(p->d_status, 0, sizeof(int)));
  *status = v;
  return DTV_OK;
}

int dtv_plan_fp_samples(const dtv_plan* plan, double* samples) {
  DTV_CHECK(plan && samples, "NULL argument");
  Plan* p = const_cast<Plan*>(reinterpret_cast<const Plan*>(plan));
  if (p->fp_samples < 0) {
    std::vector<FPView> fpv(p->gp.n_views);
    DTV_CUDA_TRY(cudaMemcpy(fpv.data(), p->d_fpv, sizeof(FPView) * p->gp.n_views,
                            cudaMemcpyDeviceToHost));
    p->fp_samples = count_fp_samples(p->gp, fpv.data());
  }
  *samples = p->fp_samples;
  return DTV_OK;
}

int dtv_forward(dtv_plan* plan, const void* vol, int32_t vol_dtype, int32_t batch, float* out,
                int32_t epilogue, const float* g, float sigma, double* abs_sum, void* stream) {
  int rc = check_plan_call(plan, batch);
  if (rc) return rc;
  DTV_CHECK(vol && out, "NULL volume or output");
  DTV_CHECK(dtype_ok(vol_dtype), "bad volume dtype %d", vol_dtype);
  DTV_CHECK(epilogue >= DTV_EPI_STORE && epilogue <= DTV_EPI_PDHG, "bad epilogue %d", epilogue);
  DTV_CHECK(epilogue == DTV_EPI_STORE || g != nullptr, "epilogue %d needs g", epilogue);
  Plan* p = reinterpret_cast<Plan*>(plan);
  DeviceGuard dg(p->device);
  return forward_impl(p, vol, vol_dtype, batch, out, epilogue, g, sigma, abs_sum, as_stream(stream));
}

int dtv_backward(dtv_plan* plan, const float* sino, int32_t batch, float* out, int32_t accumulate,
                 void* stream) {
  int rc = check_plan_call(plan, batch);
  if (rc) return rc;
  DTV_CHECK(sino && out, "NULL sinogram or output");
  Plan* p = reinterpret_cast<Plan*>(plan);
  DeviceGuard dg(p->device);
  return backward_impl(p, sino, batch, accumulate ? out : nullptr, out, as_stream(stream));
}

int dtv_backward_onto(dtv_plan* plan, const float* sino, int32_t batch, const float* base,
                      float* out, void* stream) {
  int rc = check_plan_call(plan, batch);
  if (rc) return rc;
  DTV_CHECK(sino && base && out, "NULL sinogram, base or output");
  Plan* p = reinterpret_cast<Plan*>(plan);
  DeviceGuard dg(p->device);
  return backward_impl(p, sino, batch, base, out, as_stream(stream));
}

// A texture-filtered z-pair plan and an exact-weight plan of one geometry.
static int check_refresh_pair(dtv_plan* fast, dtv_plan* exact, int batch) {
  int rc = check_plan_call(fast, batch);
  if (rc) return rc;
  rc = check_plan_call(exact, batch);
  if (rc) return rc;
  const Plan* f = reinterpret_cast<const Plan*>(fast);
  const Plan* e = reinterpret_cast<const Plan*>(exact);
  DTV_CHECK((f->flags & DTV_PLAN_TEX_PAIRS) && !(f->flags & DTV_PLAN_TMA),
            "the fast plan must be a DTV_PLAN_TEX_PAIRS plan without DTV_PLAN_TMA");
  DTV_CHECK(e->flags & DTV_PLAN_PAIRS_EXACT, "the exact plan must be a DTV_PLAN_PAIRS_EXACT plan");
  DTV_CHECK(f->device == e->device, "the plans are on different devices");
  DTV_CHECK(f->geom_key == e->geom_key, "the plans' geometries differ");
  return DTV_OK;
}

int dtv_pdhg_forward_refresh(dtv_plan* fast, dtv_plan* exact, const void* vol, int32_t vol_dtype,
                             int32_t batch, const float* g, float sigma, float* w, float* g_eff,
                             double* abs_sum, void* stream) {
  int rc = check_refresh_pair(fast, exact, batch);
  if (rc) return rc;
  DTV_CHECK(vol && g && w && g_eff, "NULL volume, data, dual or corrected data");
  DTV_CHECK(dtype_ok(vol_dtype), "bad volume dtype %d", vol_dtype);
  Plan* f = reinterpret_cast<Plan*>(fast);
  DeviceGuard dg(f->device);
  return forward_refresh_impl(f, reinterpret_cast<Plan*>(exact), vol, vol_dtype, batch, g, sigma,
                              w, g_eff, abs_sum, as_stream(stream));
}

int dtv_backward_refresh(dtv_plan* fast, dtv_plan* exact, const float* sino, int32_t batch,
                         float* out, float* e_b, void* stream) {
  int rc = check_refresh_pair(fast, exact, batch);
  if (rc) return rc;
  DTV_CHECK(sino && out && e_b, "NULL sinogram, output or difference");
  DTV_CHECK(out != e_b, "out and e_b must be different buffers");
  Plan* f = reinterpret_cast<Plan*>(fast);
  DeviceGuard dg(f->device);
  return backward_refresh_impl(f, reinterpret_cast<Plan*>(exact), sino, batch, out, e_b,
                               as_stream(stream));
}

int dtv_forward_many(dtv_plan* const* plans, const void* const* vols, int32_t vol_dtype,
                     float* const* outs, int32_t count, int32_t epilogue, const float* const* gs,
                     float sigma, void* stream) {
  DTV_CHECK(plans && vols && outs, "NULL argument");
  DTV_CHECK(count >= 1, "count %d < 1", count);
  DTV_CHECK(dtype_ok(vol_dtype), "bad volume dtype %d", vol_dtype);
  DTV_CHECK(epilogue >= DTV_EPI_STORE && epilogue <= DTV_EPI_PDHG, "bad epilogue %d", epilogue);
  DTV_CHECK(epilogue == DTV_EPI_STORE || gs != nullptr, "epilogue %d needs g", epilogue);
  std::vector<Plan*> ps(count);
  for (int k = 0; k < count; ++k) {
    DTV_CHECK(plans[k] && vols[k] && outs[k], "NULL plan, volume or output at %d", k);
    DTV_CHECK(epilogue == DTV_EPI_STORE || gs[k], "NULL g at %d", k);
    ps[k] = reinterpret_cast<Plan*>(plans[k]);
    DTV_CHECK(ps[k]->flags & DTV_PLAN_TEX_PAIRS, "plan %d is not a DTV_PLAN_TEX_PAIRS plan", k);
    DTV_CHECK(ps[k]->device == ps[0]->device, "plans %d and 0 are on different devices", k);
  }
  // each plan stages its one volume into its own texture: a plan may appear once
  std::vector<Plan*> sorted(ps);
  std::sort(sorted.begin(), sorted.end());
  DTV_CHECK(std::adjacent_find(sorted.begin(), sorted.end()) == sorted.end(),
            "a plan appears more than once");
  DeviceGuard dg(ps[0]->device);
  return forward_many_impl(ps.data(), vols, vol_dtype, outs, count, epilogue, gs, sigma,
                           as_stream(stream));
}

int dtv_backward_many(dtv_plan* const* plans, const float* const* sinos, float* const* outs,
                      int32_t count, int32_t accumulate, void* stream) {
  DTV_CHECK(plans && sinos && outs, "NULL argument");
  DTV_CHECK(count >= 1, "count %d < 1", count);
  std::vector<Plan*> ps(count);
  for (int k = 0; k < count; ++k) {
    DTV_CHECK(plans[k] && sinos[k] && outs[k], "NULL plan, sinogram or output at %d", k);
    ps[k] = reinterpret_cast<Plan*>(plans[k]);
    DTV_CHECK(ps[k]->sino_tex != nullptr,
              "plan %d has no sinogram texture (DTV_PLAN_TEX or DTV_PLAN_TEX_PAIRS)", k);
    DTV_CHECK(ps[k]->device == ps[0]->device, "plans %d and 0 are on different devices", k);
  }
  std::vector<Plan*> sorted(ps);
  std::sort(sorted.begin(), sorted.end());
  DTV_CHECK(std::adjacent_find(sorted.begin(), sorted.end()) == sorted.end(),
            "a plan appears more than once");
  DeviceGuard dg(ps[0]->device);
  return backward_many_impl(ps.data(), sinos, outs, count, accumulate ? 1 : 0, as_stream(stream));
}

int dtv_backward_adjoint(dtv_plan* plan, const float* sino, int32_t batch, float* out,
                         void* stream) {
  int rc = check_plan_call(plan, batch);
  if (rc) return rc;
  DTV_CHECK(sino && out, "NULL sinogram or output");
  Plan* p = reinterpret_cast<Plan*>(plan);
  DeviceGuard dg(p->device);
  return adjoint_impl(p, sino, batch, out, as_stream(stream));
}

static int one_shot(const dtv_geometry* g, int batch, int device, int fwd, const float* in,
                    float* out, cudaStream_t st) {
  Plan* p = nullptr;
  int rc = create_plan(g, batch, 0, device, &p);
  if (rc) return rc;
  {
    DeviceGuard dg(device);
    rc = fwd ? forward_impl(p, in, DTV_F32, batch, out, DTV_EPI_STORE, nullptr, 0.f, nullptr, st)
             : backward_impl(p, in, batch, nullptr, out, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (!rc && e != cudaSuccess) rc = fail(DTV_ERR_CUDA, "sync: %s", cudaGetErrorString(e));
  }
  dtv_plan_destroy(reinterpret_cast<dtv_plan*>(p));
  return rc;
}

int dtv_standard_forward(const float* volume, int32_t batch, const float* angles_deg,
                         int32_t n_angles, const int32_t vs[3], const int32_t ds[2], float sid,
                         float sdd, int32_t device, float* sino, void* stream) {
  DTV_CHECK(volume && sino, "NULL volume or sinogram");
  std::vector<double> views(12 * (size_t)(n_angles > 0 ? n_angles : 0));
  dtv_geometry g;
  int rc = dtv_geometry_standard(&g, views.data(), angles_deg, n_angles, vs, ds, sid, sdd);
  if (rc) return rc;
  return one_shot(&g, batch, device, 1, volume, sino, as_stream(stream));
}

int dtv_standard_backward(const float* sino, int32_t batch, const float* angles_deg,
                          int32_t n_angles, const int32_t vs[3], const int32_t ds[2], float sid,
                          float sdd, int32_t device, float* volume, void* stream) {
  DTV_CHECK(volume && sino, "NULL volume or sinogram");
  std::vector<double> views(12 * (size_t)(n_angles > 0 ? n_angles : 0));
  dtv_geometry g;
  int rc = dtv_geometry_standard(&g, views.data(), angles_deg, n_angles, vs, ds, sid, sdd);
  if (rc) return rc;
  return one_shot(&g, batch, device, 0, sino, volume, as_stream(stream));
}

int dtv_vector_forward(const float* volume, int32_t batch, const int32_t vs[3],
                       const int32_t ds[2], const float* pv, int32_t n_views, int32_t device,
                       float* sino, void* stream) {
  DTV_CHECK(volume && sino, "NULL volume or sinogram");
  std::vector<double> views(12 * (size_t)(n_views > 0 ? n_views : 0));
  dtv_geometry g;
  int rc = dtv_geometry_vector(&g, views.data(), pv, n_views, vs, ds);
  if (rc) return rc;
  return one_shot(&g, batch, device, 1, volume, sino, as_stream(stream));
}

int dtv_vector_backward(const float* sino, int32_t batch, const int32_t vs[3],
                        const int32_t ds[2], const float* pv, int32_t n_views, int32_t device,
                        float* volume, void* stream) {
  DTV_CHECK(volume && sino, "NULL volume or sinogram");
  std::vector<double> views(12 * (size_t)(n_views > 0 ? n_views : 0));
  dtv_geometry g;
  int rc = dtv_geometry_vector(&g, views.data(), pv, n_views, vs, ds);
  if (rc) return rc;
  return one_shot(&g, batch, device, 0, sino, volume, as_stream(stream));
}

}  // extern "C"
