/*
 * dtv_b200.h — C ABI of the B200 cone-beam projector pair and the unrolled
 * DTV / FISTA / PDHG update kernels.
 *
 * Conventions shared by every entry point:
 *   - volume  : [batch][1][nz][ny][nx], x fastest (reference layout,
 *               model/ConeBeamLayers/Standard/plug/kernel/backwardKernel.cu:63)
 *   - sinogram: [batch][1][n_views][nv][nu], u fastest
 *               (model/ConeBeamLayers/Standard/plug/kernel/forwardKernel.cu:96)
 *   - every data pointer is DEVICE memory owned by the caller; outputs are
 *     caller-allocated (the reference allocated them itself, :96);
 *   - `stream` is a cudaStream_t passed as void*; calls are stream-ordered and
 *     never synchronise the host (the reference synchronised once per view
 *     through .item(), forwardKernel.cu:135);
 *   - every call returns DTV_OK or an error code; dtv_error_string() names it
 *     and dtv_last_error_message() gives the detail of the last failure on the
 *     calling thread (the reference raised RuntimeError via AT_ASSERTM on bad
 *     input, forwardKernel.cu:15-17,89-94, and ignored CUDA errors).
 *   - plans are immutable after creation apart from their launch knobs
 *     (dtv_plan_set_tuning, which a launch reads when it is issued; set them
 *     before sharing the plan between threads). A plan may be used from
 *     several host threads on different streams at once EXCEPT that calls
 *     sharing one plan's staging buffers (forward/backward) on different
 *     streams race: serialise them on one stream or use one plan per stream.
 */
#ifndef DTV_B200_H
#define DTV_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define DTV_API __attribute__((visibility("default")))
#else
#define DTV_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define DTV_OK 0
#define DTV_ERR_INVALID 1     /* bad argument (null, size, dtype, ...)     */
#define DTV_ERR_CUDA 2        /* a CUDA runtime call failed                */
#define DTV_ERR_ALLOC 3       /* device allocation failed                  */
#define DTV_ERR_UNSUPPORTED 4 /* valid but not supported by the library   */

/* ---- storage types ------------------------------------------------------ */
#define DTV_F32 0
#define DTV_F16 1
#define DTV_BF16 2

/* ---- forward-projector sample phase ------------------------------------ */
/* Standard circular layer: samples at a_min-3+k*step, a_min/a_max from the
 * dominant in-plane axis against the bounds +-n/2 in world units
 * (Standard/plug/kernel/forwardKernel.cu:45-58,66-80). */
#define DTV_PHASE_STANDARD 0
/* Vector (Beijing) layer: as above, dominant axis chosen among x, y, z
 * (Beijing/plug/kernel/forwardKernel.cu:40-60). */
#define DTV_PHASE_VECTOR 1
/* Exact ray/box chord with centred samples a_in+(k+1/2)*step, k < ceil(chord/step)
 * (the general geometry; no reference counterpart). */
#define DTV_PHASE_BOX 2

/* ---- plan flags ----------------------------------------------------------- */
#define DTV_PLAN_SOFT 0x0      /* software trilinear/bilinear, FP32 weights (default) */
#define DTV_PLAN_TEX 0x1       /* hardware texture filtering (8-bit fraction weights) */
#define DTV_PLAN_STAGE_F16 0x2 /* stage the projected volume as FP16 (soft sampler)  */
/* Forward projector through a 2-D layered FP16 texture whose texel (x, y, L)
 * holds the z pair (f[L-2], f[L-1]): one bilinear fetch (8-bit x/y weights)
 * returns both planes and the z interpolation is done in FP32. Backprojector
 * as DTV_PLAN_TEX. Needs nz + 3 <= the device's layered-texture layer limit. */
#define DTV_PLAN_TEX_PAIRS 0x4
/* Keep a table of every ray's sample range (32 bytes per ray and view) and
 * (nx+1)(ny+1)nz 16-byte cell records per batch item for
 * dtv_backward_adjoint, which otherwise rebuilds each ray for every 16^3
 * brick it crosses (see DTV_TUNE_ADJOINT). */
#define DTV_PLAN_ADJOINT 0x8
/* With DTV_PLAN_TEX_PAIRS: the forward projector stages the z pairs of the
 * volume a second time as a linear array and streams 20x32x20-word boxes of
 * it into shared memory with the Tensor Memory Accelerator, one box per
 * 16x16-ray tile and chunk of 16 planes along the tile's dominant axis;
 * samples are interpolated from shared memory with FP32 x/y/z weights (exact
 * trilinear of the FP16 volume). DTV_TUNE_FP_TEX_SHARE sends a share of the
 * tiles through the texture unit instead, so both pipes work at once. */
#define DTV_PLAN_TMA 0x10
/* Exact interpolation weights in both directions. Forward projector: the FP16
 * z pairs of DTV_PLAN_TEX_PAIRS staged in a linear array with a two-texel
 * zero border, read through L1 (four 4-byte loads per sample) and
 * interpolated with FP32 x/y/z weights (exact trilinear of the FP16-rounded
 * volume). Backprojector: software bilinear with FP32 weights, as
 * DTV_PLAN_SOFT. The texture filter's 8-bit weights, whose error iterative
 * reconstructions amplify, are not used. Exclusive with DTV_PLAN_TEX,
 * DTV_PLAN_TEX_PAIRS and DTV_PLAN_TMA. */
#define DTV_PLAN_PAIRS_EXACT 0x20

/* ---- forward-projector epilogues ---------------------------------------- */
#define DTV_EPI_STORE 0    /* out = FP(vol)                                        */
#define DTV_EPI_RESIDUAL 1 /* out = FP(vol) - g                 (FISTA.py:21)       */
#define DTV_EPI_PDHG 2     /* out = (out + sigma*(FP(vol)-g))/(1+sigma) (DTVCP.py:38-39) */

/*
 * Geometry. World positions in any length unit. Voxel (i,j,k) centre is at
 *   ((i - nx/2 + vol_offset[0]) * voxel[0], (j - ny/2 + ...) , (k - nz/2 + ...)).
 * Detector pixel (u,v) centre of view n is at
 *   D_n + (u - nu/2 + det_offset[0]) U_n + (v - nv/2 + det_offset[1]) V_n,
 * with views[12n..12n+11] = source S_n(3), detector centre D_n(3), U_n(3), V_n(3),
 * where U_n, V_n are world vectors of ONE pixel step (their length is the pitch).
 * The forward projector sums trilinear samples (border value 0) of the volume
 * along the ray S_n -> pixel with spacing fp_step and multiplies by fp_scale.
 * The FDK backprojector adds, per view, the bilinear detector value at the
 * voxel's projection times bp_scale * (SDD_n / L)^bp_weight_power, where L and
 * SDD_n are the source-to-voxel and source-to-detector distances along the
 * detector normal.
 */
typedef struct dtv_geometry {
  int32_t nx, ny, nz;
  int32_t nu, nv;
  int32_t n_views;
  double voxel[3];
  double vol_offset[3];
  double det_offset[2];
  double fp_step;
  double fp_scale;
  int32_t fp_phase;        /* DTV_PHASE_* */
  int32_t bp_weight_power; /* 2: (SDD/L)^2 (Standard), 1: SDD/L (vector) */
  double bp_scale;         /* pi/N (Standard), 2*pi/(N/21) (vector)      */
  /* Vector-layer quirk: skip a view when the voxel's detector coordinate lies
   * outside [-1, nx+1] x [-1, ny+1] of the VOLUME size
   * (Beijing/plug/kernel/backwardKernel.cu:38). 0 disables. */
  int32_t bp_extent_check;
  int32_t reserved;
  const double* views; /* host memory, n_views*12 doubles */
} dtv_geometry;

typedef struct dtv_plan dtv_plan;

/* ---- library ---------------------------------------------------------------- */
DTV_API int dtv_version(void);
DTV_API const char* dtv_error_string(int code);
DTV_API const char* dtv_last_error_message(void);
/* Number of kernel launches this library has issued in the process (host-side
 * counter; a stream capture counts the kernels one graph replay launches). */
DTV_API int64_t dtv_launch_count(void);

/* ---- geometry builders (host only, no CUDA) --------------------------------- */
/* Standard circular orbit exactly as the reference Standard layer defines it:
 * beta = angle*pi/180 - pi/2, source -sid*e_x, detector centre (sdd-sid)*e_x,
 * U = e_y (pitch 1), V = e_z, voxel = sid/sdd, step = sid/sdd, scale = sid/sdd,
 * offsets 0, FDK weight (sdd/L)^2 * pi/N.
 * Replaces the geometry part of JITStandardGeometry.forward/backward
 * (Standard/plug/include/forward.h:3, backward.h:3;
 *  kernel/forwardKernel.cu:30-40,63,82,110-113; kernel/backwardKernel.cu:29-44,50).
 * `views` must hold 12*n_angles doubles; g->views is set to it. */
DTV_API int dtv_geometry_standard(dtv_geometry* g, double* views, const float* angles_deg, int32_t n_angles,
                          const int32_t volume_size[3], const int32_t detector_size[2], float sid,
                          float sdd);
/* Vector geometry of the Beijing layer: project_vector[n][12] = source(3),
 * detector(3), v(3), u(3) with the z of source and detector negated, voxel 1,
 * step 1, scale 1 (the Python layer multiplies by sampleInterval), offsets
 * volume 0 / detector 1/2, weight SDD/L * 2*pi/(n/21), extent quirk on.
 * Replaces JITBeijingGeometry.forward/backward geometry
 * (Beijing/plug/include/forward.h:3, backward.h:3;
 *  kernel/forwardKernel.cu:24-35; kernel/backwardKernel.cu:21-43). */
DTV_API int dtv_geometry_vector(dtv_geometry* g, double* views, const float* project_vector, int32_t n_views,
                        const int32_t volume_size[3], const int32_t detector_size[2]);
/* General circular orbit with explicit voxel size and detector pitch, centred
 * voxels and pixels, exact-chord sampling with step = smallest voxel edge,
 * scale = step, FDK weight (sdd/L)^2 * pi/N. No reference counterpart (the
 * reference ties voxel and pitch together, forwardKernel.cu:63). */
DTV_API int dtv_geometry_circular(dtv_geometry* g, double* views, const double* angles_deg, int32_t n_angles,
                          const int32_t volume_size[3], const double voxel[3],
                          const int32_t detector_size[2], const double pitch[2], double sod,
                          double sdd);

/* ---- plans ------------------------------------------------------------------- */
/* Uploads the per-view tables (computed in FP64 on the host) and allocates the
 * sampler staging for volumes/sinograms of up to max_batch items on `device`.
 * This is the ONLY call that allocates device memory. */
DTV_API int dtv_plan_create(const dtv_geometry* g, int32_t max_batch, int32_t flags, int32_t device,
                    dtv_plan** out);
DTV_API int dtv_plan_destroy(dtv_plan* plan);
/* Launch knobs of a plan, set by an autotuner that times the candidates; the
 * results do not depend on them (each ray's sum is the same computation):
 *   DTV_TUNE_FP_RAY_TILE: the forward projector's ray tile, 0..7, as
 *   (block tu x tv pixels, warp wu x wv pixels): 0 (16x16, 8x4) default,
 *   1 (16x16, 16x2), 2 (32x8, 32x1), 3 (16x16, 4x8), 4 (32x8, 8x4),
 *   5 (8x32, 8x4), 6 (64x4, 32x1), 7 (8x32, 4x8).
 * No counterpart in the reference (its kernels use one fixed launch shape). */
#define DTV_TUNE_FP_RAY_TILE 1
/*   DTV_TUNE_FP_TEX_SHARE: with DTV_PLAN_TMA, how many eighths of the ray
 *   tiles sample through the texture unit (0..8; the rest go through shared
 *   memory). No counterpart in the reference. */
#define DTV_TUNE_FP_TEX_SHARE 2
/*   DTV_TUNE_ADJOINT: how dtv_backward_adjoint scatters, 0 = per 16^3 brick
 *   through shared-memory atomics, 1 = into per-cell records of four floats
 *   with 16-byte vector atomics, then a gather (needs DTV_PLAN_ADJOINT; the
 *   default for such plans). No counterpart in the reference. */
#define DTV_TUNE_ADJOINT 3
/*   DTV_TUNE_FP_BAND: the order in which the forward projector's ray tiles
 *   run. 0: view by view. B > 0: bands of B tile rows, every view of a band
 *   before the next band, so the volume slab a band's rays cross stays in L2
 *   across views. Default: 4 when the plan's staged volume exceeds 32 MB, else
 *   0. 0..4096; not used by DTV_PLAN_TMA plans. No counterpart in the
 *   reference. */
#define DTV_TUNE_FP_BAND 4
/*   DTV_TUNE_BP_WARP: the backprojector's columns per warp and per quad of
 *   4 consecutive lanes: 0 = 16 x 2 (quads 4 x 1), 1 = 8 x 4 (4 x 1),
 *   2 = 4 x 8 (4 x 1), 3 = 8 x 4 (2 x 2), 4 = 4 x 8 (2 x 2, default). The
 *   texture unit serves a quad in fewer wavefronts when its four footprints
 *   are close. No counterpart in the reference. */
#define DTV_TUNE_BP_WARP 5
DTV_API int dtv_plan_set_tuning(dtv_plan* plan, int32_t key, int32_t value);
DTV_API int dtv_plan_get_tuning(const dtv_plan* plan, int32_t key, int32_t* value);
/* Device-side error bits of the plan's kernels (0: none; 1: a shared-memory
 * staging wait of the DTV_PLAN_TMA forward projector ran out of its iteration
 * limit, the outputs of that launch are invalid). Synchronises the device;
 * reset != 0 clears the bits. No counterpart in the reference. */
DTV_API int dtv_plan_device_status(dtv_plan* plan, int32_t* status, int32_t reset);
/* Number of forward-projector ray samples per volume (exact chord count under
 * the plan's phase rule, the algorithmic work unit), computed on the host. */
DTV_API int dtv_plan_fp_samples(const dtv_plan* plan, double* samples_per_volume);

/* Several plans' forward projections in ONE kernel launch (no counterpart in
 * the reference, which launched per view): plans[k] projects vols[k] (one
 * volume each, any size and view count) into outs[k], with the epilogue of
 * dtv_forward against gs[k] (no abs_sum). DTV_PLAN_TEX_PAIRS plans on one
 * device, each at most once (a plan stages its volume into its own texture);
 * the per-ray sums equal those of dtv_forward. Up to 24 plans share a launch,
 * more take further launches. */
DTV_API int dtv_forward_many(dtv_plan* const* plans, const void* const* vols, int32_t vol_dtype,
                             float* const* outs, int32_t count, int32_t epilogue,
                             const float* const* gs, float sigma, void* stream);
/* Several plans' FDK backprojections in one launch (plans with a sinogram
 * texture: DTV_PLAN_TEX or DTV_PLAN_TEX_PAIRS, each at most once); values equal
 * dtv_backward's. */
DTV_API int dtv_backward_many(dtv_plan* const* plans, const float* const* sinos,
                              float* const* outs, int32_t count, int32_t accumulate, void* stream);

/* ---- FBP filter ------------------------------------------------------------ */
/* Cosine weighting and spatial Ram-Lak ramp of the FBP layers
 * (Standard/StandardGeometry.py:51-93, Beijing/BeijingGeometry.py:57-84), fused:
 * out[r, u] = sum_t k[t] * cos(i, u + t - W/2) * in[r, u + t - W/2] over rows r of
 * `width` (W) columns, zero outside the row, with the reference's W+1-tap kernel
 * k (1/8 at the centre, -1/(2 pi^2 d^2) at odd offsets d, 0 at even ones) and
 * cos(i, j) = sdd / sqrt(sdd^2 + (i - mid_i)^2 + (j - mid_j)^2), i = r mod
 * rows_per_view. adjoint != 0 applies the transpose (ramp, then the weight).
 * W even (the reference's reshape fails for odd W), at most 8192. */
DTV_API int dtv_fbp_filter(const float* in, float* out, int64_t rows, int32_t rows_per_view,
                           int32_t width, float sdd, float mid_i, float mid_j, int32_t adjoint,
                           void* stream);

/* ---- projectors ------------------------------------------------------------- */
/* Ray-driven forward projector (Standard/plug/kernel/forwardKernel.cu:22-143;
 * Beijing/plug/kernel/forwardKernel.cu:17-135), one launch for all views and
 * batch items. vol_dtype: DTV_F32 / DTV_F16 / DTV_BF16. `g` (sinogram shaped)
 * is read by the RESIDUAL and PDHG epilogues and may be NULL for STORE.
 * If abs_sum is not NULL, sum |FP(vol) - g| (or |FP(vol)| for STORE) is ADDED
 * to *abs_sum (device double; DTVCP.py:55). */
DTV_API int dtv_forward(dtv_plan* plan, const void* vol, int32_t vol_dtype, int32_t batch, float* out,
                int32_t epilogue, const float* g, float sigma, double* abs_sum, void* stream);
/* Voxel-driven FDK-weighted backprojector, all views in one pass, each voxel
 * written once (Standard/plug/kernel/backwardKernel.cu:22-110;
 * Beijing/plug/kernel/backwardKernel.cu:18-104). out is overwritten, or
 * accumulated into when accumulate != 0. */
DTV_API int dtv_backward(dtv_plan* plan, const float* sino, int32_t batch, float* out, int32_t accumulate,
                 void* stream);
/* out = base + BP(sino), same backprojector as dtv_backward; base may equal
 * out (then it is dtv_backward with accumulate != 0), or else must not
 * overlap it. No reference
 * counterpart: DTVCP's corrected iterations add the stored backprojector
 * correction this way without copying it into out first. */
DTV_API int dtv_backward_onto(dtv_plan* plan, const float* sino, int32_t batch, const float* base,
                              float* out, void* stream);

/* The correction passes of a texture-filtered z-pair plan `fast`
 * (DTV_PLAN_TEX_PAIRS, not DTV_PLAN_TMA) against an exact-weight plan `exact`
 * (DTV_PLAN_PAIRS_EXACT) of the same geometry, one launch per operator that
 * samples through both plans. No reference counterpart (the reference has
 * one texture-filtered operator pair); the dual step is DTVCP.py:38-39.
 *
 * dtv_pdhg_forward_refresh: per ray, with e = E(vol) and a = A(vol) the exact
 * and fast projections (each with the bits dtv_forward gives on its plan),
 *   g_eff = g + (a - e),  w = (w + sigma*(e - g)) / (1 + sigma),
 * and abs_sum[0] += sum |e - g| (device double, may be NULL). g_eff must not
 * alias g or w.
 *
 * dtv_backward_refresh: out = BP_exact(sino), e_b = out - BP_fast(sino) (out
 * and e_b distinct buffers of volume shape; above 640 views e_b adds the
 * difference of each chunk of 640 views, a sum rounded per chunk). Plans of different geometry,
 * sampler or device return DTV_ERR_INVALID. */
DTV_API int dtv_pdhg_forward_refresh(dtv_plan* fast, dtv_plan* exact, const void* vol,
                                     int32_t vol_dtype, int32_t batch, const float* g, float sigma,
                                     float* w, float* g_eff, double* abs_sum, void* stream);
DTV_API int dtv_backward_refresh(dtv_plan* fast, dtv_plan* exact, const float* sino, int32_t batch,
                                 float* out, float* e_b, void* stream);
/* Exact transpose of dtv_forward's STORE map (same samples, same weights,
 * software sampler): out = A^T sino. No reference counterpart — the reference
 * paired forward with the FDK backprojector as its gradient
 * (Standard/StandardGeometry.py:17-21,30-34). out is overwritten. */
DTV_API int dtv_backward_adjoint(dtv_plan* plan, const float* sino, int32_t batch, float* out, void* stream);

/* One-shot entries with the reference's argument lists (host geometry, the
 * sizes as arrays); each builds a plan, runs, and frees it (synchronising the
 * stream). They replace JITStandardGeometry.forward/backward
 * (Standard/plug/include/forward.h:3, backward.h:3) and
 * JITBeijingGeometry.forward/backward (Beijing/plug/include/forward.h:3,
 * backward.h:3) for callers that keep no plan. */
DTV_API int dtv_standard_forward(const float* volume, int32_t batch, const float* angles_deg,
                         int32_t n_angles, const int32_t volume_size[3],
                         const int32_t detector_size[2], float sid, float sdd, int32_t device,
                         float* sino, void* stream);
DTV_API int dtv_standard_backward(const float* sino, int32_t batch, const float* angles_deg,
                          int32_t n_angles, const int32_t volume_size[3],
                          const int32_t detector_size[2], float sid, float sdd, int32_t device,
                          float* volume, void* stream);
DTV_API int dtv_vector_forward(const float* volume, int32_t batch, const int32_t volume_size[3],
                       const int32_t detector_size[2], const float* project_vector,
                       int32_t n_views, int32_t device, float* sino, void* stream);
DTV_API int dtv_vector_backward(const float* sino, int32_t batch, const int32_t volume_size[3],
                        const int32_t detector_size[2], const float* project_vector,
                        int32_t n_views, int32_t device, float* volume, void* stream);

/* ---- directional finite differences ------------------------------------------ */
/* out = D_axis f (transpose=0) or D_axis^T f (transpose=1) for axis 0,1,2 = x,y,z,
 * f and out [batch][nz][ny][nx] f32. D = shift - I with the reference's boundary
 * rows: the last index along the axis gives -f; with quirk != 0 the y operator
 * uses offset size[1] over the flat index and wraps the last row of a slice into
 * the next slice exactly as model/PDHG/Utils/Gradients.py:8-34 builds its sparse
 * matrices; quirk == 0 stops at each slice's last row. */
DTV_API int dtv_diff(const float* f, float* out, const int32_t size[3], int32_t batch, int32_t axis,
             int32_t transpose, int32_t quirk, void* stream);
/* sums[a] += sum |D_a f| over the batch, a = x, y, z (device doubles;
 * DTVCP.py:34-37). f_dtype DTV_F32 or DTV_F16. */
DTV_API int dtv_diff_abs_sums(const void* f, int32_t f_dtype, const int32_t size[3], int32_t batch,
                      int32_t quirk, double* sums, void* stream);

/* ---- L1-ball projection ------------------------------------------------------- */
/* Bytes of device workspace the L1-ball threshold search needs per channel. */
DTV_API int64_t dtv_l1ball_workspace_bytes(void);
/* w = sign(v) * max(|v| - lambda, 0) with lambda >= 0 solving
 * sum max(|v| - lambda, 0) = radius, or w = v when sum|v| < radius
 * (model/PDHG/Utils/L1ball.py:4-17, which Newton-iterates lambda with a host
 * sync per step; here an exact 3-pass radix search on the device).
 * radius: device double. workspace: dtv_l1ball_workspace_bytes() bytes of
 * device memory, 8-byte aligned, any contents (the call clears what it uses).
 * lambda_out (device double, may be NULL) receives lambda. */
DTV_API int dtv_l1ball(const float* v, float* w, int64_t n, const double* radius, void* workspace,
               double* lambda_out, void* stream);

/* dtv_l1ball for callers that cannot allocate device memory where they
 * project (a host that reserves the GPU up front and exposes no allocator, a
 * C/Fortran caller without a device allocator, a loop that must not call
 * cudaMalloc/cudaFree because cudaFree synchronises the device). No
 * counterpart in the reference. Same arguments and result as dtv_l1ball minus
 * the workspace: the search runs in a 49,200-byte array compiled into the
 * library (one per GPU, held until the process exits). n must not exceed
 * 2^31-1 (larger n returns DTV_ERR_INVALID). The first call on each device
 * looks up that array's address; make the first call before any stream
 * capture. All calls on a device share the array, so calls that overlap on
 * the GPU (different streams, or different host threads) race; each call
 * clears it before use. The address is cached per device ordinal for the
 * life of the library: do not call it after cudaDeviceReset (or any other
 * teardown of the device's primary context) in the same process. Allocates
 * nothing. */
DTV_API int dtv_l1ball_noalloc(const float* v, float* w, int64_t n, const double* radius,
                               double* lambda_out, void* stream);

/* ---- DTV by Chambolle-Pock (model/PDHG/DTVCP.py:29-60) ------------------------- */
typedef struct dtv_pdhg_params {
  float sigma;  /* dual step (DTVCP.py:27)                    */
  float tau;    /* primal step (DTVCP.py:26)                  */
  float mu;     /* non-negativity weight (DTVCP.py:22)        */
  float v[3];   /* per-direction weights v1,v2,v3 (:19-21)   */
  int32_t quirk; /* reference D_y wrap (Gradients.py:18-25)   */
  int32_t f_dtype; /* storage of fbar, the projector input: DTV_F32, DTV_F16 or DTV_BF16
                      (f itself is always FP32) */
} dtv_pdhg_params;

/* Workspace bytes of the fused dual step (three L1-ball channels). The
 * workspace is device memory, 8-byte aligned, of any contents: the dual step
 * clears it, and the primal step reads the thresholds the dual step left. */
DTV_API int64_t dtv_pdhg_workspace_bytes(void);
/* Dual step, fused: p_ = p + v1*sigma*D_x fbar (q_, s_ likewise, stored in
 * place), c = -relu(-c - sigma*mu*fbar), then the per-direction L1-ball
 * thresholds of |p_|/sigma with radii v_a * t[a] (t: device doubles, the
 * constraint levels sum|D_a f|). (DTVCP.py:41-47, L1ball.py:4-17) */
DTV_API int dtv_pdhg_dual(const void* fbar, float* p, float* q, float* s, float* c, const int32_t size[3],
                  int32_t batch, const dtv_pdhg_params* prm, const double* t, void* workspace,
                  void* stream);
/* Primal step, fused: p,q,s <- p_ - sigma*sign(p_)*l1ball(...) (clip to the
 * thresholds found by dtv_pdhg_dual), fnew = f - recon - tau*(v1 D_x^T p +
 * v2 D_y^T q + v3 D_z^T s + mu c), fbar = 2 fnew - f, f = fnew.
 * (DTVCP.py:44-54) */
DTV_API int dtv_pdhg_primal(float* f, void* fbar, const float* recon, float* p, float* q, float* s,
                    const float* c, const int32_t size[3], int32_t batch,
                    const dtv_pdhg_params* prm, const void* workspace, void* stream);
/* The same two steps with the duals' clip deferred from one iteration's
 * primal step into the next iteration's dual step, which loads the duals
 * anyway. No counterpart in the reference (an iteration of DTVCP.py:38-54
 * split differently).
 * dtv_pdhg_primal_defer computes f and fbar as dtv_pdhg_primal does but
 * stores no clipped dual: p, q, s keep the values dtv_pdhg_dual left, and
 * the three thresholds it clipped them with are written to carry (device
 * float[3], not in the workspace).
 * dtv_pdhg_dual_defer is dtv_pdhg_dual on the duals clipped to carry as it
 * loads them (carry NULL: no clip, the same as dtv_pdhg_dual).
 * A clip leaves an unclipped element's bits unchanged, so an iteration
 * sequence of dual_defer(carry) / primal_defer(carry) gives the bits of
 * dtv_pdhg_dual / dtv_pdhg_primal; ending it with dtv_pdhg_primal leaves the
 * same clipped duals too. */
DTV_API int dtv_pdhg_dual_defer(const void* fbar, float* p, float* q, float* s, float* c,
                                const int32_t size[3], int32_t batch, const dtv_pdhg_params* prm,
                                const double* t, void* workspace, const float* carry,
                                void* stream);
DTV_API int dtv_pdhg_primal_defer(float* f, void* fbar, const float* recon, float* p, float* q,
                                  float* s, const float* c, const int32_t size[3], int32_t batch,
                                  const dtv_pdhg_params* prm, const void* workspace, float* carry,
                                  void* stream);

/* ---- FISTA (model/FISTA/FISTA.py:16-27) ------------------------------------------ */
/* d = y - L*bp; x = sign(d)*max(|d| - thresh, 0); y = x + momentum*(x - x_prev);
 * x_prev = x. n elements, all f32. */
DTV_API int dtv_fista_update(float* y, float* x_prev, const float* bp, int64_t n, float L, float thresh,
                     float momentum, void* stream);
/* dtv_fista_update for several volumes (y[k], x_prev[k], bp[k] of n[k]
 * elements) with one L, threshold and momentum, in one launch. No counterpart
 * in the reference. */
DTV_API int dtv_fista_update_many(float* const* y, float* const* x_prev, const float* const* bp,
                                  const int64_t* n, int32_t count, float L, float thresh,
                                  float momentum, void* stream);

/* ---- FISTA-DTV (model/FISTA/DTVFISTA.py:23-43) ---------------------------------- */
/* z = relu(f - sigma*bp) (z may alias bp). */
DTV_API int dtv_relu_step(const float* f, const float* bp, float* z, int64_t n, float sigma, void* stream);
/* fnew = sum_a t_a D_a^T thr_a(D_a z) + z, f = fnew + momentum*(fnew - f), where
 * thr_a(x) = sign(x)*max(|x| - v_a, 0) (quirk == 0) or, reproducing the
 * reference's torch.max(tensor) call (DTVFISTA.py:34-36), sign(x)*M_a with
 * M_a = max_i(|D_a z|_i - v_a) (quirk != 0; needs `maxes`, 3 device floats
 * filled by dtv_dtvfista_maxes). quirk also selects the reference's y
 * difference (see dtv_diff). dtv_dtvfista_maxes uses maxes[0..2] as scratch. */
DTV_API int dtv_dtvfista_maxes(const float* z, const int32_t size[3], int32_t batch, const float v[3],
                       float* maxes, void* stream);
DTV_API int dtv_dtvfista_update(float* f, const float* z, const int32_t size[3], int32_t batch,
                        const float v[3], const float t[3], float momentum, int32_t quirk,
                        const float* maxes, void* stream);

/* ---- ASD-POCS (model/PDHG/ASDPOCS.py:28-47) ------------------------------------- */
/* f -= beta*bp and, if l1 is not NULL, *l1 += sum |f_old - f_new| (device
 * double; the numerator of l1_loss(f0, f), ASDPOCS.py:33-34). */
DTV_API int dtv_axpy_l1(float* f, const float* bp, float beta, double* l1, int64_t n, void* stream);
/* One normalised-TV descent step: f -= davg[0] * sum_a D_a^T (D_a f / (|grad f| + 1)),
 * |grad f| = sqrt(sum_a (D_a f)^2), computed from a snapshot copy `f_in` into
 * `f_out` (they must differ). davg is a device float. (ASDPOCS.py:38-43) */
DTV_API int dtv_tv_descent(const float* f_in, float* f_out, const int32_t size[3], int32_t batch,
                   int32_t quirk, const float* davg, void* stream);

/* out[0] = (float)(in[0] * scale) on the device (scalar glue that keeps
 * data-dependent step sizes such as davg = alpha * dp on the GPU, ASDPOCS.py:35). */
DTV_API int dtv_scale_scalar(const double* in, double scale, float* out, void* stream);

/* out = a*x + b*y over n elements (out may alias x or y). No counterpart in the
 * reference: the operator-error correction of DTVCP (exact minus fast
 * projection, added to the fast one). */
DTV_API int dtv_lincomb(const float* x, float a, const float* y, float b, float* out, int64_t n,
                        void* stream);
/* The PDHG sinogram dual step from a finished projection fp (DTVCP.py:38-39):
 * w = (w + sigma*(fp - g))/(1 + sigma); abs_sum[0] += sum|fp - g| (device
 * double, may be NULL). The forward projector's DTV_EPI_PDHG epilogue does the
 * same inside the projection. */
DTV_API int dtv_pdhg_sino_dual(float* w, const float* fp, const float* g, float sigma, int64_t n,
                               double* abs_sum, void* stream);
/* sum[0] += sum |a - b| over n elements (device double): ASD-POCS's
 * l1_loss(f, f0) as a sum (model/PDHG/ASDPOCS.py:44). */
DTV_API int dtv_l1_distance(const float* a, const float* b, int64_t n, double* sum, void* stream);
/* davg[0] *= alpha if dg_sum[0] > rmax * dp_sum[0], on the device, so the
 * adaptive step needs no host sync (ASDPOCS.py:45; dp and dg as sums over the
 * same n elements). */
DTV_API int dtv_asd_adapt(const double* dp_sum, const double* dg_sum, float rmax, float alpha,
                          float* davg, void* stream);

/* ---- roofline denominators (benchmarks only) ------------------------------------
 * No counterpart in the reference, which times nothing. The projectors are
 * bound by the texture unit and the exact adjoint by L2 vector reductions, not
 * by HBM; these time each rate on the current device with a kernel that does
 * nothing else. Both allocate, launch on the legacy default stream and
 * synchronise: do not call them inside a stream capture or on a hot path. */
/* Bilinear fetches per second from a layered 2-D texture of 384 x 384 x 64
 * texels: texel_bits 32 (half2, the forward projector's z-pair texel, and the
 * rate of the FP32 sinogram texels) or 64 (half4). */
DTV_API int dtv_measure_texture_fetch_rate(int32_t texel_bits, double* fetches_per_second);
/* The same fetch pattern on a 2-D array that holds the 64 planes as an 8 x 8
 * grid of tiles (texture gather works on 2-D arrays only): gather 0, bilinear
 * fetches of half2 texels; gather 1, gathers (the four unfiltered 32-bit
 * texels of a bilinear footprint in one fetch). */
DTV_API int dtv_measure_texture_gather_rate(int32_t gather, double* fetches_per_second);
/* 16-byte float4 atomicAdd reductions per second into `records` records
 * ([1024, 2^26]; 72 MB = 4.7M records stays in L2): pattern 0, each warp's
 * 32 lanes on 32 consecutive records (the adjoint's neighbouring rays);
 * pattern 1, every lane on a random record. */
DTV_API int dtv_measure_atomic_v4_rate(int64_t records, int32_t pattern, double* atomics_per_second);

#ifdef __cplusplus
}
#endif

#endif /* DTV_B200_H */
