// Forward projector with shared-memory staging of the z-pair volume.
//
// Same ray sums as the z-pair samplers of forward.cu (uniform samples along
// each source-to-pixel ray, trilinear interpolation with border value 0, as in
// Standard/plug/kernel/forwardKernel.cu:22-86 and
// Beijing/plug/kernel/forwardKernel.cu:17-76), restructured so that most
// samples are served from shared memory instead of the texture unit:
//   - a block projects a 16x16-pixel tile of one view. Its rays form a thin
//     pyramid, cut into chunks of up to 16 planes along the tile's dominant
//     in-plane axis (x or y);
//   - per chunk one thread issues a Tensor Memory Accelerator box load
//     (20 x 32 x 20 words of the linear z-pair copy, word = half2(f[z], f[z+1]))
//     into shared memory. The box covers every sample of the chunk with its
//     trilinear footprint; its extent across the chunk is bounded by the four
//     corner rays of the tile (the rays through a pixel rectangle meet any
//     plane inside the quadrilateral of the corner rays' intersections);
//   - each thread interpolates its ray's samples of the chunk from shared
//     memory: 4 word loads per sample, x/y weights in FP16 (both planes at once
//     in half2 arithmetic), z weight and ray sum in FP32.
// A sample belongs to the chunk that holds the floor of its chunk-axis
// coordinate, computed exactly as it is sampled, so every sample is summed
// once. Chunks whose box does not fit the footprint (steep rays, wide tiles)
// read the same words from global memory; tiles whose corner rays do not all
// advance the same way along the chunk axis use the texture unit.
#include <climits>
#include <cuda.h>
#include <cuda_fp16.h>
#include <mutex>

#include "ray.cuh"

namespace dtv {

constexpr int kQA = 20;  // box extent along the chunk axis: 16 planes + 1 + x alignment slack
constexpr int kQO = 32;  // box extent along the other in-plane axis
constexpr int kQL = 20;  // box extent in z-pair layers
constexpr int kQWords = kQA * kQO * kQL;
constexpr unsigned kQBytes = kQWords * 4u;
constexpr int kQTile = 16;                  // tile edge (pixels)
constexpr int kQChunk = 16;                 // longest chunk (planes)
constexpr unsigned kQWaitLimit = 1u << 24;  // polls of one staging wait

struct ChunkBox {
  int lo, hi;  // chunk-axis planes whose samples this chunk sums
  int o0, l0;  // box origin along the other in-plane axis and in layers
  int ok;      // the box holds every footprint of the chunk
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (unsigned i = 0; i < kQWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ float pair_lerp(unsigned w00, unsigned w01, unsigned w10, unsigned w11,
                                           float ax, float ay, float az) {
  const float2 a00 = __half22float2(*reinterpret_cast<const __half2*>(&w00));
  const float2 a01 = __half22float2(*reinterpret_cast<const __half2*>(&w01));
  const float2 a10 = __half22float2(*reinterpret_cast<const __half2*>(&w10));
  const float2 a11 = __half22float2(*reinterpret_cast<const __half2*>(&w11));
  const float l0 = fmaf(ax, a01.x - a00.x, a00.x), l1 = fmaf(ax, a11.x - a10.x, a10.x);
  const float h0 = fmaf(ax, a01.y - a00.y, a00.y), h1 = fmaf(ax, a11.y - a10.y, a10.y);
  const float lo = fmaf(ay, l1 - l0, l0), hi = fmaf(ay, h1 - h0, h0);
  return fmaf(az, hi - lo, lo);
}

// Box in shared memory: word (L, y, x) at ((L - gl0) * by + (y - gy0)) * bx + (x - gx0),
// i.e. floor(z) * bxy + floor(y) * bx + floor(x) - off for the sample's layer
// L = floor(z) + 2. The word index is clamped into the box (a no-op for samples
// of the box's chunk). The x/y interpolation of both planes runs in half2
// arithmetic (FP16 weights, finer than the texture unit's 8-bit ones), the z
// interpolation and the ray sum in FP32.
struct SmemPairSampler {
  const unsigned int* box;
  int bx, bxy, off;
  __device__ __forceinline__ float operator()(float x, float y, float z) const {
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    int q = (int)fz * bxy + (int)fy * bx + (int)fx - off;
    q = min(max(q, 0), kQWords - bx - 2);
    const unsigned int w00 = box[q], w01 = box[q + 1], w10 = box[q + bx], w11 = box[q + bx + 1];
    const __half2 a00 = *reinterpret_cast<const __half2*>(&w00);
    const __half2 a01 = *reinterpret_cast<const __half2*>(&w01);
    const __half2 a10 = *reinterpret_cast<const __half2*>(&w10);
    const __half2 a11 = *reinterpret_cast<const __half2*>(&w11);
    const __half2 hx = __float2half2_rn(x - fx), hy = __float2half2_rn(y - fy);
    const __half2 r0 = __hfma2(hx, __hsub2(a01, a00), a00);
    const __half2 r1 = __hfma2(hx, __hsub2(a11, a10), a10);
    const float2 c = __half22float2(__hfma2(hy, __hsub2(r1, r0), r0));
    return fmaf(z - fz, c.y - c.x, c.x);
  }
};

// The same words read from global memory with explicit zero borders.
struct GlobalPairSampler {
  const unsigned int* lin;  // this batch item
  int nx, ny, pitch, lmax;
  __device__ __forceinline__ unsigned word(int ix, int iy, int L) const {
    return (ix >= 0 && ix < nx && iy >= 0 && iy < ny)
               ? __ldg(lin + ((int64_t)L * ny + iy) * pitch + ix)
               : 0u;
  }
  __device__ __forceinline__ float operator()(float x, float y, float z) const {
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    const int ix = (int)fx, iy = (int)fy;
    const int L = min(max((int)fz + 2, 0), lmax);
    return pair_lerp(word(ix, iy, L), word(ix + 1, iy, L), word(ix, iy + 1, L),
                     word(ix + 1, iy + 1, L), x - fx, y - fy, z - fz);
  }
};

template <class Sampler>
__device__ __forceinline__ void sum_range(const Sampler& smp, const RaySetup& rs, int k, int ke,
                                          float& a0, float& a1) {
  for (; k + 3 < ke; k += 4) {
    float s[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float kf = (float)(k + j);
      s[j] = smp(fmaf(kf, rs.dp[0], rs.p0[0]), fmaf(kf, rs.dp[1], rs.p0[1]),
                 fmaf(kf, rs.dp[2], rs.p0[2]));
    }
    a0 += s[0];
    a1 += s[1];
    a0 += s[2];
    a1 += s[3];
  }
  for (; k < ke; ++k) {
    const float kf = (float)k;
    a0 += smp(fmaf(kf, rs.dp[0], rs.p0[0]), fmaf(kf, rs.dp[1], rs.p0[1]),
              fmaf(kf, rs.dp[2], rs.p0[2]));
  }
}

__global__ void __launch_bounds__(kFPThreads, 4)
    fp_tma_kernel(RayParams rp, const FPView* __restrict__ views,
                  const __grid_constant__ CUtensorMap map_x, const __grid_constant__ CUtensorMap map_y,
                  const cudaTextureObject_t* texs, const unsigned int* __restrict__ lin, int pitch,
                  int max_chunks, int tex_share, FPOut o, int* status) {
  extern __shared__ unsigned char dsm[];
  __shared__ __align__(8) unsigned long long bar;
  __shared__ float s_corner[4][4];  // per corner ray: q_o, c_o, q_z, c_z
  __shared__ int s_amin, s_amax, s_sign_ok;

  const int tiles_u = (rp.nu + kQTile - 1) / kQTile;
  const int tu0 = (blockIdx.x % tiles_u) * kQTile, tv0 = (blockIdx.x / tiles_u) * kQTile;
  const int t = threadIdx.x, w = t >> 5, l = t & 31;
  const int u = tu0 + (w & 1) * 8 + (l & 7), v = tv0 + (w >> 1) * 4 + (l >> 3);
  const int n = blockIdx.y, b = blockIdx.z;
  const bool live = u < rp.nu && v < rp.nv;
  const FPView& f = views[n];
  float res = 0.f;

  // chunk axis: the larger in-plane component of the tile's central ray
  double rc[3];
#pragma unroll
  for (int c = 0; c < 3; ++c)
    rc[c] = f.d0ms[c] + (tu0 + 0.5 * (kQTile - 1)) * f.u[c] + (tv0 + 0.5 * (kQTile - 1)) * f.v[c];
  const int ax = fabs(rc[0]) >= fabs(rc[1]) ? 0 : 1;
  const int oa = 1 - ax;
  const int sg = rc[ax] > 0.0 ? 1 : -1;

  if (t == 0) {
    s_amin = INT_MAX;
    s_amax = INT_MIN;
    s_sign_ok = 1;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  if (t < 4) {
    const double cu = tu0 + (t & 1) * (kQTile - 1), cv = tv0 + (t >> 1) * (kQTile - 1);
    double r[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) r[c] = f.d0ms[c] + cu * f.u[c] + cv * f.v[c];
    if (r[ax] * rc[ax] > 0.0) {
      const double qo = r[oa] / r[ax], qz = r[2] / r[ax];
      s_corner[t][0] = (float)qo;
      s_corner[t][1] = (float)(f.s[oa] - f.s[ax] * qo);
      s_corner[t][2] = (float)qz;
      s_corner[t][3] = (float)(f.s[2] - f.s[ax] * qz);
    } else {
      s_sign_ok = 0;
    }
  }
  RaySetup rs;
  rs.count = 0;
  if (live) rs = setup_ray(rp, f, u, v, 0.f, 0.f);
  const float p0a = ax == 0 ? rs.p0[0] : rs.p0[1];
  const float dpa = ax == 0 ? rs.dp[0] : rs.dp[1];
  if (rs.count > 0) {
    const int fa0 = (int)floorf(p0a), fa1 = (int)floorf(fmaf((float)(rs.count - 1), dpa, p0a));
    atomicMin(&s_amin, min(fa0, fa1));
    atomicMax(&s_amax, max(fa0, fa1));
  }
  __syncthreads();
  const int amin = s_amin, amax = s_amax;
  const int span = amax - amin + 1;  // <= 0: no samples in the tile

  // Tiles sent to the texture unit (a share of them, or those the chunking
  // cannot serve): the z-pair texture sampler of forward.cu.
  const bool via_tex = ((blockIdx.x + blockIdx.y) & 7) < tex_share || !s_sign_ok ||
                       (span > 0 && (span + 3) / 4 > max_chunks);
  if (via_tex) {
    if (live) {
      const RaySetup rt = setup_ray(rp, f, u, v, 0.5f, 0.f);
      PairSampler smp{texs[b], (float)(rp.nz + 2)};
      const float val = rt.count > 0 ? ray_sum(smp, rt) * rp.scale : 0.f;
      fp_store(rp, o, n, b, u, v, val, res);
    }
    if (o.abs_sum) block_add_double((double)fabsf(res), o.abs_sum);
    return;
  }

  // shared memory: the box (128-byte aligned for the TMA), then the schedule
  const uint32_t dsm_addr = smem_u32(dsm);
  unsigned int* box = reinterpret_cast<unsigned int*>(dsm + (((dsm_addr + 127u) & ~127u) - dsm_addr));
  ChunkBox* sched = reinterpret_cast<ChunkBox*>(box + kQWords);

  // Chunk schedule: the longest chunk length whose boxes all fit; with the
  // shortest one, chunks that still do not fit fall back to global memory.
  int C = kQChunk, nch = 0;
  if (span > 0) {
    for (;;) {
      nch = (span + C - 1) / C;
      int fit = 1;
      for (int c = t; c < nch; c += kFPThreads) {
        ChunkBox cb;
        if (sg > 0) {
          cb.lo = amin + c * C;
          cb.hi = min(cb.lo + C - 1, amax);
        } else {
          cb.hi = amax - c * C;
          cb.lo = max(cb.hi - C + 1, amin);
        }
        const float P0 = (float)cb.lo, P1 = (float)(cb.hi + 1);
        float omn = 3e38f, omx = -3e38f, zmn = 3e38f, zmx = -3e38f;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const float oA = fmaf(P0, s_corner[i][0], s_corner[i][1]);
          const float oB = fmaf(P1, s_corner[i][0], s_corner[i][1]);
          const float zA = fmaf(P0, s_corner[i][2], s_corner[i][3]);
          const float zB = fmaf(P1, s_corner[i][2], s_corner[i][3]);
          omn = fminf(omn, fminf(oA, oB));
          omx = fmaxf(omx, fmaxf(oA, oB));
          zmn = fminf(zmn, fminf(zA, zB));
          zmx = fmaxf(zmx, fmaxf(zA, zB));
        }
        cb.ok = (omx - omn) < 64.f && (zmx - zmn) < 64.f && fabsf(omn) < 1e6f &&
                fabsf(zmn) < 1e6f;
        cb.o0 = 0;
        cb.l0 = 0;
        if (cb.ok) {
          const int fo0 = (int)floorf(omn), fo1 = (int)floorf(omx);
          const int fz0 = (int)floorf(zmn), fz1 = (int)floorf(zmx);
          cb.o0 = fo0 - 1;
          if (ax == 1) cb.o0 &= ~3;  // x origin on a 16-byte boundary
          cb.l0 = fz0 + 1;           // layer of floor(z) + 2, one layer of margin
          cb.ok = (fo1 + 2 - cb.o0 + 1 <= kQO) && (fz1 + 3 - cb.l0 + 1 <= kQL);
        }
        sched[c] = cb;
        fit &= cb.ok;
      }
      if (__syncthreads_and(fit) || C == 4) break;
      C -= 4;
    }
  }

  const int lin_items = pitch * rp.ny * (rp.nz + 3);
  const GlobalPairSampler gsm{lin + (int64_t)b * lin_items, rp.nx, rp.ny, pitch, rp.nz + 2};
  const float inv = rs.count > 0 ? 1.f / dpa : 0.f;
  const uint32_t bar_addr = smem_u32(&bar);
  const uint64_t map_addr =
      reinterpret_cast<uint64_t>(ax == 0 ? &map_x : &map_y);
  uint32_t phase = 0;
  float a0 = 0.f, a1 = 0.f;
  int k = 0;
  for (int c = 0; c < nch; ++c) {
    const ChunkBox cb = sched[c];
    // box origin (x, y) in the volume and extents
    const int gx0 = ax == 0 ? (cb.lo & ~3) : cb.o0;
    const int gy0 = ax == 0 ? cb.o0 : cb.lo;
    const int bx = ax == 0 ? kQA : kQO, by = ax == 0 ? kQO : kQA;
    if (cb.ok) {
      // one thread issues the load and one warp waits for it; the others wait
      // at the block barrier (spinning warps would take issue slots)
      if (t == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_addr),
                     "r"(kQBytes)
                     : "memory");
        asm volatile(
            "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(box)),
            "l"(map_addr), "r"(gx0), "r"(gy0), "r"(cb.l0), "r"(b), "r"(bar_addr)
            : "memory");
      }
      if (w == 0 && !mbar_wait(bar_addr, phase) && l == 0) atomicOr(status, 1);
      phase ^= 1u;
      __syncthreads();
    }
    if (k < rs.count) {
      // first sample past this chunk (the chunk-axis coordinate is monotone in k)
      const float edge = sg > 0 ? (float)(cb.hi + 1) : (float)cb.lo;
      float est = ceilf((edge - p0a) * inv);
      est = fminf(fmaxf(est, (float)k), (float)rs.count);
      int ke = (int)est;
      auto beyond = [&](int kk) {
        const float pa = fmaf((float)kk, dpa, p0a);
        return sg > 0 ? pa >= edge : pa < edge;
      };
      while (ke > k && beyond(ke - 1)) --ke;
      while (ke < rs.count && !beyond(ke)) ++ke;
      if (cb.ok) {
        const SmemPairSampler smp{box, bx, bx * by, (cb.l0 - 2) * bx * by + gy0 * bx + gx0};
        sum_range(smp, rs, k, ke, a0, a1);
      } else {
        sum_range(gsm, rs, k, ke, a0, a1);
      }
      k = ke;
    }
    __syncthreads();  // the box is rewritten by the next chunk's load
  }
  if (live) fp_store(rp, o, n, b, u, v, (a0 + a1) * rp.scale, res);
  if (o.abs_sum) block_add_double((double)fabsf(res), o.abs_sum);
}

// ---- host side ------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = [] {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (EncodeTiledFn) nullptr;
    return reinterpret_cast<EncodeTiledFn>(ptr);
  }();
  return fn;
}

static int tma_max_chunks(const GeomParams& g) {
  // chunk-axis span of a tile's samples: the volume plus one sample step
  // (at most step / voxel planes) and one plane of rounding on each side
  const int ext = (int)ceil(g.step / fmin(g.voxel[0], g.voxel[1])) + 2;
  return (std::max(g.nx, g.ny) + 2 * ext + 4) / 4 + 2;
}

static size_t tma_smem_bytes(const GeomParams& g) {
  return 128 + (size_t)kQBytes + sizeof(ChunkBox) * tma_max_chunks(g);
}

int encode_pair_maps(Plan* p) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return fail(DTV_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  const GeomParams& g = p->gp;
  const size_t smem = tma_smem_bytes(g);
  if (smem > 200 * 1024)
    return fail(DTV_ERR_UNSUPPORTED, "volume too wide for DTV_PLAN_TMA (%zu bytes of staging)", smem);
  const cuuint64_t dims[4] = {(cuuint64_t)g.nx, (cuuint64_t)g.ny, (cuuint64_t)(g.nz + 3),
                              (cuuint64_t)p->max_batch};
  const cuuint64_t row = (cuuint64_t)p->pair_pitch * 4;
  const cuuint64_t strides[3] = {row, row * g.ny, row * g.ny * (g.nz + 3)};
  const cuuint32_t box_x[4] = {kQA, kQO, kQL, 1}, box_y[4] = {kQO, kQA, kQL, 1};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  for (int m = 0; m < 2; ++m) {
    const CUresult r =
        enc(reinterpret_cast<CUtensorMap*>(p->tmap[m]), CU_TENSOR_MAP_DATA_TYPE_UINT32, 4,
            p->d_pair_lin, dims, strides, m == 0 ? box_x : box_y, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(DTV_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  }
  // the kernel's dynamic shared-memory limit is per function: raise it to the
  // largest plan's need (outside any stream capture)
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  cudaFuncAttributes fa;
  DTV_CUDA_TRY(cudaFuncGetAttributes(&fa, fp_tma_kernel));
  if ((size_t)fa.maxDynamicSharedSizeBytes < smem)
    DTV_CUDA_TRY(cudaFuncSetAttribute(fp_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
  return DTV_OK;
}

int fp_tma_launch(Plan* p, const RayParams& rp, const FPOut& o, int batch, cudaStream_t st) {
  const GeomParams& g = p->gp;
  const int tiles = ((g.nu + kQTile - 1) / kQTile) * ((g.nv + kQTile - 1) / kQTile);
  dim3 grid(tiles, g.n_views, batch);
  CUtensorMap mx, my;
  memcpy(&mx, p->tmap[0], sizeof(mx));
  memcpy(&my, p->tmap[1], sizeof(my));
  fp_tma_kernel<<<grid, kFPThreads, tma_smem_bytes(g), st>>>(
      rp, p->d_fpv, mx, my, p->pair_tex_dev, p->d_pair_lin, p->pair_pitch, tma_max_chunks(g),
      p->fp_tex_share, o, p->d_status);
  note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

}  // namespace dtv
