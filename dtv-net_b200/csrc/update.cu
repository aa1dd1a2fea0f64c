// Directional finite differences, the L1-ball threshold search and the fused
// DTV / FISTA / ASD-POCS update kernels.
//
// Finite differences restate model/PDHG/Utils/Gradients.py:8-34, where each
// operator is a sparse matrix D = shift - I: row i is -e_i plus e_{i+o} when
// row i is "valid" (x: (i+1) % X != 0; y: i < N - size[1], with offset
// size[1]; z: i < N - X*Y). The stencils below apply those matrices and their
// transposes without building them. Volume kernels run on a (x, y, z-slab)
// grid: a warp is 32 consecutive x of one row, and each thread marches
// up to kZS slices along z (fewer on small volumes, so the grid fills the
// GPU), carrying the z-neighbour from one slice to the next.
//
// The L1-ball projection (model/PDHG/Utils/L1ball.py:4-17) needs the threshold
// lambda solving sum_i max(a_i - lambda, 0) = r. The reference Newton-iterates
// lambda with a host sync per step. Here it is found exactly by a three-level
// radix search over the IEEE-754 bit patterns of a_i >= 0 (monotone in a_i):
// 1024 / 1024 / 2048 bins on key bits [30:21] / [20:11] / [10:0]. Every bin of
// a level shares one exponent, so its sum is kept exactly as an integer sum of
// 24-bit significands. After the last level the bin is a single value and
// lambda follows in closed form from the counts and sums above it.
#include <atomic>
#include <cstddef>
#include <math.h>

#include <algorithm>
#include <mutex>

#include "common.cuh"

namespace dtv {

// ---- launch helpers ----------------------------------------------------------------
static inline int blocks_for(int64_t n, int threads = 256, int per_sm = 8) {
  int64_t b = (n + threads - 1) / threads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148LL * per_sm));
}

// Shared-memory histogram words are 32-bit; a block may add at most this many
// elements to one (see hist_add).
constexpr int64_t kHistBlockElems = 1LL << 20;

// Grid of a histogram pass over n elements: enough blocks that none adds
// more than kHistBlockElems elements.
static inline int hist_blocks(int64_t n, int threads, int per_sm, int64_t per_thread) {
  const int64_t need = (n + kHistBlockElems - 1) / kHistBlockElems;
  return (int)std::max<int64_t>(blocks_for((n + per_thread - 1) / per_thread, threads, per_sm),
                                need);
}

struct Dims {
  int X, Y, Z;
  int64_t N;  // X*Y*Z
  int quirk;
  int zs;  // slices per thread, 1 .. kZS
};

// block of 64 x 4 threads (each warp 32 consecutive x of one row; a block's
// rows are 256 contiguous bytes, which streams better than 32 x 8), up to 8
// slices per thread
constexpr int kTX = 64, kTY = 4, kZS = 8;
// Blocks a launch should have: four resident blocks of 256 threads on each of
// the 148 SMs. Small volumes take fewer slices per thread to get there.
constexpr int64_t kWantBlocks = 4 * 148;

static Dims make_dims(const int32_t s[3], int quirk, int batch) {
  Dims d;
  d.X = s[0]; d.Y = s[1]; d.Z = s[2];
  d.N = (int64_t)s[0] * s[1] * s[2];
  d.quirk = quirk;
  const int64_t cols = (int64_t)((d.X + kTX - 1) / kTX) * ((d.Y + kTY - 1) / kTY);
  d.zs = kZS;
  while (d.zs > 1 && cols * ((d.Z + d.zs - 1) / d.zs) * batch < kWantBlocks &&
         (int64_t)((d.Z + d.zs / 2 - 1) / (d.zs / 2)) * batch <= 65535)
    d.zs /= 2;
  return d;
}

static int check_dims(const int32_t s[3], int batch) {
  DTV_CHECK(s != nullptr, "NULL size");
  DTV_CHECK(s[0] > 0 && s[1] > 0 && s[2] > 0 && batch > 0, "bad size (%d,%d,%d) x %d", s[0],
            s[1], s[2], batch);
  DTV_CHECK((int64_t)((s[2] + kZS - 1) / kZS) * batch <= 65535,
            "z slabs x batch exceeds the grid limit");
  DTV_CHECK((s[1] + kTY - 1) / kTY <= 65535, "ny too large");
  DTV_CHECK((int64_t)s[0] * s[1] * s[2] <= 2147483647LL, "volume exceeds 2^31-1 voxels");
  return DTV_OK;
}

static dim3 grid3(const Dims& d, int batch) {
  return dim3((d.X + kTX - 1) / kTX, (d.Y + kTY - 1) / kTY, ((d.Z + d.zs - 1) / d.zs) * batch);
}
static const dim3 kBlock3(kTX, kTY);

// Position of this thread: column (x, y) of batch item b, slices [z0, z0+zs).
struct Col {
  int x, y, z0, nz;  // nz = slices this thread handles
  int64_t base;      // b * N
  bool in;
};
__device__ __forceinline__ Col col3(const Dims& d) {
  Col c;
  c.x = blockIdx.x * kTX + threadIdx.x;
  c.y = blockIdx.y * kTY + threadIdx.y;
  const int zslabs = (d.Z + d.zs - 1) / d.zs;
  const int zb = blockIdx.z % zslabs;
  const int b = blockIdx.z / zslabs;
  c.z0 = zb * d.zs;
  c.nz = min(d.zs, d.Z - c.z0);
  c.base = (int64_t)b * d.N;
  c.in = c.x < d.X && c.y < d.Y;
  return c;
}
// The same position for tile `tile` of that grid, in its launch order (x
// tiles fastest, then y tiles, then z-slabs and batch items).
__device__ __forceinline__ Col col3_tile(const Dims& d, int64_t tile) {
  const int tx = (d.X + kTX - 1) / kTX, ty = (d.Y + kTY - 1) / kTY;
  const int bx = (int)(tile % tx);
  const int64_t r = tile / tx;
  const int by = (int)(r % ty);
  const int bz = (int)(r / ty);
  const int zslabs = (d.Z + d.zs - 1) / d.zs;
  Col c;
  c.x = bx * kTX + threadIdx.x;
  c.y = by * kTY + threadIdx.y;
  c.z0 = (bz % zslabs) * d.zs;
  c.nz = min(d.zs, d.Z - c.z0);
  c.base = (int64_t)(bz / zslabs) * d.N;
  c.in = c.x < d.X && c.y < d.Y;
  return c;
}
__device__ __forceinline__ int ltid() { return threadIdx.y * blockDim.x + threadIdx.x; }
__device__ __forceinline__ int lthreads() { return blockDim.x * blockDim.y; }

__device__ __forceinline__ int64_t axis_off(const Dims& d, int a) {
  return a == 0 ? 1 : (a == 1 ? (d.quirk ? d.Y : d.X) : (int64_t)d.X * d.Y);
}
// row i (flat index inside one item) carries the +1 entry at i + off
__device__ __forceinline__ bool row_valid(const Dims& d, int a, int64_t i, int x, int y, int z) {
  if (a == 0) return x < d.X - 1;
  if (a == 1) return d.quirk ? (i < d.N - d.Y) : (y < d.Y - 1);
  return z < d.Z - 1;
}
// column j receives the +1 entry of row j - off
__device__ __forceinline__ bool col_valid(const Dims& d, int a, int64_t j, int x, int y, int z) {
  if (a == 0) return x >= 1;
  if (a == 1) return d.quirk ? (j >= d.Y) : (y >= 1);
  return z >= 1;
}

template <class T>
__device__ __forceinline__ float dfwd(const T* f, const Dims& d, int a, int64_t i, int x, int y,
                                      int z) {
  const float c = load_as_float(f, i);
  return row_valid(d, a, i, x, y, z) ? load_as_float(f, i + axis_off(d, a)) - c : -c;
}

// (x, y, z) of flat index i inside one item (i < 2^31, checked on the host);
// used only for the few neighbour rows that need it
__device__ __forceinline__ void decompose(const Dims& d, int64_t i, int& x, int& y, int& z) {
  const unsigned int ii = (unsigned int)i;
  const unsigned int plane = (unsigned int)d.X * (unsigned int)d.Y;
  const unsigned int zz = ii / plane;
  const unsigned int r = ii - zz * plane;
  const unsigned int yy = r / (unsigned int)d.X;
  z = (int)zz;
  y = (int)yy;
  x = (int)(r - yy * (unsigned int)d.X);
}

// (x, y, z) of row j = i - axis_off(d, a), the row whose +1 entry lands on
// column i of voxel (x, y, z): a step back along axis a, except that the
// quirk's y offset wraps across rows and slices.
__device__ __forceinline__ void prev_row(const Dims& d, int a, int64_t j, int x, int y, int z,
                                         int& xj, int& yj, int& zj) {
  xj = x;
  yj = y;
  zj = z;
  if (a == 0) xj = x - 1;
  else if (a == 2) zj = z - 1;
  else if (!d.quirk) yj = y - 1;
  else decompose(d, j, xj, yj, zj);
}

// ---- warp / block reductions ------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int C>
__device__ __forceinline__ void block_sums_atomic(double (&v)[C], double* dst) {
  __shared__ double red[C][32];
  const int t = ltid(), w = t >> 5, l = t & 31, nw = lthreads() >> 5;
#pragma unroll
  for (int c = 0; c < C; ++c) {
    v[c] = warp_sum(v[c]);
    if (l == 0) red[c][w] = v[c];
  }
  __syncthreads();
  if (t < 32) {
#pragma unroll
    for (int c = 0; c < C; ++c) {
      double s = l < nw ? red[c][l] : 0.0;
      s = warp_sum(s);
      if (l == 0 && s != 0.0) atomicAdd(dst + c, s);
    }
  }
}

// ---- finite differences ---------------------------------------------------------------------
__global__ void __launch_bounds__(256) diff_kernel(const float* __restrict__ f, float* __restrict__ out,
                                                   Dims d, int a, int transpose) {
  const Col c = col3(d);
  if (!c.in) return;
  const float* fb = f + c.base;
  for (int k = 0; k < c.nz; ++k) {
    const int z = c.z0 + k;
    const int64_t i = ((int64_t)z * d.Y + c.y) * d.X + c.x;
    float r;
    if (!transpose) {
      r = dfwd(fb, d, a, i, c.x, c.y, z);
    } else {
      r = -__ldg(fb + i);
      if (col_valid(d, a, i, c.x, c.y, z)) r += __ldg(fb + i - axis_off(d, a));
    }
    out[c.base + i] = r;
  }
}

template <class T>
__global__ void __launch_bounds__(256) diff_abs_sums_kernel(const T* __restrict__ f, Dims d,
                                                            double* __restrict__ sums) {
  const Col c = col3(d);
  double acc[3] = {0.0, 0.0, 0.0};
  if (c.in) {
    const T* fb = f + c.base;
    float s0 = 0.f, s1 = 0.f, s2 = 0.f;
    // unrolled: the slices' loads are independent and can all be in flight
#pragma unroll 4
    for (int k = 0; k < c.nz; ++k) {
      const int z = c.z0 + k;
      const int64_t i = ((int64_t)z * d.Y + c.y) * d.X + c.x;
      s0 += fabsf(dfwd(fb, d, 0, i, c.x, c.y, z));
      s1 += fabsf(dfwd(fb, d, 1, i, c.x, c.y, z));
      s2 += fabsf(dfwd(fb, d, 2, i, c.x, c.y, z));
    }
    acc[0] = s0; acc[1] = s1; acc[2] = s2;
  }
  block_sums_atomic<3>(acc, sums);
}

// ---- L1-ball radix search ------------------------------------------------------------------
constexpr int kL1B1 = 1024, kL1B2 = 1024, kL1B3 = 2048;
constexpr int kL1S1 = 21, kL1S2 = 11;  // key >> 21: level-1 bin; >> 11: level-2 prefix

struct L1Chan {
  double radius;
  double c_above;
  double t_above;
  double lambda;
  unsigned int prefix;  // key bits above the current level's bins
  unsigned int maxkey;
  int done;
  float thresh;
  unsigned int cnt1[kL1B1];
  unsigned int cnt2[kL1B2];
  unsigned int cnt3[kL1B3];
  unsigned long long sum1[kL1B1];
  unsigned long long sum2[kL1B2];
  unsigned long long sum3[kL1B3];
};
static_assert(sizeof(L1Chan) % 16 == 0, "L1Chan alignment");
static_assert(sizeof(L1Chan) == 49200, "L1Chan size is part of the documented interface");

__device__ __forceinline__ unsigned int sig24(unsigned int key) {
  const unsigned int m = key & 0x7FFFFFu;
  return (key & 0x7F800000u) ? (m | 0x800000u) : m;
}

// Shared-memory histograms hold three 32-bit words per bin: the count and
// the sums of the low and high 12 bits of each element's 24-bit significand
// (h[0..nb) counts, h[nb..2nb) low sums, h[2nb..3nb) high sums). Each block
// adds at most 2^20 elements, so no word overflows; hist_flush folds them
// into the exact 64-bit sums of the global histogram.

__device__ __forceinline__ void hist_add(unsigned int* h, int nb, int bin, unsigned int key,
                                         bool active) {
  if (!active) return;
  const unsigned int sig = sig24(key);
  atomicAdd(h + bin, 1u);
  atomicAdd(h + nb + bin, sig & 0xFFFu);
  atomicAdd(h + 2 * nb + bin, sig >> 12);
}

// Four elements (a thread's four consecutive x in the four-x dual step): one
// add of all four when they are active and share a bin, else one add each.
// The duals of a reconstruction concentrate in a few bins as the iterations
// go on (clipped to a common bound, then moved by one small step), and lanes
// adding to one shared-memory word serialise; neighbours usually share their
// bin then. The four significands sum to S < 2^26, added as S mod 2^12 to
// the low word and S / 2^12 to the high word: the flushed sum
// low + high * 2^12 is the same integer, and the high word's adds still
// total at most the block's significand sum / 2^12 < 2^32.
__device__ __forceinline__ void hist_add4(unsigned int* h, int nb, const int (&bin)[4],
                                          const unsigned int (&key)[4], const bool (&act)[4]) {
  if (act[0] && act[1] && act[2] && act[3] && bin[0] == bin[1] && bin[1] == bin[2] &&
      bin[2] == bin[3]) {
    const unsigned int S = sig24(key[0]) + sig24(key[1]) + sig24(key[2]) + sig24(key[3]);
    atomicAdd(h + bin[0], 4u);
    atomicAdd(h + nb + bin[0], S & 0xFFFu);
    atomicAdd(h + 2 * nb + bin[0], S >> 12);
    return;
  }
#pragma unroll
  for (int e = 0; e < 4; ++e) hist_add(h, nb, bin[e], key[e], act[e]);
}

__device__ __forceinline__ void hist_clear(unsigned int* h, int nb) {
  for (int i = ltid(); i < 3 * nb; i += lthreads()) h[i] = 0u;
}

__device__ __forceinline__ void hist_flush(const unsigned int* h, int nb, unsigned int* gcnt,
                                           unsigned long long* gsum) {
  for (int i = ltid(); i < nb; i += lthreads()) {
    if (h[i]) {
      atomicAdd(gcnt + i, h[i]);
      atomicAdd(gsum + i, (unsigned long long)h[nb + i] +
                              ((unsigned long long)h[2 * nb + i] << 12));
    }
  }
}

// Level-2 / level-3 histogram pass over one channel (keys of |x|), static
// shared memory for the largest (level-3) bin count.
template <int C>
__global__ void l1_hist_kernel(const float* __restrict__ x0, const float* __restrict__ x1,
                               const float* __restrict__ x2, int64_t n, L1Chan* chans, int level) {
  static_assert(C == 1, "one channel");
  __shared__ unsigned int hs[3 * kL1B3];
  L1Chan& ch = chans[0];
  if (ch.done) return;
  const int nb = level == 2 ? kL1B2 : kL1B3;
  hist_clear(hs, nb);
  const unsigned int pre = ch.prefix;
  const int pshift = level == 2 ? kL1S1 : kL1S2;
  __syncthreads();
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const unsigned int key = __float_as_uint(__ldg(x0 + t)) & 0x7FFFFFFFu;
    const int bin = level == 2 ? (int)((key >> kL1S2) & (kL1B2 - 1)) : (int)(key & (kL1B3 - 1));
    hist_add(hs, nb, bin, key, (key >> pshift) == pre);
  }
  __syncthreads();
  if (level == 2) hist_flush(hs, nb, ch.cnt2, ch.sum2);
  else hist_flush(hs, nb, ch.cnt3, ch.sum3);
}

// Level-2 or level-3 pass over three channels at once (the fused PDHG path);
// dynamic shared memory: 3 channels x 3 words x bins. Each thread loads 4
// consecutive elements of each channel per step (16-byte loads); the arrays
// are 16-byte aligned and the last n % 4 elements are done by block 0.
__device__ __forceinline__ void hist3_one(unsigned int* hs, int nb, int level, const bool* live,
                                          const unsigned int* pre, int pshift, const float (&x)[3]) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const unsigned int key = __float_as_uint(x[c]) & 0x7FFFFFFFu;
    const int bin = level == 2 ? (int)((key >> kL1S2) & (kL1B2 - 1)) : (int)(key & (kL1B3 - 1));
    hist_add(hs + c * 3 * nb, nb, bin, key, live[c] && (key >> pshift) == pre[c]);
  }
}

__global__ void __launch_bounds__(512) l1_hist3_kernel(const float* __restrict__ x0,
                                                       const float* __restrict__ x1,
                                                       const float* __restrict__ x2, int64_t n,
                                                       L1Chan* chans, int level) {
  extern __shared__ unsigned int hs[];
  const int nb = level == 2 ? kL1B2 : kL1B3;
  bool live[3];
  unsigned int pre[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    live[c] = !chans[c].done;
    pre[c] = chans[c].prefix;
  }
  if (!live[0] && !live[1] && !live[2]) return;
  for (int i = threadIdx.x; i < 9 * nb; i += blockDim.x) hs[i] = 0u;
  __syncthreads();
  const int pshift = level == 2 ? kL1S1 : kL1S2;
  const int64_t n4 = n / 4;
  const float4* v0 = reinterpret_cast<const float4*>(x0);
  const float4* v1 = reinterpret_cast<const float4*>(x1);
  const float4* v2 = reinterpret_cast<const float4*>(x2);
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n4;
       t += (int64_t)gridDim.x * blockDim.x) {
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a, c = a;
    if (live[0]) a = __ldg(v0 + t);
    if (live[1]) b = __ldg(v1 + t);
    if (live[2]) c = __ldg(v2 + t);
    const float e0[3] = {a.x, b.x, c.x}, e1[3] = {a.y, b.y, c.y};
    const float e2[3] = {a.z, b.z, c.z}, e3[3] = {a.w, b.w, c.w};
    hist3_one(hs, nb, level, live, pre, pshift, e0);
    hist3_one(hs, nb, level, live, pre, pshift, e1);
    hist3_one(hs, nb, level, live, pre, pshift, e2);
    hist3_one(hs, nb, level, live, pre, pshift, e3);
  }
  if (blockIdx.x == 0) {  // tail: the last n % 4 elements
    const int64_t t = n4 * 4 + threadIdx.x;
    if (t < n) {
      const float e[3] = {live[0] ? x0[t] : 0.f, live[1] ? x1[t] : 0.f, live[2] ? x2[t] : 0.f};
      hist3_one(hs, nb, level, live, pre, pshift, e);
    }
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (!live[c]) continue;
    if (level == 2) hist_flush(hs + c * 3 * nb, nb, chans[c].cnt2, chans[c].sum2);
    else hist_flush(hs + c * 3 * nb, nb, chans[c].cnt3, chans[c].sum3);
  }
}

// Level-1 histogram of a plain array (standalone L1-ball).
__global__ void l1_hist1_kernel(const float* __restrict__ v, int64_t n, L1Chan* ch) {
  __shared__ unsigned int hs[3 * kL1B1];
  hist_clear(hs, kL1B1);
  __syncthreads();
  unsigned int kmax = 0;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const unsigned int key = __float_as_uint(__ldg(v + t)) & 0x7FFFFFFFu;
    kmax = max(kmax, key);
    hist_add(hs, kL1B1, (int)(key >> kL1S1), key, true);
  }
  __syncthreads();
  hist_flush(hs, kL1B1, ch->cnt1, ch->sum1);
  for (int o = 16; o > 0; o >>= 1) kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
  if ((threadIdx.x & 31) == 0 && kmax) atomicMax(&ch->maxkey, kmax);
}

__device__ __forceinline__ double bin_scale(unsigned int key_lo) {
  const int e = (int)((key_lo >> 23) & 0xFFu);
  return ldexp(1.0, (e > 0 ? e : 1) - 150);
}

// One block (1024 threads) per channel: picks the bin holding lambda at
// `level`, records the counts/sums above it, zeroes that level's histogram,
// and after level 3 stores the threshold.
__global__ void __launch_bounds__(1024) l1_select_kernel(L1Chan* chans, int level) {
  L1Chan& ch = chans[blockIdx.x];
  if (ch.done) return;
  const int nb = level == 1 ? kL1B1 : (level == 2 ? kL1B2 : kL1B3);
  unsigned int* cnt = level == 1 ? ch.cnt1 : (level == 2 ? ch.cnt2 : ch.cnt3);
  unsigned long long* sum = level == 1 ? ch.sum1 : (level == 2 ? ch.sum2 : ch.sum3);
  const int per = nb / 1024;  // 1 or 2 bins per thread, thread t owns bins [t*per, t*per+per)
  const unsigned int kbase =
      level == 1 ? 0u : (level == 2 ? (ch.prefix << kL1S1) : (ch.prefix << kL1S2));
  const int bshift = level == 1 ? kL1S1 : (level == 2 ? kL1S2 : 0);
  double c_loc = 0.0, t_loc = 0.0;
  double cb[2] = {0.0, 0.0}, tb[2] = {0.0, 0.0};
  const int t = threadIdx.x;
  for (int q = 0; q < per; ++q) {
    const int j = t * per + q;
    const unsigned int klo = kbase | ((unsigned int)j << bshift);
    cb[q] = (double)cnt[j];
    tb[q] = (double)sum[j] * bin_scale(klo);
    c_loc += cb[q];
    t_loc += tb[q];
  }
  // inclusive suffix scan over threads (higher t = higher bins)
  __shared__ double wc[32], wt[32];
  __shared__ int best;
  const int w = t >> 5, l = t & 31;
  double c_s = c_loc, t_s = t_loc;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double c2 = __shfl_down_sync(0xffffffffu, c_s, o);
    const double t2 = __shfl_down_sync(0xffffffffu, t_s, o);
    if (l + o < 32) {
      c_s += c2;
      t_s += t2;
    }
  }
  if (l == 0) {
    wc[w] = c_s;
    wt[w] = t_s;
  }
  if (t == 0) best = -1;
  __syncthreads();
  double c_hi = 0.0, t_hi = 0.0;  // warps above this one
  for (int ww = w + 1; ww < 32; ++ww) {
    c_hi += wc[ww];
    t_hi += wt[ww];
  }
  // C/T over bins strictly above this thread's bins, plus what earlier levels fixed
  const double c_above = ch.c_above + c_hi + (c_s - c_loc);
  const double t_above = ch.t_above + t_hi + (t_s - t_loc);
  const double radius = ch.radius;
  if (level == 1 && t == 0) {
    double ttot = 0.0;
    for (int ww = 0; ww < 32; ++ww) ttot += wt[ww];
    if (ttot < radius) {  // sum|v| < b: the reference returns v (L1ball.py:5-6)
      ch.done = 1;
      ch.thresh = 0.f;
      ch.lambda = 0.0;
    } else if (radius <= 0.0) {  // every lambda >= max|v| solves it; take max|v|
      ch.done = 1;
      ch.thresh = __uint_as_float(ch.maxkey);
      ch.lambda = (double)ch.thresh;
    }
  }
  __syncthreads();
  if (!ch.done) {
    // scan this thread's bins from the top down
    double ca = c_above, ta = t_above;
    for (int q = per - 1; q >= 0; --q) {
      const int j = t * per + q;
      const unsigned int klo = kbase | ((unsigned int)j << bshift);
      const double lo = (double)__uint_as_float(klo);
      const double cj = ca + cb[q], tj = ta + tb[q];
      if (tj - lo * cj >= radius) {
        atomicMax(&best, j);
        break;
      }
      ca = cj;
      ta = tj;
    }
  }
  __syncthreads();
  // Below level 1 the parent bin passed the test at its lower edge, so the
  // lowest bin of this level passes too in exact arithmetic; if the sums,
  // added in another order, round just under the radius, take that bin.
  const int J = (best < 0 && level > 1) ? 0 : best;
  if (!ch.done && J >= 0 && J >= t * per && J < t * per + per) {
    // this thread owns bin J: fix the new "above" totals
    double ca = c_above, ta = t_above;
    for (int q = per - 1; q >= 0; --q) {
      const int j = t * per + q;
      if (j == J) break;
      ca += cb[q];
      ta += tb[q];
    }
    const unsigned int klo = kbase | ((unsigned int)J << bshift);
    if (level < 3) {
      ch.c_above = ca;
      ch.t_above = ta;
      ch.prefix = klo >> bshift;
    } else {
      const double a_star = (double)__uint_as_float(klo);
      const double a_next = (double)__uint_as_float(klo + 1u);
      double lam = ca > 0.0 ? (ta - radius) / ca : a_star;
      lam = fmin(fmax(lam, a_star), a_next);
      ch.lambda = lam;
      ch.thresh = (float)lam;
      ch.done = 1;
    }
  }
}

// Resets channels for a new search, one block per channel: radius from
// device doubles, or s_c * t[c] (a scale times a device constraint level),
// and every histogram bin of the three levels cleared, so a search starts
// from a defined state whatever the workspace held before (fresh
// cudaMalloc'd memory, or a search that stopped part-way).
constexpr int kL1ResetThreads = 256;
__global__ void __launch_bounds__(kL1ResetThreads)
l1_reset_kernel(L1Chan* chans, int C, const double* radius, const double* t, float s0, float s1,
                float s2) {
  const int c = blockIdx.x;
  if (c >= C) return;
  L1Chan& ch = chans[c];
  // cnt1..cnt3 and sum1..sum3 are contiguous: 4096 32-bit and 4096 64-bit words
  unsigned int* bins = ch.cnt1;
  constexpr int kWords = (kL1B1 + kL1B2 + kL1B3) * (1 + 2);
  for (int i = threadIdx.x; i < kWords; i += kL1ResetThreads) bins[i] = 0u;
  if (threadIdx.x == 0) {
    const float sc = c == 0 ? s0 : (c == 1 ? s1 : s2);
    ch.radius = radius ? radius[c] : (double)sc * t[c];
    ch.c_above = 0.0;
    ch.t_above = 0.0;
    ch.lambda = 0.0;
    ch.prefix = 0;
    ch.maxkey = 0;
    ch.done = 0;
    ch.thresh = 0.f;
  }
}
static_assert(offsetof(L1Chan, sum3) + sizeof(((L1Chan*)0)->sum3) ==
                  offsetof(L1Chan, cnt1) + (kL1B1 + kL1B2 + kL1B3) * 3 * sizeof(unsigned int),
              "histogram words are contiguous");

__global__ void l1_apply_kernel(const float* __restrict__ v, float* __restrict__ w, int64_t n,
                                const L1Chan* ch, double* lambda_out) {
  const float lam = ch->thresh;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const float x = __ldg(v + t);
    const float m = fmaxf(fabsf(x) - lam, 0.f);
    w[t] = x > 0.f ? m : (x < 0.f ? -m : 0.f);
  }
  if (lambda_out && blockIdx.x == 0 && threadIdx.x == 0) *lambda_out = ch->lambda;
}

// ---- fused PDHG dual step (DTVCP.py:41-47) + level-1 histograms --------------------------------
// Slices per thread of the dual step (its duals of all slices are held in
// registers before any store, so fewer slices mean more resident blocks).
constexpr int kDualZS = 4;
// clip(x, m) = sign(x) * min(|x|, m): the duals' projection by the L1-ball
// threshold m. Wherever the result compares equal to x it has x's own bits
// (-0 included: the sign is copied from x), so storing it in place of an
// unclipped element changes no memory.
__device__ __forceinline__ float clipf(float x, float m) { return copysignf(fminf(fabsf(x), m), x); }

// The thresholds a deferred clip applies to the duals a dual step loads:
// those the previous primal step clipped with (carry), or +inf (no clip).
__device__ __forceinline__ float carry_thresh(const float* carry, int a) {
  return carry ? carry[a] : __int_as_float(0x7f800000);
}

template <class T>
__global__ void __launch_bounds__(256, 6) pdhg_dual_kernel(const T* __restrict__ fbar, float* __restrict__ p,
                                                        float* __restrict__ q, float* __restrict__ s,
                                                        float* __restrict__ c, Dims d, float a0,
                                                        float a1, float a2, float smu,
                                                        L1Chan* chans, int64_t n_tiles,
                                                        const float* carry) {
  __shared__ unsigned int hs[3][3 * kL1B1];
  const float m0 = carry_thresh(carry, 0), m1 = carry_thresh(carry, 1),
              m2 = carry_thresh(carry, 2);
  for (int i = ltid(); i < 9 * kL1B1; i += lthreads()) (&hs[0][0])[i] = 0u;
  __syncthreads();
  unsigned int kmax[3] = {0u, 0u, 0u};
  // a block walks several tiles and flushes its histograms once
  for (int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
  const Col cl = col3_tile(d, tile);
  const T* fb = fbar + cl.base;
  const int64_t plane = (int64_t)d.X * d.Y;
  const int64_t oy = axis_off(d, 1);
  const int64_t i0 = ((int64_t)cl.z0 * d.Y + cl.y) * d.X + cl.x;
  const bool xv = cl.x < d.X - 1;
  const bool yv_clean = cl.y < d.Y - 1;
  // phase 1: the duals of all slices are loaded first (a later slice's loads
  // cannot move above an earlier slice's stores to the same arrays), then
  // stencils and stores
  float pv[kDualZS], qv[kDualZS], sv[kDualZS], cv[kDualZS];
#pragma unroll
  for (int k = 0; k < kDualZS; ++k) {
    pv[k] = qv[k] = sv[k] = cv[k] = 0.f;
    if (cl.in && k < cl.nz) {
      const int64_t t = cl.base + i0 + k * plane;
      pv[k] = clipf(p[t], m0);
      qv[k] = clipf(q[t], m1);
      sv[k] = clipf(s[t], m2);
      cv[k] = c[t];
    }
  }
  unsigned int keys[3][kDualZS];
#pragma unroll
  for (int k = 0; k < kDualZS; ++k) {
    keys[0][k] = keys[1][k] = keys[2][k] = 0u;
    if (cl.in && k < cl.nz) {
      const int64_t i = i0 + k * plane;
      const int z = cl.z0 + k;
      const float fc = load_as_float(fb, i);
      const float gx = xv ? load_as_float(fb, i + 1) - fc : -fc;
      const bool yv = d.quirk ? (i < d.N - d.Y) : yv_clean;
      const float gy = yv ? load_as_float(fb, i + oy) - fc : -fc;
      const float gz = z < d.Z - 1 ? load_as_float(fb, i + plane) - fc : -fc;
      const int64_t t = cl.base + i;
      const float np = fmaf(a0, gx, pv[k]), nq = fmaf(a1, gy, qv[k]), ns = fmaf(a2, gz, sv[k]);
      p[t] = np;
      q[t] = nq;
      s[t] = ns;
      // -relu(-c - sigma*mu*fbar): stays 0 wherever fbar >= 0, stored only on change
      const float cn = fminf(fmaf(smu, fc, cv[k]), 0.f);
      if (cn != cv[k]) c[t] = cn;
      keys[0][k] = __float_as_uint(np) & 0x7FFFFFFFu;
      keys[1][k] = __float_as_uint(nq) & 0x7FFFFFFFu;
      keys[2][k] = __float_as_uint(ns) & 0x7FFFFFFFu;
    }
  }
  // phase 2: level-1 histograms (warp-synchronous; every lane takes part)
#pragma unroll
  for (int k = 0; k < kDualZS; ++k) {
    const bool in = cl.in && k < cl.nz;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      kmax[a] = max(kmax[a], keys[a][k]);
      hist_add(hs[a], kL1B1, (int)(keys[a][k] >> kL1S1), keys[a][k], in);
    }
  }
  }
  __syncthreads();
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    hist_flush(hs[a], kL1B1, chans[a].cnt1, chans[a].sum1);
    unsigned int km = kmax[a];
    for (int o = 16; o > 0; o >>= 1) km = max(km, __shfl_xor_sync(0xffffffffu, km, o));
    if ((ltid() & 31) == 0 && km) atomicMax(&chans[a].maxkey, km);
  }
}

// Four consecutive values as floats (16-byte aligned for float, 8-byte for
// the 16-bit types).
__device__ __forceinline__ float4 load4_as_float(const float* p, int64_t i) {
  return __ldg(reinterpret_cast<const float4*>(p + i));
}
__device__ __forceinline__ float4 load4_as_float(const __half* p, int64_t i) {
  const uint2 w = __ldg(reinterpret_cast<const uint2*>(p + i));
  const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&w.x));
  const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&w.y));
  return make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float4 load4_as_float(const __nv_bfloat16* p, int64_t i) {
  const uint2 w = __ldg(reinterpret_cast<const uint2*>(p + i));
  const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w.x));
  const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w.y));
  return make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float4 clip4(float4 v, float m) {
  return make_float4(clipf(v.x, m), clipf(v.y, m), clipf(v.z, m), clipf(v.w, m));
}
__device__ __forceinline__ float4 f4_zero() { return make_float4(0.f, 0.f, 0.f, 0.f); }

// The same dual step with four consecutive x per thread: the duals move as
// 16-byte vectors and f-bar's x-neighbours come from the thread's own vector,
// for about a third of the instructions per voxel. For rows of a multiple of
// 4 voxels (and, with the D_y wrap, a multiple of 4 rows: the wrapped
// neighbour vector then stays aligned). A block of 64 x 4 threads covers
// 256 x 4 columns and kX4ZS slices; the duals of all its slices are loaded
// before any store, as in pdhg_dual_kernel.
constexpr int kX4TX = 256, kX4ZS = 2;
template <class T>
__global__ void __launch_bounds__(256, 4) pdhg_dual_x4_kernel(const T* __restrict__ fbar,
                                                           float* __restrict__ p,
                                                           float* __restrict__ q,
                                                           float* __restrict__ s,
                                                           float* __restrict__ c, Dims d,
                                                           float a0, float a1, float a2,
                                                           float smu, L1Chan* chans,
                                                           int n_tiles, const float* carry) {
  __shared__ unsigned int hs[3][3 * kL1B1];
  __shared__ float msh[3];  // thresholds of the deferred clip
  for (int i = ltid(); i < 9 * kL1B1; i += lthreads()) (&hs[0][0])[i] = 0u;
  if (ltid() < 3) msh[ltid()] = carry_thresh(carry, ltid());
  __syncthreads();
  unsigned int kmax[3] = {0u, 0u, 0u};
  const int tx = (d.X + kX4TX - 1) / kX4TX, ty = (d.Y + kTY - 1) / kTY;
  const int zslabs = (d.Z + kX4ZS - 1) / kX4ZS;
  const int64_t plane = (int64_t)d.X * d.Y;
  const int64_t oy = axis_off(d, 1);
  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const int bx = tile % tx, r = tile / tx;
    const int by = r % ty, bz = r / ty;
    const int x0 = bx * kX4TX + (int)threadIdx.x * 4, y = by * kTY + (int)threadIdx.y;
    const int z0 = (bz % zslabs) * kX4ZS;
    const int nz = min(kX4ZS, d.Z - z0);
    const int64_t base = (int64_t)(bz / zslabs) * d.N;
    const bool in = x0 < d.X && y < d.Y;
    const int64_t i0 = ((int64_t)z0 * d.Y + y) * d.X + x0;
    const T* fb = fbar + base;
    float4 P[kX4ZS], Q[kX4ZS], S[kX4ZS], C[kX4ZS];
#pragma unroll
    for (int k = 0; k < kX4ZS; ++k) {
      P[k] = Q[k] = S[k] = C[k] = f4_zero();
      if (in && k < nz) {
        const int64_t t = base + i0 + k * plane;
        P[k] = clip4(*reinterpret_cast<const float4*>(p + t), msh[0]);
        Q[k] = clip4(*reinterpret_cast<const float4*>(q + t), msh[1]);
        S[k] = clip4(*reinterpret_cast<const float4*>(s + t), msh[2]);
        C[k] = *reinterpret_cast<const float4*>(c + t);
      }
    }
    float4 fc = in ? load4_as_float(fb, i0) : f4_zero();
#pragma unroll
    for (int k = 0; k < kX4ZS; ++k) {
      if (!(in && k < nz)) continue;
      const int64_t i = i0 + k * plane;
      const int z = z0 + k;
      const bool zv = z < d.Z - 1;
      const float4 fn = zv ? load4_as_float(fb, i + plane) : f4_zero();
      // with the wrap, i and N - Y are multiples of 4: all four share the test
      const bool yv = d.quirk ? (i < d.N - d.Y) : (y < d.Y - 1);
      const float4 fy = yv ? load4_as_float(fb, i + oy) : f4_zero();
      const bool xlast = x0 + 3 < d.X - 1;  // the 4th voxel has an x-neighbour
      const float fx4 = xlast ? load_as_float(fb, i + 4) : 0.f;
      const float fcs[4] = {fc.x, fc.y, fc.z, fc.w};
      const float gxs[4] = {fc.y - fc.x, fc.z - fc.y, fc.w - fc.z, xlast ? fx4 - fc.w : -fc.w};
      const float fys[4] = {fy.x, fy.y, fy.z, fy.w};
      const float fns[4] = {fn.x, fn.y, fn.z, fn.w};
      const float ps[4] = {P[k].x, P[k].y, P[k].z, P[k].w};
      const float qs[4] = {Q[k].x, Q[k].y, Q[k].z, Q[k].w};
      const float ss[4] = {S[k].x, S[k].y, S[k].z, S[k].w};
      const float cs[4] = {C[k].x, C[k].y, C[k].z, C[k].w};
      float np[4], nq[4], ns[4], cw[4];
      bool cc = false;
      const int64_t t = base + i;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float gy = yv ? fys[e] - fcs[e] : -fcs[e];
        const float gz = zv ? fns[e] - fcs[e] : -fcs[e];
        np[e] = fmaf(a0, gxs[e], ps[e]);
        nq[e] = fmaf(a1, gy, qs[e]);
        ns[e] = fmaf(a2, gz, ss[e]);
        // -relu(-c - sigma*mu*fbar): stays 0 wherever fbar >= 0; a vector is
        // stored only if one of its elements changes, the others keeping
        // their own bytes
        const float cn = fminf(fmaf(smu, fcs[e], cs[e]), 0.f);
        cc |= cn != cs[e];
        cw[e] = cn != cs[e] ? cn : cs[e];
      }
      if (cc) *reinterpret_cast<float4*>(c + t) = make_float4(cw[0], cw[1], cw[2], cw[3]);
      *reinterpret_cast<float4*>(p + t) = make_float4(np[0], np[1], np[2], np[3]);
      *reinterpret_cast<float4*>(q + t) = make_float4(nq[0], nq[1], nq[2], nq[3]);
      *reinterpret_cast<float4*>(s + t) = make_float4(ns[0], ns[1], ns[2], ns[3]);
      const bool all[4] = {true, true, true, true};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const float* nv = a == 0 ? np : (a == 1 ? nq : ns);
        unsigned int k[4];
        int b[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          k[e] = __float_as_uint(nv[e]) & 0x7FFFFFFFu;
          b[e] = (int)(k[e] >> kL1S1);
          kmax[a] = max(kmax[a], k[e]);
        }
        hist_add4(hs[a], kL1B1, b, k, all);
      }
      fc = fn;
    }
  }
  __syncthreads();
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    hist_flush(hs[a], kL1B1, chans[a].cnt1, chans[a].sum1);
    unsigned int km = kmax[a];
    for (int o = 16; o > 0; o >>= 1) km = max(km, __shfl_xor_sync(0xffffffffu, km, o));
    if ((ltid() & 31) == 0 && km) atomicMax(&chans[a].maxkey, km);
  }
}

// ---- fused PDHG primal step (DTVCP.py:44-54) ----------------------------------------------------
// Without carry the duals are clipped in place; neighbours may read a value
// before or after its clip, and clipping is idempotent, so both give the same
// result. With carry (the deferred clip) they are only read.
template <class T>
__global__ void __launch_bounds__(256) pdhg_primal_kernel(float* __restrict__ f, T* __restrict__ fbar,
                                                          const float* __restrict__ recon, float* p,
                                                          float* q, float* s,
                                                          const float* __restrict__ c, Dims d,
                                                          float tau, float mu, float v0, float v1,
                                                          float v2, const L1Chan* chans,
                                                          float* carry) {
  const float m0 = chans[0].thresh, m1 = chans[1].thresh, m2 = chans[2].thresh;
  // carry: the clipped duals are not stored; the thresholds go to carry, and
  // the next dual step clips the duals as it loads them
  if (carry && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && ltid() < 3)
    carry[ltid()] = chans[ltid()].thresh;
  const Col cl = col3(d);
  if (!cl.in) return;
  const int64_t plane = (int64_t)d.X * d.Y;
  const int64_t oy = axis_off(d, 1);
  float* pb = p + cl.base;
  float* qb = q + cl.base;
  float* sb = s + cl.base;
  int64_t i = ((int64_t)cl.z0 * d.Y + cl.y) * d.X + cl.x;
  float sprev = cl.z0 >= 1 ? clipf(sb[i - plane], m2) : 0.f;  // s(i - XY), carried along z
  for (int k = 0; k < cl.nz; ++k, i += plane) {
    const float pr = pb[i], qr = qb[i], sr = sb[i];
    const float ps = clipf(pr, m0), qs = clipf(qr, m1), ss = clipf(sr, m2);
    float dx = -ps, dy = -qs, dz = -ss;
    if (cl.x >= 1) dx += clipf(pb[i - 1], m0);
    const bool yv = d.quirk ? (i >= d.Y) : (cl.y >= 1);
    if (yv) dy += clipf(qb[i - oy], m1);
    if (cl.z0 + k >= 1) dz += sprev;
    // only clipped duals change; the others keep their bytes without a store
    if (!carry) {
      if (ps != pr) pb[i] = ps;
      if (qs != qr) qb[i] = qs;
      if (ss != sr) sb[i] = ss;
    }
    sprev = ss;
    const int64_t t = cl.base + i;
    const float reg = fmaf(v0, dx, fmaf(v1, dy, fmaf(v2, dz, mu * c[t])));
    const float fo = f[t];
    // explicit FMAs: every instance of the step rounds the same way
    const float fn = fmaf(-tau, reg, fo - recon[t]);
    store_from_float(fbar, t, fmaf(2.f, fn, -fo));
    f[t] = fn;
  }
}

// Four floats as a 16-bit or 32-bit vector store (16-byte aligned for float,
// 8-byte for the 16-bit types).
__device__ __forceinline__ void store4_from_float(float* p, int64_t i, float4 v) {
  *reinterpret_cast<float4*>(p + i) = v;
}
__device__ __forceinline__ void store4_from_float(__half* p, int64_t i, float4 v) {
  const __half2 a = __floats2half2_rn(v.x, v.y), b = __floats2half2_rn(v.z, v.w);
  uint2 w;
  w.x = *reinterpret_cast<const unsigned int*>(&a);
  w.y = *reinterpret_cast<const unsigned int*>(&b);
  *reinterpret_cast<uint2*>(p + i) = w;
}
__device__ __forceinline__ void store4_from_float(__nv_bfloat16* p, int64_t i, float4 v) {
  const __nv_bfloat162 a = __floats2bfloat162_rn(v.x, v.y), b = __floats2bfloat162_rn(v.z, v.w);
  uint2 w;
  w.x = *reinterpret_cast<const unsigned int*>(&a);
  w.y = *reinterpret_cast<const unsigned int*>(&b);
  *reinterpret_cast<uint2*>(p + i) = w;
}

// The primal step with four consecutive x per thread (the conditions of
// pdhg_dual_x4_kernel): 16-byte loads of f, the backprojection, the duals
// and c; the x-neighbour of the first voxel comes from one scalar load, the
// others from the thread's own vector. Same arithmetic per voxel as
// pdhg_primal_kernel.
template <class T>
__global__ void __launch_bounds__(256, 4) pdhg_primal_x4_kernel(float* __restrict__ f,
                                                             T* __restrict__ fbar,
                                                             const float* __restrict__ recon,
                                                             float* p, float* q, float* s,
                                                             const float* __restrict__ c, Dims d,
                                                             float tau, float mu, float v0,
                                                             float v1, float v2,
                                                             const L1Chan* chans, float* carry) {
  if (carry && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && ltid() < 3)
    carry[ltid()] = chans[ltid()].thresh;
  const int x0 = (blockIdx.x * kTX + (int)threadIdx.x) * 4;
  const int y = blockIdx.y * kTY + (int)threadIdx.y;
  const int zslabs = (d.Z + d.zs - 1) / d.zs;
  const int z0 = (int)(blockIdx.z % zslabs) * d.zs;
  const int nz = min(d.zs, d.Z - z0);
  if (x0 >= d.X || y >= d.Y) return;
  const int64_t base = (int64_t)(blockIdx.z / zslabs) * d.N;
  const float m0 = chans[0].thresh, m1 = chans[1].thresh, m2 = chans[2].thresh;
  const int64_t plane = (int64_t)d.X * d.Y;
  const int64_t oy = axis_off(d, 1);
  float* pb = p + base;
  float* qb = q + base;
  float* sb = s + base;
  int64_t i = ((int64_t)z0 * d.Y + y) * d.X + x0;
  float sprev[4] = {0.f, 0.f, 0.f, 0.f};  // clipped s(i - XY), carried along z
  if (z0 >= 1) {
    const float4 sv = *reinterpret_cast<const float4*>(sb + i - plane);
    sprev[0] = clipf(sv.x, m2); sprev[1] = clipf(sv.y, m2);
    sprev[2] = clipf(sv.z, m2); sprev[3] = clipf(sv.w, m2);
  }
  for (int k = 0; k < nz; ++k, i += plane) {
    const float4 P = *reinterpret_cast<const float4*>(pb + i);
    const float4 Q = *reinterpret_cast<const float4*>(qb + i);
    const float4 S = *reinterpret_cast<const float4*>(sb + i);
    const int64_t t = base + i;
    const float4 Cv = __ldg(reinterpret_cast<const float4*>(c + t));
    const float4 Fv = *reinterpret_cast<const float4*>(f + t);
    const float4 Rv = __ldg(reinterpret_cast<const float4*>(recon + t));
    const float pr[4] = {P.x, P.y, P.z, P.w}, qr[4] = {Q.x, Q.y, Q.z, Q.w};
    const float sr[4] = {S.x, S.y, S.z, S.w}, cs[4] = {Cv.x, Cv.y, Cv.z, Cv.w};
    const float fo[4] = {Fv.x, Fv.y, Fv.z, Fv.w}, rc[4] = {Rv.x, Rv.y, Rv.z, Rv.w};
    float ps[4], qs[4], ss[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      ps[e] = clipf(pr[e], m0);
      qs[e] = clipf(qr[e], m1);
      ss[e] = clipf(sr[e], m2);
    }
    const float pl = x0 >= 1 ? clipf(pb[i - 1], m0) : 0.f;  // the first voxel's x-neighbour
    const bool yv = d.quirk ? (i >= d.Y) : (y >= 1);        // shared by the four (aligned)
    float qn[4] = {0.f, 0.f, 0.f, 0.f};
    if (yv) {
      const float4 Qn = *reinterpret_cast<const float4*>(qb + i - oy);
      qn[0] = clipf(Qn.x, m1); qn[1] = clipf(Qn.y, m1);
      qn[2] = clipf(Qn.z, m1); qn[3] = clipf(Qn.w, m1);
    }
    const bool zv = z0 + k >= 1;
    // only vectors with a clipped dual are stored, as one 16-byte store. An
    // unclipped element's clip has its own bits (clipf), so the store writes
    // the same memory as element stores would, and a neighbour reading
    // concurrently sees the value or its clip, which are equal. With carry
    // nothing is stored: the next dual step clips the duals as it loads them.
    if (!carry) {
      bool cp = false, cq = false, cs_ = false;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        cp |= ps[e] != pr[e];
        cq |= qs[e] != qr[e];
        cs_ |= ss[e] != sr[e];
      }
      if (cp) *reinterpret_cast<float4*>(pb + i) = make_float4(ps[0], ps[1], ps[2], ps[3]);
      if (cq) *reinterpret_cast<float4*>(qb + i) = make_float4(qs[0], qs[1], qs[2], qs[3]);
      if (cs_) *reinterpret_cast<float4*>(sb + i) = make_float4(ss[0], ss[1], ss[2], ss[3]);
    }
    float fn[4], fb[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      float dx = -ps[e], dy = -qs[e], dz = -ss[e];
      if (e > 0) dx += ps[e - 1];
      else if (x0 >= 1) dx += pl;
      if (yv) dy += qn[e];
      if (zv) dz += sprev[e];
      sprev[e] = ss[e];
      const float reg = fmaf(v0, dx, fmaf(v1, dy, fmaf(v2, dz, mu * cs[e])));
      fn[e] = fmaf(-tau, reg, fo[e] - rc[e]);
      fb[e] = fmaf(2.f, fn[e], -fo[e]);
    }
    store4_from_float(fbar, t, make_float4(fb[0], fb[1], fb[2], fb[3]));
    *reinterpret_cast<float4*>(f + t) = make_float4(fn[0], fn[1], fn[2], fn[3]);
  }
}

// ---- FISTA (FISTA.py:21-26) --------------------------------------------------------------------------
__global__ void fista_kernel(float* __restrict__ y, float* __restrict__ xp, const float* __restrict__ bp,
                             int64_t n, float L, float thr, float mom) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const float dd = y[t] - L * bp[t];
    const float m = fmaxf(fabsf(dd) - thr, 0.f);
    const float xi = dd > 0.f ? m : (dd < 0.f ? -m : 0.f);
    y[t] = xi + mom * (xi - xp[t]);
    xp[t] = xi;
  }
}

// The same update for several volumes in one launch: a flat index over the
// volumes' elements, each thread finding its volume from the prefix offsets
// held in the launch parameters.
constexpr int kFistaMany = 64;
struct FistaMany {
  float* y[kFistaMany];
  float* xp[kFistaMany];
  const float* bp[kFistaMany];
  int64_t start[kFistaMany + 1];
  int count;
};

__global__ void fista_many_kernel(const __grid_constant__ FistaMany m, float L, float thr,
                                  float mom) {
  const int64_t total = m.start[m.count];
  int k = 0;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    while (g >= m.start[k + 1]) ++k;  // g only grows within a thread
    const int64_t t = g - m.start[k];
    float* y = m.y[k];
    float* xp = m.xp[k];
    const float dd = y[t] - L * m.bp[k][t];
    const float mm = fmaxf(fabsf(dd) - thr, 0.f);
    const float xi = dd > 0.f ? mm : (dd < 0.f ? -mm : 0.f);
    y[t] = xi + mom * (xi - xp[t]);
    xp[t] = xi;
  }
}

// ---- FISTA-DTV (DTVFISTA.py:29-38) -------------------------------------------------------------------
__global__ void relu_step_kernel(const float* __restrict__ f, const float* bp, float* z, int64_t n,
                                 float sigma) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x)
    z[t] = fmaxf(f[t] - sigma * bp[t], 0.f);
}

__global__ void __launch_bounds__(256) dtvfista_maxes_kernel(const float* __restrict__ z, Dims d,
                                                             unsigned int* maxbits) {
  const Col c = col3(d);
  unsigned int km[3] = {0u, 0u, 0u};
  if (c.in) {
    const float* zb = z + c.base;
    for (int k = 0; k < c.nz; ++k) {
      const int zz = c.z0 + k;
      const int64_t i = ((int64_t)zz * d.Y + c.y) * d.X + c.x;
#pragma unroll
      for (int a = 0; a < 3; ++a)
        km[a] = max(km[a], __float_as_uint(fabsf(dfwd(zb, d, a, i, c.x, c.y, zz))));
    }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    unsigned int k = km[a];
    for (int o = 16; o > 0; o >>= 1) k = max(k, __shfl_xor_sync(0xffffffffu, k, o));
    if ((ltid() & 31) == 0) atomicMax(maxbits + a, k);
  }
}

__global__ void finish_maxes_kernel(const unsigned int* bits, float v0, float v1, float v2,
                                    float* maxes) {
  const int a = threadIdx.x;
  if (a < 3) maxes[a] = __uint_as_float(bits[a]) - (a == 0 ? v0 : (a == 1 ? v1 : v2));
}

__global__ void __launch_bounds__(256) dtvfista_update_kernel(float* __restrict__ f,
                                                              const float* __restrict__ z, Dims d,
                                                              float v0, float v1, float v2,
                                                              float t0, float t1, float t2,
                                                              float mom, int quirk,
                                                              const float* __restrict__ maxes) {
  const Col c = col3(d);
  if (!c.in) return;
  const float vs[3] = {v0, v1, v2}, ts[3] = {t0, t1, t2};
  const float* zb = z + c.base;
  for (int k = 0; k < c.nz; ++k) {
    const int zz = c.z0 + k;
    const int64_t i = ((int64_t)zz * d.Y + c.y) * d.X + c.x;
    float fn = zb[i];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float m = quirk ? maxes[a] : 0.f;
      auto thr = [&](float g) {
        if (quirk) return g > 0.f ? m : (g < 0.f ? -m : 0.f);  // sign(g) * max_i(|g_i| - v)
        const float r = fmaxf(fabsf(g) - vs[a], 0.f);
        return g > 0.f ? r : (g < 0.f ? -r : 0.f);
      };
      float dt = -thr(dfwd(zb, d, a, i, c.x, c.y, zz));
      if (col_valid(d, a, i, c.x, c.y, zz)) {
        const int64_t j = i - axis_off(d, a);
        int xj, yj, zj;
        prev_row(d, a, j, c.x, c.y, zz, xj, yj, zj);
        dt += thr(dfwd(zb, d, a, j, xj, yj, zj));
      }
      fn = fmaf(ts[a], dt, fn);
    }
    const int64_t t = c.base + i;
    const float fo = f[t];
    f[t] = fn + mom * (fn - fo);
  }
}

// ---- ASD-POCS (ASDPOCS.py:33-43) ---------------------------------------------------------------------
__global__ void axpy_l1_kernel(float* __restrict__ f, const float* __restrict__ bp, float beta,
                               double* l1, int64_t n) {
  double acc[1] = {0.0};
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const float o = f[t];
    const float nv = o - beta * bp[t];
    f[t] = nv;
    acc[0] += fabsf(o - nv);
  }
  if (l1) block_sums_atomic<1>(acc, l1);
}

// out = a x + b y.
__global__ void lincomb_kernel(const float* __restrict__ x, float a, const float* __restrict__ y,
                               float b, float* __restrict__ out, int64_t n) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x)
    out[t] = fmaf(a, __ldg(x + t), b * __ldg(y + t));
}

// The PDHG sinogram dual step from a finished projection:
// w = (w + sigma (fp - g)) / (1 + sigma), abs_sum += sum |fp - g|.
__global__ void sino_dual_kernel(float* __restrict__ w, const float* __restrict__ fp,
                                 const float* __restrict__ g, float sigma, int64_t n,
                                 double* abs_sum) {
  double acc[1] = {0.0};
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const float res = __ldg(fp + t) - __ldg(g + t);
    w[t] = (w[t] + sigma * res) / (1.f + sigma);
    acc[0] += fabsf(res);
  }
  if (abs_sum) block_sums_atomic<1>(acc, abs_sum);
}

// sum += sum |a - b| (FP64 accumulation): ASD-POCS's TV-change measure.
__global__ void l1_distance_kernel(const float* __restrict__ a, const float* __restrict__ b,
                                   double* sum, int64_t n) {
  double acc[1] = {0.0};
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x)
    acc[0] += fabsf(__ldg(a + t) - __ldg(b + t));
  block_sums_atomic<1>(acc, sum);
}

// ASD-POCS step-size rule on the device: davg *= alpha when the TV steps
// moved the iterate more than rmax times the data step did.
__global__ void asd_adapt_kernel(const double* dp_sum, const double* dg_sum, float rmax,
                                 float alpha, float* davg) {
  if (threadIdx.x == 0 && *dg_sum > (double)rmax * *dp_sum) *davg *= alpha;
}

__device__ __forceinline__ void grad3(const float* f, const Dims& d, int64_t i, int x, int y, int z,
                                      float g[3]) {
#pragma unroll
  for (int a = 0; a < 3; ++a) g[a] = dfwd(f, d, a, i, x, y, z);
}

__global__ void __launch_bounds__(256) tv_descent_kernel(const float* __restrict__ fin,
                                                         float* __restrict__ fout, Dims d,
                                                         const float* __restrict__ davg) {
  const Col c = col3(d);
  if (!c.in) return;
  const float step = davg[0];
  const float* fb = fin + c.base;
  for (int k = 0; k < c.nz; ++k) {
    const int z = c.z0 + k;
    const int64_t i = ((int64_t)z * d.Y + c.y) * d.X + c.x;
    float g[3];
    grad3(fb, d, i, c.x, c.y, z, g);
    const float nrm = sqrtf(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]) + 1.f;
    float grad = 0.f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      grad -= g[a] / nrm;
      if (col_valid(d, a, i, c.x, c.y, z)) {
        const int64_t j = i - axis_off(d, a);
        int xj, yj, zj;
        prev_row(d, a, j, c.x, c.y, z, xj, yj, zj);
        float gj[3];
        grad3(fb, d, j, xj, yj, zj, gj);
        const float nj = sqrtf(gj[0] * gj[0] + gj[1] * gj[1] + gj[2] * gj[2]) + 1.f;
        grad += gj[a] / nj;
      }
    }
    fout[c.base + i] = fb[i] - step * grad;
  }
}

__global__ void scale_scalar_kernel(const double* in, double scale, float* out) {
  if (threadIdx.x == 0) out[0] = (float)(in[0] * scale);
}

}  // namespace dtv

using namespace dtv;

extern "C" {

int dtv_diff(const float* f, float* out, const int32_t size[3], int32_t batch, int32_t axis,
             int32_t transpose, int32_t quirk, void* stream) {
  DTV_CHECK(f && out && size, "NULL argument");
  DTV_CHECK(f != out, "dtv_diff cannot run in place");
  int rc = check_dims(size, batch);
  if (rc) return rc;
  DTV_CHECK(axis >= 0 && axis <= 2, "axis must be 0, 1 or 2");
  Dims d = make_dims(size, quirk, batch);
  diff_kernel<<<grid3(d, batch), kBlock3, 0, as_stream(stream)>>>(f, out, d, axis, transpose); note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

int dtv_diff_abs_sums(const void* f, int32_t dt, const int32_t size[3], int32_t batch,
                      int32_t quirk, double* sums, void* stream) {
  DTV_CHECK(f && sums && size, "NULL argument");
  DTV_CHECK(dt == DTV_F32 || dt == DTV_F16, "dtype must be f32 or f16");
  int rc = check_dims(size, batch);
  if (rc) return rc;
  Dims d = make_dims(size, quirk, batch);
  if (dt == DTV_F32) {
    diff_abs_sums_kernel<float><<<grid3(d, batch), kBlock3, 0, as_stream(stream)>>>(
        (const float*)f, d, sums); note_launch();
  } else {
    diff_abs_sums_kernel<__half><<<grid3(d, batch), kBlock3, 0, as_stream(stream)>>>(
        (const __half*)f, d, sums); note_launch();
  }
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

int64_t dtv_l1ball_workspace_bytes(void) { return (int64_t)sizeof(L1Chan); }

int dtv_l1ball(const float* v, float* w, int64_t n, const double* radius, void* ws,
               double* lambda_out, void* stream) {
  DTV_CHECK(v && w && radius && ws, "NULL argument");
  DTV_CHECK(n > 0, "n must be positive");
  DTV_CHECK(n <= 2147483647LL, "n = %lld exceeds 2^31-1 (32-bit bin counts)", (long long)n);
  cudaStream_t st = as_stream(stream);
  L1Chan* ch = reinterpret_cast<L1Chan*>(ws);
  l1_reset_kernel<<<1, kL1ResetThreads, 0, st>>>(ch, 1, radius, nullptr, 0.f, 0.f, 0.f); note_launch();
  l1_hist1_kernel<<<hist_blocks(n, 256, 4, 1), 256, 0, st>>>(v, n, ch); note_launch();
  l1_select_kernel<<<1, 1024, 0, st>>>(ch, 1); note_launch();
  l1_hist_kernel<1><<<hist_blocks(n, 256, 4, 1), 256, 0, st>>>(v, nullptr, nullptr, n, ch, 2); note_launch();
  l1_select_kernel<<<1, 1024, 0, st>>>(ch, 2); note_launch();
  l1_hist_kernel<1><<<hist_blocks(n, 256, 4, 1), 256, 0, st>>>(v, nullptr, nullptr, n, ch, 3); note_launch();
  l1_select_kernel<<<1, 1024, 0, st>>>(ch, 3); note_launch();
  l1_apply_kernel<<<blocks_for(n), 256, 0, st>>>(v, w, n, ch, lambda_out); note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

int64_t dtv_pdhg_workspace_bytes(void) { return (int64_t)(3 * sizeof(L1Chan)); }

static int pdhg_dual_impl(const void* fbar, float* p, float* q, float* s, float* c,
                          const int32_t size[3], int32_t batch, const dtv_pdhg_params* prm,
                          const double* t, void* ws, const float* carry, void* stream) {
  DTV_CHECK(fbar && p && q && s && c && size && prm && t && ws, "NULL argument");
  DTV_CHECK(prm->f_dtype == DTV_F32 || prm->f_dtype == DTV_F16 || prm->f_dtype == DTV_BF16,
            "f_dtype must be f32, f16 or bf16");
  int rc = check_dims(size, batch);
  if (rc) return rc;
  Dims d = make_dims(size, prm->quirk, batch);
  const int64_t total = d.N * batch;
  DTV_CHECK(total <= 2147483647LL, "volume x batch exceeds 2^31-1 elements");
  cudaStream_t st = as_stream(stream);
  L1Chan* ch = reinterpret_cast<L1Chan*>(ws);
  const float sg = prm->sigma;
  // radius on |p_| directly: sigma * v_a * t_a (the reference projects |p_|/sigma
  // onto the ball of radius v_a * t_a)
  Dims dd = d;
  dd.zs = std::min(d.zs, kDualZS);
  // tiles of the (x, y, z-slab) grid, walked by at most six resident blocks
  // per SM, each adding at most 2^20 elements to its histograms
  const int64_t tiles = (int64_t)((d.X + kTX - 1) / kTX) * ((d.Y + kTY - 1) / kTY) *
                        ((d.Z + dd.zs - 1) / dd.zs) * batch;
  const int64_t per_block = kHistBlockElems / (kTX * kTY * kDualZS);
  const int grid = (int)std::max<int64_t>(std::min<int64_t>(tiles, 148LL * 6),
                                          (tiles + per_block - 1) / per_block);
  l1_reset_kernel<<<3, kL1ResetThreads, 0, st>>>(ch, 3, nullptr, t, sg * prm->v[0], sg * prm->v[1],
                                    sg * prm->v[2]); note_launch();
  // four x per thread where rows (and, with the D_y wrap, the row count) are
  // multiples of 4 and the arrays allow 16-byte (8-byte for 16-bit fbar) access
  const int fb_align = prm->f_dtype == DTV_F32 ? 16 : 8;
  const bool x4 = d.X % 4 == 0 && (!d.quirk || d.Y % 4 == 0) &&
                  ((uintptr_t)p | (uintptr_t)q | (uintptr_t)s | (uintptr_t)c) % 16 == 0 &&
                  (uintptr_t)fbar % fb_align == 0;
  if (x4) {
    const int64_t t4 = (int64_t)((d.X + kX4TX - 1) / kX4TX) * ((d.Y + kTY - 1) / kTY) *
                       ((d.Z + kX4ZS - 1) / kX4ZS) * batch;
    const int64_t per4 = kHistBlockElems / (kX4TX * kTY * kX4ZS);
    const int g4 = (int)std::max<int64_t>(std::min<int64_t>(t4, 148LL * 4), (t4 + per4 - 1) / per4);
    const float b0 = prm->v[0] * sg, b1 = prm->v[1] * sg, b2 = prm->v[2] * sg, sm = sg * prm->mu;
    if (prm->f_dtype == DTV_F32)
      pdhg_dual_x4_kernel<float><<<g4, kBlock3, 0, st>>>((const float*)fbar, p, q, s, c, d, b0,
                                                          b1, b2, sm, ch, (int)t4, carry);
    else if (prm->f_dtype == DTV_F16)
      pdhg_dual_x4_kernel<__half><<<g4, kBlock3, 0, st>>>((const __half*)fbar, p, q, s, c, d, b0,
                                                           b1, b2, sm, ch, (int)t4, carry);
    else
      pdhg_dual_x4_kernel<__nv_bfloat16><<<g4, kBlock3, 0, st>>>(
          (const __nv_bfloat16*)fbar, p, q, s, c, d, b0, b1, b2, sm, ch, (int)t4, carry);
    note_launch();
  } else if (prm->f_dtype == DTV_F32) {
    pdhg_dual_kernel<float><<<grid, kBlock3, 0, st>>>(
        (const float*)fbar, p, q, s, c, dd, prm->v[0] * sg, prm->v[1] * sg, prm->v[2] * sg,
        sg * prm->mu, ch, tiles, carry); note_launch();
  } else if (prm->f_dtype == DTV_F16) {
    pdhg_dual_kernel<__half><<<grid, kBlock3, 0, st>>>(
        (const __half*)fbar, p, q, s, c, dd, prm->v[0] * sg, prm->v[1] * sg, prm->v[2] * sg,
        sg * prm->mu, ch, tiles, carry); note_launch();
  } else {
    pdhg_dual_kernel<__nv_bfloat16><<<grid, kBlock3, 0, st>>>(
        (const __nv_bfloat16*)fbar, p, q, s, c, dd, prm->v[0] * sg, prm->v[1] * sg,
        prm->v[2] * sg, sg * prm->mu, ch, tiles, carry); note_launch();
  }
  DTV_LAUNCH_CHECK();
  // the shared-memory limit is a per-device function attribute
  static std::atomic<unsigned long long> attr_set{0};
  const int smem3 = 9 * kL1B3 * (int)sizeof(unsigned int);
  int dev = 0;
  DTV_CUDA_TRY(cudaGetDevice(&dev));
  const unsigned long long bit = 1ull << (dev & 63);
  if (!(attr_set.load() & bit)) {
    DTV_CUDA_TRY(cudaFuncSetAttribute(l1_hist3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      smem3));
    attr_set |= bit;
  }
  const int smem2 = 9 * kL1B2 * (int)sizeof(unsigned int);
  l1_select_kernel<<<3, 1024, 0, st>>>(ch, 1); note_launch();
  DTV_CHECK(((uintptr_t)p | (uintptr_t)q | (uintptr_t)s) % 16 == 0, "p, q, s must be 16-byte aligned");
  l1_hist3_kernel<<<hist_blocks(total, 512, 2, 4), 512, smem2, st>>>(p, q, s, total, ch, 2); note_launch();
  l1_select_kernel<<<3, 1024, 0, st>>>(ch, 2); note_launch();
  l1_hist3_kernel<<<hist_blocks(total, 512, 2, 4), 512, smem3, st>>>(p, q, s, total, ch, 3); note_launch();
  l1_select_kernel<<<3, 1024, 0, st>>>(ch, 3); note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

static int pdhg_primal_impl(float* f, void* fbar, const float* recon, float* p, float* q,
                            float* s, const float* c, const int32_t size[3], int32_t batch,
                            const dtv_pdhg_params* prm, const void* ws, float* carry,
                            void* stream) {
  DTV_CHECK(f && fbar && recon && p && q && s && c && size && prm && ws, "NULL argument");
  DTV_CHECK(prm->f_dtype == DTV_F32 || prm->f_dtype == DTV_F16 || prm->f_dtype == DTV_BF16,
            "f_dtype must be f32, f16 or bf16");
  int rc = check_dims(size, batch);
  if (rc) return rc;
  Dims d = make_dims(size, prm->quirk, batch);
  const L1Chan* ch = reinterpret_cast<const L1Chan*>(ws);
  // four x per thread under the conditions of the dual step's vector path
  const int fb_align = prm->f_dtype == DTV_F32 ? 16 : 8;
  const bool x4 = d.X % 4 == 0 && (!d.quirk || d.Y % 4 == 0) &&
                  ((uintptr_t)f | (uintptr_t)recon | (uintptr_t)p | (uintptr_t)q | (uintptr_t)s |
                   (uintptr_t)c) % 16 == 0 &&
                  (uintptr_t)fbar % fb_align == 0;
  if (x4) {
    // a quarter of the x blocks: halve the slices per thread while the grid
    // has fewer than four blocks per SM
    Dims d4 = d;
    const int64_t cols = (int64_t)((d.X / 4 + kTX - 1) / kTX) * ((d.Y + kTY - 1) / kTY);
    while (d4.zs > 1 && cols * ((d.Z + d4.zs - 1) / d4.zs) * batch < kWantBlocks &&
           (int64_t)((d.Z + d4.zs / 2 - 1) / (d4.zs / 2)) * batch <= 65535)
      d4.zs /= 2;
    const dim3 g4((d.X / 4 + kTX - 1) / kTX, (d.Y + kTY - 1) / kTY,
                  ((d.Z + d4.zs - 1) / d4.zs) * batch);
    cudaStream_t st = as_stream(stream);
    if (prm->f_dtype == DTV_F32)
      pdhg_primal_x4_kernel<float><<<g4, kBlock3, 0, st>>>(f, (float*)fbar, recon, p, q, s, c,
                                                           d4, prm->tau, prm->mu, prm->v[0],
                                                           prm->v[1], prm->v[2], ch, carry);
    else if (prm->f_dtype == DTV_F16)
      pdhg_primal_x4_kernel<__half><<<g4, kBlock3, 0, st>>>(f, (__half*)fbar, recon, p, q, s, c,
                                                            d4, prm->tau, prm->mu, prm->v[0],
                                                            prm->v[1], prm->v[2], ch, carry);
    else
      pdhg_primal_x4_kernel<__nv_bfloat16><<<g4, kBlock3, 0, st>>>(
          f, (__nv_bfloat16*)fbar, recon, p, q, s, c, d4, prm->tau, prm->mu, prm->v[0],
          prm->v[1], prm->v[2], ch, carry);
    note_launch();
  } else if (prm->f_dtype == DTV_F32) {
    pdhg_primal_kernel<float><<<grid3(d, batch), kBlock3, 0, as_stream(stream)>>>(
        f, (float*)fbar, recon, p, q, s, c, d, prm->tau, prm->mu, prm->v[0], prm->v[1],
        prm->v[2], ch, carry); note_launch();
  } else if (prm->f_dtype == DTV_F16) {
    pdhg_primal_kernel<__half><<<grid3(d, batch), kBlock3, 0, as_stream(stream)>>>(
        f, (__half*)fbar, recon, p, q, s, c, d, prm->tau, prm->mu, prm->v[0], prm->v[1],
        prm->v[2], ch, carry); note_launch();
  } else {
    pdhg_primal_kernel<__nv_bfloat16><<<grid3(d, batch), kBlock3, 0, as_stream(stream)>>>(
        f, (__nv_bfloat16*)fbar, recon, p, q, s, c, d, prm->tau, prm->mu, prm->v[0], prm->v[1],
        prm->v[2], ch, carry); note_launch();
  }
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

int dtv_pdhg_dual(const void* fbar, float* p, float* q, float* s, float* c, const int32_t size[3],
                  int32_t batch, const dtv_pdhg_params* prm, const double* t, void* ws,
                  void* stream) {
  return pdhg_dual_impl(fbar, p, q, s, c, size, batch, prm, t, ws, nullptr, stream);
}

int dtv_pdhg_dual_defer(const void* fbar, float* p, float* q, float* s, float* c,
                        const int32_t size[3], int32_t batch, const dtv_pdhg_params* prm,
                        const double* t, void* ws, const float* carry, void* stream) {
  return pdhg_dual_impl(fbar, p, q, s, c, size, batch, prm, t, ws, carry, stream);
}

int dtv_pdhg_primal(float* f, void* fbar, const float* recon, float* p, float* q, float* s,
                    const float* c, const int32_t size[3], int32_t batch,
                    const dtv_pdhg_params* prm, const void* ws, void* stream) {
  return pdhg_primal_impl(f, fbar, recon, p, q, s, c, size, batch, prm, ws, nullptr, stream);
}

int dtv_pdhg_primal_defer(float* f, void* fbar, const float* recon, float* p, float* q,
                          float* s, const float* c, const int32_t size[3], int32_t batch,
                          const dtv_pdhg_params* prm, const void* ws, float* carry,
                          void* stream) {
  DTV_CHECK(carry, "NULL argument");
  return pdhg_primal_impl(f, fbar, recon, p, q, s, c, size, batch, prm, ws, carry, stream);
}

int dtv_fista_update(float* y, float* x_prev, const float* bp, int64_t n, float L, float thresh,
                     float momentum, void* stream) {
  DTV_CHECK(y && x_prev && bp && n > 0, "bad argument");
  fista_kernel<<<blocks_for(n), 256, 0, as_stream(stream)>>>(y, x_prev, bp, n, L, thresh, momentum); note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

int dtv_fista_update_many(float* const* y, float* const* x_prev, const float* const* bp,
                          const int64_t* n, int32_t count, float L, float thresh, float momentum,
                          void* stream) {
  DTV_CHECK(y && x_prev && bp && n && count >= 1, "bad argument");
  FistaMany m;
  for (int c0 = 0; c0 < count; c0 += kFistaMany) {
    const int cnt = std::min(kFistaMany, count - c0);
    m.count = cnt;
    m.start[0] = 0;
    for (int k = 0; k < cnt; ++k) {
      DTV_CHECK(y[c0 + k] && x_prev[c0 + k] && bp[c0 + k] && n[c0 + k] > 0, "bad volume %d",
                c0 + k);
      m.y[k] = y[c0 + k];
      m.xp[k] = x_prev[c0 + k];
      m.bp[k] = bp[c0 + k];
      m.start[k + 1] = m.start[k] + n[c0 + k];
    }
    fista_many_kernel<<<blocks_for(m.start[cnt]), 256, 0, as_stream(stream)>>>(m, L, thresh,
                                                                                momentum); note_launch();
    DTV_LAUNCH_CHECK();
  }
  return DTV_OK;
}

int dtv_relu_step(const float* f, const float* bp, float* z, int64_t n, float sigma, void* stream) {
  DTV_CHECK(f && bp && z && n > 0, "bad argument");
  relu_step_kernel<<<blocks_for(n), 256, 0, as_stream(stream)>>>(f, bp, z, n, sigma); note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

int dtv_dtvfista_maxes(const float* z, const int32_t size[3], int32_t batch, const float v[3],
                       float* maxes, void* stream) {
  DTV_CHECK(z && size && v && maxes, "NULL argument");
  int rc = check_dims(size, batch);
  if (rc) return rc;
  Dims d = make_dims(size, 1, batch);
  cudaStream_t st = as_stream(stream);
  // the three max bit patterns live in maxes[0..2] during the reduction
  unsigned int* bits = reinterpret_cast<unsigned int*>(maxes);
  DTV_CUDA_TRY(cudaMemsetAsync(bits, 0, 3 * sizeof(unsigned int), st));
  dtvfista_maxes_kernel<<<grid3(d, batch), kBlock3, 0, st>>>(z, d, bits); note_launch();
  finish_maxes_kernel<<<1, 32, 0, st>>>(bits, v[0], v[1], v[2], maxes); note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

int dtv_dtvfista_update(float* f, const float* z, const int32_t size[3], int32_t batch,
                        const float v[3], const float t[3], float momentum, int32_t quirk,
                        const float* maxes, void* stream) {
  DTV_CHECK(f && z && size && v && t, "NULL argument");
  DTV_CHECK(!quirk || maxes, "quirk mode needs maxes");
  int rc = check_dims(size, batch);
  if (rc) return rc;
  Dims d = make_dims(size, quirk, batch);
  dtvfista_update_kernel<<<grid3(d, batch), kBlock3, 0, as_stream(stream)>>>(
      f, z, d, v[0], v[1], v[2], t[0], t[1], t[2], momentum, quirk, maxes); note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

int dtv_axpy_l1(float* f, const float* bp, float beta, double* l1, int64_t n, void* stream) {
  DTV_CHECK(f && bp && n > 0, "bad argument");
  axpy_l1_kernel<<<blocks_for(n), 256, 0, as_stream(stream)>>>(f, bp, beta, l1, n); note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

int dtv_tv_descent(const float* f_in, float* f_out, const int32_t size[3], int32_t batch,
                   int32_t quirk, const float* davg, void* stream) {
  DTV_CHECK(f_in && f_out && size && davg, "NULL argument");
  DTV_CHECK(f_in != f_out, "f_in and f_out must differ");
  int rc = check_dims(size, batch);
  if (rc) return rc;
  Dims d = make_dims(size, quirk, batch);
  tv_descent_kernel<<<grid3(d, batch), kBlock3, 0, as_stream(stream)>>>(f_in, f_out, d, davg); note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

int dtv_lincomb(const float* x, float a, const float* y, float b, float* out, int64_t n,
                void* stream) {
  DTV_CHECK(x && y && out && n > 0, "bad argument");
  lincomb_kernel<<<blocks_for(n), 256, 0, as_stream(stream)>>>(x, a, y, b, out, n); note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

int dtv_pdhg_sino_dual(float* w, const float* fp, const float* g, float sigma, int64_t n,
                       double* abs_sum, void* stream) {
  DTV_CHECK(w && fp && g && n > 0, "bad argument");
  sino_dual_kernel<<<blocks_for(n), 256, 0, as_stream(stream)>>>(w, fp, g, sigma, n, abs_sum); note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

int dtv_l1_distance(const float* a, const float* b, int64_t n, double* sum, void* stream) {
  DTV_CHECK(a && b && sum && n > 0, "bad argument");
  l1_distance_kernel<<<blocks_for(n), 256, 0, as_stream(stream)>>>(a, b, sum, n); note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

int dtv_asd_adapt(const double* dp_sum, const double* dg_sum, float rmax, float alpha,
                  float* davg, void* stream) {
  DTV_CHECK(dp_sum && dg_sum && davg, "NULL argument");
  asd_adapt_kernel<<<1, 32, 0, as_stream(stream)>>>(dp_sum, dg_sum, rmax, alpha, davg); note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

int dtv_scale_scalar(const double* in, double scale, float* out, void* stream) {
  DTV_CHECK(in && out, "NULL argument");
  scale_scalar_kernel<<<1, 32, 0, as_stream(stream)>>>(in, scale, out); note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

}  // extern "C"

// ---- L1-ball projection without a caller-supplied workspace ---------------------------
//
// dtv_l1ball needs a ~48 KB device workspace for its threshold search, which
// its caller allocates. Some callers cannot allocate device memory at the
// point where they project: a host that reserves the whole GPU at start-up
// and hands out no allocator, a C or Fortran caller on the far side of the
// ABI with no device allocator of its own, or a latency-bound pipeline that
// must not call cudaMalloc/cudaFree in its loop (cudaFree synchronises the
// device). dtv_l1ball_noalloc serves them with the same kernels, whose
// workspace is the array below instead. Each GPU that loads this library
// holds one copy until the process exits.
namespace dtv {

static __device__ __align__(256) unsigned char g_l1ball_scratch[sizeof(L1Chan)];

constexpr int64_t kL1NoallocMaxN = 2147483647LL;  // per-bin counts are 32-bit
constexpr int kMaxDevices = 64;
static std::mutex g_l1ball_scratch_mu;
static void* g_l1ball_scratch_ptr[kMaxDevices] = {};

// Device address of g_l1ball_scratch on the current device. Host code cannot
// pass the array's name to a kernel (that is a host-side stand-in), so the
// address is looked up once per device, with that device current.
static int l1ball_scratch(L1Chan** out) {
  int dev = -1;
  DTV_CUDA_TRY(cudaGetDevice(&dev));
  DTV_CHECK(dev >= 0 && dev < kMaxDevices, "device %d outside [0, %d)", dev, kMaxDevices);
  std::lock_guard<std::mutex> lock(g_l1ball_scratch_mu);
  if (g_l1ball_scratch_ptr[dev] == nullptr) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_l1ball_scratch);
    if (e != cudaSuccess || p == nullptr)
      return fail(DTV_ERR_CUDA, "cudaGetSymbolAddress(l1ball scratch) on device %d: %s", dev,
                  cudaGetErrorString(e));
    g_l1ball_scratch_ptr[dev] = p;
  }
  *out = reinterpret_cast<L1Chan*>(g_l1ball_scratch_ptr[dev]);
  return DTV_OK;
}

}  // namespace dtv

extern "C" int dtv_l1ball_noalloc(const float* v, float* w, int64_t n, const double* radius,
                                  double* lambda_out, void* stream) {
  using namespace dtv;
  DTV_CHECK(v && w && radius, "NULL argument");
  DTV_CHECK(n > 0, "n must be positive");
  DTV_CHECK(n <= kL1NoallocMaxN,
            "n = %lld exceeds the maximum %lld elements of dtv_l1ball_noalloc",
            (long long)n, (long long)kL1NoallocMaxN);
  L1Chan* ch = nullptr;
  int rc = l1ball_scratch(&ch);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  // The array keeps whatever the previous call left; the histograms must
  // start at zero, so clear the whole workspace first.
  DTV_CUDA_TRY(cudaMemsetAsync(ch, 0, sizeof(L1Chan), st));
  l1_reset_kernel<<<1, kL1ResetThreads, 0, st>>>(ch, 1, radius, nullptr, 0.f, 0.f, 0.f); note_launch();
  l1_hist1_kernel<<<hist_blocks(n, 256, 4, 1), 256, 0, st>>>(v, n, ch); note_launch();
  l1_select_kernel<<<1, 1024, 0, st>>>(ch, 1); note_launch();
  l1_hist_kernel<1><<<hist_blocks(n, 256, 4, 1), 256, 0, st>>>(v, nullptr, nullptr, n, ch, 2); note_launch();
  l1_select_kernel<<<1, 1024, 0, st>>>(ch, 2); note_launch();
  l1_hist_kernel<1><<<hist_blocks(n, 256, 4, 1), 256, 0, st>>>(v, nullptr, nullptr, n, ch, 3); note_launch();
  l1_select_kernel<<<1, 1024, 0, st>>>(ch, 3); note_launch();
  l1_apply_kernel<<<blocks_for(n), 256, 0, st>>>(v, w, n, ch, lambda_out); note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}
