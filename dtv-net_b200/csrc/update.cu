// Directional finite differences, the L1-ball threshold search and the fused
// DTV / FISTA / ASD-POCS update kernels.
//
// Finite differences restate model/PDHG/Utils/Gradients.py:8-34, where each
// operator is a sparse matrix D = shift - I: row i is -e_i plus e_{i+o} when
// row i is "valid" (x: (i+1) % X != 0; y: i < N - size[1], with offset
// size[1]; z: i < N - X*Y). The stencils below apply those matrices and their
// transposes without building them.
//
// The L1-ball projection (model/PDHG/Utils/L1ball.py:4-17) needs the threshold
// lambda solving sum_i max(a_i - lambda, 0) = r. The reference Newton-iterates
// lambda with a host sync per step. Here it is found exactly by a three-level
// radix search over the IEEE-754 bit patterns of a_i >= 0 (monotone in a_i):
// 2048 / 1024 / 1024 bins on key bits [30:20] / [19:10] / [9:0]. Every bin of
// a level shares one exponent, so its sum is kept exactly as an integer sum of
// 24-bit significands. After the last level the bin is a single value and
// lambda follows in closed form from the counts and sums above it.
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

struct Dims {
  int X, Y, Z;
  int64_t N;  // X*Y*Z
  int quirk;
};

static Dims make_dims(const int32_t s[3], int quirk) {
  Dims d;
  d.X = s[0]; d.Y = s[1]; d.Z = s[2];
  d.N = (int64_t)s[0] * s[1] * s[2];
  d.quirk = quirk;
  return d;
}

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

__device__ __forceinline__ void decompose(const Dims& d, int64_t i, int& x, int& y, int& z) {
  x = (int)(i % d.X);
  const int64_t r = i / d.X;
  y = (int)(r % d.Y);
  z = (int)(r / d.Y);
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
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
#pragma unroll
  for (int c = 0; c < C; ++c) {
    v[c] = warp_sum(v[c]);
    if (l == 0) red[c][w] = v[c];
  }
  __syncthreads();
  if (threadIdx.x < 32) {
#pragma unroll
    for (int c = 0; c < C; ++c) {
      double s = l < nw ? red[c][l] : 0.0;
      s = warp_sum(s);
      if (l == 0 && s != 0.0) atomicAdd(dst + c, s);
    }
  }
}

// ---- finite differences ---------------------------------------------------------------------
__global__ void diff_kernel(const float* __restrict__ f, float* __restrict__ out, Dims d,
                            int64_t total, int a, int transpose) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = t / d.N, i = t - b * d.N;
    int x, y, z;
    decompose(d, i, x, y, z);
    const float* fb = f + b * d.N;
    float r;
    if (!transpose) {
      r = dfwd(fb, d, a, i, x, y, z);
    } else {
      r = -__ldg(fb + i);
      if (col_valid(d, a, i, x, y, z)) r += __ldg(fb + i - axis_off(d, a));
    }
    out[t] = r;
  }
}

template <class T>
__global__ void diff_abs_sums_kernel(const T* __restrict__ f, Dims d, int64_t total,
                                     double* __restrict__ sums) {
  double acc[3] = {0.0, 0.0, 0.0};
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = t / d.N, i = t - b * d.N;
    int x, y, z;
    decompose(d, i, x, y, z);
    const T* fb = f + b * d.N;
#pragma unroll
    for (int a = 0; a < 3; ++a) acc[a] += fabsf(dfwd(fb, d, a, i, x, y, z));
  }
  block_sums_atomic<3>(acc, sums);
}

// ---- L1-ball radix search ------------------------------------------------------------------
constexpr int kL1Bins1 = 2048, kL1Bins2 = 1024, kL1Bins3 = 1024;

struct L1Chan {
  double radius;
  double c_above;
  double t_above;
  double lambda;
  unsigned int prefix;  // key bits above the current level's bins
  unsigned int maxkey;
  int done;
  float thresh;
  unsigned int cnt1[kL1Bins1];
  unsigned int cnt2[kL1Bins2];
  unsigned int cnt3[kL1Bins3];
  unsigned long long sum1[kL1Bins1];
  unsigned long long sum2[kL1Bins2];
  unsigned long long sum3[kL1Bins3];
};
static_assert(sizeof(L1Chan) % 16 == 0, "L1Chan alignment");

__device__ __forceinline__ unsigned int sig24(unsigned int key) {
  const unsigned int m = key & 0x7FFFFFu;
  return (key & 0x7F800000u) ? (m | 0x800000u) : m;
}

// Adds `key` to a shared histogram with warp aggregation (all lanes call;
// lanes with active == false contribute nothing).
__device__ __forceinline__ void hist_add(unsigned int* cnt, unsigned long long* sum, int bin,
                                         unsigned int key, bool active) {
  const unsigned int act = __ballot_sync(0xffffffffu, active);
  if (!active) return;
  const unsigned int grp = __match_any_sync(act, bin);
  const unsigned int s = __reduce_add_sync(grp, sig24(key));
  if ((threadIdx.x & 31) == (unsigned)(__ffs(grp) - 1)) {
    atomicAdd(cnt + bin, (unsigned int)__popc(grp));
    atomicAdd(sum + bin, (unsigned long long)s);
  }
}

template <int NB>
__device__ __forceinline__ void hist_flush(const unsigned int* scnt, const unsigned long long* ssum,
                                           unsigned int* gcnt, unsigned long long* gsum) {
  for (int i = threadIdx.x; i < NB; i += blockDim.x) {
    if (scnt[i]) {
      atomicAdd(gcnt + i, scnt[i]);
      atomicAdd(gsum + i, ssum[i]);
    }
  }
}

// Level-2 / level-3 histogram pass over C channels (keys of |x|).
template <int C>
__global__ void l1_hist_kernel(const float* __restrict__ x0, const float* __restrict__ x1,
                               const float* __restrict__ x2, int64_t n, L1Chan* chans, int level) {
  __shared__ unsigned int scnt[C][1024];
  __shared__ unsigned long long ssum[C][1024];
  bool any = false;
#pragma unroll
  for (int c = 0; c < C; ++c) any |= !chans[c].done;
  if (!any) return;
  for (int i = threadIdx.x; i < 1024; i += blockDim.x)
#pragma unroll
    for (int c = 0; c < C; ++c) {
      scnt[c][i] = 0;
      ssum[c][i] = 0;
    }
  unsigned int pre[C];
  bool live[C];
#pragma unroll
  for (int c = 0; c < C; ++c) {
    pre[c] = chans[c].prefix;
    live[c] = !chans[c].done;
  }
  __syncthreads();
  const int pshift = level == 2 ? 20 : 10;
  const float* xs[3] = {x0, x1, x2};
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t nround = (n + stride - 1) / stride * stride;  // all lanes iterate together
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nround; t += stride) {
#pragma unroll
    for (int c = 0; c < C; ++c) {
      unsigned int key = 0;
      bool act = false;
      if (t < n && live[c]) {
        key = __float_as_uint(__ldg(xs[c] + t)) & 0x7FFFFFFFu;
        act = (key >> pshift) == pre[c];
      }
      const int bin = level == 2 ? (int)((key >> 10) & 1023u) : (int)(key & 1023u);
      hist_add(scnt[c], ssum[c], bin, key, act);
    }
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < C; ++c) {
    if (!live[c]) continue;
    if (level == 2) hist_flush<1024>(scnt[c], ssum[c], chans[c].cnt2, chans[c].sum2);
    else hist_flush<1024>(scnt[c], ssum[c], chans[c].cnt3, chans[c].sum3);
  }
}

// Level-1 histogram of a plain array (standalone L1-ball).
__global__ void l1_hist1_kernel(const float* __restrict__ v, int64_t n, L1Chan* ch) {
  __shared__ unsigned int scnt[kL1Bins1];
  __shared__ unsigned long long ssum[kL1Bins1];
  for (int i = threadIdx.x; i < kL1Bins1; i += blockDim.x) {
    scnt[i] = 0;
    ssum[i] = 0;
  }
  __syncthreads();
  unsigned int kmax = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t nround = (n + stride - 1) / stride * stride;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nround; t += stride) {
    unsigned int key = 0;
    if (t < n) key = __float_as_uint(__ldg(v + t)) & 0x7FFFFFFFu;
    kmax = max(kmax, key);
    hist_add(scnt, ssum, (int)(key >> 20), key, t < n);
  }
  __syncthreads();
  hist_flush<kL1Bins1>(scnt, ssum, ch->cnt1, ch->sum1);
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
  const int nb = level == 1 ? kL1Bins1 : (level == 2 ? kL1Bins2 : kL1Bins3);
  unsigned int* cnt = level == 1 ? ch.cnt1 : (level == 2 ? ch.cnt2 : ch.cnt3);
  unsigned long long* sum = level == 1 ? ch.sum1 : (level == 2 ? ch.sum2 : ch.sum3);
  const int per = nb / 1024;  // 2 or 1 bins per thread, thread t owns bins [t*per, t*per+per)
  const unsigned int kbase = level == 1 ? 0u : (level == 2 ? (ch.prefix << 20) : (ch.prefix << 10));
  const int bshift = level == 1 ? 20 : (level == 2 ? 10 : 0);
  double c_loc = 0.0, t_loc = 0.0;
  double cb[2], tb[2];
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
  double c_above = ch.c_above + c_hi + (c_s - c_loc);
  double t_above = ch.t_above + t_hi + (t_s - t_loc);
  const double radius = ch.radius;
  if (level == 1 && t == 0) {
    // totals for the special cases
    double ctot = 0.0, ttot = 0.0;
    for (int ww = 0; ww < 32; ++ww) {
      ctot += wc[ww];
      ttot += wt[ww];
    }
    (void)ctot;
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
  const int J = best;
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
  __syncthreads();
  for (int q = 0; q < per; ++q) {  // leave the histogram zeroed for the next search
    cnt[t * per + q] = 0;
    sum[t * per + q] = 0;
  }
}

// Resets a channel for a new search (radius from a device double, optionally
// scaled and multiplied by a device constraint level).
__global__ void l1_reset_kernel(L1Chan* chans, int C, const double* radius, const double* t,
                                float s0, float s1, float s2) {
  const int c = threadIdx.x;
  if (c >= C) return;
  L1Chan& ch = chans[c];
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
template <class T>
__global__ void __launch_bounds__(256) pdhg_dual_kernel(const T* __restrict__ fbar, float* __restrict__ p,
                                                        float* __restrict__ q, float* __restrict__ s,
                                                        float* __restrict__ c, Dims d, int64_t total,
                                                        float a0, float a1, float a2, float smu,
                                                        L1Chan* chans) {
  extern __shared__ unsigned char smem[];
  unsigned int* scnt = reinterpret_cast<unsigned int*>(smem);                      // [3][2048]
  unsigned long long* ssum = reinterpret_cast<unsigned long long*>(smem + 3 * kL1Bins1 * 4);
  for (int i = threadIdx.x; i < 3 * kL1Bins1; i += blockDim.x) {
    scnt[i] = 0;
    ssum[i] = 0;
  }
  __syncthreads();
  unsigned int kmax[3] = {0u, 0u, 0u};
  float* outs[3] = {p, q, s};
  const float as[3] = {a0, a1, a2};
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t nround = (total + stride - 1) / stride * stride;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nround; t += stride) {
    const bool in = t < total;
    unsigned int key[3] = {0u, 0u, 0u};
    if (in) {
      const int64_t b = t / d.N, i = t - b * d.N;
      int x, y, z;
      decompose(d, i, x, y, z);
      const T* fb = fbar + b * d.N;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const float g = dfwd(fb, d, a, i, x, y, z);
        const float nv = fmaf(as[a], g, outs[a][t]);  // p + v*sigma*D fbar
        outs[a][t] = nv;
        key[a] = __float_as_uint(nv) & 0x7FFFFFFFu;
        kmax[a] = max(kmax[a], key[a]);
      }
      const float cv = fmaf(smu, load_as_float(fb, i), c[t]);
      c[t] = fminf(cv, 0.f);  // -relu(-c - sigma*mu*fbar)
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
      hist_add(scnt + a * kL1Bins1, ssum + a * kL1Bins1, (int)(key[a] >> 20), key[a], in);
  }
  __syncthreads();
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    hist_flush<kL1Bins1>(scnt + a * kL1Bins1, ssum + a * kL1Bins1, chans[a].cnt1, chans[a].sum1);
    unsigned int km = kmax[a];
    for (int o = 16; o > 0; o >>= 1) km = max(km, __shfl_xor_sync(0xffffffffu, km, o));
    if ((threadIdx.x & 31) == 0 && km) atomicMax(&chans[a].maxkey, km);
  }
}

__device__ __forceinline__ float clipf(float x, float m) { return copysignf(fminf(fabsf(x), m), x); }

// ---- fused PDHG primal step (DTVCP.py:44-54) ----------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256) pdhg_primal_kernel(T* __restrict__ f, T* __restrict__ fbar,
                                                          const float* __restrict__ recon, float* p,
                                                          float* q, float* s,
                                                          const float* __restrict__ c, Dims d,
                                                          int64_t total, float tau, float mu,
                                                          float v0, float v1, float v2,
                                                          const L1Chan* chans) {
  const float m0 = chans[0].thresh, m1 = chans[1].thresh, m2 = chans[2].thresh;
  float* duals[3] = {p, q, s};
  const float ms[3] = {m0, m1, m2};
  const float vs[3] = {v0, v1, v2};
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = t / d.N, i = t - b * d.N;
    int x, y, z;
    decompose(d, i, x, y, z);
    float reg = mu * c[t];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float* g = duals[a] + b * d.N;
      const float self = clipf(g[i], ms[a]);
      float dt = -self;
      if (col_valid(d, a, i, x, y, z)) dt += clipf(g[i - axis_off(d, a)], ms[a]);
      reg = fmaf(vs[a], dt, reg);
      g[i] = self;  // idempotent: neighbours re-clip whatever they read
    }
    const float fo = load_as_float(f, t);
    const float fn = fo - recon[t] - tau * reg;
    store_from_float(fbar, t, 2.f * fn - fo);
    store_from_float(f, t, fn);
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

// ---- FISTA-DTV (DTVFISTA.py:29-38) -------------------------------------------------------------------
__global__ void relu_step_kernel(const float* __restrict__ f, const float* bp, float* z, int64_t n,
                                 float sigma) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x)
    z[t] = fmaxf(f[t] - sigma * bp[t], 0.f);
}

__global__ void dtvfista_maxes_kernel(const float* __restrict__ z, Dims d, int64_t total,
                                      unsigned int* maxbits) {
  unsigned int km[3] = {0u, 0u, 0u};
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = t / d.N, i = t - b * d.N;
    int x, y, zz;
    decompose(d, i, x, y, zz);
#pragma unroll
    for (int a = 0; a < 3; ++a)
      km[a] = max(km[a], __float_as_uint(fabsf(dfwd(z + b * d.N, d, a, i, x, y, zz))));
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    unsigned int k = km[a];
    for (int o = 16; o > 0; o >>= 1) k = max(k, __shfl_xor_sync(0xffffffffu, k, o));
    if ((threadIdx.x & 31) == 0) atomicMax(maxbits + a, k);
  }
}

__global__ void finish_maxes_kernel(const unsigned int* bits, float v0, float v1, float v2,
                                    float* maxes) {
  const int a = threadIdx.x;
  if (a < 3) maxes[a] = __uint_as_float(bits[a]) - (a == 0 ? v0 : (a == 1 ? v1 : v2));
}

__global__ void dtvfista_update_kernel(float* __restrict__ f, const float* __restrict__ z, Dims d,
                                       int64_t total, float v0, float v1, float v2, float t0,
                                       float t1, float t2, float mom, int quirk,
                                       const float* __restrict__ maxes) {
  const float vs[3] = {v0, v1, v2}, ts[3] = {t0, t1, t2};
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = t / d.N, i = t - b * d.N;
    int x, y, zz;
    decompose(d, i, x, y, zz);
    const float* zb = z + b * d.N;
    float fn = zb[i];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float m = quirk ? maxes[a] : 0.f;
      auto thr = [&](float g) {
        if (quirk) return g > 0.f ? m : (g < 0.f ? -m : 0.f);  // sign(g) * max_i(|g_i| - v)
        const float r = fmaxf(fabsf(g) - vs[a], 0.f);
        return g > 0.f ? r : (g < 0.f ? -r : 0.f);
      };
      float dt = -thr(dfwd(zb, d, a, i, x, y, zz));
      if (col_valid(d, a, i, x, y, zz)) {
        const int64_t j = i - axis_off(d, a);
        int xj, yj, zj;
        decompose(d, j, xj, yj, zj);
        dt += thr(dfwd(zb, d, a, j, xj, yj, zj));
      }
      fn = fmaf(ts[a], dt, fn);
    }
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

__device__ __forceinline__ void grad3(const float* f, const Dims& d, int64_t i, float g[3]) {
  int x, y, z;
  decompose(d, i, x, y, z);
#pragma unroll
  for (int a = 0; a < 3; ++a) g[a] = dfwd(f, d, a, i, x, y, z);
}

__global__ void tv_descent_kernel(const float* __restrict__ fin, float* __restrict__ fout, Dims d,
                                  int64_t total, const float* __restrict__ davg) {
  const float step = davg[0];
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = t / d.N, i = t - b * d.N;
    const float* fb = fin + b * d.N;
    int x, y, z;
    decompose(d, i, x, y, z);
    float g[3];
    grad3(fb, d, i, g);
    const float nrm = sqrtf(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]) + 1.f;
    float grad = 0.f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      grad -= g[a] / nrm;
      if (col_valid(d, a, i, x, y, z)) {
        float gj[3];
        grad3(fb, d, i - axis_off(d, a), gj);
        const float nj = sqrtf(gj[0] * gj[0] + gj[1] * gj[1] + gj[2] * gj[2]) + 1.f;
        grad += gj[a] / nj;
      }
    }
    fout[t] = fb[i] - step * grad;
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
  DTV_CHECK(size[0] > 0 && size[1] > 0 && size[2] > 0 && batch > 0, "bad size");
  DTV_CHECK(axis >= 0 && axis <= 2, "axis must be 0, 1 or 2");
  Dims d = make_dims(size, quirk);
  const int64_t total = d.N * batch;
  diff_kernel<<<blocks_for(total), 256, 0, as_stream(stream)>>>(f, out, d, total, axis, transpose); note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

int dtv_diff_abs_sums(const void* f, int32_t dt, const int32_t size[3], int32_t batch,
                      int32_t quirk, double* sums, void* stream) {
  DTV_CHECK(f && sums && size, "NULL argument");
  DTV_CHECK(dt == DTV_F32 || dt == DTV_F16, "dtype must be f32 or f16");
  DTV_CHECK(size[0] > 0 && size[1] > 0 && size[2] > 0 && batch > 0, "bad size");
  Dims d = make_dims(size, quirk);
  const int64_t total = d.N * batch;
  if (dt == DTV_F32) {
    diff_abs_sums_kernel<float><<<blocks_for(total), 256, 0, as_stream(stream)>>>(
        (const float*)f, d, total, sums); note_launch();
  }
  else {
    diff_abs_sums_kernel<__half><<<blocks_for(total), 256, 0, as_stream(stream)>>>(
        (const __half*)f, d, total, sums); note_launch();
  }
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

int64_t dtv_l1ball_workspace_bytes(void) { return (int64_t)sizeof(L1Chan); }

int dtv_l1ball(const float* v, float* w, int64_t n, const double* radius, void* ws,
               double* lambda_out, void* stream) {
  DTV_CHECK(v && w && radius && ws, "NULL argument");
  DTV_CHECK(n > 0, "n must be positive");
  cudaStream_t st = as_stream(stream);
  L1Chan* ch = reinterpret_cast<L1Chan*>(ws);
  l1_reset_kernel<<<1, 32, 0, st>>>(ch, 1, radius, nullptr, 0.f, 0.f, 0.f); note_launch();
  l1_hist1_kernel<<<blocks_for(n, 256, 4), 256, 0, st>>>(v, n, ch); note_launch();
  l1_select_kernel<<<1, 1024, 0, st>>>(ch, 1); note_launch();
  l1_hist_kernel<1><<<blocks_for(n, 256, 4), 256, 0, st>>>(v, nullptr, nullptr, n, ch, 2); note_launch();
  l1_select_kernel<<<1, 1024, 0, st>>>(ch, 2); note_launch();
  l1_hist_kernel<1><<<blocks_for(n, 256, 4), 256, 0, st>>>(v, nullptr, nullptr, n, ch, 3); note_launch();
  l1_select_kernel<<<1, 1024, 0, st>>>(ch, 3); note_launch();
  l1_apply_kernel<<<blocks_for(n), 256, 0, st>>>(v, w, n, ch, lambda_out); note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

int64_t dtv_pdhg_workspace_bytes(void) { return (int64_t)(3 * sizeof(L1Chan)); }

int dtv_pdhg_dual(const void* fbar, float* p, float* q, float* s, float* c, const int32_t size[3],
                  int32_t batch, const dtv_pdhg_params* prm, const double* t, void* ws,
                  void* stream) {
  DTV_CHECK(fbar && p && q && s && c && size && prm && t && ws, "NULL argument");
  DTV_CHECK(prm->f_dtype == DTV_F32 || prm->f_dtype == DTV_F16, "f_dtype must be f32 or f16");
  DTV_CHECK(size[0] > 0 && size[1] > 0 && size[2] > 0 && batch > 0, "bad size");
  Dims d = make_dims(size, prm->quirk);
  const int64_t total = d.N * batch;
  cudaStream_t st = as_stream(stream);
  L1Chan* ch = reinterpret_cast<L1Chan*>(ws);
  const float sg = prm->sigma;
  // radius on |p_| directly: sigma * v_a * t_a (the reference projects |p_|/sigma
  // onto the ball of radius v_a * t_a)
  l1_reset_kernel<<<1, 32, 0, st>>>(ch, 3, nullptr, t, sg * prm->v[0], sg * prm->v[1],
                                    sg * prm->v[2]); note_launch();
  const size_t smem = 3 * kL1Bins1 * (sizeof(unsigned int) + sizeof(unsigned long long));
  const int nb = blocks_for(total, 256, 2);
  if (prm->f_dtype == DTV_F32) {
    static bool attr_f32 = false;
    if (!attr_f32) {
      DTV_CUDA_TRY(cudaFuncSetAttribute(pdhg_dual_kernel<float>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      attr_f32 = true;
    }
    pdhg_dual_kernel<float><<<nb, 256, smem, st>>>((const float*)fbar, p, q, s, c, d, total,
                                                   prm->v[0] * sg, prm->v[1] * sg, prm->v[2] * sg,
                                                   sg * prm->mu, ch); note_launch();
  } else {
    static bool attr_f16 = false;
    if (!attr_f16) {
      DTV_CUDA_TRY(cudaFuncSetAttribute(pdhg_dual_kernel<__half>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      attr_f16 = true;
    }
    pdhg_dual_kernel<__half><<<nb, 256, smem, st>>>((const __half*)fbar, p, q, s, c, d, total,
                                                    prm->v[0] * sg, prm->v[1] * sg, prm->v[2] * sg,
                                                    sg * prm->mu, ch); note_launch();
  }
  DTV_LAUNCH_CHECK();
  l1_select_kernel<<<3, 1024, 0, st>>>(ch, 1); note_launch();
  l1_hist_kernel<3><<<blocks_for(total, 256, 2), 256, 0, st>>>(p, q, s, total, ch, 2); note_launch();
  l1_select_kernel<<<3, 1024, 0, st>>>(ch, 2); note_launch();
  l1_hist_kernel<3><<<blocks_for(total, 256, 2), 256, 0, st>>>(p, q, s, total, ch, 3); note_launch();
  l1_select_kernel<<<3, 1024, 0, st>>>(ch, 3); note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

int dtv_pdhg_primal(void* f, void* fbar, const float* recon, float* p, float* q, float* s,
                    const float* c, const int32_t size[3], int32_t batch,
                    const dtv_pdhg_params* prm, const void* ws, void* stream) {
  DTV_CHECK(f && fbar && recon && p && q && s && c && size && prm && ws, "NULL argument");
  DTV_CHECK(prm->f_dtype == DTV_F32 || prm->f_dtype == DTV_F16, "f_dtype must be f32 or f16");
  DTV_CHECK(size[0] > 0 && size[1] > 0 && size[2] > 0 && batch > 0, "bad size");
  Dims d = make_dims(size, prm->quirk);
  const int64_t total = d.N * batch;
  const L1Chan* ch = reinterpret_cast<const L1Chan*>(ws);
  if (prm->f_dtype == DTV_F32) {
    pdhg_primal_kernel<float><<<blocks_for(total), 256, 0, as_stream(stream)>>>(
        (float*)f, (float*)fbar, recon, p, q, s, c, d, total, prm->tau, prm->mu, prm->v[0],
        prm->v[1], prm->v[2], ch); note_launch();
  }
  else {
    pdhg_primal_kernel<__half><<<blocks_for(total), 256, 0, as_stream(stream)>>>(
        (__half*)f, (__half*)fbar, recon, p, q, s, c, d, total, prm->tau, prm->mu, prm->v[0],
        prm->v[1], prm->v[2], ch); note_launch();
  }
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

int dtv_fista_update(float* y, float* x_prev, const float* bp, int64_t n, float L, float thresh,
                     float momentum, void* stream) {
  DTV_CHECK(y && x_prev && bp && n > 0, "bad argument");
  fista_kernel<<<blocks_for(n), 256, 0, as_stream(stream)>>>(y, x_prev, bp, n, L, thresh, momentum); note_launch();
  DTV_LAUNCH_CHECK();
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
  DTV_CHECK(size[0] > 0 && size[1] > 0 && size[2] > 0 && batch > 0, "bad size");
  Dims d = make_dims(size, 1);
  const int64_t total = d.N * batch;
  cudaStream_t st = as_stream(stream);
  // the three max bit patterns live in maxes[0..2] during the reduction
  unsigned int* bits = reinterpret_cast<unsigned int*>(maxes);
  DTV_CUDA_TRY(cudaMemsetAsync(bits, 0, 3 * sizeof(unsigned int), st));
  dtvfista_maxes_kernel<<<blocks_for(total), 256, 0, st>>>(z, d, total, bits); note_launch();
  finish_maxes_kernel<<<1, 32, 0, st>>>(bits, v[0], v[1], v[2], maxes); note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}

int dtv_dtvfista_update(float* f, const float* z, const int32_t size[3], int32_t batch,
                        const float v[3], const float t[3], float momentum, int32_t quirk,
                        const float* maxes, void* stream) {
  DTV_CHECK(f && z && size && v && t, "NULL argument");
  DTV_CHECK(!quirk || maxes, "quirk mode needs maxes");
  DTV_CHECK(size[0] > 0 && size[1] > 0 && size[2] > 0 && batch > 0, "bad size");
  Dims d = make_dims(size, quirk);
  const int64_t total = d.N * batch;
  dtvfista_update_kernel<<<blocks_for(total), 256, 0, as_stream(stream)>>>(
      f, z, d, total, v[0], v[1], v[2], t[0], t[1], t[2], momentum, quirk, maxes); note_launch();
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
  DTV_CHECK(size[0] > 0 && size[1] > 0 && size[2] > 0 && batch > 0, "bad size");
  Dims d = make_dims(size, quirk);
  const int64_t total = d.N * batch;
  tv_descent_kernel<<<blocks_for(total), 256, 0, as_stream(stream)>>>(f_in, f_out, d, total, davg); note_launch();
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
  l1_reset_kernel<<<1, 32, 0, st>>>(ch, 1, radius, nullptr, 0.f, 0.f, 0.f); note_launch();
  l1_hist1_kernel<<<blocks_for(n, 256, 4), 256, 0, st>>>(v, n, ch); note_launch();
  l1_select_kernel<<<1, 1024, 0, st>>>(ch, 1); note_launch();
  l1_hist_kernel<1><<<blocks_for(n, 256, 4), 256, 0, st>>>(v, nullptr, nullptr, n, ch, 2); note_launch();
  l1_select_kernel<<<1, 1024, 0, st>>>(ch, 2); note_launch();
  l1_hist_kernel<1><<<blocks_for(n, 256, 4), 256, 0, st>>>(v, nullptr, nullptr, n, ch, 3); note_launch();
  l1_select_kernel<<<1, 1024, 0, st>>>(ch, 3); note_launch();
  l1_apply_kernel<<<blocks_for(n), 256, 0, st>>>(v, w, n, ch, lambda_out); note_launch();
  DTV_LAUNCH_CHECK();
  return DTV_OK;
}
