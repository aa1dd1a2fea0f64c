// Host-side geometry: the reference conventions expressed as per-view world
// vectors, and the FP64 derivation of the device tables. No CUDA calls here.
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>

#include "common.cuh"

namespace dtv {

// The reference's value of pi (Standard/plug/kernel/forwardKernel.cu:14).
static const double kRefPi = 3.14159265359;
static const double kPi = 3.14159265358979323846;

static thread_local char g_err[512] = "";
static std::atomic<long long> g_launches{0};

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

static inline void cross(const double* a, const double* b, double* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
static inline double dot(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

int validate_geometry(const dtv_geometry* g) {
  DTV_CHECK(g != nullptr, "geometry is NULL");
  DTV_CHECK(g->nx > 0 && g->ny > 0 && g->nz > 0, "volume size must be positive (%d,%d,%d)",
            g->nx, g->ny, g->nz);
  DTV_CHECK(g->nu > 0 && g->nv > 0, "detector size must be positive (%d,%d)", g->nu, g->nv);
  DTV_CHECK(g->n_views > 0, "n_views must be positive");
  DTV_CHECK(g->views != nullptr, "geometry views pointer is NULL");
  DTV_CHECK(g->voxel[0] > 0 && g->voxel[1] > 0 && g->voxel[2] > 0, "voxel size must be positive");
  DTV_CHECK(g->fp_step > 0, "fp_step must be positive");
  DTV_CHECK(g->fp_phase >= DTV_PHASE_STANDARD && g->fp_phase <= DTV_PHASE_BOX, "bad fp_phase %d",
            g->fp_phase);
  DTV_CHECK(g->bp_weight_power >= 0 && g->bp_weight_power <= 2, "bad bp_weight_power");
  // index arithmetic in the kernels is 32-bit within one volume / sinogram view
  const double vpad = double(g->nx + 2 * kPad) * (g->ny + 2 * kPad) * (g->nz + 2 * kPad);
  DTV_CHECK(vpad < 2147483647.0, "volume too large for 32-bit in-volume indexing");
  DTV_CHECK(double(g->nu) * g->nv < 2147483647.0, "detector too large");
  for (int n = 0; n < g->n_views; ++n) {
    const double* v = g->views + 12 * n;
    for (int c = 0; c < 12; ++c)
      DTV_CHECK(isfinite(v[c]), "view %d has a non-finite entry", n);
    double nr[3];
    cross(v + 6, v + 9, nr);
    DTV_CHECK(dot(nr, nr) > 0, "view %d: U and V are parallel", n);
    double dms[3] = {v[3] - v[0], v[4] - v[1], v[5] - v[2]};
    DTV_CHECK(fabs(dot(dms, nr)) > 0, "view %d: source lies in the detector plane", n);
  }
  return DTV_OK;
}

int build_tables(const dtv_geometry* g, GeomParams* gp, FPView* fpv, BPView* bpv) {
  int rc = validate_geometry(g);
  if (rc) return rc;
  gp->nx = g->nx; gp->ny = g->ny; gp->nz = g->nz;
  gp->nu = g->nu; gp->nv = g->nv; gp->n_views = g->n_views;
  gp->phase = g->fp_phase;
  gp->bp_power = g->bp_weight_power;
  gp->bp_extent = g->bp_extent_check;
  for (int c = 0; c < 3; ++c) {
    gp->voxel[c] = g->voxel[c];
    gp->vol_offset[c] = g->vol_offset[c];
  }
  gp->det_offset[0] = g->det_offset[0];
  gp->det_offset[1] = g->det_offset[1];
  gp->step = g->fp_step;
  gp->scale = g->fp_scale;
  gp->bp_scale = g->bp_scale;

  const int n3[3] = {g->nx, g->ny, g->nz};
  double O[3];  // world centre of voxel (0,0,0)
  for (int c = 0; c < 3; ++c) O[c] = (-n3[c] / 2.0 + g->vol_offset[c]) * g->voxel[c];
  const double cu = -g->nu / 2.0 + g->det_offset[0];
  const double cv = -g->nv / 2.0 + g->det_offset[1];

  for (int n = 0; n < g->n_views; ++n) {
    const double* w = g->views + 12 * n;
    const double *S = w, *D = w + 3, *U = w + 6, *V = w + 9;
    FPView& f = fpv[n];
    memset(&f, 0, sizeof(f));
    for (int c = 0; c < 3; ++c) {
      const double P00 = D[c] + cu * U[c] + cv * V[c];
      f.s[c] = (S[c] - O[c]) / g->voxel[c];
      f.sw[c] = S[c];
      f.d0ms[c] = (P00 - S[c]) / g->voxel[c];
      f.u[c] = U[c] / g->voxel[c];
      f.v[c] = V[c] / g->voxel[c];
    }
    // projective map for the backprojector
    double nr[3], vxn[3], nxu[3];
    cross(U, V, nr);
    cross(V, nr, vxn);
    cross(nr, U, nxu);
    const double dms[3] = {D[0] - S[0], D[1] - S[1], D[2] - S[2]};
    const double sdd = dot(dms, nr);
    double Ut[3], Vt[3];
    const double du = dot(U, vxn), dv = dot(V, nxu);
    for (int c = 0; c < 3; ++c) {
      Ut[c] = vxn[c] / du;
      Vt[c] = nxu[c] / dv;
    }
    const double smd[3] = {S[0] - D[0], S[1] - D[1], S[2] - D[2]};
    const double au = dot(Ut, smd) / sdd, av = dot(Vt, smd) / sdd;
    double Wu[3], Wv[3], Wh[3];
    for (int c = 0; c < 3; ++c) {
      Wh[c] = nr[c] / sdd;
      Wu[c] = au * nr[c] + Ut[c] - cu * Wh[c];
      Wv[c] = av * nr[c] + Vt[c] - cv * Wh[c];
    }
    const double oms[3] = {O[0] - S[0], O[1] - S[1], O[2] - S[2]};
    const double* rows[3] = {Wu, Wv, Wh};
    BPView& b = bpv[n];
    memset(&b, 0, sizeof(b));
    for (int r = 0; r < 3; ++r) {
      for (int c = 0; c < 3; ++c) b.m[4 * r + c] = (float)(rows[r][c] * g->voxel[c]);
      b.m[4 * r + 3] = (float)dot(rows[r], oms);
    }
  }
  return DTV_OK;
}

// Exact ray/box chord count (host, FP64): sum over rays of ceil(chord/step).
double count_fp_samples(const GeomParams& gp, const FPView* fpv) {
  const int n3[3] = {gp.nx, gp.ny, gp.nz};
  double total = 0.0;
  for (int n = 0; n < gp.n_views; ++n) {
    const FPView& f = fpv[n];
    for (int v = 0; v < gp.nv; ++v)
      for (int u = 0; u < gp.nu; ++u) {
        double r[3], rw[3];
        for (int c = 0; c < 3; ++c) {
          r[c] = f.d0ms[c] + u * f.u[c] + v * f.v[c];
          rw[c] = r[c] * gp.voxel[c];
        }
        const double len = sqrt(dot(rw, rw));
        double lo = -INFINITY, hi = INFINITY;
        bool miss = false;
        for (int c = 0; c < 3 && !miss; ++c) {
          const double d = r[c] / len;
          if (d == 0.0) {
            if (f.s[c] < -0.5 || f.s[c] > n3[c] - 0.5) miss = true;
            continue;
          }
          double t0 = (-0.5 - f.s[c]) / d, t1 = (n3[c] - 0.5 - f.s[c]) / d;
          if (t0 > t1) std::swap(t0, t1);
          lo = std::max(lo, t0);
          hi = std::min(hi, t1);
        }
        if (!miss && hi > lo) total += ceil((hi - lo) / gp.step);
      }
  }
  return total;
}

}  // namespace dtv

using namespace dtv;

extern "C" {

int dtv_version(void) { return 10000; }

int64_t dtv_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

const char* dtv_error_string(int code) {
  switch (code) {
    case DTV_OK: return "ok";
    case DTV_ERR_INVALID: return "invalid argument";
    case DTV_ERR_CUDA: return "CUDA error";
    case DTV_ERR_ALLOC: return "device allocation failed";
    case DTV_ERR_UNSUPPORTED: return "unsupported";
    default: return "unknown error";
  }
}

const char* dtv_last_error_message(void) { return g_err; }

int dtv_geometry_standard(dtv_geometry* g, double* views, const float* angles_deg, int32_t n,
                          const int32_t vs[3], const int32_t ds[2], float sid, float sdd) {
  DTV_CHECK(g && views && angles_deg && vs && ds, "NULL argument");
  DTV_CHECK(n > 0, "need at least one angle");
  DTV_CHECK(sid > 0 && sdd > sid, "need 0 < sid < sdd (got %g, %g)", (double)sid, (double)sdd);
  memset(g, 0, sizeof(*g));
  g->nx = vs[0]; g->ny = vs[1]; g->nz = vs[2];
  g->nu = ds[0]; g->nv = ds[1];
  g->n_views = n;
  const double s = (double)(sid / sdd);  // float quotient, forwardKernel.cu:63
  for (int c = 0; c < 3; ++c) {
    g->voxel[c] = s;
    g->vol_offset[c] = 0.0;
  }
  g->det_offset[0] = g->det_offset[1] = 0.0;
  g->fp_step = s;
  g->fp_scale = s;
  g->fp_phase = DTV_PHASE_STANDARD;
  g->bp_weight_power = 2;
  g->bp_scale = kRefPi / n;
  g->bp_extent_check = 0;
  for (int a = 0; a < n; ++a) {
    // forwardKernel.cu:30-40 / backwardKernel.cu:32-36
    const double beta = (double)angles_deg[a] / 180.0 * kRefPi - kRefPi / 2.0;
    const double ex = cos(beta), ey = sin(beta);
    double* o = views + 12 * a;
    o[0] = -ex * sid; o[1] = -ey * sid; o[2] = 0.0;
    o[3] = ex * ((double)sdd - sid); o[4] = ey * ((double)sdd - sid); o[5] = 0.0;
    o[6] = -ey; o[7] = ex; o[8] = 0.0;
    o[9] = 0.0; o[10] = 0.0; o[11] = 1.0;
  }
  g->views = views;
  return validate_geometry(g);
}

int dtv_geometry_vector(dtv_geometry* g, double* views, const float* pv, int32_t n,
                        const int32_t vs[3], const int32_t ds[2]) {
  DTV_CHECK(g && views && pv && vs && ds, "NULL argument");
  DTV_CHECK(n > 0, "need at least one view");
  memset(g, 0, sizeof(*g));
  g->nx = vs[0]; g->ny = vs[1]; g->nz = vs[2];
  g->nu = ds[0]; g->nv = ds[1];
  g->n_views = n;
  for (int c = 0; c < 3; ++c) {
    g->voxel[c] = 1.0;
    g->vol_offset[c] = 0.0;
  }
  g->det_offset[0] = g->det_offset[1] = 0.5;  // forwardKernel.cu:33 (0.5 + detX)
  g->fp_step = 1.0;                           // forwardKernel.cu:72
  g->fp_scale = 1.0;
  g->fp_phase = DTV_PHASE_VECTOR;
  g->bp_weight_power = 1;                              // backwardKernel.cu:37
  // backwardKernel.cu:43,96: 2*pi / (N / 21) in integer division. With fewer than
  // 21 views the reference divides by zero; the scale is 0 here instead.
  g->bp_scale = n >= 21 ? 2.0 * kRefPi / (n / 21) : 0.0;
  g->bp_extent_check = 1;                              // backwardKernel.cu:38
  for (int a = 0; a < n; ++a) {
    const float* p = pv + 12 * a;
    double* o = views + 12 * a;
    o[0] = p[0]; o[1] = p[1]; o[2] = -(double)p[2];  // source, :27
    o[3] = p[3]; o[4] = p[4]; o[5] = -(double)p[5];  // detector, :28
    o[6] = p[9]; o[7] = p[10]; o[8] = p[11];         // U = u, :30
    o[9] = p[6]; o[10] = p[7]; o[11] = p[8];         // V = v, :29
  }
  g->views = views;
  return validate_geometry(g);
}

int dtv_geometry_circular(dtv_geometry* g, double* views, const double* angles_deg, int32_t n,
                          const int32_t vs[3], const double voxel[3], const int32_t ds[2],
                          const double pitch[2], double sod, double sdd) {
  DTV_CHECK(g && views && angles_deg && vs && voxel && ds && pitch, "NULL argument");
  DTV_CHECK(n > 0, "need at least one angle");
  DTV_CHECK(sod > 0 && sdd > sod, "need 0 < sod < sdd");
  DTV_CHECK(pitch[0] > 0 && pitch[1] > 0, "pitch must be positive");
  memset(g, 0, sizeof(*g));
  g->nx = vs[0]; g->ny = vs[1]; g->nz = vs[2];
  g->nu = ds[0]; g->nv = ds[1];
  g->n_views = n;
  double step = voxel[0];
  for (int c = 0; c < 3; ++c) {
    g->voxel[c] = voxel[c];
    g->vol_offset[c] = 0.5;
    step = std::min(step, voxel[c]);
  }
  g->det_offset[0] = g->det_offset[1] = 0.5;
  g->fp_step = step;
  g->fp_scale = step;
  g->fp_phase = DTV_PHASE_BOX;
  g->bp_weight_power = 2;
  g->bp_scale = kPi / n;
  g->bp_extent_check = 0;
  for (int a = 0; a < n; ++a) {
    const double beta = angles_deg[a] / 180.0 * kPi - kPi / 2.0;
    const double ex = cos(beta), ey = sin(beta);
    double* o = views + 12 * a;
    o[0] = -ex * sod; o[1] = -ey * sod; o[2] = 0.0;
    o[3] = ex * (sdd - sod); o[4] = ey * (sdd - sod); o[5] = 0.0;
    o[6] = -ey * pitch[0]; o[7] = ex * pitch[0]; o[8] = 0.0;
    o[9] = 0.0; o[10] = 0.0; o[11] = pitch[1];
  }
  g->views = views;
  return validate_geometry(g);
}

}  // extern "C"
