/*
 * oracle.c — FP64 CPU restatement of the reference cone-beam projectors.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the correctness oracle and the timed
 * CPU baseline. The product (dtv-net_b200/) never links, loads or calls it;
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
 * arm use it, always as the checker.
 *
 * Two layers:
 *   1. literal restatements of the reference kernels, line by line, in double
 *      precision (oracle_*_literal), citing the file:line each step follows;
 *   2. the same operators over a per-view vector description (source, detector
 *      centre, one-pixel steps U and V) that also expresses the general
 *      geometry; tests pin layer 2 to layer 1 on the reference conventions.
 * Texture sampling is restated as trilinear/bilinear interpolation with border
 * value 0 in unnormalised texel coordinates (the reference's texture setup,
 * Standard/plug/kernel/forwardKernel.cu:102-107). With tex_quant != 0 the
 * interpolation weights are rounded to 1/256, the 8-bit fraction the CUDA
 * programming guide documents for hardware linear filtering; tex_quant == 2
 * rounds only the x/y weights (bilinear hardware filtering of z-plane pairs).
 *
 * Parity pin: the literal layer is compared against the reference kernels
 * themselves (built from their unmodified sources, run on a GPU) through the
 * fixtures in tests/golden/.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* The reference's own value of pi (Standard/plug/kernel/forwardKernel.cu:14). */
#define REF_PI 3.14159265359
/* Exact pi for the general geometry (no reference counterpart). */
#define EXACT_PI 3.14159265358979323846

typedef struct og_geometry {
  int32_t nx, ny, nz, nu, nv, n_views;
  int32_t phase;     /* 0 standard, 1 vector, 2 box */
  int32_t bp_pow;    /* FDK weight exponent */
  int32_t bp_extent; /* vector-layer extent quirk */
  int32_t pad;
  double voxel[3];
  double vol_off[3];
  double det_off[2];
  double step, scale, bp_scale;
} og_geometry;

/* ------------------------------------------------------------------------ */
/* sampling                                                                  */
/* ------------------------------------------------------------------------ */
static inline double qw(double a, int q) { return q ? nearbyint(a * 256.0) / 256.0 : a; }

/* Trilinear sample at voxel-index coordinate (x,y,z) (voxel i centred at i),
 * value 0 outside: tex3D(t, x+0.5, y+0.5, z+0.5) with cudaAddressModeBorder
 * and cudaFilterModeLinear (forwardKernel.cu:77,102-107). */
static double tri(const double* v, int nx, int ny, int nz, double x, double y, double z, int q) {
  double fx = floor(x), fy = floor(y), fz = floor(z);
  if (fx < -1.0 || fy < -1.0 || fz < -1.0 || fx > nx || fy > ny || fz > nz) return 0.0;
  int ix = (int)fx, iy = (int)fy, iz = (int)fz;
  /* q == 2: x/y weights at 1/256, z weight exact (the z-pair sampler) */
  double ax = qw(x - fx, q), ay = qw(y - fy, q), az = qw(z - fz, q == 1);
  double acc = 0.0;
  for (int dz = 0; dz < 2; ++dz) {
    int zz = iz + dz;
    if (zz < 0 || zz >= nz) continue;
    double wz = dz ? az : 1.0 - az;
    for (int dy = 0; dy < 2; ++dy) {
      int yy = iy + dy;
      if (yy < 0 || yy >= ny) continue;
      double wy = dy ? ay : 1.0 - ay;
      for (int dx = 0; dx < 2; ++dx) {
        int xx = ix + dx;
        if (xx < 0 || xx >= nx) continue;
        double wx = dx ? ax : 1.0 - ax;
        acc += wz * wy * wx * v[((int64_t)zz * ny + yy) * nx + xx];
      }
    }
  }
  return acc;
}

/* Bilinear sample of one detector view at pixel-index coordinate (u,v),
 * value 0 outside (tex3D(sino, u+0.5, v+0.5, view+0.5), backwardKernel.cu:49). */
static double bil(const double* s, int nu, int nv, double u, double v, int q) {
  double fu = floor(u), fv = floor(v);
  if (fu < -1.0 || fv < -1.0 || fu > nu || fv > nv) return 0.0;
  int iu = (int)fu, iv = (int)fv;
  double au = qw(u - fu, q), av = qw(v - fv, q);
  double acc = 0.0;
  for (int dv = 0; dv < 2; ++dv) {
    int vv = iv + dv;
    if (vv < 0 || vv >= nv) continue;
    double wv = dv ? av : 1.0 - av;
    for (int du = 0; du < 2; ++du) {
      int uu = iu + du;
      if (uu < 0 || uu >= nu) continue;
      double wu = du ? au : 1.0 - au;
      acc += wv * wu * s[(int64_t)vv * nu + uu];
    }
  }
  return acc;
}

/* ------------------------------------------------------------------------ */
/* layer 1: literal restatements                                             */
/* ------------------------------------------------------------------------ */

/* Standard forward projector, model/ConeBeamLayers/Standard/plug/kernel/
 * forwardKernel.cu:22-86 (kernel) and :110-136 (host sizes and loops). */
void oracle_forward_standard_literal(const double* vol, int batch, const double* angles_deg,
                                     int n_angles, int X, int Y, int Z, int W, int H, double sid,
                                     double sdd, int q, double* sino) {
  const double vcx = X / -2.0, vcy = Y / -2.0, vcz = Z / -2.0; /* :111 */
  const double dcx = W / -2.0, dcy = H / -2.0;                 /* :113 */
#pragma omp parallel for collapse(2) schedule(dynamic)
  for (int b = 0; b < batch; ++b)
    for (int a = 0; a < n_angles; ++a) {
      const double* V = vol + (int64_t)b * X * Y * Z;
      double angle = angles_deg[a] / 180.0 * REF_PI - REF_PI / 2.0; /* :30 */
      double exx = cos(angle), exy = sin(angle);                    /* :31 */
      double eyx = -exy, eyy = exx;                                 /* :32 */
      for (int j = 0; j < H; ++j)
        for (int i = 0; i < W; ++i) {
          double detX = i + dcx, detY = j + dcy;                   /* :33-34 */
          double wx = exx * sdd + eyx * detX, wy = exy * sdd + eyy * detX; /* :37 */
          double rz = detY;                                        /* :38 */
          double nrm = sqrt(wx * wx + wy * wy + rz * rz);          /* :39 */
          double rx = wx / nrm, ry = wy / nrm;
          rz /= nrm;
          double sx = -exx * sid, sy = -exy * sid, sz = 0.0; /* :40 */
          double a0, a1;
          if (fabs(rx) >= fabs(ry)) { /* :45-50 */
            a0 = (vcx - sx) / rx;
            a1 = (X + vcx - sx) / rx;
          } else { /* :51-56 */
            a0 = (vcy - sy) / ry;
            a1 = (Y + vcy - sy) / ry;
          }
          double amin = fmin(a0, a1) - 3, amax = fmax(a0, a1) + 3; /* :57-58 */
          double s = sid / sdd;                                     /* :63 */
          double pix = 0.0;
          while (amin < amax) { /* :66-80 */
            double px = (sx + amin * rx) / s - vcx;
            double py = (sy + amin * ry) / s - vcy;
            double pz = (sz + amin * rz) / s - vcz;
            pix += tri(V, X, Y, Z, px, py, pz, q);
            amin += s;
          }
          pix *= s; /* :82 */
          sino[(((int64_t)b * n_angles + a) * H + j) * W + i] = pix; /* :84-85 */
        }
    }
}

/* 2-D line intersection, model/ConeBeamLayers/Standard/plug/include/
 * helper_geometry.h:26-42 (same formula and degeneracy threshold). */
static void isect2(double p1x, double p1y, double p2x, double p2y, double p3x, double p3y,
                   double p4x, double p4y, double* ox, double* oy) {
  double dn = (p1x - p2x) * (p3y - p4y) - (p1y - p2y) * (p3x - p4x);
  if (dn < 0.000001 && dn > -0.000001) {
    *ox = NAN;
    *oy = NAN;
    return;
  }
  double x = (p1x * p2y - p1y * p2x) * (p3x - p4x) - (p1x - p2x) * (p3x * p4y - p3y * p4x);
  double y = (p1x * p2y - p1y * p2x) * (p3y - p4y) - (p1y - p2y) * (p3x * p4y - p3y * p4x);
  *ox = x / dn;
  *oy = y / dn;
}

/* Standard FDK-weighted backprojector, model/ConeBeamLayers/Standard/plug/
 * kernel/backwardKernel.cu:22-53 (kernel) and :77-103 (host loops). */
void oracle_backward_standard_literal(const double* sino, int batch, const double* angles_deg,
                                      int n_angles, int X, int Y, int Z, int W, int H, double sid,
                                      double sdd, int q, double* vol) {
  const double vcx = X / -2.0, vcy = Y / -2.0, vcz = Z / -2.0; /* :78 */
  const double dcx = W / -2.0, dcy = H / -2.0;                 /* :80 */
  memset(vol, 0, sizeof(double) * (size_t)batch * X * Y * Z);
#pragma omp parallel for collapse(3) schedule(static)
  for (int b = 0; b < batch; ++b)
    for (int y = 0; y < Y; ++y)
      for (int x = 0; x < X; ++x) {
        double* Vb = vol + (int64_t)b * X * Y * Z;
        for (int a = 0; a < n_angles; ++a) { /* :101-103, views in order */
          const double* S = sino + ((int64_t)b * n_angles + a) * W * H;
          double s = sid / sdd;                                   /* :29 */
          double cx = (vcx + x) * s, cy = (vcy + y) * s;          /* :30 */
          double angle = angles_deg[a] / 180.0 * REF_PI - REF_PI / 2.0; /* :32 */
          double exx = cos(angle), exy = sin(angle);              /* :33 */
          double eyx = -exy, eyy = exx;                           /* :34 */
          double srcx = exx * sid, srcy = exy * sid;              /* :35 */
          double detx = exx * (sdd - sid), dety = exy * (sdd - sid); /* :36 */
          double ix, iy;
          isect2(cx, cy, -srcx, -srcy, detx, dety, detx + eyx, dety + eyy, &ix, &iy); /* :37 */
          double u = ix * eyx + iy * eyy - dcx;                  /* :38 */
          double bx = srcx + cx, by = srcy + cy;                  /* :40 */
          double dz = sdd / (bx * exx + by * exy) * s;            /* :41 */
          double z = vcz * dz - dcy;                              /* :42 */
          double coff = dz / s;                                   /* :44 */
          for (int k = 0; k < Z; ++k) {                           /* :47-52 */
            double val = bil(S, W, H, u, z, q);
            Vb[((int64_t)k * Y + y) * X + x] += val * coff * coff * REF_PI / n_angles;
            z += dz;
          }
        }
      }
}

/* Vector-geometry forward projector, model/ConeBeamLayers/Beijing/plug/kernel/
 * forwardKernel.cu:17-76 (kernel) and :102-128 (host). pv is [n][12]. */
void oracle_forward_vector_literal(const double* vol, int batch, const double* pv, int n_views,
                                   int X, int Y, int Z, int W, int H, int q, double* sino) {
  const double vcx = X / -2.0, vcy = Y / -2.0, vcz = Z / -2.0; /* :103 */
  const double dcx = W / -2.0, dcy = H / -2.0;                 /* :105 */
#pragma omp parallel for collapse(2) schedule(dynamic)
  for (int b = 0; b < batch; ++b)
    for (int n = 0; n < n_views; ++n) {
      const double* V = vol + (int64_t)b * X * Y * Z;
      const double* P = pv + 12 * n;
      double s[3] = {P[0], P[1], -P[2]};  /* :27 */
      double d[3] = {P[3], P[4], -P[5]};  /* :28 */
      double vv[3] = {P[6], P[7], P[8]};  /* :29 */
      double uu[3] = {P[9], P[10], P[11]}; /* :30 */
      for (int j = 0; j < H; ++j)
        for (int i = 0; i < W; ++i) {
          double detX = i + dcx, detY = j + dcy; /* :24-25 */
          double px[3], r[3];
          for (int c = 0; c < 3; ++c) px[c] = d[c] + (0.5 + detX) * uu[c] + (0.5 + detY) * vv[c]; /* :33 */
          for (int c = 0; c < 3; ++c) r[c] = px[c] - s[c];
          double nrm = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]); /* :35 */
          for (int c = 0; c < 3; ++c) r[c] /= nrm;
          double dom = fmax(fabs(r[0]), fmax(fabs(r[2]), fabs(r[1]))); /* :40 */
          double a0, a1;
          if (fabs(r[0]) == dom) {
            a0 = (vcx - s[0]) / r[0];
            a1 = (X + vcx - s[0]) / r[0];
          } else if (fabs(r[1]) == dom) {
            a0 = (vcy - s[1]) / r[1];
            a1 = (Y + vcy - s[1]) / r[1];
          } else {
            a0 = (vcz - s[2]) / r[2];
            a1 = (Z + vcz - s[2]) / r[2];
          }
          double amin = fmin(a0, a1) - 3, amax = fmax(a0, a1) + 3; /* :59-60 */
          double pix = 0.0;
          while (amin < amax) { /* :63-73 */
            double x = s[0] + amin * r[0] - vcx;
            double y = s[1] + amin * r[1] - vcy;
            double z = s[2] + amin * r[2] - vcz;
            pix += tri(V, X, Y, Z, x, y, z, q);
            amin += 1.0;
          }
          sino[(((int64_t)b * n_views + n) * H + j) * W + i] = pix; /* :74-75 */
        }
    }
}

static inline double det3(const double* a, const double* b, const double* c) {
  /* Beijing/plug/include/helper_math.h det3: a . (b x c) */
  return a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) +
         a[2] * (b[0] * c[1] - b[1] * c[0]);
}

/* Vector-geometry backprojector, model/ConeBeamLayers/Beijing/plug/kernel/
 * backwardKernel.cu:18-45 (kernel) and :47-104 (host), for any view count
 * (the reference requires a multiple of 1512 through its texture chunking). */
void oracle_backward_vector_literal(const double* sino, int batch, const double* pv, int n_views,
                                    int X, int Y, int Z, int W, int H, int q, double* vol) {
  const double vcx = X / -2.0, vcy = Y / -2.0, vcz = Z / -2.0; /* :73 */
  const double dcx = W / -2.0, dcy = H / -2.0;                 /* :74 */
  const int blocks = n_views / 21;                             /* :96 angles/21 */
  memset(vol, 0, sizeof(double) * (size_t)batch * X * Y * Z);
#pragma omp parallel for collapse(3) schedule(static)
  for (int b = 0; b < batch; ++b)
    for (int y = 0; y < Y; ++y)
      for (int x = 0; x < X; ++x) {
        double* Vb = vol + (int64_t)b * X * Y * Z;
        for (int k = 0; k < Z; ++k) {
          double acc_all = 0.0;
          for (int a0 = 0; a0 < n_views; a0 += 21) { /* one launch per 21 views (:95-96) */
            double value = 0.0;
            int found = 0;
            for (int a = a0; a < a0 + 21 && a < n_views; ++a) { /* :28 */
              const double* P = pv + 12 * a;
              double s[3] = {P[0], P[1], -P[2]}, d[3] = {P[3], P[4], -P[5]};
              double vv[3] = {P[6], P[7], P[8]}, uu[3] = {P[9], P[10], P[11]};
              double c[3] = {vcx + x, vcy + y, vcz + k}; /* :33 */
              double smc[3], cms[3], smd[3];
              for (int t = 0; t < 3; ++t) {
                smc[t] = s[t] - c[t];
                cms[t] = c[t] - s[t];
                smd[t] = s[t] - d[t];
              }
              double fs = 1.0 / det3(uu, vv, smc);            /* :34 */
              double dX = fs * det3(cms, vv, smd) - dcx;       /* :35 */
              double dY = fs * det3(uu, cms, smd) - dcy;       /* :36 */
              double fr = fs * det3(uu, vv, smd);              /* :37 */
              if (dX < -1 || dX > X + 1 || dY < -1 || dY > Y + 1) continue; /* :38 */
              found = 1;
              /* tex3D(sino, dX, dY, a%TEXA+0.5): texel coordinate dX is pixel
               * coordinate dX-0.5 (:40) */
              value += fr * bil(sino + ((int64_t)b * n_views + a) * W * H, W, H, dX - 0.5,
                                dY - 0.5, q);
            }
            if (found) acc_all += value * 2 * REF_PI / blocks; /* :43 */
          }
          Vb[((int64_t)k * Y + y) * X + x] = acc_all;
        }
      }
}

/* ------------------------------------------------------------------------ */
/* layer 2: per-view vector form                                             */
/* ------------------------------------------------------------------------ */

/* Circular views in the Standard convention (forwardKernel.cu:30-40). */
void oracle_standard_views(const double* angles_deg, int n, double sid, double sdd, double* views) {
  for (int a = 0; a < n; ++a) {
    double angle = angles_deg[a] / 180.0 * REF_PI - REF_PI / 2.0;
    double exx = cos(angle), exy = sin(angle);
    double* o = views + 12 * a;
    o[0] = -exx * sid; o[1] = -exy * sid; o[2] = 0.0;                 /* source */
    o[3] = exx * (sdd - sid); o[4] = exy * (sdd - sid); o[5] = 0.0;   /* detector centre */
    o[6] = -exy; o[7] = exx; o[8] = 0.0;                              /* U = e_y */
    o[9] = 0.0; o[10] = 0.0; o[11] = 1.0;                             /* V = e_z */
  }
}

/* Circular views with explicit pitch (general geometry). */
void oracle_circular_views(const double* angles_deg, int n, double sod, double sdd, double pu,
                           double pv, double* views) {
  for (int a = 0; a < n; ++a) {
    double angle = angles_deg[a] / 180.0 * EXACT_PI - EXACT_PI / 2.0;
    double exx = cos(angle), exy = sin(angle);
    double* o = views + 12 * a;
    o[0] = -exx * sod; o[1] = -exy * sod; o[2] = 0.0;
    o[3] = exx * (sdd - sod); o[4] = exy * (sdd - sod); o[5] = 0.0;
    o[6] = -exy * pu; o[7] = exx * pu; o[8] = 0.0;
    o[9] = 0.0; o[10] = 0.0; o[11] = pv;
  }
}

static void ray_of(const og_geometry* g, const double* vw, int u, int v, double* S, double* r) {
  for (int c = 0; c < 3; ++c) {
    S[c] = vw[c];
    double P = vw[3 + c] + (u - g->nu / 2.0 + g->det_off[0]) * vw[6 + c] +
               (v - g->nv / 2.0 + g->det_off[1]) * vw[9 + c];
    r[c] = P - S[c];
  }
  double nrm = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
  for (int c = 0; c < 3; ++c) r[c] /= nrm;
}

/* Exact ray / voxel-edge box chord in world units; returns 0 if missed. */
static int box_chord(const og_geometry* g, const double* S, const double* r, double* tin,
                     double* tout) {
  const int n[3] = {g->nx, g->ny, g->nz};
  double lo = -INFINITY, hi = INFINITY;
  for (int c = 0; c < 3; ++c) {
    double o = (-n[c] / 2.0 + g->vol_off[c]) * g->voxel[c];
    double bmin = o - 0.5 * g->voxel[c], bmax = o + (n[c] - 0.5) * g->voxel[c];
    if (r[c] == 0.0) {
      if (S[c] < bmin || S[c] > bmax) return 0;
      continue;
    }
    double t0 = (bmin - S[c]) / r[c], t1 = (bmax - S[c]) / r[c];
    if (t0 > t1) { double t = t0; t0 = t1; t1 = t; }
    if (t0 > lo) lo = t0;
    if (t1 < hi) hi = t1;
  }
  *tin = lo;
  *tout = hi;
  return hi > lo;
}

/* Sample range of one ray under the geometry's phase rule:
 * samples at a0 + k*step for 0 <= k < nk. */
static void ray_samples(const og_geometry* g, const double* S, const double* r, double* a0,
                        long* nk) {
  const int n[3] = {g->nx, g->ny, g->nz};
  if (g->phase == 2) {
    double ti, to;
    if (!box_chord(g, S, r, &ti, &to)) { *a0 = 0; *nk = 0; return; }
    *nk = (long)ceil((to - ti) / g->step);
    *a0 = ti + 0.5 * g->step;
    return;
  }
  int ax;
  if (g->phase == 0) {
    ax = fabs(r[0]) >= fabs(r[1]) ? 0 : 1; /* Standard forwardKernel.cu:45 */
  } else {
    double dom = fmax(fabs(r[0]), fmax(fabs(r[2]), fabs(r[1]))); /* Beijing :40-58 */
    ax = fabs(r[0]) == dom ? 0 : (fabs(r[1]) == dom ? 1 : 2);
  }
  double e0 = -n[ax] / 2.0, e1 = n[ax] / 2.0; /* bounds in world units (the quirk) */
  double t0 = (e0 - S[ax]) / r[ax], t1 = (e1 - S[ax]) / r[ax];
  double lo = fmin(t0, t1) - 3, hi = fmax(t0, t1) + 3;
  *a0 = lo;
  *nk = (long)ceil((hi - lo) / g->step);
}

void oracle_forward(const og_geometry* g, const double* views, const double* vol, int batch, int q,
                    double* sino) {
  const int nx = g->nx, ny = g->ny, nz = g->nz, nu = g->nu, nv = g->nv;
  /* one task per detector row, so that a few views still use every core */
#pragma omp parallel for collapse(3) schedule(dynamic)
  for (int b = 0; b < batch; ++b)
    for (int n = 0; n < g->n_views; ++n)
      for (int v = 0; v < nv; ++v) {
        const double* V = vol + (int64_t)b * nx * ny * nz;
        const double* vw = views + 12 * n;
        for (int u = 0; u < nu; ++u) {
          double S[3], r[3], a0;
          long nk;
          ray_of(g, vw, u, v, S, r);
          ray_samples(g, S, r, &a0, &nk);
          double acc = 0.0;
          for (long k = 0; k < nk; ++k) {
            double a = a0 + k * g->step, p[3];
            for (int c = 0; c < 3; ++c) {
              double w = S[c] + a * r[c];
              p[c] = w / g->voxel[c] + (c == 0 ? nx : c == 1 ? ny : nz) / 2.0 - g->vol_off[c];
            }
            acc += tri(V, nx, ny, nz, p[0], p[1], p[2], q);
          }
          sino[(((int64_t)b * g->n_views + n) * nv + v) * nu + u] = acc * g->scale;
        }
    }
}

/* Exact transpose of oracle_forward with q = 0: vol = A^T sino. */
void oracle_adjoint(const og_geometry* g, const double* views, const double* sino, int batch,
                    double* vol) {
  const int nx = g->nx, ny = g->ny, nz = g->nz, nu = g->nu, nv = g->nv;
  const int64_t V1 = (int64_t)nx * ny * nz;
  memset(vol, 0, sizeof(double) * (size_t)batch * V1);
  for (int b = 0; b < batch; ++b) {
#pragma omp parallel
    {
      double* acc = (double*)calloc((size_t)V1, sizeof(double));
#pragma omp for schedule(dynamic)
      for (int n = 0; n < g->n_views; ++n) {
        const double* vw = views + 12 * n;
        for (int v = 0; v < nv; ++v)
          for (int u = 0; u < nu; ++u) {
            double y = sino[(((int64_t)b * g->n_views + n) * nv + v) * nu + u] * g->scale;
            if (y == 0.0) continue;
            double S[3], r[3], a0;
            long nk;
            ray_of(g, vw, u, v, S, r);
            ray_samples(g, S, r, &a0, &nk);
            for (long k = 0; k < nk; ++k) {
              double a = a0 + k * g->step, p[3];
              for (int c = 0; c < 3; ++c)
                p[c] = (S[c] + a * r[c]) / g->voxel[c] + (c == 0 ? nx : c == 1 ? ny : nz) / 2.0 -
                       g->vol_off[c];
              double fx = floor(p[0]), fy = floor(p[1]), fz = floor(p[2]);
              if (fx < -1 || fy < -1 || fz < -1 || fx > nx || fy > ny || fz > nz) continue;
              int ix = (int)fx, iy = (int)fy, iz = (int)fz;
              double ax = p[0] - fx, ay = p[1] - fy, az = p[2] - fz;
              for (int dz = 0; dz < 2; ++dz) {
                int zz = iz + dz;
                if (zz < 0 || zz >= nz) continue;
                for (int dy = 0; dy < 2; ++dy) {
                  int yy = iy + dy;
                  if (yy < 0 || yy >= ny) continue;
                  for (int dx = 0; dx < 2; ++dx) {
                    int xx = ix + dx;
                    if (xx < 0 || xx >= nx) continue;
                    double w = (dz ? az : 1 - az) * (dy ? ay : 1 - ay) * (dx ? ax : 1 - ax);
                    acc[((int64_t)zz * ny + yy) * nx + xx] += w * y;
                  }
                }
              }
            }
          }
      }
#pragma omp critical
      {
        double* out = vol + (int64_t)b * V1;
        for (int64_t i = 0; i < V1; ++i) out[i] += acc[i];
      }
      free(acc);
    }
  }
}

/* FDK-weighted voxel-driven backprojector over the vector description. */
void oracle_backward(const og_geometry* g, const double* views, const double* sino, int batch,
                     int q, double* vol) {
  const int nx = g->nx, ny = g->ny, nz = g->nz, nu = g->nu, nv = g->nv;
  const int64_t V1 = (int64_t)nx * ny * nz;
#pragma omp parallel for collapse(3) schedule(static)
  for (int b = 0; b < batch; ++b)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j) {
        for (int i = 0; i < nx; ++i) {
          double x[3] = {(i - nx / 2.0 + g->vol_off[0]) * g->voxel[0],
                         (j - ny / 2.0 + g->vol_off[1]) * g->voxel[1],
                         (k - nz / 2.0 + g->vol_off[2]) * g->voxel[2]};
          double acc = 0.0;
          for (int n = 0; n < g->n_views; ++n) {
            const double* vw = views + 12 * n;
            const double *S = vw, *D = vw + 3, *U = vw + 6, *Vv = vw + 9;
            double nr[3] = {U[1] * Vv[2] - U[2] * Vv[1], U[2] * Vv[0] - U[0] * Vv[2],
                            U[0] * Vv[1] - U[1] * Vv[0]};
            double dms[3] = {D[0] - S[0], D[1] - S[1], D[2] - S[2]};
            double rr[3] = {x[0] - S[0], x[1] - S[1], x[2] - S[2]};
            double sdd = dms[0] * nr[0] + dms[1] * nr[1] + dms[2] * nr[2];
            double L = rr[0] * nr[0] + rr[1] * nr[1] + rr[2] * nr[2];
            double t = sdd / L;
            double P[3] = {S[0] + t * rr[0] - D[0], S[1] + t * rr[1] - D[1],
                           S[2] + t * rr[2] - D[2]};
            /* P = a U + b V: solve the 2x2 normal equations */
            double uu = U[0] * U[0] + U[1] * U[1] + U[2] * U[2];
            double vv = Vv[0] * Vv[0] + Vv[1] * Vv[1] + Vv[2] * Vv[2];
            double uv = U[0] * Vv[0] + U[1] * Vv[1] + U[2] * Vv[2];
            double pu = P[0] * U[0] + P[1] * U[1] + P[2] * U[2];
            double pv = P[0] * Vv[0] + P[1] * Vv[1] + P[2] * Vv[2];
            double det = uu * vv - uv * uv;
            double a = (pu * vv - pv * uv) / det, bb = (pv * uu - pu * uv) / det;
            double u = a + nu / 2.0 - g->det_off[0];
            double v = bb + nv / 2.0 - g->det_off[1];
            if (g->bp_extent) {
              double tx = u + 0.5, ty = v + 0.5; /* texel coordinates */
              if (tx < -1 || tx > nx + 1 || ty < -1 || ty > ny + 1) continue;
            }
            double val = bil(sino + ((int64_t)b * g->n_views + n) * nu * nv, nu, nv, u, v, q);
            acc += val * g->bp_scale * pow(sdd / L, (double)g->bp_pow);
          }
          vol[(int64_t)b * V1 + ((int64_t)k * ny + j) * nx + i] = acc;
        }
      }
}

/* Algorithmic work count: sum over rays of ceil(chord/step) over the exact
 * voxel-edge box (independent of the phase rule). */
double oracle_fp_samples(const og_geometry* g, const double* views) {
  double total = 0.0;
#pragma omp parallel for reduction(+ : total) collapse(2) schedule(dynamic)
  for (int n = 0; n < g->n_views; ++n)
    for (int v = 0; v < g->nv; ++v)
      for (int u = 0; u < g->nu; ++u) {
        double S[3], r[3], ti, to;
        ray_of(g, views + 12 * n, u, v, S, r);
        if (box_chord(g, S, r, &ti, &to)) total += ceil((to - ti) / g->step);
      }
  return total;
}

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
