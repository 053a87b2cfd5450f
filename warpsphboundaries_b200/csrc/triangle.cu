// Conditioned single triangles (2-D): the twelve channels of a solid triangle by float64 area quadrature, for the
// rows where the closed form would lose digits -- the triangle is small (longest edge <= 0.02 h) or a sliver
// (2 area <= 0.01 longest edge^2).  Other rows keep the closed form (status 0).
//
// Reference: src/warpSPHBoundaries/edge/warptriangle.py:126-277 (channels, _triangle_kernel, _panel, _line, _cuts,
// prepare) and its use as a per-row override in src/warpSPHBoundaries/scene/fused.py:556-564 / scene.py:405-409.
//
// Integration (unit support, y relative to the query, body frame): the triangle is mapped from the unit square by
// y(u, t) = a + u b + t (1 - u) c (a = v0, b = v1 - v0, c = v2 - v0 with c the shortest edge, so the inner lines
// t -> y are short), dA = 2 area (1 - u) du dt.  Inner lines: split where they cross the kernel's knot and support
// circles and at the foot of the perpendicular from the query, then Gauss-Legendre (16 nodes) on panels graded by
// distance from the foot (d 2^k, d = the line's distance to the query), so the branch points of r on each line stay
// away from every panel.  Outer direction: the cuts where the edges cross the circles and where the lines pass
// through the query or touch a circle (u = (+-R |c| - a x c) / (b x c)), then adaptive bisection comparing 16- and
// 8-node Gauss-Legendre: a panel is accepted when max |fine - coarse| <= tol (width + max |fine|) over the twelve
// channels (each scaled by the triangle's extent from the query), until `max_panels` panels were visited; a row
// whose budget runs out gets status -1 and NaN channels.
#include "common.cuh"

namespace wsb {
namespace {

constexpr int kTriThreads = 64;

template <class K>
__device__ __forceinline__ void tri_prof(double r, double& w, double& rho) {
  if constexpr (K::kPieces > 1) {
    if (r >= K::kKnot) {
      K::template eval<1>(r, w, rho);
      return;
    }
  }
  K::template eval<0>(r, w, rho);
}

struct TriGeo {
  double a[2], b[2], c[2];
  double sc[12];       // 1 / channel scales
};

// wt * f(y) / scale into acc: W, y W, -W'/r y, y (x) (-W'/r y), y y W (pi W units)
template <class K>
__device__ __forceinline__ void add_point(double y0, double y1, double wt, const double* isc, double* acc) {
  const double r = sqrt(fma(y0, y0, y1 * y1));
  if (r >= 1.0) return;
  double w, rho;
  tri_prof<K>(r, w, rho);
  const double W = wt * w, gx = wt * rho * y0, gy = wt * rho * y1;
  acc[0] += W * isc[0];
  acc[1] += y0 * W * isc[1];
  acc[2] += y1 * W * isc[2];
  acc[3] += gx * isc[3];
  acc[4] += gy * isc[4];
  acc[5] += y0 * gx * isc[5];
  acc[6] += y0 * gy * isc[6];
  acc[7] += y1 * gx * isc[7];
  acc[8] += y1 * gy * isc[8];
  acc[9] += y0 * y0 * W * isc[9];
  acc[10] += y0 * y1 * W * isc[10];
  acc[11] += y1 * y1 * W * isc[11];
}

__device__ __forceinline__ void gl16(int g, double& x, double& w) {
  // 16-node Gauss-Legendre on [-1, 1] (kTriGx16 / kTriGw16 of the generated tables)
  x = kTriGx16[g];
  w = kTriGw16[g];
}

// int_0^1 f(y(u, t)) dt along the line y = S + t D, added into acc times wscale.  Panels live in t itself (their
// widths, hence the weights, keep full relative precision however short the segment is next to its distance from
// the query); their ends sit at the support circle, the knot circle, the foot of the perpendicular t* and at
// distances d 2^k from the foot (d = the line's distance to the query).
template <class K>
__device__ void line_integral(double u, const TriGeo& T, double wscale, double* acc) {
  const double S[2] = {fma(u, T.b[0], T.a[0]), fma(u, T.b[1], T.a[1])};
  const double D[2] = {(1.0 - u) * T.c[0], (1.0 - u) * T.c[1]};
  const double DD = fma(D[0], D[0], D[1] * D[1]);
  if (!(DD > 0.0)) return;
  const double Dl = sqrt(DD), iDl = 1.0 / Dl;
  const double ts = -fma(S[0], D[0], S[1] * D[1]) / DD;                   // foot of the perpendicular
  const double d = fabs(S[0] * D[1] - S[1] * D[0]) * iDl;                 // distance of the line to the query
  if (d >= 1.0) return;
  const double L1 = sqrt((1.0 - d) * (1.0 + d));
  const double tlo = fmax(0.0, ts - L1 * iDl), thi = fmin(1.0, ts + L1 * iDl);
  if (!(thi > tlo)) return;
  double knot = -1.0;
  if constexpr (K::kPieces > 1) {
    if (d < K::kKnot) knot = sqrt((K::kKnot - d) * (K::kKnot + d));
  }
  const double base = fmax(d, (thi - tlo) * Dl * 9.313225746154785e-10);  // 2^-30 of the span
  for (int side = 0; side < 2; ++side) {
    const double sgn = side == 0 ? -1.0 : 1.0;
    // this side's range in t and in distance from the foot
    const double ta = side == 0 ? tlo : fmax(tlo, ts), tb = side == 0 ? fmin(thi, ts) : thi;
    if (!(tb > ta)) continue;
    const double x0 = side == 0 ? (ts - tb) * Dl : (ta - ts) * Dl;       // nearest distance from the foot
    const double x1 = side == 0 ? (ts - ta) * Dl : (tb - ts) * Dl;
    double dd = base;
    for (int it = 0; it < 200 && dd <= x0; ++it) dd *= 2.0;
    double x = x0, tcur = side == 0 ? tb : ta;                           // walk away from the foot
    for (int it = 0; it < 100 && x < x1; ++it) {
      double nxt = fmin(x1, dd);
      if (knot > x && knot < nxt) nxt = knot;
      const double tn = nxt >= x1 ? (side == 0 ? ta : tb) : ts + sgn * nxt * iDl;
      const double t0 = fmin(tcur, tn), t1 = fmax(tcur, tn);
      if (t1 > t0) {
        const double hc = 0.5 * (t1 - t0), mc = 0.5 * (t1 + t0);
        for (int g = 0; g < 16; ++g) {
          double xg, wg;
          gl16(g, xg, wg);
          const double t = fma(hc, xg, mc);
          add_point<K>(fma(t, D[0], S[0]), fma(t, D[1], S[1]), wg * hc * wscale, T.sc, acc);
        }
      }
      if (nxt >= dd) dd *= 2.0;
      x = nxt;
      tcur = tn;
    }
  }
}

// outer panel [lo, hi] in u: n-node Gauss of (1 - u) * line integral
template <class K>
__device__ void outer_panel(double lo, double hi, const TriGeo& T, bool fine, double* acc) {
#pragma unroll
  for (int k = 0; k < 12; ++k) acc[k] = 0.0;
  const double hc = 0.5 * (hi - lo), mc = 0.5 * (hi + lo);
  const int n = fine ? 16 : 8;
  for (int g = 0; g < n; ++g) {
    const double x = fine ? kTriGx16[g] : kTriGx8[g], w = fine ? kTriGw16[g] : kTriGw8[g];
    const double u = fma(hc, x, mc);
    line_integral<K>(u, T, w * hc * (1.0 - u), acc);
  }
}

__device__ __forceinline__ void add_cut(double* cuts, int& n, double t) {
  if (t > 0.0 && t < 1.0 && n < 24) cuts[n++] = t;
}

// u where the segment p + u q crosses the circles (and its closest point)
template <class K>
__device__ void segment_cuts(double* cuts, int& n, const double p[2], const double q[2]) {
  const double qq = fma(q[0], q[0], q[1] * q[1]);
  if (!(qq > 0.0)) return;
  const double t = -fma(p[0], q[0], p[1] * q[1]) / qq;
  add_cut(cuts, n, t);
  const double cx = fma(t, q[0], p[0]), cy = fma(t, q[1], p[1]);
  const double rr = fma(cx, cx, cy * cy);
  for (int j = 0; j < K::kPieces; ++j) {
    const double R = (K::kPieces > 1 && j == 0) ? K::kKnot : 1.0;
    const double del = (R * R - rr) / qq;
    if (del >= 0.0) {
      const double root = sqrt(del);
      add_cut(cuts, n, t - root);
      add_cut(cuts, n, t + root);
    }
  }
}

template <class K>
__global__ void __launch_bounds__(kTriThreads) k_triangle(const double* __restrict__ lpos,
                                                          const double* __restrict__ sup,
                                                          const int32_t* __restrict__ valid, int64_t n, double v0x,
                                                          double v0y, double v1x, double v1y, double v2x, double v2y,
                                                          double area2, double sign, int background, double tol,
                                                          int max_panels, double* __restrict__ values,
                                                          double* __restrict__ estimate,
                                                          int32_t* __restrict__ status) {
  const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  double* out = values + 12 * row;
  double* est = estimate ? estimate + 12 * row : nullptr;
  if (valid && valid[row] == 0) {
    status[row] = 0;
    for (int k = 0; k < 12; ++k) {
      out[k] = 0.0;
      if (est) est[k] = __longlong_as_double(0x7ff8000000000000LL);
    }
    return;
  }
  const double h = sup[row];
  const double e0x = v1x - v0x, e0y = v1y - v0y, e1x = v2x - v0x, e1y = v2y - v0y;
  const double l0 = fma(e0x, e0x, e0y * e0y), l1 = fma(e1x, e1x, e1y * e1y);
  const double l2 = fma(e1x - e0x, e1x - e0x, (e1y - e0y) * (e1y - e0y));
  const double longest2 = fmax(l0, fmax(l1, l2));
  if (longest2 > 0.02 * 0.02 * h * h && area2 > 0.01 * longest2) {
    status[row] = 0;                                   // well conditioned: the closed form serves this row
    for (int k = 0; k < 12; ++k) {
      out[k] = 0.0;
      if (est) est[k] = __longlong_as_double(0x7ff8000000000000LL);
    }
    return;
  }
  const double ih = 1.0 / h;
  TriGeo T;
  T.a[0] = (v0x - lpos[2 * row]) * ih;
  T.a[1] = (v0y - lpos[2 * row + 1]) * ih;
  T.b[0] = e0x * ih;
  T.b[1] = e0y * ih;
  T.c[0] = e1x * ih;
  T.c[1] = e1y * ih;
  double sx = fmax(fabs(T.a[0]), fmax(fabs(T.a[0] + T.b[0]), fabs(T.a[0] + T.c[0])));
  double sy = fmax(fabs(T.a[1]), fmax(fabs(T.a[1] + T.b[1]), fabs(T.a[1] + T.c[1])));
  sx = fmax(sx, 1e-150);
  sy = fmax(sy, 1e-150);
  const double scl[12] = {1.0, sx, sy, sx, sy, sx * sx, sx * sy, sy * sx, sy * sy, sx * sx, sx * sy, sy * sy};
#pragma unroll
  for (int k = 0; k < 12; ++k) T.sc[k] = 1.0 / scl[k];
  // outer cuts
  double cuts[24];
  int nc = 0;
  cuts[nc++] = 0.0;
  cuts[nc++] = 1.0;
  segment_cuts<K>(cuts, nc, T.a, T.b);
  const double ac_[2] = {T.a[0] + T.c[0], T.a[1] + T.c[1]}, bmc[2] = {T.b[0] - T.c[0], T.b[1] - T.c[1]};
  segment_cuts<K>(cuts, nc, ac_, bmc);
  const double bc = T.b[0] * T.c[1] - T.b[1] * T.c[0], acr = T.a[0] * T.c[1] - T.a[1] * T.c[0];
  if (bc != 0.0) {
    add_cut(cuts, nc, -acr / bc);
    const double cl = sqrt(fma(T.c[0], T.c[0], T.c[1] * T.c[1]));
    for (int j = 0; j < K::kPieces; ++j) {
      const double R = (K::kPieces > 1 && j == 0) ? K::kKnot : 1.0;
      add_cut(cuts, nc, (R * cl - acr) / bc);
      add_cut(cuts, nc, (-R * cl - acr) / bc);
    }
  }
  for (int i = 1; i < nc; ++i) {                        // insertion sort
    const double key = cuts[i];
    int j = i - 1;
    while (j >= 0 && cuts[j] > key) {
      cuts[j + 1] = cuts[j];
      --j;
    }
    cuts[j + 1] = key;
  }
  double total[12], errs[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) total[k] = errs[k] = 0.0;
  int st = 1, visited = 0;
  double slo[64], shi[64];
  for (int part = 0; part + 1 < nc; ++part) {
    int size = 1;
    slo[0] = cuts[part];
    shi[0] = cuts[part + 1];
    while (size > 0) {
      --size;
      const double lo = slo[size], hi = shi[size];
      if (!(hi > lo)) continue;
      double fine[12], coarse[12];
      outer_panel<K>(lo, hi, T, true, fine);
      outer_panel<K>(lo, hi, T, false, coarse);
      double err = 0.0, norm = 0.0;
#pragma unroll
      for (int k = 0; k < 12; ++k) {
        err = fmax(err, fabs(fine[k] - coarse[k]));
        norm = fmax(norm, fabs(fine[k]));
      }
      ++visited;
      const bool accept = err <= tol * (hi - lo + norm);
      if (!accept && size < 62 && visited < max_panels && hi - lo > 1e-14) {
        const double mid = 0.5 * (lo + hi);
        slo[size] = mid;
        shi[size] = hi;
        slo[size + 1] = lo;
        shi[size + 1] = mid;
        size += 2;
      } else {
        if (!accept) st = -1;
#pragma unroll
        for (int k = 0; k < 12; ++k) {
          total[k] += fine[k];
          errs[k] += fabs(fine[k] - coarse[k]);
        }
      }
    }
  }
  status[row] = st;
  const double jac = area2 * ih * ih * kInvPi;
  double plane[12];
  {
    // whole-support constants: mass on lam and the g1 diagonal, the plane second moment on m20 / m02
    plane[0] = plane[5] = plane[8] = 1.0;
    plane[9] = plane[11] = K::kPlane2;
    plane[1] = plane[2] = plane[3] = plane[4] = plane[6] = plane[7] = plane[10] = 0.0;
  }
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    out[k] = st < 0 ? __longlong_as_double(0x7ff8000000000000LL)
                    : (double)background * plane[k] + sign * total[k] * scl[k] * jac;
    if (est) est[k] = errs[k] * scl[k] * jac;
  }
}

// rows with status != 0 take the quadrature (unit support, body frame, legacy order lam m1 G g1 m2) rotated into the
// world frame and scaled; the other rows take the closed form `c*`; both assigned or added into the outputs
__global__ void k_triangle_combine(const double* __restrict__ q, const int32_t* __restrict__ status,
                                   const double* __restrict__ sup, const double* __restrict__ pose, int64_t n,
                                   int add, const double* __restrict__ clam, const double* __restrict__ cG,
                                   const double* __restrict__ ccov, const double* __restrict__ cm1,
                                   const double* __restrict__ cm2, double* __restrict__ lam, double* __restrict__ G,
                                   double* __restrict__ cov, double* __restrict__ m1, double* __restrict__ m2) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double L, g[2], C[4], a1[2], a2[4];
  if (status[i] != 0) {
    const double* v = q + 12 * i;
    const double h = sup[i], c = pose[2], s = pose[3];
    auto rot = [&](double x, double y, double* o) {
      o[0] = c * x - s * y;
      o[1] = s * x + c * y;
    };
    // R M R^T for a 2 x 2 tensor M = [[m00, m01], [m10, m11]]
    auto rot2 = [&](double m00, double m01, double m10, double m11, double* o) {
      const double r00 = c * m00 - s * m10, r01 = c * m01 - s * m11, r10 = s * m00 + c * m10, r11 = s * m01 + c * m11;
      o[0] = r00 * c - r01 * s;
      o[1] = r00 * s + r01 * c;
      o[2] = r10 * c - r11 * s;
      o[3] = r10 * s + r11 * c;
    };
    L = v[0];
    rot(v[1] * h, v[2] * h, a1);
    rot(v[3] / h, v[4] / h, g);
    rot2(v[5], v[6], v[7], v[8], C);
    rot2(v[9] * h * h, v[10] * h * h, v[10] * h * h, v[11] * h * h, a2);
  } else {
    L = clam[i];
    g[0] = cG[2 * i];
    g[1] = cG[2 * i + 1];
    a1[0] = cm1[2 * i];
    a1[1] = cm1[2 * i + 1];
    for (int k = 0; k < 4; ++k) {
      C[k] = ccov[4 * i + k];
      a2[k] = cm2[4 * i + k];
    }
  }
  if (add) {
    lam[i] += L;
    for (int k = 0; k < 2; ++k) {
      G[2 * i + k] += g[k];
      m1[2 * i + k] += a1[k];
    }
    for (int k = 0; k < 4; ++k) {
      cov[4 * i + k] += C[k];
      m2[4 * i + k] += a2[k];
    }
  } else {
    lam[i] = L;
    for (int k = 0; k < 2; ++k) {
      G[2 * i + k] = g[k];
      m1[2 * i + k] = a1[k];
    }
    for (int k = 0; k < 4; ++k) {
      cov[4 * i + k] = C[k];
      m2[4 * i + k] = a2[k];
    }
  }
}

template <class K>
int launch_tri(const double* v, double area2, double sign, int background, const double* lpos, const double* sup,
               const int32_t* valid, int64_t n, double tol, int max_panels, double* values, double* estimate,
               int32_t* status, cudaStream_t st) {
  k_triangle<K><<<(unsigned)((n + kTriThreads - 1) / kTriThreads), kTriThreads, 0, st>>>(
      lpos, sup, valid, n, v[0], v[1], v[2], v[3], v[4], v[5], area2, sign, background, tol, max_panels, values,
      estimate, status);
  WSB_CUDA(cudaGetLastError());
  return WSB_OK;
}

}  // namespace
}  // namespace wsb

using namespace wsb;

extern "C" int wsb_triangle_channels(const double* tri, double area2, double sign, int background, int kernel,
                                     const double* lpos, const double* sup, const int32_t* valid, int64_t n,
                                     double tolerance, int max_panels, double* values, double* estimate,
                                     int32_t* status, void* stream) {
  if (!tri) return fail(WSB_ERR_ARG, "wsb_triangle_channels: NULL triangle");
  if (n < 0) return fail(WSB_ERR_ARG, "wsb_triangle_channels: negative size");
  if (!(tolerance > 0.0) || max_panels < 1)
    return fail(WSB_ERR_ARG, "wsb_triangle_channels: positive tolerance and max_panels required");
  if (!(area2 > 0.0) || (sign != 1.0 && sign != -1.0) || (background != 0 && background != 1))
    return fail(WSB_ERR_ARG, "wsb_triangle_channels: area2 > 0, sign +-1 and background 0/1 required");
  if (n == 0) return WSB_OK;
  if (!lpos || !sup || !values || !status) return fail(WSB_ERR_ARG, "wsb_triangle_channels: NULL array");
  cudaStream_t st = (cudaStream_t)stream;
  switch (kernel) {
    case WSB_KERNEL_CUBIC: return launch_tri<Tri_cubic>(tri, area2, sign, background, lpos, sup, valid, n, tolerance, max_panels, values, estimate, status, st);
    case WSB_KERNEL_W2: return launch_tri<Tri_w2>(tri, area2, sign, background, lpos, sup, valid, n, tolerance, max_panels, values, estimate, status, st);
    case WSB_KERNEL_W4: return launch_tri<Tri_w4>(tri, area2, sign, background, lpos, sup, valid, n, tolerance, max_panels, values, estimate, status, st);
    case WSB_KERNEL_W6: return launch_tri<Tri_w6>(tri, area2, sign, background, lpos, sup, valid, n, tolerance, max_panels, values, estimate, status, st);
    case WSB_KERNEL_POLY6: return launch_tri<Tri_poly6>(tri, area2, sign, background, lpos, sup, valid, n, tolerance, max_panels, values, estimate, status, st);
    default:
      return fail(WSB_ERR_UNSUPPORTED, "wsb_triangle_channels: the conditioned triangle rule serves kernels with at "
                                       "most two radii (cubic, w2, w4, w6, poly6)");
  }
}

extern "C" int wsb_triangle_combine(const double* values, const int32_t* status, const double* sup,
                                    const double* pose, int64_t n, int add, const double* clam, const double* cG,
                                    const double* ccov, const double* cm1, const double* cm2, double* lam, double* G,
                                    double* cov, double* m1, double* m2, void* stream) {
  if (n < 0) return fail(WSB_ERR_ARG, "wsb_triangle_combine: negative size");
  if (n == 0) return WSB_OK;
  if (!values || !status || !sup || !pose || !clam || !cG || !ccov || !cm1 || !cm2 || !lam || !G || !cov || !m1 || !m2)
    return fail(WSB_ERR_ARG, "wsb_triangle_combine: NULL array");
  k_triangle_combine<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
      values, status, sup, pose, n, add, clam, cG, ccov, cm1, cm2, lam, G, cov, m1, m2);
  WSB_CUDA(cudaGetLastError());
  return WSB_OK;
}
