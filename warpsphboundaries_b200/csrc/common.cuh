// Shared device code of libwsb: the surface handle, rounding-exact predicates, the winding-number
// indicator and the closed-form chord engine of the twelve edge channels.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <string>

#include "../../include/wsb.h"
#include "kernel_tables.h"

namespace wsb {

constexpr double kInvPi = 0.318309886183790671537767526745028724;
constexpr double kTwoPi = 6.283185307179586;

// device-side status codes written into the optional status word (atomicMax)
enum : int32_t { kStatusOk = 0, kStatusBadEdge = 1, kStatusBadCell = 2 };

void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* where);

#define WSB_CUDA(call)                                   \
  do {                                                   \
    cudaError_t e__ = (call);                            \
    if (e__ != cudaSuccess) return cuda_fail(e__, #call); \
  } while (0)

// ----------------------------------------------------------------------------------------------- surface
struct Surface {
  int device = 0;
  int64_t n_verts = 0, n_edges = 0;
  int background = 0;
  double support_max = 0;
  // edge cell grid
  int32_t nx = 0, ny = 0;
  double lo_x = 0, lo_y = 0, cell = 0;
  int32_t K = 1;
  int64_t n_items = 0;
  // y bins
  int32_t nb = 1;
  double y0 = 0, dy = 1;
  int64_t n_bitems = 0;
  double bbox[4] = {0, 0, 0, 0};
  // device arrays
  double* verts = nullptr;      // [n_verts*2]
  int32_t* edges = nullptr;     // [n_edges*2]
  int32_t* cstart = nullptr;    // [nx*ny+1]
  int32_t* citems = nullptr;    // [n_items]
  double4* crec = nullptr;      // [n_items] (ax, ay, bx, by) of the item's edge, cell-list order
  double* cind = nullptr;       // [nx*ny] winding + background at the cell centre
  int32_t* cok = nullptr;       // [nx*ny] 1 where the centre's winding is certain (clear of every edge line it tests)
  int32_t* cempty = nullptr;    // [nx*ny]
  int32_t* ccompact = nullptr;  // [nx*ny] index of a cell among the cells with edges (cell order), -1 for an empty one
  int32_t n_nonempty = 0;       // cells with edges
  int32_t* bstart = nullptr;    // [nb+1]
  int32_t* bitems = nullptr;    // [n_bitems]
  double4* erec = nullptr;      // [n_edges] (ax, ay, bx, by) by edge id
  double4* brec = nullptr;      // [n_bitems] the records of the y-bin items, bin order
  // host copies (tests, signed distance set-up)
  std::string err;
};

// ----------------------------------------------------------------------------------------------- rounding-exact helpers
// a x b with both products rounded before the subtraction (no FMA contraction): the orientation predicate shared by the
// indicator and the edge terms, src/warpSPHBoundaries/edge/predicates.py:21-31
__device__ __forceinline__ double cross2_rn(double ax, double ay, double bx, double by) {
  return __dsub_rn(__dmul_rn(ax, by), __dmul_rn(ay, bx));
}

__device__ __forceinline__ double dot2_rn(double ax, double ay, double bx, double by) {
  return __dadd_rn(__dmul_rn(ax, bx), __dmul_rn(ay, by));
}

// Pose.toLocal (scene.py:75-79): d = p - c;  (d0 c + d1 s, d1 c - d0 s), every operation rounded on its own
__device__ __forceinline__ void to_local_rn(double px, double py, double cx, double cy, double c, double s, double& lx,
                                            double& ly) {
  const double d0 = __dsub_rn(px, cx), d1 = __dsub_rn(py, cy);
  lx = __dadd_rn(__dmul_rn(d0, c), __dmul_rn(d1, s));
  ly = __dsub_rn(__dmul_rn(d1, c), __dmul_rn(d0, s));
}

// the neighbour predicate |x - seg(a, b)| < h in float64 with the operation order of
// scene.py:135-139 / fixedadj.py:92-96 and no contraction
__device__ __forceinline__ bool seg_within(double px, double py, double ax, double ay, double bx, double by, double h) {
  const double dx = __dsub_rn(bx, ax), dy = __dsub_rn(by, ay);
  const double num = __dadd_rn(__dmul_rn(__dsub_rn(px, ax), dx), __dmul_rn(__dsub_rn(py, ay), dy));
  const double den = fmax(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), 1e-300);
  double t = __ddiv_rn(num, den);
  t = fmin(fmax(t, 0.0), 1.0);
  const double ex = __dsub_rn(px, __dadd_rn(ax, __dmul_rn(t, dx)));
  const double ey = __dsub_rn(py, __dadd_rn(ay, __dmul_rn(t, dy)));
  return __dsqrt_rn(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey))) < h;
}

// The same predicate decided in float first: the float squared distance of the relative vectors (formed in double,
// then rounded) is off by at most ~1e-6 relative for candidates of one cell, so outside a band of 1e-4 around h^2 the
// float answer equals the double answer and the exact test only runs inside the band.
__device__ __forceinline__ bool seg_within_fast(double px, double py, double ax, double ay, double bx, double by,
                                                double h) {
  const float dx = (float)(bx - ax), dy = (float)(by - ay);
  const float rx = (float)(px - ax), ry = (float)(py - ay);
  const float den = dx * dx + dy * dy;
  if (den > 1e-30f) {
    const float t = fminf(fmaxf(__fdividef(rx * dx + ry * dy, den), 0.0f), 1.0f);
    const float ex = rx - t * dx, ey = ry - t * dy;
    const float d2 = ex * ex + ey * ey;
    const float h2 = (float)(h * h);
    if (d2 < h2 * 0.9999f) return true;
    if (d2 > h2 * 1.0001f) return false;
  }
  return seg_within(px, py, ax, ay, bx, by, h);
}

// ----------------------------------------------------------------------------------------------- indicator
struct SurfView {        // the device pointers and scalars a kernel needs (passed by value)
  const double* verts;
  const int32_t* edges;
  int64_t n_edges;
  const int32_t* cstart;
  const double4* crec;
  const int32_t* citems;
  const double* cind;
  const int32_t* cok;
  const int32_t* cempty;
  const int32_t* ccompact;
  const int32_t* bstart;
  const int32_t* bitems;
  const double4* brec;
  const double4* erec;
  int32_t nx, ny, nb, K, nne;
  double lo_x, lo_y, cell, y0, dy;
  double background;
};

// Winding number + background of a point in the body frame, relative coordinates normalised by h (h = 1: none), with the
// logic of the fixed-topology kernel (fixedadj.py:98-145): the cell cache for edge-free cells, ray casting along the y bin
// otherwise, the principal-value angle sum over all edges for points on the boundary; outside the grid the background.
__device__ __forceinline__ double indicator_at(const SurfView& S, double px, double py, double h, bool in_grid,
                                               int32_t cid) {
  if (!in_grid) return S.background;
  if (S.cempty[cid] != 0) return S.cind[cid];
  const double iyd = floor(__ddiv_rn(__dsub_rn(py, S.y0), S.dy));
  if (!(iyd >= 0.0 && iyd <= (double)S.nb)) return S.background;
  int iy = (int)iyd;
  if (iy > S.nb - 1) iy = S.nb - 1;
  double w = 0.0;
  bool boundary = false;
  for (int i = S.bstart[iy]; i < S.bstart[iy + 1]; ++i) {
    const double4 r = S.brec[i];
    const bool up = r.y <= py && py < r.w, down = r.w <= py && py < r.y;
    const double ax = __dsub_rn(r.x, px), ay = __dsub_rn(r.y, py), cx = __dsub_rn(r.z, px), cy = __dsub_rn(r.w, py);
    // the sign of the support-normalised, product-rounded cross product is certain when the unnormalised one
    // clears 1e-10 of its terms' magnitude (the normalised form is accurate to a few ulp of that magnitude)
    const double cu = ax * cy - ay * cx, mag = fabs(ax * cy) + fabs(ay * cx);
    double cr;
    if (fabs(cu) > 1e-10 * mag) {
      cr = cu;
    } else {
      const double arx = __ddiv_rn(ax, h), ary = __ddiv_rn(ay, h), crx = __ddiv_rn(cx, h), cry = __ddiv_rn(cy, h);
      cr = cross2_rn(arx, ary, crx, cry);
      if (cr == 0.0 && dot2_rn(arx, ary, crx, cry) <= 0.0) boundary = true;
    }
    if (up && cr > 0.0) w += 1.0;
    if (down && cr < 0.0) w -= 1.0;
  }
  if (boundary) {
    double ang = 0.0;
    for (int64_t e = 0; e < S.n_edges; ++e) {
      const double4 r = S.erec[e];
      const double arx = __ddiv_rn(__dsub_rn(r.x, px), h), ary = __ddiv_rn(__dsub_rn(r.y, py), h);
      const double crx = __ddiv_rn(__dsub_rn(r.z, px), h), cry = __ddiv_rn(__dsub_rn(r.w, py), h);
      const double cr = cross2_rn(arx, ary, crx, cry);
      if (cr != 0.0) ang += atan2(cr, dot2_rn(arx, ary, crx, cry));
    }
    w = ang / kTwoPi;
  }
  return w + S.background;
}

// orientation of x against the line a -> b with a certainty test: returns +1 / -1, or 0 when |(b - a) x (x - a)| is
// within 1e-10 of its terms (then the caller falls back to the reference's rounded ray cast)
__device__ __forceinline__ int orient_certain(double ax, double ay, double bx, double by, double x, double y) {
  const double ux = bx - ax, uy = by - ay, vx = x - ax, vy = y - ay;
  const double o = ux * vy - uy * vx, mag = fabs(ux * vy) + fabs(uy * vx);
  if (!(fabs(o) > 1e-10 * mag)) return 0;
  return o > 0.0 ? 1 : -1;
}

// signed crossing of the segment r -> p with the edge a -> b (+1 when p lies on the edge's left = solid side and r on
// its right, -1 the other way, 0 when they do not cross); *degenerate set when any orientation is uncertain
__device__ __forceinline__ int segment_crossing(double rx, double ry, double px, double py, const double4& e,
                                                bool* degenerate) {
  const int orr = orient_certain(e.x, e.y, e.z, e.w, rx, ry), op = orient_certain(e.x, e.y, e.z, e.w, px, py);
  if (orr == op && orr != 0) return 0;                               // same side of the edge line: no crossing
  const int oa = orient_certain(rx, ry, px, py, e.x, e.y), ob = orient_certain(rx, ry, px, py, e.z, e.w);
  if (orr == 0 || op == 0) {
    // uncertain side of the edge line: it only matters if the segment reaches the edge
    if (oa == ob && oa != 0) return 0;
    *degenerate = true;
    return 0;
  }
  if (oa == ob && oa != 0) return 0;                                 // the edge is on one side of the segment
  if (oa == 0 || ob == 0) {
    *degenerate = true;
    return 0;
  }
  return op > 0 ? 1 : -1;
}

__device__ __forceinline__ bool cell_of(const SurfView& S, double px, double py, int32_t& cid) {
  const double fx = floor(__ddiv_rn(__dsub_rn(px, S.lo_x), S.cell));
  const double fy = floor(__ddiv_rn(__dsub_rn(py, S.lo_y), S.cell));
  if (!(fx >= 0.0 && fx < (double)S.nx && fy >= 0.0 && fy < (double)S.ny)) {
    cid = -1;
    return false;
  }
  cid = (int32_t)fx * S.ny + (int32_t)fy;
  return true;
}

// ----------------------------------------------------------------------------------------------- the chord engine
struct PairGeo {
  double t0, t1, n0, n1, z, s0, s1;
};

// edge frame of a pair from the relative vertices p, q (units of h): warpbc.py:628-643
__device__ __forceinline__ bool pair_geo(double p0, double p1, double q0, double q1, PairGeo& g) {
  const double d0 = q0 - p0, d1 = q1 - p1;
  const double ll = d0 * d0 + d1 * d1;
  if (ll == 0.0) return false;
  const double ie = rsqrt(ll);             // 1 / |d|: every edge-frame quantity is a product with it
  g.t0 = d0 * ie;
  g.t1 = d1 * ie;
  g.n0 = g.t1;
  g.n1 = -g.t0;
  g.z = cross2_rn(p0, p1, q0, q1) * ie;   // the same rounded orientation as the indicator
  g.s0 = (d0 * p0 + d1 * p1) * ie;
  g.s1 = (d0 * q0 + d1 * q1) * ie;
  return true;
}

// The edge frame of the pair (row at (px, py), support h, 1/h = ih; edge a -> b).  The relative vertices are formed by
// multiplying with 1/h; where the orientation is so close to zero that the rounding of that form could decide its sign
// (|cross| <= 1e-10 of its terms), they are re-formed by division, exactly as the indicator forms them, so the sign of
// z and the winding indicator always agree.
__device__ __forceinline__ bool pair_geo_row(double px, double py, double h, double ih, const double4& e, PairGeo& g) {
  double p0 = (e.x - px) * ih, p1 = (e.y - py) * ih, q0 = (e.z - px) * ih, q1 = (e.w - py) * ih;
  const double cu = p0 * q1 - p1 * q0;
  if (!(fabs(cu) > 1e-10 * (fabs(p0 * q1) + fabs(p1 * q0)))) {
    p0 = __ddiv_rn(__dsub_rn(e.x, px), h);
    p1 = __ddiv_rn(__dsub_rn(e.y, py), h);
    q0 = __ddiv_rn(__dsub_rn(e.z, px), h);
    q1 = __ddiv_rn(__dsub_rn(e.w, py), h);
  }
  return pair_geo(p0, p1, q0, q1, g);
}

// asinh(hi/|z|) - asinh(lo/|z|) as one logarithm of positive factors (no cancellation of a + sqrt(a^2 + 1) for a < 0):
// the chord on the far side of the foot (lo >= 0), on the near side (hi <= 0), or across it; the factors are selected
// and one logarithm taken, so a warp whose lanes fall in different cases still evaluates a single log
template <typename T>
__device__ __forceinline__ T asinh_diff(T lo, T hi, T rlo, T rhi, T zz) {
  const bool far = lo >= T(0), near = hi <= T(0);
  const T num = far ? hi + rhi : (near ? rlo - lo : (hi + rhi) * (rlo - lo));
  const T den = far ? lo + rlo : (near ? rhi - hi : zz);
  return log(num / den);
}

// The MIXED route evaluates the chord angle in float.  The angle enters every channel only through M(R) * angle and
// MPsi(R) * angle with |M(R)| <= 1/2, so float rounding (<= 2.4e-7 absolute for |angle| <= pi) moves lam by < 1.2e-7.
// The logarithm stays in double: its coefficient in the monomial sums reaches 1.7e3 (w6 gradient profile at |z| -> 1),
// which would amplify float rounding to 1e-4.  The float angle keeps the sign of y = z (hi - lo), so its jump across
// z = 0 agrees with the float64 winding indicator; only where y would leave float's normal range (|y| < 2^-100) is
// the angle taken in double.
constexpr double kMixedGuardY = 0x1p-100;

template <int PREC>
__device__ __forceinline__ void special_fns(double lo, double hi, double rlo, double rhi, double z, double zz,
                                            double& dasinh, double& dang) {
  dasinh = 0.0;
  dang = 0.0;
  if (z == 0.0) return;
  const double y = z * (hi - lo), x = zz + lo * hi;
  dasinh = asinh_diff<double>(lo, hi, rlo, rhi, zz);
  if (PREC == WSB_PREC_MIXED && fabs(y) >= kMixedGuardY) {
    dang = (double)atan2f((float)y, (float)x);
    return;
  }
  dang = (y == 0.0 && x == 0.0) ? 0.0 : atan2(y, x);
}

// The chord [s0, s1] of the edge line clipped to the circle r <= R around the row, with one square root per end: an
// end outside the circle moves to -+L = -+sqrt(R^2 - z^2), where its radius is R; an end inside keeps its radius
// sqrt(s^2 + z^2).  False when the clipped chord is empty.
__device__ __forceinline__ bool clip_chord(const PairGeo& g, const double R, double& lo, double& hi, double& rlo,
                                           double& rhi, double& zz) {
  const double az = fabs(g.z);
  if (!(az < R)) return false;
  zz = g.z * g.z;
  const double LL = fmax((R - az) * (R + az), 0.0);
  const double q0 = g.s0 * g.s0 + zz, q1 = g.s1 * g.s1 + zz;
  const bool c0 = g.s0 < 0.0 && q0 > R * R, c1 = g.s1 > 0.0 && q1 > R * R;
  const double t0 = sqrt(c0 ? LL : q0), t1 = sqrt(c1 ? LL : q1);
  lo = c0 ? -t0 : g.s0;
  hi = c1 ? t1 : g.s1;
  if (!(lo < hi)) return false;
  rlo = c0 ? R : t0;
  rhi = c1 ? R : t1;
  return true;
}

// The monomial chord integrals A_n = int_lo^hi r^n ds, n < NA, by the parity recurrence: A_0 = hi - lo, A_1 through
// the asinh difference, A_n = (hi rhi^n - lo rlo^n + n z^2 A_{n-2}) / (n + 1).
template <int NA>
__device__ __forceinline__ void chord_monomials(double lo, double hi, double rlo, double rhi, double zz, double dasinh,
                                                double* A) {
  A[0] = hi - lo;
  if (NA > 1) A[1] = 0.5 * (hi * rhi - lo * rlo + zz * dasinh);
  double ph = rhi, pl = rlo;
#pragma unroll
  for (int n = 2; n < NA; ++n) {
    ph *= rhi;
    pl *= rlo;
    A[n] = (hi * ph - lo * pl + (double)n * zz * A[n - 2]) * (1.0 / (double)(n + 1));
  }
}

// The contribution of one block's chord sums S (chord angle dang) to the twelve channels (before the common 1/pi).
// acc layout: 0 lam, 1-2 m1, 3-4 G, 5-8 g1 (g(1,0)_x, g(1,0)_y, g(0,1)_x, g(0,1)_y), 9-11 m20, m11, m02 -- the
// per-edge values of the reference plan (warpbc.py:98-117, 970-991).  acc: a double* or any type whose operator[]
// gives the channel's accumulator by reference.
template <class Acc>
__device__ __forceinline__ void add_block(const PairGeo& g, const BlockSums& S, double dang, Acc acc) {
  const double Vl = g.z * S.Lreg - S.Mhat * dang;
  const double Vp = g.z * S.Preg - S.MPhat * dang;
  acc[0] += Vl;
  acc[1] += g.n0 * S.P0;
  acc[2] += g.n1 * S.P0;
  acc[3] -= g.n0 * S.W0;
  acc[4] -= g.n1 * S.W0;
  const double zW = g.z * S.W0;
  const double Y0 = g.n0 * zW + g.t0 * S.W1, Y1 = g.n1 * zW + g.t1 * S.W1;
  acc[5] += Vl - g.n0 * Y0;
  acc[6] -= g.n1 * Y0;
  acc[7] -= g.n0 * Y1;
  acc[8] += Vl - g.n1 * Y1;
  const double zP = g.z * S.P0;
  const double Z0 = g.n0 * zP + g.t0 * S.P1, Z1 = g.n1 * zP + g.t1 * S.P1;
  acc[9] += g.n0 * Z0 - Vp;
  acc[10] += g.n0 * Z1;
  acc[11] += g.n1 * Z1 - Vp;
}

// int_lo^hi pi*W(sqrt(s^2 + z^2)) ds of a quadrature kernel (KT::poly = pi*W on r <= 1), the chord [lo, hi] already
// clipped to the support: Gauss-Legendre panels on both sides of the foot s = 0, graded from it -- the first up to
// 2 max(|z|, 2^-24), then doubling.  pi*W is analytic except through r, whose branch points s = +-iz lie a panel's
// half-length away from the first panel (Bernstein parameter ~2.9: 20 nodes, 2.9^-40 ~ 3e-19 times the polynomial's
// growth on the ellipse; measured against adaptive quadrature at 1.2e-14 of the chord scale).  A panel [d, 2d]
// with d >= 2 |z| sees them at least its own length away (parameter >= 3 + sqrt 8 = 5.8: 12 nodes reach 5.8^-24 =
// 5e-19 times the growth of the degree-25 / 40 polynomial on the ellipse, ~1e3), so those take the 12-node rule.
template <class KT>
__device__ __forceinline__ double quad_chord(double lo, double hi, double z) {
  const double zz = z * z, base = fmax(fabs(z), 0x1p-24);
  double sum = 0.0;
  for (int side = 0; side < 2; ++side) {
    const double u0 = side == 0 ? fmax(-hi, 0.0) : fmax(lo, 0.0);
    const double u1 = side == 0 ? -lo : hi;
    if (!(u1 > u0)) continue;
    double d = 2.0 * base;
    for (int it = 0; it < 64 && d <= u0; ++it) d *= 2.0;
    double u = u0;
    for (int it = 0; it < 64 && u < u1; ++it) {
      const double nxt = fmin(u1, d);
      const double hc = 0.5 * (nxt - u), mc = 0.5 * (nxt + u);
      double ps = 0.0;
      if (u < 2.0 * base) {
#pragma unroll
        for (int k = 0; k < kQuadGaussChord; ++k) {
          const double x = fma(hc, kQuadCx[k], mc);
          ps = fma(kQuadCw[k], KT::poly(fmin(sqrt(fma(x, x, zz)), 1.0)), ps);
        }
      } else {
#pragma unroll
        for (int k = 0; k < kQuadGaussFar; ++k) {
          const double x = fma(hc, kQuadFx[k], mc);
          ps = fma(kQuadFw[k], KT::poly(fmin(sqrt(fma(x, x, zz)), 1.0)), ps);
        }
      }
      sum = fma(hc, ps, sum);
      if (nxt >= d) d *= 2.0;
      u = nxt;
    }
  }
  return sum;
}

// One kernel block (truncated monomial profile on r <= R_B) of one pair: the clipped chord, its monomial integrals,
// the six chord sums of the block and their contribution to the twelve channels.
template <class KT, int B, int PREC, class Acc>
__device__ __forceinline__ void block_channels(const PairGeo& g, Acc acc) {
  constexpr double R = KT::kR[B];
  constexpr int NA = KT::kNA[B];
  double lo, hi, rlo, rhi, zz;
  if (!clip_chord(g, R, lo, hi, rlo, rhi, zz)) return;
  double dasinh, dang;
  special_fns<PREC>(lo, hi, rlo, rhi, g.z, zz, dasinh, dang);
  double A[NA];
  chord_monomials<NA>(lo, hi, rlo, rhi, zz, dasinh, A);
  BlockSums S;
  KT::template sums<B>(A, rlo, rhi, S);
  add_block(g, S, dang, acc);
}

// the adjoint chord sums of one block: int s^j P ds, j = 0..3 (units of h, pi-free)
template <class KT, int B>
__device__ __forceinline__ bool block_adjoint(const PairGeo& g, AdjSums& o) {
  constexpr double R = KT::kR[B];
  constexpr int NA = KT::kNAadj[B];
  double lo, hi, rlo, rhi, zz;
  if (!clip_chord(g, R, lo, hi, rlo, rhi, zz)) return false;
  double dasinh, dang;
  special_fns<WSB_PREC_FP64>(lo, hi, rlo, rhi, g.z, zz, dasinh, dang);
  double A[NA];
  chord_monomials<NA>(lo, hi, rlo, rhi, zz, dasinh, A);
  KT::template adj<B>(A, rlo, rhi, zz, o);
  return true;
}

// per-row contraction of slot channels (src/warpSPHBoundaries/scene/fused.py:69-154): fixed slot order, + indicator *
// plane channels, physical scaling, rotation R v, R M R^T; added into the outputs
__device__ __forceinline__ void put(double* p, double v, bool assign) {
  if (assign)
    *p = v;
  else
    *p += v;
}

// The vector stores below are streaming (evict-first) stores: they serve output passes that write every row once, so
// their lines should not push the pass's own inputs out of L2.
// two consecutive outputs by one 16-byte store (p 16-byte aligned), assigned or added
__device__ __forceinline__ void put2(double* p, double a, double b, bool assign) {
  double2* q = reinterpret_cast<double2*>(p);
  if (assign) {
    __stcs(q, make_double2(a, b));
  } else {
    const double2 o = *q;
    __stcs(q, make_double2(o.x + a, o.y + b));
  }
}

// Programmatic dependent launch (sm_90 and later).  A kernel launched with the programmatic-serialization attribute
// may be scheduled before the preceding kernel of its stream has finished; pdl_wait() blocks until that kernel has
// completed and its memory operations are visible (at once when there is no such dependency), so it comes before any
// access to memory the predecessors touch.  pdl_trigger() lets the next such kernel be scheduled as this grid's
// blocks retire, which overlaps its launch and block start with this grid's tail.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// four consecutive outputs by one 32-byte store (p 32-byte aligned: st.global.cs.v4.f64, sm_100), assigned or added
__device__ __forceinline__ void put4(double* p, double a, double b, double c, double d, bool assign) {
  if (!assign) {
    const double2 o0 = reinterpret_cast<const double2*>(p)[0], o1 = reinterpret_cast<const double2*>(p)[1];
    a = o0.x + a;
    b = o0.y + b;
    c = o1.x + c;
    d = o1.y + d;
  }
  // no memory clobber: the stored values depend on any load of the same outputs above, and no other access of this
  // thread touches them, so the compiler may keep scheduling independent loads across the store
  asm volatile("st.global.cs.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(a), "d"(b), "d"(c), "d"(d));
}

// four consecutive doubles by one 32-byte read-only load (p 32-byte aligned, sm_100; memory that no thread writes
// during the kernel, so the load may be hoisted and overlapped freely)
__device__ __forceinline__ void ld4_nc(const double* p, double& a, double& b, double& c, double& d) {
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(a), "=d"(b), "=d"(c), "=d"(d) : "l"(p));
}

// a*b + c*d with its roundings fixed (one product, then one fused multiply-add): the compiler may not re-contract it,
// so every instantiation of the row finish -- any store width, any kernel pack, direct or staged -- gives the same bits
__device__ __forceinline__ double dot2(double a, double b, double c, double d) { return __fma_rn(a, b, __dmul_rn(c, d)); }

// VEC 0: scalar stores; 1: the pairs of G, m1, cov, m2 as 16-byte stores (pointers 16-byte aligned); 2: also the four
// values of cov and m2 as one 32-byte store (cov, m2 32-byte aligned), so every store of a warp writes whole sectors.
// The values are the same in every mode: the rotation to the world frame is written with explicit roundings.
template <int VEC = 0>
__device__ __forceinline__ void write_outputs(const double ch[12], double h, const double* rot, int64_t r, double* lam,
                                              double* G, double* cov, double* m1, double* m2, bool assign = false) {
  const double R00 = rot[0], R01 = rot[1], R10 = rot[2], R11 = rot[3];
  auto put_pair = [&](double* p, double a, double b) {
    if constexpr (VEC > 0) {
      put2(p, a, b, assign);
    } else {
      put(p, a, assign);
      put(p + 1, b, assign);
    }
  };
  auto put_quad = [&](double* p, double a, double b, double c, double d) {
    if constexpr (VEC > 1) {
      put4(p, a, b, c, d, assign);
    } else {
      put_pair(p, a, b);
      put_pair(p + 2, c, d);
    }
  };
  if (lam) {
    if constexpr (VEC > 0) {
      if (assign)
        __stcs(&lam[r], ch[0]);
      else
        __stcs(&lam[r], __dadd_rn(lam[r], ch[0]));
    } else {
      put(&lam[r], ch[0], assign);
    }
  }
  if (m1) {
    const double vx = __dmul_rn(h, ch[1]), vy = __dmul_rn(h, ch[2]);
    put_pair(&m1[2 * r], dot2(R00, vx, R01, vy), dot2(R10, vx, R11, vy));
  }
  if (G) {
    const double vx = __ddiv_rn(ch[3], h), vy = __ddiv_rn(ch[4], h);
    put_pair(&G[2 * r], dot2(R00, vx, R01, vy), dot2(R10, vx, R11, vy));
  }
  if (cov) {
    // R C R^T with C = [[a, b], [c, d]]: rows of C R^T first, then R times them
    const double a = ch[5], b = ch[6], c = ch[7], d = ch[8];
    const double u00 = dot2(a, R00, b, R01), u01 = dot2(a, R10, b, R11);
    const double u10 = dot2(c, R00, d, R01), u11 = dot2(c, R10, d, R11);
    put_quad(&cov[4 * r], dot2(R00, u00, R01, u10), dot2(R00, u01, R01, u11), dot2(R10, u00, R11, u10),
             dot2(R10, u01, R11, u11));
  }
  if (m2) {
    // R M R^T with M = [[xx, xy], [xy, yy]] symmetric: the off-diagonal entry written twice
    const double hh = __dmul_rn(h, h);
    const double xx = __dmul_rn(ch[9], hh), xy = __dmul_rn(ch[10], hh), yy = __dmul_rn(ch[11], hh);
    const double u00 = dot2(xx, R00, xy, R01), u01 = dot2(xx, R10, xy, R11);
    const double u10 = dot2(xy, R00, yy, R01), u11 = dot2(xy, R10, yy, R11);
    const double off = dot2(R10, u00, R11, u10);
    put_quad(&m2[4 * r], dot2(R00, u00, R01, u10), off, off, dot2(R10, u01, R11, u11));
  }
}

// dispatch a functor templated on the kernel table type
template <class F>
inline int dispatch_kernel(int kernel, F&& f) {
  switch (kernel) {
    case WSB_KERNEL_CUBIC: return f(Kern_cubic{});
    case WSB_KERNEL_W2: return f(Kern_w2{});
    case WSB_KERNEL_W4: return f(Kern_w4{});
    case WSB_KERNEL_W6: return f(Kern_w6{});
    case WSB_KERNEL_QUARTIC: return f(Kern_quartic{});
    case WSB_KERNEL_QUINTIC: return f(Kern_quintic{});
    case WSB_KERNEL_POLY6: return f(Kern_poly6{});
    case WSB_KERNEL_CONE: return f(Kern_cone{});
    case WSB_KERNEL_LW2: return f(Kern_lw2{});
    case WSB_KERNEL_LW4: return f(Kern_lw4{});
    default: return fail(WSB_ERR_UNSUPPORTED, "unknown kernel id " + std::to_string(kernel));
  }
}

SurfView view_of(const Surface* s);

}  // namespace wsb
