// The disk element: the twelve channels of solid disks (fibre bundles, solid disk bodies) at every particle,
// exactly, in float64 -- the drop-in for the reference's table lookup per (query, disk)
// (src/warpSPHBoundaries/edge/warpdisk.py:1-199, edge/disktables.py, scene/scene.py:808-905 DiskArrayRep,
// scene/fixedadj.py:199-246 fixed_disk_topology).
//
// Math (h = 1, P = pi W as truncated polynomial blocks).  The channels of the region Omega = disk cap support follow
// from the divergence theorem with the radial potentials F1(r) = int_0^r t P dt and F2(r) = int_0^r t F1 dt:
//   lam  = oint F1/r^2 (y.n)        m1 = oint F1 n         G = -oint P n
//   g1_dj = delta_dj lam - oint y_d P n_j                m2_dj = oint y_d F1 n_j - delta_dj oint F2/r^2 (y.n)
// over the boundary of Omega: the arc of the disk's circle inside the support and the arc of the support circle
// inside the disk (r = 1, n = y: closed forms in its half-angle).  In the frame whose x axis points at the disk
// centre (distance D, radius R) the disk arc is symmetric about the point nearest the particle; with u the angle from
// that point the integrand is analytic except at u = +-i acosh((D^2 + R^2) / (2 D R)), where r vanishes.  The arc is
// integrated by 24-node Gauss-Legendre panels graded from u = 0 (the first up to twice that distance, then doubling,
// as the edge quadrature of the tensile kernels) and split where r crosses a block radius; every quantity that cancels
// near the particle is formed from sin^2(u/2):  r^2 = (D - R)^2 + 4 D R sin^2(u/2), y.n = (R - D) + 2 D sin^2(u/2).
// The arc ends and the support arc's half-angle come from the same stable forms.  Near-tangent rows (|D - R| -> 0)
// take more panels (about log2(pi / |D - R|)), never fewer digits.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>
#include <type_traits>
#include <vector>

#include "common.cuh"

namespace wsb {

struct Disks {
  int device = 0;
  int64_t m = 0;
  double support_max = 0;
  int32_t nx = 0, ny = 0;
  double lo_x = 0, lo_y = 0, cell = 1;
  int64_t n_items = 0;
  int32_t* cstart = nullptr;   // [nx*ny+1]
  double4* items = nullptr;    // [n_items] (cx, cy, R, 0) of the disks that reach the cell, cell-list order
};

constexpr int kDiskThreads = 128;

// the sum over the warp's lanes, in a fixed butterfly order, on every lane
__device__ __forceinline__ double warp_allsum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// The seven non-zero channels of one disk in its aligned frame (before 1/pi): lam, m1_x, G_x, g1_xx, g1_yy, m2_xx,
// m2_yy.  D = centre distance, R = radius (h = 1), D < 1 + R.  Called by a whole warp with the same (D, R): lane q
// takes node q of every panel, the eight sums are reduced by a fixed butterfly, every lane returns the totals.
template <int KID>
__device__ void disk_pair(double D, double R, int lane, double out[7]) {
  double lam = 0.0, m1 = 0.0, G = 0.0, gxx = 0.0, gyy = 0.0, mxx = 0.0, myy = 0.0, SF = 0.0;
  const double dm = D - R;
  // the arc of the disk's circle inside the support: u in [0, U] (and its mirror image)
  if (fabs(dm) < 1.0) {   // (D = 0: a concentric circle, one panel: the singularity distance is infinite)
    const double U = D + R <= 1.0 ? 0.5 * kTwoPi : 2.0 * asin(fmin(1.0, sqrt((1.0 - dm * dm) / (4.0 * D * R))));
    const double x = 0.5 * dm * dm / (D * R);                  // acosh(1 + x): the distance of the singularity
    const double base = fmax(log1p(x + sqrt(x * (x + 2.0))), 0x1p-24);
    double radii[kDiskMaxKnots], knots[kDiskMaxKnots];
    const int nr = disk_knots<KID>(radii);
    int nk = 0;
    for (int k = 0; k < nr; ++k) {
      const double Rb = radii[k];
      if (fabs(dm) < Rb && Rb < D + R) {
        const double kn = 2.0 * asin(fmin(1.0, sqrt((Rb * Rb - dm * dm) / (4.0 * D * R))));
        if (kn > 0.0 && kn < U) knots[nk++] = kn;
      }
    }
    for (int a = 1; a < nk; ++a)                                   // ascending (at most kDiskMaxKnots knots)
      for (int b = a; b > 0 && knots[b] < knots[b - 1]; --b) {
        const double t = knots[b];
        knots[b] = knots[b - 1];
        knots[b - 1] = t;
      }
    auto node = [&](double uu, double wq) {
      double sh, ch;
      sincos(0.5 * uu, &sh, &ch);                                  // one half-angle evaluation per node
      const double s2 = sh * sh, su = 2.0 * sh * ch, cu = fma(-2.0, s2, 1.0);
      const double yx = fma(2.0 * R, s2, dm), yy = R * su, nx = -cu, ny = su;
      const double yn = fma(2.0 * D, s2, -dm);
      const double r = sqrt(fma(4.0 * D * R, s2, dm * dm));
      double P, Fl, F2l;
      disk_profile<KID>(r, 1.0 / (r * r), P, Fl, F2l);
      const double F1 = Fl * r * r;
      const double w = 2.0 * R * wq;
      lam = fma(w * Fl, yn, lam);
      m1 = fma(w * F1, nx, m1);
      G = fma(-w * P, nx, G);
      gxx = fma(-w * P * yx, nx, gxx);
      gyy = fma(-w * P * yy, ny, gyy);
      mxx = fma(w * F1 * yx, nx, mxx);
      myy = fma(w * F1 * yy, ny, myy);
      SF = fma(w * F2l, yn, SF);
    };
    // the panel after u: up to the doubling bound d or the next knot, whichever is first
    double d = 2.0 * base;
    int ki = 0;
    auto next_panel = [&](double u) {
      double nxt = fmin(U, d);
      while (ki < nk && knots[ki] <= u) ++ki;
      if (ki < nk && knots[ki] < nxt) nxt = knots[ki];
      if (nxt >= d) d *= 2.0;
      return nxt;
    };
    // panels next to the nearest point (start below 2 * base) take 24 nodes on lanes 0-23; farther panels, whose
    // singularities lie at least their own length away (Bernstein parameter >= 5.8), 12 nodes, two panels at a time
    // (lanes 0-11 and 12-23)
    double u = 0.0;
    for (int it = 0; it < 160 && u < U; ++it) {
      const double a0 = u, a1 = next_panel(u);
      if (a0 < 2.0 * base) {
        const double hc = 0.5 * (a1 - a0), mc = 0.5 * (a1 + a0);
        if (lane < kQuadGauss) node(fma(hc, kQuadGx[lane], mc), hc * kQuadGw[lane]);
        u = a1;
        continue;
      }
      const double b1 = a1 < U ? next_panel(a1) : a1;
      const bool second = lane >= kQuadGaussFar;
      const double lo = second ? a1 : a0, hi = second ? b1 : a1;
      const int q = second ? lane - kQuadGaussFar : lane;
      if (q < kQuadGaussFar && hi > lo) {
        const double hc = 0.5 * (hi - lo), mc = 0.5 * (hi + lo);
        node(fma(hc, kQuadFx[q], mc), hc * kQuadFw[q]);
      }
      u = b1;
    }
  }
  lam = warp_allsum(lam);
  m1 = warp_allsum(m1);
  G = warp_allsum(G);
  gxx = warp_allsum(gxx);
  gyy = warp_allsum(gyy);
  mxx = warp_allsum(mxx);
  myy = warp_allsum(myy);
  SF = warp_allsum(SF);
  // the arc of the support circle inside the disk: |phi| < beta
  double beta = -1.0;
  if (R >= D + 1.0)
    beta = 0.5 * kTwoPi;
  else if (fabs(D - 1.0) < R && D > 0.0)
    beta = 2.0 * asin(fmin(1.0, sqrt((R * R - (D - 1.0) * (D - 1.0)) / (4.0 * D))));
  if (beta > 0.0) {
    double P1, Fl1, F2l1;
    disk_profile<KID>(1.0, 1.0, P1, Fl1, F2l1);
    const double sb = sin(beta), s2b = sin(2.0 * beta);
    const double cxx = beta + 0.5 * s2b, cyy = beta - 0.5 * s2b;
    lam += 2.0 * beta * Fl1;
    m1 += 2.0 * sb * Fl1;
    G -= 2.0 * sb * P1;
    gxx -= P1 * cxx;
    gyy -= P1 * cyy;
    mxx += Fl1 * cxx;
    myy += Fl1 * cyy;
    SF += 2.0 * beta * F2l1;
  }
  out[0] = lam;
  out[1] = m1;
  out[2] = G;
  out[3] = gxx + lam;
  out[4] = gyy + lam;
  out[5] = mxx - SF;
  out[6] = myy - SF;
}

// the body-frame position of particle i and its cell (false outside the grid or outside `allowed`)
__device__ __forceinline__ bool disk_row(const double* __restrict__ pos, const int32_t* __restrict__ allowed,
                                         const double* __restrict__ pose, int64_t i, int32_t nx, int32_t ny,
                                         double lo_x, double lo_y, double cell, double& lx, double& ly, int32_t& cid) {
  if (allowed && allowed[i] == 0) return false;
  to_local_rn(pos[2 * i], pos[2 * i + 1], pose[0], pose[1], pose[2], pose[3], lx, ly);
  const double fx = floor((lx - lo_x) / cell), fy = floor((ly - lo_y) / cell);
  if (!(fx >= 0.0 && fx < (double)nx && fy >= 0.0 && fy < (double)ny)) return false;
  cid = (int32_t)fx * ny + (int32_t)fy;
  return true;
}

// Pass 1, one thread per particle: a particle that reaches no disk gets its zero channels (when the call assigns);
// the others are appended to the work list (warp-aggregated).
__global__ void __launch_bounds__(kDiskThreads) k_disk_rows(const int32_t* __restrict__ cstart,
                                                           const double4* __restrict__ items, int32_t nx,
                                                           int32_t ny, double lo_x, double lo_y, double cell,
                                                           const double* __restrict__ pos,
                                                           const double* __restrict__ sup,
                                                           const int32_t* __restrict__ allowed, int64_t n,
                                                           const double* __restrict__ pose, bool assign,
                                                           int32_t* __restrict__ work, int32_t* __restrict__ nwork,
                                                           double* lam, double* G, double* cov, double* m1,
                                                           double* m2) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  bool has = false;
  if (i < n) {
    double lx, ly;
    int32_t cid;
    if (disk_row(pos, allowed, pose, i, nx, ny, lo_x, lo_y, cell, lx, ly, cid)) {
      const double ih = 1.0 / sup[i];
      for (int32_t k = cstart[cid]; k < cstart[cid + 1] && !has; ++k) {
        const double4 e = items[k];
        const double vx = (e.x - lx) * ih, vy = (e.y - ly) * ih;
        has = sqrt(vx * vx + vy * vy) < 1.0 + e.z * ih;
      }
    }
    if (!has && assign) {
      double acc[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
      const double c = pose[2], s = pose[3];
      const double rot[4] = {c, -s, s, c};
      write_outputs(acc, sup[i], rot, i, lam, G, cov, m1, m2, true);
    }
  }
  const unsigned ballot = __ballot_sync(0xffffffffu, has);
  const int lane = threadIdx.x & 31;
  int base = 0;
  if (lane == 0 && ballot) base = atomicAdd(nwork, __popc(ballot));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (has) work[base + __popc(ballot & ((1u << lane) - 1))] = (int32_t)i;
}

// Pass 2, one warp per listed particle (grid-stride): every disk of the particle's cell within reach, in cell-list
// order, integrated by the whole warp, rotated from its aligned frame and summed; lane 0 scales, rotates to the world
// frame and writes.  Each particle is one warp's work in a fixed order: the result does not depend on the list order.
template <int KID>
__global__ void __launch_bounds__(kDiskThreads, 4) k_disk_warp(const int32_t* __restrict__ cstart,
                                                           const double4* __restrict__ items, int32_t nx,
                                                           int32_t ny, double lo_x, double lo_y, double cell,
                                                           const double* __restrict__ pos,
                                                           const double* __restrict__ sup,
                                                           const int32_t* __restrict__ work,
                                                           const int32_t* __restrict__ nwork_p,
                                                           const double* __restrict__ pose, bool assign, double* lam,
                                                           double* G, double* cov, double* m1, double* m2) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (kDiskThreads / 32);
  const int64_t nwork = *nwork_p;
  for (int64_t j = (int64_t)blockIdx.x * (kDiskThreads / 32) + threadIdx.x / 32; j < nwork; j += warps) {
    const int64_t i = work[j];
    double lx, ly;
    int32_t cid = 0;
    disk_row(pos, nullptr, pose, i, nx, ny, lo_x, lo_y, cell, lx, ly, cid);   // listed: inside the grid
    const double h = sup[i], ih = 1.0 / h;
    double acc[12];
#pragma unroll
    for (int c = 0; c < 12; ++c) acc[c] = 0.0;
    for (int32_t k = cstart[cid]; k < cstart[cid + 1]; ++k) {
      const double4 e = items[k];
      const double vx = (e.x - lx) * ih, vy = (e.y - ly) * ih, R = e.z * ih;
      const double D = sqrt(vx * vx + vy * vy);
      if (!(D < 1.0 + R)) continue;
      double o[7];
      disk_pair<KID>(D, R, lane, o);
      const double ca = D > 0.0 ? vx / D : 1.0, sa = D > 0.0 ? vy / D : 0.0;
      acc[0] += o[0];
      acc[1] += ca * o[1];
      acc[2] += sa * o[1];
      acc[3] += ca * o[2];
      acc[4] += sa * o[2];
      const double dg = o[3] - o[4], dmm = o[5] - o[6];
      acc[5] += ca * ca * o[3] + sa * sa * o[4];
      acc[6] += ca * sa * dg;
      acc[7] += ca * sa * dg;
      acc[8] += sa * sa * o[3] + ca * ca * o[4];
      acc[9] += ca * ca * o[5] + sa * sa * o[6];
      acc[10] += ca * sa * dmm;
      acc[11] += sa * sa * o[5] + ca * ca * o[6];
    }
    if (lane == 0) {
#pragma unroll
      for (int c = 0; c < 12; ++c) acc[c] *= kInvPi;
      const double c = pose[2], s = pose[3];
      const double rot[4] = {c, -s, s, c};
      write_outputs(acc, h, rot, i, lam, G, cov, m1, m2, assign);
    }
  }
}

// ------------------------------------------------------------------------------------------------ detector inputs
// The cone area and the direction extreme of solid disks (src/warpSPHBoundaries/scene/fused.py:310-475, 741-835):
// closed forms per (particle, disk), one thread per particle over the disks of its cell.

// the angle in [-pi, pi)
__device__ __forceinline__ double disk_wrap(double a) {
  const double r = a + 0.5 * kTwoPi;
  return r - kTwoPi * floor(r / kTwoPi) - 0.5 * kTwoPi;
}

// int t^2 dphi along a ray family through the disk: t = D cos(phi) -+ q, q = sqrt(R^2 - D^2 sin^2(phi)), gives
// t^2 = R^2 + D^2 cos(2 phi) -+ 2 D cos(phi) q, whose antiderivative is R^2 phi + s c -+ (s q + R^2 asin(s / R))
// (s = D sin(phi), c = D cos(phi)).  q is formed as sqrt((R - D)(R + D) + c^2) and asin(s / R) as atan2(s, q): near
// the tangent ray s / R -> 1, where asin of a rounded quotient loses half the digits, both stay accurate.
__device__ __forceinline__ double disk_q(double D, double R, double c) {
  return sqrt(fmax(fma(c, c, (R - D) * (R + D)), 0.0));
}

__device__ __forceinline__ double disk_ray_antideriv(double D, double R, double phi, double sign) {
  double sp, cp;
  sincos(phi, &sp, &cp);
  const double s = D * sp, c = D * cp, q = disk_q(D, R, c);
  return R * R * phi + s * c + sign * (s * q + R * R * atan2(s, q));
}

// The area of disk cap unit ball swept by the rays from the particle at angles [0, psi] (psi in [0, pi]) from the
// direction of the centre (distance D, radius R, support 1): 1/2 int (min(t_far, 1)^2 - min(max(t_near, 0), 1)^2)
// dphi, in closed form on the pieces between the tangent ray asin(R / D) and the rays through the crossings of the
// disk's circle with the support circle (where a clip switches on or off).
__device__ double disk_sweep(double D, double R, double psi) {
  double c[2];
  int nc = 0;
  if (D >= R && D > 0.0) {   // (D = R: the particle on the circle; the far end reaches the particle at pi/2)
    const double a = atan2(R, sqrt((D - R) * (D + R)));   // the tangent ray
    if (a > 0.0 && a < psi) c[nc++] = a;
  }
  if (D > 1e-12) {
    const double arg = (D * D + 1.0 - R * R) / (2.0 * D);
    if (fabs(arg) <= 1.0) {
      const double a = acos(arg);
      if (a > 0.0 && a < psi) c[nc++] = a;
    }
  }
  if (nc == 2 && c[1] < c[0]) {
    const double tmp = c[0];
    c[0] = c[1];
    c[1] = tmp;
  }
  double total = 0.0, lo = 0.0;
  for (int k = 0; k <= nc; ++k) {
    const double hi = k < nc ? c[k] : psi;
    if (hi > lo) {
      const double m = 0.5 * (lo + hi), sm = D * sin(m);
      if (fabs(sm) < R) {
        const double cm = D * cos(m), q = disk_q(D, R, cm), t1 = cm - q, t2 = cm + q;
        if (t2 > 0.0) {
          const double far = t2 >= 1.0 ? hi - lo : disk_ray_antideriv(D, R, hi, 1.0) - disk_ray_antideriv(D, R, lo, 1.0);
          const double near = t1 >= 1.0 ? hi - lo
                              : t1 > 0.0 ? disk_ray_antideriv(D, R, hi, -1.0) - disk_ray_antideriv(D, R, lo, -1.0)
                                         : 0.0;
          total += 0.5 * (far - near);
        }
      }
    }
    lo = hi;
  }
  return total;
}

// the swept area at any real angle: odd in the angle, and each full turn adds the whole area
__device__ __forceinline__ double disk_sweep_any(double D, double R, double psi) {
  const double p0 = disk_wrap(psi);
  const double k = floor((psi - p0) / kTwoPi + 0.5);
  double v = disk_sweep(D, R, fabs(p0));
  if (p0 < 0.0) v = -v;
  if (k != 0.0) v += k * 2.0 * disk_sweep(D, R, 0.5 * kTwoPi);
  return v;
}

// per particle: area[i] += the area of the disks' solid cap disk(x, H) cap wedge(x, axis, half_angle) and
// area[n + i] += the full-disk area, summed over the disks of its cell within reach
__global__ void __launch_bounds__(kDiskThreads) k_disk_cone(const int32_t* __restrict__ cstart,
                                                           const double4* __restrict__ items, int32_t nx, int32_t ny,
                                                           double lo_x, double lo_y, double cell,
                                                           const double* __restrict__ pos,
                                                           const double* __restrict__ sup,
                                                           const int32_t* __restrict__ allowed, int64_t n,
                                                           const double* __restrict__ pose,
                                                           const double* __restrict__ axes, double half_angle,
                                                           double* __restrict__ area) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double lx, ly;
  int32_t cid;
  if (!disk_row(pos, allowed, pose, i, nx, ny, lo_x, lo_y, cell, lx, ly, cid)) return;
  const double H = sup[i], ih = 1.0 / H;
  const double ax = axes[2 * i], ay = axes[2 * i + 1], pc = pose[2], ps = pose[3];
  const double th = atan2(-ps * ax + pc * ay, pc * ax + ps * ay);     // the world axis in the body frame
  const bool wedge = half_angle < 0.5 * kTwoPi;
  double a_wedge = 0.0, a_full = 0.0;
  for (int32_t k = cstart[cid]; k < cstart[cid + 1]; ++k) {
    const double4 e = items[k];
    const double vx = (e.x - lx) * ih, vy = (e.y - ly) * ih, R = e.z * ih;
    const double D = sqrt(vx * vx + vy * vy);
    if (!(D < 1.0 + R)) continue;
    const double full = 2.0 * disk_sweep(D, R, 0.5 * kTwoPi);
    a_full += full;
    if (wedge) {
      const double g = disk_wrap(th - atan2(vy, vx));
      a_wedge += disk_sweep_any(D, R, g + half_angle) - disk_sweep_any(D, R, g - half_angle);
    } else {
      a_wedge += full;
    }
  }
  area[i] += a_wedge * H * H;
  area[n + i] += a_full * H * H;
}

// per particle: out[i] = max(out[i], the largest |cos| between its world vector and a direction towards a disk point
// within its support).  The directions to the points of one disk within the support form the interval [-b, b] about
// the centre direction: b = asin(R / d) when the tangent points lie inside the support, else the angle at which the
// disk's circle meets the support circle; with psi the angle between the line of the vector and the centre direction
// the extreme is cos(max(0, psi - b)); a particle inside the disk sees it in every direction.
__global__ void __launch_bounds__(kDiskThreads) k_disk_dir(const int32_t* __restrict__ cstart,
                                                          const double4* __restrict__ items, int32_t nx, int32_t ny,
                                                          double lo_x, double lo_y, double cell,
                                                          const double* __restrict__ pos,
                                                          const double* __restrict__ sup,
                                                          const int32_t* __restrict__ allowed, int64_t n,
                                                          const double* __restrict__ pose,
                                                          const double* __restrict__ vecs, double* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double lx, ly;
  int32_t cid;
  if (!disk_row(pos, allowed, pose, i, nx, ny, lo_x, lo_y, cell, lx, ly, cid)) return;
  const double wx = vecs[2 * i], wy = vecs[2 * i + 1], pc = pose[2], ps = pose[3];
  const double bx = pc * wx + ps * wy, by = -ps * wx + pc * wy;      // R^T w
  const double nb = sqrt(bx * bx + by * by);
  if (!(nb > 0.0)) return;
  const double H = sup[i];
  double best = 0.0;
  for (int32_t k = cstart[cid]; k < cstart[cid + 1] && best < 1.0; ++k) {
    const double4 e = items[k];
    const double cx = e.x - lx, cy = e.y - ly, R = e.z;
    const double d = sqrt(cx * cx + cy * cy);
    double f = 0.0;
    if (d <= R) {
      f = 1.0;
    } else if (d - R < H) {
      const double b = d * d - R * R <= H * H ? asin(fmin(R / d, 1.0))
                                              : acos(fmin(fmax((d * d + H * H - R * R) / (2.0 * d * H), -1.0), 1.0));
      const double psi = acos(fmin(fabs(cx * bx + cy * by) / (d * nb), 1.0));
      f = psi <= b ? 1.0 : cos(psi - b);
    }
    best = fmax(best, f);
  }
  out[i] = fmax(out[i], best);
}

}  // namespace wsb

using namespace wsb;

extern "C" int wsb_disks_create(const double* centres, const double* radii, int64_t m, double support_max, int device,
                                wsb_disks** out) {
  if (!out) return fail(WSB_ERR_ARG, "wsb_disks_create: NULL output handle");
  *out = nullptr;
  if (m < 0 || m > (int64_t)INT32_MAX) return fail(WSB_ERR_ARG, "wsb_disks_create: disk count out of range");
  if (m > 0 && (!centres || !radii)) return fail(WSB_ERR_ARG, "wsb_disks_create: NULL array");
  if (!(support_max > 0.0) || !std::isfinite(support_max))
    return fail(WSB_ERR_ARG, "wsb_disks_create: support_max must be positive and finite");
  double lo_x = 0, lo_y = 0, hi_x = 0, hi_y = 0;
  for (int64_t k = 0; k < m; ++k) {
    const double cx = centres[2 * k], cy = centres[2 * k + 1], R = radii[k];
    if (!std::isfinite(cx) || !std::isfinite(cy) || !(R > 0.0) || !std::isfinite(R))
      return fail(WSB_ERR_ARG, "wsb_disks_create: disk " + std::to_string(k) + " has a non-finite centre or a "
                                   "radius that is not positive");
    if (k == 0 || cx - R < lo_x) lo_x = cx - R;
    if (k == 0 || cy - R < lo_y) lo_y = cy - R;
    if (k == 0 || cx + R > hi_x) hi_x = cx + R;
    if (k == 0 || cy + R > hi_y) hi_y = cy + R;
  }
  Disks* d = new Disks();
  d->device = device;
  d->m = m;
  d->support_max = support_max;
  // a cell grid over the disks' boxes grown by one support; a disk is listed in every cell whose box comes within
  // R + support_max of its centre (interior cells included: a particle deep inside still has the disk's plane terms)
  const double s = support_max;
  double cell = s;
  lo_x -= s;
  lo_y -= s;
  hi_x += s;
  hi_y += s;
  auto dims = [&](double c, int64_t& gx, int64_t& gy) {
    gx = std::max<int64_t>(1, (int64_t)std::ceil((hi_x - lo_x) / c));
    gy = std::max<int64_t>(1, (int64_t)std::ceil((hi_y - lo_y) / c));
  };
  int64_t gx = 1, gy = 1;
  if (m > 0) {
    dims(cell, gx, gy);
    while (gx * gy > ((int64_t)1 << 22)) {   // at most 4M cells: a coarser grid only lengthens the cell lists
      cell *= 2.0;
      dims(cell, gx, gy);
    }
  }
  d->nx = (int32_t)gx;
  d->ny = (int32_t)gy;
  d->lo_x = lo_x;
  d->lo_y = lo_y;
  d->cell = cell;
  std::vector<int32_t> counts((size_t)(gx * gy) + 1, 0);
  auto each = [&](auto&& f) {
    for (int64_t k = 0; k < m; ++k) {
      const double cx = centres[2 * k], cy = centres[2 * k + 1], reach = radii[k] + s;
      const int64_t x0 = std::max<int64_t>(0, (int64_t)std::floor((cx - reach - lo_x) / cell));
      const int64_t x1 = std::min<int64_t>(gx - 1, (int64_t)std::floor((cx + reach - lo_x) / cell));
      const int64_t y0 = std::max<int64_t>(0, (int64_t)std::floor((cy - reach - lo_y) / cell));
      const int64_t y1 = std::min<int64_t>(gy - 1, (int64_t)std::floor((cy + reach - lo_y) / cell));
      for (int64_t ix = x0; ix <= x1; ++ix)
        for (int64_t iy = y0; iy <= y1; ++iy) {
          const double bx0 = lo_x + ix * cell, by0 = lo_y + iy * cell;
          const double ex = std::max({bx0 - cx, 0.0, cx - (bx0 + cell)});
          const double ey = std::max({by0 - cy, 0.0, cy - (by0 + cell)});
          if (std::sqrt(ex * ex + ey * ey) < reach * (1.0 + 1e-12)) f(ix * gy + iy, k);
        }
    }
  };
  each([&](int64_t c, int64_t) { ++counts[(size_t)c + 1]; });
  for (size_t c = 1; c < counts.size(); ++c) counts[c] += counts[c - 1];
  d->n_items = counts.back();
  std::vector<double4> items((size_t)std::max<int64_t>(d->n_items, 1));
  std::vector<int32_t> fill(counts.begin(), counts.end() - 1);
  each([&](int64_t c, int64_t k) {
    items[(size_t)fill[(size_t)c]++] = make_double4(centres[2 * k], centres[2 * k + 1], radii[k], 0.0);
  });
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaMalloc(&d->cstart, sizeof(int32_t) * counts.size());
  if (e == cudaSuccess) e = cudaMalloc(&d->items, sizeof(double4) * items.size());
  if (e == cudaSuccess)
    e = cudaMemcpy(d->cstart, counts.data(), sizeof(int32_t) * counts.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d->items, items.data(), sizeof(double4) * items.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(d->cstart);
    cudaFree(d->items);
    delete d;
    return cuda_fail(e, "wsb_disks_create");
  }
  *out = reinterpret_cast<wsb_disks*>(d);
  return WSB_OK;
}

extern "C" int wsb_disks_destroy(wsb_disks* d_) {
  Disks* d = reinterpret_cast<Disks*>(d_);
  if (!d) return WSB_OK;
  cudaSetDevice(d->device);
  cudaFree(d->cstart);
  cudaFree(d->items);
  delete d;
  return WSB_OK;
}

static inline size_t disk_align256(size_t x) { return (x + 255) & ~(size_t)255; }

extern "C" size_t wsb_disk_workspace_size(const wsb_disks* d, int64_t n) {
  if (!d || n < 0) return 0;
  return disk_align256(sizeof(int32_t) * (size_t)std::max<int64_t>(n, 1)) + 256;
}

extern "C" int wsb_disk_aggregate(const wsb_disks* d_, int kernel, const double* pos, const double* sup,
                                  const int32_t* allowed, int64_t n, const double* pose, int out_mask, double* lam,
                                  double* G, double* cov, double* m1, double* m2, void* workspace,
                                  size_t workspace_bytes, void* stream) {
  const Disks* d = reinterpret_cast<const Disks*>(d_);
  if (!d) return fail(WSB_ERR_ARG, "wsb_disk_aggregate: NULL disks");
  if (kernel < 0 || kernel >= kNumKernels)
    return fail(WSB_ERR_UNSUPPORTED, "wsb_disk_aggregate: kernel id " + std::to_string(kernel) +
                                         " has no disk element (exact-table kernels only)");
  if (n < 0 || n > (int64_t)INT32_MAX) return fail(WSB_ERR_ARG, "wsb_disk_aggregate: row count out of range");
  if (n == 0) return WSB_OK;
  if (!pos || !sup || !pose) return fail(WSB_ERR_ARG, "wsb_disk_aggregate: NULL array");
  const size_t need = wsb_disk_workspace_size(d_, n);
  if (!workspace || workspace_bytes < need)
    return fail(WSB_ERR_SIZE, "wsb_disk_aggregate: workspace of " + std::to_string(workspace_bytes) +
                                  " bytes, need " + std::to_string(need));
  WSB_CUDA(cudaSetDevice(d->device));
  cudaStream_t st = (cudaStream_t)stream;
  const bool assign = (out_mask & WSB_OUT_ASSIGN) != 0;
  double* L = (out_mask & WSB_OUT_LAM) ? lam : nullptr;
  double* Gp = (out_mask & WSB_OUT_G) ? G : nullptr;
  double* C = (out_mask & WSB_OUT_COV) ? cov : nullptr;
  double* M1 = (out_mask & WSB_OUT_M1) ? m1 : nullptr;
  double* M2 = (out_mask & WSB_OUT_M2) ? m2 : nullptr;
  int32_t* work = static_cast<int32_t*>(workspace);
  int32_t* nwork = reinterpret_cast<int32_t*>(static_cast<char*>(workspace) + need - 256);
  WSB_CUDA(cudaMemsetAsync(nwork, 0, sizeof(int32_t), st));
  const unsigned grid = (unsigned)((n + kDiskThreads - 1) / kDiskThreads);
  k_disk_rows<<<grid, kDiskThreads, 0, st>>>(d->cstart, d->items, d->nx, d->ny, d->lo_x, d->lo_y, d->cell, pos, sup,
                                             allowed, n, pose, assign, work, nwork, L, Gp, C, M1, M2);
  // warps per listed particle, grid-stride: at most 16 blocks of 4 warps per SM, never more warps than particles
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d->device);
  const int64_t wgrid = std::min<int64_t>((n + 3) / 4, (int64_t)sms * 16);
  auto launch = [&](auto kid) {
    k_disk_warp<decltype(kid)::value><<<(unsigned)wgrid, kDiskThreads, 0, st>>>(
        d->cstart, d->items, d->nx, d->ny, d->lo_x, d->lo_y, d->cell, pos, sup, work, nwork, pose, assign, L, Gp, C,
        M1, M2);
  };
  switch (kernel) {
    case 0: launch(std::integral_constant<int, 0>{}); break;
    case 1: launch(std::integral_constant<int, 1>{}); break;
    case 2: launch(std::integral_constant<int, 2>{}); break;
    case 3: launch(std::integral_constant<int, 3>{}); break;
    case 4: launch(std::integral_constant<int, 4>{}); break;
    case 5: launch(std::integral_constant<int, 5>{}); break;
    case 6: launch(std::integral_constant<int, 6>{}); break;
    case 7: launch(std::integral_constant<int, 7>{}); break;
    case 8: launch(std::integral_constant<int, 8>{}); break;
    case 9: launch(std::integral_constant<int, 9>{}); break;
    default: return fail(WSB_ERR_UNSUPPORTED, "wsb_disk_aggregate: unknown kernel id");
  }
  WSB_CUDA(cudaGetLastError());
  return WSB_OK;
}

extern "C" int wsb_disk_cone_area(const wsb_disks* d_, const double* pos, const double* sup, const int32_t* allowed,
                                  int64_t n, const double* pose, const double* axes, double half_angle, double* area,
                                  void* stream) {
  const Disks* d = reinterpret_cast<const Disks*>(d_);
  if (!d) return fail(WSB_ERR_ARG, "wsb_disk_cone_area: NULL disks");
  if (n < 0 || n > (int64_t)INT32_MAX) return fail(WSB_ERR_ARG, "wsb_disk_cone_area: row count out of range");
  if (!(half_angle >= 0.0) || !std::isfinite(half_angle))
    return fail(WSB_ERR_ARG, "wsb_disk_cone_area: the half angle must be finite and >= 0");
  if (n == 0) return WSB_OK;
  if (!pos || !sup || !pose || !axes || !area) return fail(WSB_ERR_ARG, "wsb_disk_cone_area: NULL array");
  WSB_CUDA(cudaSetDevice(d->device));
  k_disk_cone<<<(unsigned)((n + kDiskThreads - 1) / kDiskThreads), kDiskThreads, 0, (cudaStream_t)stream>>>(
      d->cstart, d->items, d->nx, d->ny, d->lo_x, d->lo_y, d->cell, pos, sup, allowed, n, pose, axes, half_angle, area);
  WSB_CUDA(cudaGetLastError());
  return WSB_OK;
}

extern "C" int wsb_disk_dir_extreme(const wsb_disks* d_, const double* pos, const double* sup, const int32_t* allowed,
                                    int64_t n, const double* pose, const double* vecs, double* out, void* stream) {
  const Disks* d = reinterpret_cast<const Disks*>(d_);
  if (!d) return fail(WSB_ERR_ARG, "wsb_disk_dir_extreme: NULL disks");
  if (n < 0 || n > (int64_t)INT32_MAX) return fail(WSB_ERR_ARG, "wsb_disk_dir_extreme: row count out of range");
  if (n == 0) return WSB_OK;
  if (!pos || !sup || !pose || !vecs || !out) return fail(WSB_ERR_ARG, "wsb_disk_dir_extreme: NULL array");
  WSB_CUDA(cudaSetDevice(d->device));
  k_disk_dir<<<(unsigned)((n + kDiskThreads - 1) / kDiskThreads), kDiskThreads, 0, (cudaStream_t)stream>>>(
      d->cstart, d->items, d->nx, d->ny, d->lo_x, d->lo_y, d->cell, pos, sup, allowed, n, pose, vecs, out);
  WSB_CUDA(cudaGetLastError());
  return WSB_OK;
}
