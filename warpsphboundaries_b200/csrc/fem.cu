// Finite-element pair weights: for every (query, P1 triangle) pair the kernel-weighted integrals of the triangle's
// three barycentric (hat) functions and of their products with the kernel gradient -- the drop-in for the reference's
// pair kernel of its P1 boundary-operation interface (src/warpSPHBoundaries/edge/warpbc.py:226-345 _pair_weights_kernel,
// :486-510 pair_weights; called from scene/boundaryOps.py:213).
//
//   w_k = int_T W_h(x' - x) phi_k(x') dx'          G_k = int_T grad_x W_h(x' - x) phi_k(x') dx'
//
// With y = (x' - x) / h and phi_k(x + h y) = l_k + g_k . y (the barycentric functions in the query's frame, from the
// vertices in the element's own order) both follow from the triangle's channels: w_k = l_k lam + g_k . m1 and
// G_kj = (l_k G_j + sum_d g_kd g1_dj) / h, where lam, m1, G, g1 are the exact closed forms of the triangle as a
// polygon (three edges and the winding indicator).  A triangle far from the query relative to its size, over which the
// kernel has no kink (or one no larger than 0.05 h), is integrated instead by the reference's far-field rule -- 8 x 8
// Gauss-Legendre on the collapsed square, the same nodes and the same sums -- where the closed form would cancel.
#include <cmath>
#include <string>
#include <type_traits>

#include "common.cuh"

namespace wsb {

constexpr int kFemThreads = 128;
constexpr double kFemFarRatio = 1.0;   // |centroid - x| >= ratio * longest edge
constexpr double kFemTiny = 0.05;      // elements this small (units of h) take the far-field rule across a kink

template <class KT, int B>
__device__ __forceinline__ void fem_blocks(const PairGeo& g, double* acc) {
  if constexpr (B < KT::kBlocks) {
    block_channels<KT, B, WSB_PREC_FP64>(g, acc);
    fem_blocks<KT, B + 1>(g, acc);
  }
}

// a block radius of the kernel strictly between the element's nearest and farthest distance (a kink inside it)
template <class KT, int B>
__device__ __forceinline__ bool fem_straddle(double rmin, double rmax) {
  if constexpr (B < KT::kBlocks) {
    constexpr double R = KT::kR[B];
    return (rmin < R && R < rmax) || fem_straddle<KT, B + 1>(rmin, rmax);
  } else {
    return false;
  }
}

template <class KT>
__global__ void __launch_bounds__(kFemThreads) k_pair_weights(const int32_t* __restrict__ pair_q,
                                                             const int32_t* __restrict__ pair_e, int64_t n_pairs,
                                                             const double* __restrict__ pos,
                                                             const double* __restrict__ sup, int64_t n_pos,
                                                             const double* __restrict__ verts, int64_t n_verts,
                                                             const int32_t* __restrict__ elems, int64_t n_elems,
                                                             double* __restrict__ w, double* __restrict__ G,
                                                             int32_t* __restrict__ bad) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n_pairs) return;
  const int64_t q = pair_q[t], e = pair_e[t];
  // an index outside its array: the pair's outputs are NaN and the error word is set, nothing out of range is read
  bool in_range = q >= 0 && q < n_pos && e >= 0 && e < n_elems;
  if (in_range) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int32_t v = elems[3 * e + k];
      in_range = in_range && v >= 0 && v < n_verts;
    }
  }
  if (!in_range) {
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      w[3 * t + k] = nan;
      G[6 * t + 2 * k] = nan;
      G[6 * t + 2 * k + 1] = nan;
    }
    atomicExch(bad, 1);
    return;
  }
  const double h = sup[q], x0 = pos[2 * q], x1 = pos[2 * q + 1];
  double r[3][2];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int32_t v = elems[3 * e + k];
    r[k][0] = (verts[2 * v] - x0) / h;
    r[k][1] = (verts[2 * v + 1] - x1) / h;
  }
  // barycentric functions l_k + g_k . y from the element's own vertex order (orientation independent)
  const double d2 = (r[1][0] - r[0][0]) * (r[2][1] - r[0][1]) - (r[1][1] - r[0][1]) * (r[2][0] - r[0][0]);
  double l[3], gx[3], gy[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double* a = r[(k + 1) % 3];
    const double* b = r[(k + 2) % 3];
    l[k] = (a[0] * b[1] - a[1] * b[0]) / d2;
    gx[k] = (a[1] - b[1]) / d2;
    gy[k] = (b[0] - a[0]) / d2;
  }
  // far from the query relative to its size, and the kernel smooth on it (or the element tiny)
  const double rho = sqrt(((r[0][0] + r[1][0] + r[2][0]) / 3.0) * ((r[0][0] + r[1][0] + r[2][0]) / 3.0) +
                          ((r[0][1] + r[1][1] + r[2][1]) / 3.0) * ((r[0][1] + r[1][1] + r[2][1]) / 3.0));
  double emax = 0.0, rmin = 1e300, rmax = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double* pa = r[k];
    const double* pb = r[(k + 1) % 3];
    const double dx = pb[0] - pa[0], dy = pb[1] - pa[1];
    const double ln = sqrt(dx * dx + dy * dy);
    emax = fmax(emax, ln);
    const double tt = fmin(fmax(-(pa[0] * dx + pa[1] * dy) / (ln * ln), 0.0), 1.0);
    const double qx = pa[0] + tt * dx, qy = pa[1] + tt * dy;
    rmin = fmin(rmin, sqrt(qx * qx + qy * qy));
    rmax = fmax(rmax, sqrt(pa[0] * pa[0] + pa[1] * pa[1]));
  }
  const bool straddle = fem_straddle<KT, 0>(rmin, rmax);
  double wk[3] = {0.0, 0.0, 0.0}, Gx[3] = {0.0, 0.0, 0.0}, Gy[3] = {0.0, 0.0, 0.0};
  if (rho >= kFemFarRatio * emax && (!straddle || emax <= kFemTiny)) {
    const double area2 = fabs(d2);
    for (int ia = 0; ia < kFemGauss; ++ia)
      for (int ib = 0; ib < kFemGauss; ++ib) {
        const double ua = kFemGx[ia], vb = kFemGx[ib];
        const double m1 = ua, m2 = vb * (1.0 - ua), m0 = 1.0 - m1 - m2;
        const double wt = kFemGw[ia] * kFemGw[ib] * (1.0 - ua) * area2;
        const double yx = m0 * r[0][0] + m1 * r[1][0] + m2 * r[2][0];
        const double yy = m0 * r[0][1] + m1 * r[1][1] + m2 * r[2][1];
        const double rr = sqrt(yx * yx + yy * yy);
        double P = 0.0, dP = 0.0;
        if (rr < 1.0) pi_w_deriv<KT::kId>(rr, P, dP);
        const double Wv = P * kInvPi, dWr = dP * kInvPi / fmax(rr, 1e-300);
        const double m[3] = {m0, m1, m2};
#pragma unroll
        for (int k = 0; k < 3; ++k) {              // grad_x W = -(W'/r) y
          wk[k] += wt * m[k] * Wv;
          Gx[k] += -wt * m[k] * dWr * yx;
          Gy[k] += -wt * m[k] * dWr * yy;
        }
      }
  } else {
    // the triangle as a counter-clockwise polygon: three edges' closed forms and the winding indicator
    const int i1 = d2 < 0.0 ? 2 : 1, i2 = d2 < 0.0 ? 1 : 2;
    const double* p[3] = {r[0], r[i1], r[i2]};
    double acc[12];
#pragma unroll
    for (int c = 0; c < 12; ++c) acc[c] = 0.0;
    double ang = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double* a = p[k];
      const double* b = p[(k + 1) % 3];
      PairGeo g;
      if (pair_geo(a[0], a[1], b[0], b[1], g)) fem_blocks<KT, 0>(g, acc);
      const double cr = cross2_rn(a[0], a[1], b[0], b[1]);
      if (cr != 0.0) ang += atan2(cr, dot2_rn(a[0], a[1], b[0], b[1]));
    }
    const double ind = ang / kTwoPi;
#pragma unroll
    for (int c = 0; c < 12; ++c) acc[c] *= kInvPi;
    acc[0] += ind * KT::kMass;
    acc[5] += ind * KT::kMass;
    acc[8] += ind * KT::kMass;
    const double lam = acc[0], m1x = acc[1], m1y = acc[2], Gcx = acc[3], Gcy = acc[4];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      wk[k] = l[k] * lam + gx[k] * m1x + gy[k] * m1y;
      Gx[k] = l[k] * Gcx + gx[k] * acc[5] + gy[k] * acc[7];
      Gy[k] = l[k] * Gcy + gx[k] * acc[6] + gy[k] * acc[8];
    }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    w[3 * t + k] = wk[k];
    G[6 * t + 2 * k] = Gx[k] / h;
    G[6 * t + 2 * k + 1] = Gy[k] / h;
  }
}

}  // namespace wsb

using namespace wsb;

// The launch runs on the device that holds `pos` (made current for the call, the caller's current device restored
// afterwards), so a caller whose current device is another one still gets the launch in the right context.
extern "C" int wsb_pair_weights(int kernel, const int32_t* pair_q, const int32_t* pair_e, int64_t n_pairs,
                                const double* pos, const double* sup, int64_t n_pos, const double* verts,
                                int64_t n_verts, const int32_t* elems, int64_t n_elems, double* w, double* G,
                                int32_t* status, void* stream) {
  if (n_pairs < 0 || n_pairs > (int64_t)INT32_MAX) return fail(WSB_ERR_ARG, "wsb_pair_weights: pair count out of range");
  if (n_pos < 0 || n_verts < 0 || n_elems < 0) return fail(WSB_ERR_ARG, "wsb_pair_weights: negative array size");
  if (kernel < 0 || kernel >= kNumKernels)
    return fail(WSB_ERR_UNSUPPORTED, "wsb_pair_weights: kernel id " + std::to_string(kernel) +
                                         " (exact-table kernels only)");
  if (n_pairs == 0) return WSB_OK;
  if (!pair_q || !pair_e || !pos || !sup || !verts || !elems || !w || !G || !status)
    return fail(WSB_ERR_ARG, "wsb_pair_weights: NULL array");
  cudaPointerAttributes attr{};
  WSB_CUDA(cudaPointerGetAttributes(&attr, pos));
  if (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged)
    return fail(WSB_ERR_ARG, "wsb_pair_weights: positions are not device memory");
  int prev = 0;
  WSB_CUDA(cudaGetDevice(&prev));
  if (prev != attr.device) WSB_CUDA(cudaSetDevice(attr.device));
  const unsigned grid = (unsigned)((n_pairs + kFemThreads - 1) / kFemThreads);
  cudaStream_t st = (cudaStream_t)stream;
  const int rc = dispatch_kernel(kernel, [&](auto kt) {
    k_pair_weights<decltype(kt)><<<grid, kFemThreads, 0, st>>>(pair_q, pair_e, n_pairs, pos, sup, n_pos, verts,
                                                                 n_verts, elems, n_elems, w, G, status);
    return 0;
  });
  const cudaError_t launch = cudaGetLastError();
  if (prev != attr.device) WSB_CUDA(cudaSetDevice(prev));
  if (rc) return rc;
  WSB_CUDA(launch);
  return WSB_OK;
}
