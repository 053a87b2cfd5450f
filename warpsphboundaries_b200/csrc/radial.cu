// Solid half-spaces and solid spheres in 3-D: the nine axial invariants of the kernel integrals over the part of a
// query's support that lies inside the solid, and their rotation into Cartesian channels (the 28 baseline requests
// |alpha| + |derivative| <= 2, or any subset).
//
// Reference: src/warpSPHBoundaries/fluxbridge/radial.py:20-71 (functions: element + select + batch) and the native
// element of src/warpSPHBoundaries/fluxbridge/_radial_code.py:43-148.  The invariants are the shell integrals of
// fluxbridge/radial_reference.py:17-56: at radius r the support sphere meets the solid in a spherical cap mu >= cap
// along the inward axis (cap = -d/r for a half-space, (R^2 - D^2 - r^2) / (2 D r) with D = R + d for a sphere of
// radius R whose surface is at signed distance d), and integrating the monomials over the cap gives
//   a0 = 2 pi (1 + cap), a1 = pi (cap^2 - 1), at = pi (cap - cap^3/3 + 2/3), an = 2 pi (cap^3 + 1) / 3.
// The reference integrates products of linear factors in Bernstein form; here each radial sub-interval (per kernel
// piece: the full-ball region [0, min(1, -d)] and the cap region [|d|, min(1, 2R + d)]) is integrated by 12-node
// Gauss-Legendre, which is exact for the polynomial integrands (degree <= 18) and leaves < 1e-17 relative on cubic's
// outer Laurent piece (r >= 1/2).  Cancellation is avoided by factoring the angular terms:
//   u = 1 + cap = (r - d)(2R + d - r) / (2 D r),  v = 1 - cap = (r + d)(r + d + 2R) / (2 D r)   (sphere)
//   u = (r - d) / r,                              v = (r + d) / r                               (half-space)
//   a0 = 2u, a1 = -u v, at = u^2 (1 + v) / 3, an = 2/3 u (cap^2 - cap + 1)          (times pi; pi cancels against W)
// and the kernel profiles W, W'/r and (W'/r)' are evaluated as r^p (hi - r)^k g(r) with exact factors.
#include "common.cuh"


namespace wsb {
namespace {

struct RadialRequests {            // up to 28 requests: degree, i, j, order (reference metadata, radial.py:124-128)
  int n;
  signed char meta[28][4];
};

template <typename T>
struct Inv9 {
  T v[9];
};

// one piece's contribution: the full-ball region [lo, hi] (cap = 1) and the cap region [clo, chi]
template <class KR, int P, typename T>
__device__ __forceinline__ void radial_piece(T d, T R, T D, bool sphere, T full_end, T cap_end, Inv9<T>& acc) {
  const T plo = T(KR::kLo[P]), phi = T(KR::kHi[P]);
  {
    const T lo = plo, hi = fmin(phi, full_end);
    if (hi > lo) {
      const T c = T(0.5) * (hi + lo), hw = T(0.5) * (hi - lo);
      T s0 = 0, s2 = 0, s5 = 0, s7 = 0;
#pragma unroll
      for (int g = 0; g < kRadialGauss; ++g) {
        const T r = fma_t(hw, T(kRadialGx[g]), c), wg = T(kRadialGw[g]);
        T w, l, dl;
        KR::template eval<P, T>(r, w, l, dl);
        const T r2 = r * r, r3 = r2 * r, r4 = r2 * r2;
        s0 = fma_t(wg, r2 * w, s0);
        s2 = fma_t(wg, r4 * w, s2);
        s5 = fma_t(wg, r4 * l, s5);
        s7 = fma_t(wg, fma_t(T(4), r2 * l, T(4.0 / 3.0) * r3 * dl), s7);
      }
      acc.v[0] += hw * T(4) * s0;
      acc.v[2] += hw * T(4.0 / 3.0) * s2;
      acc.v[3] += hw * T(4.0 / 3.0) * s2;
      acc.v[5] -= hw * T(4.0 / 3.0) * s5;
      acc.v[6] -= hw * T(4.0 / 3.0) * s5;
      acc.v[7] += hw * s7;
      acc.v[8] += hw * s7;
    }
  }
  {
    const T lo = fmax(plo, fabs(d)), hi = fmin(phi, cap_end);
    if (hi > lo) {
      const T c = T(0.5) * (hi + lo), hw = T(0.5) * (hi - lo);
      T s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      const T inv2D = sphere ? T(1) / (T(2) * D) : T(0);
#pragma unroll
      for (int g = 0; g < kRadialGauss; ++g) {
        const T r = fma_t(hw, T(kRadialGx[g]), c), wg = T(kRadialGw[g]);
        T w, l, dl;
        KR::template eval<P, T>(r, w, l, dl);
        const T ir = T(1) / r;
        T u, v;
        if (sphere) {
          u = (r - d) * ((R - r) + (R + d)) * inv2D * ir;
          v = (r + d) * ((r + d) + T(2) * R) * inv2D * ir;
        } else {
          u = (r - d) * ir;
          v = (r + d) * ir;
        }
        const T cap = T(0.5) * (u - v);
        const T a0 = T(2) * u, a1 = -u * v, at = u * u * (T(1) + v) * T(1.0 / 3.0),
                an = T(2.0 / 3.0) * u * fma_t(cap, cap - T(1), T(1));
        const T r2 = r * r, r3 = r2 * r, r4 = r2 * r2;
        const T ww = wg * w, wl = wg * l;
        s[0] = fma_t(ww, r2 * a0, s[0]);
        s[1] = fma_t(ww, r3 * a1, s[1]);
        s[2] = fma_t(ww, r4 * at, s[2]);
        s[3] = fma_t(ww, r4 * an, s[3]);
        s[4] = fma_t(wl, r3 * a1, s[4]);
        s[5] = fma_t(wl, r4 * at, s[5]);
        s[6] = fma_t(wl, r4 * an, s[6]);
        const T base = wl * r2 * a0, wdl = wg * dl * r3;
        s[7] += fma_t(wdl, at, base);
        s[8] += fma_t(wdl, an, base);
      }
      acc.v[0] += hw * s[0];
      acc.v[1] += hw * s[1];
      acc.v[2] += hw * s[2];
      acc.v[3] += hw * s[3];
      acc.v[4] -= hw * s[4];
      acc.v[5] -= hw * s[5];
      acc.v[6] -= hw * s[6];
      acc.v[7] += hw * s[7];
      acc.v[8] += hw * s[8];
    }
  }
}

// the nine invariants at unit support: (lam, m1_axial, m2_tangent, m2_axial, G_axial, g1_tangent, g1_axial,
// H_tangent, H_axial); d = signed outward distance / h, R = radius / h (ignored for a half-space)
template <class KR, typename T>
__device__ __forceinline__ void radial_invariants(T d, T R, bool sphere, Inv9<T>& acc) {
#pragma unroll
  for (int j = 0; j < 9; ++j) acc.v[j] = T(0);
  const T cap_end = sphere ? fmin(T(1), T(2) * R + d) : T(1);
  if (d <= T(-1)) {
    // the whole support lies in the solid (for a sphere |x - c| + h <= R): exact constants
    KR::template full<T>(acc.v);
    return;
  }
  if (d >= T(1)) return;                       // the support does not reach the solid
  const T full_end = fmin(T(1), fmax(T(0), -d));
  radial_piece<KR, 0, T>(d, R, R + d, sphere, full_end, cap_end, acc);
  if constexpr (KR::kPieces > 1) radial_piece<KR, 1, T>(d, R, R + d, sphere, full_end, cap_end, acc);
  static_assert(KR::kPieces <= 2, "radial kernels have at most two pieces");
}

constexpr int kRadialThreads = 128;

__device__ __forceinline__ double pick3(int i, double x, double y, double z) { return i == 0 ? x : (i == 1 ? y : z); }

// one thread per row; the block's rows are contiguous, so their outputs [row0 .. row0 + 128) x n_requests are one
// contiguous range: each thread writes its row into shared memory, then the block stores the range coalesced
template <class KR, typename T>
__global__ void __launch_bounds__(kRadialThreads, 6) k_radial(const double* __restrict__ dist,
                                                              const double* __restrict__ radii,
                                                              const double* __restrict__ normals,
                                                              const double* __restrict__ supports, int64_t n,
                                                              int sphere, RadialRequests req,
                                                              double* __restrict__ out, double* __restrict__ inv_out,
                                                              int32_t* __restrict__ status) {
  __shared__ double stage[kRadialThreads * 28];
  const int64_t row0 = (int64_t)blockIdx.x * kRadialThreads;
  const int64_t row = row0 + threadIdx.x;
  const int nreq = req.n;
  if (row < n) {
    const double h = supports[row], dd = dist[row];
    const double Rr = sphere ? radii[row] : 0.0;
    const double nx = normals[3 * row], ny = normals[3 * row + 1], nz = normals[3 * row + 2];
    const bool ok = h > 0.0 && isfinite(h) && isfinite(dd) && isfinite(nx) && isfinite(ny) && isfinite(nz) &&
                    (!sphere || (Rr > 0.0 && isfinite(Rr) && dd >= -Rr));
    Inv9<T> acc;
    double inv[9];
    if (ok) {
      radial_invariants<KR, T>(T(dd / h), T(Rr / h), sphere != 0, acc);
      const double ih = 1.0 / h;
      const double scale[9] = {1.0, h, h * h, h * h, ih, 1.0, 1.0, ih * ih, ih * ih};
#pragma unroll
      for (int j = 0; j < 9; ++j) inv[j] = (double)acc.v[j] * scale[j];
    } else {
#pragma unroll
      for (int j = 0; j < 9; ++j) inv[j] = __longlong_as_double(0x7ff8000000000000LL);
    }
    if (status) status[row] = ok ? 0 : 1;
    if (inv_out) {
#pragma unroll
      for (int j = 0; j < 9; ++j) inv_out[row * 9 + j] = inv[j];
    }
#pragma unroll 4
    for (int c = 0; c < nreq; ++c) {
      const int degree = req.meta[c][0], i = req.meta[c][1], j = req.meta[c][2], order = req.meta[c][3];
      const double ni = pick3(i, nx, ny, nz), nj = pick3(j, nx, ny, nz);
      double v;
      if (degree == 0 && order == 0) {
        v = inv[0];
      } else if (degree == 1 && order == 0) {
        v = inv[1] * ni;
      } else if (degree == 0 && order == 1) {
        v = inv[4] * ni;
      } else {
        // tangent / axial pair of the second-order entry: m2 (2, 3), g1 (5, 6), Hessian (7, 8)
        const double tan = order == 0 ? inv[2] : (order == 1 ? inv[5] : inv[7]);
        const double axi = order == 0 ? inv[3] : (order == 1 ? inv[6] : inv[8]);
        v = (axi - tan) * ni * nj + (i == j ? tan : 0.0);
      }
      stage[threadIdx.x * nreq + c] = v;
    }
  }
  __syncthreads();
  const int64_t rows_here = n - row0 < kRadialThreads ? n - row0 : kRadialThreads;
  const int count = (int)rows_here * nreq;
  double* dst = out + row0 * nreq;
  for (int k = threadIdx.x; k < count; k += kRadialThreads) dst[k] = stage[k];
}

template <typename T>
int launch_radial(int kernel, const double* d, const double* r, const double* nrm, const double* h, int64_t n,
                  int sphere, const RadialRequests& req, double* out, double* inv, int32_t* status,
                  cudaStream_t st) {
  const unsigned grid = (unsigned)((n + kRadialThreads - 1) / kRadialThreads);
  constexpr int B = kRadialThreads;
  switch (kernel) {
    case WSB_KERNEL_CUBIC: k_radial<Rad_cubic, T><<<grid, B, 0, st>>>(d, r, nrm, h, n, sphere, req, out, inv, status); break;
    case WSB_KERNEL_W2: k_radial<Rad_w2, T><<<grid, B, 0, st>>>(d, r, nrm, h, n, sphere, req, out, inv, status); break;
    case WSB_KERNEL_W4: k_radial<Rad_w4, T><<<grid, B, 0, st>>>(d, r, nrm, h, n, sphere, req, out, inv, status); break;
    case WSB_KERNEL_W6: k_radial<Rad_w6, T><<<grid, B, 0, st>>>(d, r, nrm, h, n, sphere, req, out, inv, status); break;
    default: return fail(WSB_ERR_UNSUPPORTED, "wsb_radial_channels: the radial family serves cubic, w2, w4, w6");
  }
  WSB_CUDA(cudaGetLastError());
  return WSB_OK;
}

}  // namespace
}  // namespace wsb

using namespace wsb;

extern "C" int wsb_radial_channels(int kind, int kernel, int precision, const double* distances, const double* radii,
                                   const double* normals, const double* supports, int64_t n, const int32_t* requests,
                                   int n_requests, double* out, double* invariants, int32_t* status, void* stream) {
  if (kind != WSB_RADIAL_PLANE && kind != WSB_RADIAL_SPHERE)
    return fail(WSB_ERR_ARG, "wsb_radial_channels: kind must be WSB_RADIAL_PLANE or WSB_RADIAL_SPHERE");
  if (n < 0) return fail(WSB_ERR_ARG, "wsb_radial_channels: negative size");
  if (n_requests < 0 || n_requests > 28) return fail(WSB_ERR_ARG, "wsb_radial_channels: 0..28 requests");
  if (precision != WSB_PREC_FP64 && precision != WSB_PREC_FP32)
    return fail(WSB_ERR_UNSUPPORTED, "wsb_radial_channels: precision must be WSB_PREC_FP64 or WSB_PREC_FP32");
  if (kernel < 0 || kernel > WSB_KERNEL_W6)
    return fail(WSB_ERR_UNSUPPORTED, "wsb_radial_channels: the radial family serves cubic, w2, w4, w6");
  RadialRequests req{};
  req.n = n_requests;
  for (int c = 0; c < n_requests; ++c) {
    const int32_t* m = requests + 4 * c;
    const int degree = m[0], i = m[1], j = m[2], order = m[3];
    if (degree < 0 || order < 0 || degree + order > 2 || i < 0 || i > 2 || j < 0 || j > 2)
      return fail(WSB_ERR_ARG, "wsb_radial_channels: request rows are (degree, i, j, order) with degree + order <= 2");
    for (int q = 0; q < 4; ++q) req.meta[c][q] = (signed char)m[q];
  }
  if (n == 0) return WSB_OK;
  if (!distances || !normals || !supports || (n_requests && !out) || (kind == WSB_RADIAL_SPHERE && !radii))
    return fail(WSB_ERR_ARG, "wsb_radial_channels: NULL array");
  cudaStream_t st = (cudaStream_t)stream;
  return precision == WSB_PREC_FP64
             ? launch_radial<double>(kernel, distances, radii, normals, supports, n, kind, req, out, invariants, status, st)
             : launch_radial<float>(kernel, distances, radii, normals, supports, n, kind, req, out, invariants, status, st);
}
