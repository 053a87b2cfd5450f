// Fixed-capacity topology (slots + indicator) and the plain FP64 route: the reference's per-pair plan interpreter
// and its per-row contraction, restated in CUDA for sm_100a.
#include "common.cuh"

namespace wsb {

// ------------------------------------------------------------------------------------------------ fixed topology
// one thread per row: the edges of the row's cell that pass the float64 predicate, in cell-list order, into K slots,
// and the winding indicator (src/warpSPHBoundaries/scene/fixedadj.py:67-147)
__global__ void k_fixed_topology(SurfView S, const double* __restrict__ lpos, const double* __restrict__ lsup,
                                 const int32_t* __restrict__ valid, int64_t n, int32_t* __restrict__ slots,
                                 double* __restrict__ ind) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  int32_t* sl = slots + r * S.K;
  for (int k = 0; k < S.K; ++k) sl[k] = -1;
  if (valid && valid[r] == 0) {
    ind[r] = 0.0;
    return;
  }
  const double px = lpos[2 * r], py = lpos[2 * r + 1], h = lsup[r];
  int32_t cid;
  const bool in_grid = cell_of(S, px, py, cid);
  if (in_grid) {
    int m = 0;
    for (int i = S.cstart[cid]; i < S.cstart[cid + 1]; ++i) {
      const double4 e = S.crec[i];
      if (seg_within(px, py, e.x, e.y, e.z, e.w, h)) sl[m++] = S.citems[i];
    }
  }
  ind[r] = indicator_at(S, px, py, h, in_grid, cid);
}

// ------------------------------------------------------------------------------------------------ reference plan tables
__constant__ int c_planE[kPlanEdgeTerms][7];
__constant__ int c_planVi[kPlanValueTerms][4];
__constant__ double c_planVmR[kPlanValueTerms];
__constant__ int c_planCn[kPlanCoeffs];
__constant__ double c_planCc[kPlanCoeffs];
__constant__ double c_planRadii[kPlanNumRadii];
__constant__ PlanOffsets c_planOffs[kNumKernels];

static int upload_plan_once(int device) {
  static bool done[64] = {false};
  if (device < 0 || device >= 64) return fail(WSB_ERR_ARG, "device id out of range");
  if (done[device]) return WSB_OK;
  WSB_CUDA(cudaMemcpyToSymbol(c_planE, kPlanE, sizeof(kPlanE)));
  WSB_CUDA(cudaMemcpyToSymbol(c_planVi, kPlanVi, sizeof(kPlanVi)));
  WSB_CUDA(cudaMemcpyToSymbol(c_planVmR, kPlanVmR, sizeof(kPlanVmR)));
  WSB_CUDA(cudaMemcpyToSymbol(c_planCn, kPlanCn, sizeof(kPlanCn)));
  WSB_CUDA(cudaMemcpyToSymbol(c_planCc, kPlanCc, sizeof(kPlanCc)));
  WSB_CUDA(cudaMemcpyToSymbol(c_planRadii, kPlanRadii, sizeof(kPlanRadii)));
  WSB_CUDA(cudaMemcpyToSymbol(c_planOffs, kPlanOffsets, sizeof(kPlanOffsets)));
  done[device] = true;
  return WSB_OK;
}

// ------------------------------------------------------------------------------------------------ reference primitives
// src/warpSPHBoundaries/edge/warp2d.py:28-149, evaluated as the reference evaluates them (pow of r^2, binomial loops)
__device__ double ref_asinh(double u) {
  const double a = fabs(u);
  double v = log(a + sqrt(a * a + 1.0));
  return u < 0.0 ? -v : v;
}

__device__ double ref_Im(int m, double s, double z) {
  const double zz = z * z, r2 = s * s + zz;
  const double r = r2 > 0.0 ? sqrt(r2) : 0.0;
  double val = s;
  int idx = 0;
  if (m % 2 == 1) {
    double tail = 0.0;
    if (z != 0.0) tail = zz * ref_asinh(s / fabs(z));
    val = (s * r + tail) / 2.0;
    idx = 1;
  }
  while (idx < m) {
    idx += 2;
    const double rp = (idx % 2 == 0) ? pow(r2, (double)(idx / 2)) : r * pow(r2, (double)((idx - 1) / 2));
    val = (s * rp + (double)idx * zz * val) / (double)(idx + 1);
  }
  return val;
}

__device__ double ref_binom(int n, int k) {
  double v = 1.0;
  for (int i = 0; i < k; ++i) v = v * (double)(n - i) / (double)(i + 1);
  return v;
}

__device__ double ref_S(int j, int m, double s, double z) {
  const double zz = z * z;
  double tot = 0.0;
  if (j % 2 == 0) {
    const int h = j / 2;
    for (int i = 0; i <= h; ++i) {
      const double sg = ((h - i) % 2 == 1) ? -1.0 : 1.0;
      tot += ref_binom(h, i) * sg * pow(zz, (double)(h - i)) * ref_Im(m + 2 * i, s, z);
    }
  } else {
    const int h = (j - 1) / 2;
    const double r2 = s * s + zz;
    const double r = r2 > 0.0 ? sqrt(r2) : 0.0;
    for (int i = 0; i <= h; ++i) {
      const int mm = m + 2 * i;
      const double rp = (mm % 2 == 0) ? pow(r2, (double)((mm + 2) / 2)) : r * pow(r2, (double)((mm + 1) / 2));
      const double sg = ((h - i) % 2 == 1) ? -1.0 : 1.0;
      tot += ref_binom(h, i) * sg * pow(zz, (double)(h - i)) * rp / (double)(mm + 2);
    }
  }
  return tot;
}

__device__ double ref_ypoly_coef(int a, int b, int j, double z, double n0, double n1, double t0, double t1) {
  double tot = 0.0;
  for (int ja = 0; ja <= a; ++ja) {
    const int jb = j - ja;
    if (jb >= 0 && jb <= b) {
      const double ca = ref_binom(a, ja) * pow(t0, (double)ja) * pow(z * n0, (double)(a - ja));
      const double cb = ref_binom(b, jb) * pow(t1, (double)jb) * pow(z * n1, (double)(b - jb));
      tot += ca * cb;
    }
  }
  return tot;
}

__device__ double ref_dangle(double z, double lo, double hi) {
  if (z == 0.0) return 0.0;
  const double y = z * (hi - lo), x = z * z + lo * hi;
  if (y == 0.0 && x == 0.0) return 0.0;
  return atan2(y, x);
}

// one thread per slot: the twelve channels of the slot's (row, edge) pair by the plan interpreter
// (src/warpSPHBoundaries/edge/warpbc.py:619-661 with the term plan of warpbc.py:98-117, 970-991)
__global__ void k_slot_channels_plain(SurfView S, int kernel, const double* __restrict__ lpos,
                                      const double* __restrict__ lsup, const int32_t* __restrict__ slots, int64_t n,
                                      double* __restrict__ c) {
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (tid >= n * S.K) return;
  double* out = c + tid * 12;
  for (int k = 0; k < 12; ++k) out[k] = 0.0;
  const int32_t e = slots[tid];
  if (e < 0) return;
  const int64_t r = tid / S.K;
  const double h = lsup[r], xv0 = lpos[2 * r], xv1 = lpos[2 * r + 1];
  const int v0 = S.edges[2 * e], v1 = S.edges[2 * e + 1];
  const double p0 = (S.verts[2 * v0] - xv0) / h, p1 = (S.verts[2 * v0 + 1] - xv1) / h;
  const double q0 = (S.verts[2 * v1] - xv0) / h, q1 = (S.verts[2 * v1 + 1] - xv1) / h;
  const double d0 = q0 - p0, d1 = q1 - p1;
  const double ell = sqrt(d0 * d0 + d1 * d1);
  if (ell == 0.0) return;
  const double t0 = d0 / ell, t1 = d1 / ell, n0 = t1, n1 = -t0;
  const double z = cross2_rn(p0, p1, q0, q1) / ell;
  const double s0 = (d0 * p0 + d1 * p1) / ell, s1 = (d0 * q0 + d1 * q1) / ell;
  const double az = fabs(z);
  double ch[12];
  for (int k = 0; k < 12; ++k) ch[k] = 0.0;
  const PlanOffsets po = c_planOffs[kernel];
  for (int t = po.e0; t < po.e1; ++t) {
    const double R = c_planRadii[c_planE[t][4]];
    if (az < R) {
      const double a2 = (R - az) * (R + az);
      const double L = a2 > 0.0 ? sqrt(a2) : 0.0;
      const double lo = fmax(s0, -L), hi = fmin(s1, L);
      if (lo < hi) {
        const int a = c_planE[t][2], b = c_planE[t][3];
        double tot = 0.0;
        for (int j = 0; j <= a + b; ++j) {
          const double yc = ref_ypoly_coef(a, b, j, z, n0, n1, t0, t1);
          if (yc != 0.0) {
            double inner = 0.0;
            for (int k = c_planE[t][5]; k < c_planE[t][6]; ++k)
              inner += c_planCc[k] * (ref_S(j, c_planCn[k], hi, z) - ref_S(j, c_planCn[k], lo, z));
            tot += yc * inner;
          }
        }
        ch[c_planE[t][0]] += (c_planE[t][1] == 0 ? n0 : n1) * tot;
      }
    }
  }
  for (int t = po.v0; t < po.v1; ++t) {
    const double R = c_planRadii[c_planVi[t][1]];
    if (az < R) {
      const double a2 = (R - az) * (R + az);
      const double L = a2 > 0.0 ? sqrt(a2) : 0.0;
      const double lo = fmax(s0, -L), hi = fmin(s1, L);
      if (lo < hi) {
        double poly = 0.0;
        for (int k = c_planVi[t][2]; k < c_planVi[t][3]; ++k)
          poly += c_planCc[k] * (ref_S(0, c_planCn[k], hi, z) - ref_S(0, c_planCn[k], lo, z));
        ch[c_planVi[t][0]] += z * poly - c_planVmR[t] * ref_dangle(z, lo, hi);
      }
    }
  }
  for (int k = 0; k < 12; ++k) out[k] = kInvPi * ch[k];
}

__global__ void k_contract(int K, double mass, double plane2, const int32_t* __restrict__ slots,
                           const double* __restrict__ c, const double* __restrict__ ind, const double* __restrict__ lsup,
                           int64_t n, const double* __restrict__ rot, double* lam, double* G, double* cov, double* m1,
                           double* m2) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  double ch[12];
  for (int k = 0; k < 12; ++k) ch[k] = 0.0;
  for (int s = 0; s < K; ++s) {
    const double* cs = c + (r * K + s) * 12;
    for (int k = 0; k < 12; ++k) ch[k] += cs[k];
  }
  const double w = ind[r];
  ch[0] += w * mass;
  ch[5] += w * mass;
  ch[8] += w * mass;
  ch[9] += w * plane2;
  ch[11] += w * plane2;
  write_outputs(ch, lsup[r], rot, r, lam, G, cov, m1, m2);
}

// ------------------------------------------------------------------------------------------------ pair-list channels
// One thread per (query, edge) pair of a pair list (the (qi, e) lists of SurfaceRep.topology): the pair's twelve
// edge-local channels, units of h, x 1/pi, by the closed-form chord engine block by block -- the reference's
// warpbc.edge_channels + second_channels over a pair list (src/warpSPHBoundaries/edge/warpbc.py:919-991), which
// SurfaceRep.moments sums per query (scene.py:384-416).  A tensile (quadrature) kernel defines its G channels only; the
// others are NaN.  A query or edge index outside its array gives NaN channels and sets the status word.
template <class KT, int PREC, int B>
__device__ __forceinline__ void pair_blocks(const PairGeo& g, double* acc) {
  if constexpr (B < KT::kBlocks) {
    block_channels<KT, B, PREC>(g, acc);
    pair_blocks<KT, PREC, B + 1>(g, acc);
  }
}

template <class KT, int PREC>
__global__ void k_pair_channels(SurfView S, const int32_t* __restrict__ qi, const int32_t* __restrict__ e,
                                int64_t n_pairs, const double* __restrict__ lpos, const double* __restrict__ lsup,
                                int64_t n_rows, double* __restrict__ c, int32_t* __restrict__ status) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n_pairs) return;
  const double nan = __longlong_as_double(0x7ff8000000000000LL);
  double acc[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) acc[k] = 0.0;
  const int64_t q = qi[t], ei = e[t];
  if (q < 0 || q >= n_rows || ei < 0 || ei >= S.n_edges) {
#pragma unroll
    for (int k = 0; k < 12; ++k) c[12 * t + k] = nan;
    atomicExch(status, 1);
    return;
  }
  const double h = lsup[q];
  PairGeo g;
  if (pair_geo_row(lpos[2 * q], lpos[2 * q + 1], h, 1.0 / h, S.erec[ei], g)) {
    if constexpr (KT::kQuad) {
      double lo, hi, rlo, rhi, zz;
      if (clip_chord(g, 1.0, lo, hi, rlo, rhi, zz)) {
        const double W0 = quad_chord<KT>(lo, hi, g.z);
        acc[3] = -g.n0 * W0;
        acc[4] = -g.n1 * W0;
      }
    } else {
      pair_blocks<KT, PREC, 0>(g, acc);
    }
  }
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    const bool defined = !KT::kQuad || k == 3 || k == 4;
    c[12 * t + k] = defined ? acc[k] * kInvPi : nan;
  }
}

}  // namespace wsb

using namespace wsb;

extern "C" int wsb_pair_channels(const wsb_surface* s_, int kernel, int precision, const int32_t* qi, const int32_t* e,
                                 int64_t n_pairs, const double* lpos, const double* lsup, int64_t n_rows, double* c,
                                 int32_t* status, void* stream) {
  const Surface* s = reinterpret_cast<const Surface*>(s_);
  if (!s) return fail(WSB_ERR_ARG, "wsb_pair_channels: NULL surface");
  if (n_pairs < 0 || n_rows < 0) return fail(WSB_ERR_ARG, "wsb_pair_channels: negative size");
  if (precision != WSB_PREC_FP64 && precision != WSB_PREC_MIXED)
    return fail(WSB_ERR_UNSUPPORTED, "wsb_pair_channels: precision " + std::to_string(precision));
  const bool quad = kernel == Kern_w2p5::kId || kernel == Kern_w4p5::kId;
  if (!quad && (kernel < 0 || kernel >= kNumKernels)) return fail(WSB_ERR_UNSUPPORTED, "unknown kernel id");
  if (n_pairs == 0) return WSB_OK;
  if (!qi || !e || !lpos || !lsup || !c || !status) return fail(WSB_ERR_ARG, "wsb_pair_channels: NULL array");
  WSB_CUDA(cudaSetDevice(s->device));
  const unsigned grid = (unsigned)((n_pairs + 127) / 128);
  cudaStream_t st = (cudaStream_t)stream;
  const SurfView v = view_of(s);
  auto launch = [&](auto kt) {
    using KT = decltype(kt);
    if (precision == WSB_PREC_MIXED)
      k_pair_channels<KT, WSB_PREC_MIXED><<<grid, 128, 0, st>>>(v, qi, e, n_pairs, lpos, lsup, n_rows, c, status);
    else
      k_pair_channels<KT, WSB_PREC_FP64><<<grid, 128, 0, st>>>(v, qi, e, n_pairs, lpos, lsup, n_rows, c, status);
    return 0;
  };
  int rc;
  if (kernel == Kern_w2p5::kId)
    rc = launch(Kern_w2p5{});
  else if (kernel == Kern_w4p5::kId)
    rc = launch(Kern_w4p5{});
  else
    rc = dispatch_kernel(kernel, launch);
  if (rc) return rc;
  WSB_CUDA(cudaGetLastError());
  return WSB_OK;
}

static double kernel_plane2(int kernel) {
  double v = 0.0;
  dispatch_kernel(kernel, [&](auto kt) {
    v = decltype(kt)::kPlane2;
    return 0;
  });
  return v;
}

extern "C" int wsb_fixed_topology(const wsb_surface* s_, const double* lpos, const double* lsup, const int32_t* valid,
                                  int64_t n, int32_t* slots, double* ind, void* stream) {
  const Surface* s = reinterpret_cast<const Surface*>(s_);
  if (!s) return fail(WSB_ERR_ARG, "wsb_fixed_topology: NULL surface");
  if (n < 0) return fail(WSB_ERR_ARG, "wsb_fixed_topology: negative row count");
  if (n == 0) return WSB_OK;
  if (!lpos || !lsup || !slots || !ind) return fail(WSB_ERR_ARG, "wsb_fixed_topology: NULL array");
  WSB_CUDA(cudaSetDevice(s->device));
  k_fixed_topology<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(view_of(s), lpos, lsup, valid, n,
                                                                                   slots, ind);
  WSB_CUDA(cudaGetLastError());
  return WSB_OK;
}

extern "C" int wsb_slot_channels_plain(const wsb_surface* s_, int kernel, const double* lpos, const double* lsup,
                                       const int32_t* slots, int64_t n, double* c, void* stream) {
  const Surface* s = reinterpret_cast<const Surface*>(s_);
  if (!s) return fail(WSB_ERR_ARG, "wsb_slot_channels_plain: NULL surface");
  if (kernel < 0 || kernel >= kNumKernels) return fail(WSB_ERR_UNSUPPORTED, "unknown kernel id");
  if (n < 0) return fail(WSB_ERR_ARG, "wsb_slot_channels_plain: negative row count");
  if (n == 0) return WSB_OK;
  if (!lpos || !lsup || !slots || !c) return fail(WSB_ERR_ARG, "wsb_slot_channels_plain: NULL array");
  WSB_CUDA(cudaSetDevice(s->device));
  int rc = upload_plan_once(s->device);
  if (rc) return rc;
  const int64_t total = n * s->K;
  k_slot_channels_plain<<<(unsigned)((total + 127) / 128), 128, 0, (cudaStream_t)stream>>>(view_of(s), kernel, lpos,
                                                                                           lsup, slots, n, c);
  WSB_CUDA(cudaGetLastError());
  return WSB_OK;
}

extern "C" int wsb_contract(const wsb_surface* s_, int kernel, const int32_t* slots, const double* c, const double* ind,
                            const double* lsup, int64_t n, const double* rot, double* lam, double* G, double* cov,
                            double* m1, double* m2, void* stream) {
  const Surface* s = reinterpret_cast<const Surface*>(s_);
  if (!s) return fail(WSB_ERR_ARG, "wsb_contract: NULL surface");
  if (kernel < 0 || kernel >= kNumKernels) return fail(WSB_ERR_UNSUPPORTED, "unknown kernel id");
  if (n < 0) return fail(WSB_ERR_ARG, "wsb_contract: negative row count");
  if (n == 0) return WSB_OK;
  if (!slots || !c || !ind || !lsup || !rot) return fail(WSB_ERR_ARG, "wsb_contract: NULL array");
  WSB_CUDA(cudaSetDevice(s->device));
  k_contract<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
      s->K, 1.0, kernel_plane2(kernel), slots, c, ind, lsup, n, rot, lam, G, cov, m1, m2);
  WSB_CUDA(cudaGetLastError());
  return WSB_OK;
}
