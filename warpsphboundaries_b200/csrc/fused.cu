// The fused aggregate route: rows sorted by edge cell (integer counting sort), one pass per row that forms the
// body-frame position, runs the float64 neighbour predicate over the row's cell and accumulates the closed-form
// channels of every neighbour pair in registers, then adds the indicator, scales and rotates.  Also the adjoint of the
// moments, signed distance and rigid-body kinematics.
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <atomic>
#include <mutex>
#include <tuple>
#include <utility>

#include "common.cuh"

namespace wsb {

constexpr int kThreads = 128;
constexpr int kKeys = 65;          // count keys: 0..63 rows with pairs (63 - min(pairs, 63)), 64 rows without

static inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

constexpr int kMaxPackStaged = 4;   // kernels of the largest pack: channel sums a staged work row holds

// the neighbour mask of a row covers the first kMaskBits candidates of its cell; later candidates (cells holding more
// edges) are found again by the predicate in the pair kernel
constexpr int kMaskBits = 128;

// one work row (a row with neighbour pairs) as the pair and adjoint kernels read it: one coalesced 64-byte load
struct __align__(16) WorkRec {
  double lx, ly;           // [0, 16)  body-frame position
  double h;                // [16, 24) support
  int32_t row, kb;         // [24, 32) row index, first candidate of the row's cell
  uint64_t m0, m1;         // [32, 48) neighbour mask of the first kMaskBits candidates
  int32_t ke, pad[3];      // [48, 64) end of the cell's candidates
};
static_assert(sizeof(WorkRec) == 64 && offsetof(WorkRec, h) == 16 && offsetof(WorkRec, row) == 24 &&
                  offsetof(WorkRec, kb) == 28 && offsetof(WorkRec, m0) == 32 && offsetof(WorkRec, ke) == 48,
              "work record layout");

struct Workspace {
  int32_t* key;      // [n] cell of a row in a cell with edges (sorted by it), -1 for rows settled by k_agg_prep
  double* lpos;      // [2n] body-frame positions
  int32_t* counts;   // [nbk + 1]   } zeroed together (buckets: the cells with edges, by compact index)
  int32_t* cursor;   // [nbk]       }
  int32_t* offs;     // [nbk + 1] exclusive prefix sums of counts
  int32_t* order;    // [n] rows sorted by bucket
  double* ind;       // [n] indicator of a row (by row index)
  int32_t* flag;     // [n] 0 not a candidate, 1 candidate without neighbour pairs, 2 row with pairs (by row index)
  int32_t* rkey;     // [n] count key of a sorted row: 63 - min(pairs, 63) for rows with pairs, 64 otherwise
  uint64_t* mask;    // [2n] by sorted row: bit k set when candidate k (< kMaskBits) of the row's cell is a neighbour
  int32_t* khist;    // [kKeys] rows per key   } zeroed together
  int32_t* kcur;     // [kKeys] fill cursors   }
  WorkRec* wrec;     // [n] work rows by decreasing pair count (slots < nwork used)
  int32_t* nwork;    // [1] number of rows with pairs
  size_t total;
  // optional staging region after `total` (a workspace of total + staging bytes): the channel sums of every work row,
  // [slot][kernel][12], written by the pair pass and expanded to the outputs by k_agg_expand; nullptr without it
  double* wacc;
  size_t staging;
};

static Workspace carve(const Surface* s, int64_t n, void* base) {
  Workspace w{};
  const int64_t nbk = (int64_t)s->n_nonempty + 2;   // buckets: the cells with edges
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += align256(bytes);
    return (char*)base + o;
  };
  w.key = (int32_t*)take(sizeof(int32_t) * std::max<int64_t>(n, 1));
  w.lpos = (double*)take(sizeof(double) * 2 * std::max<int64_t>(n, 1));
  w.counts = (int32_t*)take(sizeof(int32_t) * (2 * nbk + 1));
  w.cursor = w.counts + nbk + 1;
  w.offs = (int32_t*)take(sizeof(int32_t) * (nbk + 1));
  w.order = (int32_t*)take(sizeof(int32_t) * std::max<int64_t>(n, 1));
  w.ind = (double*)take(sizeof(double) * std::max<int64_t>(n, 1));
  w.flag = (int32_t*)take(sizeof(int32_t) * std::max<int64_t>(n, 1));
  w.rkey = (int32_t*)take(sizeof(int32_t) * std::max<int64_t>(n, 1));
  w.mask = (uint64_t*)take(sizeof(uint64_t) * 2 * std::max<int64_t>(n, 1));
  w.khist = (int32_t*)take(sizeof(int32_t) * 2 * kKeys);
  w.kcur = w.khist + kKeys;
  w.wrec = (WorkRec*)take(sizeof(WorkRec) * std::max<int64_t>(n, 1));
  w.nwork = (int32_t*)take(sizeof(int32_t));
  w.total = off;
  w.staging = align256(sizeof(double) * 12 * kMaxPackStaged * std::max<int64_t>(n, 1));
  w.wacc = nullptr;
  return w;
}

// the staging region when the workspace holds it (workspace_bytes >= total + staging) and it starts on a 32-byte
// boundary (the expansion reads it by 32-byte loads); otherwise the evaluation stores its outputs directly
static void attach_staging(Workspace& w, void* base, size_t workspace_bytes) {
  char* p = base ? (char*)base + w.total : nullptr;
  w.wacc = (p && workspace_bytes >= w.total + w.staging && ((uintptr_t)p & 31u) == 0) ? (double*)p : nullptr;
}

// body-frame position (bit-for-bit Pose.toLocal), broadphase (fixedadj.py:257-265) and the bucket of every row
__global__ void k_agg_prep(SurfView S, const double* __restrict__ pos, const double* __restrict__ sup,
                           const int32_t* __restrict__ allowed, int64_t n, const double* __restrict__ pose,
                           double4 obb, int unbounded, int32_t* __restrict__ key, double* __restrict__ lpos,
                           int32_t* __restrict__ counts, double* __restrict__ ind, int32_t* __restrict__ flag) {
  pdl_wait();      // the preceding kernel of the stream has completed and its writes are visible
  pdl_trigger();   // the next kernel of the stream may be scheduled into the SMs this grid frees
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double lx, ly;
  to_local_rn(pos[2 * i], pos[2 * i + 1], pose[0], pose[1], pose[2], pose[3], lx, ly);
  lpos[2 * i] = lx;
  lpos[2 * i + 1] = ly;
  const int32_t ncells = S.nx * S.ny;
  bool valid = allowed ? (allowed[i] != 0) : true;
  if (valid && !unbounded) {
    const double dx = __dadd_rn(fmax(__dsub_rn(obb.x, lx), 0.0), fmax(__dsub_rn(lx, obb.z), 0.0));
    const double dy = __dadd_rn(fmax(__dsub_rn(obb.y, ly), 0.0), fmax(__dsub_rn(ly, obb.w), 0.0));
    valid = __dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy))) < sup[i];
  }
  int32_t b;
  if (!valid) {
    b = ncells + 1;
  } else {
    int32_t cid;
    b = cell_of(S, lx, ly, cid) ? cid : ncells;
  }
  if (b < ncells && S.cempty[b] == 0) {        // a cell with candidates: the row is sorted and row info takes it
    key[i] = b;
    atomicAdd(&counts[S.ccompact[b]], 1);        // bucketed by the cell's index among the cells with edges
    return;
  }
  // no candidates: not a candidate of the body (flag 0), outside the grid (the background), or an edge-free cell, whose
  // cached centre winding is the indicator of all its points; these rows never enter the sort
  key[i] = -1;
  flag[i] = b == ncells + 1 ? 0 : 1;
  ind[i] = b == ncells + 1 ? 0.0 : (b == ncells ? S.background : S.cind[b]);
}

__global__ void k_agg_scatter(SurfView S, const int32_t* __restrict__ key, int64_t n, const int32_t* __restrict__ offs,
                              int32_t* __restrict__ cursor, int32_t* __restrict__ order) {
  pdl_wait();      // the preceding kernel of the stream has completed and its writes are visible
  pdl_trigger();   // the next kernel of the stream may be scheduled into the SMs this grid frees
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t b = key[i];
  if (b >= 0) {
    const int32_t c = S.ccompact[b];
    order[offs[c] + atomicAdd(&cursor[c], 1)] = (int32_t)i;
  }
}

// index of the lowest set bit of the 128-bit mask (m0 low word), cleared; -1 when the mask is empty
__device__ __forceinline__ int pop_bit(uint64_t& m0, uint64_t& m1) {
  if (m0) {
    const int b = __ffsll((long long)m0) - 1;
    m0 &= m0 - 1;
    return b;
  }
  if (m1) {
    const int b = 63 + __ffsll((long long)m1);
    m1 &= m1 - 1;
    return b;
  }
  return -1;
}

// one thread's channel accumulators in a [12][kThreads] shared array
struct SmemAcc {
  double* p;
  __device__ __forceinline__ double& operator[](int c) const { return p[c * kThreads]; }
};

// a work record by three 16-byte loads and one 4-byte load through the read-only path
__device__ __forceinline__ WorkRec load_workrec(const WorkRec* p) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(p));
  const longlong2 b = __ldg(reinterpret_cast<const longlong2*>(p) + 1);
  const ulonglong2 m = __ldg(reinterpret_cast<const ulonglong2*>(p) + 2);
  WorkRec r;
  r.lx = a.x;
  r.ly = a.y;
  r.h = __longlong_as_double(b.x);
  r.row = (int32_t)(uint32_t)((unsigned long long)b.y & 0xffffffffull);
  r.kb = (int32_t)(uint32_t)((unsigned long long)b.y >> 32);
  r.m0 = m.x;
  r.m1 = m.y;
  r.ke = __ldg(reinterpret_cast<const int32_t*>(p) + 12);
  return r;
}

// an asynchronous copy of a 32-byte record into shared memory (two 16-byte cp.async, L1-allocating) and the waits on it:
// the copy is in flight while the thread computes, without holding registers
__device__ __forceinline__ void cp_async_rec(double4* dst, const double4* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(d + 16), "l"(reinterpret_cast<const char*>(src) + 16)
               : "memory");
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// a 32-byte record through the read-only data path (two 16-byte loads)
__device__ __forceinline__ double4 ldg4(const double4* p) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(p)), b = __ldg(reinterpret_cast<const double2*>(p) + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

constexpr int kStageRecs = 768;   // candidate records a row-info block stages in shared memory (24 KiB)

// Per sorted row: its number of neighbour pairs (float-prefiltered exact predicate over its cell's candidates) as a
// radix key with the neighbour mask, and its winding indicator -- both kernel independent, computed once per position
// set.

__global__ void __launch_bounds__(kThreads) k_agg_rowinfo(SurfView S, const double* __restrict__ sup,
                                                         const int32_t* __restrict__ key,
                                                         const double* __restrict__ lpos,
                                                         const int32_t* __restrict__ offs,
                                                         const int32_t* __restrict__ order, int64_t n,
                                                         double* __restrict__ ind, int32_t* __restrict__ flag,
                                                         int32_t* __restrict__ rkey, uint64_t* __restrict__ mask,
                                                         int32_t* __restrict__ khist) {
  pdl_wait();      // the preceding kernel of the stream has completed and its writes are visible
  pdl_trigger();   // the next kernel of the stream may be scheduled into the SMs this grid frees
  // The block's rows are consecutive in cell order, so the candidates of all their cells are one contiguous range of
  // the cell-list records: it is staged in shared memory with coalesced loads when it fits, and every row's pass
  // over its cell's candidates reads it there.
  __shared__ double4 s_rec[kStageRecs];
  __shared__ int32_t s_lo, s_hi;
  __shared__ int32_t s_hist[kKeys - 1];
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (threadIdx.x == 0) {
    s_lo = INT32_MAX;
    s_hi = -1;
  }
  for (int k = threadIdx.x; k < kKeys - 1; k += kThreads) s_hist[k] = 0;
  // sorted rows: the rows in cells with candidates (k_agg_prep settles all others)
  int32_t i = 0, b = 0;
  const bool cand = j < (int64_t)offs[S.nne];
  if (cand) {
    i = order[j];
    b = key[i];
  }
  __syncthreads();
  if (cand) {
    atomicMin(&s_lo, b);
    atomicMax(&s_hi, b);
  }
  __syncthreads();
  int r0 = 0;
  bool staged = false;
  if (s_hi >= 0) {
    r0 = S.cstart[s_lo];
    const int r1 = S.cstart[s_hi + 1];
    staged = r1 - r0 <= kStageRecs;
    if (staged)
      for (int k = threadIdx.x; k < r1 - r0; k += kThreads) s_rec[k] = ldg4(S.crec + r0 + k);
  }
  __syncthreads();
  int cnt = 0;
  if (j < n) {
    if (cand) {
      const double lx = lpos[2 * i], ly = lpos[2 * i + 1], h = sup[i];
      // one pass over the cell's candidates: the neighbour count and the signed crossings of the segment from the
      // cell centre (whose exact winding is stored) to the row; an uncertain orientation falls back to the ray cast
      const int64_t cx = b / S.ny, cy = b % S.ny;
      const double rx = __dadd_rn(S.lo_x, __dmul_rn(__dadd_rn((double)cx, 0.5), S.cell));
      const double ry = __dadd_rn(S.lo_y, __dmul_rn(__dadd_rn((double)cy, 0.5), S.cell));
      bool degenerate = S.cok[b] == 0;
      int cross = 0;
      uint64_t m0 = 0, m1 = 0;
      const int k0 = S.cstart[b], k1 = S.cstart[b + 1];
      for (int k = k0; k < k1; ++k) {
        const double4 e = staged ? s_rec[k - r0] : ldg4(S.crec + k);
        if (seg_within_fast(lx, ly, e.x, e.y, e.z, e.w, h)) {
          ++cnt;
          const int r = k - k0;
          if (r < 64)
            m0 |= 1ull << r;
          else if (r < kMaskBits)
            m1 |= 1ull << (r - 64);
        }
        if (!degenerate) cross += segment_crossing(rx, ry, lx, ly, e, &degenerate);
      }
      reinterpret_cast<ulonglong2*>(mask)[j] = make_ulonglong2(m0, m1);
      const double w = degenerate ? indicator_at(S, lx, ly, h, true, b) : S.cind[b] + (double)cross;
      ind[i] = w;
      flag[i] = cnt > 0 ? 2 : 1;
    }
    rkey[j] = cnt > 0 ? 63 - min(cnt, 63) : kKeys - 1;
  }
  // histogram of the keys of the rows with pairs (the rows without are never scattered, so their key is not
  // counted): warp-aggregated into the block's counts, then one global add per key the block has -- a global atomic
  // per warp and key would serialise on the few hot keys of millions of rows
  const int ckey = j < n && cnt > 0 ? 63 - min(cnt, 63) : -1;
  const unsigned peers = __match_any_sync(0xffffffffu, ckey);
  if (ckey >= 0 && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&s_hist[ckey], __popc(peers));
  __syncthreads();
  for (int k = threadIdx.x; k < kKeys - 1; k += kThreads)
    if (s_hist[k]) atomicAdd(&khist[k], s_hist[k]);
}

template <int VEC = 0>
__device__ __forceinline__ void finish_row(double acc[12], double ind, double mass, double plane2, double h,
                                           const double* pose, int64_t i, bool assign, double* lam, double* G,
                                           double* cov, double* m1, double* m2) {
  acc[0] = __fma_rn(ind, mass, acc[0]);
  acc[5] = __fma_rn(ind, mass, acc[5]);
  acc[8] = __fma_rn(ind, mass, acc[8]);
  acc[9] = __fma_rn(ind, plane2, acc[9]);
  acc[11] = __fma_rn(ind, plane2, acc[11]);
  const double c = pose[2], s = pose[3];
  const double rot[4] = {c, -s, s, c};
  write_outputs<VEC>(acc, h, rot, i, lam, G, cov, m1, m2, assign);
}

// ------------------------------------------------------------------------------------------------ kernel packs
// A pack of kernel tables is evaluated in one pass over the neighbour pairs: the kernel groups of one aggregate, as
// FusedWall evaluates a tuple of groups in one launch family (src/warpSPHBoundaries/scene/fused.py:506-547,
// warpfused.fused_channels over every group).  The blocks of all the pack's kernels are grouped by support radius R;
// per pair the clipped chord, its special functions and its monomial integrals are formed once per distinct R (up to
// the highest power any block of that radius needs), then every (kernel, block) of that radius adds its chord sums
// into the kernel's own accumulators.  A pack of one kernel is the single-kernel evaluation.
template <int M>
struct PackRadii {
  double r[M];   // distinct block radii in first-seen order (pack order, then block order)
  int na[M];     // monomial integrals formed at each radius: the most any block of that radius uses
  int n;
};

template <int M>
constexpr void pack_radii_add(PackRadii<M>& a, const double* r, const int* na, int nb) {
  for (int b = 0; b < nb; ++b) {
    int d = 0;
    while (d < a.n && a.r[d] != r[b]) ++d;
    if (d == a.n) {
      a.r[d] = r[b];
      a.na[d] = na[b];
      ++a.n;
    } else if (na[b] > a.na[d]) {
      a.na[d] = na[b];
    }
  }
}

template <class... KTs>
constexpr PackRadii<(KTs::kBlocks + ...)> pack_radii() {
  PackRadii<(KTs::kBlocks + ...)> a{};
  (pack_radii_add(a, KTs::kR, KTs::kNA, KTs::kBlocks), ...);
  return a;
}

template <class... KTs>
struct KPack {
  static constexpr int kN = sizeof...(KTs);
  static constexpr auto kRadii = pack_radii<KTs...>();
  template <int K>
  using Kern = std::tuple_element_t<K, std::tuple<KTs...>>;
};

constexpr int kMaxPack = 4;

// output pointers of the pack's kernels, by pack position (NULL: not written)
struct PackOut {
  double* lam[kMaxPack];
  double* G[kMaxPack];
  double* cov[kMaxPack];
  double* m1[kMaxPack];
  double* m2[kMaxPack];
};

// resident CTAs of 128 threads per SM for a pack of n kernels: the 12 n float64 channel sums of a thread live in shared
// memory (12 KiB a kernel per CTA), at most 7 CTAs (measured on B200 with one kernel on the 2^20-particle scene:
// 12.2e9 pairs/s with 7 CTAs at 72 registers, 12.0e9 with 6 or 8, 11.6e9 with the sums in registers at 6 CTAs)
constexpr int pack_min_blocks(int n) {
  const int by_smem = (227 * 1024) / (12 * n * kThreads * 8 + 32 * kThreads + 1024);
  return by_smem < 7 ? by_smem : 7;
}

// every (kernel, block) of the pack whose radius is the D-th distinct radius: its chord sums into its accumulators
template <class Pack, int D, int K, int B>
__device__ __forceinline__ void pack_blocks_at(const PairGeo& g, double lo, double hi, const double* A, double rlo,
                                               double rhi, double dang, double* acc_t) {
  if constexpr (K < Pack::kN) {
    using KT = typename Pack::template Kern<K>;
    if constexpr (B < KT::kBlocks) {
      if constexpr (KT::kR[B] == Pack::kRadii.r[D]) {
        if constexpr (KT::kQuad) {
          // a quadrature kernel contributes its gradient channels only: G = -n int W ds (no indicator term, W and
          // W' vanish at the support edge)
          const double W0 = quad_chord<KT>(lo, hi, g.z);
          const SmemAcc a{acc_t + K * 12 * kThreads};
          a[3] -= g.n0 * W0;
          a[4] -= g.n1 * W0;
        } else {
          BlockSums S;
          KT::template sums<B>(A, rlo, rhi, S);
          add_block(g, S, dang, SmemAcc{acc_t + K * 12 * kThreads});
        }
      }
      pack_blocks_at<Pack, D, K, B + 1>(g, lo, hi, A, rlo, rhi, dang, acc_t);
    } else {
      pack_blocks_at<Pack, D, K + 1, 0>(g, lo, hi, A, rlo, rhi, dang, acc_t);
    }
  }
}

// one pair, every kernel of the pack: per distinct radius the clipped chord, special functions and monomials once
template <class Pack, int PREC, int D>
__device__ __forceinline__ void pack_pair(const PairGeo& g, double* acc_t) {
  if constexpr (D < Pack::kRadii.n) {
    constexpr double R = Pack::kRadii.r[D];
    constexpr int NA = Pack::kRadii.na[D];
    double lo, hi, rlo, rhi, zz;
    if (clip_chord(g, R, lo, hi, rlo, rhi, zz)) {
      double dasinh, dang;
      special_fns<PREC>(lo, hi, rlo, rhi, g.z, zz, dasinh, dang);
      double A[NA];
      chord_monomials<NA>(lo, hi, rlo, rhi, zz, dasinh, A);
      pack_blocks_at<Pack, D, 0, 0>(g, lo, hi, A, rlo, rhi, dang, acc_t);
    }
    pack_pair<Pack, PREC, D + 1>(g, acc_t);
  }
}

// ------------------------------------------------------------------------------------------------ the float route
// WSB_PREC_FP32: per (pair, support radius) the chord is clipped in float64 and its angle taken in float (float64 only
// where y leaves float's normal range); the four integrated profiles (P, Psi, M/r^2, MPsi/r^2) of every (kernel, block)
// at that radius are evaluated in float by Clenshaw's recurrence on their Chebyshev series on [0, R] and integrated by
// 8-node Gauss-Legendre on panels graded from the foot of the perpendicular -- 0, |z|, 2|z|, 4|z|, ... up to the
// chord end, the reference's stable route (src/warpSPHBoundaries/edge/warpbc.py:519-575) without its cap on the
// panel count -- the node radius shared by every block of the pack; the odd chord sums come from the potentials M,
// MPsi at the chord ends; the edge-frame combination and the row sums stay in float64.  The tensile (quadrature)
// kernels keep their float64 chord quadrature.  Float slot of (kernel K, block B): K * kF32MaxBlocks + B.
constexpr int kF32MaxBlocks = 3;

template <class Pack, int D, int K, int B>
__device__ __forceinline__ void f32_node(float x, float w, float* q) {
  if constexpr (K < Pack::kN) {
    using KT = typename Pack::template Kern<K>;
    if constexpr (B < KT::kBlocks) {
      if constexpr (!KT::kQuad && KT::kR[B] == Pack::kRadii.r[D]) {
        static_assert(B < kF32MaxBlocks, "blocks per kernel");
        constexpr int o = 4 * (K * kF32MaxBlocks + B);
        float P, Psi, Fl, Fp;
        ChebOf<KT>::template integrands<B>(x, P, Psi, Fl, Fp);
        q[o] = fmaf(w, P, q[o]);
        q[o + 1] = fmaf(w, Psi, q[o + 1]);
        q[o + 2] = fmaf(w, Fl, q[o + 2]);
        q[o + 3] = fmaf(w, Fp, q[o + 3]);
      }
      f32_node<Pack, D, K, B + 1>(x, w, q);
    } else {
      f32_node<Pack, D, K + 1, 0>(x, w, q);
    }
  }
}

template <class Pack, int D, int K, int B>
__device__ __forceinline__ void f32_finish(const PairGeo& g, const float* q, double lo, double hi, double rlo,
                                           double rhi, double dang, double* acc_t) {
  if constexpr (K < Pack::kN) {
    using KT = typename Pack::template Kern<K>;
    if constexpr (B < KT::kBlocks) {
      if constexpr (KT::kR[B] == Pack::kRadii.r[D]) {
        const SmemAcc a{acc_t + K * 12 * kThreads};
        if constexpr (KT::kQuad) {
          const double W0 = quad_chord<KT>(lo, hi, g.z);
          a[3] -= g.n0 * W0;
          a[4] -= g.n1 * W0;
        } else {
          constexpr int o = 4 * (K * kF32MaxBlocks + B);
          constexpr float s2R = (float)(2.0 / KT::kR[B]);
          float Mh, MPh, Ml, MPl;
          ChebOf<KT>::template potentials<B>(fminf(fmaf((float)rhi, s2R, -1.0f), 1.0f), Mh, MPh);
          ChebOf<KT>::template potentials<B>(fminf(fmaf((float)rlo, s2R, -1.0f), 1.0f), Ml, MPl);
          BlockSums S;
          S.W0 = (double)q[o];
          S.P0 = (double)q[o + 1];
          S.Lreg = (double)q[o + 2];
          S.Preg = (double)q[o + 3];
          S.W1 = (double)Mh - (double)Ml;
          S.P1 = (double)MPh - (double)MPl;
          S.Mhat = ChebOf<KT>::kMhat[B];
          S.MPhat = ChebOf<KT>::kMPhat[B];
          add_block(g, S, dang, a);
        }
      }
      f32_finish<Pack, D, K, B + 1>(g, q, lo, hi, rlo, rhi, dang, acc_t);
    } else {
      f32_finish<Pack, D, K + 1, 0>(g, q, lo, hi, rlo, rhi, dang, acc_t);
    }
  }
}

template <class Pack, int D>
__device__ __forceinline__ void pack_pair_f32(const PairGeo& g, double* acc_t) {
  if constexpr (D < Pack::kRadii.n) {
    constexpr double R = Pack::kRadii.r[D];
    double lo, hi, rlo, rhi, zz;
    if (clip_chord(g, R, lo, hi, rlo, rhi, zz)) {
      double dang = 0.0;
      if (g.z != 0.0) {
        const double y = g.z * (hi - lo), x = zz + lo * hi;
        dang = fabs(y) >= kMixedGuardY ? (double)atan2f((float)y, (float)x)
                                       : ((y == 0.0 && x == 0.0) ? 0.0 : atan2(y, x));
      }
      constexpr int kSlots = 4 * Pack::kN * kF32MaxBlocks;
      float q[kSlots];
#pragma unroll
      for (int i = 0; i < kSlots; ++i) q[i] = 0.0f;
      const float az = (float)fabs(g.z), zzf = az * az;
      constexpr float s2R = (float)(2.0 / R);
      for (int side = 0; side < 2; ++side) {
        const float u0 = (float)(side == 0 ? fmax(-hi, 0.0) : fmax(lo, 0.0));
        const float u1 = (float)(side == 0 ? -lo : hi);
        if (!(u1 > u0)) continue;
        // panels [0, |z|], [|z|, 2|z|], ... (the first breakpoint at least 2^-30 of the side's length: nearer the foot
        // the integrand differs from its z = 0 polynomial by O(z^2)); z = 0 integrates a polynomial in s: one panel
        float d = az > 0.0f ? fmaxf(az, u1 * 0x1p-30f) : u1;
        for (int it = 0; it < 40 && d <= u0; ++it) d *= 2.0f;
        float u = u0;
        for (int it = 0; it < 40 && u < u1; ++it) {
          const float nxt = fminf(u1, d);
          const float hc = 0.5f * (nxt - u), mc = 0.5f * (nxt + u);
#pragma unroll
          for (int k = 0; k < kF32Gauss; ++k) {
            const float s = fmaf(hc, kF32Gx[k], mc);
            const float r = sqrtf(fmaf(s, s, zzf));
            const float x = fminf(fmaf(r, s2R, -1.0f), 1.0f);
            f32_node<Pack, D, 0, 0>(x, hc * kF32Gw[k], q);
          }
          if (nxt >= d) d *= 2.0f;
          u = nxt;
        }
      }
      f32_finish<Pack, D, 0, 0>(g, q, lo, hi, rlo, rhi, dang, acc_t);
    }
    pack_pair_f32<Pack, D + 1>(g, acc_t);
  }
}

// the outputs of a row of a quadrature kernel: its gradient channels G (scaled, rotated); the other outputs are not
// defined for it and are written as NaN
template <int VEC = 0>
__device__ __forceinline__ void finish_row_quad(const double acc[12], double h, const double* pose, int64_t i,
                                                bool assign, double* lam, double* G, double* cov, double* m1,
                                                double* m2) {
  const double c = pose[2], s = pose[3], nan = __longlong_as_double(0x7ff8000000000000LL);
  if (lam) put(&lam[i], nan, assign);
  if (G) {
    const double vx = __ddiv_rn(acc[3], h), vy = __ddiv_rn(acc[4], h);
    if constexpr (VEC > 0) {
      put2(&G[2 * i], dot2(c, vx, -s, vy), dot2(s, vx, c, vy), assign);
    } else {
      put(&G[2 * i], dot2(c, vx, -s, vy), assign);
      put(&G[2 * i + 1], dot2(s, vx, c, vy), assign);
    }
  }
  for (int k = 0; k < 4; ++k) {
    if (cov) put(&cov[4 * i + k], nan, assign);
    if (m2) put(&m2[4 * i + k], nan, assign);
  }
  if (m1) {
    put(&m1[2 * i], nan, assign);
    put(&m1[2 * i + 1], nan, assign);
  }
}

// a row without neighbour pairs, every kernel of the pack: the indicator w times the whole-plane channels (w = 0 for
// a non-candidate when the outputs are assigned)
template <class Pack, int K, int VEC = 0>
__device__ __forceinline__ void pack_constant_row(int64_t i, double w, double h, const double* pose, bool assign,
                                                  const PackOut& o) {
  if constexpr (K < Pack::kN) {
    using KT = typename Pack::template Kern<K>;
    double acc[12];
#pragma unroll
    for (int c = 0; c < 12; ++c) acc[c] = 0.0;
    if constexpr (KT::kQuad)
      finish_row_quad<VEC>(acc, h, pose, i, assign, o.lam[K], o.G[K], o.cov[K], o.m1[K], o.m2[K]);
    else
      finish_row<VEC>(acc, w, KT::kMass, KT::kPlane2, h, pose, i, assign, o.lam[K], o.G[K], o.cov[K], o.m1[K],
                      o.m2[K]);
    pack_constant_row<Pack, K + 1, VEC>(i, w, h, pose, assign, o);
  }
}

// a work row, every kernel of the pack: the G lanes' sums combined by an xor butterfly (every lane of the warp takes
// part), then the lane that writes adds the indicator terms and stores the outputs
template <class Pack, int G, int K>
__device__ __forceinline__ void pack_finish(const double* acc_t, bool write, int64_t i, double w, double h,
                                            const double* pose, bool assign, const PackOut& o) {
  if constexpr (K < Pack::kN) {
    using KT = typename Pack::template Kern<K>;
    double acc[12];
#pragma unroll
    for (int c = 0; c < 12; ++c) acc[c] = acc_t[(K * 12 + c) * kThreads];
#pragma unroll
    for (int off = 1; off < G; off <<= 1) {
#pragma unroll
      for (int c = 0; c < 12; ++c) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], off);
    }
    if (write) {
      // a rounded multiply of its own (no contraction with the indicator terms), as the staged path stores the sums
#pragma unroll
      for (int c = 0; c < 12; ++c) acc[c] = __dmul_rn(acc[c], kInvPi);
      if constexpr (KT::kQuad)
        finish_row_quad(acc, h, pose, i, assign, o.lam[K], o.G[K], o.cov[K], o.m1[K], o.m2[K]);
      else
        finish_row(acc, w, KT::kMass, KT::kPlane2, h, pose, i, assign, o.lam[K], o.G[K], o.cov[K], o.m1[K], o.m2[K]);
    }
    pack_finish<Pack, G, K + 1>(acc_t, write, i, w, h, pose, assign, o);
  }
}

// a work row's channel sums (the G lanes' sums by the xor butterfly, x 1/pi) into its staging slot [kernel][12]
template <class Pack, int G, int K>
__device__ __forceinline__ void pack_stage(const double* acc_t, bool write, double* dst) {
  if constexpr (K < Pack::kN) {
    double acc[12];
#pragma unroll
    for (int c = 0; c < 12; ++c) acc[c] = acc_t[(K * 12 + c) * kThreads];
#pragma unroll
    for (int off = 1; off < G; off <<= 1) {
#pragma unroll
      for (int c = 0; c < 12; ++c) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], off);
    }
    if (write) {
      double2* d2 = reinterpret_cast<double2*>(dst + K * 12);
#pragma unroll
      for (int c = 0; c < 6; ++c) d2[c] = make_double2(__dmul_rn(acc[2 * c], kInvPi), __dmul_rn(acc[2 * c + 1], kInvPi));
    }
    pack_stage<Pack, G, K + 1>(acc_t, write, dst);
  }
}

// Rows with neighbour pairs (compacted, by decreasing pair count), then the rows without: the first
// ceil(nwork G / kThreads) blocks take the work rows, the next ceil(n / kThreads) blocks the constant rows (one row a
// thread, coalesced), so the constant rows' stores overlap the last wave of pair blocks instead of running as a launch
// of their own; the grid is sized for nwork = n and blocks past both ranges return.  A group of G adjacent lanes owns
// one work row and splits its neighbours: the row's neighbour mask (set by k_agg_rowinfo) lists them among the first
// kMaskBits candidates of its cell, and lane g takes those of rank g, g + G, ... in candidate order; candidates past
// the mask are split g, g + G, ... and found by the float-prefiltered predicate.  Work rows are sorted by pair count,
// so the lanes of a warp evaluate nearly the same number of closed forms.  The G partial sums are combined by an xor
// butterfly (the same additions on every lane, commutative, so the result is deterministic and identical on the G
// lanes).  The channel sums live in shared memory ([kernel][channel][thread]), which keeps the registers for the
// closed form.
template <class Pack, int PREC, int G, int MINB, bool STAGED>
__global__ void __launch_bounds__(kThreads, MINB) k_agg_pairs(SurfView S, const double* __restrict__ sup,
                                                             const WorkRec* __restrict__ wrec,
                                                             const int32_t* __restrict__ nwork_p, int64_t n,
                                                             const double* __restrict__ ind,
                                                             const int32_t* __restrict__ flag,
                                                             const double* __restrict__ pose, bool assign,
                                                             const PackOut out, double* __restrict__ wacc) {
  pdl_wait();      // the preceding kernel of the stream has completed and its writes are visible
  pdl_trigger();   // the next kernel of the stream may be scheduled into the SMs this grid frees
  static_assert(G == 1 || G == 2 || G == 4 || G == 8 || G == 16, "lanes per row");
  static_assert(Pack::kN >= 1 && Pack::kN <= kMaxPack, "pack size");
  // dynamic shared memory: the channel sums [kernel][channel][thread], then each thread's next edge record
  extern __shared__ double4 s_dyn[];
  double* const s_acc = reinterpret_cast<double*>(s_dyn + kThreads);
  double4* const s_next = s_dyn;
  const int64_t nwork = *nwork_p;
  const int64_t wblocks = (nwork + kThreads / G - 1) / (kThreads / G);
  if ((int64_t)blockIdx.x >= wblocks) {                             // a tail block: constant rows
    if constexpr (STAGED) return;                                   // (staged: k_agg_expand writes every row)
    const int64_t i = ((int64_t)blockIdx.x - wblocks) * kThreads + threadIdx.x;
    if (i < n) {
      const int32_t f = flag[i];
      if (f == 1 || (f == 0 && assign)) pack_constant_row<Pack, 0>(i, f == 1 ? ind[i] : 0.0, sup[i], pose, assign, out);
    }
    return;
  }
  const int64_t w = (int64_t)blockIdx.x * (blockDim.x / G) + threadIdx.x / G;
  const int sub = threadIdx.x % G;
  const bool ok = w < nwork;
  int32_t i = 0;
  int kb = 0, kt = 0, e1 = 0;
  uint64_t mk0 = 0, mk1 = 0;
  double lx = 0.0, ly = 0.0, h = 1.0;
  if (ok) {
    const WorkRec r = load_workrec(wrec + w);
    i = r.row;
    lx = r.lx;
    ly = r.ly;
    h = r.h;
    kb = r.kb;
    e1 = r.ke;
    kt = kb + kMaskBits + sub;                                      // past the mask: lane sub scans kt, kt + G, ...
    mk0 = r.m0;
    mk1 = r.m1;
  }
  // lane sub takes the neighbours of rank sub, sub + G, ... of the mask (in candidate order), then its share of the
  // candidates past the mask by the predicate
  for (int s = 0; s < sub; ++s) pop_bit(mk0, mk1);
  int nb = pop_bit(mk0, mk1);
  const double ih = 1.0 / h;
  double* const acc_t = s_acc + threadIdx.x;
#pragma unroll
  for (int c = 0; c < Pack::kN * 12; ++c) acc_t[c * kThreads] = 0.0;
  // the next neighbour's (or tail candidate's) record is copied into the thread's shared-memory slot one step ahead
  // (cp.async), so its latency hides behind the current pair's closed form
  const double4 zero = make_double4(0.0, 0.0, 0.0, 0.0);
  double4* const slot = s_next + threadIdx.x;
  if (nb >= 0)
    cp_async_rec(slot, S.crec + kb + nb);
  else if (kt < e1)
    cp_async_rec(slot, S.crec + kt);
  while (__any_sync(0xffffffffu, nb >= 0 || kt < e1)) {
    double4 e = zero;
    bool have = false;
    if (nb >= 0) {
      cp_async_wait_all();
      e = *slot;
      have = true;
      for (int s = 1; s < G; ++s) pop_bit(mk0, mk1);
      nb = pop_bit(mk0, mk1);
      if (nb >= 0)
        cp_async_rec(slot, S.crec + kb + nb);
      else if (kt < e1)
        cp_async_rec(slot, S.crec + kt);
    } else {
      while (kt < e1) {
        cp_async_wait_all();
        e = *slot;
        kt += G;
        if (kt < e1) cp_async_rec(slot, S.crec + kt);
        if (seg_within_fast(lx, ly, e.x, e.y, e.z, e.w, h)) {
          have = true;
          break;
        }
      }
    }
    __syncwarp();
    if (have) {
      PairGeo g;
      if (pair_geo_row(lx, ly, h, ih, e, g)) {
        if constexpr (PREC == WSB_PREC_FP32)
          pack_pair_f32<Pack, 0>(g, acc_t);
        else
          pack_pair<Pack, PREC, 0>(g, acc_t);
      }
    }
  }
  const bool write = ok && sub == 0;
  if constexpr (STAGED)
    pack_stage<Pack, G, 0>(acc_t, write, wacc + w * (Pack::kN * 12));
  else
    pack_finish<Pack, G, 0>(acc_t, write, i, write ? ind[i] : 0.0, h, pose, assign, out);
}

// Staged expansion: one thread per row, consecutive rows in consecutive threads, so every output array is written in
// full coalesced sectors -- a work row's outputs from its staged channel sums (key[i] is its work slot), any other row
// the indicator times the whole-plane channels.  A work row's outputs, every kernel of the pack, from its staged sums
// (already loaded: a[kernel * 12 + c]).
template <class Pack, int K, int VEC>
__device__ __forceinline__ void pack_expand_row(const double* a, int64_t i, double w, double h, const double* pose,
                                                bool assign, const PackOut& o) {
  if constexpr (K < Pack::kN) {
    using KT = typename Pack::template Kern<K>;
    double acc[12];
#pragma unroll
    for (int c = 0; c < 12; ++c) acc[c] = a[K * 12 + c];
    if constexpr (KT::kQuad)
      finish_row_quad<VEC>(acc, h, pose, i, assign, o.lam[K], o.G[K], o.cov[K], o.m1[K], o.m2[K]);
    else
      finish_row<VEC>(acc, w, KT::kMass, KT::kPlane2, h, pose, i, assign, o.lam[K], o.G[K], o.cov[K], o.m1[K],
                      o.m2[K]);
    pack_expand_row<Pack, K + 1, VEC>(a, i, w, h, pose, assign, o);
  }
}

// a work row's staged sums, every kernel: 3 Pack::kN 32-byte loads issued together (a row's slot is 96 bytes a
// kernel, 32-byte aligned: each load reads one whole sector), so their latencies overlap instead of each kernel's
// loads following the previous kernel's stores (measured on B200, four-kernel pack on the 2^20-particle scene: the
// expansion from 148 to 140 us)
template <class Pack>
__device__ __forceinline__ void load_staged(const double* src, double* a) {
#pragma unroll
  for (int c = 0; c < Pack::kN * 3; ++c) ld4_nc(src + 4 * c, a[4 * c], a[4 * c + 1], a[4 * c + 2], a[4 * c + 3]);
}

// VEC (write_outputs): 2 when G / m1 are 16-byte and cov / m2 32-byte aligned, so every store of a warp writes whole
// 32-byte sectors (no read-modify-write of partly written sectors); 1 when all are 16-byte aligned; 0 otherwise
// (121 registers, 4 CTAs per SM: capping the registers at 5 / 6 / 8 CTAs measured 0.340 / 0.356 / 0.390 ms for the
// grouped pass on the 2^20-particle scene against 0.306 ms -- the spilled staged sums cost more than the occupancy
// gains)
template <class Pack, int VEC>
__global__ void __launch_bounds__(kThreads) k_agg_expand(const double* __restrict__ sup,
                                                         const int32_t* __restrict__ flag,
                                                         const double* __restrict__ ind,
                                                         const int32_t* __restrict__ slot,
                                                         const double* __restrict__ wacc, int64_t n,
                                                         const double* __restrict__ pose, bool assign,
                                                         const PackOut out) {
  pdl_wait();      // the preceding kernel of the stream has completed and its writes are visible
  pdl_trigger();   // the next kernel of the stream may be scheduled into the SMs this grid frees
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int32_t f = flag[i];
  if (f == 0 && !assign) return;                                   // not a candidate, outputs added to: nothing
  // one code path for every row, so a warp issues each of its output stores once (work and constant rows of a warp
  // in separate branches would store every sector twice with partial masks): a constant row is a work row with zero
  // sums and the same finish (the indicator terms, w = 0 for a non-candidate)
  double a[Pack::kN * 12];
#pragma unroll
  for (int c = 0; c < Pack::kN * 12; ++c) a[c] = 0.0;
  if (f == 2) load_staged<Pack>(wacc + (int64_t)slot[i] * (Pack::kN * 12), a);
  pack_expand_row<Pack, 0, VEC>(a, i, f != 0 ? ind[i] : 0.0, sup[i], pose, assign, out);
}

static int pack_out_vec(const PackOut& o, int n) {
  auto al = [](const double* p, uintptr_t a) { return p == nullptr || ((uintptr_t)p & (a - 1)) == 0; };
  bool v16 = true, v32 = true;
  for (int k = 0; k < n; ++k) {
    v16 = v16 && al(o.G[k], 16) && al(o.m1[k], 16) && al(o.cov[k], 16) && al(o.m2[k], 16);
    v32 = v32 && al(o.cov[k], 32) && al(o.m2[k], 32);
  }
  return v16 ? (v32 ? 2 : 1) : 0;
}

// the pair kernel of a pack over a prepared workspace (two lanes per work row: measured fastest on the 2^20-particle
// scene, 1 / 2 lanes give 10.4 / 11.3e9 pairs/s with one kernel, 1 / 2 / 4 lanes 0.448 / 0.421 / 0.471 ms for the
// four-kernel pack, which also beat the four kernels as two two-kernel packs, 0.426 ms)
// instrumentation: events recorded on the launching stream right before and after each fused pair kernel (set by
// wsb_set_pair_events; NULL: none)
static cudaEvent_t g_pair_ev[2] = {nullptr, nullptr};

template <class Pack>
constexpr size_t pack_smem_bytes() {
  return sizeof(double4) * kThreads + sizeof(double) * Pack::kN * 12 * kThreads;
}

template <class Pack, int PREC>
static int launch_pack(const SurfView& v, const double* sup, const Workspace& w, int64_t n, const double* pose,
                       bool assign, const PackOut& out, cudaStream_t st) {
  constexpr int G = 2;
  constexpr size_t smem = pack_smem_bytes<Pack>();
  const bool staged = w.wacc != nullptr;
  auto kern = staged ? k_agg_pairs<Pack, PREC, G, pack_min_blocks(Pack::kN), true>
                     : k_agg_pairs<Pack, PREC, G, pack_min_blocks(Pack::kN), false>;
  if (smem > 48 * 1024) {       // above the default limit: opt in once per device for this instantiation
    static std::atomic<uint64_t> opted[2] = {{0}, {0}};
    int dev = 0;
    WSB_CUDA(cudaGetDevice(&dev));
    const uint64_t bit = 1ull << (dev & 63);
    if (!(opted[staged].load() & bit)) {
      WSB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      opted[staged].fetch_or(bit);
    }
  }
  const unsigned rows = (unsigned)((n + kThreads - 1) / kThreads);
  const unsigned grid = (unsigned)((n * G + kThreads - 1) / kThreads) + (staged ? 0u : rows);
  if (g_pair_ev[0]) WSB_CUDA(cudaEventRecord(g_pair_ev[0], st));
  WSB_CUDA(launch_dep(kern, grid, kThreads, smem, st, v, sup, (const WorkRec*)w.wrec, (const int32_t*)w.nwork, n,
                      (const double*)w.ind, (const int32_t*)w.flag, pose, assign, out, w.wacc));
  if (g_pair_ev[1]) WSB_CUDA(cudaEventRecord(g_pair_ev[1], st));
  if (staged) {
    const int vec = pack_out_vec(out, Pack::kN);
    if (vec == 2)
      WSB_CUDA(launch_dep(k_agg_expand<Pack, 2>, rows, kThreads, 0, st, sup, (const int32_t*)w.flag,
                          (const double*)w.ind, (const int32_t*)w.key, (const double*)w.wacc, n, pose, assign, out));
    else if (vec == 1)
      WSB_CUDA(launch_dep(k_agg_expand<Pack, 1>, rows, kThreads, 0, st, sup, (const int32_t*)w.flag,
                          (const double*)w.ind, (const int32_t*)w.key, (const double*)w.wacc, n, pose, assign, out));
    else
      WSB_CUDA(launch_dep(k_agg_expand<Pack, 0>, rows, kThreads, 0, st, sup, (const int32_t*)w.flag,
                          (const double*)w.ind, (const int32_t*)w.key, (const double*)w.wacc, n, pose, assign, out));
  }
  return WSB_OK;
}

// ------------------------------------------------------------------------------------------------ adjoint
// d/dx and d/dvertex of lam, m1, m2 by recomputation of the chord integrals int s^j W ds (j <= 3) of every neighbour
// pair: grad_x m_alpha = -sum_e n_e int y^alpha W ds, d m_alpha / d p_e = n_e int (1 - tau) y^alpha W ds,
// d m_alpha / d q_e = n_e int tau y^alpha W ds (np2d.py:554-565, 626-652)
template <class KT, int B>
__device__ __forceinline__ void adj_blocks(const PairGeo& g, AdjSums& tot) {
  if constexpr (B < KT::kBlocks) {
    AdjSums o;
    if (block_adjoint<KT, B>(g, o)) {
      tot.W0 += o.W0;
      tot.W1 += o.W1;
      tot.W2 += o.W2;
      tot.W3 += o.W3;
    }
    adj_blocks<KT, B + 1>(g, tot);
  }
}

// G lanes per work row split its neighbours (lane g takes the neighbours of rank g, g + G, ... of the row's mask, then
// candidates past the mask g, g + G, ... by the float-prefiltered predicate, exact where the float decision is within
// its margin); their d_pos partial sums are combined by a fixed xor butterfly
template <class KT, int G>
__global__ void __launch_bounds__(kThreads) k_agg_backward(SurfView S, const double* __restrict__ sup,
                                                          const WorkRec* __restrict__ wrec,
                                                          const int32_t* __restrict__ nwork_p, int64_t n,
                                                          const double* __restrict__ pose,
                                                          const double* __restrict__ g_lam,
                                                          const double* __restrict__ g_m1,
                                                          const double* __restrict__ g_m2, double* d_pos,
                                                          double* d_verts) {
  const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / G;
  const int sub = threadIdx.x % G;
  const bool ok = w < n && w < (int64_t)*nwork_p;    // work rows only (rows with neighbour pairs)
  WorkRec r{};
  if (ok) r = load_workrec(wrec + w);
  const int32_t i = ok ? r.row : 0;
  const double lx = ok ? r.lx : 0.0, ly = ok ? r.ly : 0.0, h = ok ? r.h : 1.0;
  const double c = pose[2], s = pose[3];
  // upstream gradients in the body frame and in channel units: m1_world = R m1, m2_world = R m2 R^T
  const double gl = g_lam && ok ? g_lam[i] : 0.0;
  double g10 = 0.0, g01 = 0.0, g20 = 0.0, g11 = 0.0, g02 = 0.0;
  if (g_m1 && ok) {
    const double wx = g_m1[2 * i], wy = g_m1[2 * i + 1];
    g10 = c * wx + s * wy;
    g01 = -s * wx + c * wy;
  }
  if (g_m2 && ok) {
    const double a = g_m2[4 * i], bb = g_m2[4 * i + 1], cc = g_m2[4 * i + 2], d = g_m2[4 * i + 3];
    // GL = R^T Gw R with R = [[c, -s], [s, c]]
    const double t00 = c * a + s * cc, t01 = c * bb + s * d, t10 = -s * a + c * cc, t11 = -s * bb + c * d;
    const double l00 = t00 * c + t01 * s, l01 = -t00 * s + t01 * c, l10 = t10 * c + t11 * s, l11 = -t10 * s + t11 * c;
    g20 = l00;
    g11 = l01 + l10;
    g02 = l11;
  }
  // physical units: d m_alpha = h^(|alpha| - 1) / pi * (unit integral)
  const double u0 = gl / h, u1x = g10, u1y = g01, u2x = g20 * h, u2m = g11 * h, u2y = g02 * h;
  double dx = 0.0, dy = 0.0;
  // the row's neighbours: lane sub takes ranks sub, sub + G, ... of the neighbour mask, then its share of the
  // candidates past the mask by the predicate
  const int kb = ok ? r.kb : 0, kend = ok ? r.ke : 0;
  int kt = kb + kMaskBits + sub;
  uint64_t mk0 = ok ? r.m0 : 0, mk1 = ok ? r.m1 : 0;
  for (int r = 0; r < sub; ++r) pop_bit(mk0, mk1);
  for (;;) {
    int k = pop_bit(mk0, mk1);
    if (k >= 0) {
      k += kb;
      for (int r = 1; r < G; ++r) pop_bit(mk0, mk1);
    } else {
      while (kt < kend) {
        const double4 c4 = S.crec[kt];
        const int kk = kt;
        kt += G;
        if (seg_within_fast(lx, ly, c4.x, c4.y, c4.z, c4.w, h)) {
          k = kk;
          break;
        }
      }
      if (k < 0) break;
    }
    const double4 e = S.crec[k];
    PairGeo g;
    if (!pair_geo_row(lx, ly, h, 1.0 / h, e, g)) continue;
    AdjSums W = {0.0, 0.0, 0.0, 0.0};
    adj_blocks<KT, 0>(g, W);
    const double z = g.z, zn0 = z * g.n0, zn1 = z * g.n1;
    // F = sum_alpha u_alpha y^alpha as a polynomial in s: F0 + F1 s + F2 s^2
    const double F0 = u0 + u1x * zn0 + u1y * zn1 + u2x * zn0 * zn0 + u2m * zn0 * zn1 + u2y * zn1 * zn1;
    const double F1 = u1x * g.t0 + u1y * g.t1 + 2.0 * u2x * zn0 * g.t0 + u2m * (zn0 * g.t1 + zn1 * g.t0) +
                      2.0 * u2y * zn1 * g.t1;
    const double F2 = u2x * g.t0 * g.t0 + u2m * g.t0 * g.t1 + u2y * g.t1 * g.t1;
    const double I0 = F0 * W.W0 + F1 * W.W1 + F2 * W.W2;     // int F W ds
    const double I1 = F0 * W.W1 + F1 * W.W2 + F2 * W.W3;     // int s F W ds
    dx -= g.n0 * I0;
    dy -= g.n1 * I0;
    if (d_verts) {
      const double ell = g.s1 - g.s0;
      const double a1 = (I1 - g.s0 * I0) / ell;              // int tau F W ds
      const double a0 = I0 - a1;                             // int (1 - tau) F W ds
      const int32_t ei = S.citems[k];
      const int v0 = S.edges[2 * ei], v1 = S.edges[2 * ei + 1];
      atomicAdd(&d_verts[2 * v0], kInvPi * g.n0 * a0);
      atomicAdd(&d_verts[2 * v0 + 1], kInvPi * g.n1 * a0);
      atomicAdd(&d_verts[2 * v1], kInvPi * g.n0 * a1);
      atomicAdd(&d_verts[2 * v1 + 1], kInvPi * g.n1 * a1);
    }
  }
#pragma unroll
  for (int off = 1; off < G; off <<= 1) {
    dx += __shfl_xor_sync(0xffffffffu, dx, off);
    dy += __shfl_xor_sync(0xffffffffu, dy, off);
  }
  if (!ok || sub != 0) return;
  dx *= kInvPi;
  dy *= kInvPi;
  // world frame: x_local = R^T (x - c)  =>  dL/dx = R dL/dx_local
  d_pos[2 * i] += c * dx - s * dy;
  d_pos[2 * i + 1] += s * dx + c * dy;
}

// ------------------------------------------------------------------------------------------------ signed distance
// the segment distance of a point to edge record r with the rounding of the reference's brute force; the nearest
// edge wins, the lower edge id on an exact tie (the order of a scan over all edges)
__device__ __forceinline__ void nearest_edge(double px, double py, const double4& r, int64_t e, double& best,
                                             double& bx, double& by, int64_t& be) {
  const double ex = __dsub_rn(r.z, r.x), ey = __dsub_rn(r.w, r.y);
  double t = __ddiv_rn(__dadd_rn(__dmul_rn(__dsub_rn(px, r.x), ex), __dmul_rn(__dsub_rn(py, r.y), ey)),
                       __dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)));
  t = fmin(fmax(t, 0.0), 1.0);
  const double cx = __dadd_rn(r.x, __dmul_rn(t, ex)), cy = __dadd_rn(r.y, __dmul_rn(t, ey));
  const double ddx = __dsub_rn(px, cx), ddy = __dsub_rn(py, cy);
  const double dist = __dsqrt_rn(__dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy)));
  if (dist < best || (dist == best && e < be)) {
    best = dist;
    bx = cx;
    by = cy;
    be = e;
  }
}

// Signed distance to the nearest edge.  Inside the cell grid the search visits square rings of cells around the
// point's cell: every edge is listed in each cell it passes through, so after ring k an edge not yet seen is farther
// than k cells and the search stops once the best distance is below that; outside the grid (farther than one
// support from every edge) all edges are scanned.  Same distances, closest points and edges as a scan over all edges.
__global__ void k_signed_distance(SurfView S, const double* __restrict__ lpos, int64_t m, double norm_support,
                                  double* d, double* cp, double* nl, int32_t* edge) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  const double px = lpos[2 * i], py = lpos[2 * i + 1];
  double best = INFINITY, bx = 0.0, by = 0.0;
  int64_t be = -1;
  int32_t cid;
  const bool in_grid = cell_of(S, px, py, cid);
  if (in_grid) {
    const int cx = cid / S.ny, cy = cid % S.ny;
    const int kmax = max(S.nx, S.ny);
    auto scan_cell = [&](int x, int y) {
      const int32_t c = x * S.ny + y;
      for (int32_t k = S.cstart[c]; k < S.cstart[c + 1]; ++k) nearest_edge(px, py, ldg4(S.crec + k), S.citems[k], best, bx, by, be);
    };
    for (int k = 0; k <= kmax; ++k) {
      const int x0 = max(cx - k, 0), x1 = min(cx + k, S.nx - 1);
      for (int x = x0; x <= x1; ++x) {
        if (x == cx - k || x == cx + k) {                  // a full column of the ring
          for (int y = max(cy - k, 0); y <= min(cy + k, S.ny - 1); ++y) scan_cell(x, y);
        } else {                                           // its top and bottom cells
          if (cy - k >= 0) scan_cell(x, cy - k);
          if (cy + k < S.ny && k > 0) scan_cell(x, cy + k);
        }
      }
      if (best < (double)k * S.cell * (1.0 - 1e-12)) break;
    }
  } else {
    for (int64_t e = 0; e < S.n_edges; ++e) nearest_edge(px, py, S.erec[e], e, best, bx, by, be);
  }
  const double ind = indicator_at(S, px, py, norm_support > 0.0 ? norm_support : 1.0, in_grid, cid);
  const bool ins = ind > 0.5;
  d[i] = ins ? -best : best;
  cp[2 * i] = bx;
  cp[2 * i + 1] = by;
  edge[i] = (int32_t)be;
  double n0 = 0.0, n1 = 0.0;
  if (be >= 0) {
    const double4 r = S.erec[be];
    const double ex = r.z - r.x, ey = r.w - r.y;
    const double el = sqrt(ex * ex + ey * ey);
    n0 = ey / el;
    n1 = -ex / el;
  }
  const double vx = px - bx, vy = py - by;
  const double dn = sqrt(vx * vx + vy * vy);
  if (dn > 1e-12 && !ins) {
    n0 = vx / fmax(dn, 1e-300);
    n1 = vy / fmax(dn, 1e-300);
  }
  nl[2 * i] = n0;
  nl[2 * i + 1] = n1;
}

// ------------------------------------------------------------------------------------------------ kinematics
__global__ void k_kinematics(const double* __restrict__ bodies, int32_t nb, const double* __restrict__ x, int64_t n,
                             double* rel, double* local, double* vel, double* acc) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= (int64_t)nb * n) return;
  const int64_t b = t / n, i = t % n;
  const double* B = bodies + 10 * b;
  const double px = x[2 * i], py = x[2 * i + 1];
  const double r0 = __dsub_rn(px, B[0]), r1 = __dsub_rn(py, B[1]);
  if (rel) {
    rel[2 * t] = r0;
    rel[2 * t + 1] = r1;
  }
  if (local) {
    double lx, ly;
    to_local_rn(px, py, B[0], B[1], B[2], B[3], lx, ly);
    local[2 * t] = lx;
    local[2 * t + 1] = ly;
  }
  const double w = B[6];
  if (vel) {      // v + w * (-r1, r0)
    vel[2 * t] = __dadd_rn(B[4], __dmul_rn(w, -r1));
    vel[2 * t + 1] = __dadd_rn(B[5], __dmul_rn(w, r0));
  }
  if (acc) {      // a + alpha * (-r1, r0) - (w * w) * r
    const double ww = __dmul_rn(w, w), al = B[9];
    acc[2 * t] = __dsub_rn(__dadd_rn(B[7], __dmul_rn(al, -r1)), __dmul_rn(ww, r0));
    acc[2 * t + 1] = __dsub_rn(__dadd_rn(B[8], __dmul_rn(al, r0)), __dmul_rn(ww, r1));
  }
}

// exclusive prefix sums of m counts in one block, tile by tile: a tile of kScanThreads x kScanItems counts is loaded
// coalesced into shared memory (padded one word every 32 against bank conflicts), each thread scans its kScanItems
// consecutive counts, the thread totals are scanned with warp shuffles, and the tile is written back coalesced with
// the running total of the earlier tiles added (the bucket counts of the row sort: one cell grid's worth of entries)
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;
__device__ __forceinline__ int scan_pad(int k) { return k + (k >> 5); }

__global__ void __launch_bounds__(kScanThreads) k_scan_block(const int32_t* __restrict__ in, int32_t* __restrict__ out,
                                                            int64_t m) {
  pdl_wait();      // the preceding kernel of the stream has completed and its writes are visible
  pdl_trigger();   // the next kernel of the stream may be scheduled into the SMs this grid frees
  __shared__ int32_t s_data[kScanTile + kScanTile / 32];
  __shared__ int32_t s_warp[kScanThreads / 32];
  __shared__ int32_t s_carry;
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  if (t == 0) s_carry = 0;
  for (int64_t base = 0; base < m; base += kScanTile) {
    const int tile = (int)min((int64_t)kScanTile, m - base);
    for (int k = t; k < kScanTile; k += kScanThreads) s_data[scan_pad(k)] = k < tile ? in[base + k] : 0;
    __syncthreads();
    int32_t sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) sum += s_data[scan_pad(t * kScanItems + i)];
    int32_t x = sum;                                   // inclusive scan of the thread totals within the warp
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int32_t y = __shfl_up_sync(0xffffffffu, x, d);
      if (lane >= d) x += y;
    }
    if (lane == 31) s_warp[wid] = x;
    __syncthreads();
    if (wid == 0) {                                    // inclusive scan of the 32 warp totals
      int32_t v = s_warp[lane];
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += y;
      }
      s_warp[lane] = v;
    }
    __syncthreads();
    int32_t run = s_carry + (wid ? s_warp[wid - 1] : 0) + (x - sum);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
      const int p = scan_pad(t * kScanItems + i);
      const int32_t v = s_data[p];
      s_data[p] = run;
      run += v;
    }
    __syncthreads();
    if (t == kScanThreads - 1) s_carry = run;          // the total of this and the earlier tiles
    for (int k = t; k < tile; k += kScanThreads) out[base + k] = s_data[scan_pad(k)];
    __syncthreads();
  }
}

// rows with pairs into `work`, grouped by count key (decreasing pair count): the prefix of the key histogram per
// block, then warp-aggregated cursor atomics (the order inside a key group is arbitrary; every row's result is
// independent of it)
__global__ void k_key_scatter(SurfView S, const int32_t* __restrict__ rkey, int64_t n, const int32_t* __restrict__ khist,
                              int32_t* __restrict__ kcur, const int32_t* __restrict__ order,
                              int32_t* __restrict__ bucket, const double* __restrict__ lpos,
                              const double* __restrict__ sup, const uint64_t* __restrict__ mask,
                              WorkRec* __restrict__ wrec, int32_t* __restrict__ nwork) {
  pdl_wait();      // the preceding kernel of the stream has completed and its writes are visible
  pdl_trigger();   // the next kernel of the stream may be scheduled into the SMs this grid frees
  constexpr int kWork = kKeys - 1;                                  // keys of rows with pairs: 0 .. 63
  static_assert(kWork == 64, "two keys a lane in the prefix scan");
  __shared__ int32_t s_pre[kWork + 1];                              // exclusive prefix of the key counts
  __shared__ int32_t s_cnt[kWork];                                  // this block's rows per key, then its base
  if (threadIdx.x < 32) {
    // the prefix of the 64 key counts by one warp: lane l scans keys l and l + 32
    const int l = threadIdx.x;
    const int a = khist[l], b = khist[l + 32];
    int sa = a, sb = b;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int ta = __shfl_up_sync(0xffffffffu, sa, o), tb = __shfl_up_sync(0xffffffffu, sb, o);
      if (l >= o) {
        sa += ta;
        sb += tb;
      }
    }
    const int tot_a = __shfl_sync(0xffffffffu, sa, 31), tot_b = __shfl_sync(0xffffffffu, sb, 31);
    s_pre[l] = sa - a;
    s_pre[l + 32] = tot_a + sb - b;
    if (l == 0) {
      s_pre[kWork] = tot_a + tot_b;
      if (blockIdx.x == 0) *nwork = tot_a + tot_b;                  // rows with key < 64
    }
  }
  for (int k = threadIdx.x; k < kWork; k += kThreads) s_cnt[k] = 0;
  __syncthreads();
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int key = j < n ? rkey[j] : -1;
  const bool mine = key >= 0 && key < kWork;
  // the row's rank among the block's rows of its key (warp-aggregated shared atomics), then one global cursor add
  // per key the block has: the block's base in that key's range
  const unsigned peers = __match_any_sync(0xffffffffu, mine ? key : -1);
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(peers) - 1;
  int rank = 0;
  if (mine && lane == leader) rank = atomicAdd(&s_cnt[key], __popc(peers));
  rank = __shfl_sync(0xffffffffu, rank, leader) + __popc(peers & ((1u << lane) - 1));
  __syncthreads();
  for (int k = threadIdx.x; k < kWork; k += kThreads)
    if (s_cnt[k]) s_cnt[k] = atomicAdd(&kcur[k], s_cnt[k]);
  __syncthreads();
  if (mine) {
    // gather the row's record once here, so the evaluations read one coalesced record per work row
    const int32_t i = order[j];
    const int32_t b = bucket[i];
    const ulonglong2 mm = reinterpret_cast<const ulonglong2*>(mask)[j];
    WorkRec r;
    r.lx = lpos[2 * i];
    r.ly = lpos[2 * i + 1];
    r.h = sup[i];
    r.row = i;
    r.kb = S.cstart[b];
    r.ke = S.cstart[b + 1];
    r.pad[0] = r.pad[1] = r.pad[2] = 0;
    r.m0 = mm.x;
    r.m1 = mm.y;
    const int32_t slot = s_pre[key] + s_cnt[key] + rank;
    wrec[slot] = r;
    bucket[i] = slot;            // from here on a work row's key is its work slot (read by the staged expansion)
  }
}

// ------------------------------------------------------------------------------------------------ cone area, direction
// Two detector inputs of the delta+ scheme over the prepared rows (src/warpSPHBoundaries/scene/fused.py:155-308,
// 741-835): the area of the solid inside the support disk and a wedge about a per-row axis, and the largest |cos|
// between a per-row vector and the directions from the row to the solid within its support.  Both visit the same
// neighbour edges as the channel pass (the float64 predicate |x - seg| < h over the row's cell candidates), one thread
// per work row, in float64.

// a - 2 pi round((a + pi) / 2 pi - 1/2): the angle in [-pi, pi)
__device__ __forceinline__ double wrap_pi(double a) {
  const double r = a + 0.5 * kTwoPi;
  return r - kTwoPi * floor(r / kTwoPi) - 0.5 * kTwoPi;
}

// every neighbour edge of a work row, in candidate order: the candidates the row's mask marks, then those past the
// mask that pass the predicate
template <class F>
__device__ __forceinline__ void for_each_neighbour(const SurfView& S, const WorkRec& r, F&& f) {
  uint64_t m0 = r.m0, m1 = r.m1;
  for (int b = pop_bit(m0, m1); b >= 0; b = pop_bit(m0, m1)) f(ldg4(S.crec + r.kb + b));
  for (int k = r.kb + kMaskBits; k < r.ke; ++k) {
    const double4 e = ldg4(S.crec + k);
    if (seg_within_fast(r.lx, r.ly, e.x, e.y, e.z, e.w, r.h)) f(e);
  }
}

// The sector of the support disk that an edge a -> b sweeps about the row, seen through its chord: s = the edge's
// orientation about the row (+1 counter-clockwise), z = the row's distance to the edge line, [lo, hi] = the swept
// angles (|hi - lo| < pi), pn = the angle of the foot of the perpendicular (on the branch of lo) and be = acos(z / H),
// the half-angle under which the chord inside the disk is seen.  False for a degenerate edge, a row on the edge line
// or an edge line that misses the open disk (scene/cone_area.py:20-40 per edge; fused.py:200-225 in the local form).
struct ConeEdge {
  double s, z, lo, hi, pn, be;
};

__device__ __forceinline__ bool cone_edge(double px, double py, double H, const double4& e, ConeEdge& c) {
  const double ax = e.x - px, ay = e.y - py, bx = e.z - px, by = e.w - py;
  const double cr = ax * by - ay * bx;
  const double dx = bx - ax, dy = by - ay;
  const double L = sqrt(dx * dx + dy * dy);
  if (!(L > 0.0) || !(fabs(cr) >= 1e-300)) return false;
  c.z = fabs(cr) / L;
  if (!(c.z < H)) return false;
  c.s = cr < 0.0 ? -1.0 : 1.0;
  const double pa = atan2(ay, ax);
  const double dphi = wrap_pi(atan2(by, bx) - pa);
  c.lo = dphi < 0.0 ? pa + dphi : pa;
  c.hi = dphi < 0.0 ? pa : pa + dphi;
  const double ux = dx / L, uy = dy / L, t = ax * ux + ay * uy;
  c.pn = c.lo + wrap_pi(atan2(ay - t * uy, ax - t * ux) - c.lo);
  c.be = acos(c.z / H);
  return true;
}

// What the chord removes from the sector 1/2 H^2 (h - l) of the angles [l, h] (inside [lo, hi]): where the edge is
// nearer than H -- the copy of (pn - be, pn + be) whose centre is nearest the interval's midpoint -- the ray ends on
// the edge at z / cos(phi - pn), so the sector 1/2 H^2 dphi gives way to the triangle 1/2 z^2 d tan(phi - pn).
__device__ __forceinline__ double chord_deficit(double l, double h, const ConeEdge& c, double H) {
  const double k = floor((0.5 * (l + h) - c.pn) / kTwoPi + 0.5);
  const double c0 = fmax(l, c.pn + kTwoPi * k - c.be), c1 = fmin(h, c.pn + kTwoPi * k + c.be);
  if (!(c0 < c1)) return 0.0;
  return 0.5 * H * H * (c1 - c0) - 0.5 * c.z * c.z * (tan(c1 - c.pn) - tan(c0 - c.pn));
}

// Per row: area += 1/2 H^2 W ind - sum_e s_e (chord deficit of e inside the wedge) and full += pi H^2 ind - sum_e s_e
// (chord deficit of e), W = 2 half_angle (2 pi for half_angle >= pi).  The sectors of the edges beyond the disk sum
// along every ray to the winding indicator, which is why only the neighbour edges enter.  A row outside the
// broadphase of a surface whose solid is the unbounded outside lies deep in it: the whole sector.  Work blocks first,
// then tail blocks for the rows without neighbour edges (as the channel pass).
__global__ void __launch_bounds__(kThreads) k_cone_area(SurfView S, const double* __restrict__ sup,
                                                       const WorkRec* __restrict__ wrec,
                                                       const int32_t* __restrict__ nwork_p, int64_t n,
                                                       const double* __restrict__ ind,
                                                       const int32_t* __restrict__ flag,
                                                       const double* __restrict__ pose,
                                                       const double* __restrict__ axes, double half_angle,
                                                       double* __restrict__ area) {
  const int64_t nwork = *nwork_p;
  const int64_t wblocks = (nwork + kThreads - 1) / kThreads;
  const bool wedge = half_angle < 0.5 * kTwoPi;
  const double W = wedge ? 2.0 * half_angle : kTwoPi;
  if ((int64_t)blockIdx.x >= wblocks) {
    const int64_t i = ((int64_t)blockIdx.x - wblocks) * kThreads + threadIdx.x;
    if (i >= n) return;
    const int32_t f = flag[i];
    if (f == 2) return;
    const double w = f == 1 ? ind[i] : S.background;
    if (w != 0.0) {
      const double H = sup[i];
      area[i] += 0.5 * H * H * W * w;
      area[n + i] += 0.5 * H * H * kTwoPi * w;
    }
    return;
  }
  const int64_t j = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (j >= nwork) return;
  const WorkRec r = load_workrec(wrec + j);
  const int64_t i = r.row;
  const double H = r.h;
  const double ax = axes[2 * i], ay = axes[2 * i + 1], pc = pose[2], ps = pose[3];
  const double th = atan2(-ps * ax + pc * ay, pc * ax + ps * ay);      // the world axis in the body frame
  double a_wedge = 0.0, a_full = 0.0;
  for_each_neighbour(S, r, [&](const double4& e) {
    ConeEdge c;
    if (!cone_edge(r.lx, r.ly, H, e, c)) return;
    a_full += c.s * chord_deficit(c.lo, c.hi, c, H);
    if (!wedge) return;
    const double mid = c.lo + wrap_pi(th - c.lo);                     // the wedge centre on the branch of lo
#pragma unroll
    for (int k = -1; k <= 1; ++k) {
      const double l = fmax(c.lo, mid + kTwoPi * k - half_angle), h = fmin(c.hi, mid + kTwoPi * k + half_angle);
      if (l < h) a_wedge += c.s * chord_deficit(l, h, c, H);
    }
  });
  if (!wedge) a_wedge = a_full;
  const double w = ind[i];
  area[i] += 0.5 * H * H * W * w - a_wedge;
  area[n + i] += 0.5 * H * H * kTwoPi * w - a_full;
}

// Per row: max |v . x| over the unit directions x from the row to the solid within its support, v the row's world
// vector in the body frame, normalised; max-accumulated into out[i] (0 for a zero vector or no solid in support).  A
// row inside the solid sees it in every direction (1).  Otherwise the solid inside the disk is seen under the angular
// spans of the edge pieces inside it; |cos| peaks where a span contains the line of v (1) or at a span's end (a vertex
// inside the disk or the edge's crossing of the support circle): fused.py:248-308.
__device__ __forceinline__ double edge_extreme(double px, double py, double H, const double4& e, double vx,
                                               double vy) {
  const double ax = e.x - px, ay = e.y - py, dx = e.z - e.x, dy = e.w - e.y;
  const double a = dx * dx + dy * dy;
  if (!(a > 0.0)) return 0.0;
  const double b = ax * dx + ay * dy;
  const double disc = b * b - a * (ax * ax + ay * ay - H * H);
  if (!(disc > 0.0)) return 0.0;
  const double sq = sqrt(disc);
  const double t0 = fmax(0.0, (-b - sq) / a), t1 = fmin(1.0, (-b + sq) / a);
  if (!(t0 < t1)) return 0.0;
  const double cd = dx * vy - dy * vx;
  if (fabs(cd) > 0.0) {
    const double ts = -(ax * vy - ay * vx) / cd;                       // where the line of v crosses the edge
    if (ts >= t0 && ts <= t1) return 1.0;
  }
  double f = 0.0;
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const double t = k == 0 ? t0 : t1;
    const double rx = ax + t * dx, ry = ay + t * dy, rr = sqrt(rx * rx + ry * ry);
    if (rr > 0.0) f = fmax(f, fabs(rx * vx + ry * vy) / rr);
  }
  return f;
}

__global__ void __launch_bounds__(kThreads) k_dir_extreme(SurfView S, const WorkRec* __restrict__ wrec,
                                                         const int32_t* __restrict__ nwork_p, int64_t n,
                                                         const double* __restrict__ ind,
                                                         const int32_t* __restrict__ flag,
                                                         const double* __restrict__ pose,
                                                         const double* __restrict__ vecs, double* __restrict__ out) {
  const int64_t nwork = *nwork_p;
  const int64_t wblocks = (nwork + kThreads - 1) / kThreads;
  if ((int64_t)blockIdx.x >= wblocks) {
    const int64_t i = ((int64_t)blockIdx.x - wblocks) * kThreads + threadIdx.x;
    if (i >= n) return;
    const int32_t f = flag[i];
    if (f == 2) return;
    const double w = f == 1 ? ind[i] : S.background;
    if (w > 0.5 && (vecs[2 * i] != 0.0 || vecs[2 * i + 1] != 0.0)) out[i] = 1.0;
    return;
  }
  const int64_t j = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (j >= nwork) return;
  const WorkRec r = load_workrec(wrec + j);
  const int64_t i = r.row;
  const double wx = vecs[2 * i], wy = vecs[2 * i + 1], pc = pose[2], ps = pose[3];
  double vx = pc * wx + ps * wy, vy = -ps * wx + pc * wy;             // R^T w
  const double nv = sqrt(vx * vx + vy * vy);
  if (!(nv > 0.0)) return;
  vx /= nv;
  vy /= nv;
  double best = ind[i] > 0.5 ? 1.0 : 0.0;
  if (best < 1.0)
    for_each_neighbour(S, r, [&](const double4& e) { best = fmax(best, edge_extreme(r.lx, r.ly, r.h, e, vx, vy)); });
  out[i] = fmax(out[i], best);
}

// shared front half of the aggregate and its adjoint: body frame, broadphase, counting sort of the rows by cell
// a launch that may start while the preceding kernel of the stream finishes (its kernel calls pdl_wait() before
// touching memory): the seven kernels of one aggregate (prepare, pair pass, expansion) follow each other this way
template <class... P, class... A>
static cudaError_t launch_dep(void (*k)(P...), unsigned grid, unsigned block, size_t smem, cudaStream_t st,
                             A&&... a) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, std::forward<A>(a)...);
}

static int sort_rows(const Surface* s, const double* pos, const double* sup, const int32_t* allowed, int64_t n,
                     const double* pose, const double* obb, int unbounded, const Workspace& w, cudaStream_t st) {
  const int64_t nbk = (int64_t)s->n_nonempty + 2;   // buckets: the cells with edges
  WSB_CUDA(cudaMemsetAsync(w.counts, 0, sizeof(int32_t) * (2 * nbk + 1), st));
  WSB_CUDA(cudaMemsetAsync(w.khist, 0, sizeof(int32_t) * 2 * kKeys, st));
  const SurfView v = view_of(s);
  const unsigned grid = (unsigned)((n + kThreads - 1) / kThreads);
  k_agg_prep<<<grid, kThreads, 0, st>>>(v, pos, sup, allowed, n, pose, make_double4(obb[0], obb[1], obb[2], obb[3]),
                                        unbounded, w.key, w.lpos, w.counts, w.ind, w.flag);
  WSB_CUDA(launch_dep(k_scan_block, 1, kScanThreads, 0, st, (const int32_t*)w.counts, w.offs, nbk + 1));
  WSB_CUDA(launch_dep(k_agg_scatter, grid, kThreads, 0, st, v, (const int32_t*)w.key, n, (const int32_t*)w.offs,
                      w.cursor, w.order));
  WSB_CUDA(launch_dep(k_agg_rowinfo, grid, kThreads, 0, st, v, sup, (const int32_t*)w.key, (const double*)w.lpos,
                      (const int32_t*)w.offs, (const int32_t*)w.order, n, w.ind, w.flag, w.rkey, w.mask, w.khist));
  WSB_CUDA(launch_dep(k_key_scatter, grid, kThreads, 0, st, v, (const int32_t*)w.rkey, n, (const int32_t*)w.khist,
                      w.kcur, (const int32_t*)w.order, w.key, (const double*)w.lpos, sup, (const uint64_t*)w.mask,
                      w.wrec, w.nwork));
  WSB_CUDA(cudaGetLastError());
  return WSB_OK;
}

// kernel ids the fused aggregate serves: the exact-table kernels and the quadrature kernels (the tensile group)
static bool is_quad_kernel(int k) { return k == Kern_w2p5::kId || k == Kern_w4p5::kId; }
static bool aggregate_kernel_ok(int k) { return (k >= 0 && k < kNumKernels) || is_quad_kernel(k); }

static int check_common(const Surface* s, int kernel, const double* pos, const double* sup, int64_t n,
                        const double* pose, const double* obb, const char* who) {
  if (!s) return fail(WSB_ERR_ARG, std::string(who) + ": NULL surface");
  if (!aggregate_kernel_ok(kernel)) return fail(WSB_ERR_UNSUPPORTED, std::string(who) + ": unknown kernel id");
  if (n < 0 || n > (int64_t)INT32_MAX) return fail(WSB_ERR_ARG, std::string(who) + ": row count out of range");
  if (n > 0 && (!pos || !sup || !pose || !obb)) return fail(WSB_ERR_ARG, std::string(who) + ": NULL array");
  return WSB_OK;
}

}  // namespace wsb

using namespace wsb;

extern "C" size_t wsb_aggregate_workspace_size(const wsb_surface* s_, int64_t n) {
  const Surface* s = reinterpret_cast<const Surface*>(s_);
  if (!s || n < 0) return 0;
  return carve(s, n, nullptr).total;
}

extern "C" int wsb_set_pair_events(void* start, void* end) {
  if ((start == nullptr) != (end == nullptr)) return fail(WSB_ERR_ARG, "wsb_set_pair_events: both events or neither");
  g_pair_ev[0] = (cudaEvent_t)start;
  g_pair_ev[1] = (cudaEvent_t)end;
  return WSB_OK;
}

extern "C" size_t wsb_aggregate_staging_size(const wsb_surface* s_, int64_t n) {
  const Surface* s = reinterpret_cast<const Surface*>(s_);
  if (!s || n < 0) return 0;
  return carve(s, n, nullptr).staging;
}

extern "C" int wsb_aggregate_prepare(const wsb_surface* s_, const double* pos, const double* sup,
                                     const int32_t* allowed, int64_t n, const double* pose, const double* obb,
                                     int unbounded, void* workspace, size_t workspace_bytes, void* stream) {
  const Surface* s = reinterpret_cast<const Surface*>(s_);
  int rc = check_common(s, 0, pos, sup, n, pose, obb, "wsb_aggregate_prepare");
  if (rc) return rc;
  if (n == 0) return WSB_OK;
  const Workspace w = carve(s, n, workspace);
  if (!workspace || workspace_bytes < w.total)
    return fail(WSB_ERR_SIZE, "wsb_aggregate_prepare: workspace of " + std::to_string(workspace_bytes) +
                                  " bytes, need " + std::to_string(w.total));
  WSB_CUDA(cudaSetDevice(s->device));
  return sort_rows(s, pos, sup, allowed, n, pose, obb, unbounded, w, (cudaStream_t)stream);
}

extern "C" int wsb_aggregate_evaluate(const wsb_surface* s_, int kernel, int precision, const double* sup, int64_t n,
                                      const double* pose, int out_mask, double* lam, double* G, double* cov,
                                      double* m1, double* m2, const void* workspace, size_t workspace_bytes,
                                      void* stream) {
  const Surface* s = reinterpret_cast<const Surface*>(s_);
  if (!s) return fail(WSB_ERR_ARG, "wsb_aggregate_evaluate: NULL surface");
  if (!aggregate_kernel_ok(kernel)) return fail(WSB_ERR_UNSUPPORTED, "wsb_aggregate_evaluate: unknown kernel id");
  if (precision != WSB_PREC_FP64 && precision != WSB_PREC_MIXED && precision != WSB_PREC_FP32)
    return fail(WSB_ERR_UNSUPPORTED, "wsb_aggregate_evaluate: unknown precision mode");
  if (n < 0 || n > (int64_t)INT32_MAX) return fail(WSB_ERR_ARG, "wsb_aggregate_evaluate: row count out of range");
  if (n == 0) return WSB_OK;
  if (!sup || !pose) return fail(WSB_ERR_ARG, "wsb_aggregate_evaluate: NULL array");
  Workspace w = carve(s, n, const_cast<void*>(workspace));
  attach_staging(w, const_cast<void*>(workspace), workspace_bytes);
  if (!workspace || workspace_bytes < w.total) return fail(WSB_ERR_SIZE, "wsb_aggregate_evaluate: workspace too small");
  WSB_CUDA(cudaSetDevice(s->device));
  cudaStream_t st = (cudaStream_t)stream;
  double* L = (out_mask & WSB_OUT_LAM) ? lam : nullptr;
  double* Gp = (out_mask & WSB_OUT_G) ? G : nullptr;
  double* C = (out_mask & WSB_OUT_COV) ? cov : nullptr;
  double* M1 = (out_mask & WSB_OUT_M1) ? m1 : nullptr;
  double* M2 = (out_mask & WSB_OUT_M2) ? m2 : nullptr;
  const SurfView v = view_of(s);
  const bool assign = (out_mask & WSB_OUT_ASSIGN) != 0;
  PackOut o{};
  o.lam[0] = L;
  o.G[0] = Gp;
  o.cov[0] = C;
  o.m1[0] = M1;
  o.m2[0] = M2;
  auto launch1 = [&](auto kt) {
    using P1 = KPack<decltype(kt)>;
    if (precision == WSB_PREC_MIXED) return launch_pack<P1, WSB_PREC_MIXED>(v, sup, w, n, pose, assign, o, st);
    if (precision == WSB_PREC_FP32) return launch_pack<P1, WSB_PREC_FP32>(v, sup, w, n, pose, assign, o, st);
    return launch_pack<P1, WSB_PREC_FP64>(v, sup, w, n, pose, assign, o, st);
  };
  int rc = 0;
  if (kernel == Kern_w2p5::kId)
    rc = launch1(Kern_w2p5{});
  else if (kernel == Kern_w4p5::kId)
    rc = launch1(Kern_w4p5{});
  else
    rc = dispatch_kernel(kernel, launch1);
  if (rc) return rc;
  WSB_CUDA(cudaGetLastError());
  return WSB_OK;
}

// The kernel sets evaluated in one pass over the neighbour pairs, largest first: the smoothing-kernel families, and
// the exact groups of the delta+ layout (scheme kernel, cone, wall-Laplacian kernel).  The first set contained in the
// groups (each of its kernels exactly once, any order) runs as one pack; every other group runs its own pass.
static const int32_t kPackCW[4] = {WSB_KERNEL_CUBIC, WSB_KERNEL_W2, WSB_KERNEL_W4, WSB_KERNEL_W6};
static const int32_t kPackW[3] = {WSB_KERNEL_W2, WSB_KERNEL_W4, WSB_KERNEL_W6};
static const int32_t kPackD2L[3] = {WSB_KERNEL_W2, WSB_KERNEL_CONE, WSB_KERNEL_LW2};
static const int32_t kPackD4L[3] = {WSB_KERNEL_W4, WSB_KERNEL_CONE, WSB_KERNEL_LW4};
static const int32_t kPackD2[2] = {WSB_KERNEL_W2, WSB_KERNEL_CONE};
static const int32_t kPackD4[2] = {WSB_KERNEL_W4, WSB_KERNEL_CONE};

// perm[p] = the group holding pack kernel p when each of the pack's kernels is exactly one of the groups
static bool match_pack(const int32_t* kernels, int n_groups, const int32_t* pack, int m, int* perm) {
  if (n_groups < m) return false;
  for (int p = 0; p < m; ++p) {
    perm[p] = -1;
    for (int g = 0; g < n_groups; ++g)
      if (kernels[g] == pack[p]) {
        if (perm[p] >= 0) return false;
        perm[p] = g;
      }
    if (perm[p] < 0) return false;
  }
  return true;
}

extern "C" int wsb_aggregate_evaluate_groups(const wsb_surface* s_, int n_groups, const int32_t* kernels,
                                             int precision, const double* sup, int64_t n, const double* pose,
                                             int out_mask, double* const* lam, double* const* G, double* const* cov,
                                             double* const* m1, double* const* m2, const void* workspace,
                                             size_t workspace_bytes, void* stream) {
  const Surface* s = reinterpret_cast<const Surface*>(s_);
  if (!s) return fail(WSB_ERR_ARG, "wsb_aggregate_evaluate_groups: NULL surface");
  if (n_groups < 1 || n_groups > WSB_MAX_GROUPS || !kernels)
    return fail(WSB_ERR_ARG, "wsb_aggregate_evaluate_groups: 1 to " + std::to_string(WSB_MAX_GROUPS) +
                                 " kernel groups expected");
  for (int g = 0; g < n_groups; ++g)
    if (!aggregate_kernel_ok(kernels[g]))
      return fail(WSB_ERR_UNSUPPORTED, "wsb_aggregate_evaluate_groups: unknown kernel id");
  if (precision != WSB_PREC_FP64 && precision != WSB_PREC_MIXED && precision != WSB_PREC_FP32)
    return fail(WSB_ERR_UNSUPPORTED, "wsb_aggregate_evaluate_groups: unknown precision mode");
  if (n < 0 || n > (int64_t)INT32_MAX) return fail(WSB_ERR_ARG, "wsb_aggregate_evaluate_groups: row count out of range");
  if (n == 0) return WSB_OK;
  if (!sup || !pose) return fail(WSB_ERR_ARG, "wsb_aggregate_evaluate_groups: NULL array");
  auto pick = [&](double* const* a, int g, int bit) { return (a && (out_mask & bit)) ? a[g] : nullptr; };
  int perm[kMaxPack];
  int which = -1, m = 0;
  const int32_t* packs[6] = {kPackCW, kPackW, kPackD2L, kPackD4L, kPackD2, kPackD4};
  const int sizes[6] = {4, 3, 3, 3, 2, 2};
  for (int k = 0; k < 6 && which < 0; ++k)
    if (match_pack(kernels, n_groups, packs[k], sizes[k], perm)) {
      which = k;
      m = sizes[k];
    }
  bool in_pack[WSB_MAX_GROUPS] = {false};
  for (int p = 0; p < m; ++p) in_pack[perm[p]] = true;
  for (int g = 0; g < n_groups; ++g) {                              // the groups outside the pack: one pass each
    if (in_pack[g]) continue;
    const int rc = wsb_aggregate_evaluate(s_, kernels[g], precision, sup, n, pose, out_mask, pick(lam, g, WSB_OUT_LAM),
                                          pick(G, g, WSB_OUT_G), pick(cov, g, WSB_OUT_COV), pick(m1, g, WSB_OUT_M1),
                                          pick(m2, g, WSB_OUT_M2), workspace, workspace_bytes, stream);
    if (rc) return rc;
  }
  if (which < 0) return WSB_OK;
  Workspace w = carve(s, n, const_cast<void*>(workspace));
  attach_staging(w, const_cast<void*>(workspace), workspace_bytes);
  if (!workspace || workspace_bytes < w.total)
    return fail(WSB_ERR_SIZE, "wsb_aggregate_evaluate_groups: workspace too small");
  WSB_CUDA(cudaSetDevice(s->device));
  cudaStream_t st = (cudaStream_t)stream;
  const SurfView v = view_of(s);
  const bool assign = (out_mask & WSB_OUT_ASSIGN) != 0;
  PackOut o{};
  for (int p = 0; p < m; ++p) {
    o.lam[p] = pick(lam, perm[p], WSB_OUT_LAM);
    o.G[p] = pick(G, perm[p], WSB_OUT_G);
    o.cov[p] = pick(cov, perm[p], WSB_OUT_COV);
    o.m1[p] = pick(m1, perm[p], WSB_OUT_M1);
    o.m2[p] = pick(m2, perm[p], WSB_OUT_M2);
  }
  auto run = [&](auto pack) {
    using P = decltype(pack);
    if (precision == WSB_PREC_MIXED) return launch_pack<P, WSB_PREC_MIXED>(v, sup, w, n, pose, assign, o, st);
    if (precision == WSB_PREC_FP32) return launch_pack<P, WSB_PREC_FP32>(v, sup, w, n, pose, assign, o, st);
    return launch_pack<P, WSB_PREC_FP64>(v, sup, w, n, pose, assign, o, st);
  };
  int rc;
  switch (which) {
    case 0: rc = run(KPack<Kern_cubic, Kern_w2, Kern_w4, Kern_w6>{}); break;
    case 1: rc = run(KPack<Kern_w2, Kern_w4, Kern_w6>{}); break;
    case 2: rc = run(KPack<Kern_w2, Kern_cone, Kern_lw2>{}); break;
    case 3: rc = run(KPack<Kern_w4, Kern_cone, Kern_lw4>{}); break;
    case 4: rc = run(KPack<Kern_w2, Kern_cone>{}); break;
    default: rc = run(KPack<Kern_w4, Kern_cone>{}); break;
  }
  if (rc) return rc;
  WSB_CUDA(cudaGetLastError());
  return WSB_OK;
}

extern "C" int wsb_aggregate(const wsb_surface* s_, int kernel, int precision, const double* pos, const double* sup,
                             const int32_t* allowed, int64_t n, const double* pose, const double* obb, int unbounded,
                             int out_mask, double* lam, double* G, double* cov, double* m1, double* m2,
                             void* workspace, size_t workspace_bytes, int32_t* status, void* stream) {
  const Surface* s = reinterpret_cast<const Surface*>(s_);
  int rc = check_common(s, kernel, pos, sup, n, pose, obb, "wsb_aggregate");
  if (rc) return rc;
  if (precision != WSB_PREC_FP64 && precision != WSB_PREC_MIXED && precision != WSB_PREC_FP32)
    return fail(WSB_ERR_UNSUPPORTED, "wsb_aggregate: unknown precision mode");
  if (n == 0) return WSB_OK;
  if (status) {
    WSB_CUDA(cudaSetDevice(s->device));
    WSB_CUDA(cudaMemsetAsync(status, 0, sizeof(int32_t), (cudaStream_t)stream));
  }
  rc = wsb_aggregate_prepare(s_, pos, sup, allowed, n, pose, obb, unbounded, workspace, workspace_bytes, stream);
  if (rc) return rc;
  return wsb_aggregate_evaluate(s_, kernel, precision, sup, n, pose, out_mask, lam, G, cov, m1, m2, workspace,
                                workspace_bytes, stream);
}

extern "C" int wsb_aggregate_groups(const wsb_surface* s_, int n_groups, const int32_t* kernels, int precision,
                                    const double* pos, const double* sup, const int32_t* allowed, int64_t n,
                                    const double* pose, const double* obb, int unbounded, int out_mask,
                                    double* const* lam, double* const* G, double* const* cov, double* const* m1,
                                    double* const* m2, void* workspace, size_t workspace_bytes, void* stream) {
  const Surface* s = reinterpret_cast<const Surface*>(s_);
  int rc = check_common(s, 0, pos, sup, n, pose, obb, "wsb_aggregate_groups");
  if (rc) return rc;
  if (n_groups < 1 || n_groups > WSB_MAX_GROUPS || !kernels)
    return fail(WSB_ERR_ARG, "wsb_aggregate_groups: 1 to " + std::to_string(WSB_MAX_GROUPS) + " kernel groups expected");
  for (int g = 0; g < n_groups; ++g)
    if (!aggregate_kernel_ok(kernels[g]))
      return fail(WSB_ERR_UNSUPPORTED, "wsb_aggregate_groups: unknown kernel id");
  if (precision != WSB_PREC_FP64 && precision != WSB_PREC_MIXED && precision != WSB_PREC_FP32)
    return fail(WSB_ERR_UNSUPPORTED, "wsb_aggregate_groups: unknown precision mode");
  if (n == 0) return WSB_OK;
  rc = wsb_aggregate_prepare(s_, pos, sup, allowed, n, pose, obb, unbounded, workspace, workspace_bytes, stream);
  if (rc) return rc;
  return wsb_aggregate_evaluate_groups(s_, n_groups, kernels, precision, sup, n, pose, out_mask, lam, G, cov, m1, m2,
                                       workspace, workspace_bytes, stream);
}

extern "C" int wsb_aggregate_backward(const wsb_surface* s_, int kernel, const double* pos, const double* sup,
                                      const int32_t* allowed, int64_t n, const double* pose, const double* obb,
                                      int unbounded, const double* g_lam, const double* g_m1, const double* g_m2,
                                      double* d_pos, double* d_verts, void* workspace, size_t workspace_bytes,
                                      void* stream) {
  const Surface* s = reinterpret_cast<const Surface*>(s_);
  int rc = check_common(s, kernel, pos, sup, n, pose, obb, "wsb_aggregate_backward");
  if (rc) return rc;
  if (is_quad_kernel(kernel))
    return fail(WSB_ERR_UNSUPPORTED, "wsb_aggregate_backward: the quadrature (tensile) kernels have no adjoint");
  if (n == 0) return WSB_OK;
  if (!d_pos) return fail(WSB_ERR_ARG, "wsb_aggregate_backward: d_pos is NULL");
  const Workspace w = carve(s, n, workspace);
  if (!workspace || workspace_bytes < w.total) return fail(WSB_ERR_SIZE, "wsb_aggregate_backward: workspace too small");
  WSB_CUDA(cudaSetDevice(s->device));
  cudaStream_t st = (cudaStream_t)stream;
  rc = sort_rows(s, pos, sup, allowed, n, pose, obb, unbounded, w, st);
  if (rc) return rc;
  const SurfView v = view_of(s);
  constexpr int G = 2;
  const unsigned grid = (unsigned)((n * G + kThreads - 1) / kThreads);
  rc = dispatch_kernel(kernel, [&](auto kt) {
    using KT = decltype(kt);
    k_agg_backward<KT, G><<<grid, kThreads, 0, st>>>(v, sup, w.wrec, w.nwork, n, pose, g_lam, g_m1, g_m2, d_pos,
                                                     d_verts);
    return 0;
  });
  if (rc) return rc;
  WSB_CUDA(cudaGetLastError());
  return WSB_OK;
}

extern "C" int wsb_signed_distance(const wsb_surface* s_, const double* lpos, int64_t m, double norm_support,
                                   double* d, double* cp, double* n_loc, int32_t* edge, void* stream) {
  const Surface* s = reinterpret_cast<const Surface*>(s_);
  if (!s) return fail(WSB_ERR_ARG, "wsb_signed_distance: NULL surface");
  if (m < 0) return fail(WSB_ERR_ARG, "wsb_signed_distance: negative point count");
  if (m == 0) return WSB_OK;
  if (!lpos || !d || !cp || !n_loc || !edge) return fail(WSB_ERR_ARG, "wsb_signed_distance: NULL array");
  WSB_CUDA(cudaSetDevice(s->device));
  k_signed_distance<<<(unsigned)((m + kThreads - 1) / kThreads), kThreads, 0, (cudaStream_t)stream>>>(
      view_of(s), lpos, m, norm_support, d, cp, n_loc, edge);
  WSB_CUDA(cudaGetLastError());
  return WSB_OK;
}

extern "C" int wsb_kinematics(const double* bodies, int32_t n_bodies, const double* x, int64_t n, double* rel,
                              double* local, double* velocity, double* acceleration, void* stream) {
  if (n_bodies < 0 || n < 0) return fail(WSB_ERR_ARG, "wsb_kinematics: negative size");
  if ((int64_t)n_bodies * n == 0) return WSB_OK;
  if (!bodies || !x) return fail(WSB_ERR_ARG, "wsb_kinematics: NULL array");
  const int64_t total = (int64_t)n_bodies * n;
  k_kinematics<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>(bodies, n_bodies, x, n, rel, local,
                                                                                  velocity, acceleration);
  WSB_CUDA(cudaGetLastError());
  return WSB_OK;
}

// the workspace of a prepared position set, checked against the surface and the row count
static int prepared(const Surface* s, int64_t n, const void* workspace, size_t workspace_bytes, const char* who,
                    Workspace* w) {
  *w = carve(s, n, const_cast<void*>(workspace));
  if (!workspace || workspace_bytes < w->total)
    return fail(WSB_ERR_SIZE, std::string(who) + ": workspace of " + std::to_string(workspace_bytes) + " bytes, need " +
                                  std::to_string(w->total));
  return WSB_OK;
}

extern "C" int wsb_cone_area(const wsb_surface* s_, const double* sup, int64_t n, const double* pose,
                             const double* axes, double half_angle, double* area, const void* workspace,
                             size_t workspace_bytes, void* stream) {
  const Surface* s = reinterpret_cast<const Surface*>(s_);
  if (!s) return fail(WSB_ERR_ARG, "wsb_cone_area: NULL surface");
  if (n < 0 || n > (int64_t)INT32_MAX) return fail(WSB_ERR_ARG, "wsb_cone_area: row count out of range");
  if (!(half_angle >= 0.0) || !std::isfinite(half_angle))
    return fail(WSB_ERR_ARG, "wsb_cone_area: the half angle must be finite and >= 0");
  if (n == 0) return WSB_OK;
  if (!sup || !pose || !axes || !area) return fail(WSB_ERR_ARG, "wsb_cone_area: NULL array");
  Workspace w;
  int rc = prepared(s, n, workspace, workspace_bytes, "wsb_cone_area", &w);
  if (rc) return rc;
  WSB_CUDA(cudaSetDevice(s->device));
  const unsigned grid = (unsigned)(2 * ((n + kThreads - 1) / kThreads));   // work blocks (at most n rows), then tails
  k_cone_area<<<grid, kThreads, 0, (cudaStream_t)stream>>>(view_of(s), sup, w.wrec, w.nwork, n, w.ind, w.flag, pose,
                                                           axes, half_angle, area);
  WSB_CUDA(cudaGetLastError());
  return WSB_OK;
}

extern "C" int wsb_dir_extreme(const wsb_surface* s_, int64_t n, const double* pose, const double* vecs, double* out,
                               const void* workspace, size_t workspace_bytes, void* stream) {
  const Surface* s = reinterpret_cast<const Surface*>(s_);
  if (!s) return fail(WSB_ERR_ARG, "wsb_dir_extreme: NULL surface");
  if (n < 0 || n > (int64_t)INT32_MAX) return fail(WSB_ERR_ARG, "wsb_dir_extreme: row count out of range");
  if (n == 0) return WSB_OK;
  if (!pose || !vecs || !out) return fail(WSB_ERR_ARG, "wsb_dir_extreme: NULL array");
  Workspace w;
  int rc = prepared(s, n, workspace, workspace_bytes, "wsb_dir_extreme", &w);
  if (rc) return rc;
  WSB_CUDA(cudaSetDevice(s->device));
  const unsigned grid = (unsigned)(2 * ((n + kThreads - 1) / kThreads));
  k_dir_extreme<<<grid, kThreads, 0, (cudaStream_t)stream>>>(view_of(s), w.wrec, w.nwork, n, w.ind, w.flag, pose, vecs,
                                                             out);
  WSB_CUDA(cudaGetLastError());
  return WSB_OK;
}

// ------------------------------------------------------------------------------------------------ allocation-free aggregate
// Some hosts cannot give this library device memory: a solver whose allocator has already reserved the GPU's memory
// for its own pool, or a time-step loop that must not call cudaMalloc / cudaFree (they synchronise the whole device),
// and that links the library through the C ABI with no workspace buffer to lend.  For them the aggregate can run on
// a scratch area compiled into the library: a static device array of kNoAllocScratchBytes per GPU, resident for as
// long as the library is loaded.  The address of that array is looked up once per device (cudaGetSymbolAddress with
// the device current) on the first call for that device; host code must never pass the array's own name to a kernel,
// since on the host that name only stands in for the device symbol.
constexpr size_t kNoAllocScratchBytes = (size_t)16 << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];
static void* g_noalloc_addr[64] = {nullptr};
static std::mutex g_noalloc_mu;

static int noalloc_scratch(int device, void** out) {
  if (device < 0 || device >= 64) return fail(WSB_ERR_ARG, "wsb_aggregate_noalloc: device id out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "wsb_aggregate_noalloc: cudaGetSymbolAddress(scratch)");
    g_noalloc_addr[device] = p;
  }
  *out = g_noalloc_addr[device];
  return WSB_OK;
}

extern "C" int wsb_aggregate_noalloc(const wsb_surface* s_, int kernel, int precision, const double* pos,
                                     const double* sup, const int32_t* allowed, int64_t n, const double* pose,
                                     const double* obb, int unbounded, int out_mask, double* lam, double* G,
                                     double* cov, double* m1, double* m2, int32_t* status, void* stream) {
  const Surface* s = reinterpret_cast<const Surface*>(s_);
  int rc = check_common(s, kernel, pos, sup, n, pose, obb, "wsb_aggregate_noalloc");
  if (rc) return rc;
  const size_t need = carve(s, n, nullptr).total;
  if (need > kNoAllocScratchBytes)
    return fail(WSB_ERR_SIZE, "wsb_aggregate_noalloc: " + std::to_string(n) + " rows on a " + std::to_string(s->nx) +
                                  " x " + std::to_string(s->ny) + " cell grid need " + std::to_string(need) +
                                  " bytes of scratch; the built-in scratch holds " +
                                  std::to_string(kNoAllocScratchBytes) + " bytes (use wsb_aggregate with a workspace)");
  if (n == 0) return WSB_OK;
  WSB_CUDA(cudaSetDevice(s->device));
  void* scratch = nullptr;
  rc = noalloc_scratch(s->device, &scratch);
  if (rc) return rc;
  return wsb_aggregate(s_, kernel, precision, pos, sup, allowed, n, pose, obb, unbounded, out_mask, lam, G, cov, m1, m2,
                       scratch, kNoAllocScratchBytes, status, stream);
}
