// Closed triangle surfaces in 3-D: the 28 baseline kernel integrals over the part of each query's support inside the
// solid (value moments |alpha| <= 2, kernel-gradient moments |alpha| <= 1, the kernel Hessian).
//
// Reference: the closed-surface element of src/warpSPHBoundaries/fluxbridge/wp_func.py:119-333 (face -> edge
// reductions, solid-angle term summed over every face), its exact mpmath counterpart
// src/warpSPHBoundaries/mesh3d/reference.py:221-311 (ClosedSurface), the whole-element search of
// fluxbridge/geometry.py:86-170 / device_search.py:158-212 and the per-query reduction of
// fluxbridge/evaluate.py:177-187.
//
// Reduction (unit support: y = (vertex - query) / h, W~ = pi W):
//  * volume -> faces.  For |alpha| = k, y y^alpha G_k(r) with (r^(3+k) G_k)' = r^(2+k) W~ has divergence y^alpha W~;
//    splitting off the homogeneous field y y^alpha Q_k(1) / r^(3+k), whose flux through the closed surface is
//    ind * int_{S^2} yhat^alpha (ind = 1 inside the solid), leaves the compact profile
//    K_k = (Q_k(r) - Q_k(1)) / r^(3+k):   M_alpha = sum_faces z_f int_f y^alpha K_k dS + ind Q_k(1) int yhat^alpha.
//    Kernel-gradient moments are -sum_f N_j int_f y^alpha W~ dS (+ alpha_j M_(alpha - e_j)); the Hessian is
//    sum_f N_i int_f y_j W~'/r dS.  Only faces within the support contribute: no solid-angle sum over all faces.
//  * face -> edges.  With y = z N + u (u in the face plane, r^2 = z^2 + |u|^2) and the compact potential
//    A_F(r) = -int_r^1 t F(t) dt of a profile F:   int_f F = sum_e w_e int_e (A_F(r) - A_F(|z|)) / (r^2 - z^2) ds,
//    int_f u F = sum_e mu_e int_e A_F ds,  int_f u u^T F = sum_e mu_e (x) int_e u A_F ds - P int_f A_F
//    (w_e: signed distance of the foot point to the edge line, mu_e: in-plane outward edge normal, P = I - N N^T).
//  * edges.  Beyond the support the first integrand is -A_F(|z|) / rho^2: an angle.  Inside, every integrand is a
//    smooth function of s along the edge (a divided difference of a Laurent polynomial in r = sqrt(c^2 + s^2)); it is
//    integrated by 12-node Gauss-Legendre on panels split at the foot of the perpendicular, at the kernel's knot and
//    at distances c 2^k from the foot (the dyadic grading of the reference's stable route, edge/warpbc.py:522-575),
//    which keeps the branch points s = +-ic of r away from every panel: relative error below 1e-12.
//    Powers z^p multiply the profiles whose potentials hold r^-m (m <= p) so that every face term stays bounded as
//    the query approaches the face plane.
// The exact rational potentials are generated by warpsphboundaries_b200/kernels.py (mesh_tables, emit_mesh).
#include <algorithm>
#include <cmath>
#include <map>
#include <vector>

#include "common.cuh"

namespace wsb {

struct Mesh {
  int device = 0;
  int64_t n_verts = 0, n_faces = 0;
  double support_max = 0;
  double lo[3] = {0, 0, 0};
  double cell = 1;
  int32_t nx = 1, ny = 1, nz = 1;
  int64_t n_items = 0, n_col_items = 0;
  double* fdata = nullptr;     // [n_faces * kFaceDoubles]
  int32_t* fcell = nullptr;    // [n_faces * 3] lowest cell of the face's box
  int32_t* fvid = nullptr;     // [n_faces * 3] vertex ids
  int32_t* cstart = nullptr;   // [nx*ny*nz + 1]
  int32_t* citems = nullptr;   // faces per cell
  int32_t* colstart = nullptr; // [nx*ny + 1] faces per (x, y) column
  int32_t* colitems = nullptr;
  uint8_t* cflag = nullptr;    // [nx*ny*nz] kCellEmpty | kCellInside | kCellNear
};

// per-cell flags: no face box meets the cell (so the surface does not cross it and every point of it has the inside
// status of its centre); that status; a face box meets one of the 27 cells around it (a query in the cell may have
// candidate faces)
enum : uint8_t { kCellEmpty = 1, kCellInside = 2, kCellNear = 4 };

// per face: v0 v1 v2 (9), unit normal N (3), edge tangents t0 t1 t2 (9), edge normals mu_e = t_e x N (9),
// edge lengths (3), box lo (3), box hi (3)
constexpr int kFaceDoubles = 39;
enum { kFV = 0, kFN = 9, kFT = 12, kFMU = 21, kFLEN = 30, kFLO = 33, kFHI = 36 };

struct MeshView {
  const double* fdata;
  const int32_t* fcell;
  const int32_t* fvid;
  const int32_t* cstart;
  const int32_t* citems;
  const int32_t* colstart;
  const int32_t* colitems;
  const uint8_t* cflag;
  double lo0, lo1, lo2, cell;
  int32_t nx, ny, nz;
};

namespace {

MeshView view_of(const Mesh* m) {
  return MeshView{m->fdata, m->fcell, m->fvid, m->cstart, m->citems, m->colstart, m->colitems, m->cflag,
                  m->lo[0], m->lo[1], m->lo[2], m->cell, m->nx, m->ny, m->nz};
}

__device__ __forceinline__ int cell_coord(double x, double lo, double cell, int n) {
  const double f = floor((x - lo) / cell);
  return f < -1.0 ? -2 : (f > (double)n ? n + 1 : (int)f);
}

// ------------------------------------------------------------------------------------------ inside indicator
// Parity of the crossings of the vertical ray {(x, y, t): t > z} with the surface.  A face's projection owns the
// point when every edge function is positive, or zero on an edge that the ownership rule gives to this side: edge
// functions are evaluated with the edge's vertices in id order (so the two faces of an edge see exactly opposite
// values) and an edge with zero value belongs to the face for which its counter-clockwise direction d has
// d.y > 0 or (d.y == 0 and d.x < 0) -- exactly one of the two faces of a shared edge.
// rounded products and differences (never contracted into an fma): a query on a vertex gives exactly 0, and the
// two faces of an edge compute bit-identical values
__device__ __forceinline__ double edge_fn(double ax, double ay, double bx, double by, double qx, double qy) {
  return __dsub_rn(__dmul_rn(__dsub_rn(bx, ax), __dsub_rn(qy, ay)), __dmul_rn(__dsub_rn(by, ay), __dsub_rn(qx, ax)));
}

// whether the vertical ray {(x, y, t): t > z} crosses face f of the column (its projection owns (x, y) and the face
// lies above z)
__device__ __forceinline__ bool column_cross(const MeshView& M, int f, double x, double y, double z) {
  const double* F = M.fdata + (int64_t)f * kFaceDoubles;
  const double nzf = F[kFN + 2];
  if (nzf == 0.0) return false;                     // vertical face: its projection has no interior
  const int* vid = M.fvid + 3 * f;
  const double sgn = nzf > 0.0 ? 1.0 : -1.0;        // counter-clockwise projection for N.z > 0
  for (int e = 0; e < 3; ++e) {
    const int a = e, b = (e + 1) % 3;
    const bool fwd = vid[a] < vid[b];
    const double* A = F + kFV + 3 * (fwd ? a : b);
    const double* B = F + kFV + 3 * (fwd ? b : a);
    double E = edge_fn(A[0], A[1], B[0], B[1], x, y);
    if (!fwd) E = -E;
    E *= sgn;
    if (E < 0.0) return false;
    if (E == 0.0) {
      const double* P0 = F + kFV + 3 * a;
      const double* P1 = F + kFV + 3 * b;
      const double dx = (P1[0] - P0[0]) * sgn, dy = (P1[1] - P0[1]) * sgn;
      if (!(dy > 0.0 || (dy == 0.0 && dx < 0.0))) return false;
    }
  }
  const double zt = F[kFV + 2] - (F[kFN] * (x - F[kFV]) + F[kFN + 1] * (y - F[kFV + 1])) / nzf;
  return zt > z;
}

__device__ int mesh_inside(const MeshView& M, double x, double y, double z) {
  const int ix = cell_coord(x, M.lo0, M.cell, M.nx), iy = cell_coord(y, M.lo1, M.cell, M.ny);
  if (ix < 0 || iy < 0 || ix >= M.nx || iy >= M.ny) return 0;
  const int col = iy * M.nx + ix;
  int parity = 0;
  for (int k = M.colstart[col]; k < M.colstart[col + 1]; ++k)
    if (column_cross(M, M.colitems[k], x, y, z)) parity ^= 1;
  return parity;
}

// mesh_inside for a whole warp (every lane calls it with the same point): the lanes test the column's faces 32 at a
// time; the parity of the crossings (an integer count) is the same as the serial walk's
__device__ __forceinline__ int mesh_inside_warp(const MeshView& M, double x, double y, double z, int lane) {
  const int ix = cell_coord(x, M.lo0, M.cell, M.nx), iy = cell_coord(y, M.lo1, M.cell, M.ny);
  if (ix < 0 || iy < 0 || ix >= M.nx || iy >= M.ny) return 0;
  const int col = iy * M.nx + ix;
  const int e = M.colstart[col + 1];
  int crossings = 0;
  for (int base = M.colstart[col]; base < e; base += 32) {
    const int k = base + lane;
    crossings += __popc(__ballot_sync(0xffffffffu, k < e && column_cross(M, M.colitems[k], x, y, z)));
  }
  return crossings & 1;
}

// squared distance from the origin to the triangle P (unit coordinates relative to the query)
__device__ __forceinline__ double tri_dist2(const double P[3][3]) {
  // closest point by the Voronoi-region tests on the barycentric parameters (vertex, edge or interior region)
  const double* A = P[0];
  const double ab[3] = {P[1][0] - A[0], P[1][1] - A[1], P[1][2] - A[2]};
  const double ac[3] = {P[2][0] - A[0], P[2][1] - A[1], P[2][2] - A[2]};
  const double ap[3] = {-A[0], -A[1], -A[2]};
  auto dot = [](const double* x, const double* y) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]; };
  const double d1 = dot(ab, ap), d2 = dot(ac, ap);
  double cp[3];
  auto setp = [&](double v, double w) {
    for (int k = 0; k < 3; ++k) cp[k] = A[k] + v * ab[k] + w * ac[k];
  };
  if (d1 <= 0.0 && d2 <= 0.0) {
    setp(0.0, 0.0);
  } else {
    const double bp[3] = {-P[1][0], -P[1][1], -P[1][2]};
    const double e3 = dot(ab, bp), e4 = dot(ac, bp);
    if (e3 >= 0.0 && e4 <= e3) {
      setp(1.0, 0.0);
    } else {
      const double vc = d1 * e4 - e3 * d2;
      if (vc <= 0.0 && d1 >= 0.0 && e3 <= 0.0) {
        setp(d1 / (d1 - e3), 0.0);
      } else {
        const double cpn[3] = {-P[2][0], -P[2][1], -P[2][2]};
        const double e5 = dot(ab, cpn), e6 = dot(ac, cpn);
        if (e6 >= 0.0 && e5 <= e6) {
          setp(0.0, 1.0);
        } else {
          const double vb = e5 * d2 - d1 * e6;
          if (vb <= 0.0 && d2 >= 0.0 && e6 <= 0.0) {
            setp(0.0, d2 / (d2 - e6));
          } else {
            const double va = e3 * e6 - e5 * e4;
            if (va <= 0.0 && (e4 - e3) >= 0.0 && (e5 - e6) >= 0.0) {
              const double t = (e4 - e3) / ((e4 - e3) + (e5 - e6));
              setp(1.0 - t, t);
            } else {
              const double den = 1.0 / (va + vb + vc);
              setp(vb * den, vc * den);
            }
          }
        }
      }
    }
  }
  return cp[0] * cp[0] + cp[1] * cp[1] + cp[2] * cp[2];
}

// ------------------------------------------------------------------------------------------ candidate faces
// The cells of the block x0..x1, y0..y1, z0..z1 (at most 27) for a warp: lane l < number of cells takes cell ordinal
// l (z outermost, then y, then x -- the order of nested loops) and returns its first item (beg) and the exclusive
// prefix of the items of the cells before it (pref; a cell `keep` rejects has none).  Returns the block's total.
template <class Keep>
__device__ __forceinline__ int block_cells(const MeshView& M, int x0, int x1, int y0, int y1, int z0, int z1, int lane,
                                           Keep&& keep, int& beg, int& pref) {
  const int nxr = x1 - x0 + 1, nyr = y1 - y0 + 1, nc = nxr * nyr * (z1 - z0 + 1);
  int cnt = 0;
  beg = 0;
  if (lane < nc) {
    const int i = x0 + lane % nxr, j = y0 + (lane / nxr) % nyr, k = z0 + lane / (nxr * nyr);
    if (keep(i, j, k)) {
      const int c = (k * M.ny + j) * M.nx + i;
      beg = M.cstart[c];
      cnt = M.cstart[c + 1] - beg;
    }
  }
  int inc = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += v;
  }
  pref = inc - cnt;
  return __shfl_sync(0xffffffffu, inc, 31);
}

// the cell ordinal of flattened item t (< total): the last lane whose prefix is <= t (prefixes do not decrease with
// the lane; an empty cell shares the next cell's prefix, lanes past the cells hold the total), by a binary search over
// the lanes; every lane of the warp takes part
__device__ __forceinline__ int cell_ordinal(int pref, int t) {
  int lo = 0;
#pragma unroll
  for (int step = 16; step > 0; step >>= 1) {
    const int pv = __shfl_sync(0xffffffffu, pref, lo + step);
    if (pv <= t) lo += step;
  }
  return lo;
}

// The faces of the 27 cells around the query's cell that come within h of the query (box first, then the exact
// triangle distance, both tested by the lanes in parallel); a face listed in several of those cells is taken in one of
// them only (the lowest corner of its box inside the 27-cell block).  Called by a whole warp with one query: the (cell, item) pairs of the block are flattened over the lanes (32 at a time, whatever
// cell they belong to), and the faces that pass are visited one after the other, warp-uniformly, in cell order and
// item order within a cell -- a fixed order, so the sums the visits accumulate do not depend on the launch.
template <class Visit>
__device__ __forceinline__ void for_candidates_warp(const MeshView& M, const double q[3], double h, int lane,
                                                    Visit&& visit) {
  const int cx = cell_coord(q[0], M.lo0, M.cell, M.nx), cy = cell_coord(q[1], M.lo1, M.cell, M.ny),
            cz = cell_coord(q[2], M.lo2, M.cell, M.nz);
  const int x0 = max(cx - 1, 0), x1 = min(cx + 1, M.nx - 1), y0 = max(cy - 1, 0), y1 = min(cy + 1, M.ny - 1),
            z0 = max(cz - 1, 0), z1 = min(cz + 1, M.nz - 1);
  if (x0 > x1 || y0 > y1 || z0 > z1) return;
  const double h2 = h * h;
  const int nxr = x1 - x0 + 1, nyr = y1 - y0 + 1;
  int beg, pref;
  const int total = block_cells(M, x0, x1, y0, y1, z0, z1, lane, [](int, int, int) { return true; }, beg, pref);
  for (int base = 0; base < total; base += 32) {
    const int t = base + lane;
    const int o = cell_ordinal(pref, t);
    const int b = __shfl_sync(0xffffffffu, beg, o), p = __shfl_sync(0xffffffffu, pref, o);
    int f = -1;
    bool hit = false;
    if (t < total) {
      const int i = x0 + o % nxr, j = y0 + (o / nxr) % nyr, k = z0 + o / (nxr * nyr);
      f = M.citems[b + (t - p)];
      const int* fc = M.fcell + 3 * f;
      if (max(fc[0], cx - 1) == i && max(fc[1], cy - 1) == j && max(fc[2], cz - 1) == k) {
        const double* F = M.fdata + (int64_t)f * kFaceDoubles;
        double d2 = 0.0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const double dl = F[kFLO + a] - q[a], dh = q[a] - F[kFHI + a];
          const double d = fmax(0.0, fmax(dl, dh));
          d2 = fma(d, d, d2);
        }
        if (d2 < h2) {
          // the exact triangle distance (unit coordinates relative to the query, the operations of the visit's P)
          const double ih = 1.0 / h;
          double P[3][3];
#pragma unroll
          for (int v = 0; v < 3; ++v)
#pragma unroll
            for (int a = 0; a < 3; ++a) P[v][a] = (F[kFV + 3 * v + a] - q[a]) * ih;
          hit = tri_dist2(P) < 1.0;
        }
      }
    }
    unsigned m = __ballot_sync(0xffffffffu, hit);
    while (m) {
      const int bl = __ffs(m) - 1;
      m &= m - 1;
      visit(__shfl_sync(0xffffffffu, f, bl));
    }
  }
}

// whether any face box comes within h of the query (the cells of for_candidates_warp, stopping at the first hit),
// for a whole warp (every lane calls it with the same query): the (cell, item) pairs are flattened over the lanes.
// A cell whose own box is h or more from the query is skipped: a face box within h of the query has its point nearest
// to the query in a cell within h, and every cell its box overlaps lists the face (a relative margin far above the
// rounding of the cell boxes: a cell is only skipped when clearly out of reach).
__device__ __forceinline__ bool has_candidate_warp(const MeshView& M, const double q[3], double h, int lane) {
  const int cx = cell_coord(q[0], M.lo0, M.cell, M.nx), cy = cell_coord(q[1], M.lo1, M.cell, M.ny),
            cz = cell_coord(q[2], M.lo2, M.cell, M.nz);
  const int x0 = max(cx - 1, 0), x1 = min(cx + 1, M.nx - 1), y0 = max(cy - 1, 0), y1 = min(cy + 1, M.ny - 1),
            z0 = max(cz - 1, 0), z1 = min(cz + 1, M.nz - 1);
  if (x0 > x1 || y0 > y1 || z0 > z1) return false;
  const double h2 = h * h;
  auto gap2 = [&](double x, double lo, int i) {
    const double a = fma((double)i, M.cell, lo), d = fmax(0.0, fmax(a - x, x - (a + M.cell)));
    return d * d;
  };
  auto reach = [&](int i, int j, int k) {
    return gap2(q[0], M.lo0, i) + gap2(q[1], M.lo1, j) + gap2(q[2], M.lo2, k) < h2 * (1.0 + 1e-9);
  };
  int beg, pref;
  const int total = block_cells(M, x0, x1, y0, y1, z0, z1, lane, reach, beg, pref);
  for (int base = 0; base < total; base += 32) {
    const int t = base + lane;
    const int o = cell_ordinal(pref, t);
    const int b = __shfl_sync(0xffffffffu, beg, o), p = __shfl_sync(0xffffffffu, pref, o);
    bool hit = false;
    if (t < total) {
      const double* F = M.fdata + (int64_t)M.citems[b + (t - p)] * kFaceDoubles;
      double d2 = 0.0;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const double d = fmax(0.0, fmax(F[kFLO + a] - q[a], q[a] - F[kFHI + a]));
        d2 = fma(d, d, d2);
      }
      hit = d2 < h2;
    }
    if (__any_sync(0xffffffffu, hit)) return true;
  }
  return false;
}

// ------------------------------------------------------------------------------------------ profiles
template <class M, int Fn>
__device__ __forceinline__ double fpoly(int p, double x) {
  if constexpr (M::kPieces > 1) {
    if (p) return MeshFn<M, Fn>::poly1(x);
  }
  return MeshFn<M, Fn>::poly0(x);
}
template <class M, int Fn>
__device__ __forceinline__ double fdd(int p, double x, double a) {
  if constexpr (M::kPieces > 1) {
    if (p) return MeshFn<M, Fn>::dd1(x, a);
  }
  return MeshFn<M, Fn>::dd0(x, a);
}
// the divided difference fdd in two halves: the synthetic-division coefficients of piece p at a (kMeshDD slots), and
// Horner's rule over them at x -- the same fma sequence as fdd, so the same value
constexpr int kMeshDD = 24;
template <class M, int Fn>
__device__ __forceinline__ void fddb(int p, double a, double* b) {
  static_assert(MeshFn<M, Fn>::kDD0 <= kMeshDD, "coefficient slots");
  if constexpr (M::kPieces > 1) {
    static_assert(MeshFn<M, Fn>::kDD1 <= kMeshDD, "coefficient slots");
    if (p) {
      MeshFn<M, Fn>::ddb1(a, b);
      return;
    }
  }
  MeshFn<M, Fn>::ddb0(a, b);
}
template <class M, int Fn>
__device__ __forceinline__ double fddh(int p, double x, const double* b) {
  if constexpr (M::kPieces > 1) {
    if (p) return MeshFn<M, Fn>::ddh1(x, b);
  }
  return MeshFn<M, Fn>::ddh0(x, b);
}
template <class M, int Fn>
__device__ __forceinline__ double fnu(int p) {
  if constexpr (M::kPieces > 1) {
    if (p) return MeshFn<M, Fn>::kNu1;
  }
  return MeshFn<M, Fn>::kNu0;
}
template <int K>
__device__ __forceinline__ double zpow(double z) {
  if constexpr (K == 0) return 1.0;
  else if constexpr (K == 1) return z;
  else if constexpr (K == 2) return z * z;
  else return z * z * z;
}
// sum_{i < m} x^i a^(m-1-i)
template <int m>
__device__ __forceinline__ double smix(double x, double a) {
  if constexpr (m == 1) return 1.0;
  else if constexpr (m == 2) return x + a;
  else return fma(x, x + a, a * a);
}
template <class M>
__device__ __forceinline__ int piece(double x) {
  if constexpr (M::kPieces > 1) return x < M::kBreak ? 0 : 1;
  return 0;
}

// A_F(r) (r inside the support); ir = 1 / r
template <class M, int Fn>
__device__ __forceinline__ double aval(double r, double ir) {
  constexpr int m = MeshFn<M, Fn>::kNeg;
  const int p = piece<M>(r);
  double v = fpoly<M, Fn>(p, r);
  if constexpr (m > 0) v = fma(fnu<M, Fn>(p), zpow<m>(ir), v);
  return v;
}

// z^ZP A_F(|z|), |z| = a (0 outside the support); sg = sign(z)
template <class M, int Fn, int ZP>
__device__ __forceinline__ double aval_a(double a, double z, double sg) {
  constexpr int m = MeshFn<M, Fn>::kNeg;
  static_assert(ZP >= m, "z power must absorb the negative power");
  if (a >= 1.0) return 0.0;
  const int p = piece<M>(a);
  double v = fpoly<M, Fn>(p, a) * zpow<ZP>(z);
  if constexpr (m > 0) v += fnu<M, Fn>(p) * zpow<ZP - m>(z) * zpow<m>(sg);
  return v;
}

// node quantities shared by the six divided differences: r, 1/r, 1/(r + a), 1/rho^2, and whether the segment
// [a, r] crosses the kernel's knot
struct Node {
  double r, ir, irpa, irho2;
  bool split;
};

// z^ZP (A_F(r) - A_F(a)) / (r^2 - a^2) for a = |z| < r < 1.  Within one piece the divided difference of the
// polynomial part comes from synthetic division (no cancellation between A(r) and A(a)); the negative power
// nu r^-m gives -nu S_m(r, a) / (r^m a^m), whose 1 / a^m is absorbed by z^ZP.  Across the knot B the two pieces'
// differences are weighted by (B - a) and (r - B) over r - a = rho^2 / (r + a).
template <class M, int Fn, int ZP>
__device__ __forceinline__ double dd2(const Node& nd, double a, double z, double sg, const double* fb) {
  constexpr int m = MeshFn<M, Fn>::kNeg;
  static_assert(ZP >= m, "z power must absorb the negative power");
  const int pa = piece<M>(a);
  if (!nd.split) {
    double d0 = fddh<M, Fn>(pa, nd.r, fb + Fn * kMeshDD) * zpow<ZP>(z);
    if constexpr (m > 0) d0 -= fnu<M, Fn>(pa) * smix<m>(nd.r, a) * zpow<m>(nd.ir) * zpow<ZP - m>(z) * zpow<m>(sg);
    return d0 * nd.irpa;
  }
  constexpr double B = M::kBreak;
  double d0 = fdd<M, Fn>(0, B, a) * zpow<ZP>(z);
  if constexpr (m > 0) d0 -= fnu<M, Fn>(0) * smix<m>(B, a) * (1.0 / zpow<m>(B)) * zpow<ZP - m>(z) * zpow<m>(sg);
  double d1 = fdd<M, Fn>(1, nd.r, B);
  if constexpr (m > 0) d1 -= fnu<M, Fn>(1) * smix<m>(nd.r, B) * zpow<m>(nd.ir) * (1.0 / zpow<m>(B));
  d1 *= zpow<ZP>(z);
  return ((B - a) * d0 + (nd.r - B) * d1) * nd.irho2;
}

__device__ __forceinline__ double angle_between(double w, double x0, double x1) {
  return atan2(w * (x1 - x0), fma(w, w, x0 * x1));
}

// the 28 accumulators of one row (W~ units, unit support): M0, M1[3], M2[6] (00 01 02 11 12 22), G0[3],
// G1[9] (i-major), H[6]
enum { kAM0 = 0, kAM1 = 1, kAM2 = 4, kAG0 = 10, kAG1 = 13, kAH = 22 };
struct Acc28 {
  double v[28];
};

__device__ __forceinline__ void acc_zero(Acc28& A) {
#pragma unroll
  for (int i = 0; i < 28; ++i) A.v[i] = 0.0;
}

// per-edge integrals accumulated over the panels of one side of the foot point
struct EdgeSums {
  double J[6];   // w int z^p DD_F ds for A_K0 (p1) A_K1 (p2) A_K2 (p3) A_W A_L A2_K2 (p1)
  double LK1, LK2, LK2b, TK2, LW, LL;   // int z A_K1, int z^2 A_K2, int z A_K2, int s z A_K2, int A_W, int A_L
};

// one quadrature node u (distance from the foot along the edge, s = sgn_side * u) with weight wt, in two parts that
// each form r and 1 / r themselves, so that fewer values are live at once: the six divided differences (w != 0 only),
// then the six potential sums (one loop over an edge's nodes calls both: measured 9.2 ms for the c3 leg against 9.7
// ms with a loop for each)
template <class M>
__device__ __forceinline__ void node_eval_dd(double u, double wt, double c2, double a, double z, double sg, double w,
                                             const double* fb, EdgeSums& S) {
  const double rho2 = fma(u, u, w * w);
  Node nd;
  nd.r = sqrt(fma(u, u, c2));
  nd.ir = 1.0 / nd.r;
  nd.split = M::kPieces > 1 && a < M::kBreak && nd.r > M::kBreak;
  nd.irpa = 1.0 / (nd.r + a);
  nd.irho2 = nd.split ? 1.0 / rho2 : 0.0;
  const double ww = w * wt;
  S.J[0] = fma(ww, dd2<M, 0, 1>(nd, a, z, sg, fb), S.J[0]);
  S.J[1] = fma(ww, dd2<M, 1, 2>(nd, a, z, sg, fb), S.J[1]);
  S.J[2] = fma(ww, dd2<M, 2, 3>(nd, a, z, sg, fb), S.J[2]);
  S.J[3] = fma(ww, dd2<M, 3, 0>(nd, a, z, sg, fb), S.J[3]);
  S.J[4] = fma(ww, dd2<M, 4, 0>(nd, a, z, sg, fb), S.J[4]);
  S.J[5] = fma(ww, dd2<M, 5, 1>(nd, a, z, sg, fb), S.J[5]);
}

template <class M>
__device__ __forceinline__ void node_eval_pot(double u, double wt, double sgn_side, double c2, double z,
                                              EdgeSums& S) {
  const double s = sgn_side * u;
  const double r = sqrt(fma(u, u, c2));
  const double ir = 1.0 / r;
  const double k1 = aval<M, 1>(r, ir) * z, k2 = aval<M, 2>(r, ir) * z;
  S.LK1 = fma(wt, k1, S.LK1);
  S.LK2b = fma(wt, k2, S.LK2b);
  S.LK2 = fma(wt, k2 * z, S.LK2);
  S.TK2 = fma(wt * s, k2, S.TK2);
  S.LW = fma(wt, aval<M, 3>(r, ir), S.LW);
  S.LL = fma(wt, aval<M, 4>(r, ir), S.LL);
}

// the panels of one edge (both sides of the foot of the perpendicular): [u0, u1] of distances from the foot, split
// at the kernel's knot and at c 2^k (k >= 1); at most 26 panels a side (c 2^k runs from 2^-24 to 1).  A panel that
// starts within 2c of the foot (the branch points of r sit at distance c from the foot) takes 16 Gauss-Legendre
// nodes (relative error below 2e-15 on [0, 2c]), the graded ones further out 12 (below 1e-18 on [2^k c, 2^(k+1) c]).
// A typical edge (side lengths up to 2c) is then 32 nodes: one round of the warp's lanes.
constexpr int kMaxPanels = 64;
struct PanelList {
  double lo[kMaxPanels], hi[kMaxPanels], sg[kMaxPanels];
  int off[kMaxPanels + 1];    // first node of each panel; off[np] = all nodes
};

// an edge of the face being evaluated, relative to the query in units of the support: tangent t and in-plane normal
// mu, the foot's signed distance w to the edge line, the edge's ends lo, hi along t from the foot, c^2 = z^2 + w^2,
// the part [s0, s1] inside the support, and its panel count
struct EdgeGeo {
  double t[3], mu[3], w, lo, hi, c2, s0, s1;
  int np;
};

template <class M>
__device__ int build_panels(PanelList& PL, double s0, double s1, double c) {
  int np = 0, nodes = 0;
  double knot = -1.0;
  if constexpr (M::kPieces > 1) {
    if (c < M::kBreak) knot = sqrt((M::kBreak - c) * (M::kBreak + c));
  }
  const double base = fmax(c, 1.0 / 16777216.0);
  for (int side = 0; side < 2; ++side) {
    const double sgn = side == 0 ? -1.0 : 1.0;
    const double u0 = side == 0 ? fmax(-s1, 0.0) : fmax(s0, 0.0);
    const double u1 = side == 0 ? -s0 : s1;
    if (!(u1 > u0)) continue;
    double d = 2.0 * base;
    for (int it = 0; it < 64 && d <= u0; ++it) d *= 2.0;
    double u = u0;
    for (int it = 0; it < 96 && u < u1 && np < kMaxPanels; ++it) {
      double nxt = fmin(u1, d);
      if (knot > u && knot < nxt) nxt = knot;
      PL.lo[np] = u;
      PL.hi[np] = nxt;
      PL.sg[np] = sgn;
      PL.off[np] = nodes;
      nodes += u < 2.0 * base ? 16 : 12;
      ++np;
      if (nxt >= d) d *= 2.0;
      u = nxt;
    }
  }
  PL.off[np] = nodes;
  return np;
}

// the warp's sums of twelve values, in every lane: lanes 16 apart swap six values and keep the sums of the other six,
// lanes 8 apart swap three, a butterfly over the last three lane bits completes each group of eight lanes' three sums,
// and each total is broadcast from its group (a fixed order: deterministic)
__device__ __forceinline__ void warp_sum12(double v[12]) {
  const int lane = threadIdx.x & 31;
  const bool up = (lane >> 4) & 1, b3 = (lane >> 3) & 1;
  double a[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const double give = up ? v[k] : v[k + 6];
    const double keep = up ? v[k + 6] : v[k];
    a[k] = keep + __shfl_xor_sync(0xffffffffu, give, 16);
  }
  double b[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double give = b3 ? a[k] : a[k + 3];
    const double keep = b3 ? a[k + 3] : a[k];
    b[k] = keep + __shfl_xor_sync(0xffffffffu, give, 8);
  }
#pragma unroll
  for (int off = 4; off > 0; off >>= 1)
#pragma unroll
    for (int k = 0; k < 3; ++k) b[k] += __shfl_xor_sync(0xffffffffu, b[k], off);
#pragma unroll
  for (int x = 0; x < 12; ++x) v[x] = __shfl_sync(0xffffffffu, b[x % 3], 8 * (x / 3));
}


// Assembly (W~ units), per edge:  M0 += J0;  M1_i += N_i J1 + mu_i LK1;
// M2_ij += N_i N_j (J2 + J5) + (N_i mu_j + mu_i N_j) LK2 + mu_i mu_j w LK2b + (mu_i t_j + mu_j t_i) TK2 / 2 - d_ij J5;
// G0_i -= N_i J3;  G1_ij -= z N_i N_j J3 + mu_i N_j LW;  H_ij += z N_i N_j J4 + (N_i mu_j + mu_i N_j) LL / 2.
// Lane k < 28 adds the term of accumulator k: every term is one bilinear form in the vectors N, mu, t whose
// coefficients a lane selects by its accumulator's type, so all lanes run the same instructions.  The J terms multiply
// face quantities (N, z) only, so they are added once per face with J summed over the face's edges; the LK / TK / LW
// / LL terms, which carry the edge's mu and t, once per edge.
enum { kTM0, kTM1, kTM2, kTG0, kTG1, kTH, kTNone };
struct AccSlot {
  int type, i, j;
};

__device__ __forceinline__ AccSlot acc_slot(int k) {
  auto sym_i = [](int x) { return x < 3 ? 0 : (x < 5 ? 1 : 2); };
  auto sym_j = [](int x) { return x < 3 ? x : (x < 5 ? x - 2 : 2); };
  if (k == kAM0) return {kTM0, 0, 0};
  if (k < kAM2) return {kTM1, k - kAM1, 0};
  if (k < kAG0) return {kTM2, sym_i(k - kAM2), sym_j(k - kAM2)};
  if (k < kAG1) return {kTG0, k - kAG0, 0};
  if (k < kAH) return {kTG1, (k - kAG1) / 3, (k - kAG1) % 3};
  if (k < 28) return {kTH, sym_i(k - kAH), sym_j(k - kAH)};
  return {kTNone, 0, 0};
}

__device__ __forceinline__ double pick3(const double v[3], int i) { return i == 0 ? v[0] : (i == 1 ? v[1] : v[2]); }

// the terms of accumulator sl with the edge's vectors mu, t (per edge)
__device__ __forceinline__ double edge_term_mu(const AccSlot& sl, const double N[3], const double t[3],
                                               const double mu[3], double w, const EdgeSums& S) {
  const double Ni = pick3(N, sl.i), Nj = pick3(N, sl.j), mi = pick3(mu, sl.i), mj = pick3(mu, sl.j);
  const double ti = pick3(t, sl.i), tj = pick3(t, sl.j);
  const double X = Ni * mj + mi * Nj, MN = mi * Nj, MM = mi * mj, MT = 0.5 * (mi * tj + mj * ti);
  const int ty = sl.type;
  const double cMi = ty == kTM1 ? S.LK1 : 0.0;
  const double cX = ty == kTM2 ? S.LK2 : (ty == kTH ? 0.5 * S.LL : 0.0);
  const double cMN = ty == kTG1 ? -S.LW : 0.0;
  const double cMM = ty == kTM2 ? w * S.LK2b : 0.0;
  const double cMT = ty == kTM2 ? S.TK2 : 0.0;
  return mi * cMi + X * cX + MN * cMN + MM * cMM + MT * cMT;
}

// the terms of accumulator sl with the J sums (face quantities N, z only: once per face, J summed over its edges)
__device__ __forceinline__ double face_term_j(const AccSlot& sl, const double N[3], double z, const double J[6]) {
  const double Ni = pick3(N, sl.i), Nj = pick3(N, sl.j);
  const double NN = Ni * Nj, dij = sl.i == sl.j ? 1.0 : 0.0;
  const int ty = sl.type;
  const double cC = ty == kTM0 ? J[0] : 0.0;
  const double cNi = ty == kTM1 ? J[1] : (ty == kTG0 ? -J[3] : 0.0);
  const double cNN = ty == kTM2 ? J[2] + J[5] : (ty == kTG1 ? -z * J[3] : (ty == kTH ? z * J[4] : 0.0));
  const double cD = ty == kTM2 ? -J[5] : 0.0;
  return cC + Ni * cNi + NN * cNN + dij * cD;
}

// the contribution of face f to the row's accumulators (lane k < 28 holds accumulator k in acc), computed by the
// whole warp: the geometry is the same in every lane, the quadrature nodes of an edge (12 or 16 per panel) are spread over the lanes and
// their sums reduced by a fixed butterfly, then lane k adds the edge's term of accumulator k (slot: this lane's).
// Everything is linear in the per-edge integrals.  Faces that do not meet the support contribute exactly nothing:
// the candidate search visits only faces within the support.  q in world units, ih = 1 / support.
template <class M>
__device__ void face_contrib_warp(const MeshView& Mv, int f, const double q[3], double ih, PanelList* PL3,
                                  EdgeGeo* G3, double* FB, int lane, const AccSlot& slot, double& acc) {
  const double* F = Mv.fdata + (int64_t)f * kFaceDoubles;
  double P[3][3];
#pragma unroll
  for (int v = 0; v < 3; ++v)
#pragma unroll
    for (int k = 0; k < 3; ++k) P[v][k] = (F[kFV + 3 * v + k] - q[k]) * ih;
  const double N[3] = {F[kFN], F[kFN + 1], F[kFN + 2]};
  const double z = N[0] * P[0][0] + N[1] * P[0][1] + N[2] * P[0][2];
  const double a = fabs(z), sg = z > 0.0 ? 1.0 : (z < 0.0 ? -1.0 : 0.0);
  // the three edges' geometry and panel lists, lane e for edge e, side by side (the previous face's lists are read)
  __syncwarp();
  if (lane < 3) {
    const int e = lane;
    EdgeGeo& ge = G3[e];
    // the edge's first vertex relative to the query: the same operations as P[e]
    const double pe[3] = {(F[kFV + 3 * e] - q[0]) * ih, (F[kFV + 3 * e + 1] - q[1]) * ih,
                          (F[kFV + 3 * e + 2] - q[2]) * ih};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      ge.t[k] = F[kFT + 3 * e + k];
      ge.mu[k] = F[kFMU + 3 * e + k];
    }
    const double len = F[kFLEN + e] * ih;
    ge.w = ge.mu[0] * pe[0] + ge.mu[1] * pe[1] + ge.mu[2] * pe[2];
    ge.lo = ge.t[0] * pe[0] + ge.t[1] * pe[1] + ge.t[2] * pe[2];
    ge.hi = ge.lo + len;
    ge.c2 = fma(z, z, ge.w * ge.w);
    const double c = sqrt(ge.c2);
    double s0 = 0.0, s1 = 0.0;
    if (c < 1.0) {
      const double L = sqrt((1.0 - c) * (1.0 + c));
      s0 = fmax(ge.lo, -L);
      s1 = fmin(ge.hi, L);
    }
    ge.s0 = s0;
    ge.s1 = s1;
    ge.np = s1 > s0 ? build_panels<M>(PL3[e], s0, s1, c) : 0;
  } else if (lane == 3) {
    // the synthetic-division coefficients of the six divided differences at a = |z| (a face constant), once per face
    // instead of once per node
    const int pa = piece<M>(a);
    fddb<M, 0>(pa, a, FB);
    fddb<M, 1>(pa, a, FB + kMeshDD);
    fddb<M, 2>(pa, a, FB + 2 * kMeshDD);
    fddb<M, 3>(pa, a, FB + 3 * kMeshDD);
    fddb<M, 4>(pa, a, FB + 4 * kMeshDD);
    fddb<M, 5>(pa, a, FB + 5 * kMeshDD);
  }
  __syncwarp();
  double Jf[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};          // the face's J sums over its edges
  double out = 0.0;                                       // the face's summed angles beyond the support
  for (int e = 0; e < 3; ++e) {
    const EdgeGeo& ge = G3[e];
    const PanelList& PL = PL3[e];
    const double t[3] = {ge.t[0], ge.t[1], ge.t[2]}, mu[3] = {ge.mu[0], ge.mu[1], ge.mu[2]};
    const double w = ge.w, lo = ge.lo, hi = ge.hi, c2 = ge.c2, s0 = ge.s0, s1 = ge.s1;
    EdgeSums S;
#pragma unroll
    for (int i = 0; i < 6; ++i) S.J[i] = 0.0;
    S.LK1 = S.LK2 = S.LK2b = S.TK2 = S.LW = S.LL = 0.0;
    if (s1 > s0) {
      const int np = ge.np;
      int p = 0;
      for (int k = lane; k < PL.off[np]; k += 32) {
        while (k >= PL.off[p + 1]) ++p;
        const int g = k - PL.off[p];
        const bool n16 = PL.off[p + 1] - PL.off[p] == 16;
        const double xg = n16 ? kTriGx16[g] : kRadialGx[g], wg = n16 ? kTriGw16[g] : kRadialGw[g];
        const double x0 = PL.lo[p], x1 = PL.hi[p];
        const double hc = 0.5 * (x1 - x0);
        const double u = fma(hc, xg, 0.5 * (x1 + x0)), wt = wg * hc;
        if (w != 0.0) node_eval_dd<M>(u, wt, c2, a, z, sg, w, FB, S);
        node_eval_pot<M>(u, wt, PL.sg[p], c2, z, S);
      }
      double v[12] = {S.J[0], S.J[1], S.J[2], S.J[3], S.J[4], S.J[5], S.LK1, S.LK2, S.LK2b, S.TK2, S.LW, S.LL};
      warp_sum12(v);
#pragma unroll
      for (int i = 0; i < 6; ++i) S.J[i] = v[i];
      S.LK1 = v[6];
      S.LK2 = v[7];
      S.LK2b = v[8];
      S.TK2 = v[9];
      S.LW = v[10];
      S.LL = v[11];
    }
    if (w != 0.0) {
      if (s1 > s0) {
        if (lo < s0) out += angle_between(w, lo, s0);
        if (s1 < hi) out += angle_between(w, s1, hi);
      } else {
        out += angle_between(w, lo, hi);
      }
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) Jf[i] += S.J[i];
    // assembly of the terms with the edge's vectors: lane k adds its accumulator's (the sums are in every lane)
    if (lane < 28) acc += edge_term_mu(slot, N, t, mu, w, S);
  }
  // the J terms multiply face quantities only: the face's three edges summed, with the angle part of the edges
  // beyond the support (a face constant times the summed angle) taken once
  if (out != 0.0) {
    Jf[0] -= aval_a<M, 0, 1>(a, z, sg) * out;
    Jf[1] -= aval_a<M, 1, 2>(a, z, sg) * out;
    Jf[2] -= aval_a<M, 2, 3>(a, z, sg) * out;
    Jf[3] -= aval_a<M, 3, 0>(a, z, sg) * out;
    Jf[4] -= aval_a<M, 4, 0>(a, z, sg) * out;
    Jf[5] -= aval_a<M, 5, 1>(a, z, sg) * out;
  }
  if (lane < 28) acc += face_term_j(slot, N, z, Jf);
}

// ------------------------------------------------------------------------------------------ kernels
constexpr int kMeshThreads = 128;

// the per-cell flags, once per mesh: emptiness, the inside status of an empty cell's centre (the column parity test),
// whether any of the 27 cells around holds a face
__global__ void k_mesh_cellflags(MeshView M, uint8_t* __restrict__ flags) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nxy = (int64_t)M.nx * M.ny;
  if (c >= nxy * M.nz) return;
  const int i = (int)(c % M.nx), j = (int)((c / M.nx) % M.ny), k = (int)(c / nxy);
  uint8_t f = 0;
  if (M.cstart[c] == M.cstart[c + 1]) {
    f |= kCellEmpty;
    const double x = M.lo0 + (i + 0.5) * M.cell, y = M.lo1 + (j + 0.5) * M.cell, z = M.lo2 + (k + 0.5) * M.cell;
    if (mesh_inside(M, x, y, z)) f |= kCellInside;
  }
  for (int dk = -1; dk <= 1; ++dk)
    for (int dj = -1; dj <= 1; ++dj)
      for (int di = -1; di <= 1; ++di) {
        const int a = i + di, b = j + dj, e = k + dk;
        if (a < 0 || b < 0 || e < 0 || a >= M.nx || b >= M.ny || e >= M.nz) continue;
        const int64_t n = ((int64_t)e * M.ny + b) * M.nx + a;
        if (M.cstart[n] != M.cstart[n + 1]) f |= kCellNear;
      }
  flags[c] = f;
}

// Per query, first pass: the cell's flags settle the rows away from the surface (inside status of an empty cell, no
// faces within the support when no face box meets the 27 cells around); the others are appended to `near`, so the
// second pass runs the parity walk and the face search on full warps of such rows.  Invalid rows (a support above the
// grid cell would reach faces outside the 27-cell block, non-finite input) are marked -1 and come back as NaN.
__global__ void __launch_bounds__(kMeshThreads) k_mesh_rowinfo(MeshView M, const double* __restrict__ pos,
                                                              const double* __restrict__ sup, int64_t n,
                                                              int32_t* __restrict__ ind, int32_t* __restrict__ near,
                                                              int32_t* __restrict__ nnear) {
  const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool listed = false;
  if (row < n) {
    const double q[3] = {pos[3 * row], pos[3 * row + 1], pos[3 * row + 2]};
    const double h = sup[row];
    const bool ok = h > 0.0 && h <= M.cell && isfinite(q[0]) && isfinite(q[1]) && isfinite(q[2]);
    if (!ok) {
      ind[row] = -1;
    } else {
      const int cx = cell_coord(q[0], M.lo0, M.cell, M.nx), cy = cell_coord(q[1], M.lo1, M.cell, M.ny),
                cz = cell_coord(q[2], M.lo2, M.cell, M.nz);
      const bool in_grid = cx >= 0 && cy >= 0 && cz >= 0 && cx < M.nx && cy < M.ny && cz < M.nz;
      // more than a cell outside the grid along some axis (cell_coord gives -2 or n + 1): the grid reaches a cell
      // (>= the support) past the surface's box, so no face is within the support and the query is outside the solid
      const bool far = cx == -2 || cy == -2 || cz == -2 || cx == M.nx + 1 || cy == M.ny + 1 || cz == M.nz + 1;
      const uint8_t f = in_grid ? M.cflag[((int64_t)cz * M.ny + cy) * M.nx + cx] : (uint8_t)(far ? 0 : kCellNear);
      if (!(f & kCellNear)) {
        ind[row] = (f & kCellInside) ? 1 : 0;     // no face box in the 27 cells: the cell is empty as well
      } else {
        listed = true;
      }
    }
  }
  const unsigned mask = __ballot_sync(0xffffffffu, listed);
  if (mask) {
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(nnear, __popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (listed) near[base + __popc(mask & ((1u << lane) - 1))] = (int32_t)row;
  }
}

// Second pass over the listed rows: the inside test (the cell's flag where the cell is empty, the parity walk
// otherwise) and whether any face is within the support; rows with faces are appended to `work`
__global__ void __launch_bounds__(kMeshThreads) k_mesh_rownear(MeshView M, const double* __restrict__ pos,
                                                              const double* __restrict__ sup,
                                                              const int32_t* __restrict__ near,
                                                              const int32_t* __restrict__ nnear,
                                                              int32_t* __restrict__ ind, int32_t* __restrict__ work,
                                                              int32_t* __restrict__ nwork) {
  // one warp per listed row (the warps of the grid stride over them): the column's faces and the candidate cells'
  // items are tested 32 at a time
  const int lane = threadIdx.x & 31;
  const int64_t m = *nnear;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x / 32);
  for (int64_t t = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; t < m; t += warps) {
    const int32_t row = near[t];
    const double q[3] = {pos[3 * row], pos[3 * row + 1], pos[3 * row + 2]};
    const double h = sup[row];
    const int cx = cell_coord(q[0], M.lo0, M.cell, M.nx), cy = cell_coord(q[1], M.lo1, M.cell, M.ny),
              cz = cell_coord(q[2], M.lo2, M.cell, M.nz);
    const bool in_grid = cx >= 0 && cy >= 0 && cz >= 0 && cx < M.nx && cy < M.ny && cz < M.nz;
    const uint8_t f = in_grid ? M.cflag[((int64_t)cz * M.ny + cy) * M.nx + cx] : (uint8_t)0;
    const int inside = (f & kCellEmpty) ? ((f & kCellInside) ? 1 : 0) : mesh_inside_warp(M, q[0], q[1], q[2], lane);
    const bool has = has_candidate_warp(M, q, h, lane);
    if (lane == 0) {
      ind[row] = inside;
      if (has) work[atomicAdd(nwork, 1)] = row;     // (the order is irrelevant: each row is computed alone)
    }
  }
}

template <class M>
__device__ __forceinline__ void write_row(double* __restrict__ out, int64_t row, const Acc28& A, double ind, double h) {
  const double ip = kInvPi;
  const double M0 = A.v[kAM0] * ip + ind * 4.0 * M::kQ0;
  const double m2c = ind * (4.0 / 3.0) * M::kQ2;
  const double h2 = h * h, ih = 1.0 / h, ih2 = ih * ih;
  double* o = out + row * 28;
  o[0] = M0;
#pragma unroll
  for (int i = 0; i < 3; ++i) o[1 + i] = A.v[kAM1 + i] * ip * h;
#pragma unroll
  for (int k = 0; k < 6; ++k) o[4 + k] = (A.v[kAM2 + k] * ip + (k == 0 || k == 3 || k == 5 ? m2c : 0.0)) * h2;
#pragma unroll
  for (int i = 0; i < 3; ++i) o[10 + i] = A.v[kAG0 + i] * ip * ih;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) o[13 + 3 * i + j] = A.v[kAG1 + 3 * i + j] * ip + (i == j ? M0 : 0.0);
#pragma unroll
  for (int k = 0; k < 6; ++k) o[22 + k] = A.v[kAH + k] * ip * ih2;
}

// rows without faces in their support: whole-support constants inside, zeros outside, NaN for invalid rows.  Each
// thread builds its row in shared memory (stride 29 doubles against bank conflicts) and the block writes its
// contiguous slab of 128 x 28 outputs coalesced.
constexpr int kRowStride = 29;

template <class M>
__global__ void __launch_bounds__(kMeshThreads) k_mesh_rows(const double* __restrict__ sup, int64_t n,
                                                           const int32_t* __restrict__ ind, double* __restrict__ out) {
  __shared__ double s_rows[kMeshThreads * kRowStride];
  const int64_t row0 = (int64_t)blockIdx.x * kMeshThreads;
  const int64_t row = row0 + threadIdx.x;
  double* const mine = s_rows + threadIdx.x * kRowStride;
  if (row < n) {
    if (ind[row] < 0) {
      for (int k = 0; k < 28; ++k) mine[k] = __longlong_as_double(0x7ff8000000000000LL);
    } else {
      Acc28 A;
      acc_zero(A);
      write_row<M>(mine, 0, A, (double)ind[row], sup[row]);
    }
  }
  __syncthreads();
  const int rows = (int)min((int64_t)kMeshThreads, n - row0);
  for (int k = threadIdx.x; k < rows * 28; k += kMeshThreads)
    out[row0 * 28 + k] = s_rows[(k / 28) * kRowStride + k % 28];
}

// one warp per work row; warps take rows from a counter (rows differ in their number of faces), and the row's
// result does not depend on which warp computes it
// 4 resident CTAs per SM (at most 128 registers a thread): with the divided-difference coefficients formed once per
// face the c3 leg measured 8.14 ms on B200 against 8.26 ms with 3 CTAs (before that change 3 CTAs were best: 9.0 ms
// against 9.9 ms with 2 and 10.2 ms with 4)
#ifndef WSB_MESH_MIN_BLOCKS
#define WSB_MESH_MIN_BLOCKS 4
#endif
template <class M>
__global__ void __launch_bounds__(kMeshThreads, WSB_MESH_MIN_BLOCKS) k_mesh_eval(MeshView Mv, const double* __restrict__ pos,
                                                           const double* __restrict__ sup,
                                                           const int32_t* __restrict__ ind,
                                                           const int32_t* __restrict__ work,
                                                           const int32_t* __restrict__ nwork,
                                                           int32_t* __restrict__ grab, double* __restrict__ out) {
  __shared__ PanelList pl[kMeshThreads / 32][3];
  __shared__ EdgeGeo eg[kMeshThreads / 32][3];
  __shared__ double fb[kMeshThreads / 32][6 * kMeshDD];
  __shared__ double acc[kMeshThreads / 32][28];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const AccSlot aslot = acc_slot(lane);                  // the accumulator this lane assembles
  const int nw = *nwork;
  for (int it = 0; it < (1 << 30); ++it) {
    int slot = 0;
    if (lane == 0) slot = atomicAdd(grab, 1);
    slot = __shfl_sync(0xffffffffu, slot, 0);
    if (slot >= nw) break;
    const int64_t row = work[slot];
    const double q[3] = {pos[3 * row], pos[3 * row + 1], pos[3 * row + 2]};
    const double h = sup[row], ih = 1.0 / h;
    double mine = 0.0;                                   // accumulator `lane` of the row (lanes < 28)
    for_candidates_warp(Mv, q, h, lane, [&](int f) {
      face_contrib_warp<M>(Mv, f, q, ih, pl[wib], eg[wib], fb[wib], lane, aslot, mine);
    });
    if (lane < 28) acc[wib][lane] = mine;
    __syncwarp();
    if (lane == 0) {
      Acc28 A;
#pragma unroll
      for (int i = 0; i < 28; ++i) A.v[i] = acc[wib][i];
      write_row<M>(out, row, A, (double)ind[row], h);
    }
    __syncwarp();
  }
}

__global__ void k_mesh_inside_only(MeshView M, const double* __restrict__ pos, int64_t n, int32_t* __restrict__ ind) {
  const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  ind[row] = mesh_inside(M, pos[3 * row], pos[3 * row + 1], pos[3 * row + 2]);
}

template <typename T>
int upload_vec(T** dst, const std::vector<T>& src) {
  const size_t bytes = std::max<size_t>(src.size(), 1) * sizeof(T);
  WSB_CUDA(cudaMalloc((void**)dst, bytes));
  if (!src.empty()) WSB_CUDA(cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
  return WSB_OK;
}

void free_mesh(Mesh* m) {
  void* ptrs[] = {m->fdata, m->fcell, m->fvid, m->cstart, m->citems, m->colstart, m->colitems, m->cflag};
  for (void* p : ptrs)
    if (p) cudaFree(p);
}

inline size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

template <class M>
int launch_mesh(const Mesh* m, const double* pos, const double* sup, int64_t n, double* out, int32_t* ind,
                int32_t* work, int32_t* nwork, int32_t* near, cudaStream_t st) {
  const MeshView v = view_of(m);
  const unsigned grid = (unsigned)((n + kMeshThreads - 1) / kMeshThreads);
  WSB_CUDA(cudaMemsetAsync(nwork, 0, 3 * sizeof(int32_t), st));      // work rows, grab counter, listed rows
  k_mesh_rowinfo<<<grid, kMeshThreads, 0, st>>>(v, pos, sup, n, ind, near, nwork + 2);
  WSB_CUDA(cudaGetLastError());
  const unsigned grid_near = (unsigned)std::min<int64_t>((n + kMeshThreads / 32 - 1) / (kMeshThreads / 32), 8192);
  k_mesh_rownear<<<grid_near, kMeshThreads, 0, st>>>(v, pos, sup, near, nwork + 2, ind, work, nwork);
  WSB_CUDA(cudaGetLastError());
  k_mesh_rows<M><<<grid, kMeshThreads, 0, st>>>(sup, n, ind, out);
  WSB_CUDA(cudaGetLastError());
  // enough warps to fill the GPU; each loops over rows taken from the counter
  const int64_t warps = std::min<int64_t>(n, (int64_t)148 * 64);
  const unsigned egrid = (unsigned)((warps * 32 + kMeshThreads - 1) / kMeshThreads);
  k_mesh_eval<M><<<egrid, kMeshThreads, 0, st>>>(v, pos, sup, ind, work, nwork, nwork + 1, out);
  WSB_CUDA(cudaGetLastError());
  return WSB_OK;
}

}  // namespace
}  // namespace wsb

using namespace wsb;

struct wsb_mesh : public Mesh {};

extern "C" int wsb_mesh_create(const double* verts, int64_t n_verts, const int32_t* faces, int64_t n_faces,
                               double support_max, int device, wsb_mesh** out) {
  if (!out) return fail(WSB_ERR_ARG, "wsb_mesh_create: NULL handle pointer");
  *out = nullptr;
  if (!verts || !faces || n_verts < 3 || n_faces < 4)
    return fail(WSB_ERR_ARG, "wsb_mesh_create: a closed surface needs >= 3 vertices and >= 4 faces");
  if (n_faces > (int64_t)(INT32_MAX / 8)) return fail(WSB_ERR_SIZE, "wsb_mesh_create: too many faces");
  if (!(support_max > 0.0) || !std::isfinite(support_max))
    return fail(WSB_ERR_ARG, "wsb_mesh_create: support_max must be positive and finite");
  for (int64_t i = 0; i < 3 * n_verts; ++i)
    if (!std::isfinite(verts[i])) return fail(WSB_ERR_ARG, "wsb_mesh_create: non-finite vertex");
  // watertight, consistently oriented 2-manifold: every undirected edge twice, once in each direction
  std::map<std::pair<int32_t, int32_t>, int> dir;
  for (int64_t f = 0; f < n_faces; ++f) {
    const int32_t* v = faces + 3 * f;
    for (int k = 0; k < 3; ++k)
      if (v[k] < 0 || v[k] >= n_verts) return fail(WSB_ERR_ARG, "wsb_mesh_create: face index out of range");
    if (v[0] == v[1] || v[1] == v[2] || v[0] == v[2]) return fail(WSB_ERR_ARG, "wsb_mesh_create: repeated vertex");
    for (int k = 0; k < 3; ++k) {
      const int32_t a = v[k], b = v[(k + 1) % 3];
      const auto key = std::make_pair(std::min(a, b), std::max(a, b));
      const int bit = a < b ? 1 : 2;
      int& d = dir[key];
      if (d & bit) return fail(WSB_ERR_ARG, "wsb_mesh_create: surface must be watertight and consistently oriented");
      d |= bit;
    }
  }
  for (const auto& kv : dir)
    if (kv.second != 3) return fail(WSB_ERR_ARG, "wsb_mesh_create: surface must be watertight and consistently oriented");
  // face records, box, signed volume (relative to the first vertex: outward normals give a positive volume)
  double vol6 = 0.0;
  const double* o = verts;
  std::vector<double> hf((size_t)n_faces * kFaceDoubles);
  std::vector<int32_t> hvid((size_t)n_faces * 3);
  double blo[3] = {INFINITY, INFINITY, INFINITY}, bhi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t f = 0; f < n_faces; ++f) {
    const int32_t* v = faces + 3 * f;
    double P[3][3];
    for (int i = 0; i < 3; ++i)
      for (int k = 0; k < 3; ++k) P[i][k] = verts[3 * v[i] + k];
    const double a[3] = {P[0][0] - o[0], P[0][1] - o[1], P[0][2] - o[2]};
    const double b[3] = {P[1][0] - o[0], P[1][1] - o[1], P[1][2] - o[2]};
    const double c[3] = {P[2][0] - o[0], P[2][1] - o[1], P[2][2] - o[2]};
    vol6 += a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) + a[2] * (b[0] * c[1] - b[1] * c[0]);
    double* F = hf.data() + f * kFaceDoubles;
    for (int i = 0; i < 3; ++i)
      for (int k = 0; k < 3; ++k) F[kFV + 3 * i + k] = P[i][k];
    const double e1[3] = {P[1][0] - P[0][0], P[1][1] - P[0][1], P[1][2] - P[0][2]};
    const double e2[3] = {P[2][0] - P[0][0], P[2][1] - P[0][1], P[2][2] - P[0][2]};
    const double N[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    const double nl = std::sqrt(N[0] * N[0] + N[1] * N[1] + N[2] * N[2]);
    if (!(nl > 0.0)) return fail(WSB_ERR_ARG, "wsb_mesh_create: degenerate (zero-area) face");
    for (int k = 0; k < 3; ++k) F[kFN + k] = N[k] / nl;
    for (int e = 0; e < 3; ++e) {
      const double* A = P[e];
      const double* B = P[(e + 1) % 3];
      double t[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]};
      const double len = std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
      for (int k = 0; k < 3; ++k) t[k] /= len;
      const double* n = F + kFN;
      const double mu[3] = {t[1] * n[2] - t[2] * n[1], t[2] * n[0] - t[0] * n[2], t[0] * n[1] - t[1] * n[0]};
      for (int k = 0; k < 3; ++k) {
        F[kFT + 3 * e + k] = t[k];
        F[kFMU + 3 * e + k] = mu[k];
      }
      F[kFLEN + e] = len;
    }
    for (int k = 0; k < 3; ++k) {
      F[kFLO + k] = std::min(P[0][k], std::min(P[1][k], P[2][k]));
      F[kFHI + k] = std::max(P[0][k], std::max(P[1][k], P[2][k]));
      blo[k] = std::min(blo[k], F[kFLO + k]);
      bhi[k] = std::max(bhi[k], F[kFHI + k]);
      hvid[3 * f + k] = v[k];
    }
  }
  if (!(vol6 > 0.0)) return fail(WSB_ERR_ARG, "wsb_mesh_create: surface must have positive signed volume");
  // cell grid over the box grown by one cell; the cell is support_max, enlarged if the grid would pass 2^26 cells
  double cell = support_max;
  int64_t nx = 0, ny = 0, nz = 0;
  double lo[3] = {0, 0, 0};
  for (int tries = 0; tries < 64; ++tries) {
    for (int k = 0; k < 3; ++k) lo[k] = blo[k] - cell;
    nx = (int64_t)std::floor((bhi[0] + cell - lo[0]) / cell) + 1;
    ny = (int64_t)std::floor((bhi[1] + cell - lo[1]) / cell) + 1;
    nz = (int64_t)std::floor((bhi[2] + cell - lo[2]) / cell) + 1;
    if (nx * ny * nz <= ((int64_t)1 << 26)) break;
    cell *= 1.5;
  }
  const int64_t n3[3] = {nx, ny, nz};
  auto cidx = [&](double x, int k) {
    const int64_t i = (int64_t)std::floor((x - lo[k]) / cell);
    return std::min<int64_t>(std::max<int64_t>(i, 0), n3[k] - 1);
  };
  const int64_t ncell = nx * ny * nz, ncol = nx * ny;
  std::vector<int64_t> cnt(ncell + 1, 0), ccnt(ncol + 1, 0);
  std::vector<int32_t> fcell((size_t)n_faces * 3);
  std::vector<int64_t> range((size_t)n_faces * 6);
  for (int64_t f = 0; f < n_faces; ++f) {
    const double* F = hf.data() + f * kFaceDoubles;
    for (int k = 0; k < 3; ++k) {
      range[6 * f + 2 * k] = cidx(F[kFLO + k], k);
      range[6 * f + 2 * k + 1] = cidx(F[kFHI + k], k);
      fcell[3 * f + k] = (int32_t)range[6 * f + 2 * k];
    }
    for (int64_t kz = range[6 * f + 4]; kz <= range[6 * f + 5]; ++kz)
      for (int64_t jy = range[6 * f + 2]; jy <= range[6 * f + 3]; ++jy)
        for (int64_t ix = range[6 * f]; ix <= range[6 * f + 1]; ++ix) ++cnt[(kz * ny + jy) * nx + ix + 1];
    for (int64_t jy = range[6 * f + 2]; jy <= range[6 * f + 3]; ++jy)
      for (int64_t ix = range[6 * f]; ix <= range[6 * f + 1]; ++ix) ++ccnt[jy * nx + ix + 1];
  }
  for (int64_t c = 0; c < ncell; ++c) cnt[c + 1] += cnt[c];
  for (int64_t c = 0; c < ncol; ++c) ccnt[c + 1] += ccnt[c];
  if (cnt[ncell] > INT32_MAX || ccnt[ncol] > INT32_MAX)
    return fail(WSB_ERR_SIZE, "wsb_mesh_create: cell lists exceed 2^31 items");
  std::vector<int32_t> items((size_t)cnt[ncell]), citems((size_t)ccnt[ncol]);
  std::vector<int32_t> start(cnt.begin(), cnt.end()), cstart(ccnt.begin(), ccnt.end());
  {
    std::vector<int64_t> cur(cnt.begin(), cnt.end() - 1), ccur(ccnt.begin(), ccnt.end() - 1);
    for (int64_t f = 0; f < n_faces; ++f) {
      for (int64_t kz = range[6 * f + 4]; kz <= range[6 * f + 5]; ++kz)
        for (int64_t jy = range[6 * f + 2]; jy <= range[6 * f + 3]; ++jy)
          for (int64_t ix = range[6 * f]; ix <= range[6 * f + 1]; ++ix)
            items[cur[(kz * ny + jy) * nx + ix]++] = (int32_t)f;
      for (int64_t jy = range[6 * f + 2]; jy <= range[6 * f + 3]; ++jy)
        for (int64_t ix = range[6 * f]; ix <= range[6 * f + 1]; ++ix) citems[ccur[jy * nx + ix]++] = (int32_t)f;
    }
  }
  WSB_CUDA(cudaSetDevice(device));
  Mesh* m = new wsb_mesh();
  m->device = device;
  m->n_verts = n_verts;
  m->n_faces = n_faces;
  m->support_max = support_max;
  for (int k = 0; k < 3; ++k) m->lo[k] = lo[k];
  m->cell = cell;
  m->nx = (int32_t)nx;
  m->ny = (int32_t)ny;
  m->nz = (int32_t)nz;
  m->n_items = (int64_t)items.size();
  m->n_col_items = (int64_t)citems.size();
  int rc;
  if ((rc = upload_vec(&m->fdata, hf)) || (rc = upload_vec(&m->fcell, fcell)) || (rc = upload_vec(&m->fvid, hvid)) ||
      (rc = upload_vec(&m->cstart, start)) || (rc = upload_vec(&m->citems, items)) ||
      (rc = upload_vec(&m->colstart, cstart)) || (rc = upload_vec(&m->colitems, citems)) ||
      (rc = upload_vec(&m->cflag, std::vector<uint8_t>((size_t)m->nx * m->ny * m->nz, 0)))) {
    free_mesh(m);
    delete m;
    return rc;
  }
  const int64_t ncells = (int64_t)m->nx * m->ny * m->nz;
  k_mesh_cellflags<<<(unsigned)((ncells + 255) / 256), 256>>>(view_of(m), m->cflag);
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    free_mesh(m);
    delete m;
    return cuda_fail(e, "wsb_mesh_create: cell flags");
  }
  *out = static_cast<wsb_mesh*>(m);
  return WSB_OK;
}

extern "C" int wsb_mesh_destroy(wsb_mesh* m) {
  if (!m) return WSB_OK;
  cudaSetDevice(m->device);
  free_mesh(m);
  delete m;
  return WSB_OK;
}

extern "C" size_t wsb_mesh_workspace_size(const wsb_mesh* m, int64_t n) {
  if (!m || n < 0) return 0;
  return al256(sizeof(int32_t) * (size_t)std::max<int64_t>(n, 1)) * 3 + 256;
}

extern "C" int wsb_mesh_inside(const wsb_mesh* m, const double* pos, int64_t n, int32_t* inside, void* stream) {
  if (!m) return fail(WSB_ERR_ARG, "wsb_mesh_inside: NULL mesh");
  if (n < 0) return fail(WSB_ERR_ARG, "wsb_mesh_inside: negative size");
  if (n == 0) return WSB_OK;
  if (!pos || !inside) return fail(WSB_ERR_ARG, "wsb_mesh_inside: NULL array");
  WSB_CUDA(cudaSetDevice(m->device));
  k_mesh_inside_only<<<(unsigned)((n + kMeshThreads - 1) / kMeshThreads), kMeshThreads, 0, (cudaStream_t)stream>>>(
      view_of(m), pos, n, inside);
  WSB_CUDA(cudaGetLastError());
  return WSB_OK;
}

extern "C" int wsb_mesh_channels(const wsb_mesh* m, int kernel, const double* pos, const double* sup, int64_t n,
                                 double* out, int32_t* inside, void* workspace, size_t workspace_bytes, void* stream) {
  if (!m) return fail(WSB_ERR_ARG, "wsb_mesh_channels: NULL mesh");
  if (n < 0) return fail(WSB_ERR_ARG, "wsb_mesh_channels: negative size");
  if (kernel < 0 || kernel > WSB_KERNEL_W6)
    return fail(WSB_ERR_UNSUPPORTED, "wsb_mesh_channels: closed surfaces serve cubic, w2, w4, w6");
  if (n == 0) return WSB_OK;
  if (!pos || !sup || !out || !workspace) return fail(WSB_ERR_ARG, "wsb_mesh_channels: NULL array");
  if (n > (int64_t)INT32_MAX / 8) return fail(WSB_ERR_SIZE, "wsb_mesh_channels: more than 2^28 queries");
  if (workspace_bytes < wsb_mesh_workspace_size(m, n))
    return fail(WSB_ERR_SIZE, "wsb_mesh_channels: workspace smaller than wsb_mesh_workspace_size");
  WSB_CUDA(cudaSetDevice(m->device));
  char* base = (char*)workspace;
  const size_t s = al256(sizeof(int32_t) * (size_t)n);
  int32_t* work = (int32_t*)base;
  int32_t* ind = inside ? inside : (int32_t*)(base + s);
  int32_t* nwork = (int32_t*)(base + 2 * s);     // [3]: work rows, grab counter, listed rows
  int32_t* near = (int32_t*)(base + 2 * s + 256);
  cudaStream_t st = (cudaStream_t)stream;
  switch (kernel) {
    case WSB_KERNEL_CUBIC: return launch_mesh<Mesh_cubic>(m, pos, sup, n, out, ind, work, nwork, near, st);
    case WSB_KERNEL_W2: return launch_mesh<Mesh_w2>(m, pos, sup, n, out, ind, work, nwork, near, st);
    case WSB_KERNEL_W4: return launch_mesh<Mesh_w4>(m, pos, sup, n, out, ind, work, nwork, near, st);
    default: return launch_mesh<Mesh_w6>(m, pos, sup, n, out, ind, work, nwork, near, st);
  }
}
