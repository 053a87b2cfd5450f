// Static structures of a closed surface (SurfaceRep): edge cell list by integer counting sort, y bins, per-cell
// indicator cache; error plumbing of the C ABI.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace wsb {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* where) {
  g_last_error = std::string(where) + ": " + cudaGetErrorString(e);
  return WSB_ERR_CUDA;
}

SurfView view_of(const Surface* s) {
  SurfView v;
  v.verts = s->verts;
  v.edges = s->edges;
  v.n_edges = s->n_edges;
  v.cstart = s->cstart;
  v.crec = s->crec;
  v.citems = s->citems;
  v.cind = s->cind;
  v.cok = s->cok;
  v.cempty = s->cempty;
  v.ccompact = s->ccompact;
  v.nne = s->n_nonempty;
  v.bstart = s->bstart;
  v.bitems = s->bitems;
  v.brec = s->brec;
  v.erec = s->erec;
  v.nx = s->nx;
  v.ny = s->ny;
  v.nb = s->nb;
  v.K = s->K;
  v.lo_x = s->lo_x;
  v.lo_y = s->lo_y;
  v.cell = s->cell;
  v.y0 = s->y0;
  v.dy = s->dy;
  v.background = (double)s->background;
  return v;
}

// winding + background at every cell centre (h = 1: no normalisation) by the ray cast of scene.py:350-372.  For an
// edge-free cell this is the indicator of every point of the cell (scene.py:281-295).  For a cell with edges it is
// the reference point of the local crossing count; cok marks whether every orientation the ray cast tested was
// certain (clear of rounding), i.e. whether the value is the exact winding number.
__global__ void k_cell_indicator(SurfView S, int64_t ncells) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  const int64_t cx = c / S.ny, cy = c % S.ny;
  const double px = __dadd_rn(S.lo_x, __dmul_rn(__dadd_rn((double)cx, 0.5), S.cell));
  const double py = __dadd_rn(S.lo_y, __dmul_rn(__dadd_rn((double)cy, 0.5), S.cell));
  const double iyd = floor(__ddiv_rn(__dsub_rn(py, S.y0), S.dy));
  double w = 0.0;
  bool certain = true;
  if (iyd >= 0.0 && iyd <= (double)S.nb) {
    int iy = (int)iyd;
    if (iy > S.nb - 1) iy = S.nb - 1;
    for (int i = S.bstart[iy]; i < S.bstart[iy + 1]; ++i) {
      const double4 r = S.brec[i];
      const double ax = r.x - px, ay = r.y - py, bx = r.z - px, by = r.w - py;
      const double cr = cross2_rn(ax, ay, bx, by);
      if (!(fabs(cr) > 1e-10 * (fabs(ax * by) + fabs(ay * bx)))) certain = false;
      if (r.y <= py && py < r.w && cr > 0.0) w += 1.0;
      if (r.w <= py && py < r.y && cr < 0.0) w -= 1.0;
    }
  }
  const_cast<double*>(S.cind)[c] = w + S.background;
  const_cast<int32_t*>(S.cok)[c] = (certain || S.cempty[c]) ? 1 : 0;
}

}  // namespace wsb

using namespace wsb;

struct wsb_surface : public Surface {};

extern "C" const char* wsb_last_error(void) { return g_last_error.c_str(); }

extern "C" int wsb_version(void) { return 100; }

template <typename T>
static int upload(T** dst, const std::vector<T>& src) {
  size_t bytes = std::max<size_t>(src.size(), 1) * sizeof(T);
  WSB_CUDA(cudaMalloc((void**)dst, bytes));
  if (!src.empty()) WSB_CUDA(cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
  return WSB_OK;
}

static void free_surface(Surface* s) {
  void* ptrs[] = {s->verts, s->edges, s->cstart, s->citems, s->crec, s->cind, s->cempty, s->ccompact, s->bstart, s->bitems, s->erec,
                  s->brec, s->cok};
  for (void* p : ptrs)
    if (p) cudaFree(p);
}

extern "C" int wsb_surface_create(const double* verts, int64_t n_verts, const int32_t* edges, int64_t n_edges,
                                  int background, double support_max, int device, wsb_surface** out) {
  if (!out) return fail(WSB_ERR_ARG, "wsb_surface_create: out is NULL");
  *out = nullptr;
  if (!verts || !edges || n_verts < 2 || n_edges < 1)
    return fail(WSB_ERR_ARG, "wsb_surface_create: a surface needs vertices and edges");
  if (!(support_max > 0.0) || !std::isfinite(support_max))
    return fail(WSB_ERR_ARG, "wsb_surface_create: support_max must be a positive finite number");
  for (int64_t e = 0; e < 2 * n_edges; ++e)
    if (edges[e] < 0 || edges[e] >= n_verts) return fail(WSB_ERR_ARG, "wsb_surface_create: edge vertex index out of range");
  for (int64_t i = 0; i < 2 * n_verts; ++i)
    if (!std::isfinite(verts[i])) return fail(WSB_ERR_ARG, "wsb_surface_create: non-finite vertex coordinate");
  WSB_CUDA(cudaSetDevice(device));
  auto* s = new wsb_surface();
  s->device = device;
  s->n_verts = n_verts;
  s->n_edges = n_edges;
  s->background = background;
  s->support_max = support_max;
  // ---- edge boxes +- support_max and the grid (scene.py:100-119, 273-279)
  const double cell = support_max;
  std::vector<double> blo(2 * n_edges), bhi(2 * n_edges);
  double gmin[2] = {INFINITY, INFINITY}, gmax[2] = {-INFINITY, -INFINITY};
  double bb[4] = {INFINITY, INFINITY, -INFINITY, -INFINITY};
  for (int64_t i = 0; i < n_verts; ++i) {
    bb[0] = std::min(bb[0], verts[2 * i]);
    bb[1] = std::min(bb[1], verts[2 * i + 1]);
    bb[2] = std::max(bb[2], verts[2 * i]);
    bb[3] = std::max(bb[3], verts[2 * i + 1]);
  }
  for (int64_t e = 0; e < n_edges; ++e) {
    const double* a = verts + 2 * edges[2 * e];
    const double* b = verts + 2 * edges[2 * e + 1];
    for (int k = 0; k < 2; ++k) {
      blo[2 * e + k] = std::min(a[k], b[k]) - support_max;
      bhi[2 * e + k] = std::max(a[k], b[k]) + support_max;
      gmin[k] = std::min(gmin[k], blo[2 * e + k]);
      gmax[k] = std::max(gmax[k], bhi[2 * e + k]);
    }
  }
  int64_t dims[2];
  for (int k = 0; k < 2; ++k) dims[k] = std::max<int64_t>((int64_t)std::ceil((gmax[k] - gmin[k]) / cell), 1);
  if (dims[0] * dims[1] > (int64_t)1 << 30) {
    delete s;
    return fail(WSB_ERR_SIZE, "wsb_surface_create: the edge cell grid exceeds 2^30 cells (support_max too small for the extent)");
  }
  const int64_t nx = dims[0], ny = dims[1], ncells = nx * ny;
  // counting sort of (cell, edge) items; within a cell by edge id (the stable argsort of the edge-major enumeration)
  std::vector<int64_t> i0(2 * n_edges), i1(2 * n_edges);
  std::vector<int32_t> counts(ncells + 1, 0);
  for (int64_t e = 0; e < n_edges; ++e) {
    for (int k = 0; k < 2; ++k) {
      i0[2 * e + k] = std::max<int64_t>((int64_t)std::floor((blo[2 * e + k] - gmin[k]) / cell), 0);
      i1[2 * e + k] = std::min<int64_t>((int64_t)std::floor((bhi[2 * e + k] - gmin[k]) / cell), dims[k] - 1);
    }
    for (int64_t cx = i0[2 * e]; cx <= i1[2 * e]; ++cx)
      for (int64_t cy = i0[2 * e + 1]; cy <= i1[2 * e + 1]; ++cy) counts[cx * ny + cy + 1]++;
  }
  std::vector<int32_t> start(ncells + 1, 0);
  int32_t K = 1;
  for (int64_t c = 0; c < ncells; ++c) {
    start[c + 1] = start[c] + counts[c + 1];
    K = std::max(K, counts[c + 1]);
  }
  const int64_t n_items = start[ncells];
  std::vector<int32_t> cursor(start.begin(), start.end() - 1), items(n_items);
  for (int64_t e = 0; e < n_edges; ++e)
    for (int64_t cx = i0[2 * e]; cx <= i1[2 * e]; ++cx)
      for (int64_t cy = i0[2 * e + 1]; cy <= i1[2 * e + 1]; ++cy) items[cursor[cx * ny + cy]++] = (int32_t)e;
  std::vector<double4> crec(n_items), erec(n_edges);
  for (int64_t e = 0; e < n_edges; ++e) {
    const double* a = verts + 2 * edges[2 * e];
    const double* b = verts + 2 * edges[2 * e + 1];
    erec[e] = make_double4(a[0], a[1], b[0], b[1]);
  }
  for (int64_t i = 0; i < n_items; ++i) crec[i] = erec[items[i]];
  std::vector<int32_t> cempty(ncells);
  for (int64_t c = 0; c < ncells; ++c) cempty[c] = (start[c + 1] == start[c]) ? 1 : 0;
  std::vector<int32_t> ccompact(ncells);
  int32_t nne = 0;
  for (int64_t c = 0; c < ncells; ++c) ccompact[c] = cempty[c] ? -1 : nne++;
  // ---- y bins (scene.py:297-314)
  const int32_t nb = std::max<int32_t>(1, (int32_t)std::sqrt((double)n_edges) * 2);
  double ylo_min = INFINITY, yhi_max = -INFINITY;
  std::vector<double> ylo(n_edges), yhi(n_edges);
  for (int64_t e = 0; e < n_edges; ++e) {
    ylo[e] = std::min(erec[e].y, erec[e].w);
    yhi[e] = std::max(erec[e].y, erec[e].w);
    ylo_min = std::min(ylo_min, ylo[e]);
    yhi_max = std::max(yhi_max, yhi[e]);
  }
  const double y0 = ylo_min;
  const double dy = std::max(yhi_max - y0, 1e-300) / nb;
  std::vector<int32_t> bcnt(nb + 1, 0), b0(n_edges), b1(n_edges);
  for (int64_t e = 0; e < n_edges; ++e) {
    b0[e] = (int32_t)std::min<int64_t>(std::max<int64_t>((int64_t)std::floor((ylo[e] - y0) / dy), 0), nb - 1);
    b1[e] = (int32_t)std::min<int64_t>(std::max<int64_t>((int64_t)std::floor((yhi[e] - y0) / dy), 0), nb - 1);
    for (int32_t b = b0[e]; b <= b1[e]; ++b) bcnt[b + 1]++;
  }
  std::vector<int32_t> bstart(nb + 1, 0);
  for (int32_t b = 0; b < nb; ++b) bstart[b + 1] = bstart[b] + bcnt[b + 1];
  std::vector<int32_t> bcur(bstart.begin(), bstart.end() - 1), bitems(bstart[nb]);
  for (int64_t e = 0; e < n_edges; ++e)
    for (int32_t b = b0[e]; b <= b1[e]; ++b) bitems[bcur[b]++] = (int32_t)e;
  s->nx = (int32_t)nx;
  s->ny = (int32_t)ny;
  s->lo_x = gmin[0];
  s->lo_y = gmin[1];
  s->cell = cell;
  s->K = K;
  s->n_nonempty = nne;
  s->n_items = n_items;
  s->nb = nb;
  s->y0 = y0;
  s->dy = dy;
  s->n_bitems = (int64_t)bitems.size();
  std::memcpy(s->bbox, bb, sizeof(bb));
  std::vector<double4> brec(bitems.size());
  for (size_t i = 0; i < bitems.size(); ++i) brec[i] = erec[bitems[i]];
  std::vector<double> hv(verts, verts + 2 * n_verts);
  std::vector<int32_t> he(edges, edges + 2 * n_edges);
  std::vector<double> cind(ncells, 0.0);
  int rc = WSB_OK;
  if ((rc = upload(&s->verts, hv)) || (rc = upload(&s->edges, he)) || (rc = upload(&s->cstart, start)) ||
      (rc = upload(&s->citems, items)) || (rc = upload(&s->crec, crec)) || (rc = upload(&s->cind, cind)) ||
      (rc = upload(&s->cempty, cempty)) || (rc = upload(&s->ccompact, ccompact)) || (rc = upload(&s->bstart, bstart)) || (rc = upload(&s->bitems, bitems)) ||
      (rc = upload(&s->erec, erec)) || (rc = upload(&s->brec, brec)) ||
      (rc = upload(&s->cok, std::vector<int32_t>(ncells, 0)))) {
    free_surface(s);
    delete s;
    return rc;
  }
  SurfView v = view_of(s);
  k_cell_indicator<<<(unsigned)((ncells + 255) / 256), 256>>>(v, ncells);
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    free_surface(s);
    delete s;
    return cuda_fail(e, "wsb_surface_create: cell indicator");
  }
  *out = s;
  return WSB_OK;
}

extern "C" int wsb_surface_destroy(wsb_surface* s) {
  if (!s) return WSB_OK;
  cudaSetDevice(s->device);
  free_surface(s);
  delete s;
  return WSB_OK;
}

extern "C" int wsb_surface_info_get(const wsb_surface* s, wsb_surface_info* o) {
  if (!s || !o) return fail(WSB_ERR_ARG, "wsb_surface_info_get: NULL argument");
  o->n_verts = s->n_verts;
  o->n_edges = s->n_edges;
  o->nx = s->nx;
  o->ny = s->ny;
  o->lo_x = s->lo_x;
  o->lo_y = s->lo_y;
  o->cell = s->cell;
  o->K = s->K;
  o->n_items = s->n_items;
  o->n_bins = s->nb;
  o->bbox_lo_x = s->bbox[0];
  o->bbox_lo_y = s->bbox[1];
  o->bbox_hi_x = s->bbox[2];
  o->bbox_hi_y = s->bbox[3];
  o->background = s->background;
  o->support_max = s->support_max;
  return WSB_OK;
}

extern "C" int wsb_surface_cells(const wsb_surface* s, int32_t* start_host, int32_t* items_host) {
  if (!s || !start_host || !items_host) return fail(WSB_ERR_ARG, "wsb_surface_cells: NULL argument");
  WSB_CUDA(cudaSetDevice(s->device));
  WSB_CUDA(cudaMemcpy(start_host, s->cstart, sizeof(int32_t) * ((int64_t)s->nx * s->ny + 1), cudaMemcpyDeviceToHost));
  if (s->n_items) WSB_CUDA(cudaMemcpy(items_host, s->citems, sizeof(int32_t) * s->n_items, cudaMemcpyDeviceToHost));
  return WSB_OK;
}
