/*
 * wsb.h -- C ABI of the B200 boundary-integral library (libwsb.so).
 *
 * Exact semi-analytic SPH boundary integrals of 2-D polygonal walls: the kernel
 * mass lambda and the twelve surface moments (m1, G, g1 = int y (x) grad W,
 * m2) at fluid particles, their adjoint, signed distance and body kinematics.
 * Plain pointers and sizes only; every array argument is DEVICE memory unless
 * its comment says "host".  Streams are cudaStream_t passed as void*.
 * Every entry point returns WSB_OK (0) or a negative WSB_ERR_* code; the text
 * of the last error of the calling thread is wsb_last_error().
 *
 * Each entry point names the reference interface (wi-re/warpSPHBoundaries,
 * path:line inside that project) it replaces.
 */
#ifndef WSB_H
#define WSB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  WSB_OK = 0,
  WSB_ERR_ARG = -1,          /* invalid argument (the Python facade raises ValueError) */
  WSB_ERR_CUDA = -2,         /* a CUDA runtime call failed */
  WSB_ERR_UNSUPPORTED = -3,  /* unsupported kernel / mode (NotImplementedError) */
  WSB_ERR_SIZE = -4,         /* a buffer or workspace is too small */
  WSB_ERR_DEVICE = -5        /* a device-side check failed (status word set) */
};

/* kernel ids (warpsphboundaries_b200/kernels.py: KERNEL_IDS) */
enum {
  WSB_KERNEL_CUBIC = 0, WSB_KERNEL_W2 = 1, WSB_KERNEL_W4 = 2, WSB_KERNEL_W6 = 3,
  WSB_KERNEL_QUARTIC = 4, WSB_KERNEL_QUINTIC = 5, WSB_KERNEL_POLY6 = 6,
  /* the wall-operator kernels of the non-lean provider layout: cone (1 - q), whose G channels are the free-surface
   * cover vector (edge/kernels.py:179-181, scene/cover.py); lw2 / lw4, W'/r of the Wendland C2 / C4 kernels, whose
   * 2 lam - tr Cov is the wall Laplacian (scene/viscosity.py:48-61, scene/fused.py:11) */
  WSB_KERNEL_CONE = 7, WSB_KERNEL_LW2 = 8, WSB_KERNEL_LW4 = 9,
  /* the tensile group of the delta+ layout: W^5 of Wendland C2 / C4 (scene/tensile.py, edge/kernels.py:214-232),
   * polynomials of degree 25 / 40 integrated along each chord by graded Gauss-Legendre panels.  Fused aggregate only
   * (wsb_aggregate, _evaluate, _groups, _noalloc); only the G output is defined (the others are written as NaN); no
   * adjoint, no plain route */
  WSB_KERNEL_W2P5 = 10, WSB_KERNEL_W4P5 = 11
};

/* arithmetic of the fused aggregate */
enum {
  WSB_PREC_FP64 = 0,   /* every step in float64 */
  WSB_PREC_MIXED = 1,  /* float32 special functions where the per-pair error bound allows, float64 guards and sums */
  WSB_PREC_FP32 = 2    /* the float route: 2-D chord sums in float32 (Chebyshev profiles, Gauss-Legendre on panels graded
                          from the foot point), chord clip, edge frame and row sums in float64; 3-D spheres: every step
                          in float32 */
};

/* solid kinds of wsb_radial_channels */
enum { WSB_RADIAL_PLANE = 0, WSB_RADIAL_SPHERE = 1 };

/* output selection bits of wsb_aggregate */
enum { WSB_OUT_LAM = 1, WSB_OUT_G = 2, WSB_OUT_COV = 4, WSB_OUT_M1 = 8, WSB_OUT_M2 = 16, WSB_OUT_ALL = 31,
       WSB_OUT_ASSIGN = 32 /* overwrite the outputs (rows that are not candidates get zeros) instead of adding */ };

typedef struct wsb_surface wsb_surface;

typedef struct {
  int64_t n_verts, n_edges;
  int32_t nx, ny;            /* edge cell grid (cell = support_max) */
  double lo_x, lo_y, cell;
  int32_t K;                 /* largest number of edges in one cell: slots per row of the fixed topology */
  int64_t n_items;           /* entries of the cell list */
  int32_t n_bins;            /* y bins of the ray-cast indicator */
  double bbox_lo_x, bbox_lo_y, bbox_hi_x, bbox_hi_y;   /* vertex bounding box (body frame) */
  int background;
  double support_max;
} wsb_surface_info;

const char* wsb_last_error(void);
int wsb_version(void);

/* Static structures of one closed surface (loops counter-clockwise around the solid) for supports <= support_max:
 * edge cell list, per-cell indicator cache, y bins.  verts [n_verts*2] and edges [n_edges*2] are HOST arrays.
 * Replaces SurfaceRep.__init__/_celllist/_cell_indicator/_ybins (src/warpSPHBoundaries/scene/scene.py:222-327)
 * and fixedadj._static (src/warpSPHBoundaries/scene/fixedadj.py:150-165). */
int wsb_surface_create(const double* verts, int64_t n_verts, const int32_t* edges, int64_t n_edges,
                       int background, double support_max, int device, wsb_surface** out);
int wsb_surface_destroy(wsb_surface* s);
int wsb_surface_info_get(const wsb_surface* s, wsb_surface_info* out);
/* host copies of the cell list (start [nx*ny+1], items [n_items]) for tests */
int wsb_surface_cells(const wsb_surface* s, int32_t* start_host, int32_t* items_host);

/* Fixed-capacity slots and indicator of rows lpos [n*2] (body frame), supports lsup [n], valid [n] (int32, may be NULL):
 * slots [n*K] int32 (-1 = empty), edges in cell-list order; ind [n] float64 (winding number + background, 0 for
 * invalid rows).  Replaces fixedadj.fixed_topology (src/warpSPHBoundaries/scene/fixedadj.py:67-147, 168-182). */
int wsb_fixed_topology(const wsb_surface* s, const double* lpos, const double* lsup, const int32_t* valid, int64_t n,
                       int32_t* slots, double* ind, void* stream);

/* Plain FP64 route, stage 1: the twelve edge channels of every slot, c [n*K*12] (units of h): one thread per slot
 * interpreting the exact truncated term plan.  Replaces warpbc.edge_channels + second_channels
 * (src/warpSPHBoundaries/edge/warpbc.py:619-661, 919-991) on a fixed topology. */
int wsb_slot_channels_plain(const wsb_surface* s, int kernel, const double* lpos, const double* lsup,
                            const int32_t* slots, int64_t n, double* c, void* stream);

/* Plain FP64 route, stage 2: per row the slot channels in slot order + ind * plane channels, physical scaling,
 * rotation to the world frame by rot [4] = (c, -s, s, c) (device), ADDED into lam [n], G [n*2], cov [n*4], m1 [n*2],
 * m2 [n*4] (any of them may be NULL).  Replaces FusedWall.evaluate's _wall_contract_kernel and
 * _second_contract_kernel (src/warpSPHBoundaries/scene/fused.py:69-154, 612-659). */
int wsb_contract(const wsb_surface* s, int kernel, const int32_t* slots, const double* c, const double* ind,
                 const double* lsup, int64_t n, const double* rot, double* lam, double* G, double* cov, double* m1,
                 double* m2, void* stream);

/* Pair-list channels: for every (query, edge) pair k of qi [n_pairs], e [n_pairs] (int32, device) the twelve
 * edge-local channels c[12k .. 12k + 11] (units of h, the 1/pi applied; 0 lam, 1-2 m1, 3-4 G, 5-8 g1, 9-11 m20 m11
 * m02) of query row qi[k] (lpos [n_rows*2] body frame, lsup [n_rows]) against edge e[k] by the closed form; kernels
 * 0 .. 11 (10, 11: the tensile kernels, G channels only, the others NaN); precision WSB_PREC_FP64 or WSB_PREC_MIXED.
 * An index outside its array gives NaN channels and sets *status (device int32, zeroed by the caller) to 1.
 * Replaces warpbc.edge_channels + second_channels over a pair list (src/warpSPHBoundaries/edge/warpbc.py:919-991) as
 * SurfaceRep.moments calls them (src/warpSPHBoundaries/scene/scene.py:384-416). */
int wsb_pair_channels(const wsb_surface* s, int kernel, int precision, const int32_t* qi, const int32_t* e,
                      int64_t n_pairs, const double* lpos, const double* lsup, int64_t n_rows, double* c,
                      int32_t* status, void* stream);

/* Workspace bytes wsb_aggregate needs for n rows. */
size_t wsb_aggregate_workspace_size(const wsb_surface* s, int64_t n);
/* Optional staging bytes for n rows: a workspace of wsb_aggregate_workspace_size + wsb_aggregate_staging_size bytes
 * (given to prepare and to every evaluation of that preparation alike) lets the evaluation write each work row's
 * channel sums to the staging region and then every row's outputs in one coalesced pass, instead of storing the work
 * rows' outputs scattered by row index.  The results are the same bits either way.  No counterpart in the reference
 * (a layout choice of this implementation). */
size_t wsb_aggregate_staging_size(const wsb_surface* s, int64_t n);
/* Instrumentation: while set, every fused pair pass records `start` (a cudaEvent_t) on its stream right before its pair
 * kernel and `end` right after it, so a profiler or benchmark can time that kernel alone; NULL, NULL clears them.  The
 * events are the caller's.  No counterpart in the reference. */
int wsb_set_pair_events(void* start, void* end);

/* Fused route: body-frame coordinates (Pose.toLocal), the body broadphase (support circle against the body box
 * [obb_lo, obb_hi]; unbounded != 0 skips it), the fixed-capacity neighbour predicate, the twelve channels of every
 * neighbour pair and the per-row contraction in ONE pass over rows sorted by cell; outputs ADDED as wsb_contract.
 * pos [n*2] world, sup [n], allowed [n] int32 (may be NULL = all), pose [4] = (cx, cy, cos, sin) (device),
 * obb [4] = (lo_x, lo_y, hi_x, hi_y) (host).  status [1] (device, may be NULL) receives a device error code.
 * Replaces AnalyticBoundary.aggregate for one (body, SurfaceRep) (src/warpSPHBoundaries/scene/provider.py:89-110:
 * fixed_adjacency fixedadj.py:249-270, FusedWall fused.py:506-564 and evaluate fused.py:612-659). */
int wsb_aggregate(const wsb_surface* s, int kernel, int precision, const double* pos, const double* sup,
                  const int32_t* allowed, int64_t n, const double* pose, const double* obb, int unbounded,
                  int out_mask, double* lam, double* G, double* cov, double* m1, double* m2,
                  void* workspace, size_t workspace_bytes, int32_t* status, void* stream);

/* The two halves of wsb_aggregate, for callers that time or overlap them separately: _prepare forms the body-frame
 * positions, the broadphase and the cell-sorted row order in the workspace; _evaluate runs the fused channel pass on a
 * prepared workspace (any kernel / precision, repeatable for several kernels over one prepared position set). */
int wsb_aggregate_prepare(const wsb_surface* s, const double* pos, const double* sup, const int32_t* allowed, int64_t n,
                          const double* pose, const double* obb, int unbounded, void* workspace,
                          size_t workspace_bytes, void* stream);
int wsb_aggregate_evaluate(const wsb_surface* s, int kernel, int precision, const double* sup, int64_t n,
                           const double* pose, int out_mask, double* lam, double* G, double* cov, double* m1,
                           double* m2, const void* workspace, size_t workspace_bytes, void* stream);

/* Several kernel groups over one position set, as FusedWall evaluates its tuple of groups in one launch family
 * (src/warpSPHBoundaries/scene/fused.py:506-547; edge/warpfused.py:58-109 FusedPlan and :190 fused_channels).
 * kernels [n_groups] (host) lists the groups' kernel ids; lam, G, cov, m1, m2 are HOST arrays of n_groups device
 * pointers each (the array, or an entry, may be NULL when out_mask leaves that output out); group g is written as
 * wsb_aggregate_evaluate with kernels[g] would write it.  The first of the kernel sets {cubic, w2, w4, w6},
 * {w2, w4, w6}, {w2, cone, lw2}, {w4, cone, lw4}, {w2, cone}, {w4, cone} that the groups contain (each kernel once,
 * any order) is evaluated in one pass over the neighbour pairs, sharing each pair's chord, special functions and
 * monomial integrals between kernel blocks of equal support radius; every other group runs its own pass.
 * At most WSB_MAX_GROUPS groups.  _groups = _prepare + _evaluate_groups. */
enum { WSB_MAX_GROUPS = 8 };
int wsb_aggregate_evaluate_groups(const wsb_surface* s, int n_groups, const int32_t* kernels, int precision,
                                  const double* sup, int64_t n, const double* pose, int out_mask, double* const* lam,
                                  double* const* G, double* const* cov, double* const* m1, double* const* m2,
                                  const void* workspace, size_t workspace_bytes, void* stream);
int wsb_aggregate_groups(const wsb_surface* s, int n_groups, const int32_t* kernels, int precision, const double* pos,
                         const double* sup, const int32_t* allowed, int64_t n, const double* pose, const double* obb,
                         int unbounded, int out_mask, double* const* lam, double* const* G, double* const* cov,
                         double* const* m1, double* const* m2, void* workspace, size_t workspace_bytes,
                         void* stream);

/* Two detector inputs of the delta+ scheme on a workspace that wsb_aggregate_prepare filled for this surface, pose
 * and position set (they visit the same neighbour edges as the channel pass, |x - seg| < sup of the row; float64).
 *
 * wsb_cone_area ADDS, per row i, the area of (solid cap disk(x_i, sup_i) cap wedge(x_i, axis_i, half_angle)) into area[i]
 * and the full-disk area of the solid into area[n + i] (area [2n], units length^2; half_angle >= pi = the full disk).
 * axes [n*2] are world vectors (only their direction matters).  A row outside the broadphase of a surface whose solid
 * is the unbounded outside (background 1) adds the whole sector.  half_angle must be finite and >= 0 (WSB_ERR_ARG).
 * Replaces FusedWall.cone_area's polygon launch and its background term (src/warpSPHBoundaries/scene/fused.py:180-246
 * _cone_area_kernel, :799-835 cone_area); the per-edge closed form it evaluates locally is scene/cone_area.py:20-60.
 *
 * wsb_dir_extreme max-accumulates, per row i, into out[i] the largest |cos| between the world vector vecs[i] (vecs
 * [n*2]) and a direction from x_i to a point of the solid within sup_i: 1 where the line of the vector meets the solid
 * there (a row inside the solid: 1), 0 for a zero vector or no solid in support.  Replaces FusedWall.dir_extreme's
 * polygon launch and its background rule (fused.py:248-308 _dir_extreme_kernel, :741-797 dir_extreme). */
int wsb_cone_area(const wsb_surface* s, const double* sup, int64_t n, const double* pose, const double* axes,
                  double half_angle, double* area, const void* workspace, size_t workspace_bytes, void* stream);
int wsb_dir_extreme(const wsb_surface* s, int64_t n, const double* pose, const double* vecs, double* out,
                    const void* workspace, size_t workspace_bytes, void* stream);

/* wsb_aggregate without a caller workspace, for hosts that cannot allocate device memory for this library (their
 * allocator owns the GPU's memory, or their step loop may not call cudaMalloc / cudaFree, which synchronise the
 * device).  No counterpart in the reference: it exists for such C-ABI callers.  The scratch is a static 16 MiB device
 * array inside libwsb.so (per GPU, held until the library is unloaded); the call allocates nothing.  It serves about
 * 120 bytes per row plus 12 bytes per cell of the surface's grid, e.g. 131072 rows over a 256 x 256 grid; larger
 * requests fail with WSB_ERR_SIZE.  The first call on a device looks the scratch address up (make that first call
 * before any stream capture).  All calls share the one array: calls that overlap on the GPU (other streams, other
 * threads) race and must be serialised by the caller; each call clears the counters it needs. */
int wsb_aggregate_noalloc(const wsb_surface* s, int kernel, int precision, const double* pos, const double* sup,
                          const int32_t* allowed, int64_t n, const double* pose, const double* obb, int unbounded,
                          int out_mask, double* lam, double* G, double* cov, double* m1, double* m2, int32_t* status,
                          void* stream);

/* Adjoint of wsb_aggregate's lam, m1, m2 (the moments m_alpha, |alpha| <= 2) by recomputation: given world-frame
 * gradients g_lam [n], g_m1 [n*2], g_m2 [n*4] (any may be NULL), ADD dL/dpos into d_pos [n*2] (world) and dL/dvertex
 * into d_verts [n_verts*2] (body frame; may be NULL).  Replaces warp2d.TorchMoment's backward and np2d
 * moment_gradient / shape_gradient (src/warpSPHBoundaries/edge/warp2d.py:287-365, 482-500;
 * src/warpSPHBoundaries/edge/np2d.py:554-565, 626-652). */
int wsb_aggregate_backward(const wsb_surface* s, int kernel, const double* pos, const double* sup,
                           const int32_t* allowed, int64_t n, const double* pose, const double* obb, int unbounded,
                           const double* g_lam, const double* g_m1, const double* g_m2, double* d_pos,
                           double* d_verts, void* workspace, size_t workspace_bytes, void* stream);

/* Signed distance of body-frame points lpos [m*2] to the surface: d [m] (> 0 in the fluid), closest point cp [m*2],
 * unit normal n_loc [m*2] into the fluid, edge [m] int32.  norm_support > 0: the indicator uses that support
 * normalisation (the sync-free route), else none.  Replaces the SurfaceRep branch of Scene.signed_distance
 * (src/warpSPHBoundaries/scene/scene.py:1312-1350). */
int wsb_signed_distance(const wsb_surface* s, const double* lpos, int64_t m, double norm_support, double* d,
                        double* cp, double* n_loc, int32_t* edge, void* stream);

/* Rigid-body fields of B bodies at world points x [n*2]: body [b] = (cx, cy, cos, sin, vx, vy, omega, ax, ay, alpha)
 * (device [B*10]); writes rel, local, velocity, acceleration [B*n*2] (any may be NULL).  Replaces BodyKinematics
 * (src/warpSPHBoundaries/scene/scene.py:1155-1225) and Body.velocityAt / accelerationAt (scene.py:934-939, 1063-1067). */
int wsb_kinematics(const double* bodies, int32_t n_bodies, const double* x, int64_t n, double* rel, double* local,
                   double* velocity, double* acceleration, void* stream);

/* Solid half-space (kind WSB_RADIAL_PLANE) or solid sphere (WSB_RADIAL_SPHERE) in 3-D, one query per row: from the
 * signed outward distance distances [n] (sphere: |x - c| - R, >= -R), radii [n] (sphere only; NULL for a plane), unit
 * outward normals [n*3] and supports [n] (all device, float64), the nine axial invariants (lam, m1_axial, m2_tangent,
 * m2_axial, G_axial, g1_tangent, g1_axial, H_tangent, H_axial) in physical units into invariants [n*9] (may be NULL)
 * and the Cartesian channel of each request row (degree, i, j, order) of the host array requests [n_requests*4]
 * (n_requests <= 28; the 28-row baseline lists value moments |alpha| <= 2, first kernel-derivative moments |alpha| <= 1
 * and the symmetric kernel Hessian) into out [n*n_requests].  Kernels cubic, w2, w4, w6; precision WSB_PREC_FP64 or
 * WSB_PREC_FP32.  Rows with invalid input (support <= 0, non-finite values, sphere radius <= 0 or distance < -radius)
 * get NaN and status [n] = 1 (status may be NULL), others 0.  Replaces fluxbridge's RadialEvaluator batch, the native
 * element and select (src/warpSPHBoundaries/fluxbridge/radial.py:20-71, 200-215;
 * src/warpSPHBoundaries/fluxbridge/_radial_code.py:43-148). */
int wsb_radial_channels(int kind, int kernel, int precision, const double* distances, const double* radii,
                        const double* normals, const double* supports, int64_t n, const int32_t* requests,
                        int n_requests, double* out, double* invariants, int32_t* status, void* stream);

/* ---- conditioned single triangles (2-D) ----
 * Float64 area quadrature of a solid triangle for the rows where the closed form would lose digits: the triangle is
 * small (longest edge <= 0.02 h) or a sliver (2 area <= 0.01 longest edge^2); the other rows get status 0 and zero
 * values (they keep the closed form).  tri [6] (host): the vertices v0 v1 v2 in the rule's order (v2 - v0 the shortest
 * edge), area2 = 2 area, sign +1 for a counter-clockwise solid triangle (-1 clockwise), background 1 for an unbounded
 * solid.  lpos [n*2] body-frame positions, sup [n], valid [n] (may be NULL), all device.  Writes values [n*12]
 * (support-normalised units, body frame, order lam m1x m1y Gx Gy g1xx g1xy g1yx g1yy m20 m11 m02), estimate [n*12]
 * (may be NULL; empirical quadrature differences, NaN where status is 0) and status [n]: 0 closed form, 1 converged,
 * -1 panel budget exhausted (values NaN).  Kernels with at most two radii (cubic, w2, w4, w6, poly6).  Replaces
 * warptriangle.channels / prepare (src/warpSPHBoundaries/edge/warptriangle.py:126-201, 258-310). */
int wsb_triangle_channels(const double* tri, double area2, double sign, int background, int kernel, const double* lpos,
                          const double* sup, const int32_t* valid, int64_t n, double tolerance, int max_panels,
                          double* values, double* estimate, int32_t* status, void* stream);

/* The per-row override of a conditioned triangle: rows with status != 0 take values (rotated into the world frame by
 * pose [4] = (cx, cy, cos, sin) and scaled by the support: m1 h, G 1/h, m2 h^2), the others the closed-form outputs
 * clam [n], cG [n*2], ccov [n*4], cm1 [n*2], cm2 [n*4]; the result is assigned (add = 0) or added into lam, G, cov, m1,
 * m2 (all device).  Replaces the quadrature override of the contraction (src/warpSPHBoundaries/scene/fused.py:556-564,
 * src/warpSPHBoundaries/scene/scene.py:405-409). */
int wsb_triangle_combine(const double* values, const int32_t* status, const double* sup, const double* pose, int64_t n,
                         int add, const double* clam, const double* cG, const double* ccov, const double* cm1,
                         const double* cm2, double* lam, double* G, double* cov, double* m1, double* m2,
                         void* stream);

/* ---- solid disks (2-D): the disk element ----
 * Non-overlapping solid disks in a body frame (a fibre bundle, or one solid disk body): centres [m*2] and radii [m]
 * on the host, copied to `device` with a cell grid (cell >= support_max) listing every disk that reaches each cell.
 * wsb_disk_aggregate writes the twelve channels of the disks at every particle exactly as wsb_aggregate writes those
 * of a surface (body frame from `pose`, world-frame outputs, out_mask with WSB_OUT_ASSIGN for the first
 * representation of a body; rows outside `allowed` get zeros), for the exact-table kernel ids (0 .. 9), on a
 * caller workspace of wsb_disk_workspace_size bytes (4 bytes per row).  The integrals are evaluated by graded
 * Gauss-Legendre quadrature along the disk's circle inside the support (float64, ~1e-13), one warp per particle
 * that reaches a disk, where the reference looks them up in Chebyshev tables (~1e-6 .. 1e-10).  Replaces DiskArrayRep's fixed
 * disk topology and the disk channel launch (src/warpSPHBoundaries/scene/fixedadj.py:199-246,
 * edge/warpdisk.py:1-199, scene/fused.py:566-574); a solid ImplicitRep disk is a one-disk set
 * (scene/scene.py:576-580). */
typedef struct wsb_disks wsb_disks;
int wsb_disks_create(const double* centres, const double* radii, int64_t m, double support_max, int device,
                     wsb_disks** out);
int wsb_disks_destroy(wsb_disks* d);
size_t wsb_disk_workspace_size(const wsb_disks* d, int64_t n);
int wsb_disk_aggregate(const wsb_disks* d, int kernel, const double* pos, const double* sup, const int32_t* allowed,
                       int64_t n, const double* pose, int out_mask, double* lam, double* G, double* cov, double* m1,
                       double* m2, void* workspace, size_t workspace_bytes, void* stream);
/* The detector inputs of disk sets, as wsb_cone_area / wsb_dir_extreme for surfaces but per call (no prepared
 * workspace): area [2n] ADDED (wedge, then full disk), out [n] max-accumulated; closed forms per (particle, disk)
 * (src/warpSPHBoundaries/scene/fused.py:310-475 _disk_cum, _disk_cone_area_kernel, _disk_dir_extreme_kernel). */
int wsb_disk_cone_area(const wsb_disks* d, const double* pos, const double* sup, const int32_t* allowed, int64_t n,
                       const double* pose, const double* axes, double half_angle, double* area, void* stream);
int wsb_disk_dir_extreme(const wsb_disks* d, const double* pos, const double* sup, const int32_t* allowed, int64_t n,
                         const double* pose, const double* vecs, double* out, void* stream);

/* ---- finite-element pair weights (2-D, P1 triangles) ----
 * For every (query, element) pair k: w[3k + i] = int_T W_h(x' - x) phi_i(x') dx' and G[6k + 2i + j] =
 * int_T d/dx_j W_h(x' - x) phi_i(x') dx' (physical units) for the three barycentric functions phi_i of triangle
 * elems[3 e .. 3 e + 2] (vertex order as given), query pos[2 q], support sup[q]; kernel ids 0 .. 9.  Exact closed
 * forms of the triangle's channels, or the reference's 8 x 8 far-field Gauss rule for a triangle far from the query
 * and smooth under the kernel.  All arrays on the device; n_pos rows of pos / sup, n_verts vertices, n_elems elements.
 * A pair whose query, element or vertex index lies outside its array gets NaN outputs and sets *status (a device
 * int32 the caller zeroes) to 1; nothing outside the arrays is read.  The launch runs on the device that holds pos.
 * Replaces warpbc.pair_weights (src/warpSPHBoundaries/edge/warpbc.py:226-345, 486-510). */
int wsb_pair_weights(int kernel, const int32_t* pair_q, const int32_t* pair_e, int64_t n_pairs, const double* pos,
                     const double* sup, int64_t n_pos, const double* verts, int64_t n_verts, const int32_t* elems,
                     int64_t n_elems, double* w, double* G, int32_t* status, void* stream);

/* ---- scenes: several rigid bodies, each with closed surfaces and a pose ----
 * A scene groups surfaces (wsb_surface handles, which must outlive the scene) into bodies with poses (cx, cy, cos,
 * sin: world = R local + c), on one device.  wsb_scene_aggregate evaluates every body at once: for each kernel group
 * g and body b, lam[g] + b*ld, G[g] + 2*b*ld, cov[g] + 4*b*ld, m1[g] + 2*b*ld, m2[g] + 4*b*ld receive that body's
 * outputs of the n rows (assigned; ld >= n is the row stride per body; a body without surfaces gets zeros), world
 * frame, as wsb_aggregate_groups per surface (the first surface of a body assigns, the others add).  The workspace
 * (wsb_scene_workspace_size) is reused surface after surface on the stream.  wsb_scene_set_pose copies the pose on
 * `stream` and returns when it has arrived.  Replaces the reference's Scene with its bodies and poses
 * (src/warpSPHBoundaries/scene/scene.py:1230-1300) evaluated by the fused wall over all bodies
 * (src/warpSPHBoundaries/scene/fused.py:506-547, called from scene/provider.py:89-110). */
typedef struct wsb_scene wsb_scene;
int wsb_scene_create(int device, wsb_scene** out);
int wsb_scene_destroy(wsb_scene* sc);
int wsb_scene_add_body(wsb_scene* sc, const double* pose, int* body);
int wsb_scene_add_surface(wsb_scene* sc, int body, const wsb_surface* surface);
int wsb_scene_set_pose(wsb_scene* sc, int body, const double* pose, void* stream);
int wsb_scene_info(const wsb_scene* sc, int* n_bodies, int* n_surfaces);
size_t wsb_scene_workspace_size(const wsb_scene* sc, int64_t n);
int wsb_scene_aggregate(const wsb_scene* sc, int n_groups, const int32_t* kernels, int precision, const double* pos,
                        const double* sup, const int32_t* allowed, int64_t n, int64_t ld, double* const* lam,
                        double* const* G, double* const* cov, double* const* m1, double* const* m2, void* workspace,
                        size_t workspace_bytes, void* stream);

/* ---- the serving loop: continuous batching of boundary queries over resident scenes ----
 * wsb_server_create: n_streams stream slots on `device`, batches of at most max_batch_rows rows, persistent device
 * buffers (inputs, outputs, workspace) grown on demand within hbm_budget bytes.  wsb_serve_submit queues one request
 * (lambda + the twelve moments of kernel `kernel` at the caller's device arrays pos [n*2], sup [n]; outputs assigned
 * into the caller's [B, n, ...] arrays lam [B*n], G [B*n*2], cov [B*n*4], m1 [B*n*2], m2 [B*n*4], any may be NULL;
 * with grad != 0 also d_pos [n*2] = d sum_b lam_b / dx), read once `stream` reaches the point of submission, and
 * returns its id; it may launch work.  wsb_serve_poll advances the scheduler (retires finished batches, admits queued
 * requests into free slots: the oldest request and every later one of the same scene, kernel, precision and grad that
 * fits the batch rows, as one launch family over their concatenated rows; a request of more than max_batch_rows rows
 * runs in chunks on its own arrays) and sets *done for request_id (for request_id 0: nothing queued or running).
 * wsb_serve_wait polls until done; wsb_serve_release forgets a completed request.  A request's result is
 * bit-identical alone and in any batch (rows are independent).  wsb_server_stats: completed requests and the p50 / p99
 * of their latency (submission to the poll that saw their completion).  One host thread drives a server.  Replaces
 * the provider call per simulation (src/warpSPHBoundaries/scene/provider.py:38-113) with a shared request loop; the
 * reference has no server of its own. */
typedef struct wsb_server wsb_server;
int wsb_server_create(int device, int n_streams, int64_t max_batch_rows, size_t hbm_budget, wsb_server** out);
int wsb_server_destroy(wsb_server* srv);
int wsb_serve_submit(wsb_server* srv, const wsb_scene* scene, int kernel, int precision, int grad, const double* pos,
                     const double* sup, int64_t n, double* lam, double* G, double* cov, double* m1, double* m2,
                     double* d_pos, void* stream, int64_t* request_id);
int wsb_serve_poll(wsb_server* srv, int64_t request_id, int* done);
int wsb_serve_wait(wsb_server* srv, int64_t request_id);
int wsb_serve_release(wsb_server* srv, int64_t request_id);
int wsb_server_stats(const wsb_server* srv, int64_t* completed, double* p50_ms, double* p99_ms,
                     size_t* reserved_bytes);

/* ---- closed triangle surfaces (3-D) ----
 * A watertight, consistently oriented triangle surface with outward normals (positive signed volume): verts
 * [n_verts*3] and faces [n_faces*3] (vertex ids) on the host, copied to `device` with a cell grid of faces (cell =
 * support_max) and (x, y) columns of faces for the inside test.  Invalid surfaces (open, inconsistently oriented,
 * negative volume, zero-area faces) return WSB_ERR_ARG.  Replaces fluxbridge's Geometry.closed_surface with its
 * whole-element search tree (src/warpSPHBoundaries/fluxbridge/geometry.py:75-170, device_search.py:125-212) and the
 * surface checks of mesh3d ClosedSurface (src/warpSPHBoundaries/mesh3d/reference.py:221-244). */
typedef struct wsb_mesh wsb_mesh;
int wsb_mesh_create(const double* verts, int64_t n_verts, const int32_t* faces, int64_t n_faces, double support_max,
                    int device, wsb_mesh** out);
int wsb_mesh_destroy(wsb_mesh* m);

/* bytes of the workspace wsb_mesh_channels needs for n queries */
size_t wsb_mesh_workspace_size(const wsb_mesh* m, int64_t n);

/* 1 where the query pos [n*3] (device) lies inside the solid, else 0 (parity of a vertical ray's crossings with
 * exact tie rules on shared edges).  Replaces the solid-angle winding sum of fluxbridge's closed-surface element
 * (src/warpSPHBoundaries/fluxbridge/wp_func.py:231-253). */
int wsb_mesh_inside(const wsb_mesh* m, const double* pos, int64_t n, int32_t* inside, void* stream);

/* The 28 baseline channels of every query (pos [n*3], supports sup [n] <= support_max, device) into out [n*28]
 * (device, float64, physical units, overwritten): value moments int_solid y^alpha W for alpha = 000 100 010 001 200
 * 110 101 020 011 002 (y = point - query), kernel-gradient moments int y^alpha dW/dx_j for alpha = 000 100 010 001 and
 * j = 0..2, and the kernel Hessian int d2W/dx_i dx_j (00 01 02 11 12 22).  `inside` [n] (may be NULL) receives the
 * inside test (-1 for a row with support above support_max, support <= 0 or a non-finite position: its outputs are
 * NaN).  Kernels cubic, w2, w4, w6.  Replaces fluxbridge's Evaluator over Geometry.closed_surface with the baseline
 * requests: Batch.launch, wp_func.element / output / batch and Batch.reduce
 * (src/warpSPHBoundaries/fluxbridge/evaluate.py:11-187, src/warpSPHBoundaries/fluxbridge/wp_func.py:119-369). */
int wsb_mesh_channels(const wsb_mesh* m, int kernel, const double* pos, const double* sup, int64_t n, double* out,
                      int32_t* inside, void* workspace, size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* WSB_H */
