/*
 * beep3_b200.h -- C ABI of the B200 (sm_100a) BEM matvec / GMRES engine.
 *
 * The engine replaces the accelerator boundary of libBEEP: the OpenCL handler
 * and its work blobs (src/opencl/opencl_handler.h:87-229,
 * src/opencl/opencl_workblob.h:20-52, src/bem/opencl_bem.h:37-295,
 * src/fmm/opencl_fmm.h) and, behind it, the bodies of
 * BEEP::init_fmm_octree, BEEP::precalc_neighbour_interactions,
 * BEEP::do_bem_fmm_iteration and BEEP::gmres (src/beep/beep.cpp).
 * BEEP's own public API (src/beep/beep.h:198-278) is unchanged: its methods
 * call these entry points instead of the OpenCL queue.
 *
 * Conventions
 *   - every function returns an int32_t status, BP_OK (0) on success; the
 *     message of the last failure on the calling thread is bp_last_error();
 *   - nothing throws across the ABI; all pointers are plain C pointers;
 *   - the unknown vector is x = [f; h] of length 2N: the N surface potentials
 *     followed by the N normal derivatives, in patch order
 *     (src/beep/beep.cpp:1275-1283);
 *   - "host" pointers are ordinary CPU memory (pinned or pageable);
 *     "device" pointers are CUDA global memory on the context's device and
 *     calls taking them are ordered on the context's stream without a host
 *     synchronisation.
 */
#ifndef BEEP3_B200_H_
#define BEEP3_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BP_ABI_VERSION 1

enum bp_status {
  BP_OK = 0,
  BP_ERR_INVALID = 1,      /* bad argument */
  BP_ERR_CUDA = 2,         /* CUDA runtime failure */
  BP_ERR_NOMEM = 3,        /* host allocation failure */
  BP_ERR_BUDGET = 4,       /* device allocation would exceed the context's HBM budget */
  BP_ERR_TIMEOUT = 5,      /* a bounded device-side wait gave up */
  BP_ERR_INTERNAL = 6,
  BP_ERR_UNSUPPORTED = 7,  /* e.g. an FMM order without quadrature tables */
  BP_ERR_NOT_CONVERGED = 8 /* GMRES stopped at its iteration limit (x is still written) */
};

enum bp_precision {
  BP_PREC_FP64 = 0,  /* near field, FMM and Krylov solve in FP64 */
  BP_PREC_MIXED = 1  /* FP32 near field and FMM, FP64 singular integrals, Krylov and energy */
};

typedef struct bp_ctx_s* bp_ctx;
typedef struct bp_geom_s* bp_geom;
typedef struct bp_problem_s* bp_problem;

const char* bp_last_error(void);
int32_t bp_abi_version(void);

/* ---------------------------------------------------------------------------
 * Context: one CUDA device, one stream, one HBM budget.
 * Replaces OpenCL_Handler construction and its 512 MB/device admission
 * budget (src/opencl/opencl_handler.cpp:19-147, :397-462).
 */
int32_t bp_ctx_create(int32_t device, uint64_t hbm_budget_bytes, bp_ctx* out);
/* Destroy problems and meshes first: while any made on the context is alive
 * (a mesh whose deletion waits for its last posed problem included) this
 * returns BP_ERR_INVALID and the context stays valid. */
int32_t bp_ctx_destroy(bp_ctx ctx);
/* cudaStream_t; NULL = the context's own.  Work already issued on the
 * previous stream is waited for before the switch, so device blocks it
 * releases are never handed to work on the new stream while still in use. */
int32_t bp_ctx_set_stream(bp_ctx ctx, void* cuda_stream);
int32_t bp_ctx_memory(bp_ctx ctx, uint64_t* used_bytes, uint64_t* budget_bytes);
/* Device blocks of destroyed problems that the context keeps for the next
 * problem of similar size (no cudaMalloc / cudaFree between poses): their
 * bytes, and with release != 0 their return to the driver.  No counterpart in
 * the reference (its OpenCL buffers are allocated per work blob). */
int32_t bp_ctx_cache(bp_ctx ctx, uint64_t* cached_bytes, int32_t release);
int32_t bp_ctx_synchronize(bp_ctx ctx);

/* ---------------------------------------------------------------------------
 * Surface preparation (host only): vertex-centred node patches and their
 * point lists from a closed triangulated surface, planar or PN-curved.
 * Mirrors Mesh::create_bezier_triangles / create_node_patches and
 * BasicNodePatch point generation (src/bem/mesh.cpp:1632-1652,
 * src/bem/node_patch.cpp:55-130, :198-273).  Points are 7 doubles:
 * x y z nx ny nz w.  qual_rule / quad_rule are the per-triangle rule orders
 * (0 = one centroid point per patch, else 1, 4, 6 or 7); galerkin points use
 * the 4-point rule.  totals[0] = curved surface area, totals[1] = planar.
 */
int32_t bp_geom_create(int32_t n_vertices, const double* vertices, const double* vertex_normals,
                       int32_t n_triangles, const int32_t* triangles, int32_t planar, int32_t qual_rule,
                       int32_t quad_rule, bp_geom* out);
int32_t bp_geom_sizes(bp_geom g, int32_t* n_patches, int32_t* n_qual, int32_t* n_quad, int32_t* n_galerkin);
int32_t bp_geom_copy(bp_geom g, double* centroid, double* normal, double* area, double* node,
                     int32_t* qual_offsets, double* qual_points, int32_t* quad_offsets, double* quad_points,
                     int32_t* galerkin_offsets, double* galerkin_points, double* totals);
int32_t bp_geom_destroy(bp_geom g);

/* ---------------------------------------------------------------------------
 * Problem: all node patches of all mesh instances in universe coordinates
 * (the contents BEEP inserts into its FMM octree, src/beep/beep.cpp:1618-1634).
 */
typedef struct {
  int32_t n_patches;
  const double* centroid;          /* [n][3] */
  const double* normal;            /* [n][3] unit */
  const double* area;              /* [n] curved patch area */
  const double* dielectric_ratio;  /* [n] eps_solvent / eps_protein */
  const double* gc;                /* [n] geometric correction, 0.5 */
  const int32_t* qual_offsets;     /* [n+1] qualocation (collocation) points */
  const double* qual_points;       /* [.][7], weights sum to 1 per patch */
  const int32_t* quad_offsets;     /* [n+1] quadrature (integration) points */
  const double* quad_points;       /* [.][7] */
  const int32_t* galerkin_offsets; /* [n+1] points of the singular self-patch integral */
  const double* galerkin_points;   /* [.][7] */
} bp_patches;

typedef struct {
  double kappa;           /* inverse Debye length, 1/Angstrom */
  double beta0;           /* screening standing in for the Laplace channels (1e-10) */
  double cube_centre[3];  /* bounding cube (BEEP::calculate_bounding_cube) */
  double cube_edge;
  int32_t nbsize;         /* target mean neighbourhood size of the adaptive tree; with
                             BP_FLAG_DEVICE_TREE the most patches a leaf may hold */
  int32_t nterms;         /* FMM order: 9, the reference's matvec order (FMM_BEM_Octree<9,9,67>);
                             other orders return BP_ERR_UNSUPPORTED */
  int32_t precision;      /* enum bp_precision */
  int32_t flags;          /* bitwise or of enum bp_flags */
} bp_params;

enum bp_flags {
  /* Near field computed in every matvec from the point lists instead of
   * cached: no coefficient storage (16 or 32 bytes per near pair), at the
   * assembly's cost per matvec.  The reference's uncached OpenCL path
   * (BEM_kernels_instant, src/bem/opencl_bem_kernels.cl:237-352;
   * src/beep/beep.cpp:999-1008); for problems whose coefficients would not
   * fit the HBM budget. */
  BP_FLAG_NEARFIELD_ON_DEMAND = 1,
  /* Octree built on the device with a cap of nbsize patches per leaf
   * instead of the reference's refinement (insertion threshold 4*nbsize,
   * then splitting the leaves with the largest neighbourhoods until the mean
   * neighbourhood size is at most nbsize: src/fmm/octree.h:867-986,
   * :1118-1148).  Patches are sorted by the Morton code of their centroid's
   * cell at depth 20; a node with more than nbsize patches splits; the
   * neighbourhood rule (the 26 neighbours of a split node split too, their
   * children being shadows) and the FMM bookkeeping are the reference's.
   * Results equal the reference-tree problem's to the FMM's accuracy, not
   * bitwise: the near/far split of pairs differs. */
  BP_FLAG_DEVICE_TREE = 2,
  /* Mixed engine only, cached near field only: each FP32 coefficient is
   * rounded to its top 24 bits (sign, exponent, 15 stored significand bits;
   * round to nearest) and stored in 12 bytes a pair instead of 16, read by
   * the apply kernel and widened in registers.  A storage option of this
   * engine with no reference counterpart (the reference caches FP32
   * coefficients, src/beep/beep.cpp:768-1064): 25 % less coefficient
   * memory and traffic per matvec for a relative error of at most 2^-16 per
   * coefficient.  Combined with BP_PREC_FP64 or
   * BP_FLAG_NEARFIELD_ON_DEMAND the call fails with BP_ERR_INVALID. */
  BP_FLAG_COMPACT_NEARFIELD = 4,
  /* Mixed engine, problems posed from device meshes (bp_problem_create_posed,
   * bp_problem_create_batch): the near-field coefficients of the pairs of
   * patches of one mesh closer than about 4.4 edges of the problem's
   * smallest leaf are integrated once, in the mesh's frame, kept with the
   * mesh (for one kappa at a time, at the radius of the problem that built
   * them; 28 bytes a pair, at most 8 GB a mesh, the radius shrunk to fit)
   * and looked up by the assembly of every later problem with that mesh and
   * kappa, whatever its pose: a rigid move does not change them.  A cache
   * that does not fit the context's budget is not built.  The other pairs are integrated as
   * usual.  No counterpart in the reference, which integrates every pair of
   * every problem (src/beep/beep.cpp:768-956); results agree with the
   * uncached assembly to FP32 rounding (the pairs' coordinates are those of
   * the mesh's frame, not the posed ones).  Ignored by the FP64 engine, the
   * on-demand near field and meshes with more than one quadrature point per
   * patch. */
  BP_FLAG_MESH_PAIR_CACHE = 8
};

typedef struct {
  int64_t n_patches;
  int64_t n_levels;
  int64_t n_nodes;
  int64_t n_leaves;
  int64_t n_nearfield_pairs; /* sum over leaves of |leaf| * |neighbourhood| */
  int64_t n_nearfield_cols;  /* sum over leaves of |neighbourhood| (stored column ids) */
  int64_t fmm_active;        /* 1 when the tree is deep enough for the far field */
  uint64_t device_bytes;
  double tree_ms;
  double assemble_ms;        /* device time of the singular + near-field assembly kernels */
  int64_t gmres_graph;       /* 1 once a solve ran its Arnoldi loop as one CUDA graph with a
                                device-side loop condition, 0 before the first solve or when the
                                host drove the loop step by step */
  double fmm_setup_ms;       /* host wall time of the far-field set-up (tables, operators, schedule) */
  double setup_ms;           /* host wall time from the tree build to a problem ready to run */
  int64_t n_scenarios;       /* independent scenarios (bp_problem_create_batch), else 1 */
  /* work of one far-field pass (0 without FMM): columns (node, channel) of
   * the multipole->plane-wave and plane-wave->local operators, plane-wave
   * translation entries (each over 12 channels), columns of the M2M / L2L
   * shifts, plane waves per direction and coefficients per channel */
  int64_t fmm_m2x_cols, fmm_x2l_cols, fmm_translations, fmm_shift_cols, fmm_plane_waves, fmm_coefficients;
} bp_problem_info;

/* Builds the adaptive octree, the singular self-patch integrals and the
 * cached near-field coefficients (BEEP::init_fmm_octree +
 * BEEP::precalc_neighbour_interactions, src/beep/beep.cpp:1585-1641,
 * :768-956). */
int32_t bp_problem_create(bp_ctx ctx, const bp_patches* patches, const bp_params* params, bp_problem* out);

/* ---------------------------------------------------------------------------
 * Device-resident meshes and posed problems (rigid-body scans).  A mesh's
 * node patches, in its own frame, are checked and uploaded once; a problem
 * is then built from instances of such meshes, each placed by a rigid move
 * p -> R (p - centre) + offset, n -> R n that runs on the device, so a new
 * pose costs no host transform and no upload of point lists.  The reference
 * moves its host patch objects for every pose instead
 * (MeshInstance::init, src/bem/mesh_instance.cpp:50-85; NodePatch
 * change_coordinate_frame, src/bem/node_patch.cpp:402-478); these entry
 * points have no counterpart there.  Problems built from a mesh keep it:
 * bp_mesh_destroy while one exists defers the deletion to the last of them
 * (bp_rhs_posed reads the mesh).  Its patches' dielectric_ratio entries are
 * ignored (the instance gives it).  The context must outlive its meshes.
 */
typedef struct bp_mesh_s* bp_mesh;
int32_t bp_mesh_create(bp_ctx ctx, const bp_patches* patches, const double centre[3], bp_mesh* out);
/* The same device-resident mesh generated on the device from a closed
 * triangulated surface (vertices [n_vertices][3], optional unit vertex
 * normals (NULL or zero rows: area-weighted), anticlockwise triangles
 * [n_triangles][3]): the node patches and point lists bp_geom_create makes on
 * the host (Mesh::create_bezier_triangles / create_node_patches,
 * src/bem/mesh.cpp:1632-1652), bit for bit, with no host point generation or
 * upload.  totals (may be NULL) = {curved area, planar area}. */
int32_t bp_mesh_create_from_surface(bp_ctx ctx, int32_t n_vertices, const double* vertices,
                                    const double* vertex_normals, int32_t n_triangles, const int32_t* triangles,
                                    int32_t planar, int32_t qual_rule, int32_t quad_rule, const double centre[3],
                                    bp_mesh* out, double* totals);
int32_t bp_mesh_destroy(bp_mesh mesh);

typedef struct {
  bp_mesh mesh;
  double rotation[9];       /* row-major R */
  double offset[3];         /* where the mesh centre goes */
  double dielectric_ratio;  /* eps_solvent / eps_protein of this instance */
} bp_instance;

/* bp_problem_create for the instances' patches, concatenated in instance
 * order. */
int32_t bp_problem_create_posed(bp_ctx ctx, const bp_instance* instances, int32_t n_instances,
                                const bp_params* params, bp_problem* out);
/* Several independent scenarios in one problem: a batch of poses whose
 * matvecs and solves share every kernel launch (BEEP::insert_mesh_instance /
 * move_mesh_instance, src/beep/beep.cpp:223-290, run once per scenario).
 * Scenario s holds instances [scenario_first[s], scenario_first[s+1])
 * (scenario_first[0] = 0, scenario_first[n_scenarios] = n_instances, every
 * scenario non-empty); its tree is built in the cube of centre
 * cube_centres[3s..3s+2] and edge params->cube_edge (one edge for all, at
 * least every scenario's own extent; params->cube_centre is ignored).  The
 * matvec is block diagonal: no interaction crosses scenarios, and each
 * block equals the matvec of bp_problem_create_posed on the scenario's
 * instances with that cube, up to rounding.  Patches are concatenated in
 * instance order; bp_rhs_posed sums each instance's charges over its own
 * scenario only; bp_solve_batch solves every scenario with its own GMRES. */
int32_t bp_problem_create_batch(bp_ctx ctx, const bp_instance* instances, int32_t n_instances,
                                const int32_t* scenario_first, int32_t n_scenarios, const double* cube_centres,
                                const bp_params* params, bp_problem* out);
int32_t bp_problem_destroy(bp_problem p);
int32_t bp_problem_info_get(bp_problem p, bp_problem_info* info);

/* Export of the adaptive octree (for inspection and cross-checks).
 * node_info: [n_nodes][18] int32 = level, ix, iy, iz, flags (1 has children,
 * 2 leaf, 4 shadow), parent, content_start, content_count, mp_idx, lc_idx,
 * child node ids 1..8 (-1 absent); nodes are level by level in the
 * reference's map order.  node_geom: [n_nodes][4] = centre xyz, edge.
 * contents: [n_contents] patch ids of every node, node after node, each in
 * insertion order (a patch appears once per level it is stored on).
 * Any output pointer may be NULL. */
int32_t bp_problem_tree(bp_problem p, int32_t* n_nodes, int32_t* n_levels, int64_t* n_contents, int32_t* node_info, double* node_geom,
                        int32_t* contents);

/* The same adaptive octree built on the host alone (no device needed):
 * BEEP::init_fmm_octree's insert + build_neighbourhoods +
 * optimize_neighbourhoods + remove_empty_nodes (src/beep/beep.cpp:1585-1641).
 * Export layout as bp_problem_tree. */
typedef struct bp_tree_s* bp_tree;
int32_t bp_tree_create(int32_t n_points, const double* points, const double cube_centre[3], double cube_edge,
                       int32_t nbsize, bp_tree* out);
int32_t bp_tree_export(bp_tree t, int32_t* n_nodes, int32_t* n_levels, int64_t* n_contents, int32_t* node_info, double* node_geom,
                       int32_t* contents);
int32_t bp_tree_destroy(bp_tree t);

/* y = A x, the BEM/FMM matvec (BEEP::do_bem_fmm_iteration,
 * src/beep/beep.cpp:1485-1583).  Host arrays of 2N doubles; blocking. */
int32_t bp_matvec(bp_problem p, const double* x, double* y);
/* Same on device arrays, stream-ordered, no synchronisation. */
int32_t bp_matvec_device(bp_problem p, const double* x_dev, double* y_dev);
/* Per-stage device time of `reps` matvecs on device arrays, averaged, in ms,
 * measured with CUDA events on the context stream, all stages serialised on
 * that stream.  stage_ms[0] = near field (+ the final near/far add),
 * [1] = P2M, [2] = M2M, [3] = multipole->exponential, [4] = exponential
 * translations fused with exponential->local, [5] = L2P per-leaf
 * preparation, [6] = L2L, [7] = L2P evaluation; *n_stages = 8.
 * stage_launches (may be NULL) receives kernel launches per stage per
 * matvec. */
int32_t bp_matvec_profile(bp_problem p, const double* x_dev, double* y_dev, int32_t reps, double* stage_ms,
                          int32_t* stage_launches, int32_t* n_stages);

/* Test of the bounded-wait timeout path (no counterpart in the reference).
 * The tensor-core kernels of the mixed engine's far field wait on their own
 * MMA-completion barriers with a bound of about a second; a wait that runs
 * out abandons the kernel's tile (after draining the MMAs it issued and
 * freeing its tensor memory) and the next bp_matvec / bp_solve on the
 * problem returns BP_ERR_TIMEOUT once.  While enable != 0 every CTA of those
 * kernels also waits, with a bound of 200000 cycles, on a barrier that
 * nothing arrives on, so that path runs on every matvec.  Returns
 * BP_ERR_UNSUPPORTED for problems without those kernels (FP64 engine, or no
 * far field).  Blocking. */
int32_t bp_problem_test_wait_timeout(bp_problem p, int32_t enable);

/* GMRES(restart) solve of A x = rhs (BEEP::gmres, src/beep/beep.cpp:1262-1483):
 * classical Gram-Schmidt Arnoldi and Givens rotations in FP64, stop when the
 * residual estimate falls below tol * ||rhs||.  x holds the initial guess on
 * entry and the solution on return.  restart <= 0 means one cycle of
 * max_iters, as in the reference.  Host arrays of 2N doubles. */
int32_t bp_solve(bp_problem p, const double* rhs, double* x, double tol, int32_t max_iters, int32_t restart,
                 int32_t* iterations, double* rel_residual);
/* bp_solve of a batch problem: every scenario runs its own GMRES (its own
 * Krylov basis, ||rhs|| and stop test) in shared launches, a converged
 * scenario sitting out the remaining steps; iterations and rel_residual
 * receive one entry per scenario.  bp_solve on a batch reports the worst
 * scenario.  BP_ERR_NOT_CONVERGED when some scenario did not converge. */
int32_t bp_solve_batch(bp_problem p, const double* rhs, double* x, double tol, int32_t max_iters, int32_t restart,
                       int32_t* iterations, double* rel_residual);
/* Same on device arrays (still blocks: the Krylov loop reads its residual). */
int32_t bp_solve_device(bp_problem p, const double* rhs_dev, double* x_dev, double tol, int32_t max_iters,
                        int32_t restart, int32_t* iterations, double* rel_residual);

/* Right-hand side from point charges (BEEP::set_rhs, src/beep/beep.cpp:1124-1260):
 * Coulomb potential and field of all charges at every qualocation point,
 * weighted and scaled by 1/(4 pi eps_solvent).  charges_xyzq: [n][4]. */
int32_t bp_rhs(bp_problem p, const double* charges_xyzq, int32_t n_charges, double eps_solvent, double* rhs);
/* The same for a problem made by bp_problem_create_posed (or _batch: each
 * instance then sees the charges of its own scenario only), from each
 * instance's charges in its mesh's own frame (the frame of the points given
 * to bp_mesh_create): charges_xyzq[k] holds n_charges[k] charges of
 * instance k.  The potential of an instance's own charges at its own
 * qualocation points does not change when the instance moves, so it is
 * computed once per mesh, charge list, eps_solvent and precision and kept
 * with the mesh (the 4 most recent); each call sums the other instances'
 * charges only.  Equal to bp_rhs with every charge placed in the problem's
 * frame, up to rounding. */
int32_t bp_rhs_posed(bp_problem p, const double* const* charges_xyzq, const int32_t* n_charges, double eps_solvent,
                     double* rhs);

/* Right-hand side without any device allocation (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc -- host applications
 * whose own allocator owns the device memory, or code that must not
 * allocate while another thread captures a CUDA graph: every argument is a
 * caller-owned device pointer (qualocation offsets [n_patches+1], points as
 * seven arrays x y z nx ny nz w of n_qual_points doubles each, charges
 * [n][4], rhs [2 n_patches]) and the kernels' per-point scratch is a fixed
 * 16 MiB array in the library, held on every GPU that loads it until exit.
 * At most 1048576 qualocation points per call (larger calls return
 * BP_ERR_INVALID).  The call runs on the calling thread's current device,
 * whose copy of the array it uses: every buffer must be device memory of
 * that device (else BP_ERR_INVALID), and cuda_stream a stream of it.
 * qual_offsets_dev must describe the point list: offsets[0] == 0,
 * non-decreasing, offsets[n_patches] == n_qual_points (the offsets are read
 * on the device only; a patch's range is clamped to [0, n_qual_points), so
 * offsets that break this give wrong sums but no out-of-bounds access).
 * The first call on a device looks the array up (do it
 * before any stream capture); calls that overlap on the GPU share the array
 * and race, so the caller serialises them.  Ordered on cuda_stream (NULL =
 * the legacy default stream), no host synchronisation. */
int32_t bp_rhs_noalloc(int32_t n_patches, const int32_t* qual_offsets_dev, const double* qual_points_soa_dev,
                       int32_t n_qual_points, const double* charges_xyzq_dev, int32_t n_charges, double eps_solvent,
                       double* rhs_dev, void* cuda_stream);

/* Energy coefficients of patches [first, first+count) from the charges of
 * their own mesh (Mesh::init_energy_precalcs + renormalise_energy_precalcs,
 * src/bem/mesh.cpp:730-925): Coulomb potential and normal field at the
 * galerkin points, corrected so that the f-coefficients satisfy Gauss's law
 * with total_area the curved area of the mesh. */
int32_t bp_energy_coefficients(bp_problem p, int32_t first, int32_t count, const double* charges_xyzq,
                               int32_t n_charges, double total_area, double* coef_f, double* coef_h);
/* Solvation energy in kJ/mol of patches [first, first+count) from a solution
 * x (host, 2N), compensated summation (Mesh::calculate_energy,
 * src/bem/mesh.cpp:1373-1404). */
int32_t bp_energy(bp_problem p, int32_t first, int32_t count, const double* coef_f, const double* coef_h,
                  double eps_ratio, const double* x, double* energy_kj_per_mol);

#ifdef __cplusplus
}
#endif

#endif /* BEEP3_B200_H_ */
