/* libporerad — B200 (sm_100a) implementation of porerad's surface-radiation path:
 * surface patches -> seeded Lambertian rays -> first-hit voxel traversal into
 * integer patch-to-patch counts -> balanced exchange operator -> gray-diffuse
 * radiosity -> wall and internal net fluxes.
 *
 * The reference (moxi000/pore-radiation-ijhmt2026, package `porerad`) exposes no C
 * interface; its boundary is the Python API of porerad.view_factors and
 * porerad.exchange.  Each entry point below names the reference function it
 * replaces (file:line within the reference project).  A Python binding with the
 * reference's exact names and signatures sits on top (package porerad_b200).
 *
 * Conventions
 *  - Every call returns PR_OK (0) or a PR_ERR_* code; pr_last_error() then holds a
 *    message for the calling thread.  No call aborts, traps or exits.
 *  - Array arguments may be host memory (pageable or pinned) or device memory of
 *    the current device; the library copies with cudaMemcpyDefault.  Calls that
 *    write host-visible outputs return after the stream has finished them.
 *  - `stream` is a cudaStream_t (NULL: the legacy default stream).  Objects are
 *    bound to the device that was current when they were created.  Distinct
 *    objects may be used concurrently from different host threads on different
 *    streams; one object must not be used by two calls at the same time.
 *  - Patch ids are int32 (at most 2^31 - 1 patches), counts are int64 at the API.
 */
#ifndef PORERAD_H
#define PORERAD_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define PR_API __attribute__((visibility("default")))
#else
#define PR_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
  PR_OK = 0,
  PR_ERR_ARG = 1,         /* invalid argument (ValueError in the Python binding) */
  PR_ERR_CUDA = 2,        /* CUDA runtime failure */
  PR_ERR_OOM = 3,         /* device memory exhausted */
  PR_ERR_UNRESOLVED = 4,  /* rays without a receiving patch: view_factors.py:268-269 (RuntimeError) */
  PR_ERR_ACCOUNTING = 5,  /* counts do not account for every ray: exchange.py:70-71 (ValueError) */
  PR_ERR_NOT_CLOSED = 6,  /* projected rows do not close: exchange.py:78-80 (RuntimeError) */
  PR_ERR_BALANCE = 7,     /* diagonal balancing did not converge: exchange.py:197 (RuntimeError) */
  PR_ERR_SERIES = 8,      /* reflection series did not converge: exchange.py:243-244 (RuntimeError) */
  PR_ERR_LIMIT = 9        /* a size beyond what this build supports */
};

/* Balancing method reported by pr_operator_info (exchange.py:153-197). */
enum { PR_BALANCE_NONE = 0, PR_BALANCE_ANDERSON = 1, PR_BALANCE_MULTIPLICATIVE = 2 };

/* Which product pr_operator_apply forms (exchange.py:82-122). */
enum {
  PR_APPLY_RAW = 0,       /* F x          raw_matvec      exchange.py:82-93   */
  PR_APPLY_RAW_T = 1,     /* F^T x        raw_rmatvec     exchange.py:95-106  */
  PR_APPLY_SYM = 2,       /* S x          symmetric_matvec exchange.py:108-112 */
  PR_APPLY_MATVEC = 3,    /* F_p x        matvec          exchange.py:114-117 */
  PR_APPLY_RMATVEC = 4    /* F_p^T x      rmatvec         exchange.py:119-122 */
};

/* Radiosity precision (pr_net_patch_power, pr_prescribed_field_channels). */
enum {
  PR_PRECISION_FP64 = 0,  /* binary64 reflection series, as the reference */
  PR_PRECISION_MIXED = 1  /* binary32 sweeps, binary64 residual refinement */
};

/* Seed of one ray block: numpy.random.PCG64(seed).state, i.e. the 128-bit LCG
 * state and increment that SeedSequence derives from the integer seed
 * (view_factors.py:149-151). */
typedef struct {
  uint64_t state_hi, state_lo, inc_hi, inc_lo;
} pr_pcg64;

typedef struct pr_case pr_case;         /* one x-oriented voxel geometry on one GPU */
typedef struct pr_counts pr_counts;     /* pooled first-hit counts, CSR by origin   */
typedef struct pr_operator pr_operator; /* projected view-factor operator F_p       */
typedef struct pr_conduction pr_conduction; /* finite-volume conduction system A, b    */

PR_API const char* pr_last_error(void);
PR_API int pr_version(void);

/* ---- geometry ------------------------------------------------------------
 * Replaces build_surface_patches(phases_x, H_m), view_factors.py:70-132.
 * phases_x: uint8 (nx, ny, nz) C order, 1 = solid, already oriented along x
 * (orient_along_x, view_factors.py:37-40). */
PR_API int pr_case_create(const uint8_t* phases_x, int64_t nx, int64_t ny, int64_t nz, double H_m,
                   void* stream, pr_case** out);
/* n_patches = SurfacePatches.n_patches (view_factors.py:65-67); n_wall = wall patches. */
PR_API int pr_case_info(const pr_case* c, int64_t* n_patches, int64_t* n_wall, size_t* device_bytes);
/* Copies the SurfacePatches fields (view_factors.py:53-63); any pointer may be NULL.
 * Shapes: solid (nx,ny,nz) u8; patch_class (P) i8; patch_cell (P) i32; patch_face (P) i8;
 * patch_origin, patch_normal (P,3) f64; patch_area_m2 (P) f64; cell_face_patch
 * (nx*ny*nz, 6) i32; hot_wall_patch, cold_wall_patch (ny,nz) i32. */
PR_API int pr_case_patches(const pr_case* c, uint8_t* solid, int8_t* patch_class, int32_t* patch_cell,
                    int8_t* patch_face, double* patch_origin, double* patch_normal,
                    double* patch_area_m2, int32_t* cell_face_patch, int32_t* hot_wall_patch,
                    int32_t* cold_wall_patch, void* stream);
PR_API void pr_case_destroy(pr_case* c);

/* ---- rays ----------------------------------------------------------------
 * Replaces generate_rays(patches, patch_start, patch_end, rays_per_patch, seed),
 * view_factors.py:135-182.  origins, directions: ((patch_end - patch_start) * R, 3) f64. */
PR_API int pr_generate_rays(const pr_case* c, int64_t patch_start, int64_t patch_end,
                     int64_t rays_per_patch, const pr_pcg64* seed, double* origins,
                     double* directions, void* stream);

/* ---- traversal -------------------------------------------------------------
 * Replaces trace_first_hit(patches, origins, directions), view_factors.py:261-270
 * (the traversal of view_factors.py:185-258).  receiver (n_rays) i32.  Returns
 * PR_ERR_UNRESOLVED with *n_failed > 0 when rays did not resolve a receiver. */
PR_API int pr_trace_first_hit(const pr_case* c, const double* origins, const double* directions,
                       int64_t n_rays, int32_t* receiver, int64_t* n_failed, void* stream);

/* ---- first-hit counts --------------------------------------------------------
 * Replaces first_hit_counts(patches, rays_per_patch, seed), view_factors.py:273-287,
 * for n_seeds blocks at once, pooled as pool_counts (view_factors.py:290-300) pools
 * them: rays are generated on the fly, traced, and the receivers of each origin
 * patch reduced into one sorted CSR row.  rays_per_origin = R * n_seeds. */
PR_API int pr_first_hit_counts(const pr_case* c, int64_t rays_per_patch, const pr_pcg64* seeds,
                        int n_seeds, void* stream, pr_counts** out);
/* first_hit_counts (view_factors.py:273-287) straight into host memory: the sorted edge list
 * of pr_first_hit_counts + pr_counts_copy, written into origin / receiver / count chunk by
 * chunk (64 M rays each) on a copy stream of its own while the next chunks trace, so that
 * with pinned arrays the copies overlap the traversal.  capacity = pairs the arrays hold
 * (n_patches * rays_per_patch * n_seeds always suffices; PR_ERR_LIMIT if exceeded); *n_pairs
 * receives the list's length.  No device table is kept. */
PR_API int pr_first_hit_counts_host(const pr_case* c, int64_t rays_per_patch, const pr_pcg64* seeds,
                                    int n_seeds, void* stream, int32_t* origin, int32_t* receiver,
                                    int64_t* count, int64_t capacity, int64_t* n_pairs);
/* pr_first_hit_counts for n_cases geometries at once (batched sweeps, serving): the rays of
 * all cases share persistent launches of the traversal, waves of up to 2^27 rays that mix
 * chunks of cases of different sizes.  seeds holds n_seeds per case (case-major); out
 * receives one count table per case, each identical to the single-case call's. */
PR_API int pr_first_hit_counts_batch(const pr_case* const* cases, int n_cases, int64_t rays_per_patch,
                                     const pr_pcg64* seeds, int n_seeds, void* stream, pr_counts** out);
/* nnz = pooled (origin, receiver) pairs; rays/steps: rays traced and DDA cells visited. */
PR_API int pr_counts_info(const pr_counts* k, int64_t* nnz, int64_t* n_patches, int64_t* rays,
                   int64_t* dda_steps);
/* The sorted edge list (origin i32, receiver i32, count i64) and rays_per_origin (i64). */
PR_API int pr_counts_copy(const pr_counts* k, int32_t* origin, int32_t* receiver, int64_t* count,
                   int64_t* rays_per_origin, void* stream);
/* The pairs of origin rows [row_begin, row_end) only, in the same sorted order: the part of
 * first_hit_counts' output (view_factors.py:273-287) whose origins lie in that patch range.
 * *n_pairs receives their number; with origin, receiver and count all NULL nothing else is
 * copied (size query).  PR_ERR_ARG for a range outside [0, n_patches]. */
PR_API int pr_counts_rows(const pr_counts* k, int64_t row_begin, int64_t row_end, int64_t* n_pairs,
                          int32_t* origin, int32_t* receiver, int64_t* count, void* stream);
/* ---- pinned host blocks for results (no counterpart in the reference) ----------------
 * first_hit_counts (view_factors.py:273-287) hands back gigabytes of NumPy arrays per call.
 * Arrays placed in a pinned block of this pool receive pr_counts_copy / pr_counts_rows
 * straight from the device at the link's rate; a released block is cached for the next
 * request that it holds with at most twice the bytes (bounded by PORERAD_HOST_CACHE_BYTES, default 32 GiB),
 * so pinning and page faults are paid once per size.  Blocks are page-aligned, rounded up
 * to 2 MiB.  release: PR_ERR_ARG for a pointer that is not a live block of the pool.
 * trim frees cached blocks, largest first, until at most keep_bytes stay cached. */
PR_API int pr_host_block(long long bytes, void** out);
PR_API int pr_host_block_release(void* block);
PR_API int pr_host_blocks_trim(long long keep_bytes);
PR_API int pr_host_blocks_stats(long long* live_bytes, long long* cached_bytes, long long* allocations,
                                long long* reuses);
/* Replaces pool_counts(tables, n_patches), view_factors.py:290-300, and the re-pooling at
 * the top of ExchangeOperator.__init__ (exchange.py:59-67): sums the counts of equal
 * (origin, receiver) pairs of an arbitrary edge list into sorted CSR rows. */
PR_API int pr_counts_from_edges(const int32_t* origin, const int32_t* receiver, const int64_t* count,
                         int64_t n_edges, int64_t n_patches, void* stream, pr_counts** out);
/* pool_counts(tables, n_patches) (view_factors.py:290-300) over a list of n_tables edge lists
 * as the reference receives them: table t is origin[t], receiver[t], count[t] of n_edges[t]
 * pairs, in host (pageable or pinned) or device memory.  The tables are copied one after the
 * other into one device edge list (pageable ones above 16 MB through pinned staging buffers)
 * and pooled there; ids outside [0, n_patches) give PR_ERR_ARG. */
PR_API int pr_counts_from_tables(const int32_t* const* origin, const int32_t* const* receiver,
                                 const int64_t* const* count, const int64_t* n_edges, int n_tables,
                                 int64_t n_patches, void* stream, pr_counts** out);
/* pool_counts (view_factors.py:290-300) of two device tables of the same patches, e.g. ray
 * sets A and B: rows merged, counts, rays per origin, rays traced and DDA steps summed. */
PR_API int pr_counts_merge(const pr_counts* a, const pr_counts* b, void* stream, pr_counts** out);
PR_API void pr_counts_destroy(pr_counts* k);

/* ---- exchange operator -------------------------------------------------------
 * Replaces ExchangeOperator.__init__, exchange.py:47-80: checks that every row
 * accounts for its rays (PR_ERR_ACCOUNTING), forms S = 0.5 (A F + F^T A) + delta A,
 * finds d > 0 with d * (S d) = A (Anderson acceleration on log d; damped
 * multiplicative iteration as fallback, exchange.py:153-197) and checks the
 * projected row closure max|F_p 1 - 1| <= 1e-10 (PR_ERR_NOT_CLOSED).  The operator
 * keeps its own reference to the counts; `counts` may be destroyed afterwards. */
PR_API int pr_operator_create(const pr_counts* counts, const int64_t* rays_per_origin,
                       const double* patch_area_m2, double support_diagonal_fraction,
                       double balance_tolerance, void* stream, pr_operator** out);
/* pr_operator_create for n_ops count tables at once (batched sweeps): each operator is
 * assembled as pr_operator_create does, then the balancing iterations of all of them run in
 * lockstep, one launch making one product of every operator still iterating.  Each out[k]
 * equals pr_operator_create of the same inputs bit for bit; out[k] is set only when every
 * operator succeeds (the first failure's status is returned). */
PR_API int pr_operator_create_batch(const pr_counts* const* counts, const int64_t* const* rays_per_origin,
                                    const double* const* patch_area_m2, int n_ops,
                                    double support_diagonal_fraction, double balance_tolerance,
                                    void* stream, pr_operator** out);
/* scale (P) f64 = ExchangeOperator.scale; the others as the attributes of the same names;
 * nnz_counts = pooled (origin, receiver) pairs, nnz_symmetric = entries of S on the union
 * pattern, spmv_calls = sparse products made with this operator so far. */
PR_API int pr_operator_info(const pr_operator* op, double* scale, int* balance_method,
                     int* balance_iterations, double* row_sum_error, int64_t* nnz_counts,
                     int64_t* nnz_symmetric, int64_t* spmv_calls);
/* y = product(x), see PR_APPLY_*. x, y: (P) f64. */
PR_API int pr_operator_apply(const pr_operator* op, int which, const double* x, double* y, void* stream);
/* ExchangeOperator.reciprocity_error(), exchange.py:124-140. */
PR_API int pr_operator_reciprocity_error(const pr_operator* op, double* out, void* stream);
/* The sampled edges with their weights n_ij / R_i (ExchangeOperator.origin, .receiver,
 * .weight, exchange.py:66-72); any pointer may be NULL. */
PR_API int pr_operator_edges(const pr_operator* op, int32_t* origin, int32_t* receiver, double* weight,
                      void* stream);
PR_API void pr_operator_destroy(pr_operator* op);

/* ---- radiosity ----------------------------------------------------------------
 * Replaces reflection_series(operator, emitted_W, emissivity, relative_tolerance=,
 * max_reflections=), exchange.py:217-245.  absorbed (P) f64; residual = sum of the
 * power still in flight; iterations = reflections summed. */
PR_API int pr_reflection_series(const pr_operator* op, const double* emitted, const double* emissivity,
                         double relative_tolerance, int64_t max_reflections, double* absorbed,
                         double* residual_power, int64_t* iterations, void* stream);
/* No counterpart in the reference.  The reflection series of pr_reflection_series for
 * callers that cannot call cudaMalloc: a host whose device memory is owned by another
 * allocator (for example a framework pool that reserves the GPU's memory up front), or
 * code that must not take the allocator's implicit synchronisation in the middle of its
 * stream work.  It allocates nothing: its scratch (two vectors, block partial sums and
 * the convergence state) is one static device array held by every GPU that loads the
 * library until the process exits (4.2 MB), sized for at most 262144 patches and for the
 * block partial sums of GPUs with up to 296 SMs (a B200 has 148); larger operators, or a
 * GPU whose launches need more partial sums, are rejected with PR_ERR_LIMIT.  emitted,
 * emissivity and absorbed must be device memory of the operator's device (PR_ERR_ARG for
 * host memory or another GPU's memory).  The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress) and should come before any stream capture.
 * Every call shares the one array: calls that overlap on the GPU (other streams, other
 * host threads) race and must be serialised by the caller. */
PR_API int pr_reflection_series_noalloc(const pr_operator* op, const double* emitted,
                                        const double* emissivity, double relative_tolerance,
                                        int64_t max_reflections, double* absorbed,
                                        double* residual_power, int64_t* iterations, void* stream);
/* Replaces net_patch_power(operator, temperature_K, emissivity, area_m2,
 * relative_tolerance=, reference_temperature_K=), exchange.py:248-271.
 * has_reference = 0 means reference_temperature_K=None.  Outputs may be NULL. */
PR_API int pr_net_patch_power(const pr_operator* op, const double* temperature_K,
                       const double* emissivity, const double* area_m2,
                       double relative_tolerance, int has_reference,
                       double reference_temperature_K, int64_t max_reflections, double* emitted,
                       double* absorbed, double* net, double* residual_power, int64_t* iterations,
                       void* stream);
/* Replaces net_patch_power_jvp(...), exchange.py:274-287.  out (P) f64. */
PR_API int pr_net_patch_power_jvp(const pr_operator* op, const double* temperature_K,
                           const double* delta_temperature_K, const double* emissivity,
                           const double* area_m2, double relative_tolerance, double* out,
                           void* stream);

/* ---- prescribed-field channels (caller of the path) -------------------------------
 * Replaces prescribed_field_channels(operator, patches, T_mean_K, delta_T_K, epsilon),
 * coupled.py:170-194: walls at T_m +/- dT/2, internal patches at the linear field of
 * their cell (coupled.py:138-143), one radiosity solve with T_ref = T_m, then
 * q[0..2] = q_h, q_c, q_i (W m^-2) and q[3] = closure_rel.  coarse (optional) =
 * 8^3 coarse source / cross-section area (coupled.py:146-153, 193), shape of
 * min(8, n) bins per axis.  precision: PR_PRECISION_*; rtol as the reference (1e-13)
 * for FP64.  stats (optional, 4 values): reflections or sweeps, SpMV calls, residual
 * power, estimated relative error of the mixed solve (0 for FP64). */
PR_API int pr_prescribed_field_channels(const pr_case* c, const pr_operator* op, double T_mean_K,
                                 double delta_T_K, double epsilon, int precision,
                                 double relative_tolerance, double* q, double* coarse,
                                 double* stats, void* stream);

/* Replaces evaluate_radiation(operator, patches, T_cells, T_hot_K, T_cold_K, epsilon,
 * relative_tolerance=, reference_temperature_K=), coupled.py:86-105, followed by the channel
 * sums of coupled.py:185-193, for an arbitrary cell temperature field: walls at T_hot_K /
 * T_cold_K, internal patches at T_cells (nx*ny*nz f64) of their owning cell.  Outputs as
 * pr_prescribed_field_channels.  The resident operator is reused across calls, as a
 * Newton-Krylov outer loop calls the radiosity at every trial field. */
PR_API int pr_cell_field_channels(const pr_case* c, const pr_operator* op, const double* T_cells,
                                  double T_hot_K, double T_cold_K, double epsilon, int has_reference,
                                  double reference_temperature_K, int precision,
                                  double relative_tolerance, double* q, double* coarse, double* stats,
                                  void* stream);

/* ---- conduction and the coupled solve (porerad/conduction.py, porerad/coupled.py) ---
 * Replaces assemble_conduction(conductivity_x, H_m), conduction.py:53-92: the
 * cell-centred finite-volume system of a conductivity field (nx*ny*nz f64, x-oriented).
 * A is held as the conductance of every cell's +x, +y, +z face (harmonic mean x dx; y, z
 * periodic; 0 on the last +x face), its diagonal and the wall responses 2 k dx. */
PR_API int pr_conduction_create(const double* conductivity, int64_t nx, int64_t ny, int64_t nz, double H_m,
                                void* stream, pr_conduction** out);
PR_API void pr_conduction_destroy(pr_conduction* conduction);
/* The stored arrays (any may be NULL): face conductances gx, gy, gz, diagonal, hot_rhs,
 * cold_rhs (ConductionSystem.hot_rhs / cold_rhs, conduction.py:25-35). */
PR_API int pr_conduction_arrays(const pr_conduction* conduction, double* gx, double* gy, double* gz, double* diag,
                                double* hot_rhs, double* cold_rhs, void* stream);
/* y = A x (ConductionSystem.matrix @ x). */
PR_API int pr_conduction_apply(const pr_conduction* conduction, const double* x, double* y, void* stream);
/* Replaces solve_conduction(system, T_hot_K, T_cold_K, rtol=), conduction.py:95-120:
 * Jacobi-PCG from the linear profile; PR_ERR_SERIES ("conduction solve did not
 * converge") unless ||A T - b|| <= 1e-9 ||b||. */
PR_API int pr_conduction_solve(const pr_conduction* conduction, double T_hot_K, double T_cold_K, double rtol,
                               double* T_out, int64_t* iterations, double* relative_residual, void* stream);
/* Replaces ConductionSystem.wall_fluxes, conduction.py:43-50. */
PR_API int pr_conduction_wall_fluxes(const pr_conduction* conduction, const double* T, double T_hot_K,
                                     double T_cold_K, double* q_hot, double* q_cold, void* stream);

#define PR_COUPLED_MAX_LINEAR 16
enum {
  PR_COUPLED_OK = 0,
  PR_COUPLED_LINEAR = 1,       /* "linear solve did not converge" */
  PR_COUPLED_LINE_SEARCH = 2,  /* "line search failed" */
  PR_COUPLED_MAX_NEWTON = 3    /* "maximum Newton iterations reached" */
};
typedef struct {
  int converged, gmres_iterations;
  double rhs_l2_W, true_residual_l2_W, true_residual_relative;
} pr_coupled_linear;
/* CoupledResult (coupled.py:314-337) of the returned attempt and the quantities of
 * wall_flux_metrics (coupled.py:443-472). */
typedef struct {
  int converged, newton_iterations, preconditioner_steps, failure, linear_residuals_pass, n_linear;
  pr_coupled_linear linear[PR_COUPLED_MAX_LINEAR];
  double final_residual_inf_W;
  double q_cond_hot_W_m2, q_rad_hot_W_m2, q_total_hot_W_m2, q_cond_cold_W_m2, q_rad_cold_W_m2, q_total_cold_W_m2;
  double radiative_fraction_hot, k_eff_apparent_W_mK, wall_flux_mismatch_rel, energy_residual_rel;
  double global_energy_residual_W, residual_power_W, T_min_K, T_max_K;
  int64_t temperature_bound_violations, series_iterations;
} pr_coupled_result;
/* Replaces solve_coupled(system, operator, patches, T_hot_K, T_cold_K, epsilon, T_initial),
 * coupled.py:423-440 (preconditioner_steps = 0: 10 steps, then 20 from the same field when
 * needed), or newton_krylov(..., preconditioner_steps), coupled.py:340-421, with
 * preconditioner_steps > 0.  Outputs (any may be NULL): the cell field (nx*ny*nz), the
 * final state's patch temperature, emitted and absorbed power (n_patches) and cell net
 * power (nx*ny*nz). */
PR_API int pr_coupled_solve(const pr_case* c, const pr_operator* op, const pr_conduction* conduction,
                            double T_hot_K, double T_cold_K, double epsilon, const double* T_initial,
                            int preconditioner_steps, double* T_out, double* patch_temperature,
                            double* patch_emitted, double* patch_absorbed, double* cell_net_power,
                            pr_coupled_result* result, void* stream);

/* ---- multi-bounce ray statistics (porerad/properties.py, porerad/penetration.py) ----
 * Rays enter the slab (the case's solid cells, x-oriented) through x = 0 at uniform
 * transverse positions, at normal incidence (properties) or with Lambertian directions
 * (penetration); at a solid surface a ray is absorbed with probability epsilon, else
 * reflected diffusely, for at most max_bounces reflections.  Restart rule of a reflected ray
 * (properties.py:14-22): */
enum { PR_RESTART_ARTICLE = 0, PR_RESTART_HIT_POINT = 1 };
typedef struct {
  int64_t events, censored, interactions, scattered;
  double event_length, censored_length, sum_mu, sum_mu2;
} pr_properties_tally;
/* Replaces the ray kernel of trace_properties(phases, axis, epsilon, n_rays=, seed=,
 * max_bounces=, restart=), properties.py:53-279: first-segment interceptions (events) and
 * right-censored crossings with their lengths in cells, surface interactions, reflections,
 * and the sums of the cosine mu between incoming and reflected directions and of mu^2. */
PR_API int pr_radiative_properties(const pr_case* c, double epsilon, int64_t n_rays, uint32_t seed, int restart,
                                   int max_bounces, pr_properties_tally* out, void* stream);
/* Replaces the ray kernel of trace_penetration(...), penetration.py:200-305: counts of rays
 * reflected (left through x = 0), transmitted (x = N), absorbed, and stopped at the
 * reflection or step limit (counts[0..3]). */
PR_API int pr_penetration(const pr_case* c, double epsilon, int64_t n_rays, uint32_t seed, int restart,
                          int max_bounces, int64_t* counts, void* stream);

/* ---- morphology descriptors ----------------------------------------------------
 * Integer counts behind the scalar and directional descriptors of porerad/descriptors.py,
 * for a uint8 phase array (nx, ny, nz) in C order (1 solid, 0 pore), on the host or the
 * device.  Always: solid and pore cells; solid/non-solid faces inside the box per normal
 * axis (interface_area, descriptors.py:38-43); pore/non-pore faces of the periodic cell
 * (interface_face_counts, descriptors.py:120-123); pore runs per axis ending at the box
 * faces (mean_pore_chords, descriptors.py:46-48: pore cells / runs).
 * PR_MORPH_CHORDS: the periodic pore chords along each axis (periodic_chords,
 * descriptors.py:82-109) as histograms chord_counts_a[0..n_a] of chord lengths (NULL skips
 * the copy), and the all-pore lines.  PR_MORPH_CONNECTIVITY: 26-connected pore clusters
 * (pore_connectivity, descriptors.py:51-60): their number, the largest, and percolation along
 * each axis.  Fields not asked for are -1.  Arrays of 2^31 - 1 cells or more: PR_ERR_LIMIT. */
enum { PR_MORPH_CHORDS = 1, PR_MORPH_CONNECTIVITY = 2 };
typedef struct {
  int64_t cells, solid_cells, pore_cells;
  int64_t interface_faces[3], periodic_faces[3], pore_runs[3], all_pore_lines[3];
  int64_t pore_clusters, largest_pore_cluster;
  int32_t pore_percolates[3];
} pr_morphology;
PR_API int pr_morphology_counts(const uint8_t* phases, int64_t nx, int64_t ny, int64_t nz, int what,
                                pr_morphology* out, int64_t* chord_counts_x, int64_t* chord_counts_y,
                                int64_t* chord_counts_z, void* stream);

/* ---- microstructure rendering ------------------------------------------------------
 * The grid work of porerad/geometry.py's generators; the random parameters, the foam graph
 * and the fiber frames are drawn on the host as the reference draws them.
 * pr_render_shapes replaces the union of shape_mask(N, center, radii, kind, R) calls
 * (geometry.py:85-121) for ellipsoids and cylinders no longer than the cell, as render_foam
 * (geometry.py:201-208) forms it: phases (device, N^3 bytes, C order) receives 1 inside any
 * shape and 0 elsewhere, evaluated cell for cell as the reference's NumPy expression is
 * (minimum-image offsets with NumPy's float remainder, R^T x as OpenBLAS's dgemm forms it).
 * pr_stamp_fibers replaces _long_cylinder (geometry.py:59-82) for n_fibers fibers: fiber f
 * marks (nodes[j] + offsets[k]) mod N for its nodes node_start[f] <= j < node_start[f+1] and
 * disk offsets offset_start[f] <= k < offset_start[f+1] (int32 triples, host or device);
 * node_start and offset_start (n_fibers + 1 entries each) are host arrays; clear = 1 zeroes
 * the array first.  solid_cells (may be NULL) receives the solid cells of the result. */
enum { PR_SHAPE_ELLIPSOID = 0, PR_SHAPE_CYLINDER = 1 };
typedef struct {
  int32_t kind;
  int32_t pad;
  double center[3];
  double R[9];     /* rotation, row-major; local axis i is column i */
  double radii[3]; /* r_x, r_y, r_z (a cylinder's half length) */
} pr_shape;
PR_API int pr_render_shapes(int64_t N, const pr_shape* shapes, int n_shapes, uint8_t* phases, int64_t* solid_cells,
                            void* stream);
PR_API int pr_stamp_fibers(int64_t N, const int32_t* nodes, const int64_t* node_start, const int32_t* offsets,
                           const int64_t* offset_start, int n_fibers, int clear, uint8_t* phases,
                           int64_t* solid_cells, void* stream);

/* Replaces the grid work of lamellar_field (geometry.py:223-239): field (device, N^3 f64) =
 * base_x[i] + 0.35 sin(two_pi_layers (i + wav[j,k]) / N) + smoothed noise, wav[j,k] = waviness
 * (0.65 sin_y[j] + 0.35 cos_z[k]); the 7-point periodic smoothing of noise (N^3 f64, host or
 * device, the reference's normal draws) is summed in the reference's order and divided by 7;
 * the sine is correctly rounded.  base_x, sin_y, cos_z: the N values the reference's cosine and
 * sines take along each axis, computed on the host. */
PR_API int pr_lamellar_field(int64_t N, const double* base_x, const double* sin_y, const double* cos_z,
                             double waviness, double two_pi_layers, const double* noise, double* field,
                             void* stream);
/* pr_stamp_fibers with any byte value (value 0 punches holes): the device work of the
 * benchmark archetypes' segment and hole stamping as well. */
PR_API int pr_stamp_cells(int64_t N, const int32_t* nodes, const int64_t* node_start, const int32_t* offsets,
                          const int64_t* offset_start, int n_groups, int clear, int value, uint8_t* phases,
                          int64_t* solid_cells, void* stream);

/* ---- benchmark archetypes (no counterpart in the reference) -------------------------
 * The grid work of porerad_b200.geometry's seeded archetypes, bit-identical to their host
 * definitions.  pr_voronoi_edge_field: field (device, N^3 f64) = d3 - d1, the distances from
 * each cell centre to its first and third nearest of n_seeds periodic points (seeds: n_seeds x 3
 * f64, host or device), as SciPy's periodic k-d tree computes them.  pr_quantile_threshold:
 * q = numpy.quantile(field, quantile) and phases = field <= q (below = 1) or field >= q; q_out
 * and solid_cells may be NULL. */
PR_API int pr_voronoi_edge_field(int64_t N, const double* seeds, int n_seeds, double* field, void* stream);
/* The archetypes' loops "add a fiber until the solid fraction is reached" and "punch a hole
 * until it falls to the target" in batches: pr_stamp_first stamps n_fibers (<= 1024) shapes at
 * once (shape f: nodes[node_start[f] .. node_start[f+1]), int32 triples, thickened by the shared
 * offsets), keeping in first (device, N^3 int32, initialised by the caller to INT32_MAX) the
 * smallest index base + f of a shape covering each cell, and returns in new_cells[f] (host) the
 * cells shape base + f covers first, counting only cells where mask (device, may be NULL) is 1.
 * pr_first_threshold: mode 0 writes phases = first <= last, mode 1 clears the cells with
 * first <= last.  node_start and new_cells are host arrays. */
PR_API int pr_stamp_first(int64_t N, const int32_t* nodes, const int64_t* node_start, const int32_t* offsets,
                          int64_t n_offsets, int n_fibers, int base, int32_t* first, const uint8_t* mask,
                          int64_t* new_cells, void* stream);
PR_API int pr_first_threshold(const int32_t* first, int64_t n, int last, int mode, uint8_t* phases, void* stream);
PR_API int pr_quantile_threshold(const double* field, int64_t n, double quantile, int below, uint8_t* phases,
                                 double* q_out, int64_t* solid_cells, void* stream);

/* ---- instrumentation (no counterpart in the reference) ----------------------------
 * Kernel classes timed with CUDA events on their launching stream while enabled:
 * 0 fused ray generation + traversal, 1 per-patch count reduction, 2 balancing
 * product, 3 reflection-series product, 4 binary32 Chebyshev sweep, 5 binary64
 * refinement residual, 6 morphology counts (one pass over the phase array), 7 pore cluster
 * labelling (union-find, sizes, summary), 8 microstructure rendering (shapes or fibers). */
PR_API void pr_timers_enable(int on);
PR_API void pr_timers_reset(void);
PR_API int pr_timers_read(int kernel_class, long long* launches, double* total_ms);
/* Traversal autotuning (no counterpart in the reference): the fused traversal has several
 * compiled variants (registers per thread, DDA steps between lane refills); by default the
 * first count pass of a problem class (grid size, rays per origin) times each on its first
 * chunk and keeps the fastest.  Results do not depend on the variant. */
PR_API int pr_trace_set_variant(int variant);  /* -1 = autotune (default) */
PR_API int pr_trace_variant_info(int* count, int* last_used, const char** name);
/* Number of the library's own kernel launches so far (CUB primitives not counted). */
PR_API long long pr_kernel_launches(void);

/* ---- device memory (no counterpart in the reference) ------------------------------
 * Library objects allocate through a per-device cache of freed blocks (size classes
 * within 12.5 %, reuse ordered after the block's last use by an in-stream event wait),
 * bounded by PORERAD_CACHE_BYTES (default a quarter of the device memory).  Stats: bytes
 * cached, bytes live in library objects, driver allocations, allocations served from the
 * cache.  release_cached returns every cached block of the device to the driver. */
PR_API int pr_memory_stats(int device, long long* cached_bytes, long long* live_bytes, long long* device_mallocs,
                           long long* cache_hits);
PR_API int pr_memory_release_cached(int device);

#ifdef __cplusplus
}
#endif

#endif /* PORERAD_H */
