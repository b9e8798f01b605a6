/* ddcb.h -- C-ABI of the B200 batched spline builder / evaluator.
 *
 * This is the drop-in boundary for DDC's batched spline hot path (CExA-project/ddc v0.15.1,
 * src/ddc/kernels/splines/). Every entry point names the reference interface it replaces. The ABI
 * carries plain pointers, sizes and strides only: device pointers for the batched data (the
 * reference's ChunkSpans live in a Kokkos memory space), host pointers for mesh descriptions.
 *
 * Conventions
 *  - Every function returns a ddcb_status; no C++ exception crosses the ABI. The text of the last
 *    failure on the calling thread is returned by ddcb_last_error_message().
 *  - Batched arrays are described by ddcb_lines: element (i, b) of line b is at
 *        base[i*stride + (b / inner)*outer_stride + (b % inner)]
 *    i.e. the dimension of interest has element stride `stride` and the batch dimensions are
 *    flattened into (outer, inner) with the inner part contiguous. This covers every
 *    layout_right dimension order of the reference's batched domains (interest dimension first,
 *    middle or last, tests/splines/batched_spline_builder.cpp:393-515).
 *  - Work is stream ordered on the ddcb_stream given (a cudaStream_t; NULL = legacy default).
 *  - Plans (bases, builders, evaluators) are immutable after creation; calls on different streams
 *    may run concurrently.
 */
#ifndef DDCB_H
#define DDCB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* cudaStream_t without requiring the CUDA headers. */
typedef struct CUstream_st* ddcb_stream;

typedef enum ddcb_status {
    DDCB_SUCCESS = 0,
    DDCB_ERR_INVALID_ARGUMENT = 1, /* bad pointer, size, layout or enum */
    DDCB_ERR_BAD_GRID = 2,         /* spline_builder.hpp:1244-1317 check_valid_grid failures */
    DDCB_ERR_SINGULAR = 3,         /* a factorisation met a zero / non-positive pivot (LAPACK info != 0) */
    DDCB_ERR_CUDA = 4,             /* a CUDA runtime call failed */
    DDCB_ERR_UNSUPPORTED = 5,      /* valid request outside this implementation's limits */
    DDCB_ERR_NOT_CONVERGED = 6,    /* iterative refinement did not reach its tolerance */
    DDCB_ERR_DEVICE = 7            /* a kernel reported a failure through its status word */
} ddcb_status;

/* ddc::SplineBuilderClosure (spline_builder_closures.hpp:18-23). */
typedef enum ddcb_closure {
    DDCB_PERIODIC = 0,
    DDCB_HERMITE = 1,
    DDCB_HOMOGENEOUS_HERMITE = 2,
    DDCB_GREVILLE = 3
} ddcb_closure;

/* The evaluator's extrapolation rules: PeriodicExtrapolationRule, NullExtrapolationRule,
 * ConstantExtrapolationRule (periodic_/null_/constant_extrapolation_rule.hpp). */
typedef enum ddcb_extrapolation {
    DDCB_EXTRAP_PERIODIC = 0,
    DDCB_EXTRAP_NULL = 1,
    DDCB_EXTRAP_CONSTANT = 2
} ddcb_extrapolation;

/* Arithmetic of the batched solves. FP64 is the drop-in (the reference's SplineSolver::LAPACK
 * arithmetic). FP32_REFINE solves in FP32 and refines with FP64 residuals; inputs and outputs stay
 * FP64. */
typedef enum ddcb_precision { DDCB_FP64 = 0, DDCB_FP32_REFINE = 1 } ddcb_precision;

typedef struct ddcb_lines {
    int64_t n;            /* extent along the dimension of interest */
    int64_t stride;       /* element stride along the dimension of interest */
    int64_t inner;        /* lines that are contiguous in memory (unit stride) */
    int64_t outer;        /* groups of `inner` lines */
    int64_t outer_stride; /* element stride between groups */
} ddcb_lines;

typedef struct ddcb_bsplines_t* ddcb_bsplines;
typedef struct ddcb_builder_t* ddcb_builder;
typedef struct ddcb_evaluator_t* ddcb_evaluator;

typedef struct ddcb_bsplines_info {
    int32_t degree, periodic, uniform;
    int64_t ncells, nbasis, size; /* nbasis(), size() of bsplines_uniform.hpp:309-354 */
    double rmin, rmax;
} ddcb_bsplines_info;

typedef struct ddcb_builder_options {
    int32_t precision;       /* ddcb_precision */
    int32_t refine_rounds;   /* FP32_REFINE: refinement rounds (1..3; 0 = 2) */
    int32_t tile_lines;      /* 0 = automatic: lines per thread block */
    int32_t chunks;          /* 0 = automatic: chunk threads per line */
    double refine_tolerance; /* FP32_REFINE: bound on the estimated relative error of a refined line,
                                ||A^-1||_inf max|b - A x| / max|x| after the last round, checked on
                                the device (0 = 1e-12); see ddcb_builder_device_status */
} ddcb_builder_options;

typedef struct ddcb_builder_info {
    int64_t nbasis, size, npoints;
    int32_t nbe_lo, nbe_hi, nbv_lo, nbv_hi; /* s_nbe_xmin/xmax, s_nbv_xmin/xmax (spline_builder.hpp:166-191) */
    int32_t offset;                         /* m_offset (spline_builder.hpp:201, 619-658) */
    double dx;                              /* m_dx (spline_builder.hpp:233-234) */
    int32_t border, kl, ku, pivoting, chunks, tile_lines; /* structure of the device solve */
} ddcb_builder_info;

/* ---- status ---------------------------------------------------------------------------- */
const char* ddcb_status_string(ddcb_status s);
const char* ddcb_last_error_message(void);
/* Device-side failures of the work queued on `stream` so far (the reference's debug builds
 * assert the same index ranges with KOKKOS_ASSERT,
 * bsplines_uniform.hpp:489-494, bsplines_non_uniform.hpp:469-479): waits for the stream; returns
 * DDCB_ERR_CUDA if a kernel failed, and, in the bounds-checked build (libddcb_check.so, built with
 * -DDDCB_CHECK_BOUNDS), DDCB_ERR_DEVICE for the first computed index (cell, knot pair, tile row)
 * that a kernel found outside its array since the previous call -- file, line, index and bound in
 * ddcb_last_error_message(); the kernel went on with the index clamped into range. Refinement
 * convergence is reported per builder by ddcb_builder_device_status. */
ddcb_status ddcb_last_device_error(ddcb_stream stream);
/* 1 in the bounds-checked build, 0 in the default one. */
int32_t ddcb_bounds_checked(void);

/* ---- basis: UniformBSplines<CDim,D>::Impl(rmin, rmax, ncells) (bsplines_uniform.hpp:145-155)
 *      and NonUniformBSplines<CDim,D>::Impl(breaks) (bsplines_non_uniform.hpp:414-457). ------- */
ddcb_status ddcb_bsplines_create_uniform(int32_t degree, int32_t periodic, double rmin, double rmax,
                                         int64_t ncells, ddcb_bsplines* out);
ddcb_status ddcb_bsplines_create_non_uniform(int32_t degree, int32_t periodic, const double* breaks,
                                             int64_t nbreaks, ddcb_bsplines* out);
ddcb_status ddcb_bsplines_destroy(ddcb_bsplines b);
ddcb_status ddcb_bsplines_get_info(ddcb_bsplines b, ddcb_bsplines_info* info);
/* Knot coordinates (ddc::coordinate of the knot elements), `count` from index `first`. */
ddcb_status ddcb_bsplines_knots(ddcb_bsplines b, int64_t first, int64_t count, double* out);
/* GrevilleInterpolationPoints<BSplines, lo, hi>::get_sampling / get_domain
 * (greville_interpolation_points.hpp:47-296): writes the interpolation points. */
ddcb_status ddcb_greville_points(ddcb_bsplines b, ddcb_closure lo, ddcb_closure hi, double* points,
                                 int64_t capacity, int64_t* npoints);
/* integrals(execution_space, int_vals) (integrals.hpp:165-177), host output of size() entries. */
ddcb_status ddcb_bsplines_integrals(ddcb_bsplines b, double* out);

/* ---- builder: SplineBuilder<..., SplineSolver> constructor (spline_builder.hpp:227-260):
 *      check_valid_grid, compute_offset, allocate_matrix / build_matrix_system / setup_solver,
 *      with the device plan created on the current CUDA device. ------------------------------ */
ddcb_status ddcb_builder_create(ddcb_bsplines basis, const double* interp_points, int64_t npoints,
                                ddcb_closure lo, ddcb_closure hi, const ddcb_builder_options* options,
                                ddcb_builder* out);
ddcb_status ddcb_builder_destroy(ddcb_builder b);
ddcb_status ddcb_builder_get_info(ddcb_builder b, ddcb_builder_info* info);
/* The outcome of the device-side checks of this builder's work queued so far on `stream`: waits for
 * the stream, returns DDCB_ERR_NOT_CONVERGED if a FP32_REFINE solve ended above refine_tolerance
 * since the previous query (the reference reports non-convergence of its iterative solver,
 * splines_linear_problem_sparse.cpp:272-275), else DDCB_SUCCESS; the flag is then cleared. */
ddcb_status ddcb_builder_device_status(ddcb_builder b, ddcb_stream stream);
/* SplineBuilder::operator()(spline, vals, derivs_xmin, derivs_xmax) (spline_builder.hpp:538-557,
 * 896-1101). derivs_* are ignored (may be NULL) unless the closure is HERMITE; their layout's n is
 * s_nbv (derivative orders odd..odd+nbv-1, unscaled). */
ddcb_status ddcb_build(ddcb_builder b, double* coefs, ddcb_lines coefs_layout, const double* vals,
                       ddcb_lines vals_layout, const double* derivs_lo, ddcb_lines derivs_lo_layout,
                       const double* derivs_hi, ddcb_lines derivs_hi_layout, ddcb_stream stream);
/* SplinesLinearProblem::solve(MultiRHS b, bool transpose) (splines_linear_problem.hpp:80-92):
 * in-place solve of A x = b (or A^T x = b) for nrhs columns of a (nbasis x nrhs) row-major device
 * array with leading dimension ld (>= nrhs). */
ddcb_status ddcb_solve_multirhs(ddcb_builder b, double* rhs, int64_t ld, int64_t nrhs, int32_t transpose,
                                ddcb_stream stream);
/* SplineBuilder::quadrature_coefficients() (spline_builder.hpp:1103-1234), host outputs of
 * nbv_lo, nbasis - nbv_lo - nbv_hi and nbv_hi entries; the Hermite parts are scaled by dx^k. The
 * weights solve A^T q = integrals with the device's transposed solve, on the builder's first
 * quadrature or ddcb_integrate_samples call (synchronously, once); this call copies them out
 * (synchronously). */
ddcb_status ddcb_quadrature_coefficients(ddcb_builder b, double* q_derivs_lo, double* q_vals, double* q_derivs_hi);
/* The same weights as one device array of nbasis entries, [q_derivs_lo, q_vals, q_derivs_hi],
 * copied stream-ordered into q_all (a device pointer): quadrature_coefficients<OutMemorySpace>()
 * with a device memory space. */
ddcb_status ddcb_quadrature_coefficients_device(ddcb_builder b, double* q_all, ddcb_stream stream);
/* SplineBuilder::operator() followed by SplineEvaluator::integrate (spline_evaluator.hpp:493-526)
 * on the same lines, fused: out[(b / inner)*out_outer_stride + b % inner] is the integral of the
 * spline interpolating line b's samples (and Hermite derivatives, read as in ddcb_build), computed
 * as the dot product of the samples with the quadrature weights -- one read of the samples, no
 * coefficient array. */
ddcb_status ddcb_integrate_samples(ddcb_builder b, double* out, int64_t out_outer_stride, const double* vals,
                                   ddcb_lines vals_layout, const double* derivs_lo, ddcb_lines derivs_lo_layout,
                                   const double* derivs_hi, ddcb_lines derivs_hi_layout, ddcb_stream stream);

/* ---- evaluator: SplineEvaluator<..., LowerExtrapolationRule, UpperExtrapolationRule>
 *      (spline_evaluator.hpp:160-186). ------------------------------------------------------- */
ddcb_status ddcb_evaluator_create(ddcb_bsplines basis, ddcb_extrapolation lo, ddcb_extrapolation hi,
                                  ddcb_evaluator* out);
ddcb_status ddcb_evaluator_destroy(ddcb_evaluator e);
/* SplineEvaluator::operator()(spline_eval, coords_eval, spline_coef) (spline_evaluator.hpp:257-294). */
ddcb_status ddcb_eval(ddcb_evaluator e, double* out, ddcb_lines out_layout, const double* coords,
                      ddcb_lines coords_layout, const double* coefs, ddcb_lines coefs_layout, ddcb_stream stream);
/* SplineEvaluator::deriv(deriv_order, spline_eval, coords_eval, spline_coef)
 * (spline_evaluator.hpp:388-430); order in 1..degree, no boundary handling (eval_no_bc). */
ddcb_status ddcb_eval_deriv(ddcb_evaluator e, int32_t order, double* out, ddcb_lines out_layout,
                            const double* coords, ddcb_lines coords_layout, const double* coefs,
                            ddcb_lines coefs_layout, ddcb_stream stream);
/* SplineEvaluator::integrate(integrals, spline_coef) (spline_evaluator.hpp:493-526): one value per
 * line, out[(b / inner)*out_outer_stride + b % inner] with the coefficient layout's batch shape. */
ddcb_status ddcb_integrate(ddcb_evaluator e, double* out, int64_t out_outer_stride, const double* coefs,
                           ddcb_lines coefs_layout, ddcb_stream stream);

/* ---- fused step: SplineBuilder::operator() followed by SplineEvaluator::operator() (order 0)
 *      or SplineEvaluator::deriv (order >= 1) on the same lines -- the semi-Lagrangian step of
 *      examples/characteristics_advection.cpp:251-259. Writes both the coefficients and the
 *      evaluated values; *fused (may be NULL) tells whether one kernel did both. ---------------- */
ddcb_status ddcb_build_eval(ddcb_builder b, ddcb_evaluator e, int32_t order, double* coefs, ddcb_lines coefs_layout,
                            const double* vals, ddcb_lines vals_layout, const double* derivs_lo,
                            ddcb_lines derivs_lo_layout, const double* derivs_hi, ddcb_lines derivs_hi_layout,
                            const double* coords, ddcb_lines coords_layout, double* out, ddcb_lines out_layout,
                            int32_t* fused, ddcb_stream stream);

/* ---- one semi-Lagrangian advection step (examples/characteristics_advection.cpp:243-259): the
 *      feet of the characteristics through the interpolation points, x_q - dt * v, the splines of
 *      the lines (SplineBuilder::operator()) and their values at the feet (SplineEvaluator::operator(),
 *      with the evaluator's periodic wrap or extrapolation rules), written to out at the
 *      interpolation points (out's n is the builder's npoints). The velocity of line b is
 *      velocity[b / velocity_div] (a device array; velocity_div = 1: one value per line, inner:
 *      one per group of inner lines), or velocity_const when velocity is NULL. coefs (may be NULL)
 *      receives the coefficients. On uniform bases one kernel does the whole step and the feet are
 *      computed in it (no coordinate array is read); *fused (may be NULL) tells whether it ran. - */
ddcb_status ddcb_advect(ddcb_builder b, ddcb_evaluator e, double dt, const double* velocity, int64_t velocity_div,
                        double velocity_const, double* out, ddcb_lines out_layout, const double* vals,
                        ddcb_lines vals_layout, const double* derivs_lo, ddcb_lines derivs_lo_layout,
                        const double* derivs_hi, ddcb_lines derivs_hi_layout, double* coefs, ddcb_lines coefs_layout,
                        int32_t* fused, ddcb_stream stream);

/* ---- reverse mode (no reference counterpart: the reference has no derivatives with respect to
 *      its inputs). The builder is linear, coefs = P A^-1 R (vals, dx^k derivs); the evaluator is
 *      y = sum_i c[jmin+i] B_i(x). Every cotangent output is overwritten, not accumulated. ---- */
/* Adjoint of ddcb_build: g_vals = R^T A^-T P^T g_coefs, with the cotangents of the periodic
 * duplicate coefficients folded back (spline_builder.hpp:1073-1100) and the transposed solve of
 * SplinesLinearProblem::solve(b, true) (splines_linear_problem.hpp:80-92). g_derivs_lo/hi (nbv_lo,
 * nbv_hi rows) receive the cotangents of the Hermite derivatives; either may be NULL. */
ddcb_status ddcb_build_adjoint(ddcb_builder b, const double* g_coefs, ddcb_lines g_coefs_layout, double* g_vals,
                               ddcb_lines g_vals_layout, double* g_derivs_lo, ddcb_lines g_derivs_lo_layout,
                               double* g_derivs_hi, ddcb_lines g_derivs_hi_layout, ddcb_stream stream);
/* Adjoint of ddcb_eval (order 0) / ddcb_eval_deriv (order 1): g_coefs[jmin+i] = sum over the
 * line's points of g_out * d out / d c[jmin+i], and g_coords = g_out * d out / dx (the spline
 * derivative of order + 1; 0 outside the domain where the extrapolation rule is constant or null).
 * coefs is read only for g_coords, which may be NULL (then coefs may be NULL too). */
ddcb_status ddcb_eval_adjoint(ddcb_evaluator e, int32_t order, const double* coords, ddcb_lines coords_layout,
                              const double* coefs, ddcb_lines coefs_layout, const double* g_out, ddcb_lines g_out_layout,
                              double* g_coefs, ddcb_lines g_coefs_layout, double* g_coords, ddcb_lines g_coords_layout,
                              ddcb_stream stream);
/* Backward of ddcb_build_eval: the evaluator adjoint scattered straight into the transposed solve
 * of the builder adjoint, so g_coefs never reaches memory. g_vals, g_derivs_lo/hi as in
 * ddcb_build_adjoint, g_coords as in ddcb_eval_adjoint; *fused (may be NULL) tells whether one
 * kernel did both. */
ddcb_status ddcb_build_eval_adjoint(ddcb_builder b, ddcb_evaluator e, int32_t order, const double* coords,
                                    ddcb_lines coords_layout, const double* coefs, ddcb_lines coefs_layout,
                                    const double* g_out, ddcb_lines g_out_layout, double* g_vals,
                                    ddcb_lines g_vals_layout, double* g_derivs_lo, ddcb_lines g_derivs_lo_layout,
                                    double* g_derivs_hi, ddcb_lines g_derivs_hi_layout, double* g_coords,
                                    ddcb_lines g_coords_layout, int32_t* fused, ddcb_stream stream);

/* ---- uneven batch: many independent one-line problems (each its own builder and evaluator:
 *      size, degree, closure and mesh may all differ) built and evaluated in one CUDA graph
 *      launch: per group of problems (band shape, arithmetic, block size) a build kernel with a
 *      block per problem, then an evaluation kernel over the group's points (no reference
 *      counterpart: the reference loops one SplineBuilder per problem). A builder solves fastest
 *      here when its chunk count fills whole warps (32 chunks per warp). The builders and
 *      evaluators must outlive the batch; each solves in its own
 *      precision (FP64, or FP32 with refinement, whose convergence ddcb_builder_device_status
 *      reports per builder). Data are packed: problem i's samples at
 *      vals[vals_off[i] .. vals_off[i+1]), its Hermite derivatives likewise in derivs_lo /
 *      derivs_hi, its coefficients in coefs, and its evaluation coordinates / values in coords /
 *      out at [evals_off[i] .. evals_off[i+1]). */
typedef struct ddcb_uneven_batch_t* ddcb_uneven_batch;
typedef struct ddcb_uneven_info {
    int64_t count, total_vals, total_derivs_lo, total_derivs_hi, total_coefs, total_evals;
    /* the schedule in use: threads = block size of the block schedule; blocks_per_sm = per-SM
     * budget in units of 256 threads (0: as many blocks as fit); order 0: largest first */
    int32_t threads, blocks_per_sm, order, shared_bytes;
    double tuned_us;       /* the tuner's best time (0: not tuned) */
    int32_t warp_schedule; /* 1: each problem's block has one thread per chunk of its plan, whole
                              warps (a warp per problem of <= 32 chunks); 0: every block `threads` */
} ddcb_uneven_info;
ddcb_status ddcb_batch_uneven_create(const ddcb_builder* builders, const ddcb_evaluator* evaluators,
                                     const int64_t* nevals, int64_t count, ddcb_uneven_batch* out);
ddcb_status ddcb_batch_uneven_destroy(ddcb_uneven_batch b);
ddcb_status ddcb_batch_uneven_get_info(ddcb_uneven_batch b, ddcb_uneven_info* info);
/* Prefix sums (count + 1 entries each; any pointer may be NULL). */
ddcb_status ddcb_batch_uneven_offsets(ddcb_uneven_batch b, int64_t* vals_off, int64_t* derivs_lo_off,
                                      int64_t* derivs_hi_off, int64_t* coefs_off, int64_t* evals_off);
/* Times the candidate schedules (warp or block schedule, block size, per-SM budget, queue order),
 * `reps` launches each, on these buffers and keeps the fastest for later runs. Overwrites coefs and
 * out. */
ddcb_status ddcb_batch_uneven_tune(ddcb_uneven_batch b, const double* vals, const double* derivs_lo,
                                   const double* derivs_hi, double* coefs, const double* coords, double* out,
                                   int32_t reps, ddcb_stream stream);
/* Builds every problem and evaluates it at its coordinates (values, with its evaluator's boundary
 * handling) in one graph launch. */
ddcb_status ddcb_batch_uneven_run(ddcb_uneven_batch b, const double* vals, const double* derivs_lo,
                                  const double* derivs_hi, double* coefs, const double* coords, double* out,
                                  ddcb_stream stream);

/* ---- host pipeline: ddcb_build_eval on HOST arrays. Where a DDC user copies host data to the
 *      device (ddc::parallel_deepcopy), builds and evaluates (examples/characteristics_advection.cpp:
 *      251-259) and copies the result back one step after the other, the pipeline cuts the batch
 *      into slices of `slice_lines` lines and overlaps the copy-in of slice i+1 and the copy-out of
 *      slice i-1 with the kernels of slice i (three streams, two device buffer sets, allocated at
 *      creation). Host layouts are ddcb_lines with outer == 1 (rows of the batch, row stride >=
 *      inner) or inner == 1 and stride == 1 (one contiguous line per batch index). Page-locked
 *      host memory lets the copies run asynchronously. ------------------------------------------ */
typedef struct ddcb_host_pipeline_t* ddcb_host_pipeline;
/* order: 0 evaluates values (with the evaluator's boundary handling), k >= 1 the k-th derivative;
 * npoints: evaluation points per line (coordinate layouts must have n == npoints). */
ddcb_status ddcb_host_pipeline_create(ddcb_builder b, ddcb_evaluator e, int32_t order, int64_t npoints,
                                      int64_t slice_lines, ddcb_host_pipeline* out);
ddcb_status ddcb_host_pipeline_destroy(ddcb_host_pipeline p);
/* Runs the step on host arrays; ordered after the work queued on `stream`, and `stream` waits
 * for the last copy-out, so synchronizing it makes `out` (and `coefs`, which may be NULL) ready.
 * derivs_lo / derivs_hi are read as in ddcb_build. Successive runs of one pipeline are ordered on
 * the device by its own events; calls from several host threads on one pipeline must not overlap
 * in time (use one pipeline per thread). */
ddcb_status ddcb_host_pipeline_run(ddcb_host_pipeline p, const double* vals, ddcb_lines vals_layout,
                                   const double* derivs_lo, ddcb_lines derivs_lo_layout, const double* derivs_hi,
                                   ddcb_lines derivs_hi_layout, const double* coords, ddcb_lines coords_layout,
                                   double* out, ddcb_lines out_layout, double* coefs, ddcb_lines coefs_layout,
                                   ddcb_stream stream);

/* ---- 2D tensor product: SplineBuilder2D / SplineEvaluator2D on two 1D plans, for the layout
 *      (x1, x2, batch) with the batch contiguous (the reference's layout_right of
 *      DiscreteDomain<X1, X2, batch...>). ----------------------------------------------------- */
/* Workspace of ddcb_build2d: the x1-pass result of one group of fields. */
ddcb_status ddcb_build2d_workspace_bytes(ddcb_builder b1, ddcb_builder b2, int64_t nbatch, uint64_t* bytes);
/* SplineBuilder2D::operator() (spline_builder_2d.hpp:455-651).
 *   vals (np1, np2, nbatch) -> coefs (size1, size2, nbatch);
 *   derivs_min1 / derivs_max1: (nbv1, np2, nbatch), read when b1's closure is HERMITE;
 *   derivs_min2 / derivs_max2: (np1, nbv2, nbatch), read when b2's closure is HERMITE;
 *   mixed_* (nbv1, nbv2, nbatch): cross derivatives at the four corners, read when both are HERMITE.
 * workspace: ddcb_build2d_workspace_bytes bytes of device memory, or NULL to have the call
 * allocate it stream-ordered (cudaMallocAsync / cudaFreeAsync on `stream`). With Hermite
 * derivatives in dimension 2 the short derivative-slab passes run on a second stream of the
 * calling host thread, forked from and joined back to `stream` with events: the work stays ordered
 * on `stream`, and a capture of `stream` takes the fork and the join in. */
ddcb_status ddcb_build2d(ddcb_builder b1, ddcb_builder b2, double* coefs, const double* vals, const double* derivs_min1,
                         const double* derivs_max1, const double* derivs_min2, const double* derivs_max2,
                         const double* mixed_min1_min2, const double* mixed_max1_min2, const double* mixed_min1_max2,
                         const double* mixed_max1_max2, int64_t nbatch, void* workspace, uint64_t workspace_bytes,
                         ddcb_stream stream);
/* 2D build that allocates nothing. No counterpart in the reference: this is an addition for callers
 * that must not allocate device memory at call time -- code running where cudaMalloc is not
 * allowed or not wanted (for instance inside a memory pool's budget, a real-time loop, or a host
 * framework that owns all device memory), which also cannot hand over a workspace.
 * Same arguments and results as ddcb_build2d with workspace == NULL, but the scratch of the x1 pass
 * is a fixed array of 48 MiB (50331648 bytes) inside the library's device image, present on every
 * GPU that loads the library until the process exits. The fields run in groups small enough for
 * the array; a build whose scratch exceeds it even with one field per group is rejected with
 * DDCB_ERR_UNSUPPORTED. The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress, once per device, kept for the life of the process: a device reset
 * between calls is not supported); make that first call before any stream capture (a first call
 * under capture is refused with DDCB_ERR_INVALID_ARGUMENT). All calls share the one array: calls
 * whose work overlaps on the GPU (other streams, other host threads) race on it and must be
 * ordered by the caller. The scratch needs no clearing: every value is written before it is read. */
ddcb_status ddcb_build2d_static_scratch(ddcb_builder b1, ddcb_builder b2, double* coefs, const double* vals,
                                        const double* derivs_min1, const double* derivs_max1, const double* derivs_min2,
                                        const double* derivs_max2, const double* mixed_min1_min2,
                                        const double* mixed_max1_min2, const double* mixed_min1_max2,
                                        const double* mixed_max1_max2, int64_t nbatch, ddcb_stream stream);
/* SplineEvaluator2D::operator() (order1 = order2 = 0, with the periodic wraps / extrapolation rules)
 * and deriv_dim_1 / deriv_dim_2 / deriv_1_and_2 (orders 0 or 1, no boundary handling)
 * (spline_evaluator_2d.hpp:376-598): coords (npoints, nbatch) pairs (x1, x2) -> out (npoints, nbatch);
 * coefs (size1, size2, nbatch). */
ddcb_status ddcb_eval2d(ddcb_evaluator e1, ddcb_evaluator e2, int32_t order1, int32_t order2, double* out,
                        const double* coords, const double* coefs, int64_t npoints, int64_t nbatch, ddcb_stream stream);
/* SplineEvaluator2D::integrate (spline_evaluator_2d.hpp:616-660): out[b] = sum c(r1, r2, b) I1[r1] I2[r2]. */
ddcb_status ddcb_integrate2d(ddcb_evaluator e1, ddcb_evaluator e2, double* out, const double* coefs, int64_t nbatch,
                             ddcb_stream stream);

/* ---- 3D tensor product: SplineBuilder3D (spline_builder_3d.hpp:597-1126) on three 1D plans, for
 *      the layout (x1, x2, x3, batch) with the batch contiguous. ------------------------------ */
/* Workspace of ddcb_build3d: the results of the dimension-1 and dimension-2 passes. */
ddcb_status ddcb_build3d_workspace_bytes(ddcb_builder b1, ddcb_builder b2, ddcb_builder b3, int64_t nbatch,
                                         uint64_t* bytes);
/* SplineBuilder3D::operator() (spline_builder_3d.hpp:934-1126): vals (np1, np2, np3, nbatch) ->
 * coefs (size1, size2, size3, nbatch). inputs holds 27 pointers; inputs[k1 + 3*k2 + 9*k3] is the
 * array whose dimension d holds values (k_d = 0, np_d rows), lower derivatives (k_d = 1, nbv_lo_d
 * rows) or upper derivatives (k_d = 2, nbv_hi_d rows), shape (rows1, rows2, rows3, nbatch). So
 * inputs[0] = vals, [1] / [2] = derivs_min1 / derivs_max1, [3] / [6] = derivs_min2 / derivs_max2,
 * [9] / [18] = derivs_min3 / derivs_max3, [4] = mixed_derivs_min1_min2, [5] = max1_min2,
 * [7] = min1_max2, [8] = max1_max2, [10] = min1_min3, [11] = max1_min3, [19] = min1_max3,
 * [20] = max1_max3, [12] = min2_min3, [15] = max2_min3, [21] = min2_max3, [24] = max2_max3, and
 * [13] = min1_min2_min3, [14], [16], [17], [22], [23], [25], [26] the other corners likewise. An
 * array is read only when every dimension with a derivative kind has a HERMITE closure on that
 * side (the others may be NULL). workspace: ddcb_build3d_workspace_bytes bytes of device memory,
 * or NULL to have the call allocate it stream-ordered. The dimension-1 derivative-slab passes
 * run on a second stream of the calling thread, forked and joined as in ddcb_build2d. */
ddcb_status ddcb_build3d(ddcb_builder b1, ddcb_builder b2, ddcb_builder b3, double* coefs, const double* const* inputs,
                         int64_t nbatch, void* workspace, uint64_t workspace_bytes, ddcb_stream stream);

/* ---- N-dimensional evaluation: SplineEvaluatorND (spline_evaluator_nd.hpp:306-590) and, with
 *      ndims = 3, SplineEvaluator3D (spline_evaluator_3d.hpp), over ndims (1..6) 1D evaluators;
 *      coefs (size_1, ..., size_N, nbatch), coords (npoints, nbatch, ndims), out (npoints, nbatch). */
/* orders == NULL: operator() -- periodic wraps, then the extrapolation rule of the first
 * non-periodic dimension outside its domain (null: 0; constant: the value at that boundary with
 * the other non-periodic coordinates clamped into their domains); else deriv(orders) with
 * orders[d] in 0..degree_d and no boundary handling (eval_no_bc, spline_evaluator_nd.hpp:766-825). */
ddcb_status ddcb_evalnd(const ddcb_evaluator* evaluators, int32_t ndims, const int32_t* orders, double* out,
                        const double* coords, const double* coefs, int64_t npoints, int64_t nbatch, ddcb_stream stream);
/* SplineEvaluatorND::integrate (spline_evaluator_nd.hpp:596-633): out[b] = sum over the coefficient
 * grid of c(i_1, ..., i_N, b) prod_d integral(B_{i_d}). */
ddcb_status ddcb_integratend(const ddcb_evaluator* evaluators, int32_t ndims, double* out, const double* coefs,
                             int64_t nbatch, ddcb_stream stream);

#ifdef __cplusplus
}
#endif

#endif /* DDCB_H */
