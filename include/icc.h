/*
 * icc.h -- C ABI of the B200 matrix-free B-spline elasticity operator and Jacobi-PCG solver.
 *
 * The operator is y = sum_e s_e K_type(e) u_e on a uniform quadratic (p = 2) tensor-product
 * B-spline grid over an axis-aligned box, with the reference's numbering:
 *   control point g = ix + ncx*(iy + ncy*iz)            (rust/src/iga/space.rs:133-147)
 *   DOF           c*ndof_sc + g (component-blocked)     (rust/src/iga/space.rs:148-155)
 *   element-local a = ax + 3*(ay + 3*az), DOF c*27 + a  (rust/src/iga/space.rs:4-9)
 *   K_type rows = test, columns = trial, row-major 81x81 (rust/src/iga/elasticity.rs:14-26)
 *
 * All entry points return an int status (ICC_OK = 0) and never abort.  Host arrays are
 * borrowed for the duration of the call; device state is owned by the handle.  A handle is
 * bound to the CUDA device that was current when it was created, and runs its work on its own
 * stream.  Handles are not thread-safe.
 */
#ifndef ICC_H
#define ICC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------------ */
#define ICC_OK 0
#define ICC_NOT_CONVERGED 1   /* PCG hit max_iter before the tolerance */
#define ICC_BREAKDOWN 2       /* p'Ap <= 0 (rust/src/solver.rs:45-49): returns the current iterate */
#define ICC_BAD_ARG (-1)
#define ICC_CUDA_ERROR (-2)
#define ICC_TIMEOUT (-3)
#define ICC_NO_DEVICE (-4)
#define ICC_OUT_OF_MEMORY (-5)
#define ICC_NAN (-6)          /* a reduction produced NaN/Inf (NaN input or a non-SPD operator) */

/* ---- mask modes (the closures the reference wraps around CsrMatrix::matvec) ------------- */
#define ICC_MASK_NONE 0       /* y = K x                                   (rust/src/sparse.rs:60-68) */
#define ICC_MASK_ZERO 1       /* y = m.*K(m.*x)                   (rust/src/topopt_iga.rs:151-159,
                                                                   rust/src/immersed.rs:558-566) */
#define ICC_MASK_IDENTITY 2   /* y = K(m.*x) on free rows, y = x on fixed (rust/tests/iga_kernel.rs:101-107) */

/* ---- precision forms of the solve ---------------------------------------------------------- */
#define ICC_FP64 0            /* all-FP64 apply, vectors and reductions */
#define ICC_MIXED 1           /* Jacobi-PCG whose iterations run in FP32 on the tensor-core apply (a
                                 3-term split-TF32 product) with FP64 reductions, an FP64 solution and
                                 FP64 residual replacement (reliable updates); stops on the FP64 true
                                 residual */

typedef struct icc_space icc_space;
typedef struct icc_op icc_op;

typedef struct icc_solve_opts {
    int32_t precision;        /* ICC_FP64 or ICC_MIXED */
    int32_t check_every;      /* PCG iterations between convergence checks on the host (0: 32) */
    double inner_tol;         /* ICC_MIXED: the FP32 residual is replaced by the FP64 true residual
                                 whenever it has fallen by this factor since the last replacement
                                 (0: 0.6) */
    int32_t max_outer;        /* ICC_MIXED: maximum residual replacements (0: 1000) */
    int32_t reserved;
} icc_solve_opts;

typedef struct icc_solve_info {
    int64_t iterations;       /* PCG iterations (ICC_FP64) or inner iterations summed (ICC_MIXED) */
    int64_t outer_iterations; /* FP64 residual replacements (ICC_MIXED), 0 otherwise */
    double rel_res;           /* final relative residual (recurrence residual for ICC_FP64, as in
                                 rust/src/solver.rs:56-58; true FP64 residual for ICC_MIXED) */
    double device_ms;         /* device time of the solve (CUDA events on the handle's stream) */
    int64_t fp64_applies;     /* FP64 operator applications */
    int64_t mixed_applies;    /* tensor-core (split-TF32) operator applications */
    int64_t kernel_launches;  /* kernels this library launched for the solve */
} icc_solve_info;

/* Text of the last error on this thread ("" if none). */
const char *icc_last_error(void);

/* ---- space (rust/src/iga/space.rs:107 SpaceBox::new) --------------------------------------
 * bounds = {x0, x1, y0, y1, z0, z1}; nsub = elements per direction; degree must be 2 and the
 * box 3-D (the hot path); open uniform knots of maximal regularity (rust/src/iga/quadrature.rs:51). */
int icc_space_create(const double bounds[6], const int64_t nsub[3], int32_t degree, icc_space **out);
void icc_space_destroy(icc_space *sp);
/* A sub-grid of a space (no reference counterpart; the domain decomposition of the multi-rank
 * solve): elements [e0[d], e1[d]) per direction, 0 <= e0 < e1 <= nel_dir, with the parent's
 * B-splines, numbered locally (control points [e0, e1 + 2) of the parent, x fastest).  Its element
 * matrices (icc_element_matrices) are the parent's elements' matrices, including next to the cut,
 * and operators on it run on the tensor cores as well. */
int icc_space_window(const icc_space *sp, const int64_t e0[3], const int64_t e1[3], icc_space **out);
/* ndof, nel, control points per direction, elements per direction */
int icc_space_dims(const icc_space *sp, int64_t *ndof, int64_t *nel, int64_t ndof_dir[3], int64_t nel_dir[3]);
/* SpaceBox::connectivity (rust/src/iga/space.rs:148-155): conn[e*81 + c*27 + a] */
int icc_space_connectivity(const icc_space *sp, int64_t *conn);

/* ---- element matrices ----------------------------------------------------------------------- */
/* rust/src/iga/elasticity.rs:173-177 lame */
void icc_lame(double young, double poisson, double *lambda, double *mu);
/* rust/src/iga/elasticity.rs:30-150 elasticity_element_matrices: writes ntypes row-major 81x81
 * matrices (capacity max_types) and the type of every element, type ids in order of first
 * appearance exactly as the reference groups them. */
int icc_element_matrices(const icc_space *sp, double lambda, double mu, double *ke_types,
                         int32_t max_types, int32_t *type_id, int32_t *ntypes);

/* ---- operator --------------------------------------------------------------------------------
 * Replaces AssemblyPattern::assemble + CsrMatrix (rust/src/sparse.rs:128-175, :60-78) by a
 * matrix-free device operator.  ke_types[ntypes*81*81], type_id[nel], scale[nel] (s_e, NULL = 1),
 * free_mask[ndof] (NULL = all free; ignored for ICC_MASK_NONE). */
int icc_op_create(const icc_space *sp, const double *ke_types, int32_t ntypes, const int32_t *type_id,
                  const double *scale, const uint8_t *free_mask, int32_t mask_mode, icc_op **out);
/* Convenience: element matrices from (lambda, mu) built on the host as icc_element_matrices does. */
int icc_op_create_lame(const icc_space *sp, double lambda, double mu, const double *scale,
                       const uint8_t *free_mask, int32_t mask_mode, icc_op **out);
void icc_op_destroy(icc_op *op);
/* Per-design-iteration rescale: replaces AssemblyPattern::assemble(|e| .., &scale)
 * (rust/src/sparse.rs:160, called from rust/src/topopt_iga.rs:131-134). */
int icc_op_update_scale(icc_op *op, const double *scale);
int icc_op_update_mask(icc_op *op, const uint8_t *free_mask, int32_t mask_mode);
/* A sparse term S added to the operator: y = mask rule of (K + S)(m .* x), i.e. the closures that
 * add a stabilisation matrix to the stiffness inside PcgSolver::solve (rust/src/topopt_immersed.rs:
 * 174-183 k.matvec + stab.matvec; rust/src/immersed.rs:514-548 + :558-566, the stabilisation
 * assembled into the stiffness).  Triplets (row, col, value) over the DOF numbering, duplicates
 * summed (CsrMatrix::from_triplets, rust/src/sparse.rs:16-58); count = 0 removes the term.  The
 * diagonal (icc_op_diagonal, and the solve's default preconditioner) includes S's diagonal; the
 * FP64 forms apply S in FP64, the tensor-core FP32 form in FP32.  Element energies stay those of
 * K alone (as the reference computes them from the element matrices). */
int icc_op_set_extra_triplets(icc_op *op, int64_t count, const int64_t *rows, const int64_t *cols,
                              const double *vals);
/* y = A x with A the masked operator (host arrays of length n = ndof); mirrors the closure
 * around CsrMatrix::matvec (rust/src/sparse.rs:60-68). */
int icc_op_apply(icc_op *op, const double *x, double *y, int64_t n);
/* Same on device arrays, enqueued on the handle's stream (see icc_op_stream). */
int icc_op_apply_dev(icc_op *op, const double *x_dev, double *y_dev, int64_t n);
/* y = A x in FP32 with the tensor-core contraction (3-term split-TF32 products, FP32
 * accumulation): the operator of the ICC_MIXED inner solve.  Host arrays / device arrays. */
int icc_op_apply_f32(icc_op *op, const float *x, float *y, int64_t n);
int icc_op_apply_f32_dev(icc_op *op, const float *x_dev, float *y_dev, int64_t n);
/* CsrMatrix::diagonal (rust/src/sparse.rs:70-78) of the unmasked operator: sum_e s_e K[a,a],
 * accumulated in element order, bit-identical to the assembled CSR diagonal. */
int icc_op_diagonal(icc_op *op, double *d, int64_t n);
/* cudaStream_t of the handle (as void*), for callers that time or order device work. */
void *icc_op_stream(icc_op *op);

/* ---- solve: PcgSolver::new(max_iter, tol).solve(n, b, diag, closure) (rust/src/solver.rs:9-76)
 * x starts at 0, Jacobi preconditioner inv_diag = |d| > 1e-12 ? 1/d : 1, stop when
 * ||r||/max(||b||, 1e-16) < tol, break when p'Ap <= 0.  diag NULL = the operator's own diagonal.
 * Returns ICC_OK, ICC_NOT_CONVERGED, ICC_BREAKDOWN or an error; x, iters and rel_res are
 * written in every non-error case (as the reference returns its current iterate). */
int icc_pcg_solve(icc_op *op, const double *b, const double *diag, int64_t n, double tol, int64_t max_iter,
                  const icc_solve_opts *opts, double *x, int64_t *iters, double *rel_res);
/* Same on device arrays (b_dev, diag_dev may be NULL for the operator diagonal). */
int icc_pcg_solve_dev(icc_op *op, const double *b_dev, const double *diag_dev, int64_t n, double tol,
                      int64_t max_iter, const icc_solve_opts *opts, double *x_dev, int64_t *iters,
                      double *rel_res);
/* Details of the last solve on this handle. */
int icc_op_last_solve_info(const icc_op *op, icc_solve_info *info);

/* ---- allocation-free apply (no counterpart in the reference) --------------------------------
 * y = K x (FP64, no mask) for callers that must not allocate device memory: applications that
 * hand libraries buffers from their own device pool and forbid cudaMalloc/cudaFree (which can
 * synchronize the device), or loops that may not allocate after start-up.  Every argument is a
 * buffer the caller owns: nel_dir (host), ke_types_dev [ntypes*81*81] row-major, type_id_dev [nel],
 * scale_dev [nel] or NULL for 1, x_dev / y_dev [ndof]; stream is a cudaStream_t (NULL = default).
 * The only scratch is a fixed 16 MiB device array inside the library (held on every GPU that loads
 * it until exit), so grids are limited to 1941 bricks of 8x4x4 elements (for example 96x48x48
 * elements); larger grids return ICC_BAD_ARG.  The first call on a device resolves that array's
 * address (make it before any stream capture).  All calls share the array: calls that overlap on
 * the GPU race and must be ordered by the caller.  Allocates nothing. */
int icc_apply_f64_noalloc(const int64_t nel_dir[3], const double *ke_types_dev, int32_t ntypes,
                          const int32_t *type_id_dev, const double *scale_dev, const double *x_dev, double *y_dev,
                          void *stream);

/* Many independent solves (designs of uneven sizes, or load cases) at once: instance i solves
 * ops[i] x[i] = b[i] as icc_pcg_solve does (diag may be NULL, or diag[i] NULL), all instances in
 * flight together on their handles' streams.  Per instance: status[i] (an icc_pcg_solve code),
 * iters[i], rel_res[i] (both may be NULL).  Returns ICC_OK when every instance ran (converged or
 * not), else the first instance's error.  The handles must be distinct. */
int icc_pcg_solve_batched(int32_t count, icc_op *const *ops, const double *const *b, const double *const *diag,
                          double tol, int64_t max_iter, const icc_solve_opts *opts, double *const *x, int64_t *iters,
                          double *rel_res, int32_t *status);

/* ---- callers of the path in the SIMP loop ------------------------------------------------------
 * rust/src/topopt_iga.rs:137-162 CantileverTopOpt::solve_state on the handle's operator (mask mode
 * ICC_MASK_ZERO = the reference's closure): b = F - K u0 on free DOFs, diag clamped at 1e-12,
 * tol' = min(pcg_tol |F_free| / |b|, 0.5) (1 when b = 0), du from the PCG (opts->precision selects
 * FP64 or MIXED), u = u0 + du on free DOFs and 0 on fixed ones; *rel_res = PCG residual * |b| /
 * |F_free| as the reference returns it.  u0 must vanish on fixed DOFs.  Host arrays of n = ndof;
 * u may alias u0. */
int icc_solve_state(icc_op *op, const double *force, const double *u0, int64_t n, double pcg_tol,
                    const icc_solve_opts *opts, double *u, int64_t *iters, double *rel_res);

/* rust/src/topopt_iga.rs:165-184 element_energies: ee[e] = u_e^T K_type(e) u_e (unscaled). */
int icc_op_element_energies(icc_op *op, const double *u, int64_t n, double *ee, int64_t nel);

/* rust/src/topopt_iga.rs:19-54 CantileverTopOptConfig (nel and degree 2 are arguments). */
typedef struct icc_topopt_cfg {
    double size[3];           /* box [0,size0] x [0,size1] x [0,size2] (reference default 1.2, 0.6, 0.3) */
    double volfrac, penal, rmin, young, poisson, emin, move_limit, pcg_tol;
    int32_t precision;        /* state solves: ICC_FP64 or ICC_MIXED */
    int32_t reserved;
} icc_topopt_cfg;

typedef struct icc_topopt icc_topopt;

/* rust/src/topopt_iga.rs:73-129 CantileverTopOpt::new: clamp x = 0, the reference's tip load, the
 * radius filter on element centres (as a stencil), the device operator. */
int icc_topopt_create(const int64_t nel[3], const icc_topopt_cfg *cfg, icc_topopt **out);
void icc_topopt_destroy(icc_topopt *t);

/* Several load cases (extends the reference's single tip load, which the handle starts with):
 * forces is nload x ndof (component-blocked, like every vector here).  Each design iteration then
 * solves every case warm-started from its previous state.  With cfg.precision = ICC_MIXED and
 * nload > 1 the cases' state solves run as one batch: every PCG iteration is one tensor-core
 * apply over the bricks of all cases and one fused vector step (per-case PCG scalars, each case
 * stops on its own tolerance).  With ICC_FP64 the cases are solved one after another.
 * Compliance and element energies are summed over the cases, and pcg_iters reports the sum. */
int icc_topopt_set_loads(icc_topopt *t, int32_t nload, const double *forces);

/* rust/src/topopt_iga.rs:187-234 CantileverTopOpt::run: densities from volfrac, per iteration the
 * SIMP scale, the warm-started state solve, compliance |F'u|, sensitivities, filter and the OC
 * bisection (candidate of its last step); stops after max_iter or when change < 0.01 and
 * iteration >= 15.  Outputs per iteration (arrays of max_iter; any may be NULL): compliance,
 * change, PCG iterations; final densities (nel); iterations run. */
int icc_topopt_run(icc_topopt *t, int32_t max_iter, double *compliance, double *change, int64_t *pcg_iters,
                   double *density, int32_t *iters_run);

/* ---- immersed set-up ------------------------------------------------------------------------------
 * rust/src/immersed.rs:88-155 classify_background_cells + element_weights on the res[0] x res[1] x
 * res[2] grid of the unit cube for the analytic solid "cube minus three orthogonal through-cylinders
 * of radius `radius` about the centre lines" (the reference evaluates a triangle mesh by ray parity;
 * the rule is the same): status 1 inside, 0 outside, -1 cut; weight 1, 0, or the fraction of
 * sub[0] x sub[1] x sub[2] cell midpoints inside.  Computed on the device; host arrays of
 * res[0] res[1] res[2] cells. */
int icc_cylinder_weights(const int64_t res[3], const int32_t sub[3], double radius, double *weights, int8_t *status);

/* ---- cut-cell stabilisation (triplets for icc_op_set_extra_triplets) ---------------------------
 * status[nel] per cell: 1 inside, 0 outside, -1 cut.  Both return *count triplets; called with
 * rows = cols = vals = NULL they only report the count, else they fill up to capacity entries.
 * rust/src/immersed.rs:224-370 ghost_penalty: gamma E h^(2p-1) sum_F int_F [d_n^p u].[d_n^p v] over
 * interior faces between two active cells of which at least one is cut, per component. */
int icc_ghost_penalty(const icc_space *sp, const int8_t *status, double gamma, double young, int64_t *rows,
                      int64_t *cols, double *vals, int64_t capacity, int64_t *count);
/* rust/src/immersed.rs:156-222 legacy_stabilization (the MATLAB heuristic kept for the reference's
 * fixture): zero-sum diagonal blocks on shared control points and springs of stiffness
 * gamma mean(h) between the faces' non-shared control points. */
int icc_legacy_stabilization(const icc_space *sp, const int8_t *status, double gamma, int64_t *rows, int64_t *cols,
                             double *vals, int64_t capacity, int64_t *count);

/* ---- diagnostics (no reference counterpart) -------------------------------------------------
 * Times `reps` FP64 applies of x_dev on the handle's stream with CUDA events around each of the
 * two kernels of an apply (the element-brick contraction and the node-side sum); returns the
 * mean milliseconds of each.  Used by the benchmark for the roofline figure. */
int icc_op_profile_apply(icc_op *op, const double *x_dev, double *y_dev, int32_t reps, double *contract_ms,
                         double *gather_ms);

/* The same for the tensor-core FP32 apply (unmasked input x_dev, FP32 device arrays). */
int icc_op_profile_apply_f32(icc_op *op, const float *x_dev, float *y_dev, int32_t reps, double *contract_ms,
                             double *gather_ms);

/* Polls of a grid-wide barrier in the mixed solve's fused vector step before it gives up and the
 * solve returns ICC_TIMEOUT (default 2^22).  The error flag and the barrier counter are cleared at
 * the start of every call, so the handle works normally after a time-out.  Lets a test make the
 * bounded wait run out without a fault; no reference counterpart. */
int icc_op_set_wait_limit(icc_op *op, int64_t grid_polls);

#ifdef __cplusplus
}
#endif

#endif /* ICC_H */
