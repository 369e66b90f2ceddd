/*
 * jxb.h -- C ABI of the B200 Galerkin linear-solve library (libjxb.so).
 *
 * The library replaces, for single-patch tensor-product NURBS spaces, the
 * traced stage of JAXIGA's Galerkin solve for linear problems:
 *
 *   evaluation at Gauss points   src/jaxiga/space/evaluation.py:95-172, 305-467
 *   element tangents             src/jaxiga/forms/library.py:54-65, 125-132, 174-181
 *   matrix-free tangent matvec   src/jaxiga/methods/galerkin.py:207-218
 *   Jacobi diagonal              src/jaxiga/methods/galerkin.py:221-237
 *   load vector / rhs            src/jaxiga/methods/galerkin.py:240-245,
 *                                src/jaxiga/methods/_common.py:280-309
 *   Krylov solve                 src/jaxiga/solvers/linear.py:399-442
 *   true-residual diagnostics    src/jaxiga/solvers/diagnostics.py:8-19
 *
 * Conventions
 *   - DOF vectors are FP64 device arrays of length n_dofs = vec * n_cp_total,
 *     component c of scalar basis i at index vec*i + c (function_space.py:300-312).
 *   - Control points and elements are numbered with the first parametric
 *     direction fastest (function_space.py:326-369, nurbs.py conventions).
 *   - Per-quadrature-point arrays are (n_elem, n_q^dim[, ncomp]) with elements
 *     and points both first-direction-fastest (pointset.py:104-112).
 *   - All device work is ordered on the caller's stream; no call blocks except
 *     jxb_plan_create, the solves (which read convergence state
 *     back to the host) and jxb_plan_destroy.
 *   - Return value 0 is success; otherwise a jxb_status code, with a message
 *     retrievable from jxb_last_error() on the calling thread.
 *   - A plan may be used by one host thread at a time; distinct plans are
 *     independent. Every device loop has an iteration cap.
 */
#ifndef JXB_H
#define JXB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* jxb_stream; /* a cudaStream_t; NULL = legacy default stream */
typedef struct jxb_plan jxb_plan;

enum jxb_status {
  JXB_OK = 0,
  JXB_ERR_INVALID = 1,      /* bad argument or unsupported configuration */
  JXB_ERR_CUDA = 2,         /* CUDA runtime error */
  JXB_ERR_NOT_CONVERGED = 3,/* iteration cap reached before the tolerance */
  JXB_ERR_NONFINITE = 4,    /* NaN/Inf met in a reduction */
  JXB_ERR_NOMEM = 5
};

enum jxb_operator {
  JXB_OP_POISSON = 0,     /* -div(a grad u) = f   (library.py:40-65)      */
  JXB_OP_ELASTICITY = 1,  /* small-strain isotropic (library.py:146-203) */
  JXB_OP_PLATE = 2,       /* Kirchhoff plate, biharmonic (library.py:68-143) */
  JXB_OP_HYPERELASTIC = 3 /* compressible neo-Hookean, Newton tangent at a state (library.py:206-225);
                             coef = {mu, lambda}; jxb_hyper_state sets the state */
};

/* Everything a plan needs; arrays are HOST pointers, copied at creation. */
typedef struct jxb_desc {
  int dim;                      /* 2 or 3 */
  int vec;                      /* 1 (Poisson, plate) or dim (elasticity) */
  int degree;                   /* p, equal in every direction, 1..5 */
  int n_quad;                   /* Gauss points per direction, p+1 */
  int n_cp[3];                  /* control points per direction */
  int n_span[3];                /* non-empty knot spans per direction */
  const int32_t* first[3];      /* first basis index of each span (bernstein.py:261-284) */
  const double* span_lo[3];     /* span bounds in [0, 1] */
  const double* span_hi[3];
  const double* extraction[3];  /* (n_span, p+1, p+1) row-major Bezier operators (bernstein.py:16-76) */
  const double* cpts;           /* (n_cp_total, dim) unweighted control points */
  const double* wgts;           /* (n_cp_total,) NURBS weights */
  const double* gauss_nodes;    /* (n_quad,) on [-1, 1] */
  const double* gauss_weights;  /* (n_quad,) */
  int op;                       /* enum jxb_operator */
  double coef[4];               /* Poisson: a0 | elasticity: E, nu | plate: E, nu, t */
  int plane_strain;             /* 2D elasticity: 0 plane stress, 1 plane strain */
  const double* coef_qp;        /* optional (n_elem, n_quad^dim) per-point a0 (PointField); NULL = coef[0] */
  const uint8_t* prescribed;    /* optional (n_dofs,) 1 = Dirichlet DOF; NULL = none */
  int want_f32;                 /* also keep FP32 copies of the point factors (mixed precision) */
  int tile[2];                  /* 2D brick shape (elements per row, rows); {0,0} = default (32 per row, up
                                   to 8 rows, fewer when the patch is small). Rows: 1..64; elements per
                                   row: 32, or 16 / 64 for the scalar operator (the batch autotuner picks) */
} jxb_desc;

typedef struct jxb_info {
  int64_t n_dofs, n_free, n_elem, n_qp;
  int64_t n_bricks;
  int64_t geo_bytes;            /* bytes of per-point factors read by one apply */
  int64_t scratch_bytes;        /* brick partial-sum buffer */
  int ngeo;                     /* factors per quadrature point */
  int rational;                 /* 1 if weights are not all equal */
} jxb_info;

typedef struct jxb_solve_opts {
  double tol;                   /* relative tolerance on ||r|| / ||b|| */
  double atol;                  /* absolute tolerance (jax semantics), usually 0 */
  int64_t maxiter;              /* <= 0: 10 * n_free (jax default) */
  int preconditioner;           /* 0 none, 1 Jacobi */
  int check_every;              /* iterations per captured graph launch (<= 0: 16) */
  /* refinement (jxb_refine_solve, jxb_mixed_pcg) */
  double inner_tol;             /* relative tolerance of each FP32 inner solve;
                                   jxb_mixed_pcg: residual drop between updates */
  int max_outer;                /* cap on outer FP64 steps / updates */
  int restarts;                 /* jxb_pcg: true-residual restarts (0..8) when the recursive residual
                                   met the tolerance but the FP64 true residual did not; they share the
                                   maxiter budget, as the reference's CPU CG (linear.py:261-321) */
} jxb_solve_opts;

typedef struct jxb_stats {
  int64_t iterations;           /* Krylov iterations (inner ones for refinement) */
  int64_t outer;                /* refinement steps */
  double residual;              /* ||b - K x|| over free DOFs, recomputed in FP64 */
  double relative_residual;
  double b_norm;
  int converged;                /* finite and residual <= max(tol * ||b||, atol) */
  int finite;
  double seconds;               /* device time of the solve (CUDA events) */
} jxb_stats;

/* ---- plan lifetime ---------------------------------------------------- */
int jxb_plan_create(const jxb_desc* desc, jxb_plan** out);
int jxb_plan_destroy(jxb_plan* plan);
int jxb_plan_info(const jxb_plan* plan, jxb_info* out);
const char* jxb_last_error(void);
int jxb_version(void);

/* ---- operator ----------------------------------------------------------
 * jxb_apply: y = K x restricted to free DOFs (src/jaxiga/methods/galerkin.py:207-218).
 *   masked != 0: prescribed entries of x are ignored and y is 0 there,
 *                i.e. y = P_f K P_f x, the operator the Krylov loop sees.
 *   masked == 0: the full, unconstrained K x (used for the Dirichlet lift).
 * jxb_apply_f32: the same operator in FP32 (factors and arithmetic), for
 *   mixed-precision inner solves; requires want_f32.
 * jxb_diag: diag(K) on free DOFs, 0 on prescribed (galerkin.py:221-237).
 */
int jxb_apply(jxb_plan* plan, jxb_stream stream, const double* x, double* y, int masked);
int jxb_apply_f32(jxb_plan* plan, jxb_stream stream, const float* x, float* y);
/* jxb_apply_static: the same result as jxb_apply, for callers that must not
 *   allocate device memory when they apply the operator (a handler inside a
 *   framework that owns every device allocation, a loop where an allocation's
 *   implicit synchronisation is unacceptable). The brick partial sums go to one
 *   fixed 16 MiB device array per GPU, present from library load to process
 *   exit, instead of the plan's scratch; plans needing more are rejected with
 *   JXB_ERR_INVALID. This call allocates nothing. Its first call on a device
 *   looks up the array's address (cudaGetSymbolAddress) and should come before
 *   any stream capture. All calls share the array: calls that overlap on the
 *   GPU race and must be ordered on one stream. The plan's device (current
 *   when the plan was created) must be current; otherwise JXB_ERR_INVALID.
 *   No counterpart in the reference, which has no device kernels. */
int jxb_apply_static(jxb_plan* plan, jxb_stream stream, const double* x, double* y, int masked);
int jxb_diag(jxb_plan* plan, jxb_stream stream, double* d);

/* ---- fields at quadrature points ---------------------------------------
 * jxb_qp_coords: physical coordinates of every Gauss point, (n_elem, n_q^dim, dim).
 * jxb_interpolate: sum_i R_i(x_q) c_i for a control-point field c (n_cp_total, ncomp),
 *   written as (n_elem, n_q^dim, ncomp) -- Solution.at / PointField construction.
 * jxb_load: F_i,c = sum_q w_q f_c(x_q) R_i(x_q) for source values f (n_elem, n_q^dim, vec)
 *   (the source work term of methods/_common.py:280-309), full length n_dofs.
 */
int jxb_qp_coords(jxb_plan* plan, jxb_stream stream, double* x);
int jxb_interpolate(jxb_plan* plan, jxb_stream stream, const double* coef, int ncomp, double* out);
/* jxb_interpolate_grad: physical gradients sum_i dR_i/dx(x_q) c_i of a control-point field
 *   (n_cp_total, ncomp), ncomp 1..3, written as (n_elem, n_q^dim, ncomp, dim)
 *   -- Solution.grad (src/jaxiga/post/solution.py:50-54) for the H1 and energy
 *   error norms (src/jaxiga/post/norms.py:59-140). */
int jxb_interpolate_grad(jxb_plan* plan, jxb_stream stream, const double* coef, int ncomp, double* out);
/* jxb_eval_points: evaluation at arbitrary points of a PointSet
 *   (src/jaxiga/space/pointset.py:27-75; evaluate, src/jaxiga/space/evaluation.py:305-467;
 *   Solution.at/grad, src/jaxiga/post/solution.py:39-54). Point k lies in element
 *   elems[k] (device int64, reference order) at reference coordinates ref[k]
 *   (device, (n, dim), in [-1, 1]^dim). Writes, for each non-NULL output:
 *   val (n, ncomp) and grad (n, ncomp, dim) of the control-point field coef
 *   (ncomp 1..3; may be NULL when only x/jac are wanted), x (n, dim) physical
 *   coordinates, jac (n) = |det J| prod(h/2), the factor the reference applies to
 *   its quadrature weights. Out-of-range element indices give NaN. */
int jxb_eval_points(jxb_plan* plan, jxb_stream stream, const double* coef, int ncomp, int64_t n,
                    const int64_t* elems, const double* ref, double* val, double* grad, double* x, double* jac);
/* Neumann loads (tractions / fluxes on boundary sides): the work term
 * neumann_work of src/jaxiga/methods/_common.py:312-318 on the boundary Gauss
 * sets of src/jaxiga/space/pointset.py:148-200.
 * jxb_boundary_points: face f is side sides[f] (2 * direction + end) of element
 *   elems[f]; its n_q points sit at ref (n_faces * n_q, dim) with reference
 *   weights wref (n_faces * n_q). Writes physical points x and outward unit
 *   normals (n_faces * n_q, dim) and surface weights w = wref * surface
 *   Jacobian * tangential half-widths (src/jaxiga/space/evaluation.py:174-193,
 *   432-455); any output may be NULL. All arrays are device arrays.
 * jxb_boundary_load: F[vec*i + c] += sum over faces and points of
 *   w t[c] R_i for tractions t (n_faces * n_q, vec) at those points. local is
 *   scratch of n_faces * (p+1)^dim * vec doubles (face-local loads); the
 *   scatter is deterministic: scalar DOF dofs[k] (k < n_touched) receives the
 *   local entries contrib[ptr[k] .. ptr[k+1]) (indices face * (p+1)^dim + a,
 *   a the element-local basis function, first direction fastest), in that order. */
int jxb_boundary_points(jxb_plan* plan, jxb_stream stream, int64_t n_faces, int n_q, const int64_t* elems,
                        const int32_t* sides, const double* ref, const double* wref, double* x, double* normal,
                        double* w);
int jxb_boundary_load(jxb_plan* plan, jxb_stream stream, int64_t n_faces, int n_q, const int64_t* elems,
                      const double* ref, const double* w, const double* traction, int64_t n_touched,
                      const int64_t* dofs, const int64_t* ptr, const int64_t* contrib, double* local, double* F);
int jxb_load(jxb_plan* plan, jxb_stream stream, const double* f_qp, double* F);
/* jxb_qp_weights: integration weights w_hat |J| prod(h/2) at every Gauss point,
 *   (n_elem, n_q^dim) -- BasisData.w of src/jaxiga/space/evaluation.py:461-463. */
int jxb_qp_weights(jxb_plan* plan, jxb_stream stream, double* w);

/* ---- solves -------------------------------------------------------------
 * jxb_pcg: preconditioned CG on the free DOFs, from x = 0, following
 *   jax.scipy.sparse.linalg.cg (the reference's matrix-free default,
 *   src/jaxiga/solvers/linear.py:399-442): stop when ||r||^2 <= max(tol^2 ||b||^2, atol^2).
 *   b is a full-length vector; its prescribed entries are ignored and x is 0
 *   there on return. Stats carry the FP64 true residual (diagnostics.py:8-19).
 *   With opts->restarts > 0, a solve whose FP64 true residual is still above
 *   the tolerance when CG stops restarts CG on that residual (tolerance
 *   min(0.5, 0.5 tol ||b|| / ||r||)) and adds the correction, at most
 *   `restarts` times, keeping only corrections that lower the true residual;
 *   stats->outer counts them.
 *   Every solve below writes x and stats and then returns JXB_ERR_NOT_CONVERGED
 *   when the true residual misses the tolerance (iteration cap, stagnation),
 *   JXB_ERR_NONFINITE when a reduction met NaN/Inf, else JXB_OK.
 * jxb_refine_solve: FP64 iterative refinement around FP32 Jacobi-PCG inner solves
 *   (jxb_apply_f32); the outer residual and correction are FP64.
 * jxb_mixed_pcg: FP32 Jacobi-PCG with reliable FP64 updates. The FP32 iterate
 *   is folded into the FP64 solution and the residual recomputed in FP64 each
 *   time the FP32 residual has fallen by opts->inner_tol (default 1e-2), and
 *   at the target; the search direction is kept across updates. Stats: outer =
 *   number of updates, iterations = FP32 iterations. Same stopping rule and
 *   true-residual stats as jxb_pcg; the plan needs want_f32. No counterpart in
 *   the reference (its solves are FP64 only).
 */
int jxb_pcg(jxb_plan* plan, jxb_stream stream, const double* b, double* x,
            const jxb_solve_opts* opts, jxb_stats* stats);
int jxb_refine_solve(jxb_plan* plan, jxb_stream stream, const double* b, double* x,
                     const jxb_solve_opts* opts, jxb_stats* stats);
int jxb_mixed_pcg(jxb_plan* plan, jxb_stream stream, const double* b, double* x,
                  const jxb_solve_opts* opts, jxb_stats* stats);

/* jxb_bicgstab: BiCGSTAB (van der Vorst) on the same masked operator, the
 *   reference's method="bicgstab" (jax.scipy.sparse.linalg.bicgstab,
 *   src/jaxiga/solvers/linear.py:152-171, 399-411): from x = 0, Jacobi (or no)
 *   right preconditioning, stop when r.r <= max(tol^2 b.b, atol^2) or at maxiter;
 *   a breakdown (rho, alpha or omega zero) returns JXB_ERR_NONFINITE. Stats and
 *   return codes as jxb_pcg. */
int jxb_bicgstab(jxb_plan* plan, jxb_stream stream, const double* b, double* x, const jxb_solve_opts* opts,
                 jxb_stats* stats);

/* jxb_pcg_snapshots: jxb_pcg (Jacobi or none, jax CG semantics) that also copies
 *   the FP64 iterate into snaps[j] (n_dofs doubles each) after every `every`
 *   iterations, up to max_snaps; *n_snaps receives the number written. With the
 *   converged x*, (K (x* - x_j), x* - x_j) are the solver's residual/error pairs. */
int jxb_pcg_snapshots(jxb_plan* plan, jxb_stream stream, const double* b, double* x,
                      const jxb_solve_opts* opts, int every, double* snaps, int64_t max_snaps,
                      int64_t* n_snaps, jxb_stats* stats);

/* ---- nonlinear elasticity (compressible neo-Hookean) ----------------------
 * W(F) = mu/2 (tr F^T F - d) - mu ln J + lambda/2 (ln J)^2, F = I + grad u
 * (src/jaxiga/forms/library.py:206-225); the reference differentiates W with jax.
 * For a JXB_OP_HYPERELASTIC plan:
 *   jxb_hyper_state    evaluates F at every Gauss point of the displacement u
 *                      (all n_dofs, Dirichlet values included) and stores the
 *                      tangent state (F^-T, mu - lambda ln J) and the first
 *                      Piola-Kirchhoff flux P(F); *energy (host, may be NULL)
 *                      receives the stored energy sum_q w_q W(F_q), summed in a
 *                      fixed order. Until it is called the state is u = 0.
 *   jxb_hyper_residual r = int P(F) : grad v over all DOFs (the internal
 *                      forces of the residual, methods/_common.py:280-309 with
 *                      the energy's gradient in place of jax.grad).
 *   jxb_apply / jxb_diag / jxb_pcg act with the tangent
 *     dP = mu dF + (mu - lambda ln J) F^-T dF^T F^-T + lambda (F^-T : dF) F^-T
 *   at the stored state (tangent_matvec at u, methods/galerkin.py:207-218).
 * A state with J <= 0 gives non-finite values, as the reference's log does. */
int jxb_hyper_state(jxb_plan* plan, jxb_stream stream, const double* u, double* energy);
int jxb_hyper_residual(jxb_plan* plan, jxb_stream stream, double* r);

/* ---- several conforming patches (multipatch spaces) ----------------------
 * A composite plan over n patch plans of one operator (created without
 * Dirichlet masks), glued by local_to_global[i] (patch i's n_cp entries: the
 * global scalar index of each control point, src/jaxiga/geometry/multipatch.py
 * compute_topology). Its K.u is sum_p S_p^T K_p S_p x (S_p the gather of patch
 * p's DOFs), the patch copies of every global DOF summed in a fixed order;
 * prescribed (n_global_scalar * vec, or NULL) marks Dirichlet DOFs. It works
 * with jxb_apply, jxb_diag, jxb_load (f_qp: the patches' points in patch order),
 * jxb_dot, jxb_pcg and jxb_plan_destroy (which leaves the patch plans alone;
 * destroy them after the composite); the other entry points reject it. */
int jxb_mp_create(jxb_plan* const* patches, int n, const int64_t* const* local_to_global, int64_t n_global_scalar,
                  const uint8_t* prescribed, jxb_plan** out);

/* ---- truncated hierarchical (THB) spaces -----------------------------------
 * Poisson, -div(a grad u) = f, or isotropic linear elasticity (src/jaxiga/forms/
 * library.py:174-181) on a space in the padded-element form of the
 * reference (src/jaxiga/space/function_space.py:23-38, built by
 * src/jaxiga/space/hierarchical.py:891-980): per leaf element, n_local_max
 * hierarchical functions (padding index n_scalar) and the extraction rows
 * (zero for the padding) that map the element's Bernstein polynomials on
 * [-1, 1]^dim to them. Replaces the reference's element tangents and CSR scatter
 * on such spaces (src/jaxiga/methods/galerkin.py:82-148, src/jaxiga/forms/
 * library.py:54-65) by a matrix-free element apply. All arrays are host arrays:
 *   elem_dofs  (n_elem, n_local_max) int64;
 *   extraction (n_elem, n_local_max, nb), nb = (degree + 1)^dim;
 *   wgts       (n_scalar) NURBS weights of the hierarchical basis;
 *   tables     (dim + 1, nq, nb): Bernstein values, then the derivative along
 *              each reference direction, at the nq = (degree + 1)^dim Gauss
 *              points (first direction fastest); the plate adds the second
 *              derivatives 11, 12, 22: (6, nq, nb);
 *   factors    (n_elem, nq, nf), Poisson: nf = (dim + 1)(dim + 2) / 2, per point
 *              the symmetric metric M = a w L^T L of the channels (numerator
 *              value, its reference gradient), L = J^-T (1/W) [-grad W / W | I],
 *              packed upper triangle row by row; elasticity: nf = dim^2 + 2 +
 *              dim, per point J^-1 (row-major, [a][k] = d xi_a / d x_k in
 *              reference coordinates), w |J|, 1/W and grad W / W; plate:
 *              nf = 21, the metric w L^T D L of the six channels (numerator
 *              value, gradient, second derivatives) with L mapping them to the
 *              curvatures -(R_xx, R_yy, 2 R_xy), packed the same way;
 *   wq         (n_elem, nq): quadrature weight over the weight function W;
 *   prescribed (n_scalar * vec) 1 = Dirichlet DOF, or NULL.
 * DOF c of function i is vec * i + c. The plan works with jxb_apply, jxb_diag,
 * jxb_load (f_qp: (n_elem, nq, vec)),
 * jxb_dot, jxb_pcg and jxb_plan_destroy; the other entry points reject it. */
typedef struct jxb_thb_desc {
  int dim, degree, n_local_max;
  int op;                      /* JXB_OP_POISSON, JXB_OP_ELASTICITY (vec = dim) or JXB_OP_PLATE (dim 2) */
  int64_t n_elem, n_scalar;
  double lam, mu;              /* elasticity: Lame parameters (plane stress or strain folded in) */
  const int64_t* elem_dofs;
  const double* extraction;
  const double* wgts;
  const double* tables;
  const double* factors;
  const double* wq;
  const uint8_t* prescribed;
} jxb_thb_desc;
int jxb_thb_create(const jxb_thb_desc* desc, jxb_plan** out);

/* ---- batches of independent problems -------------------------------------
 * The B200 form of the reference's vmap-over-params batching
 * (tests/test_advanced.py:338-356; host SciPy solves run once per member,
 * src/jaxiga/solvers/linear.py:147-149): 2D Poisson plans of any degree and
 * size, their DOF vectors concatenated in plan order (jxb_batch_size gives the
 * offsets), solved by Jacobi-PCG per instance with per-instance scalars and
 * convergence, every iteration of the whole batch captured in one CUDA graph.
 * stats receives one jxb_stats per instance; *seconds the device time. */
typedef struct jxb_batch jxb_batch;
int jxb_batch_create(jxb_plan* const* plans, int n, jxb_batch** out);
int jxb_batch_destroy(jxb_batch* batch);
int jxb_batch_size(const jxb_batch* batch, int64_t* total_dofs, int64_t* offsets /* n+1 or NULL */);
/* How a batched K.u runs: *persistent = 1 when one persistent launch walks the
 * bricks of every instance and degree (JXB_BATCH_PERSIST=1 and every plan has rows
 * of 32 elements), else 0; *brick_launches = brick launches per K.u. */
int jxb_batch_info(const jxb_batch* batch, int* persistent, int* brick_launches);
int jxb_batch_apply(jxb_batch* batch, jxb_stream stream, const double* x, double* y);
int jxb_batch_pcg(jxb_batch* batch, jxb_stream stream, const double* b, double* x, const jxb_solve_opts* opts,
                  jxb_stats* stats, double* seconds);

/* ---- learned preconditioner ---------------------------------------------
 * A 3D convolutional network on the control-point grid (FP32 weights and
 * activations, hand-written kernels), used inside flexible CG. No counterpart
 * in the reference, whose only preconditioner is Jacobi
 * (src/jaxiga/solvers/linear.py:419-431).
 *   jxb_cnn_create: a U-Net with `levels` (2..6) levels, channels[levels] per
 *     level (each in {4,8,12,16,24,32,48,64}); in_ch input channels (residual
 *     components, then features), out_ch outputs (= vec).
 *   jxb_cnn_params / jxb_cnn_grads: device pointer to the flat FP32 parameter
 *     vector / gradient accumulator and its length.
 *   jxb_cnn_forward: out[out_ch][nz][ny][nx] = N(in[in_ch][nz][ny][nx]).
 *   jxb_cnn_backward: adds to the accumulator the parameter gradient of
 *     sum(gout * N(in)); must follow a forward on the same input and dims.
 *   jxb_cnn_accumulate: forward, masked MSE against target, backward; returns the loss.
 *   jxb_cnn_accumulate_energy: forward, then, with z = P_f out_scale N(in) in DOF
 *     layout (0 on prescribed DOFs) and the plan's operator K, the loss
 *     angle == 0: weight * d^T K d, d = P_f e - z (energy norm of the error);
 *     angle == 1: weight * (1 - (z.r)^2 / ((z^T K z)(e.r))) for the pair r = K e
 *     (energy-norm angle between z and e: blind to the scale of z, which
 *     flexible CG does not use);
 *     angle == 2: the same angle for z + D^-1 r, the additive two-level map
 *     (the network learns what the Jacobi step misses).
 *     e and r are grids [vec][nz][ny][nx]; adds the parameter gradient and
 *     returns the loss.
 *   jxb_cnn_adam: one Adam step with the accumulated gradient times grad_scale.
 *   jxb_cnn_set_input_pooling: on = 1 pools the input once (2x2x2 average) and
 *     runs the U-Net on the half-resolution grid, interpolating its output back
 *     (trilinear); forward, backward and the losses keep their input-grid
 *     shapes. Drops the activation buffers.
 * jxb_fcg_learned: truncated flexible CG keeping `depth` (1..8) directions,
 *   z = ||r|| out_scale N(in_scale r/||r||, features) (cnn NULL: Jacobi only);
 *   Jacobi directions take over after `stall` learned iterations without a new
 *   lowest residual or a non-descent direction. `mode` bit 0: FP32 iterations
 *   with FP64 corrections (plan created with want_f32): reliable updates each
 *   time the residual has fallen by inner_tol (default 1e-2), the stored
 *   directions kept, as jxb_mixed_pcg, and a fallback to Jacobi lasts for the
 *   rest of the solve; with bit 2 also set, restarted FP32 solves to inner_tol
 *   inside FP64 iterative refinement instead;
 *   bit 1: two-level preconditioner z = a n + D^-1 (r - a K n), n the network
 *   output, a = (n.r)/(n^T K n) (one more operator apply per iteration);
 *   bit 3 (without bit 1): additive two-level z = n + D^-1 r, the weight of n
 *   fixed through out_scale (no extra apply).
 *   stats->outer = iterations that used the network. */
typedef struct jxb_cnn jxb_cnn;
int jxb_cnn_create(int in_ch, int out_ch, int levels, const int* channels, uint64_t seed, jxb_cnn** out);
int jxb_cnn_destroy(jxb_cnn* cnn);
int jxb_cnn_set_input_pooling(jxb_cnn* cnn, int on);
/* jxb_cnn_set_inference_bf16: on = 1 makes inference forwards (jxb_cnn_forward and
 *   the network applications inside jxb_fcg_learned) run every 3x3x3 layer of at
 *   most 32 input and output channels as a BF16 tensor-core implicit GEMM
 *   (mma.sync m16n8k16, FP32 accumulation); training forwards stay FP32, and a
 *   jxb_cnn_backward after a BF16 forward is refused. */
int jxb_cnn_set_inference_bf16(jxb_cnn* cnn, int on);
int jxb_cnn_params(jxb_cnn* cnn, float** params, int64_t* n);
int jxb_cnn_grads(jxb_cnn* cnn, float** grads, int64_t* n);
int jxb_cnn_forward(jxb_cnn* cnn, jxb_stream stream, int nx, int ny, int nz, const float* in, float* out);
int jxb_cnn_backward(jxb_cnn* cnn, jxb_stream stream, int nx, int ny, int nz, const float* in, const float* gout);
int jxb_cnn_zero_grad(jxb_cnn* cnn, jxb_stream stream);
int jxb_cnn_accumulate(jxb_cnn* cnn, jxb_stream stream, int nx, int ny, int nz, const float* in,
                       const float* target, const float* mask, double* loss);
int jxb_cnn_accumulate_energy(jxb_plan* plan, jxb_cnn* cnn, jxb_stream stream, const float* in, const float* e,
                              const float* r, float out_scale, double weight, int angle, double* loss);
int jxb_cnn_adam(jxb_cnn* cnn, jxb_stream stream, float lr, float grad_scale);
int jxb_fcg_learned(jxb_plan* plan, jxb_cnn* cnn, jxb_stream stream, const double* b, double* x,
                    const float* features, int n_features, float in_scale, double out_scale, int stall,
                    int depth, int mode, const jxb_solve_opts* opts, jxb_stats* stats);

/* ---- geometric multigrid -------------------------------------------------
 * A V-cycle over nested spline spaces of one patch (the finest first, each
 * coarser level the same patch with every other interior knot removed), used
 * as the preconditioner of CG. No counterpart in the reference, whose only
 * preconditioner is Jacobi (src/jaxiga/solvers/linear.py:419-431).
 *   jxb_transfer1d: one direction of the prolongation from level l+1 to level l,
 *     a CSR matrix (HOST arrays) of rows = control points of level l along that
 *     direction by cols = those of level l+1 (knot insertion); the tensor
 *     product over the directions maps coarse DOFs to fine ones, the
 *     restriction is its transpose.
 *   jxb_mg_create: plans[0..n_levels) of the same operator kind on those
 *     spaces (each plan listed once, its Dirichlet mask that of its level),
 *     transfer[3 l + d] for l < n_levels - 1 and d < dim, coarse_inv the dense
 *     row-major inverse of the coarsest operator on its free DOFs (zero rows and
 *     columns on prescribed DOFs), n_dofs^2 doubles, host. degree (1..8): the
 *     Chebyshev-Jacobi smoother's polynomial degree, applied before and after
 *     each coarse correction; smooth_range (> 1): the ratio lmax / lmin of the
 *     interval it damps, lmax of D^-1 K estimated at creation by a power
 *     iteration. The plans must outlive the multigrid object.
 *   jxb_mg_vcycle: z = V r on the finest level (r, z device, n_dofs).
 *   jxb_mg_pcg: CG preconditioned by the V-cycle, with the stopping rule, stats
 *     and return codes of jxb_pcg (opts->preconditioner and restarts unused).
 *   jxb_mg_info: lmax[l] of D^-1 K per level (the coarsest stays 0). */
typedef struct jxb_mg jxb_mg;
typedef struct jxb_transfer1d {
  int rows, cols;
  const int32_t* ptr;  /* rows + 1 */
  const int32_t* idx;  /* column of each entry */
  const double* val;
} jxb_transfer1d;
int jxb_mg_create(jxb_plan* const* plans, int n_levels, const jxb_transfer1d* transfer, const double* coarse_inv,
                  int degree, double smooth_range, jxb_mg** out);
int jxb_mg_destroy(jxb_mg* mg);
int jxb_mg_info(const jxb_mg* mg, double* lmax);
int jxb_mg_vcycle(jxb_mg* mg, jxb_stream stream, const double* r, double* z);
int jxb_mg_pcg(jxb_mg* mg, jxb_stream stream, const double* b, double* x, const jxb_solve_opts* opts,
               jxb_stats* stats);

/* ---- Jacobi-PCG on an assembled CSR matrix ------------------------------
 * The device CG of the staggered phase-field solver (DeviceCG,
 * src/jaxiga/solvers/phase_field.py:305-390): the pattern is set once per
 * mesh, each solve passes new values and right-hand side.
 *   jxb_csr_create: n rows, indptr (n + 1, int64) and cols (int32), HOST arrays.
 *   jxb_csr_matvec: y = A x for values (nnz), x, y device arrays.
 *   jxb_csr_pcg: Jacobi-PCG with jax CG semantics from the warm start in x
 *     (r0 = b - A x0, stop when r.r <= max(tol^2 b.b, atol^2) or at maxiter,
 *     default 10 n); the diagonal of the given values with the reference's
 *     guard (1/d where |d| > 0, else 1). Stats and return codes as jxb_pcg,
 *     the residual being |b - A x| over all rows. */
typedef struct jxb_csr jxb_csr;
int jxb_csr_create(int64_t n, const int64_t* indptr, const int32_t* cols, jxb_csr** out);
int jxb_csr_destroy(jxb_csr* csr);
int jxb_csr_matvec(jxb_csr* csr, jxb_stream stream, const double* values, const double* x, double* y);
int jxb_csr_pcg(jxb_csr* csr, jxb_stream stream, const double* values, const double* b, double* x,
                const jxb_solve_opts* opts, jxb_stats* stats);

/* ---- vector helpers used by hosts that drive their own Krylov loop ---- */
int jxb_dot(jxb_plan* plan, jxb_stream stream, const double* a, const double* b, double* out_host);

/* ---- measurement --------------------------------------------------------
 * jxb_profile_apply: runs `reps` masked applies (FP64, or FP32 when f32 != 0,
 *   x/y then being float*) and returns in ms_out[0] / ms_out[1] the average
 *   device time of one brick launch / one combine launch, measured with CUDA
 *   events on `stream`. Blocks until done. No counterpart in the reference
 *   (which has no kernels of its own to time). */
int jxb_profile_apply(jxb_plan* plan, jxb_stream stream, const void* x, void* y, int reps, int f32,
                      double* ms_out);

#ifdef __cplusplus
}
#endif
#endif /* JXB_H */
