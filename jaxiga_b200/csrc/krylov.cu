// BiCGSTAB on the device: the reference's `method="bicgstab"`
// (src/jaxiga/solvers/linear.py:152-171, 399-411), which runs
// jax.scipy.sparse.linalg.bicgstab with the Jacobi preconditioner on the
// matrix-free operator.
//
// The iteration is van der Vorst's BiCGSTAB (1992) with right
// preconditioning M = D^-1 on the free DOFs: from x0 = 0, r = b, rhat = r,
//   rho = rhat.r;  beta = (rho / rho_old) (alpha / omega);
//   p = r + beta (p - omega v);  v = K M p;  alpha = rho / rhat.v;
//   s = r - alpha v;  if s.s <= atol2: x += alpha M p, r = s, stop;
//   t = K M s;  omega = t.s / t.t;  x += alpha M p + omega M s;  r = s - omega t,
// stopping when r.r <= max(tol^2 b.b, atol^2) or at maxiter, and reporting a
// breakdown (rho, alpha or omega zero) as non-finite. Scalars live in device
// memory and every kernel first reads the done flag, so `check_every`
// iterations are one captured CUDA graph, as for CG.
#include <math.h>

#include <vector>

#include "jxb_internal.cuh"

namespace jxb {
namespace {

// cg first: the brick and combine kernels read cg.done as their skip flag
struct BsState {
  CgState cg;  // k, maxiter, atol2, done and status of the solve
  double rho, alpha, omega, beta, rs, ss;
  int early;
};

constexpr int RB = JXB_RED_BLOCKS, RT = JXB_RED_THREADS;

__global__ void __launch_bounds__(RT) k_bs_init(long long n, const double* __restrict__ b, const uint8_t* __restrict__ keep,
                                                 double* x, double* r, double* rhat, double* p, double* v,
                                                 double* part) {
  double bb = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double bi = keep[i] ? b[i] : 0.0;
    x[i] = 0;
    r[i] = bi;
    rhat[i] = bi;
    p[i] = 0;
    v[i] = 0;
    bb += bi * bi;
  }
  const double s = block_sum_all(bb);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void k_bs_start(BsState* st, const double* part, double tol, double atol, long long maxiter) {
  const double bb = reduce_partials(part);
  if (threadIdx.x == 0) {
    st->rho = st->alpha = st->omega = 1.0;
    st->beta = 0;
    st->rs = bb;
    st->cg.atol2 = fmax(tol * tol * bb, atol * atol);
    st->cg.k = 0;
    st->cg.maxiter = maxiter;
    st->cg.status = JXB_OK;
    st->early = 0;
    st->cg.done = 0;
    if (!isfinite(bb)) {
      st->cg.done = 1;
      st->cg.status = JXB_ERR_NONFINITE;
    } else if (!(bb > st->cg.atol2)) {
      st->cg.done = 1;
    } else if (maxiter <= 0) {
      st->cg.done = 1;
      st->cg.status = JXB_ERR_NOT_CONVERGED;
    }
  }
}

// partials of a . b (slot 0) and, with c, c . d (slot 1)
__global__ void __launch_bounds__(RT) k_bs_dot2(const BsState* st, long long n, const double* __restrict__ a,
                                                 const double* __restrict__ b, const double* __restrict__ c,
                                                 const double* __restrict__ d, double* part) {
  if (st->cg.done) return;
  double s0 = 0, s1 = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    s0 += a[i] * b[i];
    if (c) s1 += c[i] * d[i];
  }
  const double t0 = block_sum_all(s0), t1 = block_sum_all(s1);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = t0;
    part[RB + blockIdx.x] = t1;
  }
}

// rho_new = rhat.r; beta
__global__ void k_bs_beta(BsState* st, const double* part) {
  if (st->cg.done) return;
  const double rho = reduce_partials(part);
  if (threadIdx.x == 0) {
    if (!(rho != 0.0) || !isfinite(rho)) {
      st->cg.done = 1;
      st->cg.status = JXB_ERR_NONFINITE;
      return;
    }
    st->beta = (rho / st->rho) * (st->alpha / st->omega);
    st->rho = rho;
  }
}

// p = r + beta (p - omega v); phat = M p
__global__ void k_bs_p(const BsState* st, long long n, const double* __restrict__ r, const double* __restrict__ v,
                       const double* __restrict__ inv, double* p, double* phat) {
  if (st->cg.done) return;
  const double beta = st->beta, omega = st->omega;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double pi = r[i] + beta * (p[i] - omega * v[i]);
    p[i] = pi;
    phat[i] = inv[i] * pi;
  }
}

// alpha = rho / rhat.v (partials in slot 0 from the combine)
__global__ void k_bs_alpha(BsState* st, const double* part) {
  if (st->cg.done) return;
  const double rv = reduce_partials(part);
  if (threadIdx.x == 0) {
    const double a = st->rho / rv;
    if (!(rv != 0.0) || !isfinite(a)) {
      st->cg.done = 1;
      st->cg.status = JXB_ERR_NONFINITE;
      return;
    }
    st->alpha = a;
  }
}

// s = r - alpha v (into r's storage); shat = M s; partials s.s
__global__ void __launch_bounds__(RT) k_bs_s(const BsState* st, long long n, double* r, const double* __restrict__ v,
                                              const double* __restrict__ inv, double* shat, double* part) {
  if (st->cg.done) return;
  const double alpha = st->alpha;
  double ss = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double si = r[i] - alpha * v[i];
    r[i] = si;
    shat[i] = inv[i] * si;
    ss += si * si;
  }
  const double t = block_sum_all(ss);
  if (threadIdx.x == 0) part[2 * RB + blockIdx.x] = t;
}

__global__ void k_bs_early(BsState* st, const double* part) {
  if (st->cg.done) return;
  const double ss = reduce_partials(part + 2 * RB);
  if (threadIdx.x == 0) {
    st->ss = ss;
    st->early = !(ss > st->cg.atol2);
  }
}

// omega = t.s / t.t (slot 0: t.s, slot 1: t.t) unless the s test stopped early
__global__ void k_bs_omega(BsState* st, const double* part) {
  if (st->cg.done || st->early) return;
  const double ts = reduce_partials(part), tt = reduce_partials(part + RB);
  if (threadIdx.x == 0) {
    const double w = ts / tt;
    if (!(tt > 0) || !(w != 0.0) || !isfinite(w)) {
      st->cg.done = 1;
      st->cg.status = JXB_ERR_NONFINITE;
      return;
    }
    st->omega = w;
  }
}

// x += alpha phat (+ omega shat); r = s (- omega t); partials r.r
__global__ void __launch_bounds__(RT) k_bs_xr(const BsState* st, long long n, double* x, double* r,
                                               const double* __restrict__ phat, const double* __restrict__ shat,
                                               const double* __restrict__ t, double* part) {
  if (st->cg.done) return;
  const double alpha = st->alpha, omega = st->early ? 0.0 : st->omega;
  double rr = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    x[i] += alpha * phat[i] + omega * shat[i];
    const double ri = r[i] - omega * t[i];
    r[i] = ri;
    rr += ri * ri;
  }
  const double s = block_sum_all(rr);
  if (threadIdx.x == 0) part[3 * RB + blockIdx.x] = s;
}

__global__ void k_bs_fin(BsState* st, const double* part) {
  if (st->cg.done) return;
  const double rr = reduce_partials(part + 3 * RB);
  if (threadIdx.x == 0) {
    st->rs = rr;
    st->cg.k += 1;
    if (!isfinite(rr)) {
      st->cg.done = 1;
      st->cg.status = JXB_ERR_NONFINITE;
    } else if (!(rr > st->cg.atol2)) {
      st->cg.done = 1;
      st->cg.status = JXB_OK;
    } else if (st->cg.k >= st->cg.maxiter) {
      st->cg.done = 1;
      st->cg.status = JXB_ERR_NOT_CONVERGED;
    }
  }
}

inline unsigned grid_n(long long n) {
  long long g = (n + 255) / 256;
  return (unsigned)(g < 4 * 148 ? (g < 1 ? 1 : g) : 4 * 148);
}

}  // namespace
}  // namespace jxb

struct jxb_krylov_ws {
  double *x = nullptr, *r = nullptr, *rhat = nullptr, *p = nullptr, *v = nullptr, *phat = nullptr, *shat = nullptr,
         *t = nullptr, *b = nullptr, *part = nullptr;
  jxb::BsState* st = nullptr;
  jxb::BsState* h_st = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graph_iters = 0;
};

namespace jxb {

void free_krylov(jxb_plan* P) {
  jxb_krylov_ws* W = P->krylov;
  if (!W) return;
  if (W->graph) cudaGraphExecDestroy(W->graph);
  void* bufs[] = {W->x, W->r, W->rhat, W->p, W->v, W->phat, W->shat, W->t, W->b, W->part, W->st};
  for (void* b : bufs) cudaFree(b);
  if (W->h_st) cudaFreeHost(W->h_st);
  delete W;
  P->krylov = nullptr;
}

namespace {

int krylov_ws(jxb_plan* P) {
  if (P->krylov) return JXB_OK;
  jxb_krylov_ws* W = new jxb_krylov_ws();
  P->krylov = W;
  const size_t n = (size_t)P->n_dofs;
  cudaError_t e = cudaSuccess;
  for (double** p : {&W->x, &W->r, &W->rhat, &W->p, &W->v, &W->phat, &W->shat, &W->t, &W->b})
    if (e == cudaSuccess) e = cudaMalloc(p, n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&W->part, 4 * RB * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&W->st, sizeof(BsState));
  if (e == cudaSuccess) e = cudaMallocHost(&W->h_st, sizeof(BsState));
  if (e != cudaSuccess) {
    free_krylov(P);
    return cuda_fail(e, "bicgstab workspace");
  }
  return JXB_OK;
}

int bs_iteration(jxb_plan* P, cudaStream_t s) {
  jxb_krylov_ws* W = P->krylov;
  const long long n = P->n_dofs;
  const CgState* gate = &W->st->cg;  // the applies skip once the solve is done
  k_bs_dot2<<<RB, RT, 0, s>>>(W->st, n, W->rhat, W->r, nullptr, nullptr, W->part);
  k_bs_beta<<<1, RT, 0, s>>>(W->st, W->part);
  k_bs_p<<<grid_n(n), 256, 0, s>>>(W->st, n, W->r, W->v, P->d_invdiag, W->p, W->phat);
  int rc = launch_bricks<double>(P, s, MODE_APPLY, W->phat, nullptr, gate, 1);
  if (rc) return rc;
  if ((rc = launch_combine<double>(P, s, W->v, 1, W->rhat, W->part, gate))) return rc;
  k_bs_alpha<<<1, RT, 0, s>>>(W->st, W->part);
  k_bs_s<<<RB, RT, 0, s>>>(W->st, n, W->r, W->v, P->d_invdiag, W->shat, W->part);
  k_bs_early<<<1, RT, 0, s>>>(W->st, W->part);
  if ((rc = launch_bricks<double>(P, s, MODE_APPLY, W->shat, nullptr, gate, 1))) return rc;
  if ((rc = launch_combine<double>(P, s, W->t, 1, nullptr, nullptr, gate))) return rc;
  k_bs_dot2<<<RB, RT, 0, s>>>(W->st, n, W->t, W->r, W->t, W->t, W->part);
  k_bs_omega<<<1, RT, 0, s>>>(W->st, W->part);
  k_bs_xr<<<RB, RT, 0, s>>>(W->st, n, W->x, W->r, W->phat, W->shat, W->t, W->part);
  k_bs_fin<<<1, RT, 0, s>>>(W->st, W->part);
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

}  // namespace
}  // namespace jxb

using namespace jxb;

extern "C" int jxb_bicgstab(jxb_plan* plan, jxb_stream stream, const double* b, double* x, const jxb_solve_opts* opts,
                            jxb_stats* stats) {
  if (plan && (plan->mp || plan->thb)) return fail(JXB_ERR_INVALID, "jxb_bicgstab: not available on a multipatch or hierarchical plan");
  if (!plan || !b || !x || !opts) return fail(JXB_ERR_INVALID, "jxb_bicgstab: null argument");
  if (!(opts->tol > 0) || !isfinite(opts->tol)) return fail(JXB_ERR_INVALID, "jxb_bicgstab: tol must be finite and positive");
  cudaStream_t user = reinterpret_cast<cudaStream_t>(stream);
  if (!plan->graph_stream[0]) JXB_CUDA(cudaStreamCreateWithFlags(&plan->graph_stream[0], cudaStreamNonBlocking));
  cudaStream_t s = plan->graph_stream[0];
  SolveEvents ev;
  int rc = ev.create();
  if (rc) return rc;
  JXB_CUDA(cudaEventRecord(ev.order, user));
  JXB_CUDA(cudaStreamWaitEvent(s, ev.order, 0));
  if ((rc = ensure_workspace(plan, false))) return rc;
  if ((rc = krylov_ws(plan))) return rc;
  jxb_krylov_ws* W = plan->krylov;
  if (opts->preconditioner) {
    if ((rc = compute_invdiag(plan, s))) return rc;
  } else {
    // no preconditioner: M = identity on the free DOFs
    std::vector<double> ones(plan->n_dofs);
    std::vector<uint8_t> keep(plan->n_dofs);
    JXB_CUDA(cudaMemcpyAsync(keep.data(), plan->d_keep, plan->n_dofs, cudaMemcpyDeviceToHost, s));
    JXB_CUDA(cudaStreamSynchronize(s));
    for (long long i = 0; i < plan->n_dofs; ++i) ones[i] = keep[i] ? 1.0 : 0.0;
    JXB_CUDA(cudaMemcpyAsync(plan->d_invdiag, ones.data(), plan->n_dofs * sizeof(double), cudaMemcpyHostToDevice, s));
    JXB_CUDA(cudaStreamSynchronize(s));
    plan->diag_valid = false;  // d_invdiag now holds the identity
  }
  const long long n = plan->n_dofs;
  const long long maxiter = opts->maxiter > 0 ? opts->maxiter : 10 * plan->n_free;
  const int every = opts->check_every > 0 ? opts->check_every : 16;
  if (!W->graph || W->graph_iters != every) {
    if (W->graph) cudaGraphExecDestroy(W->graph);
    W->graph = nullptr;
    cudaGraph_t g;
    JXB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    int rci = 0;
    for (int it = 0; it < every && !rci; ++it) rci = bs_iteration(plan, s);
    cudaError_t ce = cudaStreamEndCapture(s, &g);
    if (rci) return rci;
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
    ce = cudaGraphInstantiate(&W->graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaGraphInstantiate");
    W->graph_iters = every;
  }
  JXB_CUDA(cudaMemcpyAsync(W->b, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  JXB_CUDA(cudaEventRecord(ev.e0, s));
  k_bs_init<<<RB, RT, 0, s>>>(n, W->b, plan->d_keep, W->x, W->r, W->rhat, W->p, W->v, W->part);
  k_bs_start<<<1, RT, 0, s>>>(W->st, W->part, opts->tol, opts->atol, maxiter);
  JXB_CUDA(cudaGetLastError());
  JXB_CUDA(cudaMemcpyAsync(W->h_st, W->st, sizeof(BsState), cudaMemcpyDeviceToHost, s));
  JXB_CUDA(cudaStreamSynchronize(s));
  const long long launches = maxiter / every + 2;
  for (long long l = 0; l < launches && !W->h_st->cg.done; ++l) {
    JXB_CUDA(cudaGraphLaunch(W->graph, s));
    JXB_CUDA(cudaMemcpyAsync(W->h_st, W->st, sizeof(BsState), cudaMemcpyDeviceToHost, s));
    JXB_CUDA(cudaStreamSynchronize(s));
  }
  JXB_CUDA(cudaEventRecord(ev.e1, s));
  const long long iters = W->h_st->cg.k;
  const int status = W->h_st->cg.done ? W->h_st->cg.status : JXB_ERR_NOT_CONVERGED;
  JXB_CUDA(cudaMemcpyAsync(x, W->x, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  double rn = 0, bn = 0;
  bool fin = true;
  if ((rc = true_residual(plan, s, W->b, W->x, nullptr, &rn, &bn, &fin))) return rc;
  JXB_CUDA(cudaEventRecord(ev.order, s));
  JXB_CUDA(cudaStreamWaitEvent(user, ev.order, 0));
  float ms = 0;
  JXB_CUDA(cudaEventElapsedTime(&ms, ev.e0, ev.e1));
  return finish_solve("jxb_bicgstab", stats, iters, 0, rn, bn, fin, opts->tol, opts->atol, ms,
                      status == JXB_ERR_NONFINITE);
}
