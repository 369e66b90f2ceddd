// Preconditioned CG on the device (K4), true residual (K5) and FP64
// iterative refinement around FP32 inner solves.
//
// The iteration follows jax.scipy.sparse.linalg.cg (jax 0.11.1, the solver
// behind src/jaxiga/solvers/linear.py:399-442): x0 = 0, p0 = z0 = M r0,
// stop when r.r <= max(tol^2 b.b, atol^2) or k == maxiter (10 n by default).
//
// One iteration is five launches -- brick apply, combine (+ p.Ap partials),
// x/r/z update (+ r.z, r.r partials), p update, scalar finish -- recorded
// once into a CUDA graph of `check_every` iterations. Every kernel first reads
// the device `done` flag, so iterations past convergence are no-ops and the
// iteration count is exact. The host reads the 64-byte state back once per
// graph launch. All reductions use a fixed grid and a fixed summation order,
// so results are bitwise reproducible run to run.
#include <math.h>
#include <stdio.h>

#include <string>
#include <vector>

#include "jxb_internal.cuh"

namespace jxb {

template <typename T, typename TB>
__global__ void __launch_bounds__(JXB_RED_THREADS) k_cg_init(long long n, const TB* __restrict__ b, const uint8_t* __restrict__ keep,
                          const T* __restrict__ invdiag, int precond, T* x, T* r, T* z, T* p,
                          double* partials) {
  double rz = 0, rr = 0, bb = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    T bi = keep[i] ? (T)b[i] : T(0);
    T zi = precond ? invdiag[i] * bi : bi;
    x[i] = 0;
    r[i] = bi;
    z[i] = zi;
    p[i] = zi;
    rz += (double)bi * (double)zi;
    rr += (double)bi * (double)bi;
  }
  bb = rr;
  double s0 = block_sum_all(rz), s1 = block_sum_all(rr), s2 = block_sum_all(bb);
  if (threadIdx.x == 0) {
    partials[JXB_RED_BLOCKS + blockIdx.x] = s0;
    partials[2 * JXB_RED_BLOCKS + blockIdx.x] = s1;
    partials[3 * JXB_RED_BLOCKS + blockIdx.x] = s2;
  }
}

__global__ void k_cg_init_fin(CgState* st, const double* partials, double tol, double atol,
                              long long maxiter) {
  double gamma = reduce_partials(partials + JXB_RED_BLOCKS);
  double rr = reduce_partials(partials + 2 * JXB_RED_BLOCKS);
  double bb = reduce_partials(partials + 3 * JXB_RED_BLOCKS);
  if (threadIdx.x == 0) {
    st->gamma = gamma;
    st->rr = rr;
    st->bb = bb;
    st->atol2 = fmax(tol * tol * bb, atol * atol);
    st->k = 0;
    st->maxiter = maxiter;
    st->alpha = st->beta = 0;
    st->status = JXB_OK;
    st->done = 0;
    if (!isfinite(rr) || !isfinite(gamma)) {
      st->done = 1;
      st->status = JXB_ERR_NONFINITE;
    } else if (!(rr > st->atol2)) {
      st->done = 1;
    } else if (maxiter <= 0) {
      st->done = 1;
      st->status = JXB_ERR_NOT_CONVERGED;
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(JXB_RED_THREADS) k_cg_xr(long long n, const CgState* st, double* partials, T* x, T* r, T* z,
                        const T* __restrict__ p, const T* __restrict__ Ap,
                        const T* __restrict__ invdiag, int precond) {
  if (st->done) return;
  double pAp = reduce_partials(partials);
  double alpha_d = st->gamma / pAp;
  T alpha = (T)alpha_d;
  double rz = 0, rr = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    T pi = p[i];
    x[i] += alpha * pi;
    T ri = r[i] - alpha * Ap[i];
    r[i] = ri;
    T zi = precond ? invdiag[i] * ri : ri;
    z[i] = zi;
    rz += (double)ri * (double)zi;
    rr += (double)ri * (double)ri;
  }
  double s0 = block_sum_all(rz), s1 = block_sum_all(rr);
  if (threadIdx.x == 0) {
    partials[JXB_RED_BLOCKS + blockIdx.x] = s0;
    partials[2 * JXB_RED_BLOCKS + blockIdx.x] = s1;
  }
}

template <typename T>
__global__ void __launch_bounds__(JXB_RED_THREADS) k_cg_p(long long n, const CgState* st, const double* partials, const T* __restrict__ z, T* p) {
  if (st->done) return;
  double gnew = reduce_partials(partials + JXB_RED_BLOCKS);
  T beta = (T)(gnew / st->gamma);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    p[i] = z[i] + beta * p[i];
}

__global__ void k_cg_fin(CgState* st, const double* partials) {
  if (st->done) return;
  double pAp = reduce_partials(partials);
  double gnew = reduce_partials(partials + JXB_RED_BLOCKS);
  double rr = reduce_partials(partials + 2 * JXB_RED_BLOCKS);
  if (threadIdx.x == 0) {
    st->alpha = st->gamma / pAp;
    st->beta = gnew / st->gamma;
    st->gamma = gnew;
    st->rr = rr;
    st->k += 1;
    if (!isfinite(rr) || !isfinite(gnew) || !isfinite(pAp) || pAp == 0.0) {
      st->done = 1;
      st->status = JXB_ERR_NONFINITE;
    } else if (!(rr > st->atol2)) {
      st->done = 1;
      st->status = JXB_OK;
    } else if (st->k >= st->maxiter) {
      st->done = 1;
      st->status = JXB_ERR_NOT_CONVERGED;
    }
  }
}

// res = b - Ax on free DOFs; partials: ||res||^2, ||b||^2, non-finite count of x
template <typename TX>
__global__ void __launch_bounds__(JXB_RED_THREADS) k_residual(long long n, const double* __restrict__ b, const double* __restrict__ Ax,
                           const TX* __restrict__ x, const uint8_t* __restrict__ keep, double* res,
                           double* partials) {
  double rr = 0, bb = 0, bad = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double ri = 0, bi = 0;
    if (keep[i]) {
      bi = b[i];
      ri = bi - Ax[i];
    }
    if (res) res[i] = ri;
    rr += ri * ri;
    bb += bi * bi;
    if (x && !isfinite((double)x[i])) bad += 1;
  }
  double s0 = block_sum_all(rr), s1 = block_sum_all(bb), s2 = block_sum_all(bad);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = s0;
    partials[JXB_RED_BLOCKS + blockIdx.x] = s1;
    partials[2 * JXB_RED_BLOCKS + blockIdx.x] = s2;
  }
}

__global__ void __launch_bounds__(JXB_RED_THREADS) k_dot(long long n, const double* a, const double* b, double* partials) {
  double s = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    s += a[i] * b[i];
  double t = block_sum_all(s);
  if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

__global__ void k_invdiag(long long n, const double* d, const uint8_t* keep, double* inv, float* inv32) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // solvers/linear.py:427-431: 1/d where |d| > 0, else 1 (prescribed rows never enter)
  double v = d[i];
  double w = keep[i] ? (fabs(v) > 0 ? 1.0 / v : 1.0) : 0.0;
  inv[i] = w;
  if (inv32) inv32[i] = (float)w;
}

__global__ void k_scale_to_f32(long long n, const double* r, double s, float* out) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (float)(r[i] * s);
}

__global__ void k_axpy_from_f32(long long n, double a, const float* d, double* x) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += a * (double)d[i];
}

// (Re)start of the FP32 iteration from an FP64 residual (reliable update):
// r32 = s res, z32 = M r32, x32 = 0. On the first start p32 = z32; later the
// search direction is kept and only rescaled to the new units (p32 *= ratio),
// so the Krylov recurrence carries on instead of starting over. Partials as
// k_cg_init: r.z, r.r and r.r again in the ||b||^2 slot (the FP32 right-hand
// side is the scaled residual).
__global__ void __launch_bounds__(JXB_RED_THREADS) k_ru_restart(long long n, const double* __restrict__ res,
                                                                const uint8_t* __restrict__ keep,
                                                                const float* __restrict__ inv, double s, float ratio,
                                                                int first, float* x, float* r, float* z, float* p,
                                                                double* partials) {
  double rz = 0, rr = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float ri = keep[i] ? (float)(res[i] * s) : 0.f;
    const float zi = inv[i] * ri;
    x[i] = 0.f;
    r[i] = ri;
    z[i] = zi;
    p[i] = first ? zi : p[i] * ratio;
    rz += (double)ri * (double)zi;
    rr += (double)ri * (double)ri;
  }
  double s0 = block_sum_all(rz), s1 = block_sum_all(rr);
  if (threadIdx.x == 0) {
    partials[JXB_RED_BLOCKS + blockIdx.x] = s0;
    partials[2 * JXB_RED_BLOCKS + blockIdx.x] = s1;
    partials[3 * JXB_RED_BLOCKS + blockIdx.x] = s1;
  }
}

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------
int ensure_workspace(jxb_plan* plan, bool f32) {
  size_t n = (size_t)plan->n_dofs;
  auto alloc = [&](double** p) -> int {
    if (!*p) JXB_CUDA(cudaMalloc(p, n * sizeof(double)));
    return 0;
  };
  auto allocf = [&](float** p) -> int {
    if (!*p) JXB_CUDA(cudaMalloc(p, n * sizeof(float)));
    return 0;
  };
  int e = 0;
  e |= alloc(&plan->d_x);
  e |= alloc(&plan->d_b);
  e |= alloc(&plan->d_r);
  e |= alloc(&plan->d_z);
  e |= alloc(&plan->d_p);
  e |= alloc(&plan->d_Ap);
  e |= alloc(&plan->d_invdiag);
  if (f32) {
    e |= allocf(&plan->d_x32);
    e |= allocf(&plan->d_r32);
    e |= allocf(&plan->d_z32);
    e |= allocf(&plan->d_p32);
    e |= allocf(&plan->d_Ap32);
    e |= allocf(&plan->d_invdiag32);
  }
  if (e) return e;
  if (!plan->d_state) JXB_CUDA(cudaMalloc(&plan->d_state, sizeof(CgState)));
  if (!plan->h_state) JXB_CUDA(cudaMallocHost(&plan->h_state, sizeof(CgState)));
  return JXB_OK;
}

int compute_invdiag(jxb_plan* plan, cudaStream_t s) {
  if (plan->diag_valid) return JXB_OK;
  int rc = launch_bricks<double>(plan, s, MODE_DIAG, nullptr, nullptr, nullptr, 1);
  if (rc) return rc;
  rc = launch_combine<double>(plan, s, plan->d_Ap, 1, nullptr, nullptr, nullptr);
  if (rc) return rc;
  long long n = plan->n_dofs;
  if (!plan->d_invdiag32) JXB_CUDA(cudaMalloc(&plan->d_invdiag32, n * sizeof(float)));
  k_invdiag<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, plan->d_Ap, plan->d_keep, plan->d_invdiag,
                                                         plan->d_invdiag32);
  JXB_CUDA(cudaGetLastError());
  plan->diag_valid = true;
  return JXB_OK;
}

static double host_sum(const std::vector<double>& v, int off) {
  double s = 0;
  for (int i = 0; i < JXB_RED_BLOCKS; ++i) s += v[off + i];
  return s;
}

int dot(jxb_plan* plan, cudaStream_t s, const double* a, const double* b, double* out_host) {
  k_dot<<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(plan->n_dofs, a, b, plan->d_red);
  JXB_CUDA(cudaGetLastError());
  std::vector<double> h(JXB_RED_BLOCKS);
  JXB_CUDA(cudaMemcpyAsync(h.data(), plan->d_red, JXB_RED_BLOCKS * sizeof(double), cudaMemcpyDeviceToHost, s));
  JXB_CUDA(cudaStreamSynchronize(s));
  *out_host = host_sum(h, 0);
  return JXB_OK;
}

// ||b - A x|| over free DOFs (FP64 apply); optionally keeps the residual vector.
int true_residual(jxb_plan* plan, cudaStream_t s, const double* b, const double* x,
                  double* res_out, double* rnorm, double* bnorm, bool* finite) {
  int rc = launch_bricks<double>(plan, s, MODE_APPLY, x, nullptr, nullptr, 1);
  if (rc) return rc;
  rc = launch_combine<double>(plan, s, plan->d_Ap, 1, nullptr, nullptr, nullptr);
  if (rc) return rc;
  k_residual<double><<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(plan->n_dofs, b, plan->d_Ap, x, plan->d_keep,
                                                                 res_out, plan->d_red);
  JXB_CUDA(cudaGetLastError());
  std::vector<double> h(3 * JXB_RED_BLOCKS);
  JXB_CUDA(cudaMemcpyAsync(h.data(), plan->d_red, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  JXB_CUDA(cudaStreamSynchronize(s));
  *rnorm = sqrt(host_sum(h, 0));
  *bnorm = sqrt(host_sum(h, JXB_RED_BLOCKS));
  *finite = host_sum(h, 2 * JXB_RED_BLOCKS) == 0 && isfinite(*rnorm);
  return JXB_OK;
}

// Record `iters` CG iterations into a graph on stream s.
template <typename T>
static int record_iterations(jxb_plan* plan, cudaStream_t s, int iters, int precond) {
  constexpr bool F32 = sizeof(T) == 4;
  T* x = F32 ? (T*)plan->d_x32 : (T*)plan->d_x;
  T* r = F32 ? (T*)plan->d_r32 : (T*)plan->d_r;
  T* z = F32 ? (T*)plan->d_z32 : (T*)plan->d_z;
  T* p = F32 ? (T*)plan->d_p32 : (T*)plan->d_p;
  T* Ap = F32 ? (T*)plan->d_Ap32 : (T*)plan->d_Ap;
  const T* inv = F32 ? (const T*)plan->d_invdiag32 : (const T*)plan->d_invdiag;
  long long n = plan->n_dofs;
  for (int it = 0; it < iters; ++it) {
    int rc = launch_bricks<T>(plan, s, MODE_APPLY, p, nullptr, plan->d_state, 1);
    if (rc) return rc;
    rc = launch_combine<T>(plan, s, Ap, 1, p, plan->d_red, plan->d_state);
    if (rc) return rc;
    k_cg_xr<T><<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(n, plan->d_state, plan->d_red, x, r, z, p, Ap, inv, precond);
    k_cg_p<T><<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(n, plan->d_state, plan->d_red, z, p);
    k_cg_fin<<<1, JXB_RED_THREADS, 0, s>>>(plan->d_state, plan->d_red);
  }
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

template <typename T>
static int get_graph(jxb_plan* plan, cudaStream_t s, int iters, int precond, cudaGraphExec_t* out) {
  int slot = sizeof(T) == 4 ? 1 : 0;
  if (plan->graph[slot] && plan->graph_iters[slot] == iters && plan->graph_precond[slot] == precond) {
    *out = plan->graph[slot];
    return JXB_OK;
  }
  if (plan->graph[slot]) {
    cudaGraphExecDestroy(plan->graph[slot]);
    plan->graph[slot] = nullptr;
  }
  cudaGraph_t g;
  // relaxed: the launchers set kernel attributes (not stream work) while recording
  JXB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
  int rc = record_iterations<T>(plan, s, iters, precond);
  cudaError_t e = cudaStreamEndCapture(s, &g);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(&plan->graph[slot], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
  plan->graph_iters[slot] = iters;
  plan->graph_precond[slot] = precond;
  *out = plan->graph[slot];
  return JXB_OK;
}

template <typename T>
static int iterate(jxb_plan* plan, cudaStream_t s, long long maxiter, int precond, int check_every,
                   long long* iters, int* status, double* snaps, long long max_snaps, long long* n_snaps);

// Runs CG on the plan-owned vectors (b given as TB*), solution left in plan x.
template <typename T, typename TB>
static int run_cg(jxb_plan* plan, cudaStream_t s, const TB* b, double tol, double atol, long long maxiter,
                  int precond, int check_every, long long* iters, int* status, double* snaps = nullptr,
                  long long max_snaps = 0, long long* n_snaps = nullptr) {
  constexpr bool F32 = sizeof(T) == 4;
  T* x = F32 ? (T*)plan->d_x32 : (T*)plan->d_x;
  T* r = F32 ? (T*)plan->d_r32 : (T*)plan->d_r;
  T* z = F32 ? (T*)plan->d_z32 : (T*)plan->d_z;
  T* p = F32 ? (T*)plan->d_p32 : (T*)plan->d_p;
  const T* inv = F32 ? (const T*)plan->d_invdiag32 : (const T*)plan->d_invdiag;
  long long n = plan->n_dofs;
  k_cg_init<T, TB><<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(n, b, plan->d_keep, inv, precond, x, r, z, p, plan->d_red);
  k_cg_init_fin<<<1, JXB_RED_THREADS, 0, s>>>(plan->d_state, plan->d_red, tol, atol, maxiter);
  JXB_CUDA(cudaGetLastError());
  return iterate<T>(plan, s, maxiter, precond, check_every, iters, status, snaps, max_snaps, n_snaps);
}

// Launches the captured iteration graph until the device state reports done
// (the state and the vectors were set up by the caller).
template <typename T>
static int iterate(jxb_plan* plan, cudaStream_t s, long long maxiter, int precond, int check_every,
                   long long* iters, int* status, double* snaps, long long max_snaps, long long* n_snaps) {
  const double* x = plan->d_x;
  cudaGraphExec_t ge;
  int rc = get_graph<T>(plan, s, check_every, precond, &ge);
  if (rc) return rc;
  long long launches = maxiter / check_every + 2;
  JXB_CUDA(cudaMemcpyAsync(plan->h_state, plan->d_state, sizeof(CgState), cudaMemcpyDeviceToHost, s));
  JXB_CUDA(cudaStreamSynchronize(s));
  long long ns = 0;
  for (long long l = 0; l < launches && !plan->h_state->done; ++l) {
    JXB_CUDA(cudaGraphLaunch(ge, s));
    JXB_CUDA(cudaMemcpyAsync(plan->h_state, plan->d_state, sizeof(CgState), cudaMemcpyDeviceToHost, s));
    JXB_CUDA(cudaStreamSynchronize(s));
    if constexpr (sizeof(T) == 8) {
      if (snaps && ns < max_snaps && !plan->h_state->done) {  // iterate after l+1 graph launches
        JXB_CUDA(cudaMemcpyAsync(snaps + ns * plan->n_dofs, x, plan->n_dofs * sizeof(double),
                                 cudaMemcpyDeviceToDevice, s));
        ++ns;
      }
    }
  }
  if (n_snaps) *n_snaps = ns;
  *iters = plan->h_state->k;
  *status = plan->h_state->done ? plan->h_state->status : JXB_ERR_NOT_CONVERGED;
  return JXB_OK;
}

}  // namespace jxb

using namespace jxb;

namespace jxb {

__global__ void k_add(long long n, const double* a, const double* b, double* out) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] + b[i];
}

int finish_solve(const char* who, jxb_stats* stats, long long iters, long long outer, double rn, double bn, bool fin,
                 double tol, double atol, float ms, bool nonfinite) {
  // the stopping rule of jax's CG: ||r|| <= max(tol ||b||, atol)
  const bool conv = fin && isfinite(rn) && rn <= fmax(tol * bn, atol);
  if (stats) {
    stats->iterations = iters;
    stats->outer = outer;
    stats->residual = rn;
    stats->b_norm = bn;
    stats->relative_residual = rn / (bn > 0 ? bn : 1.0);
    stats->finite = (fin && isfinite(rn)) ? 1 : 0;
    stats->converged = conv ? 1 : 0;
    stats->seconds = ms * 1e-3;
  }
  if (nonfinite) return fail(JXB_ERR_NONFINITE, std::string(who) + ": non-finite value in the Krylov reductions");
  if (!conv) {
    char buf[160];
    snprintf(buf, sizeof buf, "%s: not converged (true residual %.3e > %.3e after %lld iterations)", who, rn,
             fmax(tol * bn, atol), iters);
    return fail(JXB_ERR_NOT_CONVERGED, buf);
  }
  return JXB_OK;
}

// Solve-local stream set-up shared by the entry points: plan stream `slot`
// created on first use, ordered after the caller's stream.
static int enter_stream(jxb_plan* plan, int slot, cudaStream_t user, SolveEvents& ev, cudaStream_t* out) {
  if (!plan->graph_stream[slot])
    JXB_CUDA(cudaStreamCreateWithFlags(&plan->graph_stream[slot], cudaStreamNonBlocking));
  int rc = ev.create();
  if (rc) return rc;
  JXB_CUDA(cudaEventRecord(ev.order, user));
  JXB_CUDA(cudaStreamWaitEvent(plan->graph_stream[slot], ev.order, 0));
  *out = plan->graph_stream[slot];
  return JXB_OK;
}

// Hands the plan stream's work back to the caller's stream and reads the
// device time between e0 and e1.
static int leave_stream(cudaStream_t s, cudaStream_t user, SolveEvents& ev, float* ms) {
  JXB_CUDA(cudaEventRecord(ev.order, s));
  JXB_CUDA(cudaStreamWaitEvent(user, ev.order, 0));
  JXB_CUDA(cudaEventSynchronize(ev.e1));
  JXB_CUDA(cudaEventElapsedTime(ms, ev.e0, ev.e1));
  return JXB_OK;
}

}  // namespace jxb

extern "C" int jxb_pcg(jxb_plan* plan, jxb_stream stream, const double* b, double* x,
                       const jxb_solve_opts* opts, jxb_stats* stats) {
  if (!plan || !b || !x || !opts) return fail(JXB_ERR_INVALID, "jxb_pcg: null argument");
  if (!(opts->tol > 0) || !isfinite(opts->tol)) return fail(JXB_ERR_INVALID, "jxb_pcg: tol must be finite and positive");
  if (opts->restarts < 0 || opts->restarts > 8) return fail(JXB_ERR_INVALID, "jxb_pcg: restarts must be in 0..8");
  cudaStream_t user = reinterpret_cast<cudaStream_t>(stream), s = nullptr;
  SolveEvents ev;
  int rc = enter_stream(plan, 0, user, ev, &s);
  if (rc) return rc;
  if ((rc = ensure_workspace(plan, false))) return rc;
  const int precond = opts->preconditioner ? 1 : 0;
  if (precond && (rc = compute_invdiag(plan, s))) return rc;
  const long long n = plan->n_dofs;
  const long long maxiter = opts->maxiter > 0 ? opts->maxiter : 10 * plan->n_free;
  const int every = opts->check_every > 0 ? opts->check_every : 16;
  JXB_CUDA(cudaMemcpyAsync(plan->d_b, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  JXB_CUDA(cudaEventRecord(ev.e0, s));
  long long iters = 0;
  int status = 0;
  if ((rc = run_cg<double, double>(plan, s, plan->d_b, opts->tol, opts->atol, maxiter, precond, every, &iters,
                                   &status)))
    return rc;
  double rn = 0, bn = 0;
  bool fin = true;
  long long restarts = 0;
  if (opts->restarts == 0 || status == JXB_ERR_NONFINITE) {
    JXB_CUDA(cudaEventRecord(ev.e1, s));
    JXB_CUDA(cudaMemcpyAsync(x, plan->d_x, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if ((rc = true_residual(plan, s, plan->d_b, plan->d_x, nullptr, &rn, &bn, &fin))) return rc;
  } else {
    // True-residual restarts (the correction solves of the reference's CPU
    // CG, src/jaxiga/solvers/linear.py:261-321): CG's recursive residual
    // drifts from b - K x on ill-conditioned operators, so the FP64 residual
    // of the accumulated solution is the right-hand side of another CG solve
    // whenever it is still above the target; a correction is kept only if it
    // lowers the true residual, and all solves share the iteration budget.
    if (!plan->d_xacc) JXB_CUDA(cudaMalloc(&plan->d_xacc, n * sizeof(double)));
    if (!plan->d_res) JXB_CUDA(cudaMalloc(&plan->d_res, n * sizeof(double)));
    JXB_CUDA(cudaMemcpyAsync(plan->d_xacc, plan->d_x, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if ((rc = true_residual(plan, s, plan->d_b, plan->d_xacc, plan->d_res, &rn, &bn, &fin))) return rc;
    const double target = fmax(opts->tol * bn, opts->atol);
    const unsigned nb = (unsigned)((n + 255) / 256);
    while (restarts < opts->restarts && fin && rn > target && iters < maxiter) {
      long long it = 0;
      int st = 0;
      if ((rc = run_cg<double, double>(plan, s, plan->d_res, fmin(0.5, 0.5 * target / rn), 0.0, maxiter - iters,
                                       precond, every, &it, &st)))
        return rc;
      iters += it;
      ++restarts;
      if (st == JXB_ERR_NONFINITE) {
        status = JXB_ERR_NONFINITE;
        break;
      }
      // candidate in d_z, its residual in d_r (both free once CG has stopped)
      k_add<<<nb, 256, 0, s>>>(n, plan->d_xacc, plan->d_x, plan->d_z);
      JXB_CUDA(cudaGetLastError());
      double rn_new = 0, bn_new = 0;
      bool fin_new = true;
      if ((rc = true_residual(plan, s, plan->d_b, plan->d_z, plan->d_r, &rn_new, &bn_new, &fin_new))) return rc;
      if (!fin_new || !(rn_new < rn)) break;  // stagnation: keep the previous solution
      JXB_CUDA(cudaMemcpyAsync(plan->d_xacc, plan->d_z, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
      JXB_CUDA(cudaMemcpyAsync(plan->d_res, plan->d_r, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
      rn = rn_new;
    }
    JXB_CUDA(cudaEventRecord(ev.e1, s));
    JXB_CUDA(cudaMemcpyAsync(x, plan->d_xacc, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  }
  float ms = 0;
  if ((rc = leave_stream(s, user, ev, &ms))) return rc;
  return finish_solve("jxb_pcg", stats, iters, restarts, rn, bn, fin, opts->tol, opts->atol, ms,
                      status == JXB_ERR_NONFINITE);
}

extern "C" int jxb_refine_solve(jxb_plan* plan, jxb_stream stream, const double* b, double* x,
                                const jxb_solve_opts* opts, jxb_stats* stats) {
  if (plan && (plan->mp || plan->thb)) return fail(JXB_ERR_INVALID, "jxb_refine_solve: not available on a multipatch or hierarchical plan");
  if (!plan || !b || !x || !opts) return fail(JXB_ERR_INVALID, "jxb_refine_solve: null argument");
  if (!plan->d_geo32) return fail(JXB_ERR_INVALID, "jxb_refine_solve: plan was created without want_f32");
  if (!(opts->tol > 0) || !isfinite(opts->tol))
    return fail(JXB_ERR_INVALID, "jxb_refine_solve: tol must be finite and positive");
  cudaStream_t user = reinterpret_cast<cudaStream_t>(stream), s = nullptr;
  SolveEvents ev;
  int rc = enter_stream(plan, 0, user, ev, &s);
  if (rc) return rc;
  if ((rc = ensure_workspace(plan, true))) return rc;
  if ((rc = compute_invdiag(plan, s))) return rc;
  long long n = plan->n_dofs;
  // d_b: rhs, d_r: FP64 residual, d_z: FP64 iterate (d_x/d_r/d_z of the FP64 CG are free here)
  double* xb = plan->d_z;
  double* res = plan->d_r;
  JXB_CUDA(cudaMemcpyAsync(plan->d_b, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  JXB_CUDA(cudaMemsetAsync(xb, 0, n * sizeof(double), s));
  JXB_CUDA(cudaEventRecord(ev.e0, s));
  double inner = opts->inner_tol > 0 ? opts->inner_tol : 1e-4;
  int max_outer = opts->max_outer > 0 ? opts->max_outer : 30;
  long long maxiter = opts->maxiter > 0 ? opts->maxiter : 10 * plan->n_free;
  int every = opts->check_every > 0 ? opts->check_every : 16;
  long long total_it = 0;
  int outer = 0;
  double rn = 0, bn = 0;
  bool fin = true;
  int status = JXB_OK;
  if ((rc = true_residual(plan, s, plan->d_b, xb, res, &rn, &bn, &fin))) return rc;
  const double target = fmax(opts->tol * bn, opts->atol);
  while (outer < max_outer && fin && rn > target && total_it < maxiter) {
    // normalised residual as the FP32 right-hand side; Ap32 holds it until the
    // CG init kernel has copied it into r32 (iterations overwrite Ap32 later)
    float* rhs32 = plan->d_Ap32;
    k_scale_to_f32<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, res, 1.0 / rn, rhs32);
    long long it = 0;
    int st = 0;
    if ((rc = run_cg<float, float>(plan, s, rhs32, inner, 0.0, maxiter - total_it, 1, every, &it, &st))) return rc;
    total_it += it;
    k_axpy_from_f32<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, rn, plan->d_x32, xb);
    JXB_CUDA(cudaGetLastError());
    double prev = rn;
    if ((rc = true_residual(plan, s, plan->d_b, xb, res, &rn, &bn, &fin))) return rc;
    ++outer;
    if (st == JXB_ERR_NONFINITE) {
      status = JXB_ERR_NONFINITE;
      break;
    }
    if (!(rn < prev)) break;  // stagnation: stop, the stats report it
  }
  JXB_CUDA(cudaEventRecord(ev.e1, s));
  JXB_CUDA(cudaMemcpyAsync(x, xb, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  float ms = 0;
  if ((rc = leave_stream(s, user, ev, &ms))) return rc;
  return finish_solve("jxb_refine_solve", stats, total_it, outer, rn, bn, fin, opts->tol, opts->atol, ms,
                      status == JXB_ERR_NONFINITE);
}

// FP32 Jacobi-PCG with reliable updates (Sleijpen and van der Vorst, 1996):
// the iteration runs in FP32 on the residual scaled to unit norm. Each time
// the FP32 recursive residual has fallen by delta (opts->inner_tol) since the
// last update, or below tol ||b||, the FP32 iterate is added to the FP64
// solution, the residual is recomputed in FP64, and the FP32 iteration goes
// on from it with the same search direction. Unlike restarted refinement the
// Krylov recurrence is never thrown away, so the iteration count stays close
// to that of FP64 CG while every K p but one per update is an FP32 apply.
extern "C" int jxb_mixed_pcg(jxb_plan* plan, jxb_stream stream, const double* b, double* x,
                             const jxb_solve_opts* opts, jxb_stats* stats) {
  if (plan && (plan->mp || plan->thb)) return fail(JXB_ERR_INVALID, "jxb_mixed_pcg: not available on a multipatch or hierarchical plan");
  if (!plan || !b || !x || !opts) return fail(JXB_ERR_INVALID, "jxb_mixed_pcg: null argument");
  if (!plan->d_geo32) return fail(JXB_ERR_INVALID, "jxb_mixed_pcg: plan was created without want_f32");
  if (!(opts->tol > 0) || !isfinite(opts->tol))
    return fail(JXB_ERR_INVALID, "jxb_mixed_pcg: tol must be finite and positive");
  cudaStream_t user = reinterpret_cast<cudaStream_t>(stream), s = nullptr;
  SolveEvents ev;
  int rc = enter_stream(plan, 0, user, ev, &s);
  if (rc) return rc;
  if ((rc = ensure_workspace(plan, true))) return rc;
  if ((rc = compute_invdiag(plan, s))) return rc;
  long long n = plan->n_dofs;
  double* xb = plan->d_z;   // FP64 solution
  double* res = plan->d_r;  // FP64 residual at the last update
  JXB_CUDA(cudaMemcpyAsync(plan->d_b, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  JXB_CUDA(cudaMemsetAsync(xb, 0, n * sizeof(double), s));
  JXB_CUDA(cudaEventRecord(ev.e0, s));
  const double delta = opts->inner_tol > 0 ? opts->inner_tol : 1e-2;
  const int max_updates = opts->max_outer > 0 ? opts->max_outer : 1000;
  const long long maxiter = opts->maxiter > 0 ? opts->maxiter : 10 * plan->n_free;
  const int every = opts->check_every > 0 ? opts->check_every : 16;
  long long total_it = 0;
  int updates = 0, status = JXB_OK;
  double rn = 0, bn = 0;
  bool fin = true;
  if ((rc = true_residual(plan, s, plan->d_b, xb, res, &rn, &bn, &fin))) return rc;
  const double target = fmax(opts->tol * bn, opts->atol);
  double rn_seg = rn;  // residual norm the FP32 vectors are scaled by
  while (updates < max_updates && fin && rn > target && total_it < maxiter) {
    const float ratio = updates == 0 ? 1.f : (float)(rn_seg / rn);
    k_ru_restart<<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(n, res, plan->d_keep, plan->d_invdiag32, 1.0 / rn,
                                                            ratio, updates == 0, plan->d_x32, plan->d_r32,
                                                            plan->d_z32, plan->d_p32, plan->d_red);
    rn_seg = rn;
    // the FP32 segment stops at the update threshold or at the target, whichever comes first
    const double seg_tol = fmax(delta, target / rn);
    k_cg_init_fin<<<1, JXB_RED_THREADS, 0, s>>>(plan->d_state, plan->d_red, seg_tol, 0.0, maxiter - total_it);
    JXB_CUDA(cudaGetLastError());
    long long it = 0;
    int st = 0;
    if ((rc = iterate<float>(plan, s, maxiter - total_it, 1, every, &it, &st, nullptr, 0, nullptr))) return rc;
    total_it += it;
    k_axpy_from_f32<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, rn_seg, plan->d_x32, xb);
    JXB_CUDA(cudaGetLastError());
    if ((rc = true_residual(plan, s, plan->d_b, xb, res, &rn, &bn, &fin))) return rc;
    ++updates;
    if (st == JXB_ERR_NONFINITE) {
      status = JXB_ERR_NONFINITE;
      break;
    }
    if (!(rn < rn_seg)) break;  // no progress in FP32: stop, the stats report it
  }
  JXB_CUDA(cudaEventRecord(ev.e1, s));
  JXB_CUDA(cudaMemcpyAsync(x, xb, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  float ms = 0;
  if ((rc = leave_stream(s, user, ev, &ms))) return rc;
  return finish_solve("jxb_mixed_pcg", stats, total_it, updates, rn, bn, fin, opts->tol, opts->atol, ms,
                      status == JXB_ERR_NONFINITE);
}

extern "C" int jxb_dot(jxb_plan* plan, jxb_stream stream, const double* a, const double* b, double* out_host) {
  if (!plan || !a || !b || !out_host) return fail(JXB_ERR_INVALID, "jxb_dot: null argument");
  return dot(plan, reinterpret_cast<cudaStream_t>(stream), a, b, out_host);
}

// jxb_pcg with the iterates recorded: after every `every` iterations the current
// FP64 iterate is copied into snaps[j] (n_dofs doubles each), up to max_snaps.
// With the converged solution x*, e_j = x* - x_j and r_j = K e_j are the
// (residual, error) pairs of the solve; they train the learned preconditioner.
extern "C" int jxb_pcg_snapshots(jxb_plan* plan, jxb_stream stream, const double* b, double* x,
                                 const jxb_solve_opts* opts, int every, double* snaps, int64_t max_snaps,
                                 int64_t* n_snaps, jxb_stats* stats) {
  if (plan && (plan->mp || plan->thb)) return fail(JXB_ERR_INVALID, "jxb_pcg_snapshots: not available on a multipatch or hierarchical plan");
  if (!plan || !b || !x || !opts || !snaps || !n_snaps || every < 1 || max_snaps < 0)
    return fail(JXB_ERR_INVALID, "jxb_pcg_snapshots: bad argument");
  cudaStream_t user = reinterpret_cast<cudaStream_t>(stream);
  JXB_CUDA(cudaStreamSynchronize(user));
  if (!plan->graph_stream[0]) JXB_CUDA(cudaStreamCreateWithFlags(&plan->graph_stream[0], cudaStreamNonBlocking));
  cudaStream_t s = plan->graph_stream[0];
  int rc = ensure_workspace(plan, false);
  if (rc) return rc;
  int precond = opts->preconditioner ? 1 : 0;
  if (precond && (rc = compute_invdiag(plan, s))) return rc;
  long long maxiter = opts->maxiter > 0 ? opts->maxiter : 10 * plan->n_free;
  JXB_CUDA(cudaMemcpyAsync(plan->d_b, b, plan->n_dofs * sizeof(double), cudaMemcpyDeviceToDevice, s));
  long long iters = 0, ns = 0;
  int status = 0;
  rc = run_cg<double, double>(plan, s, plan->d_b, opts->tol, opts->atol, maxiter, precond, every, &iters, &status,
                              snaps, max_snaps, &ns);
  if (rc) return rc;
  JXB_CUDA(cudaMemcpyAsync(x, plan->d_x, plan->n_dofs * sizeof(double), cudaMemcpyDeviceToDevice, s));
  double rn, bn;
  bool fin;
  if ((rc = true_residual(plan, s, plan->d_b, plan->d_x, nullptr, &rn, &bn, &fin))) return rc;
  JXB_CUDA(cudaStreamSynchronize(s));
  *n_snaps = ns;
  return finish_solve("jxb_pcg_snapshots", stats, iters, 0, rn, bn, fin, opts->tol, opts->atol, 0.f,
                      status == JXB_ERR_NONFINITE);
}
