// Jacobi-PCG on an assembled CSR matrix, on the device: the B200 form of the
// reference's DeviceCG (src/jaxiga/solvers/phase_field.py:305-390), which runs
// jax.scipy.sparse.linalg.cg with a Jacobi preconditioner on the staggered
// phase-field subproblems, warm-started from the previous sweep's solution.
//
// The sparsity pattern (row pointers and column indices) is uploaded once per
// mesh; every solve passes new values and a new right-hand side as device
// arrays, as the reference passes `data` and `b` as arguments rather than
// constants. SpMV is one warp per row (rows of assembled IGA operators hold
// tens to a thousand entries), summing in a fixed order, so results are
// bitwise reproducible. The iteration follows jax's CG: r0 = b - A x0,
// stop when r.r <= max(tol^2 b.b, atol^2) or at maxiter; `check_every`
// iterations are one captured CUDA graph whose kernels skip their work once the
// device state says done.
#include <math.h>

#include <algorithm>
#include <vector>

#include "jxb_internal.cuh"

namespace jxb {
namespace {

constexpr int CNB = 256;

unsigned cgrid(long long n) {
  long long g = (n + CNB - 1) / CNB;
  return (unsigned)(g < 4 * 148 ? (g < 1 ? 1 : g) : 4 * 148);
}

// y = A x, warp per row; optional partial sums of dot_with . y
__global__ void __launch_bounds__(JXB_RED_THREADS) k_spmv(const CgState* st, long long n, const long long* __restrict__ ptr,
                                                          const int* __restrict__ col, const double* __restrict__ val,
                                                          const double* __restrict__ x, double* y,
                                                          const double* __restrict__ dot_with, double* partials) {
  if (st && st->done) return;
  const int lane = threadIdx.x & 31;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  double part = 0;
  for (long long row = warp; row < n; row += nw) {
    double s = 0;
    for (long long k = ptr[row] + lane; k < ptr[row + 1]; k += 32) s += val[k] * x[col[k]];
    s = warp_sum(s);
    if (lane == 0) {
      y[row] = s;
      if (dot_with) part += dot_with[row] * s;
    }
  }
  if (partials) {
    const double t = block_sum_all(part);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
  }
}

// inverse diagonal with the reference's guard: 1/d where |d| > 0, else 1
__global__ void k_csr_invdiag(long long n, const long long* __restrict__ ptr, const int* __restrict__ col,
                              const double* __restrict__ val, double* inv) {
  const long long row = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  double d = 0;
  for (long long k = ptr[row]; k < ptr[row + 1]; ++k)
    if (col[k] == row) d += val[k];
  inv[row] = fabs(d) > 0 ? 1.0 / d : 1.0;
}

// r = b - Ax0, z = M r, p = z; partials r.z, r.r, b.b
__global__ void __launch_bounds__(JXB_RED_THREADS) k_csr_init(long long n, const double* __restrict__ b,
                                                              const double* __restrict__ Ax, const double* __restrict__ inv,
                                                              double* r, double* z, double* p, double* partials) {
  double rz = 0, rr = 0, bb = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double ri = b[i] - Ax[i];
    const double zi = inv[i] * ri;
    r[i] = ri;
    z[i] = zi;
    p[i] = zi;
    rz += ri * zi;
    rr += ri * ri;
    bb += b[i] * b[i];
  }
  const double s0 = block_sum_all(rz), s1 = block_sum_all(rr), s2 = block_sum_all(bb);
  if (threadIdx.x == 0) {
    partials[JXB_RED_BLOCKS + blockIdx.x] = s0;
    partials[2 * JXB_RED_BLOCKS + blockIdx.x] = s1;
    partials[3 * JXB_RED_BLOCKS + blockIdx.x] = s2;
  }
}

__global__ void k_csr_start(CgState* st, const double* partials, double tol, double atol, long long maxiter) {
  const double gamma = reduce_partials(partials + JXB_RED_BLOCKS);
  const double rr = reduce_partials(partials + 2 * JXB_RED_BLOCKS);
  const double bb = reduce_partials(partials + 3 * JXB_RED_BLOCKS);
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

// alpha = gamma / p.Ap; x += alpha p; r -= alpha Ap; z = M r; partials r.z, r.r
__global__ void __launch_bounds__(JXB_RED_THREADS) k_csr_xr(const CgState* st, long long n, double* partials, double* x,
                                                            double* r, double* z, const double* __restrict__ p,
                                                            const double* __restrict__ Ap,
                                                            const double* __restrict__ inv) {
  if (st->done) return;
  const double alpha = st->gamma / reduce_partials(partials);
  double rz = 0, rr = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    x[i] += alpha * p[i];
    const double ri = r[i] - alpha * Ap[i];
    r[i] = ri;
    const double zi = inv[i] * ri;
    z[i] = zi;
    rz += ri * zi;
    rr += ri * ri;
  }
  const double s0 = block_sum_all(rz), s1 = block_sum_all(rr);
  if (threadIdx.x == 0) {
    partials[JXB_RED_BLOCKS + blockIdx.x] = s0;
    partials[2 * JXB_RED_BLOCKS + blockIdx.x] = s1;
  }
}

__global__ void k_csr_fin(CgState* st, const double* partials) {
  if (st->done) return;
  const double pAp = reduce_partials(partials);
  const double gnew = reduce_partials(partials + JXB_RED_BLOCKS);
  const double rr = reduce_partials(partials + 2 * JXB_RED_BLOCKS);
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

__global__ void k_csr_p(const CgState* st, long long n, const double* __restrict__ z, double* p) {
  if (st->done) return;
  const double beta = st->beta;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = z[i] + beta * p[i];
}

// partials |Ax - b|^2, |b|^2
__global__ void __launch_bounds__(JXB_RED_THREADS) k_csr_res(long long n, const double* __restrict__ b,
                                                             const double* __restrict__ Ax, double* partials) {
  double rr = 0, bb = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double d = Ax[i] - b[i];
    rr += d * d;
    bb += b[i] * b[i];
  }
  const double s0 = block_sum_all(rr), s1 = block_sum_all(bb);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = s0;
    partials[JXB_RED_BLOCKS + blockIdx.x] = s1;
  }
}

}  // namespace
}  // namespace jxb

struct jxb_csr {
  long long n = 0, nnz = 0;
  long long* ptr = nullptr;
  int* col = nullptr;
  double *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *Ap = nullptr, *inv = nullptr, *part = nullptr,
         *b = nullptr;
  jxb::CgState* st = nullptr;
  jxb::CgState* h_st = nullptr;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graph_iters = 0;
  double* val = nullptr;  // device copy of the values of the current solve
};

namespace jxb {
namespace {

void free_csr(jxb_csr* C) {
  if (!C) return;
  if (C->graph) cudaGraphExecDestroy(C->graph);
  void* bufs[] = {C->ptr, C->col, C->x, C->r, C->z, C->p, C->Ap, C->inv, C->part, C->st, C->val, C->b};
  for (void* b : bufs) cudaFree(b);
  if (C->h_st) cudaFreeHost(C->h_st);
  if (C->stream) cudaStreamDestroy(C->stream);
  delete C;
}

int csr_iteration(jxb_csr* C, cudaStream_t s) {
  k_spmv<<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(C->st, C->n, C->ptr, C->col, C->val, C->p, C->Ap, C->p, C->part);
  k_csr_xr<<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(C->st, C->n, C->part, C->x, C->r, C->z, C->p, C->Ap, C->inv);
  k_csr_fin<<<1, JXB_RED_THREADS, 0, s>>>(C->st, C->part);
  k_csr_p<<<cgrid(C->n), CNB, 0, s>>>(C->st, C->n, C->z, C->p);
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

}  // namespace
}  // namespace jxb

using namespace jxb;

extern "C" int jxb_csr_create(int64_t n, const int64_t* indptr, const int32_t* cols, jxb_csr** out) {
  if (!out || !indptr || n < 1 || (indptr[n] > 0 && !cols)) return fail(JXB_ERR_INVALID, "jxb_csr_create: bad argument");
  *out = nullptr;
  if (indptr[0] != 0) return fail(JXB_ERR_INVALID, "jxb_csr_create: indptr[0] must be 0");
  for (int64_t i = 0; i < n; ++i)
    if (indptr[i + 1] < indptr[i]) return fail(JXB_ERR_INVALID, "jxb_csr_create: indptr must not decrease");
  const int64_t nnz = indptr[n];
  for (int64_t k = 0; k < nnz; ++k)
    if (cols[k] < 0 || cols[k] >= n) return fail(JXB_ERR_INVALID, "jxb_csr_create: column index out of range");
  jxb_csr* C = new jxb_csr();
  C->n = n;
  C->nnz = nnz;
  auto bail = [&](int code) {
    if (C->stream) cudaStreamSynchronize(C->stream);
    free_csr(C);
    return code;
  };
  cudaError_t e = cudaStreamCreateWithFlags(&C->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&C->ptr, (n + 1) * sizeof(long long));
  if (e == cudaSuccess) e = cudaMalloc(&C->col, std::max<int64_t>(nnz, 1) * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&C->val, std::max<int64_t>(nnz, 1) * sizeof(double));
  for (double** p : {&C->x, &C->r, &C->z, &C->p, &C->Ap, &C->inv, &C->b})
    if (e == cudaSuccess) e = cudaMalloc(p, n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&C->part, 4 * JXB_RED_BLOCKS * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&C->st, sizeof(CgState));
  if (e == cudaSuccess) e = cudaMallocHost(&C->h_st, sizeof(CgState));
  if (e == cudaSuccess) e = cudaMemcpyAsync(C->ptr, indptr, (n + 1) * sizeof(long long), cudaMemcpyHostToDevice, C->stream);
  if (e == cudaSuccess && nnz)
    e = cudaMemcpyAsync(C->col, cols, nnz * sizeof(int), cudaMemcpyHostToDevice, C->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(C->stream);
  if (e != cudaSuccess) return bail(cuda_fail(e, "jxb_csr_create"));
  *out = C;
  return JXB_OK;
}

extern "C" int jxb_csr_destroy(jxb_csr* C) {
  if (!C) return JXB_OK;
  cudaStreamSynchronize(C->stream);
  free_csr(C);
  return JXB_OK;
}

extern "C" int jxb_csr_matvec(jxb_csr* C, jxb_stream stream, const double* values, const double* x, double* y) {
  if (!C || !values || !x || !y) return fail(JXB_ERR_INVALID, "jxb_csr_matvec: null argument");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  k_spmv<<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(nullptr, C->n, C->ptr, C->col, values, x, y, nullptr, nullptr);
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

extern "C" int jxb_csr_pcg(jxb_csr* C, jxb_stream stream, const double* values, const double* b, double* x,
                           const jxb_solve_opts* opts, jxb_stats* stats) {
  if (!C || !values || !b || !x || !opts) return fail(JXB_ERR_INVALID, "jxb_csr_pcg: null argument");
  if (!(opts->tol > 0) || !isfinite(opts->tol)) return fail(JXB_ERR_INVALID, "jxb_csr_pcg: tol must be finite and positive");
  cudaStream_t user = reinterpret_cast<cudaStream_t>(stream), s = C->stream;
  SolveEvents ev;
  int rc = ev.create();
  if (rc) return rc;
  JXB_CUDA(cudaEventRecord(ev.order, user));
  JXB_CUDA(cudaStreamWaitEvent(s, ev.order, 0));
  const long long n = C->n;
  const long long maxiter = opts->maxiter > 0 ? opts->maxiter : 10 * n;
  const int every = opts->check_every > 0 ? opts->check_every : 16;
  // the graph reads the solver's own copies of the values and the right-hand side
  JXB_CUDA(cudaMemcpyAsync(C->val, values, std::max<long long>(C->nnz, 1) * sizeof(double), cudaMemcpyDeviceToDevice, s));
  JXB_CUDA(cudaMemcpyAsync(C->b, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  JXB_CUDA(cudaMemcpyAsync(C->x, x, n * sizeof(double), cudaMemcpyDeviceToDevice, s));  // warm start x0
  if (!C->graph || C->graph_iters != every) {
    if (C->graph) cudaGraphExecDestroy(C->graph);
    C->graph = nullptr;
    cudaGraph_t g;
    JXB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    int rci = 0;
    for (int it = 0; it < every && !rci; ++it) rci = csr_iteration(C, s);
    cudaError_t ce = cudaStreamEndCapture(s, &g);
    if (rci) return rci;
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
    ce = cudaGraphInstantiate(&C->graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaGraphInstantiate");
    C->graph_iters = every;
  }
  JXB_CUDA(cudaEventRecord(ev.e0, s));
  k_csr_invdiag<<<(unsigned)((n + CNB - 1) / CNB), CNB, 0, s>>>(n, C->ptr, C->col, C->val, C->inv);
  k_spmv<<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(nullptr, n, C->ptr, C->col, C->val, C->x, C->Ap, nullptr, nullptr);
  k_csr_init<<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(n, C->b, C->Ap, C->inv, C->r, C->z, C->p, C->part);
  k_csr_start<<<1, JXB_RED_THREADS, 0, s>>>(C->st, C->part, opts->tol, opts->atol, maxiter);
  JXB_CUDA(cudaGetLastError());
  JXB_CUDA(cudaMemcpyAsync(C->h_st, C->st, sizeof(CgState), cudaMemcpyDeviceToHost, s));
  JXB_CUDA(cudaStreamSynchronize(s));
  const long long launches = maxiter / every + 2;
  for (long long l = 0; l < launches && !C->h_st->done; ++l) {
    JXB_CUDA(cudaGraphLaunch(C->graph, s));
    JXB_CUDA(cudaMemcpyAsync(C->h_st, C->st, sizeof(CgState), cudaMemcpyDeviceToHost, s));
    JXB_CUDA(cudaStreamSynchronize(s));
  }
  JXB_CUDA(cudaEventRecord(ev.e1, s));
  const long long iters = C->h_st->k;
  const int status = C->h_st->done ? C->h_st->status : JXB_ERR_NOT_CONVERGED;
  JXB_CUDA(cudaMemcpyAsync(x, C->x, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  // true residual |b - A x| against the caller's b
  k_spmv<<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(nullptr, n, C->ptr, C->col, C->val, C->x, C->Ap, nullptr, nullptr);
  k_csr_res<<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(n, C->b, C->Ap, C->part);
  std::vector<double> h(2 * JXB_RED_BLOCKS);
  JXB_CUDA(cudaMemcpyAsync(h.data(), C->part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  JXB_CUDA(cudaStreamSynchronize(s));
  double rr = 0, bb = 0;
  for (int i = 0; i < JXB_RED_BLOCKS; ++i) {
    rr += h[i];
    bb += h[JXB_RED_BLOCKS + i];
  }
  JXB_CUDA(cudaEventRecord(ev.order, s));
  JXB_CUDA(cudaStreamWaitEvent(user, ev.order, 0));
  float ms = 0;
  JXB_CUDA(cudaEventElapsedTime(&ms, ev.e0, ev.e1));
  const double rn = sqrt(rr), bn = sqrt(bb);
  return finish_solve("jxb_csr_pcg", stats, iters, 0, rn, bn, isfinite(rn), opts->tol, opts->atol, ms,
                      status == JXB_ERR_NONFINITE);
}
