// Geometric multigrid V-cycle over nested spline spaces, and CG preconditioned
// by it.
//
// The reference preconditions its matrix-free CG with Jacobi only
// (src/jaxiga/solvers/linear.py:419-431); on the clamped plate (a fourth-order
// operator, condition number ~h^-4) that takes thousands of iterations. Here
// the levels are the same patch with every other interior knot removed, so the
// coarse spaces are nested in the fine one and the prolongation is knot
// insertion: per parametric direction a banded matrix P_d (fine control points
// x coarse control points), applied to the (z, y, x, component)-ordered DOF
// array one direction at a time; the restriction is its transpose. Knot
// insertion acts on homogeneous coefficients, so on a rational patch a field
// is multiplied by the coarse weights before and divided by the fine weights
// after (and the transpose of that for the restriction). Each level
// has its own plan (its operator rediscretised on the coarse space) and the
// coarsest operator is inverted exactly (a dense inverse of its free block,
// supplied by the host).
//
// Smoothing is Chebyshev acceleration of Jacobi: the degree-k polynomial in
// D^-1 K that is smallest on [lmax / range, lmax] (lmax of D^-1 K from a power
// iteration at set-up, times 1.1), applied before and after the coarse
// correction, which keeps the V-cycle symmetric so that plain PCG can use it.
//
// The PCG follows jax.scipy.sparse.linalg.cg (x0 = 0, stop when r.r <=
// max(tol^2 b.b, atol^2) or at maxiter) with z = V r; `check_every`
// iterations, V-cycles included, are captured in one CUDA graph, and every
// kernel first reads the device `done` flag so that iterations past
// convergence do nothing.
#include <math.h>

#include <algorithm>
#include <string>
#include <vector>

#include "jxb_internal.cuh"

namespace jxb {
namespace {

struct Dir1d {  // one direction of a transfer, CSR on the device
  int rows = 1, cols = 1;
  int *ptr = nullptr, *idx = nullptr;
  double* val = nullptr;
};

struct Level {
  jxb_plan* plan = nullptr;
  long long n = 0;
  int ncp[3] = {1, 1, 1};
  Dir1d P[3], R[3];  // prolongation from the next coarser level and its transpose
  double *Rv = nullptr, *Z = nullptr, *E = nullptr, *D = nullptr, *KE = nullptr, *RES = nullptr, *T1 = nullptr,
         *T2 = nullptr, *W = nullptr;  // W: weighted copy (rational patches)
  double lmax = 0;
};

constexpr int NB = 256;

__global__ void k_apply1d(const CgState* st, int dir, int n0, int n1, int n2, int m, int vec,
                          const int* __restrict__ ptr, const int* __restrict__ idx, const double* __restrict__ val,
                          const double* __restrict__ in, double* __restrict__ out) {
  if (st && st->done) return;
  int o[3] = {n0, n1, n2};
  o[dir] = m;
  const long long total = (long long)o[0] * o[1] * o[2] * vec;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t % vec);
    long long r = t / vec;
    int i[3];
    i[0] = (int)(r % o[0]);
    r /= o[0];
    i[1] = (int)(r % o[1]);
    i[2] = (int)(r / o[1]);
    const int row = i[dir];
    double s = 0;
    for (int k = ptr[row]; k < ptr[row + 1]; ++k) {
      int j[3] = {i[0], i[1], i[2]};
      j[dir] = idx[k];
      s += val[k] * in[(((long long)j[2] * n1 + j[1]) * n0 + j[0]) * vec + c];
    }
    out[t] = s;
  }
}

__global__ void k_cheb_init(const CgState* st, long long n, const double* __restrict__ inv,
                            const double* __restrict__ r, double s, double* e, double* d) {
  if (st && st->done) return;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double v = s * inv[i] * r[i];
    e[i] = v;
    d[i] = v;
  }
}

// d = c1 d + c2 D^-1 (r - K e); e += d
__global__ void k_cheb_step(const CgState* st, long long n, const double* __restrict__ inv,
                            const double* __restrict__ r, const double* __restrict__ Ke, double c1, double c2,
                            double* d, double* e) {
  if (st && st->done) return;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double v = c1 * d[i] + c2 * inv[i] * (r[i] - Ke[i]);
    d[i] = v;
    e[i] += v;
  }
}

// out = keep ? a - b : 0
__global__ void k_sub_masked(const CgState* st, long long n, const uint8_t* __restrict__ keep,
                             const double* __restrict__ a, const double* __restrict__ b, double* out) {
  if (st && st->done) return;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = keep[i] ? a[i] - b[i] : 0.0;
}

// z += keep ? t : 0 ; with copy != 0: z = keep ? t : 0
__global__ void k_add_masked(const CgState* st, long long n, const uint8_t* __restrict__ keep,
                             const double* __restrict__ t, double* z, int copy) {
  if (st && st->done) return;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double v = keep[i] ? t[i] : 0.0;
    z[i] = copy ? v : z[i] + v;
  }
}

// out[i*vec + c] = in[i*vec + c] * w[i] (mul) or / w[i]: the NURBS weights around
// knot insertion, which acts on homogeneous coefficients
__global__ void k_weight(const CgState* st, long long n_scalar, int vec, const double* __restrict__ w,
                         const double* __restrict__ in, double* out, int mul) {
  if (st && st->done) return;
  const long long n = n_scalar * vec;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double wi = w[i / vec];
    out[i] = mul ? in[i] * wi : in[i] / wi;
  }
}

// z = A r, A dense (n x n, row-major), one warp per row, fixed summation order
__global__ void k_gemv(const CgState* st, int n, const double* __restrict__ A, const double* __restrict__ r,
                       double* z) {
  if (st && st->done) return;
  const int lane = threadIdx.x & 31;
  for (int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < n; row += (gridDim.x * blockDim.x) >> 5) {
    double s = 0;
    for (int j = lane; j < n; j += 32) s += A[(size_t)row * n + j] * r[j];
    s = warp_sum(s);
    if (lane == 0) z[row] = s;
  }
}

// PCG pieces (jax CG semantics), partial sums in slots of JXB_RED_BLOCKS
__global__ void __launch_bounds__(JXB_RED_THREADS) k_mg_init(long long n, const double* __restrict__ b,
                                                             const uint8_t* __restrict__ keep, double* x, double* r,
                                                             double* partials) {
  double bb = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double v = keep[i] ? b[i] : 0.0;
    x[i] = 0.0;
    r[i] = v;
    bb += v * v;
  }
  const double s = block_sum_all(bb);
  if (threadIdx.x == 0) partials[3 * JXB_RED_BLOCKS + blockIdx.x] = s;
}

__global__ void __launch_bounds__(JXB_RED_THREADS) k_mg_rz(const CgState* st, long long n, const double* __restrict__ r,
                                                           const double* __restrict__ z, double* partials, int with_rr) {
  if (st && st->done) return;
  double rz = 0, rr = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    rz += r[i] * z[i];
    rr += r[i] * r[i];
  }
  const double s0 = block_sum_all(rz), s1 = block_sum_all(rr);
  if (threadIdx.x == 0) {
    partials[JXB_RED_BLOCKS + blockIdx.x] = s0;
    if (with_rr) partials[2 * JXB_RED_BLOCKS + blockIdx.x] = s1;
  }
}

__global__ void k_mg_start(CgState* st, const double* partials, double tol, double atol, long long maxiter) {
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

// p = z (first)
__global__ void k_copy(long long n, const double* __restrict__ a, double* b) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = a[i];
}

// alpha = gamma / p.Ap; x += alpha p; r -= alpha Ap; partial r.r
__global__ void __launch_bounds__(JXB_RED_THREADS) k_mg_xr(const CgState* st, long long n, double* partials, double* x,
                                                           double* r, const double* __restrict__ p,
                                                           const double* __restrict__ Ap) {
  if (st->done) return;
  const double alpha = st->gamma / reduce_partials(partials);
  double rr = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    x[i] += alpha * p[i];
    const double v = r[i] - alpha * Ap[i];
    r[i] = v;
    rr += v * v;
  }
  const double s = block_sum_all(rr);
  if (threadIdx.x == 0) partials[2 * JXB_RED_BLOCKS + blockIdx.x] = s;
}

__global__ void k_mg_fin(CgState* st, const double* partials) {
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

__global__ void k_mg_p(const CgState* st, long long n, const double* __restrict__ z, double* p) {
  if (st->done) return;
  const double beta = st->beta;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = z[i] + beta * p[i];
}

// power-iteration step: y = D^-1 K x (already in y as K x) -> y *= inv; partials y.y, x.y
__global__ void __launch_bounds__(JXB_RED_THREADS) k_pow(long long n, const double* __restrict__ inv,
                                                         const double* __restrict__ x, double* y, double* partials) {
  double yy = 0, xy = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double v = inv[i] * y[i];
    y[i] = v;
    yy += v * v;
    xy += x[i] * v;
  }
  const double s0 = block_sum_all(yy), s1 = block_sum_all(xy);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = s0;
    partials[JXB_RED_BLOCKS + blockIdx.x] = s1;
  }
}

__global__ void k_scale(long long n, const double* __restrict__ a, double s, double* b) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = s * a[i];
}

// deterministic start vector of the power iteration, 0 on prescribed DOFs
__global__ void k_pow_start(long long n, const uint8_t* __restrict__ keep, double* x) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    x[i] = keep[i] ? 1.0 + 0.5 * sin(0.7 * (double)i) : 0.0;
}

unsigned grid_of(long long n) {
  long long g = (n + NB - 1) / NB;
  return (unsigned)(g < 4 * 148 ? (g < 1 ? 1 : g) : 4 * 148);
}

}  // namespace
}  // namespace jxb

struct jxb_mg {
  std::vector<jxb::Level> L;
  int degree = 3;
  double range = 20.0;
  double* coarse_inv = nullptr;
  // PCG state on the finest level
  double *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *Ap = nullptr, *b = nullptr, *part = nullptr;
  jxb::CgState* st = nullptr;
  jxb::CgState* h_st = nullptr;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graph_iters = 0;
  std::vector<void*> owned;
};

namespace jxb {
namespace {

int dalloc(jxb_mg* M, double** p, size_t n) {
  JXB_CUDA(cudaMalloc(p, std::max<size_t>(n, 1) * sizeof(double)));
  M->owned.push_back(*p);
  return JXB_OK;
}

void free_mg(jxb_mg* M) {
  if (!M) return;
  if (M->graph) cudaGraphExecDestroy(M->graph);
  for (void* p : M->owned) cudaFree(p);
  if (M->h_st) cudaFreeHost(M->h_st);
  if (M->stream) cudaStreamDestroy(M->stream);
  delete M;
}

int masked_apply(jxb_plan* P, cudaStream_t s, const double* x, double* y, const CgState* st) {
  int rc = launch_bricks<double>(P, s, MODE_APPLY, x, nullptr, st, 1);
  if (rc) return rc;
  return launch_combine<double>(P, s, y, 1, nullptr, nullptr, st);
}

// e = Chebyshev(D^-1 K) D^-1 r on level l
int smooth(jxb_mg* M, int l, cudaStream_t s, const double* r, double* e, const CgState* st) {
  Level& V = M->L[l];
  const double lmax = 1.1 * V.lmax, lmin = lmax / M->range;
  const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin), sigma = theta / delta;
  double rho = 1.0 / sigma;
  const long long n = V.n;
  const double* inv = V.plan->d_invdiag;
  k_cheb_init<<<grid_of(n), NB, 0, s>>>(st, n, inv, r, 1.0 / theta, e, V.D);
  for (int k = 1; k < M->degree; ++k) {
    int rc = masked_apply(V.plan, s, e, V.KE, st);
    if (rc) return rc;
    const double rho_new = 1.0 / (2.0 * sigma - rho);
    k_cheb_step<<<grid_of(n), NB, 0, s>>>(st, n, inv, r, V.KE, rho_new * rho, 2.0 * rho_new / delta, V.D, e);
    rho = rho_new;
  }
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

// out = T (in) with T the tensor product of one 1D matrix per direction
int transfer(jxb_mg* M, int l, cudaStream_t s, const double* in, double* out, bool prolong, const CgState* st) {
  Level& F = M->L[l];
  Level& C = M->L[l + 1];
  const int vec = F.plan->vec, dim = F.plan->dim;
  int n[3] = {prolong ? C.ncp[0] : F.ncp[0], prolong ? C.ncp[1] : F.ncp[1], prolong ? C.ncp[2] : F.ncp[2]};
  const double* src = in;
  const bool rational = F.plan->rational || C.plan->rational;
  if (rational) {  // into homogeneous coefficients: times the coarse weights / over the fine ones
    Level& S = prolong ? C : F;
    k_weight<<<grid_of(S.n), NB, 0, s>>>(st, S.plan->n_scalar, vec, S.plan->d_wgts, in, S.W, prolong ? 1 : 0);
    src = S.W;
  }
  for (int d = 0; d < dim; ++d) {
    const Dir1d& T = prolong ? F.P[d] : F.R[d];
    double* dst = d == dim - 1 ? out : (d % 2 == 0 ? F.T1 : F.T2);
    int m = T.rows;
    long long total = (long long)vec * m * (d == 0 ? n[1] * n[2] : d == 1 ? n[0] * n[2] : n[0] * n[1]);
    k_apply1d<<<grid_of(total), NB, 0, s>>>(st, d, n[0], n[1], n[2], m, vec, T.ptr, T.idx, T.val, src, dst);
    n[d] = m;
    src = dst;
  }
  if (rational) {  // back from homogeneous coefficients
    Level& S = prolong ? F : C;
    k_weight<<<grid_of(S.n), NB, 0, s>>>(st, S.plan->n_scalar, vec, S.plan->d_wgts, out, out, prolong ? 0 : 1);
  }
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

// Z_l = V(R_l)
int vcycle(jxb_mg* M, int l, cudaStream_t s, const CgState* st) {
  Level& V = M->L[l];
  const int nl = (int)M->L.size();
  const long long n = V.n;
  if (l == nl - 1) {
    k_gemv<<<(unsigned)((n * 32 + NB - 1) / NB), NB, 0, s>>>(st, (int)n, M->coarse_inv, V.Rv, V.Z);
    JXB_CUDA(cudaGetLastError());
    return JXB_OK;
  }
  Level& C = M->L[l + 1];
  int rc;
  if ((rc = smooth(M, l, s, V.Rv, V.Z, st))) return rc;
  if ((rc = masked_apply(V.plan, s, V.Z, V.KE, st))) return rc;
  k_sub_masked<<<grid_of(n), NB, 0, s>>>(st, n, V.plan->d_keep, V.Rv, V.KE, V.RES);
  if ((rc = transfer(M, l, s, V.RES, C.RES, false, st))) return rc;
  k_add_masked<<<grid_of(C.n), NB, 0, s>>>(st, C.n, C.plan->d_keep, C.RES, C.Rv, 1);
  if ((rc = vcycle(M, l + 1, s, st))) return rc;
  if ((rc = transfer(M, l, s, C.Z, V.RES, true, st))) return rc;
  k_add_masked<<<grid_of(n), NB, 0, s>>>(st, n, V.plan->d_keep, V.RES, V.Z, 0);
  if ((rc = masked_apply(V.plan, s, V.Z, V.KE, st))) return rc;
  k_sub_masked<<<grid_of(n), NB, 0, s>>>(st, n, V.plan->d_keep, V.Rv, V.KE, V.RES);
  if ((rc = smooth(M, l, s, V.RES, V.E, st))) return rc;
  k_add_masked<<<grid_of(n), NB, 0, s>>>(st, n, V.plan->d_keep, V.E, V.Z, 0);
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

int power_lmax(jxb_mg* M, int l, cudaStream_t s, int iters) {
  Level& V = M->L[l];
  const long long n = V.n;
  double* x = V.E;
  double* y = V.KE;
  double* part = M->part;
  k_pow_start<<<grid_of(n), NB, 0, s>>>(n, V.plan->d_keep, x);
  JXB_CUDA(cudaGetLastError());
  double xx = 0;
  int rc = dot(V.plan, s, x, x, &xx);
  if (rc) return rc;
  if (!(xx > 0)) return fail(JXB_ERR_INVALID, "jxb_mg_create: a level has no free DOFs");
  k_scale<<<grid_of(n), NB, 0, s>>>(n, x, 1.0 / sqrt(xx), x);
  double lam = 0;
  std::vector<double> h(JXB_RED_BLOCKS);
  for (int it = 0; it < iters; ++it) {  // |x| = 1: |D^-1 K x| -> lmax
    if ((rc = masked_apply(V.plan, s, x, y, nullptr))) return rc;
    k_pow<<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(n, V.plan->d_invdiag, x, y, part);
    JXB_CUDA(cudaGetLastError());
    JXB_CUDA(cudaMemcpyAsync(h.data(), part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    JXB_CUDA(cudaStreamSynchronize(s));
    double yy = 0;
    for (int i = 0; i < JXB_RED_BLOCKS; ++i) yy += h[i];
    if (!(yy > 0) || !isfinite(yy)) return fail(JXB_ERR_NONFINITE, "jxb_mg_create: power iteration broke down");
    lam = sqrt(yy);
    k_scale<<<grid_of(n), NB, 0, s>>>(n, y, 1.0 / lam, x);
  }
  V.lmax = lam;
  return JXB_OK;
}

}  // namespace
}  // namespace jxb

using namespace jxb;

extern "C" int jxb_mg_create(jxb_plan* const* plans, int n_levels, const jxb_transfer1d* transfer_, const double* coarse_inv,
                             int degree, double smooth_range, jxb_mg** out) {
  if (!plans || !out || n_levels < 2 || n_levels > 12 || !transfer_ || !coarse_inv)
    return fail(JXB_ERR_INVALID, "jxb_mg_create: bad argument");
  for (int l = 0; l < n_levels; ++l)
    if (plans[l] && (plans[l]->mp || plans[l]->thb)) return fail(JXB_ERR_INVALID, "jxb_mg_create: not available on a multipatch or hierarchical plan");
  if (degree < 1 || degree > 8 || !(smooth_range > 1.0))
    return fail(JXB_ERR_INVALID, "jxb_mg_create: degree must be in 1..8 and smooth_range > 1");
  *out = nullptr;
  for (int l = 0; l < n_levels; ++l) {
    if (!plans[l]) return fail(JXB_ERR_INVALID, "jxb_mg_create: null plan");
    if (plans[l]->dim != plans[0]->dim || plans[l]->vec != plans[0]->vec || plans[l]->op != plans[0]->op)
      return fail(JXB_ERR_INVALID, "jxb_mg_create: levels must share dim, vec and operator");
    for (int k = 0; k < l; ++k)
      if (plans[k] == plans[l]) return fail(JXB_ERR_INVALID, "jxb_mg_create: a plan appears twice");
  }
  jxb_mg* M = new jxb_mg();
  M->degree = degree;
  M->range = smooth_range;
  M->L.resize(n_levels);
  auto bail = [&](int code) {
    if (M->stream) cudaStreamSynchronize(M->stream);
    free_mg(M);
    return code;
  };
  if (cudaStreamCreateWithFlags(&M->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(JXB_ERR_CUDA, "jxb_mg_create: stream"));
  cudaStream_t s = M->stream;
  const int dim = plans[0]->dim, vec = plans[0]->vec;
  int rc;
  for (int l = 0; l < n_levels; ++l) {
    Level& V = M->L[l];
    V.plan = plans[l];
    V.n = plans[l]->n_dofs;
    for (int d = 0; d < 3; ++d) V.ncp[d] = d < dim ? plans[l]->n_cp[d] : 1;
    if ((rc = ensure_workspace(V.plan, false))) return bail(rc);
    if ((rc = compute_invdiag(V.plan, s))) return bail(rc);
  }
  size_t tmax = 0;
  for (int l = 0; l + 1 < n_levels; ++l) {
    Level& F = M->L[l];
    Level& C = M->L[l + 1];
    for (int d = 0; d < dim; ++d) {
      const jxb_transfer1d& T = transfer_[3 * l + d];
      if (T.rows != F.ncp[d] || T.cols != C.ncp[d] || !T.ptr || !T.idx || !T.val)
        return bail(fail(JXB_ERR_INVALID, "jxb_mg_create: transfer " + std::to_string(l) + " direction " +
                                               std::to_string(d) + " does not map the coarse control points to the fine"));
      const int nnz = T.ptr[T.rows];
      for (int i = 0; i < T.rows; ++i)
        if (T.ptr[i + 1] < T.ptr[i]) return bail(fail(JXB_ERR_INVALID, "jxb_mg_create: transfer rows must increase"));
      for (int k = 0; k < nnz; ++k)
        if (T.idx[k] < 0 || T.idx[k] >= T.cols) return bail(fail(JXB_ERR_INVALID, "jxb_mg_create: transfer column out of range"));
      // host transpose
      std::vector<int> tptr(T.cols + 1, 0), tidx(nnz);
      std::vector<double> tval(nnz);
      for (int k = 0; k < nnz; ++k) tptr[T.idx[k] + 1]++;
      for (int j = 0; j < T.cols; ++j) tptr[j + 1] += tptr[j];
      std::vector<int> fill(tptr.begin(), tptr.end() - 1);
      for (int i = 0; i < T.rows; ++i)
        for (int k = T.ptr[i]; k < T.ptr[i + 1]; ++k) {
          const int at = fill[T.idx[k]]++;
          tidx[at] = i;
          tval[at] = T.val[k];
        }
      auto up = [&](Dir1d& D, int rows, int cols, const int* p, const int* ix, const double* v) -> int {
        D.rows = rows;
        D.cols = cols;
        const int z = p[rows];
        JXB_CUDA(cudaMalloc(&D.ptr, (rows + 1) * sizeof(int)));
        M->owned.push_back(D.ptr);
        JXB_CUDA(cudaMalloc(&D.idx, std::max(z, 1) * sizeof(int)));
        M->owned.push_back(D.idx);
        JXB_CUDA(cudaMalloc(&D.val, std::max(z, 1) * sizeof(double)));
        M->owned.push_back(D.val);
        JXB_CUDA(cudaMemcpyAsync(D.ptr, p, (rows + 1) * sizeof(int), cudaMemcpyHostToDevice, s));
        JXB_CUDA(cudaMemcpyAsync(D.idx, ix, z * sizeof(int), cudaMemcpyHostToDevice, s));
        JXB_CUDA(cudaMemcpyAsync(D.val, v, z * sizeof(double), cudaMemcpyHostToDevice, s));
        JXB_CUDA(cudaStreamSynchronize(s));  // the host arrays are about to go away
        return JXB_OK;
      };
      if ((rc = up(F.P[d], T.rows, T.cols, T.ptr, T.idx, T.val))) return bail(rc);
      if ((rc = up(F.R[d], T.cols, T.rows, tptr.data(), tidx.data(), tval.data()))) return bail(rc);
    }
    // intermediate shapes of either direction's passes
    size_t a = (size_t)vec * F.ncp[0] * C.ncp[1] * C.ncp[2], bsz = (size_t)vec * F.ncp[0] * F.ncp[1] * C.ncp[2];
    size_t c2 = (size_t)vec * C.ncp[0] * F.ncp[1] * F.ncp[2], d2 = (size_t)vec * C.ncp[0] * C.ncp[1] * F.ncp[2];
    tmax = std::max({tmax, a, bsz, c2, d2});
  }
  for (int l = 0; l < n_levels; ++l) {
    Level& V = M->L[l];
    for (double** p : {&V.Rv, &V.Z, &V.E, &V.D, &V.KE, &V.RES, &V.W})
      if ((rc = dalloc(M, p, V.n))) return bail(rc);
    if ((rc = dalloc(M, &V.T1, tmax)) || (rc = dalloc(M, &V.T2, tmax))) return bail(rc);
  }
  const long long nc = M->L.back().n;
  if ((rc = dalloc(M, &M->coarse_inv, (size_t)nc * nc))) return bail(rc);
  if (cudaMemcpyAsync(M->coarse_inv, coarse_inv, (size_t)nc * nc * sizeof(double), cudaMemcpyHostToDevice, s) !=
      cudaSuccess)
    return bail(fail(JXB_ERR_CUDA, "jxb_mg_create: coarse inverse upload"));
  const long long n0 = M->L[0].n;
  for (double** p : {&M->x, &M->r, &M->z, &M->p, &M->Ap, &M->b})
    if ((rc = dalloc(M, p, n0))) return bail(rc);
  if ((rc = dalloc(M, &M->part, 4 * JXB_RED_BLOCKS))) return bail(rc);
  if (cudaMalloc(&M->st, sizeof(CgState)) != cudaSuccess) return bail(fail(JXB_ERR_NOMEM, "jxb_mg_create: state"));
  M->owned.push_back(M->st);
  if (cudaMallocHost(&M->h_st, sizeof(CgState)) != cudaSuccess) return bail(fail(JXB_ERR_NOMEM, "jxb_mg_create: state"));
  for (int l = 0; l + 1 < n_levels; ++l)
    if ((rc = power_lmax(M, l, s, 20))) return bail(rc);
  if (cudaStreamSynchronize(s) != cudaSuccess) return bail(fail(JXB_ERR_CUDA, "jxb_mg_create: set-up"));
  *out = M;
  return JXB_OK;
}

extern "C" int jxb_mg_destroy(jxb_mg* M) {
  if (!M) return JXB_OK;
  cudaStreamSynchronize(M->stream);
  free_mg(M);
  return JXB_OK;
}

extern "C" int jxb_mg_info(const jxb_mg* M, double* lmax) {
  if (!M || !lmax) return fail(JXB_ERR_INVALID, "jxb_mg_info: null argument");
  for (size_t l = 0; l < M->L.size(); ++l) lmax[l] = M->L[l].lmax;
  return JXB_OK;
}

extern "C" int jxb_mg_vcycle(jxb_mg* M, jxb_stream stream, const double* r, double* z) {
  if (!M || !r || !z) return fail(JXB_ERR_INVALID, "jxb_mg_vcycle: null argument");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  Level& V = M->L[0];
  k_add_masked<<<grid_of(V.n), NB, 0, s>>>(nullptr, V.n, V.plan->d_keep, r, V.Rv, 1);
  int rc = vcycle(M, 0, s, nullptr);
  if (rc) return rc;
  JXB_CUDA(cudaMemcpyAsync(z, V.Z, V.n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  return JXB_OK;
}

// one PCG iteration (recorded into the graph)
static int mg_iteration(jxb_mg* M, cudaStream_t s) {
  Level& V = M->L[0];
  const long long n = V.n;
  int rc = launch_bricks<double>(V.plan, s, MODE_APPLY, M->p, nullptr, M->st, 1);
  if (rc) return rc;
  if ((rc = launch_combine<double>(V.plan, s, M->Ap, 1, M->p, M->part, M->st))) return rc;
  k_mg_xr<<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(M->st, n, M->part, M->x, M->r, M->p, M->Ap);
  k_add_masked<<<grid_of(n), NB, 0, s>>>(M->st, n, V.plan->d_keep, M->r, V.Rv, 1);
  if ((rc = vcycle(M, 0, s, M->st))) return rc;
  k_mg_rz<<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(M->st, n, M->r, V.Z, M->part, 0);
  k_mg_fin<<<1, JXB_RED_THREADS, 0, s>>>(M->st, M->part);
  k_mg_p<<<grid_of(n), NB, 0, s>>>(M->st, n, V.Z, M->p);
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

extern "C" int jxb_mg_pcg(jxb_mg* M, jxb_stream stream, const double* b, double* x, const jxb_solve_opts* opts,
                          jxb_stats* stats) {
  if (!M || !b || !x || !opts) return fail(JXB_ERR_INVALID, "jxb_mg_pcg: null argument");
  if (!(opts->tol > 0) || !isfinite(opts->tol)) return fail(JXB_ERR_INVALID, "jxb_mg_pcg: tol must be finite and positive");
  cudaStream_t user = reinterpret_cast<cudaStream_t>(stream), s = M->stream;
  SolveEvents ev;
  int rc = ev.create();
  if (rc) return rc;
  JXB_CUDA(cudaEventRecord(ev.order, user));
  JXB_CUDA(cudaStreamWaitEvent(s, ev.order, 0));
  Level& V = M->L[0];
  jxb_plan* P = V.plan;
  const long long n = V.n;
  const long long maxiter = opts->maxiter > 0 ? opts->maxiter : 10 * P->n_free;
  const int every = opts->check_every > 0 ? opts->check_every : 8;
  if (!M->graph || M->graph_iters != every) {
    if (M->graph) cudaGraphExecDestroy(M->graph);
    M->graph = nullptr;
    cudaGraph_t g;
    JXB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    int rci = 0;
    for (int it = 0; it < every && !rci; ++it) rci = mg_iteration(M, s);
    cudaError_t ce = cudaStreamEndCapture(s, &g);
    if (rci) return rci;
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
    ce = cudaGraphInstantiate(&M->graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaGraphInstantiate");
    M->graph_iters = every;
  }
  JXB_CUDA(cudaMemcpyAsync(M->b, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  JXB_CUDA(cudaEventRecord(ev.e0, s));
  k_mg_init<<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(n, M->b, P->d_keep, M->x, M->r, M->part);
  k_add_masked<<<grid_of(n), NB, 0, s>>>(nullptr, n, P->d_keep, M->r, V.Rv, 1);
  if ((rc = vcycle(M, 0, s, nullptr))) return rc;
  k_mg_rz<<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(nullptr, n, M->r, V.Z, M->part, 1);
  k_copy<<<grid_of(n), NB, 0, s>>>(n, V.Z, M->p);
  k_mg_start<<<1, JXB_RED_THREADS, 0, s>>>(M->st, M->part, opts->tol, opts->atol, maxiter);
  JXB_CUDA(cudaGetLastError());
  JXB_CUDA(cudaMemcpyAsync(M->h_st, M->st, sizeof(CgState), cudaMemcpyDeviceToHost, s));
  JXB_CUDA(cudaStreamSynchronize(s));
  const long long launches = maxiter / every + 2;
  for (long long l = 0; l < launches && !M->h_st->done; ++l) {
    JXB_CUDA(cudaGraphLaunch(M->graph, s));
    JXB_CUDA(cudaMemcpyAsync(M->h_st, M->st, sizeof(CgState), cudaMemcpyDeviceToHost, s));
    JXB_CUDA(cudaStreamSynchronize(s));
  }
  JXB_CUDA(cudaEventRecord(ev.e1, s));
  const long long iters = M->h_st->k;
  const int status = M->h_st->done ? M->h_st->status : JXB_ERR_NOT_CONVERGED;
  JXB_CUDA(cudaMemcpyAsync(x, M->x, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  double rn = 0, bn = 0;
  bool fin = true;
  if ((rc = true_residual(P, s, M->b, M->x, nullptr, &rn, &bn, &fin))) return rc;
  JXB_CUDA(cudaEventRecord(ev.order, s));
  JXB_CUDA(cudaStreamWaitEvent(user, ev.order, 0));
  float ms = 0;
  JXB_CUDA(cudaEventElapsedTime(&ms, ev.e0, ev.e1));
  return finish_solve("jxb_mg_pcg", stats, iters, 0, rn, bn, fin, opts->tol, opts->atol, ms, status == JXB_ERR_NONFINITE);
}
