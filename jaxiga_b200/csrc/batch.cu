// Batched solves: many independent single-patch problems of uneven size and
// degree solved together (the B200 form of the reference's vmap-over-params
// batching, tests/test_advanced.py:338-356, where the host SciPy solve runs
// once per batch member, src/jaxiga/solvers/linear.py:147-149).
//
// The instances' DOF vectors are concatenated. One CG iteration of the whole
// batch is:
//   * one brick launch per degree group, each CTA reading its instance's
//     arguments and brick index from the group's work list (or, with
//     JXB_BATCH_PERSIST=1 and rows of 32 elements, one persistent launch whose
//     CTAs take (instance, brick, degree) items of every degree off one list);
//   * one combine launch with one CTA per instance (its p.Ap reduction stays
//     inside the CTA, so it is deterministic);
//   * two vector kernels with one CTA per instance (x/r/z update with r.z and
//     r.r; p update and the instance's scalar state).
// Every kernel skips instances that have converged. `check_every`
// iterations are captured in one CUDA graph; the host reads the instances'
// 64-byte states after each graph launch and stops when all are done.
#include <math.h>
#include <stdlib.h>

#include <algorithm>
#include <map>
#include <set>
#include <string>
#include <vector>

#include "jxb_internal.cuh"

struct jxb_batch {
  int n = 0;
  std::vector<jxb_plan*> plans;
  std::vector<long long> off;  // n + 1
  long long total = 0;
  bool rational = false;
  long long* d_off = nullptr;
  uint8_t* d_keep = nullptr;
  double *d_b = nullptr, *d_x = nullptr, *d_r = nullptr, *d_z = nullptr, *d_p = nullptr, *d_Ap = nullptr,
         *d_inv = nullptr, *d_pAp = nullptr, *d_gnew = nullptr, *d_rrnew = nullptr, *d_part = nullptr;
  jxb::CgState* d_states = nullptr;
  jxb::CgState* h_states = nullptr;
  jxb::Bricks* d_brs = nullptr;
  double** d_scratch = nullptr;
  struct Group {
    int p, variant, fp0, fp1;
    long long n_work;
    int2* d_work = nullptr;
  };
  std::vector<Group> groups;
  // the persistent path: one work list over all degrees
  bool persist = false;
  int4* d_pwork = nullptr;
  int n_pwork = 0;
  unsigned* d_next = nullptr;  // self-resetting work counter
  int pgrid = 0;
  size_t psmem = 0;
  jxb::BrickArgs<double>* d_args_p = nullptr;  // x = p (the CG direction)
  jxb::BrickArgs<double>* d_args_x = nullptr;  // x = x (true residual)
  cudaGraphExec_t graph = nullptr;
  int graph_iters = 0;
  cudaStream_t stream = nullptr;
};

namespace jxb {
namespace {

__device__ double block_sum_b(double v) {
  __shared__ double part[32];
  __shared__ double total;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) part[w] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int i = 0; i < (int)((blockDim.x + 31) >> 5); ++i) s += part[i];
    total = s;
  }
  __syncthreads();
  double r = total;
  __syncthreads();
  return r;
}

// y = combine of instance blockIdx.x (2D), optional p.y into dot_out[inst]. The
// CTA is large (one CTA serves a whole instance, up to ~17k control points)
// and issues the loads of all covering bricks of a control point together.
constexpr int BATCH_COMBINE_THREADS = 512;

__global__ void __launch_bounds__(BATCH_COMBINE_THREADS)
    k_combine_batch(const Bricks* __restrict__ brs, double* const* __restrict__ scratch,
                    const long long* __restrict__ off, const uint8_t* __restrict__ keep, double* __restrict__ y,
                    const double* __restrict__ dot_with, double* __restrict__ dot_out,
                    const CgState* __restrict__ states) {
  const int inst = blockIdx.x;
  if (states && states[inst].done) return;
  const Bricks& br = brs[inst];
  const double* sc = scratch[inst];
  const long long o = off[inst];
  const long long n_scalar = (long long)br.n_cp[0] * br.n_cp[1];
  double part = 0;
  for (long long i = threadIdx.x; i < n_scalar; i += blockDim.x) {
    const int ix = (int)(i % br.n_cp[0]), iy = (int)(i / br.n_cp[0]);
    double sv[1];
    combine_point<double, 1, 2>(br, sc, ix, iy, 0, sv);
    double s = sv[0];
    const long long dof = o + i;
    if (!keep[dof]) s = 0;
    y[dof] = s;
    if (dot_with) part += dot_with[dof] * s;
  }
  if (dot_out) {
    const double t = block_sum_b(part);
    if (threadIdx.x == 0) dot_out[inst] = t;
  }
}

__global__ void __launch_bounds__(256) k_bcg_init(const long long* __restrict__ off, const double* __restrict__ b,
                                                  const uint8_t* __restrict__ keep, const double* __restrict__ inv,
                                                  double* x, double* r, double* z, double* p, CgState* states,
                                                  double tol, double atol, long long maxiter) {
  const int inst = blockIdx.x;
  const long long lo = off[inst], hi = off[inst + 1];
  double rz = 0, rr = 0;
  for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    const double bi = keep[i] ? b[i] : 0.0;
    const double zi = inv[i] * bi;
    x[i] = 0;
    r[i] = bi;
    z[i] = zi;
    p[i] = zi;
    rz += bi * zi;
    rr += bi * bi;
  }
  rz = block_sum_b(rz);
  rr = block_sum_b(rr);
  if (threadIdx.x == 0) {
    CgState& st = states[inst];
    st.gamma = rz;
    st.rr = rr;
    st.bb = rr;
    st.atol2 = fmax(tol * tol * rr, atol * atol);
    st.k = 0;
    st.maxiter = maxiter;
    st.alpha = st.beta = 0;
    st.status = JXB_OK;
    st.done = !(rr > st.atol2) ? 1 : 0;
    if (!isfinite(rr)) {
      st.done = 1;
      st.status = JXB_ERR_NONFINITE;
    }
  }
}

__global__ void __launch_bounds__(256) k_bcg_xr(const long long* __restrict__ off, const CgState* __restrict__ states,
                                                const double* __restrict__ pAp, double* x, double* r, double* z,
                                                const double* __restrict__ p, const double* __restrict__ Ap,
                                                const double* __restrict__ inv, double* gnew, double* rrnew) {
  const int inst = blockIdx.x;
  if (states[inst].done) return;
  const long long lo = off[inst], hi = off[inst + 1];
  const double alpha = states[inst].gamma / pAp[inst];
  double rz = 0, rr = 0;
  for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    x[i] += alpha * p[i];
    const double ri = r[i] - alpha * Ap[i];
    r[i] = ri;
    const double zi = inv[i] * ri;
    z[i] = zi;
    rz += ri * zi;
    rr += ri * ri;
  }
  rz = block_sum_b(rz);
  rr = block_sum_b(rr);
  if (threadIdx.x == 0) {
    gnew[inst] = rz;
    rrnew[inst] = rr;
  }
}

__global__ void __launch_bounds__(256) k_bcg_p(const long long* __restrict__ off, CgState* states,
                                               const double* __restrict__ pAp, const double* __restrict__ gnew,
                                               const double* __restrict__ rrnew, const double* __restrict__ z,
                                               double* p) {
  const int inst = blockIdx.x;
  CgState& st = states[inst];
  if (st.done) return;
  const long long lo = off[inst], hi = off[inst + 1];
  const double g = gnew[inst], gamma = st.gamma;
  const double beta = g / gamma;
  for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) p[i] = z[i] + beta * p[i];
  __syncthreads();  // every thread has read st.gamma before it changes
  if (threadIdx.x == 0) {
    const double rr = rrnew[inst], pa = pAp[inst];
    st.alpha = gamma / pa;
    st.beta = beta;
    st.gamma = g;
    st.rr = rr;
    st.k += 1;
    if (!isfinite(rr) || !isfinite(g) || !isfinite(pa) || pa == 0.0) {
      st.done = 1;
      st.status = JXB_ERR_NONFINITE;
    } else if (!(rr > st.atol2)) {
      st.done = 1;
    } else if (st.k >= st.maxiter) {
      st.done = 1;
      st.status = JXB_ERR_NOT_CONVERGED;
    }
  }
}

// per-instance ||b - Ax||^2 and ||b||^2 over free DOFs
__global__ void __launch_bounds__(256) k_bres(const long long* __restrict__ off, const double* __restrict__ b,
                                              const double* __restrict__ Ax, const double* __restrict__ x,
                                              const uint8_t* __restrict__ keep, double* out) {
  const int inst = blockIdx.x;
  const long long lo = off[inst], hi = off[inst + 1];
  double rr = 0, bb = 0, bad = 0;
  for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    if (keep[i]) {
      const double ri = b[i] - Ax[i];
      rr += ri * ri;
      bb += b[i] * b[i];
    }
    if (!isfinite(x[i])) bad += 1;
  }
  rr = block_sum_b(rr);
  bb = block_sum_b(bb);
  bad = block_sum_b(bad);
  if (threadIdx.x == 0) {
    out[3 * inst] = rr;
    out[3 * inst + 1] = bb;
    out[3 * inst + 2] = bad;
  }
}

int batch_apply(jxb_batch* B, cudaStream_t s, const BrickArgs<double>* d_args, double* y, const double* dot_with,
                double* dot_out, const CgState* states) {
  if (B->persist) {
    int rc = launch_bricks2_persist(B->rational, d_args, B->d_pwork, B->n_pwork, B->d_next, B->pgrid, B->psmem,
                                    states, s);
    if (rc) return rc;
  }
  for (auto& g : B->groups) {
    if (B->persist) break;
    int rc = launch_bricks2_batch(g.p, B->rational, g.variant, d_args, g.d_work, g.n_work, g.fp0, g.fp1, states, s);
    if (rc) return rc;
  }
  k_combine_batch<<<B->n, BATCH_COMBINE_THREADS, 0, s>>>(B->d_brs, B->d_scratch, B->d_off, B->d_keep, y, dot_with, dot_out, states);
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

void free_batch(jxb_batch* B) {
  if (!B) return;
  void* bufs[] = {B->d_off, B->d_keep, B->d_b, B->d_x, B->d_r, B->d_z, B->d_p, B->d_Ap, B->d_inv, B->d_pAp,
                  B->d_gnew, B->d_rrnew, B->d_part, B->d_states, B->d_brs, B->d_scratch, B->d_args_p, B->d_args_x};
  for (void* p : bufs) cudaFree(p);
  for (auto& g : B->groups) cudaFree(g.d_work);
  cudaFree(B->d_pwork);
  cudaFree(B->d_next);
  if (B->h_states) cudaFreeHost(B->h_states);
  if (B->graph) cudaGraphExecDestroy(B->graph);
  if (B->stream) cudaStreamDestroy(B->stream);
  delete B;
}

}  // namespace
}  // namespace jxb

using namespace jxb;

extern "C" int jxb_batch_create(jxb_plan* const* plans, int n, jxb_batch** out) {
  if (!plans || n < 1 || !out) return fail(JXB_ERR_INVALID, "jxb_batch_create: bad argument");
  *out = nullptr;
  // Every instance writes its brick partial sums into its own plan's scratch
  // inside the shared launches, so a plan listed twice would race with itself.
  // (checked on the pointers alone, before any plan is read)
  std::set<const jxb_plan*> seen;
  for (int i = 0; i < n; ++i) {
    if (!plans[i]) return fail(JXB_ERR_INVALID, "jxb_batch_create: null plan");
    if (!seen.insert(plans[i]).second)
      return fail(JXB_ERR_INVALID, "jxb_batch_create: plan " + std::to_string(i) +
                                       " appears more than once; create one plan per instance");
  }
  for (int i = 0; i < n; ++i) {
    if (plans[i]->mp || plans[i]->thb) return fail(JXB_ERR_INVALID, "jxb_batch_create: not available on a multipatch or hierarchical plan");
    if (plans[i]->dim != 2 || plans[i]->op != JXB_OP_POISSON)
      return fail(JXB_ERR_INVALID, "jxb_batch_create: batches take 2D Poisson plans");
    if (plans[i]->rational != plans[0]->rational)
      return fail(JXB_ERR_INVALID, "jxb_batch_create: all plans must be rational or all non-rational");
  }
  jxb_batch* B = new jxb_batch();
  B->n = n;
  B->plans.assign(plans, plans + n);
  B->rational = plans[0]->rational != 0;
  B->off.resize(n + 1, 0);
  for (int i = 0; i < n; ++i) B->off[i + 1] = B->off[i] + plans[i]->n_dofs;
  B->total = B->off[n];
  auto fail_b = [&](int code) {
    if (B->stream) cudaStreamSynchronize(B->stream);
    free_batch(B);
    return code;
  };
#define JXB_CUDA_B(call)                                         \
  do {                                                           \
    cudaError_t _e = (call);                                     \
    if (_e != cudaSuccess) return fail_b(cuda_fail(_e, #call)); \
  } while (0)
  const size_t N = (size_t)B->total;
  cudaError_t e = cudaSuccess;
  auto al = [&](void** p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, std::max<size_t>(bytes, 8));
  };
  al((void**)&B->d_off, (n + 1) * sizeof(long long));
  al((void**)&B->d_keep, N);
  for (double** p : {&B->d_b, &B->d_x, &B->d_r, &B->d_z, &B->d_p, &B->d_Ap, &B->d_inv}) al((void**)p, N * sizeof(double));
  for (double** p : {&B->d_pAp, &B->d_gnew, &B->d_rrnew}) al((void**)p, n * sizeof(double));
  al((void**)&B->d_part, 3 * n * sizeof(double));
  al((void**)&B->d_states, n * sizeof(CgState));
  al((void**)&B->d_brs, n * sizeof(Bricks));
  al((void**)&B->d_scratch, n * sizeof(double*));
  al((void**)&B->d_args_p, n * sizeof(BrickArgs<double>));
  al((void**)&B->d_args_x, n * sizeof(BrickArgs<double>));
  if (e != cudaSuccess) return fail_b(cuda_fail(e, "jxb_batch_create: cudaMalloc"));
  if ((e = cudaMallocHost(&B->h_states, n * sizeof(CgState))) != cudaSuccess) return fail_b(cuda_fail(e, "cudaMallocHost"));
  if ((e = cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking)) != cudaSuccess)
    return fail_b(cuda_fail(e, "cudaStreamCreate"));
  cudaStream_t s = B->stream;
  std::vector<Bricks> brs(n);
  std::vector<double*> scr(n);
  std::vector<BrickArgs<double>> ap(n), ax(n);
  std::map<std::pair<int, int>, std::vector<int2>> work;  // (p, variant) -> work list
  std::map<std::pair<int, int>, std::pair<int, int>> fpmax;
  for (int i = 0; i < n; ++i) {
    jxb_plan* P = plans[i];
    brs[i] = P->br;
    scr[i] = P->d_scratch;
    ap[i] = make_brick_args<double>(P, B->d_p + B->off[i], nullptr, 1);
    ax[i] = make_brick_args<double>(P, B->d_x + B->off[i], nullptr, 1);
    const int v = tile2_variant(P->br.te[0], P->br.te[1]);
    if (v < 0) return fail_b(fail(JXB_ERR_INVALID, "jxb_batch_create: unsupported brick shape"));
    auto key = std::make_pair(P->p, v);
    for (long long b = 0; b < P->br.n_bricks; ++b) work[key].push_back(make_int2(i, (int)b));
    auto& f = fpmax[key];
    f.first = std::max(f.first, P->br.fp[0]);
    f.second = std::max(f.second, P->br.fp[1]);
    // keep mask of this instance into the concatenated mask
    JXB_CUDA_B(cudaMemcpyAsync(B->d_keep + B->off[i], P->d_keep, P->n_dofs, cudaMemcpyDeviceToDevice, s));
  }
  for (auto& kv : work) {
    jxb_batch::Group g;
    g.p = kv.first.first;
    g.variant = kv.first.second;
    g.fp0 = fpmax[kv.first].first;
    g.fp1 = fpmax[kv.first].second;
    // largest instances first: long bricks start early (better load balance)
    std::stable_sort(kv.second.begin(), kv.second.end(), [&](int2 a, int2 b) {
      return plans[a.x]->n_elem > plans[b.x]->n_elem;
    });
    g.n_work = (long long)kv.second.size();
    if ((e = cudaMalloc(&g.d_work, g.n_work * sizeof(int2))) != cudaSuccess) return fail_b(cuda_fail(e, "cudaMalloc"));
    JXB_CUDA_B(cudaMemcpyAsync(g.d_work, kv.second.data(), g.n_work * sizeof(int2), cudaMemcpyHostToDevice, s));
    B->groups.push_back(g);
  }
  // The persistent path on request (JXB_BATCH_PERSIST=1) when every instance has
  // rows of 32 elements: highest degree first, then the largest instances. It is
  // not the default: each of its CTAs reserves the shared memory of the largest
  // degree, which caps the resident CTAs per SM, and on the 256-annuli batch it
  // measured 0.93 ms per K.u against 0.48 ms for the per-degree launches.
  {
    const char* env = getenv("JXB_BATCH_PERSIST");
    bool ok = env && env[0] == '1';
    for (int i = 0; i < n && ok; ++i) ok = plans[i]->br.te[0] == PERSIST2_TX && plans[i]->p >= 1 && plans[i]->p <= 5;
    if (ok) {
      std::vector<int4> items;
      for (int i = 0; i < n; ++i) {
        const jxb_plan* P = plans[i];
        B->psmem = std::max(B->psmem, smem2_scalar_apply(P->p, B->rational, PERSIST2_TX, P->br.fp[0], P->br.fp[1]));
        for (long long b = 0; b < P->br.n_bricks; ++b) items.push_back(make_int4(i, (int)b, P->p, 0));
      }
      std::stable_sort(items.begin(), items.end(), [&](int4 a, int4 b) {
        if (a.z != b.z) return a.z > b.z;
        return plans[a.x]->n_elem > plans[b.x]->n_elem;
      });
      if (items.size() > (size_t)0x7fffffff) return fail_b(fail(JXB_ERR_INVALID, "jxb_batch_create: too many bricks"));
      B->n_pwork = (int)items.size();
      int rc = persist2_grid(B->rational, B->psmem, &B->pgrid);
      if (rc) return fail_b(rc);
      if ((e = cudaMalloc(&B->d_pwork, items.size() * sizeof(int4))) != cudaSuccess)
        return fail_b(cuda_fail(e, "cudaMalloc"));
      if ((e = cudaMalloc(&B->d_next, sizeof(unsigned))) != cudaSuccess) return fail_b(cuda_fail(e, "cudaMalloc"));
      JXB_CUDA_B(cudaMemsetAsync(B->d_next, 0, sizeof(unsigned), s));
      JXB_CUDA_B(cudaMemcpyAsync(B->d_pwork, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
      B->persist = true;
    }
  }
  JXB_CUDA_B(cudaMemcpyAsync(B->d_off, B->off.data(), (n + 1) * sizeof(long long), cudaMemcpyHostToDevice, s));
  JXB_CUDA_B(cudaMemcpyAsync(B->d_brs, brs.data(), n * sizeof(Bricks), cudaMemcpyHostToDevice, s));
  JXB_CUDA_B(cudaMemcpyAsync(B->d_scratch, scr.data(), n * sizeof(double*), cudaMemcpyHostToDevice, s));
  JXB_CUDA_B(cudaMemcpyAsync(B->d_args_p, ap.data(), n * sizeof(BrickArgs<double>), cudaMemcpyHostToDevice, s));
  JXB_CUDA_B(cudaMemcpyAsync(B->d_args_x, ax.data(), n * sizeof(BrickArgs<double>), cudaMemcpyHostToDevice, s));
  // Jacobi inverse diagonal of every instance, concatenated
  for (int i = 0; i < n; ++i) {
    jxb_plan* P = plans[i];
    int rc = ensure_workspace(P, false);
    if (rc) return fail_b(rc);
    if ((rc = compute_invdiag(P, s))) return fail_b(rc);
    JXB_CUDA_B(cudaMemcpyAsync(B->d_inv + B->off[i], P->d_invdiag, P->n_dofs * sizeof(double),
                             cudaMemcpyDeviceToDevice, s));
  }
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return fail_b(cuda_fail(e, "jxb_batch_create"));
  *out = B;
  return JXB_OK;
#undef JXB_CUDA_B
}

extern "C" int jxb_batch_destroy(jxb_batch* B) {
  if (!B) return JXB_OK;
  cudaStreamSynchronize(B->stream);
  free_batch(B);
  return JXB_OK;
}

extern "C" int jxb_batch_size(const jxb_batch* B, int64_t* total_dofs, int64_t* offsets) {
  if (!B || !total_dofs) return fail(JXB_ERR_INVALID, "jxb_batch_size: null argument");
  *total_dofs = B->total;
  if (offsets)
    for (int i = 0; i <= B->n; ++i) offsets[i] = B->off[i];
  return JXB_OK;
}

extern "C" int jxb_batch_info(const jxb_batch* B, int* persistent, int* brick_launches) {
  if (!B || !persistent || !brick_launches) return fail(JXB_ERR_INVALID, "jxb_batch_info: null argument");
  *persistent = B->persist ? 1 : 0;
  *brick_launches = B->persist ? 1 : (int)B->groups.size();
  return JXB_OK;
}

extern "C" int jxb_batch_apply(jxb_batch* B, jxb_stream stream, const double* x, double* y) {
  if (!B || !x || !y) return fail(JXB_ERR_INVALID, "jxb_batch_apply: null argument");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  JXB_CUDA(cudaMemcpyAsync(B->d_p, x, B->total * sizeof(double), cudaMemcpyDeviceToDevice, s));
  return batch_apply(B, s, B->d_args_p, y, nullptr, nullptr, nullptr);
}

extern "C" int jxb_batch_pcg(jxb_batch* B, jxb_stream stream, const double* b, double* x, const jxb_solve_opts* opts,
                             jxb_stats* stats, double* seconds) {
  if (!B || !b || !x || !opts) return fail(JXB_ERR_INVALID, "jxb_batch_pcg: null argument");
  cudaStream_t user = reinterpret_cast<cudaStream_t>(stream);
  cudaStream_t s = B->stream;
  SolveEvents evs;
  if (int rc0 = evs.create()) return rc0;
  cudaEvent_t ev = evs.order, e0 = evs.e0, e1 = evs.e1;
  JXB_CUDA(cudaEventRecord(ev, user));
  JXB_CUDA(cudaStreamWaitEvent(s, ev, 0));
  const int n = B->n;
  long long maxiter = opts->maxiter;
  if (maxiter <= 0) {
    maxiter = 0;
    for (auto* P : B->plans) maxiter = std::max(maxiter, 10 * P->n_free);
  }
  const int every = opts->check_every > 0 ? opts->check_every : 16;
  JXB_CUDA(cudaMemcpyAsync(B->d_b, b, B->total * sizeof(double), cudaMemcpyDeviceToDevice, s));
  JXB_CUDA(cudaEventRecord(e0, s));
  k_bcg_init<<<n, 256, 0, s>>>(B->d_off, B->d_b, B->d_keep, B->d_inv, B->d_x, B->d_r, B->d_z, B->d_p, B->d_states,
                               opts->tol, opts->atol, maxiter);
  JXB_CUDA(cudaGetLastError());
  if (!B->graph || B->graph_iters != every) {
    if (B->graph) cudaGraphExecDestroy(B->graph);
    B->graph = nullptr;
    cudaGraph_t g;
    JXB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    int rc = 0;
    for (int it = 0; it < every && !rc; ++it) {
      rc = batch_apply(B, s, B->d_args_p, B->d_Ap, B->d_p, B->d_pAp, B->d_states);
      if (rc) break;
      k_bcg_xr<<<n, 256, 0, s>>>(B->d_off, B->d_states, B->d_pAp, B->d_x, B->d_r, B->d_z, B->d_p, B->d_Ap, B->d_inv,
                                 B->d_gnew, B->d_rrnew);
      k_bcg_p<<<n, 256, 0, s>>>(B->d_off, B->d_states, B->d_pAp, B->d_gnew, B->d_rrnew, B->d_z, B->d_p);
    }
    cudaError_t ce = cudaStreamEndCapture(s, &g);
    if (rc) return rc;
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
    ce = cudaGraphInstantiate(&B->graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaGraphInstantiate");
    B->graph_iters = every;
  }
  long long launches = maxiter / every + 2;
  JXB_CUDA(cudaMemcpyAsync(B->h_states, B->d_states, n * sizeof(CgState), cudaMemcpyDeviceToHost, s));
  JXB_CUDA(cudaStreamSynchronize(s));
  auto all_done = [&]() {
    for (int i = 0; i < n; ++i)
      if (!B->h_states[i].done) return false;
    return true;
  };
  for (long long l = 0; l < launches && !all_done(); ++l) {
    JXB_CUDA(cudaGraphLaunch(B->graph, s));
    JXB_CUDA(cudaMemcpyAsync(B->h_states, B->d_states, n * sizeof(CgState), cudaMemcpyDeviceToHost, s));
    JXB_CUDA(cudaStreamSynchronize(s));
  }
  JXB_CUDA(cudaEventRecord(e1, s));
  JXB_CUDA(cudaMemcpyAsync(x, B->d_x, B->total * sizeof(double), cudaMemcpyDeviceToDevice, s));
  // FP64 true residuals of every instance
  int rc = batch_apply(B, s, B->d_args_x, B->d_Ap, nullptr, nullptr, nullptr);
  if (rc) return rc;
  k_bres<<<n, 256, 0, s>>>(B->d_off, B->d_b, B->d_Ap, B->d_x, B->d_keep, B->d_part);
  std::vector<double> h(3 * n);
  JXB_CUDA(cudaMemcpyAsync(h.data(), B->d_part, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  JXB_CUDA(cudaStreamSynchronize(s));
  float ms = 0;
  JXB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  JXB_CUDA(cudaEventRecord(ev, s));
  JXB_CUDA(cudaStreamWaitEvent(user, ev, 0));
  if (seconds) *seconds = ms * 1e-3;
  int nonfinite = -1, unconverged = -1;
  for (int i = 0; i < n; ++i) {
    const double rn = sqrt(h[3 * i]), bn = sqrt(h[3 * i + 1]);
    const bool fin = h[3 * i + 2] == 0 && isfinite(rn);
    jxb_stats one;
    const int st = finish_solve("jxb_batch_pcg", &one, B->h_states[i].k, 0, rn, bn, fin, opts->tol, opts->atol, ms,
                                B->h_states[i].status == JXB_ERR_NONFINITE);
    if (stats) stats[i] = one;
    if (st == JXB_ERR_NONFINITE && nonfinite < 0) nonfinite = i;
    if (st == JXB_ERR_NOT_CONVERGED && unconverged < 0) unconverged = i;
  }
  if (nonfinite >= 0)
    return fail(JXB_ERR_NONFINITE, "jxb_batch_pcg: non-finite value in instance " + std::to_string(nonfinite));
  if (unconverged >= 0)
    return fail(JXB_ERR_NOT_CONVERGED, "jxb_batch_pcg: instance " + std::to_string(unconverged) +
                                           " (and maybe others) missed the tolerance; see its stats");
  return JXB_OK;
}
