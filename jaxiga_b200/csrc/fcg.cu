// Flexible CG with a learned (CNN) preconditioner.
//
// FCG(1) in the form of Notay (SIAM J. Sci. Comput. 22, 2000): the search
// direction is the preconditioned residual made A-orthogonal to the previous
// direction only, p_k = z_k - (z_k . A p_{k-1} / p_{k-1} . A p_{k-1}) p_{k-1},
// alpha_k = (p_k . r_k) / (p_k . A p_k). It tolerates a preconditioner that is
// not a fixed linear SPD map, which a ReLU network is not.
//
// The preconditioner maps the residual r to z = ||r|| * out_scale * N(r / ||r|| * in_scale, features),
// N the network applied on the control-point grid (channels: the vec residual
// components, then the caller's static feature channels such as a
// log-coefficient field). Scaling by ||r|| makes the map homogeneous of degree
// one. Jacobi-PCG is the fallback: if a learned direction is not a descent
// direction (p . A p <= 0) or the residual stops decreasing for `stall`
// iterations, the remaining iterations use z = D^-1 r. Stopping rule and
// true-residual diagnostics are those of jxb_pcg.
#include <math.h>

#include <vector>

#include "jxb_internal.cuh"

extern "C" int jxb_cnn_forward(struct jxb_cnn* N, jxb_stream stream, int nx, int ny, int nz, const float* in, float* out);

namespace jxb {

__global__ void k_pack_in(long long ncp, int vec, const double* __restrict__ r, const uint8_t* __restrict__ keep,
                          float s, float* __restrict__ in) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncp * vec) return;
  long long cp = i / vec;
  int c = (int)(i % vec);
  in[(long long)c * ncp + cp] = keep[i] ? (float)(r[i] * s) : 0.f;
}

__global__ void k_unpack_out(long long ncp, int vec, const float* __restrict__ out, const uint8_t* __restrict__ keep,
                             double s, double* __restrict__ z) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncp * vec) return;
  long long cp = i / vec;
  int c = (int)(i % vec);
  z[i] = keep[i] ? s * (double)out[(long long)c * ncp + cp] : 0.0;
}

__global__ void k_jacobi(long long n, const double* __restrict__ inv, const double* __restrict__ r, double* __restrict__ z) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) z[i] = inv[i] * r[i];
}

__global__ void k_dir(long long n, const double* __restrict__ z, double beta, const double* __restrict__ pp,
                      double* __restrict__ p) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = z[i] - beta * pp[i];
}

__global__ void k_step(long long n, double alpha, const double* __restrict__ p, const double* __restrict__ Ap,
                       double* __restrict__ x, double* __restrict__ r) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    x[i] += alpha * p[i];
    r[i] -= alpha * Ap[i];
  }
}

__global__ void k_resid(long long n, const double* __restrict__ b, const double* __restrict__ Ax,
                        const uint8_t* __restrict__ keep, double* __restrict__ out) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = keep[i] ? b[i] - Ax[i] : 0.0;
}

__global__ void k_mask_copy(long long n, const double* __restrict__ b, const uint8_t* __restrict__ keep, double* __restrict__ r) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) r[i] = keep[i] ? b[i] : 0.0;
}

}  // namespace jxb

using namespace jxb;

extern "C" int jxb_fcg_learned(jxb_plan* plan, struct jxb_cnn* cnn, jxb_stream stream, const double* b, double* x,
                               const float* features, int n_features, float in_scale, double out_scale, int stall,
                               const jxb_solve_opts* opts, jxb_stats* stats) {
  if (!plan || !cnn || !b || !x || !opts) return fail(JXB_ERR_INVALID, "jxb_fcg_learned: null argument");
  if (n_features < 0 || (n_features > 0 && !features)) return fail(JXB_ERR_INVALID, "jxb_fcg_learned: bad features");
  if (!(opts->tol > 0)) return fail(JXB_ERR_INVALID, "jxb_fcg_learned: tol must be positive");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int rc = ensure_workspace(plan, false);
  if (rc) return rc;
  rc = compute_invdiag(plan, s);
  if (rc) return rc;
  const long long n = plan->n_dofs, ncp = plan->n_scalar;
  const int vec = plan->vec;
  double *tmp1 = nullptr, *tmp2 = nullptr;
  float *in = nullptr, *out = nullptr;
  JXB_CUDA(cudaMalloc(&tmp1, n * sizeof(double)));
  JXB_CUDA(cudaMalloc(&tmp2, n * sizeof(double)));
  JXB_CUDA(cudaMalloc(&in, (size_t)(vec + n_features) * ncp * sizeof(float)));
  JXB_CUDA(cudaMalloc(&out, (size_t)vec * ncp * sizeof(float)));
  if (n_features)
    JXB_CUDA(cudaMemcpyAsync(in + (size_t)vec * ncp, features, (size_t)n_features * ncp * sizeof(float),
                             cudaMemcpyDeviceToDevice, s));
  double *xv = plan->d_x, *r = plan->d_r, *z = plan->d_z;
  double *p = plan->d_p, *Ap = plan->d_Ap, *pp = tmp1, *App = tmp2;  // current / previous direction
  const unsigned nb = (unsigned)((n + 255) / 256);
  cudaEvent_t e0, e1;
  JXB_CUDA(cudaEventCreate(&e0));
  JXB_CUDA(cudaEventCreate(&e1));
  JXB_CUDA(cudaEventRecord(e0, s));
  JXB_CUDA(cudaMemsetAsync(xv, 0, n * sizeof(double), s));
  k_mask_copy<<<nb, 256, 0, s>>>(n, b, plan->d_keep, r);
  double bb = 0;
  if ((rc = dot(plan, s, r, r, &bb))) return rc;
  const double atol2 = fmax(opts->tol * opts->tol * bb, opts->atol * opts->atol);
  const long long maxiter = opts->maxiter > 0 ? opts->maxiter : 10 * plan->n_free;
  double rr = bb, best = bb, pAp_prev = 0;
  long long k = 0, since_best = 0, learned_iters = 0;
  bool use_learned = true, fresh = true;
  int status = JXB_OK;
  const int nx = plan->n_cp[0], ny = plan->n_cp[1], nz = plan->dim == 3 ? plan->n_cp[2] : 1;
  while (rr > atol2 && k < maxiter) {
    const double rn = sqrt(rr);
    if (use_learned) {
      k_pack_in<<<(unsigned)((ncp * vec + 255) / 256), 256, 0, s>>>(ncp, vec, r, plan->d_keep, (float)(in_scale / rn), in);
      if ((rc = jxb_cnn_forward(cnn, stream, nx, ny, nz, in, out))) return rc;
      k_unpack_out<<<(unsigned)((ncp * vec + 255) / 256), 256, 0, s>>>(ncp, vec, out, plan->d_keep, rn * out_scale, z);
    } else {
      k_jacobi<<<nb, 256, 0, s>>>(n, plan->d_invdiag, r, z);
    }
    if (!fresh) {
      double zAp = 0;
      if ((rc = dot(plan, s, z, App, &zAp))) return rc;
      k_dir<<<nb, 256, 0, s>>>(n, z, zAp / pAp_prev, pp, p);
    } else {
      JXB_CUDA(cudaMemcpyAsync(p, z, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    if ((rc = launch_bricks<double>(plan, s, MODE_APPLY, p, nullptr, nullptr, 1))) return rc;
    if ((rc = launch_combine<double>(plan, s, Ap, 1, nullptr, nullptr, nullptr))) return rc;
    double pAp = 0, pr = 0;
    if ((rc = dot(plan, s, p, Ap, &pAp))) return rc;
    if ((rc = dot(plan, s, p, r, &pr))) return rc;
    if (!(pAp > 0) || !isfinite(pAp) || !isfinite(pr)) {
      if (use_learned) {  // the learned direction is unusable: continue with Jacobi
        use_learned = false;
        fresh = true;
        ++k;
        continue;
      }
      status = JXB_ERR_NONFINITE;
      break;
    }
    k_step<<<nb, 256, 0, s>>>(n, pr / pAp, p, Ap, xv, r);
    std::swap(p, pp);
    std::swap(Ap, App);
    pAp_prev = pAp;
    fresh = false;
    if ((rc = dot(plan, s, r, r, &rr))) return rc;
    ++k;
    if (use_learned) ++learned_iters;
    if (rr < best) {
      best = rr;
      since_best = 0;
    } else if (++since_best >= stall && use_learned) {
      use_learned = false;  // stagnation: finish with Jacobi directions
      fresh = true;
      since_best = 0;
    }
  }
  if (status == JXB_OK && rr > atol2) status = JXB_ERR_NOT_CONVERGED;
  JXB_CUDA(cudaEventRecord(e1, s));
  JXB_CUDA(cudaMemcpyAsync(x, xv, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  // FP64 true residual (the check of src/jaxiga/solvers/diagnostics.py:8-19)
  if ((rc = launch_bricks<double>(plan, s, MODE_APPLY, xv, nullptr, nullptr, 1))) return rc;
  if ((rc = launch_combine<double>(plan, s, tmp1, 1, nullptr, nullptr, nullptr))) return rc;
  k_resid<<<nb, 256, 0, s>>>(n, b, tmp1, plan->d_keep, tmp2);
  double res2 = 0;
  if ((rc = dot(plan, s, tmp2, tmp2, &res2))) return rc;
  float ms = 0;
  JXB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(tmp1);
  cudaFree(tmp2);
  cudaFree(in);
  cudaFree(out);
  if (stats) {
    const double res = sqrt(res2), bn = sqrt(bb);
    stats->iterations = k;
    stats->outer = learned_iters;
    stats->residual = res;
    stats->b_norm = bn;
    stats->relative_residual = res / (bn > 0 ? bn : 1.0);
    stats->finite = isfinite(res) ? 1 : 0;
    stats->converged = (isfinite(res) && res <= opts->tol * bn) ? 1 : 0;
    stats->seconds = ms * 1e-3;
  }
  if (status == JXB_ERR_NONFINITE) return fail(JXB_ERR_NONFINITE, "jxb_fcg_learned: non-finite value");
  return JXB_OK;
}
