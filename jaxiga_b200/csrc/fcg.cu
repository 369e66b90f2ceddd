// Flexible CG with a learned (CNN) preconditioner, and the energy-norm
// training step of that network.
//
// Truncated flexible CG, FCG(m) in the form of Notay (SIAM J. Sci. Comput.
// 22, 2000): the search direction is the preconditioned residual made
// A-orthogonal to the last m directions,
//   p_k = z_k - sum_{j=k-m}^{k-1} (z_k . A p_j / p_j . A p_j) p_j,
//   alpha_k = (p_k . r_k) / (p_k . A p_k).
// It tolerates a preconditioner that is not a fixed linear SPD map, which a
// ReLU network is not; m > 1 keeps the global A-orthogonality that a varying
// preconditioner otherwise loses.
//
// The preconditioner maps r to z = ||r|| out_scale N(in_scale r/||r||, features),
// N the network on the control-point grid (channels: the vec residual
// components, then static features such as a log-coefficient). Scaling by
// ||r|| makes the map homogeneous of degree one. Jacobi is the fallback: a
// learned direction with p . A p <= 0, or `stall` learned iterations without
// a new lowest residual, restart the recurrence with z = D^-1 r (which, with
// a fixed SPD preconditioner, is plain PCG). Stopping rule and true-residual
// diagnostics are those of jxb_pcg (src/jaxiga/solvers/linear.py:399-442,
// src/jaxiga/solvers/diagnostics.py:8-19).
//
// Device-resident: every scalar of the recurrence lives in a device state
// block; one iteration is pack, network, unpack (or Jacobi), multi-dot,
// direction, brick apply, combine (+ p.Ap partials), p.r partials and ring
// copies, x/r update (+ r.r partials), finish. It is captured once into a
// CUDA graph (one iteration per launch for the learned mode, `check_every`
// for Jacobi) and every kernel but the network's returns at once when the
// device `done` flag is set. Reductions use a fixed grid and order.
#include <math.h>

#include <vector>

#include "jxb_internal.cuh"

namespace jxb {

constexpr int FCG_MMAX = 8;

struct FcgState {
  CgState cg;              // rr, alpha, atol2, k (= iterations), maxiter, done, status
  double pAp[FCG_MMAX];    // ring: p_j . A p_j of the stored directions
  long long nd;            // directions stored since the last restart
  int bad;                 // the last direction had p . A p <= 0 or was not finite
  int m;                   // ring length
};

template <typename T>
__global__ void k_fpack(long long ncp, int vec, const T* __restrict__ r, const uint8_t* __restrict__ keep,
                        float in_scale, const FcgState* st, float* __restrict__ in) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncp * vec) return;
  const double rr = st->cg.rr;
  const float s = (!st->cg.done && rr > 0) ? (float)(in_scale / sqrt(rr)) : 0.f;
  const long long cp = i / vec;
  const int c = (int)(i % vec);
  in[(long long)c * ncp + cp] = keep[i] ? (float)r[i] * s : 0.f;
}

template <typename T>
__global__ void k_funpack(long long ncp, int vec, const float* __restrict__ out, const uint8_t* __restrict__ keep,
                          double out_scale, const FcgState* st, T* __restrict__ z) {
  if (st->cg.done) return;
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncp * vec) return;
  const long long cp = i / vec;
  const int c = (int)(i % vec);
  z[i] = keep[i] ? (T)(sqrt(st->cg.rr) * out_scale * (double)out[(long long)c * ncp + cp]) : T(0);
}

template <typename T>
__global__ void k_fjac(long long n, const T* __restrict__ inv, const T* __restrict__ r, const FcgState* st,
                       T* __restrict__ z) {
  if (st->cg.done) return;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    z[i] = inv[i] * r[i];
}

// partials of z . r (two-level mode)
template <typename T>
__global__ void __launch_bounds__(JXB_RED_THREADS) k_fzr(long long n, const FcgState* st, const T* __restrict__ z,
                                                         const T* __restrict__ r, double* __restrict__ partials) {
  if (st->cg.done) return;
  double acc = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    acc += (double)z[i] * (double)r[i];
  const double s = block_sum_all(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// two-level preconditioner: z <- a z + D^-1 (r - a K z), a = (z.r)/(z.Kz), the
// network output taken as a coarse correction with its own line search and
// followed by one Jacobi step on the remaining residual
template <typename T>
__global__ void __launch_bounds__(JXB_RED_THREADS) k_ftwolevel(long long n, const FcgState* st, const double* __restrict__ zkz_part,
                                                               const double* __restrict__ zr_part, const T* __restrict__ Kz,
                                                               const T* __restrict__ r, const T* __restrict__ inv, T* __restrict__ z) {
  if (st->cg.done) return;
  const double zkz = reduce_partials(zkz_part), zr = reduce_partials(zr_part);
  const T a = (zkz > 0 && isfinite(zkz) && isfinite(zr)) ? (T)(zr / zkz) : T(0);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    z[i] = a * z[i] + inv[i] * (r[i] - a * Kz[i]);
}

// additive two-level preconditioner: z <- z + D^-1 r, the network output z
// (its weight folded into out_scale) plus one Jacobi step on r
template <typename T>
__global__ void k_fadd(long long n, const FcgState* st, const T* __restrict__ inv, const T* __restrict__ r,
                       T* __restrict__ z) {
  if (st->cg.done) return;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    z[i] += inv[i] * r[i];
}

// ring slot of stored direction d (0-based since the last restart)
__device__ __forceinline__ int fcg_slot(long long d, int m) { return (int)(d % m); }

// partials[j][block] = z . A p_{nd-1-j}, j < min(nd, m)
template <typename T>
__global__ void __launch_bounds__(JXB_RED_THREADS) k_fmdot(long long n, const FcgState* st, const T* __restrict__ z,
                                                           const T* __restrict__ APr, double* __restrict__ partials) {
  if (st->cg.done) return;
  const int m = st->m;
  const long long nd = st->nd;
  const int jn = (int)(nd < m ? nd : m);
  double acc[FCG_MMAX];
#pragma unroll
  for (int j = 0; j < FCG_MMAX; ++j) acc[j] = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double zi = (double)z[i];
#pragma unroll
    for (int j = 0; j < FCG_MMAX; ++j)
      if (j < jn) acc[j] += zi * (double)APr[(long long)fcg_slot(nd - 1 - j, m) * n + i];
  }
#pragma unroll
  for (int j = 0; j < FCG_MMAX; ++j) {
    if (j >= jn) break;  // jn is uniform across the block
    const double s = block_sum_all(acc[j]);
    if (threadIdx.x == 0) partials[j * JXB_RED_BLOCKS + blockIdx.x] = s;
  }
}

// p = z - sum_j beta_j p_{nd-1-j}, beta_j = (z . A p_j) / (p_j . A p_j)
template <typename T>
__global__ void __launch_bounds__(JXB_RED_THREADS) k_fdir(long long n, const FcgState* st, const T* __restrict__ z,
                                                          const T* __restrict__ Pr, const double* __restrict__ partials,
                                                          T* __restrict__ p) {
  if (st->cg.done) return;
  const int m = st->m;
  const long long nd = st->nd;
  const int jn = (int)(nd < m ? nd : m);
  T beta[FCG_MMAX];
#pragma unroll
  for (int j = 0; j < FCG_MMAX; ++j) {
    beta[j] = T(0);
    if (j < jn) beta[j] = (T)(reduce_partials(partials + j * JXB_RED_BLOCKS) / st->pAp[fcg_slot(nd - 1 - j, m)]);
  }
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    T v = z[i];
#pragma unroll
    for (int j = 0; j < FCG_MMAX; ++j)
      if (j < jn) v -= beta[j] * Pr[(long long)fcg_slot(nd - 1 - j, m) * n + i];
    p[i] = v;
  }
}

// p.r partials; p and A p copied into ring slot nd % m
template <typename T>
__global__ void __launch_bounds__(JXB_RED_THREADS) k_fpr(long long n, const FcgState* st, const T* __restrict__ p,
                                                         const T* __restrict__ Ap, const T* __restrict__ r,
                                                         T* __restrict__ Pr, T* __restrict__ APr,
                                                         double* __restrict__ partials) {
  if (st->cg.done) return;
  const long long off = (long long)fcg_slot(st->nd, st->m) * n;
  double acc = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const T pi = p[i];
    Pr[off + i] = pi;
    APr[off + i] = Ap[i];
    acc += (double)pi * (double)r[i];
  }
  const double s = block_sum_all(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// x += alpha p, r -= alpha A p (+ r.r partials); skipped for a bad direction
template <typename T>
__global__ void __launch_bounds__(JXB_RED_THREADS) k_fupdate(long long n, const FcgState* st, const double* __restrict__ pap_part,
                                                             const double* __restrict__ pr_part, const T* __restrict__ p,
                                                             const T* __restrict__ Ap, T* __restrict__ x, T* __restrict__ r,
                                                             double* __restrict__ rr_part) {
  if (st->cg.done) return;
  const double pAp = reduce_partials(pap_part), pr = reduce_partials(pr_part);
  if (!(pAp > 0) || !isfinite(pAp) || !isfinite(pr)) return;
  const T alpha = (T)(pr / pAp);
  double acc = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    x[i] += alpha * p[i];
    const T ri = r[i] - alpha * Ap[i];
    r[i] = ri;
    acc += (double)ri * (double)ri;
  }
  const double s = block_sum_all(acc);
  if (threadIdx.x == 0) rr_part[blockIdx.x] = s;
}

__global__ void k_ffin(FcgState* st, const double* __restrict__ pap_part, const double* __restrict__ pr_part,
                       const double* __restrict__ rr_part) {
  if (st->cg.done) return;
  const double pAp = reduce_partials(pap_part), pr = reduce_partials(pr_part);
  const bool bad = !(pAp > 0) || !isfinite(pAp) || !isfinite(pr);
  const double rr = bad ? 0.0 : reduce_partials(rr_part);
  if (threadIdx.x != 0) return;
  if (bad) {
    st->bad = 1;
    st->cg.done = 1;
    return;
  }
  st->pAp[fcg_slot(st->nd, st->m)] = pAp;
  st->nd += 1;
  st->cg.k += 1;
  st->cg.alpha = pr / pAp;
  st->cg.rr = rr;
  if (!isfinite(rr)) {
    st->cg.done = 1;
    st->cg.status = JXB_ERR_NONFINITE;
  } else if (!(rr > st->cg.atol2)) {
    st->cg.done = 1;
  } else if (st->cg.k >= st->cg.maxiter) {
    st->cg.done = 1;
    st->cg.status = JXB_ERR_NOT_CONVERGED;
  }
}

template <typename T, typename TB>
__global__ void __launch_bounds__(JXB_RED_THREADS) k_finit(long long n, const TB* __restrict__ b, const uint8_t* __restrict__ keep,
                                                           T* __restrict__ x, T* __restrict__ r, double* __restrict__ part) {
  double acc = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const T bi = keep[i] ? (T)b[i] : T(0);
    x[i] = T(0);
    r[i] = bi;
    acc += (double)bi * (double)bi;
  }
  const double s = block_sum_all(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void k_finit_fin(FcgState* st, const double* __restrict__ part, double tol, double atol, long long maxiter, int m) {
  const double bb = reduce_partials(part);
  if (threadIdx.x != 0) return;
  st->cg.rr = bb;
  st->cg.bb = bb;
  st->cg.gamma = 0;
  st->cg.alpha = st->cg.beta = 0;
  st->cg.atol2 = fmax(tol * tol * bb, atol * atol);
  st->cg.k = 0;
  st->cg.maxiter = maxiter;
  st->cg.status = JXB_OK;
  st->cg.done = 0;
  st->nd = 0;
  st->bad = 0;
  st->m = m;
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

// restart the recurrence (after a bad learned direction or a stall)
__global__ void k_frestart(FcgState* st) {
  st->nd = 0;
  st->bad = 0;
  if (st->cg.status == JXB_OK && st->cg.k < st->cg.maxiter && st->cg.rr > st->cg.atol2) st->cg.done = 0;
}

// Reliable update of the FP32 recurrence (mixed mode): r32 = s res (the FP64
// residual scaled to unit norm), x32 = 0, and the stored directions and their
// products rescaled to the new units (P, AP *= ratio; p.Ap *= ratio^2 in the
// finish kernel), so the A-orthogonalisation carries on across the update.
__global__ void __launch_bounds__(JXB_RED_THREADS) k_fru_restart(long long n, int m, const double* __restrict__ res,
                                                                 const uint8_t* __restrict__ keep, double s,
                                                                 float ratio, int first, float* __restrict__ x,
                                                                 float* __restrict__ r, float* __restrict__ Pr,
                                                                 float* __restrict__ APr, double* __restrict__ part) {
  double acc = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float ri = keep[i] ? (float)(res[i] * s) : 0.f;
    x[i] = 0.f;
    r[i] = ri;
    acc += (double)ri * (double)ri;
    if (!first)
      for (int j = 0; j < m; ++j) {
        Pr[(long long)j * n + i] *= ratio;
        APr[(long long)j * n + i] *= ratio;
      }
  }
  const double t = block_sum_all(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void k_fru_fin(FcgState* st, const double* __restrict__ part, double tol, long long maxiter, int m,
                          int first, double ratio) {
  const double rr = reduce_partials(part);
  if (threadIdx.x != 0) return;
  st->cg.rr = rr;
  st->cg.bb = rr;
  st->cg.gamma = 0;
  st->cg.alpha = st->cg.beta = 0;
  st->cg.atol2 = tol * tol * rr;
  st->cg.k = 0;
  st->cg.maxiter = maxiter;
  st->cg.status = JXB_OK;
  st->cg.done = 0;
  st->bad = 0;
  if (first) {
    st->nd = 0;
    st->m = m;
  } else {
    for (int j = 0; j < FCG_MMAX; ++j) st->pAp[j] *= ratio * ratio;
  }
  if (!isfinite(rr)) {
    st->cg.done = 1;
    st->cg.status = JXB_ERR_NONFINITE;
  } else if (!(rr > st->cg.atol2)) {
    st->cg.done = 1;
  } else if (maxiter <= 0) {
    st->cg.done = 1;
    st->cg.status = JXB_ERR_NOT_CONVERGED;
  }
}

template <typename T>
__global__ void k_ediff(long long ncp, int vec, const float* __restrict__ e, const float* __restrict__ out,
                        float out_scale, const uint8_t* __restrict__ keep, T* __restrict__ d) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncp * vec) return;
  const long long cp = i / vec;
  const int c = (int)(i % vec);
  const long long g = (long long)c * ncp + cp;
  d[i] = keep[i] ? (T)e[g] - (T)out_scale * (T)out[g] : T(0);
}

template <typename T>
__global__ void k_egrad(long long ncp, int vec, const T* __restrict__ Kd, const uint8_t* __restrict__ keep, double s,
                        float* __restrict__ g) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncp * 4) return;
  const int c = (int)(i / ncp);
  const long long cp = i % ncp;
  float v = 0.f;
  if (c < vec) {
    const long long dof = cp * vec + c;
    v = keep[dof] ? (float)(s * (double)Kd[dof]) : 0.f;
  }
  g[i] = v;
}

// z = keep ? out_scale * out : 0 in DOF layout
__global__ void k_zdof(long long ncp, int vec, const float* __restrict__ out, float out_scale,
                       const uint8_t* __restrict__ keep, double* __restrict__ z) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncp * vec) return;
  const long long cp = i / vec;
  const int c = (int)(i % vec);
  z[i] = keep[i] ? (double)out_scale * (double)out[(long long)c * ncp + cp] : 0.0;
}

// z += D^-1 r (r in grid layout [vec][ncp]; inv is 0 on prescribed DOFs):
// the additive two-level map whose network part is being trained
__global__ void k_zadd_jacobi(long long ncp, int vec, const float* __restrict__ r, const double* __restrict__ inv,
                              double* __restrict__ z) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncp * vec) return;
  z[i] += inv[i] * (double)r[(long long)(i % vec) * ncp + i / vec];
}

// partials of z . r and e . r over free DOFs (r, e: grid layout [vec][ncp])
__global__ void __launch_bounds__(JXB_RED_THREADS) k_angle_dots(long long ncp, int vec, const double* __restrict__ z,
                                                                const float* __restrict__ r, const float* __restrict__ e,
                                                                const uint8_t* __restrict__ keep, double* __restrict__ part) {
  double zr = 0, er = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < ncp * vec;
       i += (long long)gridDim.x * blockDim.x) {
    if (!keep[i]) continue;
    const long long g = (long long)(i % vec) * ncp + i / vec;
    const double ri = (double)r[g];
    zr += z[i] * ri;
    er += (double)e[g] * ri;
  }
  const double s0 = block_sum_all(zr), s1 = block_sum_all(er);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = s0;
    part[JXB_RED_BLOCKS + blockIdx.x] = s1;
  }
}

// gout[c][cp] = keep ? s1 * Kz - s2 * r : 0 (4 channels, the extra ones 0)
__global__ void k_angle_grad(long long ncp, int vec, const double* __restrict__ Kz, const float* __restrict__ r,
                             const uint8_t* __restrict__ keep, double s1, double s2, float* __restrict__ g) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncp * 4) return;
  const int c = (int)(i / ncp);
  const long long cp = i % ncp;
  float v = 0.f;
  if (c < vec) {
    const long long dof = cp * vec + c;
    v = keep[dof] ? (float)(s1 * Kz[dof] - s2 * (double)r[i]) : 0.f;
  }
  g[i] = v;
}

__global__ void k_to_f32(long long n, const double* __restrict__ r, double s, float* __restrict__ out) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (float)(r[i] * s);
}

__global__ void k_axpy_f32(long long n, double a, const float* __restrict__ d, double* __restrict__ x) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += a * (double)d[i];
}

namespace {

inline unsigned nb256(long long n) { return (unsigned)((n + 255) / 256); }

// One FCG run's buffers and settings.
struct FcgRun {
  jxb_plan* plan;
  jxb_cnn* cnn;
  const float* features;
  int n_features;
  float in_scale;
  double out_scale;
  int stall, m, every;
  bool two_level = false;
  bool additive = false;
  bool sticky_fallback = false;  // a fallback to Jacobi lasts for the rest of the solve
  bool net_off = false;
  FcgState *d_st = nullptr, *h_st = nullptr;
  double* part = nullptr;  // (FCG_MMAX + 3) x JXB_RED_BLOCKS
  float* in = nullptr;
  void *Pr = nullptr, *APr = nullptr;
  long long learned_iters = 0;
  ~FcgRun() {
    cudaFree(d_st);
    cudaFreeHost(h_st);
    cudaFree(part);
    cudaFree(in);
    cudaFree(Pr);
    cudaFree(APr);
  }
};

template <typename T>
int record_iteration(FcgRun& R, cudaStream_t s, bool learned, int iters) {
  jxb_plan* plan = R.plan;
  constexpr bool F32 = sizeof(T) == 4;
  T* x = F32 ? (T*)plan->d_x32 : (T*)plan->d_x;
  T* r = F32 ? (T*)plan->d_r32 : (T*)plan->d_r;
  T* z = F32 ? (T*)plan->d_z32 : (T*)plan->d_z;
  T* p = F32 ? (T*)plan->d_p32 : (T*)plan->d_p;
  T* Ap = F32 ? (T*)plan->d_Ap32 : (T*)plan->d_Ap;
  const T* inv = F32 ? (const T*)plan->d_invdiag32 : (const T*)plan->d_invdiag;
  const long long n = plan->n_dofs, ncp = plan->n_scalar;
  const int vec = plan->vec;
  double* pm = R.part;
  double* pap = R.part + FCG_MMAX * JXB_RED_BLOCKS;
  double* ppr = pap + JXB_RED_BLOCKS;
  double* prr = ppr + JXB_RED_BLOCKS;
  const int nx = plan->n_cp[0], ny = plan->n_cp[1], nz = plan->dim == 3 ? plan->n_cp[2] : 1;
  for (int it = 0; it < iters; ++it) {
    if (learned) {
      k_fpack<T><<<nb256(ncp * vec), 256, 0, s>>>(ncp, vec, r, plan->d_keep, R.in_scale, R.d_st, R.in);
      const float* out4 = nullptr;
      int rc = cnn_forward(R.cnn, s, nx, ny, nz, R.in, &out4, true);
      if (rc) return rc;
      k_funpack<T><<<nb256(ncp * vec), 256, 0, s>>>(ncp, vec, out4, plan->d_keep, R.out_scale, R.d_st, z);
      if (R.two_level) {  // K z into Ap (free until the direction's apply), z.Kz and z.r partials
        int rc2 = launch_bricks<T>(plan, s, MODE_APPLY, z, nullptr, &R.d_st->cg, 1);
        if (rc2) return rc2;
        rc2 = launch_combine<T>(plan, s, Ap, 1, z, pap, &R.d_st->cg);
        if (rc2) return rc2;
        k_fzr<T><<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(n, R.d_st, z, r, ppr);
        k_ftwolevel<T><<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(n, R.d_st, pap, ppr, Ap, r, inv, z);
      } else if (R.additive) {
        k_fadd<T><<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(n, R.d_st, inv, r, z);
      }
    } else {
      k_fjac<T><<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(n, inv, r, R.d_st, z);
    }
    k_fmdot<T><<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(n, R.d_st, z, (const T*)R.APr, pm);
    k_fdir<T><<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(n, R.d_st, z, (const T*)R.Pr, pm, p);
    int rc = launch_bricks<T>(plan, s, MODE_APPLY, p, nullptr, &R.d_st->cg, 1);
    if (rc) return rc;
    rc = launch_combine<T>(plan, s, Ap, 1, p, pap, &R.d_st->cg);
    if (rc) return rc;
    k_fpr<T><<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(n, R.d_st, p, Ap, r, (T*)R.Pr, (T*)R.APr, ppr);
    k_fupdate<T><<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(n, R.d_st, pap, ppr, p, Ap, x, r, prr);
    k_ffin<<<1, JXB_RED_THREADS, 0, s>>>(R.d_st, pap, ppr, prr);
  }
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

template <typename T>
int capture(FcgRun& R, cudaStream_t s, bool learned, int iters, cudaGraphExec_t* out) {
  cudaGraph_t g;
  JXB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
  int rc = record_iteration<T>(R, s, learned, iters);
  cudaError_t e = cudaStreamEndCapture(s, &g);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
  return JXB_OK;
}

struct GraphPair {
  cudaGraphExec_t learned = nullptr, jacobi = nullptr;
  ~GraphPair() {
    if (learned) cudaGraphExecDestroy(learned);
    if (jacobi) cudaGraphExecDestroy(jacobi);
  }
};

// Allocates the run's buffers for vectors of type T (the network input keeps
// the feature channels after the vec residual channels).
template <typename T>
int fcg_setup(FcgRun& R, cudaStream_t s) {
  jxb_plan* plan = R.plan;
  const long long n = plan->n_dofs, ncp = plan->n_scalar;
  JXB_CUDA(cudaMalloc(&R.d_st, sizeof(FcgState)));
  JXB_CUDA(cudaMallocHost(&R.h_st, sizeof(FcgState)));
  JXB_CUDA(cudaMalloc(&R.part, (FCG_MMAX + 3) * JXB_RED_BLOCKS * sizeof(double)));
  JXB_CUDA(cudaMalloc(&R.Pr, (size_t)R.m * n * sizeof(T)));
  JXB_CUDA(cudaMalloc(&R.APr, (size_t)R.m * n * sizeof(T)));
  if (R.cnn) {
    JXB_CUDA(cudaMalloc(&R.in, (size_t)(plan->vec + R.n_features) * ncp * sizeof(float)));
    JXB_CUDA(cudaMemsetAsync(R.in, 0, (size_t)plan->vec * ncp * sizeof(float), s));
    if (R.n_features)
      JXB_CUDA(cudaMemcpyAsync(R.in + (size_t)plan->vec * ncp, R.features, (size_t)R.n_features * ncp * sizeof(float),
                               cudaMemcpyDeviceToDevice, s));
    // one forward outside capture sizes the network's activation buffers
    const int nx = plan->n_cp[0], ny = plan->n_cp[1], nz = plan->dim == 3 ? plan->n_cp[2] : 1;
    int rc = cnn_forward(R.cnn, s, nx, ny, nz, R.in, nullptr, true);
    if (rc) return rc;
  }
  return JXB_OK;
}

template <typename T>
int fcg_loop(FcgRun& R, GraphPair& G, cudaStream_t s, long long maxiter, long long* iters, int* status);

// Runs FCG on rhs b (type TB) into the plan's T-typed x. Returns the status
// (JXB_OK, NOT_CONVERGED, NONFINITE) in *status and the iteration count.
template <typename T, typename TB>
int fcg_run(FcgRun& R, GraphPair& G, cudaStream_t s, const TB* b, double tol, double atol, long long maxiter,
            long long* iters, int* status) {
  jxb_plan* plan = R.plan;
  constexpr bool F32 = sizeof(T) == 4;
  T* x = F32 ? (T*)plan->d_x32 : (T*)plan->d_x;
  T* r = F32 ? (T*)plan->d_r32 : (T*)plan->d_r;
  const long long n = plan->n_dofs;
  k_finit<T, TB><<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(n, b, plan->d_keep, x, r, R.part);
  k_finit_fin<<<1, JXB_RED_THREADS, 0, s>>>(R.d_st, R.part, tol, atol, maxiter, R.m);
  JXB_CUDA(cudaGetLastError());
  return fcg_loop<T>(R, G, s, maxiter, iters, status);
}

// Launches the iteration graphs until the device state reports done (state and
// vectors set up by the caller); learned directions first, Jacobi after a fallback.
template <typename T>
int fcg_loop(FcgRun& R, GraphPair& G, cudaStream_t s, long long maxiter, long long* iters, int* status) {
  bool learned = R.cnn != nullptr && !R.net_off;
  if (learned && !G.learned) {
    int rc = capture<T>(R, s, true, 1, &G.learned);
    if (rc) return rc;
  }
  if (!G.jacobi) {
    int rc = capture<T>(R, s, false, R.every, &G.jacobi);
    if (rc) return rc;
  }
  JXB_CUDA(cudaMemcpyAsync(R.h_st, R.d_st, sizeof(FcgState), cudaMemcpyDeviceToHost, s));
  JXB_CUDA(cudaStreamSynchronize(s));
  double best = R.h_st->cg.rr;
  long long since = 0;
  const long long cap = maxiter + 2;  // every launch advances k unless done; bounded in any case
  for (long long l = 0; l < cap && !R.h_st->cg.done; ++l) {
    const long long k0 = R.h_st->cg.k;
    JXB_CUDA(cudaGraphLaunch(learned ? G.learned : G.jacobi, s));
    JXB_CUDA(cudaMemcpyAsync(R.h_st, R.d_st, sizeof(FcgState), cudaMemcpyDeviceToHost, s));
    JXB_CUDA(cudaStreamSynchronize(s));
    const FcgState& h = *R.h_st;
    if (learned) {
      R.learned_iters += h.cg.k - k0;
      if (h.cg.rr < best) {
        best = h.cg.rr;
        since = 0;
      } else {
        since += h.cg.k - k0;
      }
      if (h.bad || since >= R.stall) {  // fall back to Jacobi directions
        learned = false;
        R.net_off = R.sticky_fallback;
        k_frestart<<<1, 1, 0, s>>>(R.d_st);
        JXB_CUDA(cudaGetLastError());
        JXB_CUDA(cudaMemcpyAsync(R.h_st, R.d_st, sizeof(FcgState), cudaMemcpyDeviceToHost, s));
        JXB_CUDA(cudaStreamSynchronize(s));
      }
    } else if (h.bad) {  // Jacobi direction without descent: breakdown
      *iters = h.cg.k;
      *status = JXB_ERR_NONFINITE;
      return JXB_OK;
    }
  }
  *iters = R.h_st->cg.k;
  *status = R.h_st->cg.done ? R.h_st->cg.status : JXB_ERR_NOT_CONVERGED;
  if (R.h_st->cg.done && R.h_st->cg.status == JXB_OK && R.h_st->cg.rr > R.h_st->cg.atol2)
    *status = JXB_ERR_NOT_CONVERGED;
  return JXB_OK;
}

}  // namespace
}  // namespace jxb

using namespace jxb;

extern "C" int jxb_fcg_learned(jxb_plan* plan, jxb_cnn* cnn, jxb_stream stream, const double* b, double* x,
                               const float* features, int n_features, float in_scale, double out_scale, int stall,
                               int depth, int mode, const jxb_solve_opts* opts, jxb_stats* stats) {
  if (plan && (plan->mp || plan->thb)) return fail(JXB_ERR_INVALID, "jxb_fcg_learned: not available on a multipatch or hierarchical plan");
  const int mixed = mode & 1;
  if (!plan || !b || !x || !opts) return fail(JXB_ERR_INVALID, "jxb_fcg_learned: null argument");
  if (n_features < 0 || (n_features > 0 && !features)) return fail(JXB_ERR_INVALID, "jxb_fcg_learned: bad features");
  if (cnn && cnn_out_channels(cnn) != plan->vec)
    return fail(JXB_ERR_INVALID, "jxb_fcg_learned: the network's outputs must equal the plan's vec");
  if (!(opts->tol > 0) || !isfinite(opts->tol)) return fail(JXB_ERR_INVALID, "jxb_fcg_learned: tol must be finite and positive");
  if (depth < 1 || depth > FCG_MMAX) return fail(JXB_ERR_INVALID, "jxb_fcg_learned: depth must be in 1..8");
  if (mixed && !plan->d_geo32) return fail(JXB_ERR_INVALID, "jxb_fcg_learned: mixed needs a plan created with want_f32");
  cudaStream_t user = reinterpret_cast<cudaStream_t>(stream);
  if (!plan->graph_stream[1]) JXB_CUDA(cudaStreamCreateWithFlags(&plan->graph_stream[1], cudaStreamNonBlocking));
  cudaStream_t s = plan->graph_stream[1];
  SolveEvents ev;
  int rc = ev.create();
  if (rc) return rc;
  cudaEvent_t e0 = ev.e0, e1 = ev.e1, evu = ev.order;
  JXB_CUDA(cudaEventRecord(evu, user));
  JXB_CUDA(cudaStreamWaitEvent(s, evu, 0));
  rc = ensure_workspace(plan, mixed != 0);
  if (rc) return rc;
  rc = compute_invdiag(plan, s);
  if (rc) return rc;
  const long long n = plan->n_dofs;
  FcgRun R;
  R.plan = plan;
  R.cnn = cnn;
  R.features = features;
  R.n_features = n_features;
  R.in_scale = in_scale;
  R.out_scale = out_scale;
  R.stall = stall > 0 ? stall : 1 << 30;
  R.m = depth;
  R.every = opts->check_every > 0 ? opts->check_every : 16;
  R.two_level = (mode & 2) != 0;
  R.additive = (mode & 8) != 0 && !R.two_level;
  GraphPair G;
  rc = mixed ? fcg_setup<float>(R, s) : fcg_setup<double>(R, s);
  if (rc) return rc;
  const long long maxiter = opts->maxiter > 0 ? opts->maxiter : 10 * plan->n_free;
  JXB_CUDA(cudaMemcpyAsync(plan->d_b, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  JXB_CUDA(cudaEventRecord(e0, s));
  long long total = 0, outer = 0;
  int status = JXB_OK;
  double rn = 0, bn = 0;
  bool fin = true;
  if (!mixed) {
    rc = fcg_run<double, double>(R, G, s, plan->d_b, opts->tol, opts->atol, maxiter, &total, &status);
    if (rc) return rc;
    JXB_CUDA(cudaEventRecord(e1, s));
    JXB_CUDA(cudaMemcpyAsync(x, plan->d_x, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    rc = true_residual(plan, s, plan->d_b, plan->d_x, nullptr, &rn, &bn, &fin);
    if (rc) return rc;
  } else if (!(mode & 4)) {
    // FP32 FCG with reliable FP64 updates: each time the FP32 residual has
    // fallen by inner_tol (default 1e-2) or below the target, the FP32 iterate
    // is added to the FP64 solution and the residual recomputed in FP64; the
    // stored directions are kept (rescaled), so the recurrence goes on.
    double* xb = plan->d_z;
    double* res = plan->d_r;
    JXB_CUDA(cudaMemsetAsync(xb, 0, n * sizeof(double), s));
    const double delta = opts->inner_tol > 0 ? opts->inner_tol : 1e-2;
    const int max_updates = opts->max_outer > 0 ? opts->max_outer : 1000;
    rc = true_residual(plan, s, plan->d_b, xb, res, &rn, &bn, &fin);
    if (rc) return rc;
    double rn_seg = rn;
    R.sticky_fallback = true;  // the segments continue one recurrence
    while (outer < max_updates && fin && rn > opts->tol * bn && total < maxiter) {
      const int first = outer == 0;
      const double ratio = first ? 1.0 : rn_seg / rn;
      k_fru_restart<<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(n, R.m, res, plan->d_keep, 1.0 / rn, (float)ratio, first,
                                                               plan->d_x32, plan->d_r32, (float*)R.Pr, (float*)R.APr,
                                                               R.part);
      k_fru_fin<<<1, JXB_RED_THREADS, 0, s>>>(R.d_st, R.part, fmax(delta, opts->tol * bn / rn), maxiter - total, R.m,
                                              first, ratio);
      JXB_CUDA(cudaGetLastError());
      rn_seg = rn;
      long long it = 0;
      int st = 0;
      rc = fcg_loop<float>(R, G, s, maxiter - total, &it, &st);
      if (rc) return rc;
      total += it;
      k_axpy_f32<<<nb256(n), 256, 0, s>>>(n, rn_seg, plan->d_x32, xb);
      JXB_CUDA(cudaGetLastError());
      rc = true_residual(plan, s, plan->d_b, xb, res, &rn, &bn, &fin);
      if (rc) return rc;
      ++outer;
      if (st == JXB_ERR_NONFINITE) {
        status = JXB_ERR_NONFINITE;
        break;
      }
      if (!(rn < rn_seg)) break;  // no progress: stop, the stats report it
    }
    JXB_CUDA(cudaEventRecord(e1, s));
    JXB_CUDA(cudaMemcpyAsync(x, xb, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  } else {
    // FP64 iterative refinement: the FP64 residual, normalised, is the rhs of
    // an FP32 FCG solve to inner_tol; the correction is added in FP64.
    double* xb = plan->d_z;
    double* res = plan->d_r;
    JXB_CUDA(cudaMemsetAsync(xb, 0, n * sizeof(double), s));
    const double inner = opts->inner_tol > 0 ? opts->inner_tol : 1e-4;
    const int max_outer = opts->max_outer > 0 ? opts->max_outer : 30;
    rc = true_residual(plan, s, plan->d_b, xb, res, &rn, &bn, &fin);
    if (rc) return rc;
    while (outer < max_outer && fin && rn > opts->tol * bn && total < maxiter) {
      float* rhs32 = plan->d_Ap32;  // copied into r32 by the FCG init before Ap32 is reused
      k_to_f32<<<nb256(n), 256, 0, s>>>(n, res, 1.0 / rn, rhs32);
      // the inner tolerance never asks for more than the outer target needs
      const double itol = fmax(inner, 0.5 * opts->tol * bn / rn);
      long long it = 0;
      int st = 0;
      rc = fcg_run<float, float>(R, G, s, rhs32, itol, 0.0, maxiter - total, &it, &st);
      if (rc) return rc;
      total += it;
      k_axpy_f32<<<nb256(n), 256, 0, s>>>(n, rn, plan->d_x32, xb);
      JXB_CUDA(cudaGetLastError());
      const double prev = rn;
      rc = true_residual(plan, s, plan->d_b, xb, res, &rn, &bn, &fin);
      if (rc) return rc;
      ++outer;
      if (st == JXB_ERR_NONFINITE) {
        status = JXB_ERR_NONFINITE;
        break;
      }
      if (!(rn < prev)) break;  // stagnation: stop, the stats report it
    }
    JXB_CUDA(cudaEventRecord(e1, s));
    JXB_CUDA(cudaMemcpyAsync(x, xb, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  }
  JXB_CUDA(cudaEventRecord(evu, s));
  JXB_CUDA(cudaStreamWaitEvent(user, evu, 0));
  JXB_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  JXB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  return finish_solve("jxb_fcg_learned", stats, total, R.learned_iters, rn, bn, fin, opts->tol, opts->atol, ms,
                      status == JXB_ERR_NONFINITE);
}

extern "C" int jxb_cnn_accumulate_energy(jxb_plan* plan, jxb_cnn* cnn, jxb_stream stream, const float* in,
                                         const float* e, const float* r, float out_scale, double weight, int angle,
                                         double* loss) {
  if (plan && (plan->mp || plan->thb)) return fail(JXB_ERR_INVALID, "jxb_cnn_accumulate_energy: not available on a multipatch or hierarchical plan");
  if (!plan || !cnn || !in || !e || (angle && !r)) return fail(JXB_ERR_INVALID, "jxb_cnn_accumulate_energy: null argument");
  if (cnn_out_channels(cnn) != plan->vec)
    return fail(JXB_ERR_INVALID, "jxb_cnn_accumulate_energy: the network's outputs must equal the plan's vec");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (angle < 0 || angle > 2) return fail(JXB_ERR_INVALID, "jxb_cnn_accumulate_energy: angle must be 0, 1 or 2");
  int rc = ensure_workspace(plan, false);
  if (rc) return rc;
  if (angle == 2 && (rc = compute_invdiag(plan, s))) return rc;
  const long long ncp = plan->n_scalar;
  const int vec = plan->vec;
  const int nx = plan->n_cp[0], ny = plan->n_cp[1], nz = plan->dim == 3 ? plan->n_cp[2] : 1;
  const float* out4 = nullptr;
  if ((rc = cnn_forward(cnn, s, nx, ny, nz, in, &out4))) return rc;
  double* d = plan->d_p;
  double* Kd = plan->d_Ap;
  std::vector<double> h(3 * JXB_RED_BLOCKS);
  double value = 0;
  if (!angle) {
    // loss = weight d^T K d, d = P_f (e - s N(in)); dL/dN = -2 weight s K d
    k_ediff<double><<<nb256(ncp * vec), 256, 0, s>>>(ncp, vec, e, out4, out_scale, plan->d_keep, d);
    if ((rc = launch_bricks<double>(plan, s, MODE_APPLY, d, nullptr, nullptr, 1))) return rc;
    if ((rc = launch_combine<double>(plan, s, Kd, 1, d, plan->d_red, nullptr))) return rc;
    k_egrad<double><<<nb256(ncp * 4), 256, 0, s>>>(ncp, vec, Kd, plan->d_keep, -2.0 * weight * out_scale,
                                                    cnn_grad_out(cnn));
    JXB_CUDA(cudaGetLastError());
    JXB_CUDA(cudaMemcpyAsync(h.data(), plan->d_red, JXB_RED_BLOCKS * sizeof(double), cudaMemcpyDeviceToHost, s));
    JXB_CUDA(cudaStreamSynchronize(s));
    double dkd = 0;
    for (int i = 0; i < JXB_RED_BLOCKS; ++i) dkd += h[i];
    value = weight * dkd;
  } else {
    // scale-free: loss = weight (1 - (z.r)^2 / ((z^T K z)(e.r))), z = P_f s N(in), r = K e;
    // dL/dz = weight 2a/(b c) ((a/b) K z - r), a = z.r, b = z^T K z, c = e.r.
    // angle == 2: z = P_f s N(in) + D^-1 r (the additive two-level map), same dL/dN
    k_zdof<<<nb256(ncp * vec), 256, 0, s>>>(ncp, vec, out4, out_scale, plan->d_keep, d);
    if (angle == 2) k_zadd_jacobi<<<nb256(ncp * vec), 256, 0, s>>>(ncp, vec, r, plan->d_invdiag, d);
    if ((rc = launch_bricks<double>(plan, s, MODE_APPLY, d, nullptr, nullptr, 1))) return rc;
    if ((rc = launch_combine<double>(plan, s, Kd, 1, d, plan->d_red, nullptr))) return rc;
    k_angle_dots<<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(ncp, vec, d, r, e, plan->d_keep,
                                                             plan->d_red + JXB_RED_BLOCKS);
    JXB_CUDA(cudaGetLastError());
    JXB_CUDA(cudaMemcpyAsync(h.data(), plan->d_red, 3 * JXB_RED_BLOCKS * sizeof(double), cudaMemcpyDeviceToHost, s));
    JXB_CUDA(cudaStreamSynchronize(s));
    double bq = 0, a = 0, c = 0;
    for (int i = 0; i < JXB_RED_BLOCKS; ++i) {
      bq += h[i];
      a += h[JXB_RED_BLOCKS + i];
      c += h[2 * JXB_RED_BLOCKS + i];
    }
    if (!(bq > 0) || !(c > 0) || !isfinite(a)) return fail(JXB_ERR_NONFINITE, "jxb_cnn_accumulate_energy: degenerate pair or output");
    value = weight * (1.0 - a * a / (bq * c));
    const double f = weight * 2.0 * a / (bq * c);
    // chain rule through z = s N: dL/dN = s dL/dz
    k_angle_grad<<<nb256(ncp * 4), 256, 0, s>>>(ncp, vec, Kd, r, plan->d_keep, f * (a / bq) * out_scale, f * out_scale,
                                                cnn_grad_out(cnn));
    JXB_CUDA(cudaGetLastError());
  }
  if ((rc = cnn_backward(cnn, s, nx, ny, nz, in))) return rc;
  JXB_CUDA(cudaStreamSynchronize(s));
  if (loss) *loss = value;
  return JXB_OK;
}
