// Poisson, linear elasticity and the Kirchhoff plate on truncated hierarchical
// (THB) spaces: a plan over padded elements.
//
// The reference evaluates a hierarchical space with the tensor code through its
// padded-element contract (src/jaxiga/space/function_space.py:23-38): element e
// carries n_local_max functions u_i (padding index n_scalar, zero extraction
// rows) with N_i = sum_a C_e[i][a] B_a, B_a the Bernstein polynomials of the
// element on [-1, 1]^dim, and R_i = w_i N_i / W. It forms element tangents
// K_e = sum_q w a0 dR^T dR (src/jaxiga/forms/library.py:54-65) and scatters
// them into CSR (src/jaxiga/methods/galerkin.py:122-148).
//
// Here K.u runs matrix-free per element, one warp per element (grid-stride,
// several warps per CTA):
//   c_a = sum_i C[i][a] w_i u_i          (the numerator's Bernstein coefficients)
//   g(q) = (sum_a B_a c_a, sum_a dB_a c_a)  at every Gauss point
//   f(q) = M_q g(q)                        (M_q: the metric a w L^T L, host-made)
//   r_a = sum_q B_a f_0 + dB_a . f_1..dim
//   y_e[i] = w_i sum_a C[i][a] r_a
// into a per-element buffer, and a combine sums, for every DOF, its element
// copies in a fixed order (a CSR list built at creation), so results are
// bitwise reproducible; the combine carries the CG's p.Ap partials. Both hook
// into launch_bricks / launch_combine, so jxb_apply, jxb_diag, jxb_load and the
// CG run on this plan unchanged.
#include <algorithm>
#include <vector>

#include "jxb_internal.cuh"

struct jxb_thb_data {
  int nlm = 0, nb = 0, nq = 0, nf = 0, vec = 1;
  long long* d_dofs = nullptr;   // (n_elem, nlm)
  double* d_ext = nullptr;       // (n_elem, nlm, nb)
  double* d_w = nullptr;         // (n_scalar + 1): weights, 0 at the padding index
  double* d_tab = nullptr;       // (dim + 1, nq, nb); the plate's (6, nq, nb)
  double* d_fac = nullptr;       // (n_elem, nq, nf)
  double* d_wq = nullptr;        // (n_elem, nq)
  double* d_yl = nullptr;        // (n_elem, nlm, vec) element outputs
  long long* d_sptr = nullptr;   // (n_dofs + 1)
  long long* d_sidx = nullptr;   // element slots grouped by DOF, ascending
};

namespace jxb {
namespace {

// One warp per element: a CTA of up to THB_THREADS runs blockDim / 32 elements
// side by side (grid-stride), each warp on its own slice of A.sg doubles of
// dynamic shared memory and synchronised by __syncwarp alone; lanes stride over
// the element's functions, Bernstein coefficients and points (mostly one pass).
constexpr int THB_THREADS = 128;

__device__ __forceinline__ long long thb_first() {
  return (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
}
__device__ __forceinline__ long long thb_stride() { return (long long)gridDim.x * (blockDim.x >> 5); }

struct ThbArgs {
  long long n_elem, n;  // n: scalar functions (the padding index)
  int nlm, nb, nq, nf, vec;
  int sg;  // dynamic shared memory per warp (doubles)
  double lam, mu;
  const long long* dofs;
  const double* ext;
  const double* w;
  const double* tab;
  const double* fac;
  const double* wq;
  const uint8_t* keep;
  double* yl;
};

// NC channels per point: the numerator's value and reference gradient (Poisson,
// NC = dim + 1) or, for the plate, value, gradient and second derivatives
// (11, 12, 22): NC = 6; the metric M_q is packed, nf = NC (NC + 1) / 2.
template <int NC>
__global__ void __launch_bounds__(THB_THREADS)
    k_thb_apply(ThbArgs A, const double* __restrict__ x, int masked, const CgState* st) {
  if (st && st->done) return;
  extern __shared__ double smem[];
  double* sm = smem + (threadIdx.x >> 5) * A.sg;  // this warp's slice
  double* loc = sm;             // [nlm]  w_i u_i
  double* cb = loc + A.nlm;     // [nb]   numerator coefficients, then the residual r_a
  double* fl = cb + A.nb;       // [NC][nq] fluxes
  const int tid = threadIdx.x & 31;
  for (long long e = thb_first(); e < A.n_elem; e += thb_stride()) {
    const long long* dofs = A.dofs + e * A.nlm;
    const double* C = A.ext + e * A.nlm * A.nb;
    for (int i = tid; i < A.nlm; i += 32) {
      const long long g = dofs[i];
      double v = 0.0;
      if (g < A.n && !(masked && !A.keep[g])) v = A.w[g] * x[g];
      loc[i] = v;
    }
    __syncwarp();
    for (int a = tid; a < A.nb; a += 32) {
      double s = 0.0;
      for (int i = 0; i < A.nlm; ++i) s += C[i * A.nb + a] * loc[i];
      cb[a] = s;
    }
    __syncwarp();
    for (int q = tid; q < A.nq; q += 32) {
      double g[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const double* T = A.tab + ((size_t)c * A.nq + q) * A.nb;
        double s = 0.0;
        for (int a = 0; a < A.nb; ++a) s += __ldg(T + a) * cb[a];
        g[c] = s;
      }
      const double* M = A.fac + (e * A.nq + q) * A.nf;
      double f[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) f[c] = 0.0;
      int k = 0;
#pragma unroll
      for (int r = 0; r < NC; ++r)
#pragma unroll
        for (int c = r; c < NC; ++c) {
          const double m = M[k++];
          f[r] += m * g[c];
          if (c != r) f[c] += m * g[r];
        }
#pragma unroll
      for (int c = 0; c < NC; ++c) fl[c * A.nq + q] = f[c];
    }
    __syncwarp();
    for (int a = tid; a < A.nb; a += 32) {
      double s = 0.0;
      for (int q = 0; q < A.nq; ++q)
#pragma unroll
        for (int c = 0; c < NC; ++c) s += __ldg(A.tab + ((size_t)c * A.nq + q) * A.nb + a) * fl[c * A.nq + q];
      cb[a] = s;  // every lane is past its reads of cb (the warp barrier above)
    }
    __syncwarp();
    for (int i = tid; i < A.nlm; i += 32) {
      const long long g = dofs[i];
      double s = 0.0;
      for (int a = 0; a < A.nb; ++a) s += C[i * A.nb + a] * cb[a];
      A.yl[e * A.nlm + i] = g < A.n ? A.w[g] * s : 0.0;
    }
    __syncwarp();
  }
}

// diag K_e: for function i, w_i^2 sum_q G_i(q)^T M_q G_i(q), G_i = the channels of N_i
template <int NC>
__global__ void __launch_bounds__(THB_THREADS) k_thb_diag(ThbArgs A) {
  for (long long e = thb_first(); e < A.n_elem; e += thb_stride()) {
    const long long* dofs = A.dofs + e * A.nlm;
    const double* C = A.ext + e * A.nlm * A.nb;
    for (int i = threadIdx.x & 31; i < A.nlm; i += 32) {
      const long long g = dofs[i];
      double d = 0.0;
      for (int q = 0; q < A.nq; ++q) {
        double G[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const double* T = A.tab + ((size_t)c * A.nq + q) * A.nb;
          double s = 0.0;
          for (int a = 0; a < A.nb; ++a) s += __ldg(T + a) * C[i * A.nb + a];
          G[c] = s;
        }
        const double* M = A.fac + (e * A.nq + q) * A.nf;
        int k = 0;
#pragma unroll
        for (int r = 0; r < NC; ++r)
#pragma unroll
          for (int c = r; c < NC; ++c) d += (c == r ? 1.0 : 2.0) * M[k++] * G[r] * G[c];
      }
      A.yl[e * A.nlm + i] = g < A.n ? A.w[g] * A.w[g] * d : 0.0;
    }
  }
}

// load: F_e[i][c] = w_i sum_a C[i][a] sum_q B_a(q) wq(q) f_c(q)
__global__ void __launch_bounds__(THB_THREADS) k_thb_load(ThbArgs A, const double* __restrict__ f_qp) {
  extern __shared__ double smem[];
  double* sm = smem + (threadIdx.x >> 5) * A.sg;  // this warp's slice
  double* fb = sm;  // [nb][vec]
  const int V = A.vec;
  for (long long e = thb_first(); e < A.n_elem; e += thb_stride()) {
    const long long* dofs = A.dofs + e * A.nlm;
    const double* C = A.ext + e * A.nlm * A.nb;
    for (int k = threadIdx.x & 31; k < A.nb * V; k += 32) {
      const int a = k / V, c = k - a * V;
      double s = 0.0;
      for (int q = 0; q < A.nq; ++q)
        s += __ldg(A.tab + (size_t)q * A.nb + a) * A.wq[e * A.nq + q] * f_qp[(e * A.nq + q) * V + c];
      fb[k] = s;
    }
    __syncwarp();
    for (int k = threadIdx.x & 31; k < A.nlm * V; k += 32) {
      const int i = k / V, c = k - i * V;
      const long long g = dofs[i];
      double s = 0.0;
      for (int a = 0; a < A.nb; ++a) s += C[i * A.nb + a] * fb[a * V + c];
      A.yl[e * A.nlm * V + k] = g < A.n ? A.w[g] * s : 0.0;
    }
    __syncwarp();
  }
}

// Isotropic elasticity at one point. g[c][0] = numerator value, g[c][1 + a] its
// reference gradient for component c; Fr (DIM^2 + 2 + DIM values) = J^-1 ([a][k]),
// w |J|, 1/W, grad W / W. Writes the flux channels f[c][0..DIM] of the test
// functions' (value, reference gradient), the quotient rule transposed.
template <int DIM>
__device__ __forceinline__ void thb_elastic_point(const double* __restrict__ Fr, double lam, double mu,
                                                  const double (&g)[DIM][DIM + 1], double (&f)[DIM][DIM + 1]) {
  double Ji[DIM][DIM];
#pragma unroll
  for (int a = 0; a < DIM; ++a)
#pragma unroll
    for (int k = 0; k < DIM; ++k) Ji[a][k] = Fr[a * DIM + k];
  const double om = Fr[DIM * DIM], iW = Fr[DIM * DIM + 1];
  const double* gW = Fr + DIM * DIM + 2;
  double Gx[DIM][DIM];  // du_c / dx_k
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    double gp[DIM];
#pragma unroll
    for (int a = 0; a < DIM; ++a) gp[a] = (g[c][1 + a] - g[c][0] * gW[a]) * iW;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
      double s = 0.0;
#pragma unroll
      for (int a = 0; a < DIM; ++a) s += Ji[a][k] * gp[a];
      Gx[c][k] = s;
    }
  }
  double tr = 0.0;
#pragma unroll
  for (int k = 0; k < DIM; ++k) tr += Gx[k][k];
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    double S[DIM];
#pragma unroll
    for (int k = 0; k < DIM; ++k) S[k] = om * (mu * (Gx[c][k] + Gx[k][c]) + (c == k ? lam * tr : 0.0));
    double fv = 0.0;
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      double Fa = 0.0;
#pragma unroll
      for (int k = 0; k < DIM; ++k) Fa += S[k] * Ji[a][k];
      f[c][1 + a] = Fa * iW;
      fv -= Fa * gW[a];
    }
    f[c][0] = fv * iW;
  }
}

template <int DIM>
__global__ void __launch_bounds__(THB_THREADS)
    k_thb_apply_el(ThbArgs A, const double* __restrict__ x, int masked, const CgState* st) {
  if (st && st->done) return;
  constexpr int NC = DIM + 1;
  extern __shared__ double smem[];
  double* sm = smem + (threadIdx.x >> 5) * A.sg;  // this warp's slice
  double* loc = sm;                // [nlm][DIM]  w_i u_ic
  double* cb = loc + A.nlm * DIM;  // [nb][DIM]   numerator coefficients, then the residual
  double* fl = cb + A.nb * DIM;    // [DIM][NC][nq] fluxes
  const int tid = threadIdx.x & 31;
  for (long long e = thb_first(); e < A.n_elem; e += thb_stride()) {
    const long long* dofs = A.dofs + e * A.nlm;
    const double* C = A.ext + e * A.nlm * A.nb;
    for (int k = tid; k < A.nlm * DIM; k += 32) {
      const int i = k / DIM, c = k - i * DIM;
      const long long g = dofs[i];
      double v = 0.0;
      if (g < A.n) {
        const long long d = g * DIM + c;
        if (!(masked && !A.keep[d])) v = A.w[g] * x[d];
      }
      loc[k] = v;
    }
    __syncwarp();
    for (int k = tid; k < A.nb * DIM; k += 32) {
      const int a = k / DIM, c = k - a * DIM;
      double s = 0.0;
      for (int i = 0; i < A.nlm; ++i) s += C[i * A.nb + a] * loc[i * DIM + c];
      cb[k] = s;
    }
    __syncwarp();
    for (int q = tid; q < A.nq; q += 32) {
      double g[DIM][NC];
#pragma unroll
      for (int c = 0; c < DIM; ++c)
#pragma unroll
        for (int ch = 0; ch < NC; ++ch) g[c][ch] = 0.0;
      for (int a = 0; a < A.nb; ++a) {
        double t[NC];
#pragma unroll
        for (int ch = 0; ch < NC; ++ch) t[ch] = __ldg(A.tab + ((size_t)ch * A.nq + q) * A.nb + a);
#pragma unroll
        for (int c = 0; c < DIM; ++c) {
          const double v = cb[a * DIM + c];
#pragma unroll
          for (int ch = 0; ch < NC; ++ch) g[c][ch] += t[ch] * v;
        }
      }
      double f[DIM][NC];
      thb_elastic_point<DIM>(A.fac + (e * A.nq + q) * A.nf, A.lam, A.mu, g, f);
#pragma unroll
      for (int c = 0; c < DIM; ++c)
#pragma unroll
        for (int ch = 0; ch < NC; ++ch) fl[(c * NC + ch) * A.nq + q] = f[c][ch];
    }
    __syncwarp();
    for (int k = tid; k < A.nb * DIM; k += 32) {
      const int a = k / DIM, c = k - a * DIM;
      double s = 0.0;
      for (int q = 0; q < A.nq; ++q)
#pragma unroll
        for (int ch = 0; ch < NC; ++ch) s += __ldg(A.tab + ((size_t)ch * A.nq + q) * A.nb + a) * fl[(c * NC + ch) * A.nq + q];
      cb[k] = s;  // every lane is past its reads of cb (the warp barrier above)
    }
    __syncwarp();
    for (int k = tid; k < A.nlm * DIM; k += 32) {
      const int i = k / DIM, c = k - i * DIM;
      const long long g = dofs[i];
      double s = 0.0;
      for (int a = 0; a < A.nb; ++a) s += C[i * A.nb + a] * cb[a * DIM + c];
      A.yl[e * A.nlm * DIM + k] = g < A.n ? A.w[g] * s : 0.0;
    }
    __syncwarp();
  }
}

// diag K_e for elasticity: w_i^2 sum_q w |J| ((lam + mu) gx_c^2 + mu |gx|^2), gx the
// physical gradient of R_i / w_i with the quotient rule
template <int DIM>
__global__ void __launch_bounds__(THB_THREADS) k_thb_diag_el(ThbArgs A) {
  for (long long e = thb_first(); e < A.n_elem; e += thb_stride()) {
    const long long* dofs = A.dofs + e * A.nlm;
    const double* C = A.ext + e * A.nlm * A.nb;
    for (int i = threadIdx.x & 31; i < A.nlm; i += 32) {
      const long long g = dofs[i];
      double d[DIM];
#pragma unroll
      for (int c = 0; c < DIM; ++c) d[c] = 0.0;
      for (int q = 0; q < A.nq; ++q) {
        double G[DIM + 1];
#pragma unroll
        for (int ch = 0; ch <= DIM; ++ch) {
          const double* T = A.tab + ((size_t)ch * A.nq + q) * A.nb;
          double s = 0.0;
          for (int a = 0; a < A.nb; ++a) s += __ldg(T + a) * C[i * A.nb + a];
          G[ch] = s;
        }
        const double* Fr = A.fac + (e * A.nq + q) * A.nf;
        const double om = Fr[DIM * DIM], iW = Fr[DIM * DIM + 1];
        double gx[DIM], n2 = 0.0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
          double s = 0.0;
#pragma unroll
          for (int a = 0; a < DIM; ++a) s += Fr[a * DIM + k] * (G[1 + a] - G[0] * Fr[DIM * DIM + 2 + a]) * iW;
          gx[k] = s;
          n2 += s * s;
        }
#pragma unroll
        for (int c = 0; c < DIM; ++c) d[c] += om * ((A.lam + A.mu) * gx[c] * gx[c] + A.mu * n2);
      }
#pragma unroll
      for (int c = 0; c < DIM; ++c) A.yl[(e * A.nlm + i) * DIM + c] = g < A.n ? A.w[g] * A.w[g] * d[c] : 0.0;
    }
  }
}

// y_g = sum of DOF g's element copies in ascending slot order; optional p.y partials
__global__ void __launch_bounds__(JXB_RED_THREADS)
    k_thb_combine(const CgState* st, long long n, const long long* __restrict__ sptr,
                  const long long* __restrict__ sidx, const double* __restrict__ yl, const uint8_t* __restrict__ keep,
                  int masked, double* __restrict__ y, const double* __restrict__ dot_with,
                  double* __restrict__ partials) {
  if (st && st->done) return;
  double part = 0.0;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (long long k = sptr[g]; k < sptr[g + 1]; ++k) s += yl[sidx[k]];
    if (masked && !keep[g]) s = 0.0;
    y[g] = s;
    if (dot_with) part += dot_with[g] * s;
  }
  if (partials) {
    __shared__ double warp_part[JXB_RED_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0) warp_part[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int i = 0; i < JXB_RED_THREADS / 32; ++i) t += warp_part[i];
      partials[blockIdx.x] = t;
    }
  }
}

}  // namespace

static ThbArgs thb_args(jxb_plan* plan) {
  jxb_thb_data* T = plan->thb;
  ThbArgs A;
  A.n_elem = plan->n_elem;
  A.n = plan->n_scalar;
  A.nlm = T->nlm;
  A.nb = T->nb;
  A.nq = T->nq;
  A.nf = T->nf;
  A.vec = T->vec;
  A.sg = 0;
  A.lam = plan->mat.lam;
  A.mu = plan->mat.mu;
  A.dofs = T->d_dofs;
  A.ext = T->d_ext;
  A.w = T->d_w;
  A.tab = T->d_tab;
  A.fac = T->d_fac;
  A.wq = T->d_wq;
  A.keep = plan->d_keep;
  A.yl = T->d_yl;
  return A;
}

static unsigned thb_grid(long long n_elem) { return (unsigned)std::max(1LL, std::min(n_elem, 148LL * 16)); }

int thb_bricks(jxb_plan* plan, cudaStream_t s, int mode, const double* x, const double* f_qp, const CgState* state,
               int masked) {
  jxb_thb_data* T = plan->thb;
  ThbArgs A = thb_args(plan);
  const bool el = plan->op == JXB_OP_ELASTICITY;
  const int V = T->vec, NC = plan->op == JXB_OP_PLATE ? 6 : plan->dim + 1;
  // per-warp shared memory; as many warps (elements) per CTA as 48 KB holds, at most 4
  A.sg = mode == MODE_APPLY ? (T->nlm + T->nb) * V + V * NC * T->nq : mode == MODE_LOAD ? T->nb * V : 0;
  const size_t sg_bytes = (size_t)A.sg * sizeof(double);
  if (sg_bytes > 48 * 1024) return fail(JXB_ERR_INVALID, "hierarchical plan: element too large for shared memory");
  const int warps = sg_bytes ? (int)std::min<size_t>(THB_THREADS / 32, (48 * 1024) / sg_bytes) : THB_THREADS / 32;
  const unsigned threads = 32u * (unsigned)warps;
  const unsigned grid = thb_grid((plan->n_elem + warps - 1) / warps);
  const size_t sm = sg_bytes * warps;
  if (mode == MODE_APPLY) {
    if (el) {
      if (plan->dim == 2)
        k_thb_apply_el<2><<<grid, threads, sm, s>>>(A, x, masked, state);
      else
        k_thb_apply_el<3><<<grid, threads, sm, s>>>(A, x, masked, state);
    } else if (NC == 3) {
      k_thb_apply<3><<<grid, threads, sm, s>>>(A, x, masked, state);
    } else if (NC == 4) {
      k_thb_apply<4><<<grid, threads, sm, s>>>(A, x, masked, state);
    } else {
      k_thb_apply<6><<<grid, threads, sm, s>>>(A, x, masked, state);
    }
  } else if (mode == MODE_DIAG) {
    if (el) {
      if (plan->dim == 2)
        k_thb_diag_el<2><<<grid, threads, 0, s>>>(A);
      else
        k_thb_diag_el<3><<<grid, threads, 0, s>>>(A);
    } else if (NC == 3) {
      k_thb_diag<3><<<grid, threads, 0, s>>>(A);
    } else if (NC == 4) {
      k_thb_diag<4><<<grid, threads, 0, s>>>(A);
    } else {
      k_thb_diag<6><<<grid, threads, 0, s>>>(A);
    }
  } else if (mode == MODE_LOAD) {
    if (!f_qp) return fail(JXB_ERR_INVALID, "jxb_load: null f_qp");
    k_thb_load<<<grid, threads, sm, s>>>(A, f_qp);
  } else {
    return fail(JXB_ERR_INVALID, "hierarchical plans apply, load and give the diagonal only");
  }
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

int thb_combine(jxb_plan* plan, cudaStream_t s, double* y, int masked, const double* dot_with, double* partials,
                const CgState* state) {
  jxb_thb_data* T = plan->thb;
  k_thb_combine<<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(state, plan->n_dofs, T->d_sptr, T->d_sidx, T->d_yl,
                                                           plan->d_keep, masked, y, dot_with, partials);
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

void free_thb(jxb_plan* plan) {
  jxb_thb_data* T = plan ? plan->thb : nullptr;
  if (!T) return;
  void* bufs[] = {T->d_dofs, T->d_ext, T->d_w, T->d_tab, T->d_fac, T->d_wq, T->d_yl, T->d_sptr, T->d_sidx};
  for (void* b : bufs) cudaFree(b);
  delete T;
  plan->thb = nullptr;
}

}  // namespace jxb

using namespace jxb;

extern "C" int jxb_thb_create(const jxb_thb_desc* d, jxb_plan** out) {
  if (!d || !out) return fail(JXB_ERR_INVALID, "jxb_thb_create: null argument");
  *out = nullptr;
  if ((d->dim != 2 && d->dim != 3) || d->degree < 1 || d->degree > 4)
    return fail(JXB_ERR_INVALID, "jxb_thb_create: dimension 2 or 3 and degree 1..4 are supported");
  if (d->n_elem < 1 || d->n_scalar < 1 || d->n_local_max < 1 || !d->elem_dofs || !d->extraction || !d->wgts ||
      !d->tables || !d->factors || !d->wq)
    return fail(JXB_ERR_INVALID, "jxb_thb_create: bad sizes or null arrays");
  if (d->op != JXB_OP_POISSON && d->op != JXB_OP_ELASTICITY && !(d->op == JXB_OP_PLATE && d->dim == 2))
    return fail(JXB_ERR_INVALID,
                "jxb_thb_create: the Poisson, linear elasticity and (2D) Kirchhoff plate operators are supported");
  int nb = 1;
  for (int k = 0; k < d->dim; ++k) nb *= d->degree + 1;
  const bool el = d->op == JXB_OP_ELASTICITY, pl = d->op == JXB_OP_PLATE;
  const int V = el ? d->dim : 1;
  const int nq = nb, nlm = d->n_local_max;
  const int ntab = pl ? 6 : d->dim + 1;  // point tables: value, gradient (and second derivatives)
  const int nf = el ? d->dim * d->dim + 2 + d->dim : ntab * (ntab + 1) / 2;
  const long long ne = d->n_elem, n = d->n_scalar, nd = n * V;
  // the DOF -> element-slot lists, ascending slot order (the fixed summation
  // order); slot (e * nlm + i) * V + c holds component c of local function i
  std::vector<long long> count(nd + 1, 0);
  for (long long k = 0; k < ne * nlm; ++k) {
    const long long g = d->elem_dofs[k];
    if (g < 0 || g > n) return fail(JXB_ERR_INVALID, "jxb_thb_create: elem_dofs entry out of range");
    if (g < n)
      for (int c = 0; c < V; ++c) ++count[g * V + c + 1];
  }
  for (long long g = 0; g < nd; ++g) count[g + 1] += count[g];
  std::vector<long long> sidx(std::max<long long>(count[nd], 1)), fill(count.begin(), count.end() - 1);
  for (long long k = 0; k < ne * nlm; ++k) {
    const long long g = d->elem_dofs[k];
    if (g < n)
      for (int c = 0; c < V; ++c) sidx[fill[g * V + c]++] = k * V + c;
  }
  std::vector<double> w(n + 1, 0.0);
  for (long long g = 0; g < n; ++g) w[g] = d->wgts[g];
  std::vector<uint8_t> keep(nd, 1);
  long long nfree = nd;
  if (d->prescribed)
    for (long long g = 0; g < nd; ++g)
      if (d->prescribed[g]) {
        keep[g] = 0;
        --nfree;
      }
  int device = 0;
  JXB_CUDA(cudaGetDevice(&device));
  jxb_plan* P = new jxb_plan();
  P->thb = new jxb_thb_data();
  jxb_thb_data* T = P->thb;
  T->nlm = nlm;
  T->nb = nb;
  T->nq = nq;
  T->nf = nf;
  T->vec = V;
  P->device = device;
  P->dim = d->dim;
  P->vec = V;
  P->p = d->degree;
  P->q = d->degree + 1;
  P->op = d->op;
  P->order = pl ? 2 : 1;
  P->nqe = nq;
  P->ngeo = nf;
  P->n_elem = ne;
  P->n_qp = ne * nq;
  P->n_scalar = n;
  P->n_dofs = nd;
  P->n_free = nfree;
  P->mat.lam = el ? d->lam : 0.0;
  P->mat.mu = el ? d->mu : 0.0;
  cudaError_t e = cudaSuccess;
  auto al = [&](void** p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, std::max<size_t>(bytes, 8));
  };
  auto up = [&](void* dst, const void* src, size_t bytes) {
    if (e == cudaSuccess && bytes) e = cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
  };
  al((void**)&T->d_dofs, ne * nlm * sizeof(long long));
  al((void**)&T->d_ext, (size_t)ne * nlm * nb * sizeof(double));
  al((void**)&T->d_w, (n + 1) * sizeof(double));
  al((void**)&T->d_tab, (size_t)ntab * nq * nb * sizeof(double));
  al((void**)&T->d_fac, (size_t)ne * nq * nf * sizeof(double));
  al((void**)&T->d_wq, (size_t)ne * nq * sizeof(double));
  al((void**)&T->d_yl, (size_t)ne * nlm * V * sizeof(double));
  al((void**)&T->d_sptr, (nd + 1) * sizeof(long long));
  al((void**)&T->d_sidx, sidx.size() * sizeof(long long));
  al((void**)&P->d_keep, nd);
  al((void**)&P->d_red, (4 * JXB_RED_BLOCKS + 16) * sizeof(double));
  static_assert(sizeof(long long) == sizeof(int64_t), "int64 DOF indices");
  up(T->d_dofs, d->elem_dofs, ne * nlm * sizeof(long long));
  up(T->d_ext, d->extraction, (size_t)ne * nlm * nb * sizeof(double));
  up(T->d_w, w.data(), (n + 1) * sizeof(double));
  up(T->d_tab, d->tables, (size_t)ntab * nq * nb * sizeof(double));
  up(T->d_fac, d->factors, (size_t)ne * nq * nf * sizeof(double));
  up(T->d_wq, d->wq, (size_t)ne * nq * sizeof(double));
  up(T->d_sptr, count.data(), (nd + 1) * sizeof(long long));
  up(T->d_sidx, sidx.data(), sidx.size() * sizeof(long long));
  up(P->d_keep, keep.data(), nd);
  if (e == cudaSuccess) e = cudaMemset(P->d_red, 0, (4 * JXB_RED_BLOCKS + 16) * sizeof(double));
  if (e != cudaSuccess) {
    free_thb(P);
    cudaFree(P->d_keep);
    cudaFree(P->d_red);
    delete P;
    return cuda_fail(e, "jxb_thb_create");
  }
  *out = P;
  return JXB_OK;
}
