// Basis tables and per-quadrature-point geometry factors (FP64).
//
// 1. k_tables: for every direction, span and Gauss node, the extracted 1D
//    B-spline values N = C . B, first and second derivatives (scaled by 2/h,
//    (2/h)^2 to patch-parameter units), i.e. the per-direction factors of
//    src/jaxiga/space/evaluation.py:374-386 (N = C.B, dN = C.dB * 2/h).
// 2. k_factors: one thread per (element slot, quadrature point). It sums the
//    tensor-product basis against weights and control points, applies the
//    NURBS quotient rule (evaluation.py:95-137), forms the Jacobian, its
//    determinant and inverse (evaluation.py:141-152), the weight
//    w = w_hat |J| prod(h/2) (evaluation.py:461-463) and stores the factors
//    the apply kernels contract against:
//      Poisson    sym(d) or sym(d+1) metric  a w J^-1 J^-T  (library.py:54-65)
//      elasticity J^-1 and w (+ 1/W, grad W / W when rational) (library.py:174-181)
//      plate      sym(5|6) metric  w L^T D L with L the curvature map
//                 of the Hessian push-forward (evaluation.py:154-170,
//                 library.py:108-132)
#include <math.h>

#include <vector>

#include "jxb_internal.cuh"

#define JXB_GRAD_MAXC 3

namespace jxb {

// Bernstein recurrence of src/jaxiga/space/bernstein.py:79-156 at one point.
__device__ void bernstein_point(double xi, int deg, double* B, double* dB, double* d2B) {
  double u1 = 1.0 - xi, u2 = 1.0 + xi;
  double scale = 1.0;
  for (int i = 0; i < deg; ++i) scale *= 2.0;
  double t[JXB_MAXP + 1];
  // values
  for (int k = 0; k <= deg; ++k) t[k] = 0.0;
  t[0] = 1.0;
  for (int j = 1; j <= deg; ++j) {
    double saved = 0.0;
    for (int k = 0; k < j; ++k) {
      double temp = t[k];
      t[k] = saved + u1 * temp;
      saved = u2 * temp;
    }
    t[j] = saved;
  }
  for (int k = 0; k <= deg; ++k) B[k] = t[k] / scale;
  // first derivative: p * (B^{p-1}_{k-1} - B^{p-1}_k), lower degree scaled by 1/2^p
  for (int k = 0; k <= deg; ++k) dB[k] = 0.0;
  if (deg >= 1) {
    double l[JXB_MAXP + 2];
    for (int k = 0; k < deg; ++k) l[k] = 0.0;
    l[0] = 1.0;
    for (int j = 1; j < deg; ++j) {
      double saved = 0.0;
      for (int k = 0; k < j; ++k) {
        double temp = l[k];
        l[k] = saved + u1 * temp;
        saved = u2 * temp;
      }
      l[j] = saved;
    }
    for (int k = 0; k < deg; ++k) l[k] /= scale;
    for (int k = 0; k <= deg; ++k) {
      double left = (k >= 1) ? l[k - 1] : 0.0;
      double right = (k < deg) ? l[k] : 0.0;
      dB[k] = (left - right) * deg;
    }
  }
  for (int k = 0; k <= deg; ++k) d2B[k] = 0.0;
  if (deg >= 2) {
    double l[JXB_MAXP + 2], m[JXB_MAXP + 2];
    for (int k = 0; k < deg - 1; ++k) l[k] = 0.0;
    l[0] = 1.0;
    for (int j = 1; j < deg - 1; ++j) {
      double saved = 0.0;
      for (int k = 0; k < j; ++k) {
        double temp = l[k];
        l[k] = saved + u1 * temp;
        saved = u2 * temp;
      }
      l[j] = saved;
    }
    for (int k = 0; k < deg - 1; ++k) l[k] /= scale;
    for (int k = 0; k < deg; ++k) {  // first difference, degree-1 rows
      double left = (k >= 1) ? l[k - 1] : 0.0;
      double right = (k < deg - 1) ? l[k] : 0.0;
      m[k] = (left - right) * (deg - 1);
    }
    for (int k = 0; k <= deg; ++k) {
      double left = (k >= 1) ? m[k - 1] : 0.0;
      double right = (k < deg) ? m[k] : 0.0;
      d2B[k] = (left - right) * deg;
    }
  }
}

// tab[((span*3 + kind)*Q + qi)*(P+1) + a] = sum_j {B,dB,d2B}_j(xi_q) C[span][a][j] * (2/h)^kind
__global__ void k_tables(int p, int Q, int n_span, const double* __restrict__ ext,
                         const double* __restrict__ lo, const double* __restrict__ hi,
                         const double* __restrict__ nodes, double* __restrict__ tab,
                         float* __restrict__ tab32) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  int P1 = p + 1;
  int total = n_span * Q * P1;
  if (idx >= total) return;
  int a = idx % P1;
  int qi = (idx / P1) % Q;
  int s = idx / (P1 * Q);
  double B[JXB_MAXP + 1], dB[JXB_MAXP + 1], d2B[JXB_MAXP + 1];
  bernstein_point(nodes[qi], p, B, dB, d2B);
  const double* C = ext + (size_t)s * P1 * P1 + (size_t)a * P1;
  double v = 0.0, d = 0.0, h = 0.0;
  for (int j = 0; j < P1; ++j) {
    v += C[j] * B[j];
    d += C[j] * dB[j];
    h += C[j] * d2B[j];
  }
  double sc = 2.0 / (hi[s] - lo[s]);
  double out[3] = {v, d * sc, h * sc * sc};
  for (int k = 0; k < 3; ++k) {
    size_t o = (((size_t)s * 3 + k) * Q + qi) * P1 + a;
    tab[o] = out[k];
    if (tab32) tab32[o] = (float)out[k];
  }
}

struct FactorArgs {
  Bricks br;
  const double* tab[3];
  const double* span_lo[3];
  const double* span_hi[3];
  const double* cpts;
  const double* wgts;
  const double* gw;        // Gauss weights (Q)
  const double* coef_qp;   // optional per-point a0, reference order
  double coef[4];
  int op, rational, ngeo;
  double* geo;
  double* wq;
  double* invW;
};

__device__ __forceinline__ void elem_of_slot(const Bricks& br, long long slot, int& ex, int& ey,
                                             int& ez, bool& valid) {
  long long E = (long long)br.te[0] * br.te[1] * br.te[2];
  long long b = slot / E;
  int el = (int)(slot % E);
  int exl = el % br.te[0];
  int eyl = (el / br.te[0]) % br.te[1];
  int ezl = el / (br.te[0] * br.te[1]);
  int bx = (int)(b % br.nb[0]);
  int by = (int)((b / br.nb[0]) % br.nb[1]);
  int bz = (int)(b / ((long long)br.nb[0] * br.nb[1]));
  ex = bx * br.te[0] + exl;
  ey = by * br.te[1] + eyl;
  ez = bz * br.te[2] + ezl;
  valid = ex < br.n_span[0] && ey < br.n_span[1] && (br.dim == 2 ? ez == 0 : ez < br.n_span[2]);
}

// Sums of the weighted tensor basis over one element at one point:
// W and its derivatives, and the homogeneous coordinates P_i = sum w X_i N.
struct PointSums {
  double W, Wd[3], Wh[6];
  double P[3], Pd[3][3], Ph[3][6];
};

__device__ void point_sums(const FactorArgs& A, int ex, int ey, int ez, int q0, int q1, int q2,
                           int order, PointSums& S) {
  const Bricks& br = A.br;
  int dim = br.dim, P1 = br.p + 1, Q = br.q;
  const double* nv[3];
  const double* nd[3];
  const double* nh[3];
  int span[3] = {ex, ey, ez};
  int qq[3] = {q0, q1, q2};
  for (int d = 0; d < dim; ++d) {
    const double* base = A.tab[d] + ((size_t)span[d] * 3) * Q * P1;
    nv[d] = base + (size_t)qq[d] * P1;
    nd[d] = base + (size_t)(Q + qq[d]) * P1;
    nh[d] = base + (size_t)(2 * Q + qq[d]) * P1;
  }
  S.W = 0;
  for (int i = 0; i < 3; ++i) {
    S.Wd[i] = 0;
    S.P[i] = 0;
    for (int j = 0; j < 3; ++j) S.Pd[i][j] = 0;
    for (int j = 0; j < 6; ++j) S.Ph[i][j] = 0;
  }
  for (int j = 0; j < 6; ++j) S.Wh[j] = 0;
  int f0 = br.first[0][ex], f1 = br.first[1][ey], f2 = dim == 3 ? br.first[2][ez] : 0;
  int n2 = dim == 3 ? P1 : 1;
  for (int a2 = 0; a2 < n2; ++a2)
    for (int a1 = 0; a1 < P1; ++a1)
      for (int a0 = 0; a0 < P1; ++a0) {
        long long cp = (long long)(f0 + a0) +
                       (long long)br.n_cp[0] * ((f1 + a1) + (long long)br.n_cp[1] * (f2 + a2));
        double w = A.wgts[cp];
        double N, dN[3] = {0, 0, 0}, hN[6] = {0, 0, 0, 0, 0, 0};
        if (dim == 2) {
          N = nv[0][a0] * nv[1][a1];
          dN[0] = nd[0][a0] * nv[1][a1];
          dN[1] = nv[0][a0] * nd[1][a1];
          if (order >= 2) {
            hN[0] = nh[0][a0] * nv[1][a1];
            hN[1] = nd[0][a0] * nd[1][a1];
            hN[2] = nv[0][a0] * nh[1][a1];
          }
        } else {
          N = nv[0][a0] * nv[1][a1] * nv[2][a2];
          dN[0] = nd[0][a0] * nv[1][a1] * nv[2][a2];
          dN[1] = nv[0][a0] * nd[1][a1] * nv[2][a2];
          dN[2] = nv[0][a0] * nv[1][a1] * nd[2][a2];
        }
        S.W += w * N;
        for (int k = 0; k < dim; ++k) S.Wd[k] += w * dN[k];
        for (int k = 0; k < 3; ++k) S.Wh[k] += w * hN[k];
        for (int i = 0; i < dim; ++i) {
          double wx = w * A.cpts[cp * dim + i];
          S.P[i] += wx * N;
          for (int k = 0; k < dim; ++k) S.Pd[i][k] += wx * dN[k];
          for (int k = 0; k < 3; ++k) S.Ph[i][k] += wx * hN[k];
        }
      }
}

__device__ double det_inv(int dim, const double J[3][3], double Ji[3][3]) {
  if (dim == 2) {
    double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    double id = 1.0 / det;
    Ji[0][0] = J[1][1] * id;
    Ji[0][1] = -J[0][1] * id;
    Ji[1][0] = -J[1][0] * id;
    Ji[1][1] = J[0][0] * id;
    return det;
  }
  double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
  double id = 1.0 / det;
  Ji[0][0] = c00 * id;
  Ji[1][0] = c01 * id;
  Ji[2][0] = c02 * id;
  Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
  Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
  Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
  return det;
}

// Pack a symmetric n x n matrix, upper triangle row by row.
__device__ __forceinline__ void store_sym(double* geo, size_t stride, int n, const double M[6][6],
                                          int off) {
  int k = 0;
  for (int a = 0; a < n; ++a)
    for (int b = a; b < n; ++b) geo[stride * (k++)] = M[a + off][b + off];
}

__global__ void k_factors(FactorArgs A) {
  const Bricks& br = A.br;
  int dim = br.dim, Q = br.q;
  long long nqe = dim == 2 ? Q * Q : Q * Q * Q;
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= br.slots * nqe) return;
  long long slot = idx / nqe;
  int q = (int)(idx % nqe);
  int q0 = q % Q, q1 = (q / Q) % Q, q2 = dim == 3 ? q / (Q * Q) : 0;
  const GeoAt ga = geo_at(dim, slot, q, Q, A.ngeo, nqe, br.te[0]);
  double* g = A.geo + ga.base;
  const size_t gs = ga.stride;
  int ex, ey, ez;
  bool valid;
  elem_of_slot(br, slot, ex, ey, ez, valid);
  if (!valid) {
    for (int k = 0; k < A.ngeo; ++k) g[k * gs] = 0.0;
    A.wq[slot * nqe + q] = 0.0;
    if (A.invW) A.invW[slot * nqe + q] = 0.0;
    return;
  }
  int order = A.op == JXB_OP_PLATE ? 2 : 1;
  PointSums S;
  point_sums(A, ex, ey, ez, q0, q1, q2, order, S);
  double W = S.W, iW = 1.0 / W;
  double x[3], xd[3][3], J[3][3], Ji[3][3];
  for (int i = 0; i < dim; ++i) {
    x[i] = S.P[i] * iW;
    for (int a = 0; a < dim; ++a) {
      xd[i][a] = (S.Pd[i][a] - x[i] * S.Wd[a]) * iW;
      J[a][i] = xd[i][a];  // dxdxi[a][i] = d x_i / d xi_a
    }
  }
  double det = det_inv(dim, J, Ji);  // Ji[k][a] = (dxdxi^-1)[k][a]
  int sp[3] = {ex, ey, ez};
  double jac = 1.0, wh = 1.0;
  int qq[3] = {q0, q1, q2};
  for (int d = 0; d < dim; ++d) {
    jac *= (A.span_hi[d][sp[d]] - A.span_lo[d][sp[d]]) / 2.0;
    wh *= A.gw[qq[d]];
  }
  double om = wh * fabs(det) * jac;
  A.wq[slot * nqe + q] = om * iW;
  if (A.invW) A.invW[slot * nqe + q] = iW;

  if (A.op == JXB_OP_POISSON) {
    double a0 = A.coef[0];
    if (A.coef_qp) {
      long long eref = ex + (long long)br.n_span[0] * (ey + (long long)br.n_span[1] * ez);
      a0 = A.coef_qp[eref * nqe + q];
    }
    // rows of the parametric gradient of u in terms of channels (v, dv/dxi_a):
    // u_a = (v_a - v W_a / W) / W
    int nc = A.rational ? dim + 1 : dim, off = A.rational ? 0 : 1;
    double Lg[3][4];
    for (int k = 0; k < dim; ++k) {
      for (int c = 0; c < 4; ++c) Lg[k][c] = 0;
      for (int a = 0; a < dim; ++a) {
        // physical row k: sum_a Ji[k][a] * row(u_a)
        Lg[k][0] += Ji[k][a] * (-S.Wd[a] * iW * iW);
        Lg[k][1 + a] += Ji[k][a] * iW;
      }
    }
    double M[6][6];
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 4; ++c) {
        double s = 0;
        for (int k = 0; k < dim; ++k) s += Lg[k][r] * Lg[k][c];
        M[r][c] = a0 * om * s;
      }
    store_sym(g, gs, nc, M, off);
  } else if (A.op == JXB_OP_ELASTICITY || A.op == JXB_OP_HYPERELASTIC) {
    int k = 0;
    for (int i = 0; i < dim; ++i)
      for (int a = 0; a < dim; ++a) g[gs * (k++)] = Ji[i][a];
    g[gs * (k++)] = om;
    if (A.rational) {
      g[gs * (k++)] = iW;
      for (int a = 0; a < dim; ++a) g[gs * (k++)] = S.Wd[a] * iW;
    }
    if (A.op == JXB_OP_HYPERELASTIC) {  // the state of u = 0: F^-T = I, mu - lambda ln J = mu, no flux
      for (int i = 0; i < dim; ++i)
        for (int a = 0; a < dim; ++a) g[gs * (k++)] = i == a ? 1.0 : 0.0;
      g[gs * (k++)] = A.coef[0];
      for (int i = 0; i < dim * dim; ++i) g[gs * (k++)] = 0.0;
    }
  } else {  // plate (2D): channels (v, v0, v1, v00, v01, v11)
    double E = A.coef[0], nu = A.coef[1], t = A.coef[2];
    double Dfac = E * t * t * t / (12.0 * (1.0 - nu * nu));
    double D[3][3] = {{Dfac, Dfac * nu, 0}, {Dfac * nu, Dfac, 0}, {0, 0, Dfac * (1.0 - nu) / 2.0}};
    double ru[6] = {iW, 0, 0, 0, 0, 0};
    double rd[2][6], rh[3][6];
    for (int a = 0; a < 2; ++a)
      for (int c = 0; c < 6; ++c) rd[a][c] = ((c == 1 + a ? 1.0 : 0.0) - S.Wd[a] * ru[c]) * iW;
    const int pa[3] = {0, 0, 1}, pb[3] = {0, 1, 1};
    for (int kk = 0; kk < 3; ++kk) {
      int a = pa[kk], b = pb[kk];
      for (int c = 0; c < 6; ++c)
        rh[kk][c] = ((c == 3 + kk ? 1.0 : 0.0) - S.Wd[b] * rd[a][c] - S.Wd[a] * rd[b][c] -
                     S.Wh[kk] * ru[c]) *
                    iW;
    }
    // physical gradient rows and second derivatives of the geometry map
    double gx[2][6];
    for (int i = 0; i < 2; ++i)
      for (int c = 0; c < 6; ++c) gx[i][c] = Ji[i][0] * rd[0][c] + Ji[i][1] * rd[1][c];
    double xh[3][2];  // d2 x_i / dxi_a dxi_b
    for (int i = 0; i < 2; ++i)
      for (int kk = 0; kk < 3; ++kk) {
        int a = pa[kk], b = pb[kk];
        xh[kk][i] = (S.Ph[i][kk] - xd[i][a] * S.Wd[b] - xd[i][b] * S.Wd[a] - x[i] * S.Wh[kk]) * iW;
      }
    // T[(a,b),(i,j)] = J[a][i] J[b][j] + (J[a][j] J[b][i] if i != j)
    double T[3][3];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        int a = pa[r], b = pb[r], i = pa[c], j = pb[c];
        T[r][c] = J[a][i] * J[b][j] + (i != j ? J[a][j] * J[b][i] : 0.0);
      }
    double Ti[3][3];
    {
      double c00 = T[1][1] * T[2][2] - T[1][2] * T[2][1];
      double c01 = T[1][2] * T[2][0] - T[1][0] * T[2][2];
      double c02 = T[1][0] * T[2][1] - T[1][1] * T[2][0];
      double dT = T[0][0] * c00 + T[0][1] * c01 + T[0][2] * c02;
      double id = 1.0 / dT;
      Ti[0][0] = c00 * id;
      Ti[1][0] = c01 * id;
      Ti[2][0] = c02 * id;
      Ti[0][1] = (T[0][2] * T[2][1] - T[0][1] * T[2][2]) * id;
      Ti[1][1] = (T[0][0] * T[2][2] - T[0][2] * T[2][0]) * id;
      Ti[2][1] = (T[0][1] * T[2][0] - T[0][0] * T[2][1]) * id;
      Ti[0][2] = (T[0][1] * T[1][2] - T[0][2] * T[1][1]) * id;
      Ti[1][2] = (T[0][2] * T[1][0] - T[0][0] * T[1][2]) * id;
      Ti[2][2] = (T[0][0] * T[1][1] - T[0][1] * T[1][0]) * id;
    }
    double rhs[3][6], Hx[3][6], L[3][6];
    for (int kk = 0; kk < 3; ++kk)
      for (int c = 0; c < 6; ++c) rhs[kk][c] = rh[kk][c] - xh[kk][0] * gx[0][c] - xh[kk][1] * gx[1][c];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 6; ++c) Hx[r][c] = Ti[r][0] * rhs[0][c] + Ti[r][1] * rhs[1][c] + Ti[r][2] * rhs[2][c];
    for (int c = 0; c < 6; ++c) {  // kappa = -(H_xx, H_yy, 2 H_xy)
      L[0][c] = -Hx[0][c];
      L[1][c] = -Hx[2][c];
      L[2][c] = -2.0 * Hx[1][c];
    }
    double M[6][6];
    for (int r = 0; r < 6; ++r)
      for (int c = 0; c < 6; ++c) {
        double s = 0;
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) s += L[i][r] * D[i][j] * L[j][c];
        M[r][c] = om * s;
      }
    store_sym(g, gs, A.rational ? 6 : 5, M, A.rational ? 0 : 1);
  }
}

// Physical coordinates at the Gauss points, reference element order.
__global__ void k_coords(FactorArgs A, double* out) {
  const Bricks& br = A.br;
  int dim = br.dim, Q = br.q;
  long long nqe = dim == 2 ? Q * Q : Q * Q * Q;
  long long n_elem = (long long)br.n_span[0] * br.n_span[1] * (dim == 3 ? br.n_span[2] : 1);
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n_elem * nqe) return;
  long long e = idx / nqe;
  int q = (int)(idx % nqe);
  int ex = (int)(e % br.n_span[0]);
  int ey = (int)((e / br.n_span[0]) % br.n_span[1]);
  int ez = (int)(e / ((long long)br.n_span[0] * br.n_span[1]));
  PointSums S;
  point_sums(A, ex, ey, ez, q % Q, (q / Q) % Q, dim == 3 ? q / (Q * Q) : 0, 1, S);
  for (int i = 0; i < dim; ++i) out[idx * dim + i] = S.P[i] / S.W;
}

// sum_a R_a c_a at the Gauss points, reference order; R_a = w_a N_a / W.
__global__ void k_interp(FactorArgs A, const double* __restrict__ coef, int ncomp, double* out) {
  const Bricks& br = A.br;
  int dim = br.dim, Q = br.q, P1 = br.p + 1;
  long long nqe = dim == 2 ? Q * Q : Q * Q * Q;
  long long n_elem = (long long)br.n_span[0] * br.n_span[1] * (dim == 3 ? br.n_span[2] : 1);
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n_elem * nqe) return;
  long long e = idx / nqe;
  int q = (int)(idx % nqe);
  int sp[3] = {(int)(e % br.n_span[0]), (int)((e / br.n_span[0]) % br.n_span[1]),
               (int)(e / ((long long)br.n_span[0] * br.n_span[1]))};
  int qq[3] = {q % Q, (q / Q) % Q, dim == 3 ? q / (Q * Q) : 0};
  const double* nv[3];
  for (int d = 0; d < dim; ++d) nv[d] = A.tab[d] + ((size_t)sp[d] * 3 * Q + qq[d]) * P1;
  int f0 = br.first[0][sp[0]], f1 = br.first[1][sp[1]], f2 = dim == 3 ? br.first[2][sp[2]] : 0;
  double W = 0, acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int n2 = dim == 3 ? P1 : 1;
  for (int a2 = 0; a2 < n2; ++a2)
    for (int a1 = 0; a1 < P1; ++a1)
      for (int a0 = 0; a0 < P1; ++a0) {
        long long cp = (long long)(f0 + a0) +
                       (long long)br.n_cp[0] * ((f1 + a1) + (long long)br.n_cp[1] * (f2 + a2));
        double N = nv[0][a0] * nv[1][a1] * (dim == 3 ? nv[2][a2] : 1.0);
        double wN = A.wgts[cp] * N;
        W += wN;
        for (int c = 0; c < ncomp && c < 8; ++c) acc[c] += wN * coef[cp * ncomp + c];
      }
  for (int c = 0; c < ncomp && c < 8; ++c) out[idx * ncomp + c] = acc[c] / W;
}

// Physical gradients of sum_a R_a c_a at the Gauss points, reference order,
// (n_elem, nqe, ncomp, dim): the quotient rule for R = w N / W
// (evaluation.py:114-121) and the push-forward J^-T (evaluation.py:149-152),
// applied to the field sums U_c = sum w N c and the geometry sums at once.
__global__ void k_interp_grad(FactorArgs A, const double* __restrict__ coef, int ncomp, double* out) {
  const Bricks& br = A.br;
  const int dim = br.dim, Q = br.q, P1 = br.p + 1;
  const long long nqe = dim == 2 ? Q * Q : Q * Q * Q;
  const long long n_elem = (long long)br.n_span[0] * br.n_span[1] * (dim == 3 ? br.n_span[2] : 1);
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n_elem * nqe) return;
  const long long e = idx / nqe;
  const int q = (int)(idx % nqe);
  const int sp[3] = {(int)(e % br.n_span[0]), (int)((e / br.n_span[0]) % br.n_span[1]),
                     (int)(e / ((long long)br.n_span[0] * br.n_span[1]))};
  const int qq[3] = {q % Q, (q / Q) % Q, dim == 3 ? q / (Q * Q) : 0};
  const double* nv[3];
  const double* nd[3];
  for (int d = 0; d < dim; ++d) {
    const double* base = A.tab[d] + (size_t)sp[d] * 3 * Q * P1;
    nv[d] = base + (size_t)qq[d] * P1;
    nd[d] = base + (size_t)(Q + qq[d]) * P1;
  }
  const int f0 = br.first[0][sp[0]], f1 = br.first[1][sp[1]], f2 = dim == 3 ? br.first[2][sp[2]] : 0;
  double W = 0, Wd[3] = {0, 0, 0}, P[3] = {0, 0, 0}, Pd[3][3] = {}, U[JXB_GRAD_MAXC] = {},
         Ud[JXB_GRAD_MAXC][3] = {};
  const int n2 = dim == 3 ? P1 : 1;
  for (int a2 = 0; a2 < n2; ++a2)
    for (int a1 = 0; a1 < P1; ++a1)
      for (int a0 = 0; a0 < P1; ++a0) {
        const long long cp = (long long)(f0 + a0) +
                             (long long)br.n_cp[0] * ((f1 + a1) + (long long)br.n_cp[1] * (f2 + a2));
        const double z = dim == 3 ? nv[2][a2] : 1.0, dz = dim == 3 ? nd[2][a2] : 0.0;
        const double w = A.wgts[cp];
        const double N = w * nv[0][a0] * nv[1][a1] * z;
        const double dN[3] = {w * nd[0][a0] * nv[1][a1] * z, w * nv[0][a0] * nd[1][a1] * z,
                              w * nv[0][a0] * nv[1][a1] * dz};
        W += N;
        for (int k = 0; k < dim; ++k) Wd[k] += dN[k];
        for (int i = 0; i < dim; ++i) {
          const double X = A.cpts[cp * dim + i];
          P[i] += N * X;
          for (int k = 0; k < dim; ++k) Pd[i][k] += dN[k] * X;
        }
        for (int c = 0; c < ncomp; ++c) {
          const double v = coef[cp * ncomp + c];
          U[c] += N * v;
          for (int k = 0; k < dim; ++k) Ud[c][k] += dN[k] * v;
        }
      }
  const double iW = 1.0 / W;
  double J[3][3], Ji[3][3];
  for (int i = 0; i < dim; ++i) {
    const double x = P[i] * iW;
    for (int a = 0; a < dim; ++a) J[a][i] = (Pd[i][a] - x * Wd[a]) * iW;  // d x_i / d xi_a
  }
  det_inv(dim, J, Ji);
  for (int c = 0; c < ncomp; ++c) {
    const double u = U[c] * iW;
    double ud[3];
    for (int a = 0; a < dim; ++a) ud[a] = (Ud[c][a] - u * Wd[a]) * iW;  // d u / d xi_a
    for (int k = 0; k < dim; ++k) {
      double g = 0;
      for (int a = 0; a < dim; ++a) g += Ji[k][a] * ud[a];
      out[(idx * ncomp + c) * dim + k] = g;
    }
  }
}

// Integration weights in reference element order: w = (w / W) * W.
__global__ void k_qp_weights(Bricks br, const double* __restrict__ wq, const double* __restrict__ invW,
                             double* out) {
  int dim = br.dim, Q = br.q;
  long long nqe = dim == 2 ? Q * Q : Q * Q * Q;
  long long n_elem = (long long)br.n_span[0] * br.n_span[1] * (dim == 3 ? br.n_span[2] : 1);
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n_elem * nqe) return;
  long long e = idx / nqe;
  int q = (int)(idx % nqe);
  int ex = (int)(e % br.n_span[0]);
  int ey = (int)((e / br.n_span[0]) % br.n_span[1]);
  int ez = (int)(e / ((long long)br.n_span[0] * br.n_span[1]));
  int bx = ex / br.te[0], by = ey / br.te[1], bz = ez / br.te[2];
  long long b = bx + (long long)br.nb[0] * (by + (long long)br.nb[1] * bz);
  long long slot = b * ((long long)br.te[0] * br.te[1] * br.te[2]) + (ex % br.te[0]) +
                   (long long)br.te[0] * ((ey % br.te[1]) + (long long)br.te[1] * (ez % br.te[2]));
  double w = wq[slot * nqe + q];
  if (invW) w /= invW[slot * nqe + q];
  out[idx] = w;
}

int qp_weights(jxb_plan* plan, cudaStream_t s, double* w) {
  long long total = plan->n_elem * plan->nqe;
  k_qp_weights<<<(unsigned)((total + 127) / 128), 128, 0, s>>>(plan->br, plan->d_wq, plan->d_invW, w);
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

static FactorArgs make_args(jxb_plan* plan) {
  FactorArgs A;
  A.br = plan->br;
  for (int d = 0; d < 3; ++d) {
    A.tab[d] = plan->d_tab[d];
    A.span_lo[d] = nullptr;
    A.span_hi[d] = nullptr;
  }
  A.cpts = plan->d_cpts;
  A.wgts = plan->d_wgts;
  A.gw = nullptr;
  A.coef_qp = nullptr;
  for (int i = 0; i < 4; ++i) A.coef[i] = plan->coef[i];
  A.op = plan->op;
  A.rational = plan->rational;
  A.ngeo = plan->ngeo;
  A.geo = plan->d_geo;
  A.wq = plan->d_wq;
  A.invW = plan->d_invW;
  return A;
}

int build_tables(jxb_plan* plan, const jxb_desc* desc, cudaStream_t s) {
  int P1 = plan->p + 1, Q = plan->q;
  double* d_nodes = nullptr;
  JXB_CUDA(cudaMalloc(&d_nodes, Q * sizeof(double)));
  JXB_CUDA(cudaMemcpyAsync(d_nodes, desc->gauss_nodes, Q * sizeof(double), cudaMemcpyHostToDevice, s));
  for (int d = 0; d < plan->dim; ++d) {
    int ns = plan->n_span[d];
    double *d_ext = nullptr, *d_lo = nullptr, *d_hi = nullptr;
    JXB_CUDA(cudaMalloc(&d_ext, (size_t)ns * P1 * P1 * sizeof(double)));
    JXB_CUDA(cudaMalloc(&d_lo, ns * sizeof(double)));
    JXB_CUDA(cudaMalloc(&d_hi, ns * sizeof(double)));
    JXB_CUDA(cudaMemcpyAsync(d_ext, desc->extraction[d], (size_t)ns * P1 * P1 * sizeof(double),
                             cudaMemcpyHostToDevice, s));
    JXB_CUDA(cudaMemcpyAsync(d_lo, desc->span_lo[d], ns * sizeof(double), cudaMemcpyHostToDevice, s));
    JXB_CUDA(cudaMemcpyAsync(d_hi, desc->span_hi[d], ns * sizeof(double), cudaMemcpyHostToDevice, s));
    size_t n = (size_t)ns * 3 * Q * P1;
    JXB_CUDA(cudaMalloc(&plan->d_tab[d], n * sizeof(double)));
    JXB_CUDA(cudaMalloc(&plan->d_tab32[d], n * sizeof(float)));
    int total = ns * Q * P1;
    k_tables<<<(total + 127) / 128, 128, 0, s>>>(plan->p, Q, ns, d_ext, d_lo, d_hi, d_nodes,
                                                 plan->d_tab[d], plan->d_tab32[d]);
    JXB_CUDA(cudaGetLastError());
    // kept for evaluation at arbitrary points (jxb_eval_points)
    plan->d_ext[d] = d_ext;
    plan->d_lo[d] = d_lo;
    plan->d_hi[d] = d_hi;
  }
  JXB_CUDA(cudaStreamSynchronize(s));
  cudaFree(d_nodes);
  return JXB_OK;
}

int build_factors(jxb_plan* plan, const jxb_desc* desc, cudaStream_t s) {
  FactorArgs A = make_args(plan);
  std::vector<void*> tmp;
  auto upload = [&](const void* h, size_t bytes) -> void* {
    void* d = nullptr;
    if (cudaMalloc(&d, bytes) != cudaSuccess) return nullptr;
    cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s);
    tmp.push_back(d);
    return d;
  };
  for (int d = 0; d < plan->dim; ++d) {
    A.span_lo[d] = (const double*)upload(desc->span_lo[d], plan->n_span[d] * sizeof(double));
    A.span_hi[d] = (const double*)upload(desc->span_hi[d], plan->n_span[d] * sizeof(double));
  }
  A.gw = (const double*)upload(desc->gauss_weights, plan->q * sizeof(double));
  if (desc->coef_qp && plan->op == JXB_OP_POISSON)
    A.coef_qp = (const double*)upload(desc->coef_qp, (size_t)plan->n_elem * plan->nqe * sizeof(double));
  for (void* p : tmp)
    if (!p) return fail(JXB_ERR_NOMEM, "device allocation failed while building factors");
  long long total = plan->br.slots * plan->nqe;
  k_factors<<<(unsigned)((total + 127) / 128), 128, 0, s>>>(A);
  JXB_CUDA(cudaGetLastError());
  JXB_CUDA(cudaStreamSynchronize(s));
  for (void* p : tmp) cudaFree(p);
  return JXB_OK;
}

int qp_coords(jxb_plan* plan, cudaStream_t s, double* x) {
  FactorArgs A = make_args(plan);
  long long total = plan->n_elem * plan->nqe;
  k_coords<<<(unsigned)((total + 127) / 128), 128, 0, s>>>(A, x);
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

// Evaluation at arbitrary reference points: point k lies in element
// elems[k] (reference order, first direction fastest) at ref[k] in [-1, 1]^dim.
// The extracted 1D basis is formed on the fly from the Bernstein recurrence
// and the element's extraction rows (evaluation.py:374-386), then the same
// quotient rule and push-forward as the Gauss-point kernels. Outputs (any may
// be null): val (n, ncomp), grad (n, ncomp, dim), x (n, dim) and
// jac = |det J| prod(h/2) (n), the measure the reference multiplies its
// quadrature weights by (evaluation.py:461-463). A point whose element index
// is out of range yields NaN.
struct EvalArgs {
  Bricks br;
  const double* ext[3];
  const double* lo[3];
  const double* hi[3];
  const double* cpts;
  const double* wgts;
};

__global__ void k_eval_points(EvalArgs A, long long n, const long long* __restrict__ elems,
                              const double* __restrict__ ref, const double* __restrict__ coef, int ncomp,
                              double* val, double* grad, double* xout, double* jac) {
  const Bricks& br = A.br;
  const int dim = br.dim, P1 = br.p + 1;
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const long long n_elem = (long long)br.n_span[0] * br.n_span[1] * (dim == 3 ? br.n_span[2] : 1);
  const long long e = elems[k];
  if (e < 0 || e >= n_elem) {
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    for (int c = 0; c < ncomp; ++c) {
      if (val) val[k * ncomp + c] = nan;
      if (grad)
        for (int d = 0; d < dim; ++d) grad[(k * ncomp + c) * dim + d] = nan;
    }
    if (xout)
      for (int d = 0; d < dim; ++d) xout[k * dim + d] = nan;
    if (jac) jac[k] = nan;
    return;
  }
  const int sp[3] = {(int)(e % br.n_span[0]), (int)((e / br.n_span[0]) % br.n_span[1]),
                     (int)(e / ((long long)br.n_span[0] * br.n_span[1]))};
  double nv[3][JXB_MAXP + 1], nd[3][JXB_MAXP + 1];
  double meas = 1.0;
  for (int d = 0; d < 3; ++d)
    for (int a = 0; a < P1; ++a) {
      nv[d][a] = d < dim ? 0.0 : 1.0;
      nd[d][a] = 0.0;
    }
  for (int d = 0; d < dim; ++d) {
    double B[JXB_MAXP + 1], dB[JXB_MAXP + 1], d2B[JXB_MAXP + 1];
    bernstein_point(ref[k * dim + d], br.p, B, dB, d2B);
    const double h = A.hi[d][sp[d]] - A.lo[d][sp[d]];
    const double* C = A.ext[d] + (size_t)sp[d] * P1 * P1;
    for (int a = 0; a < P1; ++a) {
      double v = 0, g = 0;
      for (int j = 0; j < P1; ++j) {
        v += C[a * P1 + j] * B[j];
        g += C[a * P1 + j] * dB[j];
      }
      nv[d][a] = v;
      nd[d][a] = g * 2.0 / h;
    }
    meas *= h / 2.0;
  }
  const int f0 = br.first[0][sp[0]], f1 = br.first[1][sp[1]], f2 = dim == 3 ? br.first[2][sp[2]] : 0;
  double W = 0, Wd[3] = {0, 0, 0}, P[3] = {0, 0, 0}, Pd[3][3] = {}, U[JXB_GRAD_MAXC] = {},
         Ud[JXB_GRAD_MAXC][3] = {};
  const int n2 = dim == 3 ? P1 : 1;
  for (int a2 = 0; a2 < n2; ++a2)
    for (int a1 = 0; a1 < P1; ++a1)
      for (int a0 = 0; a0 < P1; ++a0) {
        const long long cp = (long long)(f0 + a0) +
                             (long long)br.n_cp[0] * ((f1 + a1) + (long long)br.n_cp[1] * (f2 + a2));
        const double w = A.wgts[cp];
        const double z = nv[2][a2], dz = nd[2][a2];
        const double N = w * nv[0][a0] * nv[1][a1] * z;
        const double dN[3] = {w * nd[0][a0] * nv[1][a1] * z, w * nv[0][a0] * nd[1][a1] * z,
                              w * nv[0][a0] * nv[1][a1] * dz};
        W += N;
        for (int q = 0; q < dim; ++q) Wd[q] += dN[q];
        for (int i = 0; i < dim; ++i) {
          const double X = A.cpts[cp * dim + i];
          P[i] += N * X;
          for (int q = 0; q < dim; ++q) Pd[i][q] += dN[q] * X;
        }
        if (coef)
          for (int c = 0; c < ncomp; ++c) {
            const double v = coef[cp * ncomp + c];
            U[c] += N * v;
            for (int q = 0; q < dim; ++q) Ud[c][q] += dN[q] * v;
          }
      }
  const double iW = 1.0 / W;
  double J[3][3], Ji[3][3], x[3];
  for (int i = 0; i < dim; ++i) {
    x[i] = P[i] * iW;
    for (int a = 0; a < dim; ++a) J[a][i] = (Pd[i][a] - x[i] * Wd[a]) * iW;
  }
  const double det = det_inv(dim, J, Ji);
  if (xout)
    for (int i = 0; i < dim; ++i) xout[k * dim + i] = x[i];
  if (jac) jac[k] = fabs(det) * meas;
  if (!coef) return;
  for (int c = 0; c < ncomp; ++c) {
    const double u = U[c] * iW;
    if (val) val[k * ncomp + c] = u;
    if (grad) {
      double ud[3];
      for (int a = 0; a < dim; ++a) ud[a] = (Ud[c][a] - u * Wd[a]) * iW;
      for (int q = 0; q < dim; ++q) {
        double g = 0;
        for (int a = 0; a < dim; ++a) g += Ji[q][a] * ud[a];
        grad[(k * ncomp + c) * dim + q] = g;
      }
    }
  }
}

int eval_points(jxb_plan* plan, cudaStream_t s, const double* coef, int ncomp, long long n,
                const long long* elems, const double* ref, double* val, double* grad, double* x, double* jac) {
  if (coef && (ncomp < 1 || ncomp > JXB_GRAD_MAXC))
    return fail(JXB_ERR_INVALID, "jxb_eval_points: ncomp must be in 1..3");
  if (n < 0) return fail(JXB_ERR_INVALID, "jxb_eval_points: negative point count");
  if (n == 0) return JXB_OK;
  EvalArgs A;
  A.br = plan->br;
  for (int d = 0; d < 3; ++d) {
    A.ext[d] = plan->d_ext[d];
    A.lo[d] = plan->d_lo[d];
    A.hi[d] = plan->d_hi[d];
  }
  A.cpts = plan->d_cpts;
  A.wgts = plan->d_wgts;
  k_eval_points<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(A, n, elems, ref, coef, ncomp, val, grad, x, jac);
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

// Geometry of boundary points: point q of face f lies on side sides[f]
// (2 * direction + end) of element elems[f] at ref[f, q]. Writes the physical
// point, the outward unit normal n ~ dxdxi^-1 e_d with the side's sign, and
// the surface weight wref * |tangent| (2D) or |t0 x t1| (3D) * prod of the
// tangential half-widths (evaluation.py:174-193, 432-455).
__device__ void boundary_geometry(const EvalArgs& A, long long e, int side, const double* xi, double* x, double* nrm,
                                  double* surf, double* nv_out, int P1) {
  const Bricks& br = A.br;
  const int dim = br.dim;
  const int sp[3] = {(int)(e % br.n_span[0]), (int)((e / br.n_span[0]) % br.n_span[1]),
                     (int)(e / ((long long)br.n_span[0] * br.n_span[1]))};
  double nv[3][JXB_MAXP + 1], nd[3][JXB_MAXP + 1], half[3] = {1, 1, 1};
  for (int d = 0; d < 3; ++d)
    for (int a = 0; a < P1; ++a) {
      nv[d][a] = d < dim ? 0.0 : 1.0;
      nd[d][a] = 0.0;
    }
  for (int d = 0; d < dim; ++d) {
    double B[JXB_MAXP + 1], dB[JXB_MAXP + 1], d2B[JXB_MAXP + 1];
    bernstein_point(xi[d], br.p, B, dB, d2B);
    const double h = A.hi[d][sp[d]] - A.lo[d][sp[d]];
    const double* C = A.ext[d] + (size_t)sp[d] * P1 * P1;
    for (int a = 0; a < P1; ++a) {
      double v = 0, g = 0;
      for (int j = 0; j < P1; ++j) {
        v += C[a * P1 + j] * B[j];
        g += C[a * P1 + j] * dB[j];
      }
      nv[d][a] = v;
      nd[d][a] = g * 2.0 / h;
    }
    half[d] = h / 2.0;
  }
  if (nv_out)
    for (int d = 0; d < 3; ++d)
      for (int a = 0; a < P1; ++a) nv_out[d * (JXB_MAXP + 1) + a] = nv[d][a];
  const int f0 = br.first[0][sp[0]], f1 = br.first[1][sp[1]], f2 = dim == 3 ? br.first[2][sp[2]] : 0;
  double W = 0, Wd[3] = {0, 0, 0}, P[3] = {0, 0, 0}, Pd[3][3] = {};
  const int n2 = dim == 3 ? P1 : 1;
  for (int a2 = 0; a2 < n2; ++a2)
    for (int a1 = 0; a1 < P1; ++a1)
      for (int a0 = 0; a0 < P1; ++a0) {
        const long long cp = (long long)(f0 + a0) +
                             (long long)br.n_cp[0] * ((f1 + a1) + (long long)br.n_cp[1] * (f2 + a2));
        const double w = A.wgts[cp];
        const double N = w * nv[0][a0] * nv[1][a1] * nv[2][a2];
        const double dN[3] = {w * nd[0][a0] * nv[1][a1] * nv[2][a2], w * nv[0][a0] * nd[1][a1] * nv[2][a2],
                              w * nv[0][a0] * nv[1][a1] * nd[2][a2]};
        W += N;
        for (int q = 0; q < dim; ++q) Wd[q] += dN[q];
        for (int i = 0; i < dim; ++i) {
          const double X = A.cpts[cp * dim + i];
          P[i] += N * X;
          for (int q = 0; q < dim; ++q) Pd[i][q] += dN[q] * X;
        }
      }
  const double iW = 1.0 / W;
  double J[3][3] = {}, Ji[3][3];
  for (int i = 0; i < dim; ++i) {
    x[i] = P[i] * iW;
    for (int a = 0; a < dim; ++a) J[a][i] = (Pd[i][a] - x[i] * Wd[a]) * iW;
  }
  det_inv(dim, J, Ji);
  const int dir = side / 2;
  const double sign = (side % 2) ? 1.0 : -1.0;
  double len = 0;
  for (int k = 0; k < dim; ++k) len += Ji[k][dir] * Ji[k][dir];
  len = sqrt(len);
  for (int k = 0; k < dim; ++k) nrm[k] = sign * Ji[k][dir] / len;
  double sj, tang = 1.0;
  if (dim == 2) {
    const int t = 1 - dir;
    sj = sqrt(J[t][0] * J[t][0] + J[t][1] * J[t][1]);
    tang = half[t];
  } else {
    const int t0 = dir == 0 ? 1 : 0, t1 = dir == 2 ? 1 : 2;
    const double c0 = J[t0][1] * J[t1][2] - J[t0][2] * J[t1][1];
    const double c1 = J[t0][2] * J[t1][0] - J[t0][0] * J[t1][2];
    const double c2 = J[t0][0] * J[t1][1] - J[t0][1] * J[t1][0];
    sj = sqrt(c0 * c0 + c1 * c1 + c2 * c2);
    tang = half[t0] * half[t1];
  }
  *surf = sj * tang;
}

__global__ void k_boundary_points(EvalArgs A, long long n_faces, int n_q, const long long* __restrict__ elems,
                                  const int* __restrict__ sides, const double* __restrict__ ref,
                                  const double* __restrict__ wref, double* x, double* normal, double* w) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_faces * n_q) return;
  const int dim = A.br.dim;
  const long long f = k / n_q;
  double xx[3], nn[3], surf;
  boundary_geometry(A, elems[f], sides[f], ref + k * dim, xx, nn, &surf, nullptr, A.br.p + 1);
  for (int i = 0; i < dim; ++i) {
    if (x) x[k * dim + i] = xx[i];
    if (normal) normal[k * dim + i] = nn[i];
  }
  if (w) w[k] = wref[k] * surf;
}

// Face-local loads: local[f, a, c] = sum_q w_q t_q[c] R_a(x_q), one thread per
// (face, local basis function a), a first-direction-fastest over the element.
__global__ void k_boundary_local(EvalArgs A, long long n_faces, int n_q, const long long* __restrict__ elems,
                                 const double* __restrict__ ref, const double* __restrict__ w,
                                 const double* __restrict__ t, int vec, double* local) {
  const Bricks& br = A.br;
  const int dim = br.dim, P1 = br.p + 1;
  const int n_loc = dim == 3 ? P1 * P1 * P1 : P1 * P1;
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_faces * n_loc) return;
  const long long f = k / n_loc;
  const int a = (int)(k % n_loc);
  const int a0 = a % P1, a1 = (a / P1) % P1, a2 = dim == 3 ? a / (P1 * P1) : 0;
  const long long e = elems[f];
  const int sp[3] = {(int)(e % br.n_span[0]), (int)((e / br.n_span[0]) % br.n_span[1]),
                     (int)(e / ((long long)br.n_span[0] * br.n_span[1]))};
  const int f0 = br.first[0][sp[0]], f1 = br.first[1][sp[1]], f2 = dim == 3 ? br.first[2][sp[2]] : 0;
  double acc[3] = {0, 0, 0};
  for (int q = 0; q < n_q; ++q) {
    const long long pq = f * n_q + q;
    double nv[3][JXB_MAXP + 1];
    for (int d = 0; d < 3; ++d)
      for (int b = 0; b < P1; ++b) nv[d][b] = d < dim ? 0.0 : 1.0;
    for (int d = 0; d < dim; ++d) {
      double B[JXB_MAXP + 1], dB[JXB_MAXP + 1], d2B[JXB_MAXP + 1];
      bernstein_point(ref[pq * dim + d], br.p, B, dB, d2B);
      const double* C = A.ext[d] + (size_t)sp[d] * P1 * P1;
      for (int b = 0; b < P1; ++b) {
        double v = 0;
        for (int j = 0; j < P1; ++j) v += C[b * P1 + j] * B[j];
        nv[d][b] = v;
      }
    }
    double W = 0;
    const int n2 = dim == 3 ? P1 : 1;
    for (int b2 = 0; b2 < n2; ++b2)
      for (int b1 = 0; b1 < P1; ++b1)
        for (int b0 = 0; b0 < P1; ++b0) {
          const long long cp = (long long)(f0 + b0) +
                               (long long)br.n_cp[0] * ((f1 + b1) + (long long)br.n_cp[1] * (f2 + b2));
          W += A.wgts[cp] * nv[0][b0] * nv[1][b1] * nv[2][b2];
        }
    const long long cpa = (long long)(f0 + a0) +
                          (long long)br.n_cp[0] * ((f1 + a1) + (long long)br.n_cp[1] * (f2 + a2));
    const double R = A.wgts[cpa] * nv[0][a0] * nv[1][a1] * nv[2][a2] / W;
    for (int c = 0; c < vec; ++c) acc[c] += w[pq] * t[pq * vec + c] * R;
  }
  for (int c = 0; c < vec; ++c) local[k * vec + c] = acc[c];
}

// F[vec * dof[i] + c] += sum over j in [ptr[i], ptr[i+1]) of local[contrib[j] * vec + c],
// in the fixed order of contrib (deterministic, no atomics).
__global__ void k_boundary_gather(long long n_touched, const long long* __restrict__ dof,
                                  const long long* __restrict__ ptr, const long long* __restrict__ contrib, int vec,
                                  const double* __restrict__ local, double* F) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_touched) return;
  for (int c = 0; c < vec; ++c) {
    double s = 0;
    for (long long j = ptr[i]; j < ptr[i + 1]; ++j) s += local[contrib[j] * vec + c];
    F[dof[i] * vec + c] += s;
  }
}

static EvalArgs eval_args(jxb_plan* plan) {
  EvalArgs A;
  A.br = plan->br;
  for (int d = 0; d < 3; ++d) {
    A.ext[d] = plan->d_ext[d];
    A.lo[d] = plan->d_lo[d];
    A.hi[d] = plan->d_hi[d];
  }
  A.cpts = plan->d_cpts;
  A.wgts = plan->d_wgts;
  return A;
}

int boundary_points(jxb_plan* plan, cudaStream_t s, long long n_faces, int n_q, const long long* elems,
                    const int* sides, const double* ref, const double* wref, double* x, double* normal, double* w) {
  if (n_faces < 0 || n_q < 1) return fail(JXB_ERR_INVALID, "jxb_boundary_points: bad sizes");
  if (n_faces == 0) return JXB_OK;
  const long long n = n_faces * n_q;
  k_boundary_points<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(eval_args(plan), n_faces, n_q, elems, sides, ref,
                                                                 wref, x, normal, w);
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

int boundary_load(jxb_plan* plan, cudaStream_t s, long long n_faces, int n_q, const long long* elems,
                  const double* ref, const double* w, const double* t, long long n_touched, const long long* dof,
                  const long long* ptr, const long long* contrib, double* local, double* F) {
  if (n_faces < 0 || n_q < 1 || n_touched < 0) return fail(JXB_ERR_INVALID, "jxb_boundary_load: bad sizes");
  if (n_faces == 0) return JXB_OK;
  const int P1 = plan->p + 1;
  const long long n_loc = plan->dim == 3 ? P1 * P1 * P1 : P1 * P1;
  const long long n = n_faces * n_loc;
  k_boundary_local<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(eval_args(plan), n_faces, n_q, elems, ref, w, t,
                                                                plan->vec, local);
  JXB_CUDA(cudaGetLastError());
  if (n_touched > 0) {
    k_boundary_gather<<<(unsigned)((n_touched + 127) / 128), 128, 0, s>>>(n_touched, dof, ptr, contrib, plan->vec,
                                                                          local, F);
    JXB_CUDA(cudaGetLastError());
  }
  return JXB_OK;
}

// Neo-Hookean state at every (element slot, Gauss point) for the displacement
// u (interleaved (n_cp, dim)): F = I + grad u, J = det F, and written after the
// elasticity geometry of the point: F^-T, c = mu - lambda ln J and the flux
// w P J^-T, P = mu (F - F^-T) + lambda ln J F^-T the gradient of the stored
// energy W = mu/2 (tr F^T F - d) - mu ln J + lambda/2 (ln J)^2
// (src/jaxiga/forms/library.py:206-225). J^-1, w|J| and the rational factors
// 1/W, grad W / W are read from the point's stored geometry (k_factors), the
// displacement gradient is summed from the tables. Each block adds its points'
// w W into partials[blockIdx.x] in a fixed order (grid JXB_RED_BLOCKS,
// grid-stride).
__global__ void __launch_bounds__(256) k_hyper_state(FactorArgs A, const double* __restrict__ u,
                                                     double* __restrict__ partials) {
  const Bricks& br = A.br;
  const int dim = br.dim, Q = br.q, P1 = br.p + 1;
  const long long nqe = dim == 2 ? Q * Q : Q * Q * Q;
  const double mu = A.coef[0], lam = A.coef[1];
  const int e0 = dim * dim + 1 + (A.rational ? dim + 1 : 0);
  double wsum = 0.0;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < br.slots * nqe;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long slot = idx / nqe;
    const int q = (int)(idx % nqe);
    int ex, ey, ez;
    bool valid;
    elem_of_slot(br, slot, ex, ey, ez, valid);
    if (!valid) continue;
    const GeoAt ga = geo_at(dim, slot, q, Q, A.ngeo, nqe, br.te[0]);
    double* g = A.geo + ga.base;
    const size_t gs = ga.stride;
    double Ji[3][3];
    for (int i = 0; i < dim; ++i)
      for (int a = 0; a < dim; ++a) Ji[i][a] = g[gs * (i * dim + a)];
    const double om = g[gs * (dim * dim)];
    double iW = 1.0, gW[3] = {0, 0, 0};
    if (A.rational) {
      iW = g[gs * (dim * dim + 1)];
      for (int a = 0; a < dim; ++a) gW[a] = g[gs * (dim * dim + 2 + a)];
    }
    const int sp[3] = {ex, ey, ez};
    const int qq[3] = {q % Q, (q / Q) % Q, dim == 3 ? q / (Q * Q) : 0};
    const double* nv[3];
    const double* nd[3];
    for (int d = 0; d < dim; ++d) {
      const double* base = A.tab[d] + (size_t)sp[d] * 3 * Q * P1;
      nv[d] = base + (size_t)qq[d] * P1;
      nd[d] = base + (size_t)(Q + qq[d]) * P1;
    }
    const int f0 = br.first[0][ex], f1 = br.first[1][ey], f2 = dim == 3 ? br.first[2][ez] : 0;
    double U[3] = {0, 0, 0}, Ud[3][3] = {};
    const int n2 = dim == 3 ? P1 : 1;
    for (int a2 = 0; a2 < n2; ++a2)
      for (int a1 = 0; a1 < P1; ++a1)
        for (int a0 = 0; a0 < P1; ++a0) {
          const long long cp = (long long)(f0 + a0) +
                               (long long)br.n_cp[0] * ((f1 + a1) + (long long)br.n_cp[1] * (f2 + a2));
          const double z = dim == 3 ? nv[2][a2] : 1.0, dz = dim == 3 ? nd[2][a2] : 0.0;
          const double w = A.rational ? A.wgts[cp] : 1.0;
          const double N = w * nv[0][a0] * nv[1][a1] * z;
          const double dN[3] = {w * nd[0][a0] * nv[1][a1] * z, w * nv[0][a0] * nd[1][a1] * z,
                                w * nv[0][a0] * nv[1][a1] * dz};
          for (int i = 0; i < dim; ++i) {
            const double v = u[cp * dim + i];
            U[i] += N * v;
            for (int k = 0; k < dim; ++k) Ud[i][k] += dN[k] * v;
          }
        }
    // F = I + du_i / dx_k, du_i / dxi_a = (Ud - u W_a) / W
    double F[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int i = 0; i < dim; ++i) {
      const double ui = U[i] * iW;
      double ud[3];
      for (int a = 0; a < dim; ++a) ud[a] = Ud[i][a] * iW - ui * gW[a];
      for (int k = 0; k < dim; ++k) {
        double gk = 0;
        for (int a = 0; a < dim; ++a) gk += Ji[k][a] * ud[a];
        F[i][k] += gk;
      }
    }
    double Fi[3][3];
    const double Jd = det_inv(dim, F, Fi);  // Fi = F^-1
    const double lnJ = log(Jd);             // J <= 0: not finite, as the reference's log
    double I1 = 0;
    for (int i = 0; i < dim; ++i)
      for (int k = 0; k < dim; ++k) I1 += F[i][k] * F[i][k];
    wsum += om * (0.5 * mu * (I1 - dim) - mu * lnJ + 0.5 * lam * lnJ * lnJ);
    int k = e0;
    for (int i = 0; i < dim; ++i)
      for (int a = 0; a < dim; ++a) g[gs * (k++)] = Fi[a][i];  // F^-T
    g[gs * (k++)] = mu - lam * lnJ;
    for (int i = 0; i < dim; ++i)
      for (int a = 0; a < dim; ++a) {  // w P J^-T, P_ik = mu (F_ik - F^-T_ik) + lambda ln J F^-T_ik
        double f = 0;
        for (int kk = 0; kk < dim; ++kk) {
          const double Pik = mu * (F[i][kk] - Fi[kk][i]) + lam * lnJ * Fi[kk][i];
          f += Pik * Ji[kk][a];
        }
        g[gs * (k++)] = om * f;
      }
  }
  // fixed-order block sum
  __shared__ double part[8];
  for (int o = 16; o > 0; o >>= 1) wsum += __shfl_down_sync(0xffffffffu, wsum, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = wsum;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += part[i];
    partials[blockIdx.x] = t;
  }
}

int hyper_state(jxb_plan* plan, cudaStream_t s, const double* u, double* energy) {
  if (plan->op != JXB_OP_HYPERELASTIC) return fail(JXB_ERR_INVALID, "jxb_hyper_state: not a hyperelastic plan");
  FactorArgs A = make_args(plan);
  k_hyper_state<<<JXB_RED_BLOCKS, 256, 0, s>>>(A, u, plan->d_red);
  JXB_CUDA(cudaGetLastError());
  plan->diag_valid = false;  // the Jacobi diagonal follows the state
  if (energy) {
    double h[JXB_RED_BLOCKS];
    JXB_CUDA(cudaMemcpyAsync(h, plan->d_red, sizeof h, cudaMemcpyDeviceToHost, s));
    JXB_CUDA(cudaStreamSynchronize(s));
    double e = 0;
    for (int i = 0; i < JXB_RED_BLOCKS; ++i) e += h[i];
    *energy = e;
  }
  return JXB_OK;
}

int interpolate_grad(jxb_plan* plan, cudaStream_t s, const double* coef, int ncomp, double* out) {
  if (ncomp < 1 || ncomp > JXB_GRAD_MAXC)
    return fail(JXB_ERR_INVALID, "jxb_interpolate_grad: ncomp must be in 1..3");
  FactorArgs A = make_args(plan);
  long long total = plan->n_elem * plan->nqe;
  k_interp_grad<<<(unsigned)((total + 127) / 128), 128, 0, s>>>(A, coef, ncomp, out);
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

int interpolate(jxb_plan* plan, cudaStream_t s, const double* coef, int ncomp, double* out) {
  if (ncomp < 1 || ncomp > 8) return fail(JXB_ERR_INVALID, "interpolate: ncomp must be in 1..8");
  FactorArgs A = make_args(plan);
  long long total = plan->n_elem * plan->nqe;
  k_interp<<<(unsigned)((total + 127) / 128), 128, 0, s>>>(A, coef, ncomp, out);
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

}  // namespace jxb
