// Matrix-free, sum-factorised stiffness application with a deterministic
// scatter-add (the B200 replacement of the JVP matvec of
// src/jaxiga/methods/galerkin.py:207-218 and of the element-tangent scatter of
// galerkin.py:122-142), plus the load vector and the Jacobi diagonal.
//
// One CTA owns one brick of elements and walks its element layers in order.
// Per layer, each element is handled by Q*Q threads (3D) or Q threads (2D):
//
//   forward   u (p+1)^d  --N_x, N'_x-->  --N_y, N'_y-->  --N_z, N'_z--> grad u at Q^d points
//   point op  flux = M_q . (value, grad[, hessian])        (per-point factors)
//   backward  the transposed contractions back to the (p+1)^d element residual
//
// The x/y contractions go through shared memory, the last direction stays in
// registers. Element residuals of a layer are staged in shared memory and
// summed into the brick's footprint accumulator by a gather in a fixed order
// (no atomics), so the result is bitwise reproducible. At the end the
// footprint is written to a scratch buffer and a combine pass adds, per
// control point, the bricks covering it, again in a fixed order.
//
// The per-point factors of one element layer are one contiguous tile in HBM.
// The 3D kernel asks the bulk-copy (TMA) engine to prefetch the next layer's
// tile into L2 (cp.async.bulk.prefetch.L2) at the start of each layer, and the
// point operator then reads its factors with coalesced read-only loads that
// hit L2. Keeping the tile out of shared memory is what lets two 256-thread
// CTAs share an SM.
#include <math.h>
#include <stdlib.h>

#include <algorithm>

#include "jxb_internal.cuh"

namespace jxb {

enum OpKind { OPK_SCALAR = 0, OPK_ELAST = 1, OPK_PLATE = 2, OPK_HYPER = 3 };

// operators with one displacement component per direction
template <int OPK>
constexpr bool vec_op() {
  return OPK == OPK_ELAST || OPK == OPK_HYPER;
}

// ---------------------------------------------------------------------------
// compile-time shapes
// ---------------------------------------------------------------------------
template <int DIM, int P>
struct BrickShape;
template <int P>
struct BrickShape<3, P> {
  static constexpr int TX = P <= 4 ? 4 : 3;
  static constexpr int TY = TX;
  static constexpr int CZ = 8;  // element layers per brick at most (the plan may take fewer)
  static constexpr int MINB = P <= 3 ? 2 : 1;  // resident CTAs per SM the kernel is built for
};
template <int P>
struct BrickShape<2, P> {
  static constexpr int TX = 32;
  static constexpr int TY = 8;  // element rows per brick
  static constexpr int CZ = 1;
};

// Resident CTAs per SM the 3D FMA brick kernel is built for. The FP32 copies
// need half the registers, so they trade registers for occupancy: scalar 4
// CTAs (64 registers, no spills), elasticity 3 (80 registers, ~100 B spilled),
// which measured 19 % and 6 % faster than 2 CTAs at p = 3.
template <typename T, int P, int OPK>
constexpr int brick3_min_blocks() {
  return OPK == OPK_HYPER ? 1 : (sizeof(T) == 4 && P <= 3) ? (OPK == OPK_ELAST ? 3 : 4) : BrickShape<3, P>::MINB;
}

// Factors per Gauss point. The hyperelastic operator stores the elasticity
// geometry (J^-1, w|J|[, 1/W, grad W / W]) and then its state: F^-T (row major),
// mu - lambda ln J, and the flux w P(F) J^-T of the residual (row major).
template <int OPK, bool RAT, int DIM>
struct GeoCount {
  static constexpr int elast = DIM * DIM + 1 + (RAT ? DIM + 1 : 0);
  static constexpr int value = OPK == OPK_SCALAR ? (RAT ? (DIM + 1) * (DIM + 2) / 2 : DIM * (DIM + 1) / 2)
                               : OPK == OPK_ELAST ? elast
                               : OPK == OPK_HYPER ? elast + 2 * DIM * DIM + 1
                                                  : (RAT ? 21 : 15);
};

// om times the neo-Hookean first Piola-Kirchhoff increment at a stored state
// (M = F^-T, c = mu - lambda ln J):
// dP = mu dF + c F^-T dF^T F^-T + lambda (F^-T : dF) F^-T.
template <typename T, int D>
__device__ __forceinline__ void hyper_dP(const T (&M)[D][D], T c, T lam, T mu, T om, const T (&dF)[D][D],
                                         T (&S)[D][D]) {
  T t1[D][D];  // F^-T dF^T
  T tr = 0;
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int b = 0; b < D; ++b) {
      T v = 0;
#pragma unroll
      for (int a = 0; a < D; ++a) v += M[i][a] * dF[b][a];
      t1[i][b] = v;
      tr += M[i][b] * dF[i][b];
    }
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int k = 0; k < D; ++k) {
      T v = 0;
#pragma unroll
      for (int b = 0; b < D; ++b) v += t1[i][b] * M[b][k];
      S[i][k] = om * (mu * dF[i][k] + c * v + lam * tr * M[i][k]);
    }
}

int host_geo_count(int op, int rational, int dim) {
  if (op == JXB_OP_POISSON) return rational ? (dim + 1) * (dim + 2) / 2 : dim * (dim + 1) / 2;
  if (op == JXB_OP_ELASTICITY) return dim * dim + 1 + (rational ? dim + 1 : 0);
  if (op == JXB_OP_HYPERELASTIC) return dim * dim + 1 + (rational ? dim + 1 : 0) + 2 * dim * dim + 1;
  return rational ? 21 : 15;
}

void host_brick_shape(int dim, int p, int* te) {
  if (dim == 3) {
    te[0] = te[1] = p <= 4 ? 4 : 3;
    te[2] = 8;
  } else {
    te[0] = 32;
    te[1] = 8;
    te[2] = 1;
  }
}

// Shared-memory strides chosen so the stage-to-stage transposes are free of
// bank conflicts for Q <= 4 (double words: a stride congruent to Q modulo 16).
template <int P, int Q>
struct Strides3 {
  static constexpr int P1 = P + 1, PP = P1 * P1;
  static constexpr int SX = PP + 1;                                    // q0 stride of bufX
  static constexpr int SY1 = Q * P1 + (((Q - Q * P1) % 16) + 16) % 16;  // q1 stride of bufY
  static constexpr int SYC = Q * SY1;                                  // channel stride of bufY
  static constexpr int SP = P1 + 1;                                    // line stride of stage
  static constexpr int SST = PP * SP;                                  // (element, component) stride of stage
};

// L2 prefetch of a contiguous byte range by the bulk-copy engine.
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}


// ---------------------------------------------------------------------------
// 3D brick kernel
// ---------------------------------------------------------------------------
template <typename T, int P, int Q, int OPK, bool RAT, int MODE>
__global__ void __launch_bounds__(BrickShape<3, P>::TX* BrickShape<3, P>::TY* Q* Q, brick3_min_blocks<T, P, OPK>())
    k_brick3(BrickArgs<T> A) {
  using S = Strides3<P, Q>;
  constexpr int P1 = P + 1, PP = P1 * P1, PPP = PP * P1;
  constexpr int TX = BrickShape<3, P>::TX, TY = BrickShape<3, P>::TY;
  constexpr int NE = TX * TY, QQ = Q * Q, NQE = Q * Q * Q, NT = NE * QQ;
  constexpr int VEC = vec_op<OPK>() ? 3 : 1;
  constexpr int NG = GeoCount<OPK, RAT, 3>::value;
  constexpr int E0 = GeoCount<OPK_ELAST, RAT, 3>::elast;  // hyperelastic: start of the state
  constexpr bool HASV = RAT || MODE == MODE_LOAD;  // value channel
  constexpr int SX = S::SX, SY1 = S::SY1, SYC = S::SYC, SP = S::SP, SST = S::SST;

  if (A.state && A.state->done) return;
  const Bricks& br = A.br;
  const int fp0 = br.fp[0], fp1 = br.fp[1], fp2 = br.fp[2];

  extern __shared__ __align__(128) unsigned char smem_raw[];
  T* stx = reinterpret_cast<T*>(smem_raw);  // [TX][2][Q][P1]
  T* sty = stx + TX * 2 * Q * P1;           // [TY][2][Q][P1]
  T* stz = sty + TY * 2 * Q * P1;           // [2][Q][P1]
  T* bufX = stz + 2 * Q * P1;               // [NE][2][Q][SX]
  T* bufY = bufX + NE * 2 * Q * SX;         // [NE][3][SYC]
  T* stage = bufY + NE * 3 * SYC;           // [NE][VEC][PP][SP]
  T* acc = stage + NE * VEC * SST;          // [VEC][fp2][fp1][fp0]
  T* su = acc + VEC * fp0 * fp1 * fp2;      // [P1][fp1][fp0][VEC] layer input tile
  const int sun = MODE == MODE_APPLY ? P1 * fp1 * fp0 * VEC : 0;
  int* soff = reinterpret_cast<int*>(su + sun);  // offx[TX], offy[TY]

  const int tid = threadIdx.x;
  const long long b = blockIdx.x;
  const int bx = (int)(b % br.nb[0]);
  const int by = (int)((b / br.nb[0]) % br.nb[1]);
  const int bz = (int)(b / ((long long)br.nb[0] * br.nb[1]));
  const int cp0x = br.bcp0[0][bx], cp0y = br.bcp0[1][by], cp0z = br.bcp0[2][bz];

  const int el = tid / QQ, t = tid % QQ;
  const int exl = el % TX, eyl = el / TX;
  const int ex = bx * TX + exl, ey = by * TY + eyl;
  const bool evalid = ex < br.n_span[0] && ey < br.n_span[1];

  const int cz = br.te[2];  // element layers per brick (<= CZ): fewer for small patches
  const long long slot_base = b * (long long)cz * NE;
  const int nlayers = min(cz, br.n_span[2] - bz * cz);
  constexpr unsigned TILE_BYTES = NE * NG * NQE * sizeof(T);
  if constexpr (MODE == MODE_APPLY) {
    if (tid == 0) prefetch_l2(A.geo + (size_t)slot_base * NG * NQE, TILE_BYTES);
  }

  // x / y tables and footprint offsets of this brick's elements
  for (int i = tid; i < TX * 2 * Q * P1; i += NT) {
    int e = i / (2 * Q * P1), r = i % (2 * Q * P1);
    int sp = min(bx * TX + e, br.n_span[0] - 1);
    stx[i] = A.tab[0][(size_t)sp * 3 * Q * P1 + r];
  }
  for (int i = tid; i < TY * 2 * Q * P1; i += NT) {
    int e = i / (2 * Q * P1), r = i % (2 * Q * P1);
    int sp = min(by * TY + e, br.n_span[1] - 1);
    sty[i] = A.tab[1][(size_t)sp * 3 * Q * P1 + r];
  }
  if (tid < TX) {
    int e = bx * TX + tid;
    soff[tid] = e < br.n_span[0] ? br.first[0][e] - cp0x : -100000;
  }
  if (tid < TY) {
    int e = by * TY + tid;
    soff[TX + tid] = e < br.n_span[1] ? br.first[1][e] - cp0y : -100000;
  }
  const int accn = VEC * fp0 * fp1 * fp2;
  for (int i = tid; i < accn; i += NT) acc[i] = T(0);

  const T* nx_v = stx + exl * 2 * Q * P1;  // [2][Q][P1] of this element
  const T* ny_v = sty + eyl * 2 * Q * P1;
  const long long nxy = (long long)br.n_cp[0] * br.n_cp[1];

  for (int lz = 0; lz < nlayers; ++lz) {
    const int ez = bz * cz + lz;
    const int fz = br.first[2][ez];
    const int offz = fz - cp0z;
    const long long slot = slot_base + (long long)lz * NE + el;
    if constexpr (MODE == MODE_APPLY) {
      // one layer ahead: 296 resident CTAs x one tile stays well inside L2
      if (tid == 0 && lz + 1 < nlayers)
        prefetch_l2(A.geo + (size_t)(slot_base + (long long)(lz + 1) * NE) * NG * NQE, TILE_BYTES);
    }
    for (int i = tid; i < 2 * Q * P1; i += NT) stz[i] = A.tab[2][(size_t)ez * 3 * Q * P1 + i];
    if constexpr (MODE == MODE_APPLY) {
      // input tile of the layer: control points [cp0x, +fp0) x [cp0y, +fp1) x [fz, +P1), coalesced
      const int rowlen = fp0 * VEC;
      for (int i = tid; i < sun; i += NT) {
        const int r = i % rowlen, rest = i / rowlen;
        const int jy = rest % fp1, jz = rest / fp1;
        const int jx = r / VEC;
        const int gx = cp0x + jx, gy = cp0y + jy;
        T v = T(0);
        if (gx < br.n_cp[0] && gy < br.n_cp[1]) {
          const long long cp = gx + (long long)br.n_cp[0] * gy + nxy * (fz + jz);
          const long long dof = cp * VEC + (r - jx * VEC);
          v = A.x[dof];
          if (A.masked && !A.keep[dof]) v = T(0);
          if constexpr (RAT) v *= A.wgts[cp];
        }
        su[i] = v;
      }
    }
    __syncthreads();

    const int fx = evalid ? br.first[0][ex] : 0, fy = evalid ? br.first[1][ey] : 0;
    const int ox = evalid ? fx - cp0x : 0, oy = evalid ? fy - cp0y : 0;

    // flux registers: [VEC][channel][q2], channels (gx, gy, gz[, v])
    T g[VEC][HASV ? 4 : 3][Q];

    if constexpr (MODE == MODE_APPLY) {
      // ---------------- forward contractions, one component at a time -------
#pragma unroll
      for (int c = 0; c < VEC; ++c) {
        if (evalid && t < PP) {  // stage X: line along x at (i1, i2)
          const int i1 = t % P1, i2 = t / P1;
          const T* line = su + ((i2 * fp1 + oy + i1) * fp0 + ox) * VEC + c;
          T u[P1];
#pragma unroll
          for (int i0 = 0; i0 < P1; ++i0) u[i0] = line[i0 * VEC];
          T* dst = bufX + el * 2 * Q * SX;
#pragma unroll
          for (int q0 = 0; q0 < Q; ++q0) {
            T sv = 0, sd = 0;
#pragma unroll
            for (int i0 = 0; i0 < P1; ++i0) {
              sv += nx_v[q0 * P1 + i0] * u[i0];
              sd += nx_v[(Q + q0) * P1 + i0] * u[i0];
            }
            dst[q0 * SX + t] = sv;
            dst[(Q + q0) * SX + t] = sd;
          }
        }
        __syncthreads();
        if (evalid && t < Q * P1) {  // stage Y: (q0, i2), line along y
          const int q0 = t % Q, i2 = t / Q;
          const T* src = bufX + el * 2 * Q * SX;
          T a[P1], ad[P1];
#pragma unroll
          for (int i1 = 0; i1 < P1; ++i1) {
            a[i1] = src[q0 * SX + i2 * P1 + i1];
            ad[i1] = src[(Q + q0) * SX + i2 * P1 + i1];
          }
          T* dst = bufY + el * 3 * SYC;
#pragma unroll
          for (int q1 = 0; q1 < Q; ++q1) {
            T vv = 0, vd = 0, dv = 0;
#pragma unroll
            for (int i1 = 0; i1 < P1; ++i1) {
              vv += ny_v[q1 * P1 + i1] * a[i1];
              vd += ny_v[(Q + q1) * P1 + i1] * a[i1];
              dv += ny_v[q1 * P1 + i1] * ad[i1];
            }
            const int o = q1 * SY1 + i2 * Q + q0;
            dst[o] = vv;
            dst[SYC + o] = vd;
            dst[2 * SYC + o] = dv;
          }
        }
        __syncthreads();
        if (evalid) {  // stage Z in registers: (q0, q1)
          const int q0 = t % Q, q1 = t / Q;
          const T* src = bufY + el * 3 * SYC;
          T vv[P1], vd[P1], dv[P1];
#pragma unroll
          for (int i2 = 0; i2 < P1; ++i2) {
            const int o = q1 * SY1 + i2 * Q + q0;
            vv[i2] = src[o];
            vd[i2] = src[SYC + o];
            dv[i2] = src[2 * SYC + o];
          }
#pragma unroll
          for (int q2 = 0; q2 < Q; ++q2) {
            T gx = 0, gy = 0, gz = 0, gv = 0;
#pragma unroll
            for (int i2 = 0; i2 < P1; ++i2) {
              const T nv = stz[q2 * P1 + i2], nd = stz[(Q + q2) * P1 + i2];
              gx += nv * dv[i2];
              gy += nv * vd[i2];
              gz += nd * vv[i2];
              if constexpr (HASV) gv += nv * vv[i2];
            }
            g[c][0][q2] = gx;
            g[c][1][q2] = gy;
            g[c][2][q2] = gz;
            if constexpr (HASV) g[c][3][q2] = gv;
          }
        }
      }
      // ---------------- point operator (factors from L2 / HBM) ---------------
      if (evalid) {
        const T* G = A.geo + (size_t)slot * NG * NQE + t;
#pragma unroll
        for (int q2 = 0; q2 < Q; ++q2) {
          const int qo = QQ * q2;
          if constexpr (OPK == OPK_SCALAR) {
            if constexpr (!RAT) {
              const T k0 = __ldg(G + 0 * NQE + qo), k1 = __ldg(G + 1 * NQE + qo), k2 = __ldg(G + 2 * NQE + qo);
              const T k3 = __ldg(G + 3 * NQE + qo), k4 = __ldg(G + 4 * NQE + qo), k5 = __ldg(G + 5 * NQE + qo);
              const T gx = g[0][0][q2], gy = g[0][1][q2], gz = g[0][2][q2];
              g[0][0][q2] = k0 * gx + k1 * gy + k2 * gz;
              g[0][1][q2] = k1 * gx + k3 * gy + k4 * gz;
              g[0][2][q2] = k2 * gx + k4 * gy + k5 * gz;
            } else {
              T m[10];
#pragma unroll
              for (int k = 0; k < 10; ++k) m[k] = __ldg(G + k * NQE + qo);
              const T v = g[0][3][q2], gx = g[0][0][q2], gy = g[0][1][q2], gz = g[0][2][q2];
              g[0][3][q2] = m[0] * v + m[1] * gx + m[2] * gy + m[3] * gz;
              g[0][0][q2] = m[1] * v + m[4] * gx + m[5] * gy + m[6] * gz;
              g[0][1][q2] = m[2] * v + m[5] * gx + m[7] * gy + m[8] * gz;
              g[0][2][q2] = m[3] * v + m[6] * gx + m[8] * gy + m[9] * gz;
            }
          } else if constexpr (OPK == OPK_ELAST || OPK == OPK_HYPER) {
            T Ji[3][3];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
              for (int a = 0; a < 3; ++a) Ji[i][a] = __ldg(G + (i * 3 + a) * NQE + qo);
            const T om = __ldg(G + 9 * NQE + qo);
            T iW = 1, gW[3] = {0, 0, 0};
            if constexpr (RAT) {
              iW = __ldg(G + 10 * NQE + qo);
#pragma unroll
              for (int a = 0; a < 3; ++a) gW[a] = __ldg(G + (11 + a) * NQE + qo);
            }
            T Gx[3][3];  // du_c / dx_k
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              T gp[3];
#pragma unroll
              for (int a = 0; a < 3; ++a) {
                if constexpr (RAT)
                  gp[a] = (g[c][a][q2] - g[c][3][q2] * gW[a]) * iW;
                else
                  gp[a] = g[c][a][q2];
              }
#pragma unroll
              for (int k = 0; k < 3; ++k) Gx[c][k] = Ji[k][0] * gp[0] + Ji[k][1] * gp[1] + Ji[k][2] * gp[2];
            }
            const T tr = Gx[0][0] + Gx[1][1] + Gx[2][2];
            const T lam = (T)A.lam, mu = (T)A.mu;
            T Sh[3][3];  // hyperelastic: om dP at the stored state
            if constexpr (OPK == OPK_HYPER) {
              T M[3][3];
#pragma unroll
              for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int k = 0; k < 3; ++k) M[i][k] = __ldg(G + (E0 + i * 3 + k) * NQE + qo);
              hyper_dP<T, 3>(M, __ldg(G + (E0 + 9) * NQE + qo), lam, mu, om, Gx, Sh);
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              T Sr[3];
#pragma unroll
              for (int k = 0; k < 3; ++k)
                Sr[k] = OPK == OPK_HYPER ? Sh[c][k] : om * (mu * (Gx[c][k] + Gx[k][c]) + (c == k ? lam * tr : T(0)));
              T F[3];
#pragma unroll
              for (int a = 0; a < 3; ++a) F[a] = Sr[0] * Ji[0][a] + Sr[1] * Ji[1][a] + Sr[2] * Ji[2][a];
              if constexpr (RAT) {
                g[c][3][q2] = -(F[0] * gW[0] + F[1] * gW[1] + F[2] * gW[2]) * iW;
#pragma unroll
                for (int a = 0; a < 3; ++a) g[c][a][q2] = F[a] * iW;
              } else {
#pragma unroll
                for (int a = 0; a < 3; ++a) g[c][a][q2] = F[a];
              }
            }
          }
        }
      }
    } else if constexpr (MODE == MODE_LOAD) {
      if (evalid) {
        const long long eref = ex + (long long)br.n_span[0] * (ey + (long long)br.n_span[1] * ez);
#pragma unroll
        for (int q2 = 0; q2 < Q; ++q2) {
          const int q = t + QQ * q2;
          const double w = A.wq[slot * NQE + q];
#pragma unroll
          for (int c = 0; c < VEC; ++c) {
            g[c][0][q2] = g[c][1][q2] = g[c][2][q2] = T(0);
            g[c][HASV ? 3 : 0][q2] = (T)(w * A.f_qp[(eref * NQE + q) * VEC + c]);
          }
        }
      }
    } else if constexpr (MODE == MODE_RESID) {  // hyperelastic: the stored flux w P J^-T
      if (evalid) {
        const T* G = A.geo + (size_t)slot * NG * NQE + t;
#pragma unroll
        for (int q2 = 0; q2 < Q; ++q2) {
          const int qo = QQ * q2;
          T iW = 1, gW[3] = {0, 0, 0};
          if constexpr (RAT) {
            iW = G[10 * NQE + qo];
#pragma unroll
            for (int a = 0; a < 3; ++a) gW[a] = G[(11 + a) * NQE + qo];
          }
#pragma unroll
          for (int c = 0; c < VEC; ++c) {
            T F[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) F[a] = G[(E0 + 10 + c * 3 + a) * NQE + qo];
            if constexpr (RAT) {
              g[c][3][q2] = -(F[0] * gW[0] + F[1] * gW[1] + F[2] * gW[2]) * iW;
#pragma unroll
              for (int a = 0; a < 3; ++a) g[c][a][q2] = F[a] * iW;
            } else {
#pragma unroll
              for (int a = 0; a < 3; ++a) g[c][a][q2] = F[a];
            }
          }
        }
      }
    }

    if constexpr (MODE == MODE_APPLY || MODE == MODE_LOAD || MODE == MODE_RESID) {
      // ---------------- backward contractions, one component at a time ------
#pragma unroll
      for (int c = 0; c < VEC; ++c) {
        if (evalid) {  // Z^T in registers: (q0, q1) -> bufY
          const int q0 = t % Q, q1 = t / Q;
          T* dst = bufY + el * 3 * SYC;
#pragma unroll
          for (int i2 = 0; i2 < P1; ++i2) {
            T vv = 0, vd = 0, dv = 0;
#pragma unroll
            for (int q2 = 0; q2 < Q; ++q2) {
              const T nv = stz[q2 * P1 + i2], nd = stz[(Q + q2) * P1 + i2];
              vv += nd * g[c][2][q2];
              if constexpr (HASV) vv += nv * g[c][3][q2];
              vd += nv * g[c][1][q2];
              dv += nv * g[c][0][q2];
            }
            const int o = q1 * SY1 + i2 * Q + q0;
            dst[o] = vv;
            dst[SYC + o] = vd;
            dst[2 * SYC + o] = dv;
          }
        }
        __syncthreads();
        if (evalid && t < Q * P1) {  // Y^T: (q0, i2) -> bufX
          const int q0 = t % Q, i2 = t / Q;
          const T* src = bufY + el * 3 * SYC;
          T vv[Q], vd[Q], dv[Q];
#pragma unroll
          for (int q1 = 0; q1 < Q; ++q1) {
            const int o = q1 * SY1 + i2 * Q + q0;
            vv[q1] = src[o];
            vd[q1] = src[SYC + o];
            dv[q1] = src[2 * SYC + o];
          }
          T* dst = bufX + el * 2 * Q * SX;
#pragma unroll
          for (int i1 = 0; i1 < P1; ++i1) {
            T a = 0, ad = 0;
#pragma unroll
            for (int q1 = 0; q1 < Q; ++q1) {
              a += ny_v[q1 * P1 + i1] * vv[q1] + ny_v[(Q + q1) * P1 + i1] * vd[q1];
              ad += ny_v[q1 * P1 + i1] * dv[q1];
            }
            dst[q0 * SX + i2 * P1 + i1] = a;
            dst[(Q + q0) * SX + i2 * P1 + i1] = ad;
          }
        }
        __syncthreads();
        if (evalid && t < PP) {  // X^T: (i1, i2) -> stage line
          const T* src = bufX + el * 2 * Q * SX;
          T a[Q], ad[Q];
#pragma unroll
          for (int q0 = 0; q0 < Q; ++q0) {
            a[q0] = src[q0 * SX + t];
            ad[q0] = src[(Q + q0) * SX + t];
          }
          T* dst = stage + (el * VEC + c) * SST + t * SP;
#pragma unroll
          for (int i0 = 0; i0 < P1; ++i0) {
            T r = 0;
#pragma unroll
            for (int q0 = 0; q0 < Q; ++q0) r += nx_v[q0 * P1 + i0] * a[q0] + nx_v[(Q + q0) * P1 + i0] * ad[q0];
            if constexpr (RAT) {
              const int i1 = t % P1, i2 = t / P1;
              const long long cp = (long long)br.n_cp[0] * ((fy + i1) + (long long)br.n_cp[1] * (fz + i2)) + fx + i0;
              r *= A.wgts[cp];
            }
            dst[i0] = r;
          }
        }
      }
    } else {  // MODE_DIAG: direct local diagonal, no sum factorisation
      if (evalid) {
        for (int a = t; a < PPP; a += QQ) {
          const int a0 = a % P1, a1 = (a / P1) % P1, a2 = a / PP;
          T d[VEC];
#pragma unroll
          for (int c = 0; c < VEC; ++c) d[c] = 0;
          for (int q = 0; q < NQE; ++q) {
            const int q0 = q % Q, q1 = (q / Q) % Q, q2 = q / QQ;
            const T vx = nx_v[q0 * P1 + a0], dx = nx_v[(Q + q0) * P1 + a0];
            const T vy = ny_v[q1 * P1 + a1], dy = ny_v[(Q + q1) * P1 + a1];
            const T vz = stz[q2 * P1 + a2], dz = stz[(Q + q2) * P1 + a2];
            const T ph[4] = {dx * vy * vz, vx * dy * vz, vx * vy * dz, vx * vy * vz};
            const T* G = A.geo + (size_t)slot * NG * NQE + q;
            if constexpr (OPK == OPK_SCALAR) {
              if constexpr (!RAT) {
                const T k0 = G[0], k1 = G[NQE], k2 = G[2 * NQE], k3 = G[3 * NQE], k4 = G[4 * NQE], k5 = G[5 * NQE];
                d[0] += k0 * ph[0] * ph[0] + k3 * ph[1] * ph[1] + k5 * ph[2] * ph[2] +
                        T(2) * (k1 * ph[0] * ph[1] + k2 * ph[0] * ph[2] + k4 * ph[1] * ph[2]);
              } else {
                const T s4[4] = {ph[3], ph[0], ph[1], ph[2]};
                int k = 0;
                T acc_ = 0;
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                  for (int j = i; j < 4; ++j) {
                    const T m = G[(k++) * NQE];
                    acc_ += (i == j ? T(1) : T(2)) * m * s4[i] * s4[j];
                  }
                d[0] += acc_;
              }
            } else {
              T Ji[3][3];
#pragma unroll
              for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int b2 = 0; b2 < 3; ++b2) Ji[i][b2] = G[(i * 3 + b2) * NQE];
              const T om = G[9 * NQE];
              T gp[3] = {ph[0], ph[1], ph[2]};
              if constexpr (RAT) {
                const T iW = G[10 * NQE];
#pragma unroll
                for (int b2 = 0; b2 < 3; ++b2) gp[b2] = (gp[b2] - ph[3] * G[(11 + b2) * NQE]) * iW;
              }
              T gx[3];
#pragma unroll
              for (int k = 0; k < 3; ++k) gx[k] = Ji[k][0] * gp[0] + Ji[k][1] * gp[1] + Ji[k][2] * gp[2];
              const T n2 = gx[0] * gx[0] + gx[1] * gx[1] + gx[2] * gx[2];
              if constexpr (OPK == OPK_HYPER) {
                // mu |g|^2 + (c + lambda) (F^-T_c . g)^2 at the stored state
                const T ch = G[(E0 + 9) * NQE] + (T)A.lam;
#pragma unroll
                for (int c = 0; c < VEC; ++c) {
                  const T mg = G[(E0 + c * 3) * NQE] * gx[0] + G[(E0 + c * 3 + 1) * NQE] * gx[1] +
                               G[(E0 + c * 3 + 2) * NQE] * gx[2];
                  d[c] += om * ((T)A.mu * n2 + ch * mg * mg);
                }
              } else {
#pragma unroll
                for (int c = 0; c < VEC; ++c) d[c] += om * ((T)(A.lam + A.mu) * gx[c] * gx[c] + (T)A.mu * n2);
              }
            }
          }
          T wsq = 1;
          if constexpr (RAT) {
            const long long cp = (long long)br.n_cp[0] * ((fy + a1) + (long long)br.n_cp[1] * (fz + a2)) + fx + a0;
            wsq = A.wgts[cp] * A.wgts[cp];
          }
#pragma unroll
          for (int c = 0; c < VEC; ++c) stage[(el * VEC + c) * SST + (a1 + P1 * a2) * SP + a0] = d[c] * wsq;
        }
      }
    }
    __syncthreads();
    // ---------------- deterministic gather of the layer into the brick ------
    {
      const int nfoot = VEC * fp0 * fp1 * P1;
      for (int i = tid; i < nfoot; i += NT) {
        const int jx = i % fp0;
        const int jy = (i / fp0) % fp1;
        const int jzl = (i / (fp0 * fp1)) % P1;
        const int c = i / (fp0 * fp1 * P1);
        T s = 0;
#pragma unroll
        for (int e1 = 0; e1 < TY; ++e1) {
          const int ly = jy - soff[TX + e1];
          if (ly < 0 || ly > P) continue;
#pragma unroll
          for (int e0 = 0; e0 < TX; ++e0) {
            const int lx = jx - soff[e0];
            if (lx < 0 || lx > P) continue;
            s += stage[((e1 * TX + e0) * VEC + c) * SST + (ly + P1 * jzl) * SP + lx];
          }
        }
        acc[((c * fp2 + offz + jzl) * fp1 + jy) * fp0 + jx] += s;
      }
    }
    // the next layer's first barrier orders these accumulator updates
  }
  __syncthreads();
  // write the brick footprint
  T* out = A.scratch + (size_t)b * accn;
  for (int i = tid; i < accn; i += NT) out[i] = acc[i];
}

#include "brick2d.cuh"
#include "brick3_mma.cuh"
#include "brick3_rf.cuh"

// The FP64 tensor-core brick kernels run the degree-3 scalar and elasticity
// applies. The environment variable JXB_BRICK3_MMA selects the variant, to
// compare them: 0 = the FMA kernel, 1 = the staged MMA kernel (stage hand-offs
// through shared memory) built for one CTA per SM, 2 = the staged kernel at
// its default occupancy (scalar: two CTAs per SM; elasticity: one), 3 = the
// register-fragment kernel built for one CTA per SM, 4 = the register-fragment
// kernel at its default occupancy (scalar: two CTAs per SM; elasticity: one)
// reading the factors from L2, 5 = the same kernel with the factor tiles copied
// into shared memory one element ahead. The default is 4 for the scalar
// operator and 5 for elasticity, the faster of the two on each (B200: Darcy
// 96^3 0.69 / 0.71 ms, elasticity 64^3 0.635 / 0.629 ms).
template <int OPK>
static int brick3_mma_mode() {
  static const int mode = [] {
    const char* e = getenv("JXB_BRICK3_MMA");
    if (e && e[0] >= '0' && e[0] <= '5' && e[1] == 0) return e[0] - '0';
    return OPK == OPK_ELAST ? 5 : 4;
  }();
  return mode;
}

// ---------------------------------------------------------------------------
// combine: y_i = sum over covering bricks (fixed order); optional p.y partials
// ---------------------------------------------------------------------------
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double warp_part[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) warp_part[w] = v;
  __syncthreads();
  double s = 0;
  if (threadIdx.x == 0) {
    int nw = (blockDim.x + 31) >> 5;
    for (int i = 0; i < nw; ++i) s += warp_part[i];
  }
  return s;  // valid in thread 0
}

// One thread per control point, every component; the grid-stride mapping of
// control points to threads is the same in both launch shapes. With `partials`
// the grid is the fixed JXB_RED_BLOCKS of the deterministic reductions (the
// per-block p.y partials); without, it covers every control point once.
template <typename T, int VEC, int DIM>
__global__ void __launch_bounds__(JXB_RED_THREADS)
    k_combine(Bricks br, const T* __restrict__ scratch, const uint8_t* __restrict__ keep, int masked,
              T* __restrict__ y, const T* __restrict__ dot_with, double* __restrict__ partials,
              const CgState* state) {
  if (state && state->done) return;
  const long long n_scalar = (long long)br.n_cp[0] * br.n_cp[1] * (DIM == 3 ? br.n_cp[2] : 1);
  double part = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_scalar;
       i += (long long)gridDim.x * blockDim.x) {
    // n_scalar < 2^31 (checked by the launcher): 32-bit index arithmetic
    const unsigned ii = (unsigned)i, n0 = (unsigned)br.n_cp[0], n1 = (unsigned)br.n_cp[1];
    const unsigned ix = ii % n0, iyz = ii / n0;
    const unsigned iy = iyz % n1, iz = DIM == 3 ? iyz / n1 : 0;
    T s[VEC];
    combine_point<T, VEC, DIM>(br, scratch, (int)ix, (int)iy, (int)iz, s);
#pragma unroll
    for (int c = 0; c < VEC; ++c) {
      const long long dof = i * VEC + c;
      T v = s[c];
      if (masked && !keep[dof]) v = T(0);
      y[dof] = v;
      if (dot_with) part += (double)dot_with[dof] * (double)v;
    }
  }
  if (partials) {
    double bs = block_sum(part);
    if (threadIdx.x == 0) partials[blockIdx.x] = bs;
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <typename T, int P, int Q, int OPK, bool RAT, int MODE>
static size_t smem3(const Bricks& br) {
  using S = Strides3<P, Q>;
  constexpr int P1 = P + 1;
  constexpr int TX = BrickShape<3, P>::TX, TY = BrickShape<3, P>::TY;
  constexpr int NE = TX * TY;
  constexpr int VEC = vec_op<OPK>() ? 3 : 1;
  size_t n = (size_t)(TX + TY + 1) * 2 * Q * P1 + (size_t)NE * 2 * Q * S::SX + (size_t)NE * 3 * S::SYC +
             (size_t)NE * VEC * S::SST + (size_t)VEC * br.fp[0] * br.fp[1] * br.fp[2] +
             (MODE == MODE_APPLY ? (size_t)P1 * br.fp[0] * br.fp[1] * VEC : 0);
  return n * sizeof(T) + (TX + TY) * sizeof(int) + 64;
}

int tile2_variant(int tx, int ty) {
  if (ty < 1 || ty > TILE2_MAX_ROWS) return -1;
  for (int v = 0; v < N_TILE2; ++v)
    if (TILE2X[v] == tx) return v;
  return -1;
}

template <typename T, int P, int Q, int OPK, bool RAT, int MODE>
static size_t smem2(const Bricks& br, const int TX, const int RG = 1) {
  constexpr int P1 = P + 1, PP = P1 * P1;
  constexpr int VEC = vec_op<OPK>() ? 2 : 1;
  constexpr int NK = OPK == OPK_PLATE ? 3 : 2;
  constexpr int SX = P1 + 1;
  const size_t group = 3 * Q * P1 + (size_t)TX * NK * Q * SX + TX * VEC * PP + (size_t)VEC * br.fp[0] * br.fp[1];
  size_t n = (size_t)TX * 3 * Q * P1 + RG * group;
  return n * sizeof(T) + TX * sizeof(int) + 64;
}

// Row groups of the 2D brick kernels: 2 when the brick has two rows or more and
// the doubled stage buffers fit in shared memory, else 1.
constexpr int RG2 = 2;
static int brick2_rg(size_t smem_rg2, int rows) { return rows >= 2 && smem_rg2 <= 227 * 1024 ? RG2 : 1; }

template <typename T, int P, int OPK, bool RAT, int MODE>
static int launch_one(const BrickArgs<T>& A, cudaStream_t s) {
  constexpr int Q = P + 1;
  const Bricks& br = A.br;
  if (br.dim == 3) {
    if constexpr (OPK == OPK_PLATE) {
      return fail(JXB_ERR_INVALID, "plate operator is 2D only");
    } else {
      if constexpr (sizeof(T) == 8 && P == 3 && (OPK == OPK_SCALAR || OPK == OPK_ELAST) && !RAT &&
                    MODE == MODE_APPLY) {
        int mode = brick3_mma_mode<OPK>();
        // a brick whose footprint leaves no room for the factor tiles reads them from L2
        if (mode == 5 && smem3_rf<OPK, true>(br) > 227 * 1024) mode = 4;
        if (mode >= 3) {
          const size_t sm = mode == 5 ? smem3_rf<OPK, true>(br) : smem3_rf<OPK, false>(br);
          if (sm > 227 * 1024) return fail(JXB_ERR_INVALID, "3D brick does not fit in shared memory");
          constexpr int MB = OPK == OPK_SCALAR ? 2 : 1;
          auto k = mode == 5 ? k_brick3_rf<OPK, MB, true> : mode == 4 ? k_brick3_rf<OPK, MB, false>
                                                                       : k_brick3_rf<OPK, 1, false>;
          JXB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
          k<<<(unsigned)br.n_bricks, brf::NT, sm, s>>>(A);
          JXB_CUDA(cudaGetLastError());
          return JXB_OK;
        }
        if (mode) {
          const size_t sm = smem3_mma<OPK>(br);
          if (sm > 227 * 1024) return fail(JXB_ERR_INVALID, "3D brick does not fit in shared memory");
          // elasticity needs the registers of the one-CTA-per-SM build
          auto k = k_brick3_mma<OPK, 1>;
          if constexpr (OPK == OPK_SCALAR) {
            if (mode == 2) k = k_brick3_mma<OPK, 2>;
          }
          JXB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
          k<<<(unsigned)br.n_bricks, bm::NT, sm, s>>>(A);
          JXB_CUDA(cudaGetLastError());
          return JXB_OK;
        }
      }
      constexpr int NT = BrickShape<3, P>::TX * BrickShape<3, P>::TY * Q * Q;
      size_t sm = smem3<T, P, Q, OPK, RAT, MODE>(br);
      if (sm > 227 * 1024) return fail(JXB_ERR_INVALID, "3D brick does not fit in shared memory for this degree/operator");
      auto k = k_brick3<T, P, Q, OPK, RAT, MODE>;
      if (sm > 48 * 1024) JXB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      k<<<(unsigned)br.n_bricks, NT, sm, s>>>(A);
    }
  } else {
    const int v = tile2_variant(br.te[0], br.te[1]);
    if (v < 0) return fail(JXB_ERR_INVALID, "unsupported 2D brick shape");
    if constexpr (OPK != OPK_SCALAR) {
      if (v != 0) return fail(JXB_ERR_INVALID, "tile variants are available for the 2D scalar operator only");
    }
#define JXB_TILE2(V_)                                                                                   \
  if (v == V_) {                                                                                        \
    constexpr int TXv = TILE2X[V_];                                                                     \
    const size_t sm2 = smem2<T, P, Q, OPK, RAT, MODE>(br, TXv, RG2);                                    \
    if (brick2_rg(sm2, br.te[1]) == RG2) {                                                              \
      auto k = k_brick2<T, P, Q, OPK, RAT, MODE, TXv, RG2>;                                             \
      if (sm2 > 48 * 1024) JXB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2)); \
      k<<<(unsigned)br.n_bricks, brick2_threads(TXv, Q, RG2), sm2, s>>>(A);                             \
    } else {                                                                                            \
      size_t sm = smem2<T, P, Q, OPK, RAT, MODE>(br, TXv);                                              \
      if (sm > 227 * 1024) return fail(JXB_ERR_INVALID, "2D brick does not fit in shared memory");      \
      auto k = k_brick2<T, P, Q, OPK, RAT, MODE, TXv, 1>;                                               \
      if (sm > 48 * 1024) JXB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)); \
      k<<<(unsigned)br.n_bricks, TXv * Q, sm, s>>>(A);                                                  \
    }                                                                                                   \
  }
    JXB_TILE2(0)
    if constexpr (OPK == OPK_SCALAR) {
      JXB_TILE2(1)
      JXB_TILE2(2)
    }
#undef JXB_TILE2
  }
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

template <typename T, int MODE>
static int dispatch(jxb_plan* plan, const BrickArgs<T>& A, cudaStream_t s) {
  bool rat = plan->rational != 0;
  if (plan->op == JXB_OP_HYPERELASTIC) {  // FP64, degrees 1..4
    if constexpr (sizeof(T) == 8) {
#define JXB_HCASE(P_) \
  case P_:            \
    return rat ? launch_one<T, P_, OPK_HYPER, true, MODE>(A, s) : launch_one<T, P_, OPK_HYPER, false, MODE>(A, s);
      switch (plan->p) {
        JXB_HCASE(1)
        JXB_HCASE(2)
        JXB_HCASE(3)
        JXB_HCASE(4)
        default:
          return fail(JXB_ERR_INVALID, "the hyperelastic operator takes degrees 1..4");
      }
#undef JXB_HCASE
    } else {
      return fail(JXB_ERR_INVALID, "the hyperelastic operator has no FP32 copy");
    }
  }
  if constexpr (MODE == MODE_RESID) {
    return fail(JXB_ERR_INVALID, "the residual mode belongs to the hyperelastic operator");
  } else {
  int opk = plan->op == JXB_OP_POISSON ? OPK_SCALAR : plan->op == JXB_OP_ELASTICITY ? OPK_ELAST : OPK_PLATE;
#define JXB_CASE(P_)                                                                         \
  case P_:                                                                                  \
    if (opk == OPK_SCALAR) return rat ? launch_one<T, P_, OPK_SCALAR, true, MODE>(A, s)     \
                                      : launch_one<T, P_, OPK_SCALAR, false, MODE>(A, s);   \
    if (opk == OPK_ELAST) return rat ? launch_one<T, P_, OPK_ELAST, true, MODE>(A, s)       \
                                     : launch_one<T, P_, OPK_ELAST, false, MODE>(A, s);     \
    return rat ? launch_one<T, P_, OPK_PLATE, true, MODE>(A, s)                             \
               : launch_one<T, P_, OPK_PLATE, false, MODE>(A, s);
  switch (plan->p) {
    JXB_CASE(1)
    JXB_CASE(2)
    JXB_CASE(3)
    JXB_CASE(4)
    JXB_CASE(5)
    default:
      return fail(JXB_ERR_INVALID, "degree must be in 1..5");
  }
#undef JXB_CASE
  }
}

template <typename T>
int launch_bricks(jxb_plan* plan, cudaStream_t s, int mode, const T* x, const double* f_qp,
                  const CgState* state, int masked) {
  if (plan->mp) {  // composite multipatch plan: gather, then every patch's bricks
    if constexpr (sizeof(T) == 8)
      return mp_bricks(plan, s, mode, x, f_qp, state);
    else
      return fail(JXB_ERR_INVALID, "multipatch plans have no FP32 copy");
  }
  if (plan->thb) {  // hierarchical plan: the padded-element apply
    if constexpr (sizeof(T) == 8)
      return thb_bricks(plan, s, mode, x, f_qp, state, masked);
    else
      return fail(JXB_ERR_INVALID, "hierarchical plans have no FP32 copy");
  }
  BrickArgs<T> A;
  A.br = plan->br;
  constexpr bool F32 = sizeof(T) == 4;
  for (int d = 0; d < 3; ++d) {
    if constexpr (F32)
      A.tab[d] = plan->d_tab32[d];
    else
      A.tab[d] = plan->d_tab[d];
  }
  if constexpr (F32) {
    A.geo = plan->d_geo32;
    A.wgts = plan->d_wgts32;
    A.scratch = plan->d_scratch32;
  } else {
    A.geo = plan->d_geo;
    A.wgts = plan->d_wgts;
    A.scratch = plan->d_scratch;
  }
  A.wq = plan->d_wq;
  A.keep = plan->d_keep;
  A.x = x;
  A.f_qp = f_qp;
  A.state = state;
  A.masked = masked;
  A.err = reinterpret_cast<int*>(plan->d_red + 4 * JXB_RED_BLOCKS);
  A.lam = plan->mat.lam;
  A.mu = plan->mat.mu;
  if (mode == MODE_APPLY) return dispatch<T, MODE_APPLY>(plan, A, s);
  if constexpr (!F32) {
    if (mode == MODE_LOAD) return dispatch<T, MODE_LOAD>(plan, A, s);
    if (mode == MODE_DIAG) return dispatch<T, MODE_DIAG>(plan, A, s);
    if (mode == MODE_RESID) return dispatch<T, MODE_RESID>(plan, A, s);
  }
  return fail(JXB_ERR_INVALID, "unsupported brick mode");
}

template <typename T>
int launch_combine(jxb_plan* plan, cudaStream_t s, T* y, int masked, const T* dot_with,
                   double* partials, const CgState* state) {
  if (plan->mp) {  // composite: the fixed-order sum of the patches' copies of every DOF
    if constexpr (sizeof(T) == 8)
      return mp_combine(plan, s, y, masked, dot_with, partials, state);
    else
      return fail(JXB_ERR_INVALID, "multipatch plans have no FP32 copy");
  }
  if (plan->thb) {  // hierarchical: the fixed-order sum of the element copies of every DOF
    if constexpr (sizeof(T) == 8)
      return thb_combine(plan, s, y, masked, dot_with, partials, state);
    else
      return fail(JXB_ERR_INVALID, "hierarchical plans have no FP32 copy");
  }
  const T* scratch;
  if constexpr (sizeof(T) == 4)
    scratch = plan->d_scratch32;
  else
    scratch = plan->d_scratch;
  if (plan->n_scalar >= (1LL << 31)) return fail(JXB_ERR_INVALID, "combine: more than 2^31 control points");
  unsigned grid = JXB_RED_BLOCKS;
  if (!partials) {
    const long long g = (plan->n_scalar + JXB_RED_THREADS - 1) / JXB_RED_THREADS;
    grid = (unsigned)std::max(1LL, std::min(g, 148LL * 64));
  }
  const Bricks& br = plan->br;
#define JXB_COMBINE(V, D)                                                                                     \
  k_combine<T, V, D><<<grid, JXB_RED_THREADS, 0, s>>>(br, scratch, plan->d_keep, masked, y, dot_with, partials, \
                                                      state)
  if (br.dim == 3 && br.vec == 1)
    JXB_COMBINE(1, 3);
  else if (br.dim == 3 && br.vec == 3)
    JXB_COMBINE(3, 3);
  else if (br.dim == 2 && br.vec == 1)
    JXB_COMBINE(1, 2);
  else if (br.dim == 2 && br.vec == 2)
    JXB_COMBINE(2, 2);
  else
    return fail(JXB_ERR_INVALID, "combine: unsupported (dimension, components)");
#undef JXB_COMBINE
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

// Batched 2D scalar apply: block i runs brick work[i].y of instance work[i].x.
template <int P, bool RAT>
static int launch_batch_p(int variant, const BrickArgs<double>* d_args, const int2* d_work, long long n_work,
                          int fp0, int fp1, const CgState* d_states, cudaStream_t s) {
  constexpr int Q = P + 1;
  Bricks br{};
  br.fp[0] = fp0;
  br.fp[1] = fp1;
#define JXB_BTILE(V_)                                                                                   \
  if (variant == V_) {                                                                                  \
    constexpr int TXv = TILE2X[V_];                                                                     \
    const size_t sm2 = smem2<double, P, Q, OPK_SCALAR, RAT, MODE_APPLY>(br, TXv, RG2);                  \
    if (brick2_rg(sm2, 2) == RG2) {  /* TY is per instance: a one-row brick leaves group 1 idle */     \
      auto k = k_brick2_batch<double, P, Q, OPK_SCALAR, RAT, MODE_APPLY, TXv, RG2>;                     \
      if (sm2 > 48 * 1024) JXB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2)); \
      k<<<(unsigned)n_work, brick2_threads(TXv, Q, RG2), sm2, s>>>(d_args, d_work, d_states);          \
    } else {                                                                                            \
      size_t sm = smem2<double, P, Q, OPK_SCALAR, RAT, MODE_APPLY>(br, TXv);                            \
      if (sm > 227 * 1024) return fail(JXB_ERR_INVALID, "batched brick does not fit in shared memory"); \
      auto k = k_brick2_batch<double, P, Q, OPK_SCALAR, RAT, MODE_APPLY, TXv, 1>;                       \
      if (sm > 48 * 1024) JXB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)); \
      k<<<(unsigned)n_work, TXv * Q, sm, s>>>(d_args, d_work, d_states);                                \
    }                                                                                                   \
    JXB_CUDA(cudaGetLastError());                                                                       \
    return JXB_OK;                                                                                      \
  }
  JXB_BTILE(0)
  JXB_BTILE(1)
  JXB_BTILE(2)
#undef JXB_BTILE
  return fail(JXB_ERR_INVALID, "unknown tile variant");
}

// Shared memory of a degree-p 2D scalar apply brick with rows of tx elements
// and footprint fp0 x fp1 (runtime degree).
size_t smem2_scalar_apply(int p, bool rational, int tx, int fp0, int fp1) {
  Bricks br{};
  br.fp[0] = fp0;
  br.fp[1] = fp1;
#define JXB_SM(P_)                                                                                    \
  case P_:                                                                                            \
    return rational ? smem2<double, P_, P_ + 1, OPK_SCALAR, true, MODE_APPLY>(br, tx)                 \
                    : smem2<double, P_, P_ + 1, OPK_SCALAR, false, MODE_APPLY>(br, tx);
  switch (p) {
    JXB_SM(1)
    JXB_SM(2)
    JXB_SM(3)
    JXB_SM(4)
    JXB_SM(5)
    default:
      return 0;
  }
#undef JXB_SM
}

// The persistent batched apply (k_brick2_persist): its launch shape for a
// batch whose largest brick needs `smem` bytes, and the launch itself.
int persist2_grid(bool rational, size_t smem, int* grid) {
  auto k = rational ? k_brick2_persist<double, OPK_SCALAR, true, MODE_APPLY>
                    : k_brick2_persist<double, OPK_SCALAR, false, MODE_APPLY>;
  // the attribute is per kernel, shared by every batch: allow the largest size
  // (227 KB less the kernel's static shared memory), each launch passes its own
  cudaFuncAttributes fa;
  JXB_CUDA(cudaFuncGetAttributes(&fa, k));
  const int max_dyn = 227 * 1024 - (int)fa.sharedSizeBytes;
  if (smem > (size_t)max_dyn) return fail(JXB_ERR_INVALID, "batched brick does not fit in shared memory");
  JXB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, max_dyn));
  int dev = 0, sms = 0, per_sm = 0;
  JXB_CUDA(cudaGetDevice(&dev));
  JXB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  JXB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, PERSIST_THREADS, smem));
  *grid = std::max(1, sms * std::max(1, per_sm));
  return JXB_OK;
}

int launch_bricks2_persist(bool rational, const BrickArgs<double>* d_args, const int4* d_work, int n_work,
                           unsigned* d_next, int grid, size_t smem, const CgState* d_states, cudaStream_t s) {
  if (n_work <= 0) return JXB_OK;
  auto k = rational ? k_brick2_persist<double, OPK_SCALAR, true, MODE_APPLY>
                    : k_brick2_persist<double, OPK_SCALAR, false, MODE_APPLY>;
  k<<<(unsigned)std::min(grid, n_work), PERSIST_THREADS, smem, s>>>(d_args, d_work, n_work, d_next, d_states);
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

int launch_bricks2_batch(int p, bool rational, int variant, const BrickArgs<double>* d_args, const int2* d_work,
                         long long n_work, int fp0, int fp1, const CgState* d_states, cudaStream_t s) {
  if (n_work <= 0) return JXB_OK;
#define JXB_BP(P_) \
  case P_:         \
    return rational ? launch_batch_p<P_, true>(variant, d_args, d_work, n_work, fp0, fp1, d_states, s) \
                    : launch_batch_p<P_, false>(variant, d_args, d_work, n_work, fp0, fp1, d_states, s);
  switch (p) {
    JXB_BP(1)
    JXB_BP(2)
    JXB_BP(3)
    JXB_BP(4)
    JXB_BP(5)
    default:
      return fail(JXB_ERR_INVALID, "degree must be in 1..5");
  }
#undef JXB_BP
}

template <typename T>
BrickArgs<T> make_brick_args(jxb_plan* plan, const T* x, const CgState* state, int masked) {
  BrickArgs<T> A;
  A.br = plan->br;
  constexpr bool F32 = sizeof(T) == 4;
  for (int d = 0; d < 3; ++d) {
    if constexpr (F32)
      A.tab[d] = plan->d_tab32[d];
    else
      A.tab[d] = plan->d_tab[d];
  }
  if constexpr (F32) {
    A.geo = plan->d_geo32;
    A.wgts = plan->d_wgts32;
    A.scratch = plan->d_scratch32;
  } else {
    A.geo = plan->d_geo;
    A.wgts = plan->d_wgts;
    A.scratch = plan->d_scratch;
  }
  A.wq = plan->d_wq;
  A.keep = plan->d_keep;
  A.x = x;
  A.f_qp = nullptr;
  A.state = state;
  A.masked = masked;
  A.err = reinterpret_cast<int*>(plan->d_red + 4 * JXB_RED_BLOCKS);
  A.lam = plan->mat.lam;
  A.mu = plan->mat.mu;
  return A;
}
template BrickArgs<double> make_brick_args<double>(jxb_plan*, const double*, const CgState*, int);

template int launch_bricks<double>(jxb_plan*, cudaStream_t, int, const double*, const double*,
                                   const CgState*, int);
template int launch_bricks<float>(jxb_plan*, cudaStream_t, int, const float*, const double*,
                                  const CgState*, int);
template int launch_combine<double>(jxb_plan*, cudaStream_t, double*, int, const double*, double*,
                                    const CgState*);
template int launch_combine<float>(jxb_plan*, cudaStream_t, float*, int, const float*, double*,
                                   const CgState*);

}  // namespace jxb
