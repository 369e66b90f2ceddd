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
// Per-point factors for a layer are one contiguous tile in HBM; they are
// streamed into shared memory with cp.async.bulk (TMA, 1D) while the previous
// layer's gather runs.
#include <math.h>

#include "jxb_internal.cuh"

namespace jxb {

enum OpKind { OPK_SCALAR = 0, OPK_ELAST = 1, OPK_PLATE = 2 };

// ---------------------------------------------------------------------------
// compile-time shapes
// ---------------------------------------------------------------------------
template <int DIM, int P>
struct BrickShape;
template <int P>
struct BrickShape<3, P> {
  static constexpr int TX = P <= 4 ? 4 : 3;
  static constexpr int TY = TX;
  static constexpr int CZ = 8;
};
template <int P>
struct BrickShape<2, P> {
  static constexpr int TX = 32;
  static constexpr int TY = 8;  // element rows per brick
  static constexpr int CZ = 1;
};

template <int OPK, bool RAT, int DIM>
struct GeoCount {
  static constexpr int value =
      OPK == OPK_SCALAR ? (RAT ? (DIM + 1) * (DIM + 2) / 2 : DIM * (DIM + 1) / 2)
      : OPK == OPK_ELAST ? (DIM * DIM + 1 + (RAT ? DIM + 1 : 0))
                         : (RAT ? 21 : 15);
};

int host_geo_count(int op, int rational, int dim) {
  if (op == JXB_OP_POISSON) return rational ? (dim + 1) * (dim + 2) / 2 : dim * (dim + 1) / 2;
  if (op == JXB_OP_ELASTICITY) return dim * dim + 1 + (rational ? dim + 1 : 0);
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

// ---------------------------------------------------------------------------
// bulk asynchronous copy (TMA, non-tensor form) into shared memory
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes,
                                              unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
// Bounded wait on the phase; returns false if the copy did not land in time.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned phase) {
  unsigned ok = 0;
  for (long long spin = 0; spin < (1ll << 26); ++spin) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(phase)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// ---------------------------------------------------------------------------
// kernel arguments
// ---------------------------------------------------------------------------
template <typename T>
struct BrickArgs {
  Bricks br;
  const T* tab[3];
  const T* geo;          // (slots, ngeo, nqe)
  const double* wq;      // load weights (slots, nqe)
  const T* wgts;         // NURBS weights (rational)
  const uint8_t* keep;   // (n_dofs) 1 = free
  const T* x;            // input DOF vector
  const double* f_qp;    // load: source values, reference order
  T* scratch;            // (n_bricks, vec, fp2, fp1, fp0)
  const CgState* state;  // optional: skip all work once done
  int masked;
  int* err;              // set when a bulk copy wait gives up
  double lam, mu;
};

// ---------------------------------------------------------------------------
// 3D brick kernel
// ---------------------------------------------------------------------------
template <typename T, int P, int Q, int OPK, bool RAT, int MODE>
__global__ void __launch_bounds__(BrickShape<3, P>::TX* BrickShape<3, P>::TY* Q* Q)
    k_brick3(BrickArgs<T> A) {
  constexpr int P1 = P + 1, PP = P1 * P1, PPP = PP * P1;
  constexpr int TX = BrickShape<3, P>::TX, TY = BrickShape<3, P>::TY, CZ = BrickShape<3, P>::CZ;
  constexpr int NE = TX * TY, QQ = Q * Q, NQE = Q * Q * Q, NT = NE * QQ;
  constexpr int VEC = OPK == OPK_ELAST ? 3 : 1;
  constexpr int NG = GeoCount<OPK, RAT, 3>::value;
  constexpr bool HASV = RAT || MODE == MODE_LOAD;  // value channel
  constexpr int SX = PP + 1;                       // padded q0 stride of bufX
  constexpr int SY1 = Q * P1 + 1;                  // padded q1 stride of bufY
  constexpr int SYC = Q * SY1;                     // channel stride of bufY
  constexpr int FX = TX + P * TX, FY = TY + P * TY;  // generous upper bounds (checked on host)
  (void)FX;
  (void)FY;

  if (A.state && A.state->done) return;
  const Bricks& br = A.br;
  const int fp0 = br.fp[0], fp1 = br.fp[1], fp2 = br.fp[2];

  extern __shared__ __align__(128) unsigned char smem_raw[];
  // layout: [geo tile][tabs x][tabs y][tab z][bufX][bufY][stage][acc][ints]
  T* sgeo = reinterpret_cast<T*>(smem_raw);
  constexpr int GEO_TILE = MODE == MODE_APPLY ? NE * NG * NQE : 0;
  T* stx = sgeo + GEO_TILE;                 // [TX][2][Q][P1]
  T* sty = stx + TX * 2 * Q * P1;           // [TY][2][Q][P1]
  T* stz = sty + TY * 2 * Q * P1;           // [2][Q][P1]
  T* bufX = stz + 2 * Q * P1;               // [NE][2][Q][SX]
  T* bufY = bufX + NE * 2 * Q * SX;         // [NE][3][SYC]
  T* stage = bufY + NE * 3 * SYC;           // [NE][VEC][PPP]
  T* acc = stage + NE * VEC * PPP;          // [VEC][fp2][fp1][fp0]
  int* soff = reinterpret_cast<int*>(acc + VEC * fp0 * fp1 * fp2);  // offx[TX], offy[TY]
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(
      (reinterpret_cast<uintptr_t>(soff + TX + TY) + 15) & ~uintptr_t(15));

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

  const long long slot_base = b * (long long)CZ * NE;
  const int nlayers = min(CZ, br.n_span[2] - bz * CZ);
  if constexpr (MODE == MODE_APPLY) {
    if (tid == 0) {
      mbar_init(bar, 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
  }
  __syncthreads();
  if constexpr (MODE == MODE_APPLY) {
    if (tid == 0) {  // first layer's factor tile
      const unsigned bytes = NE * NG * NQE * sizeof(T);
      mbar_expect_tx(bar, bytes);
      bulk_copy_g2s(sgeo, A.geo + (size_t)slot_base * NG * NQE, bytes, bar);
    }
  }

  const T* nx_v = stx + exl * 2 * Q * P1;  // [2][Q][P1] of this element
  const T* ny_v = sty + eyl * 2 * Q * P1;

  for (int lz = 0; lz < nlayers; ++lz) {
    const int ez = bz * CZ + lz;
    const int fz = br.first[2][ez];
    const int offz = fz - cp0z;
    for (int i = tid; i < 2 * Q * P1; i += NT) stz[i] = A.tab[2][(size_t)ez * 3 * Q * P1 + i];
    __syncthreads();

    const long long slot = slot_base + (long long)lz * NE + el;
    const int fx = evalid ? br.first[0][ex] : 0, fy = evalid ? br.first[1][ey] : 0;

    // flux registers: [VEC][channel][q2], channels (gx, gy, gz[, v])
    T g[VEC][HASV ? 4 : 3][Q];

    if constexpr (MODE == MODE_APPLY) {
      // ---------------- forward contractions, one component at a time -------
#pragma unroll
      for (int c = 0; c < VEC; ++c) {
        if (evalid && t < PP) {  // stage X: line along x at (i1, i2)
          const int i1 = t % P1, i2 = t / P1;
          const long long row =
              (long long)br.n_cp[0] * ((fy + i1) + (long long)br.n_cp[1] * (fz + i2)) + fx;
          T u[P1];
#pragma unroll
          for (int i0 = 0; i0 < P1; ++i0) {
            long long cp = row + i0;
            T v = A.x[cp * VEC + c];
            if (A.masked) v = A.keep[cp * VEC + c] ? v : T(0);
            if constexpr (RAT) v *= A.wgts[cp];
            u[i0] = v;
          }
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
            int o = q1 * SY1 + i2 * Q + q0;
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
            int o = q1 * SY1 + i2 * Q + q0;
            vv[i2] = src[o];
            vd[i2] = src[SYC + o];
            dv[i2] = src[2 * SYC + o];
          }
#pragma unroll
          for (int q2 = 0; q2 < Q; ++q2) {
            T gx = 0, gy = 0, gz = 0, gv = 0;
#pragma unroll
            for (int i2 = 0; i2 < P1; ++i2) {
              T nv = stz[q2 * P1 + i2], nd = stz[(Q + q2) * P1 + i2];
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
      // ---------------- point operator ------------------------------------
      if (!mbar_wait(bar, lz & 1)) {
        if (tid == 0) atomicExch(A.err, 1);
      }
      if (evalid) {
        const int q01 = t;
        const T* G = sgeo + el * NG * NQE;
#pragma unroll
        for (int q2 = 0; q2 < Q; ++q2) {
          const int q = q01 + QQ * q2;
          if constexpr (OPK == OPK_SCALAR) {
            if constexpr (!RAT) {
              T k0 = G[0 * NQE + q], k1 = G[1 * NQE + q], k2 = G[2 * NQE + q];
              T k3 = G[3 * NQE + q], k4 = G[4 * NQE + q], k5 = G[5 * NQE + q];
              T gx = g[0][0][q2], gy = g[0][1][q2], gz = g[0][2][q2];
              g[0][0][q2] = k0 * gx + k1 * gy + k2 * gz;
              g[0][1][q2] = k1 * gx + k3 * gy + k4 * gz;
              g[0][2][q2] = k2 * gx + k4 * gy + k5 * gz;
            } else {
              T m[10];
#pragma unroll
              for (int k = 0; k < 10; ++k) m[k] = G[k * NQE + q];
              T v = g[0][3][q2], gx = g[0][0][q2], gy = g[0][1][q2], gz = g[0][2][q2];
              g[0][3][q2] = m[0] * v + m[1] * gx + m[2] * gy + m[3] * gz;
              g[0][0][q2] = m[1] * v + m[4] * gx + m[5] * gy + m[6] * gz;
              g[0][1][q2] = m[2] * v + m[5] * gx + m[7] * gy + m[8] * gz;
              g[0][2][q2] = m[3] * v + m[6] * gx + m[8] * gy + m[9] * gz;
            }
          } else if constexpr (OPK == OPK_ELAST) {
            T Ji[3][3];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
              for (int a = 0; a < 3; ++a) Ji[i][a] = G[(i * 3 + a) * NQE + q];
            T om = G[9 * NQE + q];
            T gp[3][3];
            T iW = 1, gW[3] = {0, 0, 0};
            if constexpr (RAT) {
              iW = G[10 * NQE + q];
#pragma unroll
              for (int a = 0; a < 3; ++a) gW[a] = G[(11 + a) * NQE + q];
            }
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
              for (int a = 0; a < 3; ++a) {
                if constexpr (RAT)
                  gp[c][a] = (g[c][a][q2] - g[c][3][q2] * gW[a]) * iW;
                else
                  gp[c][a] = g[c][a][q2];
              }
            T Gx[3][3];  // du_c / dx_k
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
              for (int k = 0; k < 3; ++k) Gx[c][k] = Ji[k][0] * gp[c][0] + Ji[k][1] * gp[c][1] + Ji[k][2] * gp[c][2];
            T tr = Gx[0][0] + Gx[1][1] + Gx[2][2];
            T lam = (T)A.lam, mu = (T)A.mu;
            T S[3][3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
              for (int k = 0; k < 3; ++k) S[c][k] = om * (mu * (Gx[c][k] + Gx[k][c]) + (c == k ? lam * tr : T(0)));
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              T F[3];
#pragma unroll
              for (int a = 0; a < 3; ++a) F[a] = S[c][0] * Ji[0][a] + S[c][1] * Ji[1][a] + S[c][2] * Ji[2][a];
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
        const int q01 = t;
        const long long eref = ex + (long long)br.n_span[0] * (ey + (long long)br.n_span[1] * ez);
#pragma unroll
        for (int q2 = 0; q2 < Q; ++q2) {
          const int q = q01 + QQ * q2;
          double w = A.wq[slot * NQE + q];
#pragma unroll
          for (int c = 0; c < VEC; ++c) {
            g[c][0][q2] = g[c][1][q2] = g[c][2][q2] = T(0);
            g[c][HASV ? 3 : 0][q2] = (T)(w * A.f_qp[(eref * NQE + q) * VEC + c]);
          }
        }
      }
    }

    if constexpr (MODE == MODE_APPLY || MODE == MODE_LOAD) {
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
              T nv = stz[q2 * P1 + i2], nd = stz[(Q + q2) * P1 + i2];
              vv += nd * g[c][2][q2];
              if constexpr (HASV) vv += nv * g[c][3][q2];
              vd += nv * g[c][1][q2];
              dv += nv * g[c][0][q2];
            }
            int o = q1 * SY1 + i2 * Q + q0;
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
            int o = q1 * SY1 + i2 * Q + q0;
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
        if (evalid && t < PP) {  // X^T: (i1, i2) -> stage
          const T* src = bufX + el * 2 * Q * SX;
          T a[Q], ad[Q];
#pragma unroll
          for (int q0 = 0; q0 < Q; ++q0) {
            a[q0] = src[q0 * SX + t];
            ad[q0] = src[(Q + q0) * SX + t];
          }
          const int i1 = t % P1, i2 = t / P1;
          T* dst = stage + (el * VEC + c) * PPP;
#pragma unroll
          for (int i0 = 0; i0 < P1; ++i0) {
            T r = 0;
#pragma unroll
            for (int q0 = 0; q0 < Q; ++q0) r += nx_v[q0 * P1 + i0] * a[q0] + nx_v[(Q + q0) * P1 + i0] * ad[q0];
            if constexpr (RAT) {
              long long cp = (long long)br.n_cp[0] * ((fy + i1) + (long long)br.n_cp[1] * (fz + i2)) + fx + i0;
              r *= A.wgts[cp];
            }
            dst[i0 * PP + t] = r;
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
            T vx = nx_v[q0 * P1 + a0], dx = nx_v[(Q + q0) * P1 + a0];
            T vy = ny_v[q1 * P1 + a1], dy = ny_v[(Q + q1) * P1 + a1];
            T vz = stz[q2 * P1 + a2], dz = stz[(Q + q2) * P1 + a2];
            T ph[4] = {dx * vy * vz, vx * dy * vz, vx * vy * dz, vx * vy * vz};
            const T* G = A.geo + (size_t)slot * NG * NQE + q;
            if constexpr (OPK == OPK_SCALAR) {
              if constexpr (!RAT) {
                T k0 = G[0], k1 = G[NQE], k2 = G[2 * NQE], k3 = G[3 * NQE], k4 = G[4 * NQE], k5 = G[5 * NQE];
                d[0] += k0 * ph[0] * ph[0] + k3 * ph[1] * ph[1] + k5 * ph[2] * ph[2] +
                        T(2) * (k1 * ph[0] * ph[1] + k2 * ph[0] * ph[2] + k4 * ph[1] * ph[2]);
              } else {
                T s[4] = {ph[3], ph[0], ph[1], ph[2]};
                int k = 0;
                T acc_ = 0;
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                  for (int j = i; j < 4; ++j) {
                    T m = G[(k++) * NQE];
                    acc_ += (i == j ? T(1) : T(2)) * m * s[i] * s[j];
                  }
                d[0] += acc_;
              }
            } else {
              T Ji[3][3];
#pragma unroll
              for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int b2 = 0; b2 < 3; ++b2) Ji[i][b2] = G[(i * 3 + b2) * NQE];
              T om = G[9 * NQE];
              T gp[3] = {ph[0], ph[1], ph[2]};
              if constexpr (RAT) {
                T iW = G[10 * NQE];
#pragma unroll
                for (int b2 = 0; b2 < 3; ++b2) gp[b2] = (gp[b2] - ph[3] * G[(11 + b2) * NQE]) * iW;
              }
              T gx[3];
#pragma unroll
              for (int k = 0; k < 3; ++k) gx[k] = Ji[k][0] * gp[0] + Ji[k][1] * gp[1] + Ji[k][2] * gp[2];
              T n2 = gx[0] * gx[0] + gx[1] * gx[1] + gx[2] * gx[2];
#pragma unroll
              for (int c = 0; c < VEC; ++c) d[c] += om * ((T)(A.lam + A.mu) * gx[c] * gx[c] + (T)A.mu * n2);
            }
          }
          T wsq = 1;
          if constexpr (RAT) {
            long long cp = (long long)br.n_cp[0] * ((fy + a1) + (long long)br.n_cp[1] * (fz + a2)) + fx + a0;
            wsq = A.wgts[cp] * A.wgts[cp];
          }
#pragma unroll
          for (int c = 0; c < VEC; ++c) stage[(el * VEC + c) * PPP + a0 * PP + a1 + P1 * a2] = d[c] * wsq;
        }
      }
    }
    __syncthreads();
    // prefetch the next layer's factors while the gather runs
    if constexpr (MODE == MODE_APPLY) {
      if (tid == 0 && lz + 1 < nlayers) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        const unsigned bytes = NE * NG * NQE * sizeof(T);
        mbar_expect_tx(bar, bytes);
        bulk_copy_g2s(sgeo, A.geo + (size_t)(slot_base + (long long)(lz + 1) * NE) * NG * NQE, bytes, bar);
      }
    }
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
            s += stage[((e1 * TX + e0) * VEC + c) * PPP + lx * PP + ly + P1 * jzl];
          }
        }
        acc[((c * fp2 + offz + jzl) * fp1 + jy) * fp0 + jx] += s;
      }
    }
    __syncthreads();
  }
  // write the brick footprint
  T* out = A.scratch + (size_t)b * accn;
  for (int i = tid; i < accn; i += NT) out[i] = acc[i];
}

// ---------------------------------------------------------------------------
// 2D brick kernel: TX elements per row, TY rows; Q threads per element.
// ---------------------------------------------------------------------------
template <typename T, int P, int Q, int OPK, bool RAT, int MODE>
__global__ void __launch_bounds__(BrickShape<2, P>::TX* Q) k_brick2(BrickArgs<T> A) {
  constexpr int P1 = P + 1, PP = P1 * P1;
  constexpr int TX = BrickShape<2, P>::TX, TY = BrickShape<2, P>::TY;
  constexpr int NE = TX, NQE = Q * Q, NT = NE * Q;
  constexpr int VEC = OPK == OPK_ELAST ? 2 : 1;
  constexpr int NG = GeoCount<OPK, RAT, 2>::value;
  constexpr bool HASV = RAT || MODE == MODE_LOAD;
  constexpr bool HESS = OPK == OPK_PLATE;
  constexpr int NK = HESS ? 3 : 2;      // 1D table kinds used
  constexpr int NCH = HESS ? 6 : 3;     // channels (v, g0, g1[, h00, h01, h11])
  constexpr int SX = P1 + 1;            // padded q0 stride

  if (A.state && A.state->done) return;
  const Bricks& br = A.br;
  const int fp0 = br.fp[0], fp1 = br.fp[1];

  extern __shared__ __align__(128) unsigned char smem_raw[];
  T* stx = reinterpret_cast<T*>(smem_raw);   // [TX][3][Q][P1]
  T* sty = stx + TX * 3 * Q * P1;            // [3][Q][P1]
  T* bufX = sty + 3 * Q * P1;                // [NE][NK][Q][SX]
  T* stage = bufX + NE * NK * Q * SX;        // [NE][VEC][PP]
  T* acc = stage + NE * VEC * PP;            // [VEC][fp1][fp0]
  int* soff = reinterpret_cast<int*>(acc + VEC * fp0 * fp1);

  const int tid = threadIdx.x;
  const long long b = blockIdx.x;
  const int bx = (int)(b % br.nb[0]);
  const int by = (int)(b / br.nb[0]);
  const int cp0x = br.bcp0[0][bx], cp0y = br.bcp0[1][by];
  const int el = tid / Q, t = tid % Q;
  const int ex = bx * TX + el;
  const bool evalid = ex < br.n_span[0];

  for (int i = tid; i < TX * 3 * Q * P1; i += NT) {
    int e = i / (3 * Q * P1), r = i % (3 * Q * P1);
    int sp = min(bx * TX + e, br.n_span[0] - 1);
    stx[i] = A.tab[0][(size_t)sp * 3 * Q * P1 + r];
  }
  if (tid < TX) {
    int e = bx * TX + tid;
    soff[tid] = e < br.n_span[0] ? br.first[0][e] - cp0x : -100000;
  }
  const int accn = VEC * fp0 * fp1;
  for (int i = tid; i < accn; i += NT) acc[i] = T(0);
  const long long slot_base = b * (long long)TY * NE;
  const int nlayers = min(TY, br.n_span[1] - by * TY);
  const T* nx_v = stx + el * 3 * Q * P1;

  for (int ly_ = 0; ly_ < nlayers; ++ly_) {
    const int ey = by * TY + ly_;
    const int fy = br.first[1][ey];
    const int offy = fy - cp0y;
    for (int i = tid; i < 3 * Q * P1; i += NT) sty[i] = A.tab[1][(size_t)ey * 3 * Q * P1 + i];
    __syncthreads();
    const long long slot = slot_base + (long long)ly_ * NE + el;
    const int fx = evalid ? br.first[0][ex] : 0;
    T g[VEC][NCH][Q];  // channel order (v, g0, g1, h00, h01, h11) at q1

    if constexpr (MODE == MODE_APPLY) {
#pragma unroll
      for (int c = 0; c < VEC; ++c) {
        if (evalid && t < P1) {  // X: line along x at row i1 = t
          const int i1 = t;
          const long long row = (long long)br.n_cp[0] * (fy + i1) + fx;
          T u[P1];
#pragma unroll
          for (int i0 = 0; i0 < P1; ++i0) {
            long long cp = row + i0;
            T v = A.x[cp * VEC + c];
            if (A.masked) v = A.keep[cp * VEC + c] ? v : T(0);
            if constexpr (RAT) v *= A.wgts[cp];
            u[i0] = v;
          }
          T* dst = bufX + el * NK * Q * SX;
#pragma unroll
          for (int k = 0; k < NK; ++k)
#pragma unroll
            for (int q0 = 0; q0 < Q; ++q0) {
              T s = 0;
#pragma unroll
              for (int i0 = 0; i0 < P1; ++i0) s += nx_v[(k * Q + q0) * P1 + i0] * u[i0];
              dst[(k * Q + q0) * SX + i1] = s;
            }
        }
        __syncthreads();
        if (evalid) {  // Y in registers: q0 = t
          const int q0 = t;
          const T* src = bufX + el * NK * Q * SX;
          T a[NK][P1];
#pragma unroll
          for (int k = 0; k < NK; ++k)
#pragma unroll
            for (int i1 = 0; i1 < P1; ++i1) a[k][i1] = src[(k * Q + q0) * SX + i1];
#pragma unroll
          for (int q1 = 0; q1 < Q; ++q1) {
            T ch[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
            for (int i1 = 0; i1 < P1; ++i1) {
              T nv = sty[q1 * P1 + i1], nd = sty[(Q + q1) * P1 + i1];
              ch[0] += nv * a[0][i1];
              ch[1] += nv * a[1][i1];
              ch[2] += nd * a[0][i1];
              if constexpr (HESS) {
                T nh = sty[(2 * Q + q1) * P1 + i1];
                ch[3] += nv * a[2][i1];
                ch[4] += nd * a[1][i1];
                ch[5] += nh * a[0][i1];
              }
            }
#pragma unroll
            for (int k = 0; k < NCH; ++k) g[c][k][q1] = ch[k];
          }
        }
        __syncthreads();
      }
      if (evalid) {
        const T* G = A.geo + (size_t)slot * NG * NQE;
#pragma unroll
        for (int q1 = 0; q1 < Q; ++q1) {
          const int q = t + Q * q1;
          if constexpr (OPK == OPK_SCALAR) {
            if constexpr (!RAT) {
              T k0 = G[q], k1 = G[NQE + q], k2 = G[2 * NQE + q];
              T gx = g[0][1][q1], gy = g[0][2][q1];
              g[0][1][q1] = k0 * gx + k1 * gy;
              g[0][2][q1] = k1 * gx + k2 * gy;
              g[0][0][q1] = 0;
            } else {
              T m[6];
#pragma unroll
              for (int k = 0; k < 6; ++k) m[k] = G[k * NQE + q];
              T v = g[0][0][q1], gx = g[0][1][q1], gy = g[0][2][q1];
              g[0][0][q1] = m[0] * v + m[1] * gx + m[2] * gy;
              g[0][1][q1] = m[1] * v + m[3] * gx + m[4] * gy;
              g[0][2][q1] = m[2] * v + m[4] * gx + m[5] * gy;
            }
          } else if constexpr (OPK == OPK_PLATE) {
            constexpr int n = RAT ? 6 : 5, off = RAT ? 0 : 1;
            T s[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) s[k] = g[0][k][q1];
            T o[6] = {0, 0, 0, 0, 0, 0};
            int k = 0;
#pragma unroll
            for (int i = 0; i < n; ++i)
#pragma unroll
              for (int j = i; j < n; ++j) {
                T m = G[(k++) * NQE + q];
                o[i + off] += m * s[j + off];
                if (j != i) o[j + off] += m * s[i + off];
              }
#pragma unroll
            for (int kk = 0; kk < 6; ++kk) g[0][kk][q1] = o[kk];
          } else {  // 2D elasticity
            T Ji[2][2] = {{G[q], G[NQE + q]}, {G[2 * NQE + q], G[3 * NQE + q]}};
            T om = G[4 * NQE + q];
            T iW = 1, gW[2] = {0, 0};
            if constexpr (RAT) {
              iW = G[5 * NQE + q];
              gW[0] = G[6 * NQE + q];
              gW[1] = G[7 * NQE + q];
            }
            T gp[2][2];
#pragma unroll
            for (int c = 0; c < 2; ++c)
#pragma unroll
              for (int a = 0; a < 2; ++a) gp[c][a] = RAT ? (g[c][1 + a][q1] - g[c][0][q1] * gW[a]) * iW : g[c][1 + a][q1];
            T Gx[2][2];
#pragma unroll
            for (int c = 0; c < 2; ++c)
#pragma unroll
              for (int k = 0; k < 2; ++k) Gx[c][k] = Ji[k][0] * gp[c][0] + Ji[k][1] * gp[c][1];
            T tr = Gx[0][0] + Gx[1][1];
            T lam = (T)A.lam, mu = (T)A.mu;
#pragma unroll
            for (int c = 0; c < 2; ++c) {
              T S0 = om * (mu * (Gx[c][0] + Gx[0][c]) + (c == 0 ? lam * tr : T(0)));
              T S1 = om * (mu * (Gx[c][1] + Gx[1][c]) + (c == 1 ? lam * tr : T(0)));
              T F0 = S0 * Ji[0][0] + S1 * Ji[1][0];
              T F1 = S0 * Ji[0][1] + S1 * Ji[1][1];
              if constexpr (RAT) {
                g[c][0][q1] = -(F0 * gW[0] + F1 * gW[1]) * iW;
                g[c][1][q1] = F0 * iW;
                g[c][2][q1] = F1 * iW;
              } else {
                g[c][0][q1] = 0;
                g[c][1][q1] = F0;
                g[c][2][q1] = F1;
              }
            }
          }
        }
      }
    } else if constexpr (MODE == MODE_LOAD) {
      if (evalid) {
        const long long eref = ex + (long long)br.n_span[0] * ey;
#pragma unroll
        for (int q1 = 0; q1 < Q; ++q1) {
          const int q = t + Q * q1;
          double w = A.wq[slot * NQE + q];
#pragma unroll
          for (int c = 0; c < VEC; ++c) {
#pragma unroll
            for (int k = 0; k < NCH; ++k) g[c][k][q1] = T(0);
            g[c][0][q1] = (T)(w * A.f_qp[(eref * NQE + q) * VEC + c]);
          }
        }
      }
    }

    if constexpr (MODE == MODE_APPLY || MODE == MODE_LOAD) {
#pragma unroll
      for (int c = 0; c < VEC; ++c) {
        if (evalid) {  // Y^T: q0 = t -> bufX[k][q0][i1]
          const int q0 = t;
          T* dst = bufX + el * NK * Q * SX;
#pragma unroll
          for (int i1 = 0; i1 < P1; ++i1) {
            T a0 = 0, a1 = 0, a2 = 0;
#pragma unroll
            for (int q1 = 0; q1 < Q; ++q1) {
              T nv = sty[q1 * P1 + i1], nd = sty[(Q + q1) * P1 + i1];
              if constexpr (HASV || HESS) a0 += nv * g[c][0][q1];
              a0 += nd * g[c][2][q1];
              a1 += nv * g[c][1][q1];
              if constexpr (HESS) {
                T nh = sty[(2 * Q + q1) * P1 + i1];
                a0 += nh * g[c][5][q1];
                a1 += nd * g[c][4][q1];
                a2 += nv * g[c][3][q1];
              }
            }
            dst[(0 * Q + q0) * SX + i1] = a0;
            dst[(1 * Q + q0) * SX + i1] = a1;
            if constexpr (HESS) dst[(2 * Q + q0) * SX + i1] = a2;
          }
        }
        __syncthreads();
        if (evalid && t < P1) {  // X^T: row i1 = t
          const int i1 = t;
          const T* src = bufX + el * NK * Q * SX;
          T* dst = stage + (el * VEC + c) * PP;
#pragma unroll
          for (int i0 = 0; i0 < P1; ++i0) {
            T r = 0;
#pragma unroll
            for (int k = 0; k < NK; ++k)
#pragma unroll
              for (int q0 = 0; q0 < Q; ++q0) r += nx_v[(k * Q + q0) * P1 + i0] * src[(k * Q + q0) * SX + i1];
            if constexpr (RAT) r *= A.wgts[(long long)br.n_cp[0] * (fy + i1) + fx + i0];
            dst[i0 * P1 + i1] = r;
          }
        }
        __syncthreads();
      }
    } else {  // MODE_DIAG
      if (evalid) {
        for (int a = t; a < PP; a += Q) {
          const int a0 = a % P1, a1 = a / P1;
          T d[VEC];
#pragma unroll
          for (int c = 0; c < VEC; ++c) d[c] = 0;
          for (int q = 0; q < NQE; ++q) {
            const int q0 = q % Q, q1 = q / Q;
            T vx = nx_v[q0 * P1 + a0], dx = nx_v[(Q + q0) * P1 + a0], hx = nx_v[(2 * Q + q0) * P1 + a0];
            T vy = sty[q1 * P1 + a1], dy = sty[(Q + q1) * P1 + a1], hy = sty[(2 * Q + q1) * P1 + a1];
            T s[6] = {vx * vy, dx * vy, vx * dy, hx * vy, dx * dy, vx * hy};
            const T* G = A.geo + (size_t)slot * NG * NQE + q;
            if constexpr (OPK == OPK_SCALAR || OPK == OPK_PLATE) {
              constexpr int n = OPK == OPK_SCALAR ? (RAT ? 3 : 2) : (RAT ? 6 : 5);
              constexpr int off = RAT ? 0 : 1;
              int k = 0;
              T acc_ = 0;
#pragma unroll
              for (int i = 0; i < n; ++i)
#pragma unroll
                for (int j = i; j < n; ++j) {
                  T m = G[(k++) * NQE];
                  acc_ += (i == j ? T(1) : T(2)) * m * s[i + off] * s[j + off];
                }
              d[0] += acc_;
            } else {
              T Ji[2][2] = {{G[0], G[NQE]}, {G[2 * NQE], G[3 * NQE]}};
              T om = G[4 * NQE];
              T gp[2] = {s[1], s[2]};
              if constexpr (RAT) {
                T iW = G[5 * NQE];
                gp[0] = (gp[0] - s[0] * G[6 * NQE]) * iW;
                gp[1] = (gp[1] - s[0] * G[7 * NQE]) * iW;
              }
              T gx[2] = {Ji[0][0] * gp[0] + Ji[0][1] * gp[1], Ji[1][0] * gp[0] + Ji[1][1] * gp[1]};
              T n2 = gx[0] * gx[0] + gx[1] * gx[1];
#pragma unroll
              for (int c = 0; c < VEC; ++c) d[c] += om * ((T)(A.lam + A.mu) * gx[c] * gx[c] + (T)A.mu * n2);
            }
          }
          T wsq = 1;
          if constexpr (RAT) {
            T w = A.wgts[(long long)br.n_cp[0] * (fy + a1) + fx + a0];
            wsq = w * w;
          }
#pragma unroll
          for (int c = 0; c < VEC; ++c) stage[(el * VEC + c) * PP + a0 * P1 + a1] = d[c] * wsq;
        }
      }
      __syncthreads();
    }
    // gather the row into the brick footprint
    {
      const int nfoot = VEC * fp0 * P1;
      for (int i = tid; i < nfoot; i += NT) {
        const int jx = i % fp0;
        const int jyl = (i / fp0) % P1;
        const int c = i / (fp0 * P1);
        T s = 0;
#pragma unroll 4
        for (int e0 = 0; e0 < TX; ++e0) {
          const int lx = jx - soff[e0];
          if (lx < 0 || lx > P) continue;
          s += stage[(e0 * VEC + c) * PP + lx * P1 + jyl];
        }
        acc[(c * fp1 + offy + jyl) * fp0 + jx] += s;
      }
    }
    __syncthreads();
  }
  T* out = A.scratch + (size_t)b * accn;
  for (int i = tid; i < accn; i += NT) out[i] = acc[i];
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

template <typename T>
__global__ void __launch_bounds__(JXB_RED_THREADS) k_combine(Bricks br, const T* __restrict__ scratch, const uint8_t* __restrict__ keep,
                          int masked, T* __restrict__ y, const T* __restrict__ dot_with,
                          double* __restrict__ partials, const CgState* state) {
  if (state && state->done) return;
  const int vec = br.vec, dim = br.dim;
  const long long n_scalar = (long long)br.n_cp[0] * br.n_cp[1] * (dim == 3 ? br.n_cp[2] : 1);
  double part = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_scalar;
       i += (long long)gridDim.x * blockDim.x) {
    int ix = (int)(i % br.n_cp[0]);
    int iy = (int)((i / br.n_cp[0]) % br.n_cp[1]);
    int iz = dim == 3 ? (int)(i / ((long long)br.n_cp[0] * br.n_cp[1])) : 0;
    const int* cx = br.cover[0] + 2 * JXB_MAXC * ix;
    const int* cy = br.cover[1] + 2 * JXB_MAXC * iy;
    const int* cz = dim == 3 ? br.cover[2] + 2 * JXB_MAXC * iz : nullptr;
    for (int c = 0; c < vec; ++c) {
      T s = 0;
      for (int kz = 0; kz < (dim == 3 ? JXB_MAXC : 1); ++kz) {
        int bz = dim == 3 ? cz[2 * kz] : 0, oz = dim == 3 ? cz[2 * kz + 1] : 0;
        if (bz < 0) break;
        for (int ky = 0; ky < JXB_MAXC; ++ky) {
          int by = cy[2 * ky], oy = cy[2 * ky + 1];
          if (by < 0) break;
          for (int kx = 0; kx < JXB_MAXC; ++kx) {
            int bx = cx[2 * kx], ox = cx[2 * kx + 1];
            if (bx < 0) break;
            long long brick = bx + (long long)br.nb[0] * (by + (long long)br.nb[1] * bz);
            long long off = ((brick * vec + c) * (dim == 3 ? br.fp[2] : 1) + oz) * br.fp[1];
            s += scratch[(off + oy) * br.fp[0] + ox];
          }
        }
      }
      long long dof = i * vec + c;
      if (masked && !keep[dof]) s = T(0);
      y[dof] = s;
      if (dot_with) part += (double)dot_with[dof] * (double)s;
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
  constexpr int P1 = P + 1, PP = P1 * P1, PPP = PP * P1;
  constexpr int TX = BrickShape<3, P>::TX, TY = BrickShape<3, P>::TY;
  constexpr int NE = TX * TY, NQE = Q * Q * Q;
  constexpr int VEC = OPK == OPK_ELAST ? 3 : 1;
  constexpr int NG = GeoCount<OPK, RAT, 3>::value;
  constexpr int SX = PP + 1, SY1 = Q * P1 + 1, SYC = Q * SY1;
  size_t n = (MODE == MODE_APPLY ? (size_t)NE * NG * NQE : 0) + (TX + TY + 1) * 2 * Q * P1 + NE * 2 * Q * SX +
             NE * 3 * SYC + NE * VEC * PPP + (size_t)VEC * br.fp[0] * br.fp[1] * br.fp[2];
  return n * sizeof(T) + (TX + TY) * sizeof(int) + 64;
}

template <typename T, int P, int Q, int OPK, bool RAT, int MODE>
static size_t smem2(const Bricks& br) {
  constexpr int P1 = P + 1, PP = P1 * P1;
  constexpr int TX = BrickShape<2, P>::TX;
  constexpr int VEC = OPK == OPK_ELAST ? 2 : 1;
  constexpr int NK = OPK == OPK_PLATE ? 3 : 2;
  constexpr int SX = P1 + 1;
  size_t n = (size_t)TX * 3 * Q * P1 + 3 * Q * P1 + TX * NK * Q * SX + TX * VEC * PP +
             (size_t)VEC * br.fp[0] * br.fp[1];
  return n * sizeof(T) + TX * sizeof(int) + 64;
}

template <typename T, int P, int OPK, bool RAT, int MODE>
static int launch_one(const BrickArgs<T>& A, cudaStream_t s) {
  constexpr int Q = P + 1;
  const Bricks& br = A.br;
  if (br.dim == 3) {
    if constexpr (OPK == OPK_PLATE) {
      return fail(JXB_ERR_INVALID, "plate operator is 2D only");
    } else {
      constexpr int NT = BrickShape<3, P>::TX * BrickShape<3, P>::TY * Q * Q;
      size_t sm = smem3<T, P, Q, OPK, RAT, MODE>(br);
      if (sm > 227 * 1024) return fail(JXB_ERR_INVALID, "3D brick does not fit in shared memory for this degree/operator");
      auto k = k_brick3<T, P, Q, OPK, RAT, MODE>;
      if (sm > 48 * 1024) JXB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      k<<<(unsigned)br.n_bricks, NT, sm, s>>>(A);
    }
  } else {
    constexpr int NT = BrickShape<2, P>::TX * Q;
    size_t sm = smem2<T, P, Q, OPK, RAT, MODE>(br);
    if (sm > 227 * 1024) return fail(JXB_ERR_INVALID, "2D brick does not fit in shared memory");
    auto k = k_brick2<T, P, Q, OPK, RAT, MODE>;
    if (sm > 48 * 1024) JXB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k<<<(unsigned)br.n_bricks, NT, sm, s>>>(A);
  }
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

template <typename T, int MODE>
static int dispatch(jxb_plan* plan, const BrickArgs<T>& A, cudaStream_t s) {
  int opk = plan->op == JXB_OP_POISSON ? OPK_SCALAR : plan->op == JXB_OP_ELASTICITY ? OPK_ELAST : OPK_PLATE;
  bool rat = plan->rational != 0;
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

template <typename T>
int launch_bricks(jxb_plan* plan, cudaStream_t s, int mode, const T* x, const double* f_qp,
                  const CgState* state, int masked) {
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
  }
  return fail(JXB_ERR_INVALID, "unsupported brick mode");
}

template <typename T>
int launch_combine(jxb_plan* plan, cudaStream_t s, T* y, int masked, const T* dot_with,
                   double* partials, const CgState* state) {
  const T* scratch;
  if constexpr (sizeof(T) == 4)
    scratch = plan->d_scratch32;
  else
    scratch = plan->d_scratch;
  k_combine<T><<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(plan->br, scratch, plan->d_keep, masked, y,
                                                           dot_with, partials, state);
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

template int launch_bricks<double>(jxb_plan*, cudaStream_t, int, const double*, const double*,
                                   const CgState*, int);
template int launch_bricks<float>(jxb_plan*, cudaStream_t, int, const float*, const double*,
                                  const CgState*, int);
template int launch_combine<double>(jxb_plan*, cudaStream_t, double*, int, const double*, double*,
                                    const CgState*);
template int launch_combine<float>(jxb_plan*, cudaStream_t, float*, int, const float*, double*,
                                   const CgState*);

}  // namespace jxb
