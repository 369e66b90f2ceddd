// FP64 tensor-core variant of the 3D brick apply at degree 3 with 4 Gauss
// points per direction, for the scalar operator (Poisson / Darcy) and for
// linear elasticity, polynomial weights. Included by apply.cu inside
// namespace jxb.
//
// At p = 3 every 1D contraction of the sum factorisation is a product of the
// 8 x 4 table [N; N'] (rows: 4 points x value/derivative, columns: the 4
// Bernstein functions) with a 4-row slab of element data, i.e. exactly the
// shape of mma.sync.m8n8k4.f64: one instruction does the 256 multiply-adds
// that take 256 scalar FMAs (and as many table loads) otherwise. The
// backward contractions use the transposed tables [N^T; N'^T] (or the halves
// swapped, so the needed product lands in rows 0-3).
//
// Work split: the CTA owns one 4 x 4 x 8 element brick as in the FMA
// kernel, and each of its 16 warps owns one column of 8 elements along z.
// A warp runs each element's whole pipeline warp-synchronously -- per
// displacement component the forward x, y, z contractions, then the point
// operator on all components, then per component the backward z, y, x
// (28 MMAs per component) -- handing data between stages through a private,
// bank-conflict-free shared-memory area (__syncwarp between stages), and adds the element
// residual into its column's footprint in shared memory, layer after layer in
// order. Warps never wait for each other until the brick is done; then one
// fixed-order gather sums the 16 column footprints into the brick footprint
// (no atomics), so the result is bitwise reproducible. Input fragments come
// straight from the DOF vector (read one layer ahead), factor tiles are
// prefetched into L2 one layer ahead.
//
// Fragment layouts of m8n8k4 (lane l, g = l >> 2, t = l & 3):
//   A (8x4, row): a = A[g][t];  B (4x8, col): b = B[t][g];  C/D (8x8): d_i = D[g][2t + i].

namespace bm {
constexpr int P1 = 4, Q = 4, NQE = 64;
constexpr int TX = 4, TY = 4, CZ = 8, NE = TX * TY, NT = NE * 32;
// XB, FB and SB are rows of 16 doubles stored XOR-swizzled (swz below), which
// keeps both the 16-byte fragment stores and the 8-byte operand loads free of
// bank conflicts; YB and TB get the same from padding.
constexpr int YR = 8, Y2 = 68;       // YB[i2 (4)][rY (8)][rX (8)]
constexpr int FC = 64;               // FB[channel (3)][q2 (4)][n (16)], n = q0 + 4 q1   (swizzled rows)
constexpr int T2 = 24, TC = 4 * T2;  // TB[channel (3)][i2 (4)][n (16)]
constexpr int SC = 64;               // SB[type (2)][i1 (4)][m (16)], m = q0 + 4 i2      (swizzled rows)
                                     // XB[rX (8)][c (16)], c = i1 + 4 i2                 (swizzled rows)
constexpr int RA = 3 * FC;           // region A (XB, FB, SB): 192 doubles
constexpr int RB = 3 * TC;           // region B (YB, TB): 288 doubles
constexpr int WB = RA + RB;          // per-warp doubles
constexpr int CF = P1 * P1;          // one z row of a column footprint: [i1][i0]
static_assert(8 * 16 <= RA && 2 * SC <= RA && 4 * Y2 <= RB, "per-warp regions");
}  // namespace bm

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b, double c0, double c1) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%4,%5};"
      : "=d"(d0), "=d"(d1)
      : "d"(a), "d"(b), "d"(c0), "d"(c1));
}

// position of (row r, column c) in a swizzled buffer of 16-double rows: the
// row's two low bits flip column bits 3 and 2 (pairs c, c+1 stay adjacent)
__device__ __forceinline__ int swz(int r, int c) { return r * 16 + (c ^ (((r & 1) << 3) | ((r & 2) << 1))); }

__device__ __forceinline__ void st2(double* p, double a, double b) {
  *reinterpret_cast<double2*>(p) = make_double2(a, b);
}

template <int OPK>
static size_t smem3_mma(const Bricks& br) {
  using namespace bm;
  constexpr int VEC = OPK == OPK_ELAST ? 3 : 1;
  const size_t n = (size_t)NE * WB + (size_t)NE * VEC * br.fp[2] * CF;
  return n * sizeof(double) + (TX + TY) * sizeof(int) + 64;
}

// MINB resident CTAs per SM the kernel is built for: 2 caps registers at 64
// per thread, 1 allows 128 with half the warps.
template <int OPK, int MINB>
__global__ void __launch_bounds__(bm::NT, MINB) k_brick3_mma(BrickArgs<double> A) {
  using namespace bm;
  constexpr int VEC = OPK == OPK_ELAST ? 3 : 1;
  constexpr int NG = OPK == OPK_ELAST ? 10 : 6;  // factors per point: J^-1 and w|J| / the symmetric metric
  if (A.state && A.state->done) return;
  const Bricks& br = A.br;
  const int fp0 = br.fp[0], fp1 = br.fp[1], fp2 = br.fp[2];

  extern __shared__ __align__(128) unsigned char smem_raw[];
  double* wbuf = reinterpret_cast<double*>(smem_raw);  // [NE][WB] stage hand-off areas
  double* colf = wbuf + NE * WB;                         // [NE][VEC][fp2][i1][i0] column footprints
  int* soff = reinterpret_cast<int*>(colf + NE * VEC * fp2 * CF);

  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const long long b = blockIdx.x;
  const int bx = (int)(b % br.nb[0]);
  const int by = (int)((b / br.nb[0]) % br.nb[1]);
  const int bz = (int)(b / ((long long)br.nb[0] * br.nb[1]));
  const int cp0x = br.bcp0[0][bx], cp0y = br.bcp0[1][by], cp0z = br.bcp0[2][bz];
  const int exl = w % TX, eyl = w / TX;
  const int ex = bx * TX + exl, ey = by * TY + eyl;
  const bool evalid = ex < br.n_span[0] && ey < br.n_span[1];
  const int cz = br.te[2];  // element layers per brick (<= CZ): fewer for small patches
  const long long slot_base = b * (long long)cz * NE;
  const int nlayers = min(cz, br.n_span[2] - bz * cz);
  if (tid < TX) {
    const int e = bx * TX + tid;
    soff[tid] = e < br.n_span[0] ? br.first[0][e] - cp0x : -100000;
  }
  if (tid < TY) {
    const int e = by * TY + tid;
    soff[TX + tid] = e < br.n_span[1] ? br.first[1][e] - cp0y : -100000;
  }
  double* cf = colf + w * VEC * fp2 * CF;
  for (int i = lane; i < VEC * fp2 * CF; i += 32) cf[i] = 0.0;

  if (evalid) {
    // A fragments of the column's x / y tables ([2][Q][P1] per span)
    const double* tx_ = A.tab[0] + (size_t)ex * 3 * Q * P1;
    const double* ty_ = A.tab[1] + (size_t)ey * 3 * Q * P1;
    const int bo = t * 4 + (g & 3);  // [q = t][i = g & 3]
    const int ty0 = (g >> 2) * 16, ty1 = (1 - (g >> 2)) * 16;
    const double ax = tx_[lane], ay = ty_[lane];
    const double axb = tx_[ty0 + bo], axb2 = tx_[ty1 + bo];
    const double ayb = ty_[ty0 + bo], ayb2 = ty_[ty1 + bo];
    double* RA_ = wbuf + w * WB;
    double* RB_ = RA_ + RA;
    const bool hi = lane >= 16;
    const int hh = hi ? 1 : 0;
    const long long ncx = br.n_cp[0], nxy = (long long)br.n_cp[0] * br.n_cp[1];
    // this lane's input entries (x-stage B fragments): i0 = t, i1 = g & 3, i2 = 2j + (g >> 2)
    const long long cxy = (long long)(br.first[0][ex] + t) + ncx * (br.first[1][ey] + (g & 3));
    auto load_in = [&](int ez_, double (&u)[VEC][2]) {
      const long long c0 = cxy + nxy * (br.first[2][ez_] + (g >> 2));
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const long long cp = c0 + 2 * j * nxy;
#pragma unroll
        for (int c = 0; c < VEC; ++c) {
          const long long dof = cp * VEC + c;
          double v = A.x[dof];
          if (A.masked && !A.keep[dof]) v = 0.0;
          u[c][j] = v;
        }
      }
    };
    const int qoff = 16 * (g & 3) + 8 * hh + 2 * t;
    if (lane == 0) prefetch_l2(A.geo + (size_t)(slot_base + w) * NG * NQE, NG * NQE * sizeof(double));
    double un[VEC][2];
    load_in(bz * cz, un);
    for (int lz = 0; lz < nlayers; ++lz) {
      const int ez = bz * cz + lz;
      const int offz = br.first[2][ez] - cp0z;
      const long long slot = slot_base + (long long)lz * NE + w;
      if (lane == 0 && lz + 1 < nlayers) prefetch_l2(A.geo + (size_t)(slot + NE) * NG * NQE, NG * NQE * sizeof(double));
      double u[VEC][2];
#pragma unroll
      for (int c = 0; c < VEC; ++c) {
        u[c][0] = un[c][0];
        u[c][1] = un[c][1];
      }
      if (lz + 1 < nlayers) load_in(ez + 1, un);
      const double* tz_ = A.tab[2] + (size_t)ez * 3 * Q * P1;
      const double az = tz_[lane], azb = tz_[ty0 + bo], azb2 = tz_[ty1 + bo];
      const double* G = A.geo + (size_t)slot * NG * NQE + qoff;
      double2 kf[NG];
      // gradients of each component at this lane's two points
      double GX[VEC][2], GY[VEC][2], GZ[VEC][2];
#pragma unroll
      for (int c = 0; c < VEC; ++c) {
        // ---- forward x: D[rX = (type, q0)][c = i1 + 4 i2] -> XB
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          double d0, d1;
          dmma(d0, d1, ax, u[c][j], 0.0, 0.0);
          st2(RA_ + swz(g, 8 * j + 2 * t), d0, d1);
        }
        __syncwarp();
        // ---- forward y (i2 = jj): D[rY = (type, q1)][rX] -> YB[i2][rY][rX]
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const double bv = RA_[swz(g, t + 4 * jj)];
          double d0, d1;
          dmma(d0, d1, ay, bv, 0.0, 0.0);
          st2(RB_ + jj * Y2 + g * YR + 2 * t, d0, d1);
        }
        __syncwarp();
        if (c == VEC - 1) {  // the factors (L2 hits after the prefetch), in flight during the last z stage
#pragma unroll
          for (int k = 0; k < NG; ++k) kf[k] = __ldg(reinterpret_cast<const double2*>(G + k * NQE));
        }
        // ---- forward z, columns n = 8h + g -> (q0, q1) = (g & 3, 2h + (g >> 2))
        double gxr[2][2], gyr[2][2], gzr[2][2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const double* yb = RB_ + t * Y2 + (2 * h + (g >> 2)) * YR + (g & 3);
          const double bdv = yb[4];       // rY = (v, q1), rX = (d, q0): x-derivative
          const double bvd = yb[4 * YR];  // rY = (d, q1), rX = (v, q0): y-derivative
          const double bvv = yb[0];       // both values
          dmma(gxr[h][0], gxr[h][1], az, bdv, 0.0, 0.0);  // rows 0-3: d/dxi
          dmma(gyr[h][0], gyr[h][1], az, bvd, 0.0, 0.0);  // rows 0-3: d/deta
          dmma(gzr[h][0], gzr[h][1], az, bvv, 0.0, 0.0);  // rows 4-7: d/dzeta
        }
        // lanes 0-15 keep the points of h = 0, lanes 16-31 those of h = 1
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const double r1 = __shfl_xor_sync(0xffffffffu, hi ? gzr[0][i] : gxr[1][i], 16);
          const double r2 = __shfl_xor_sync(0xffffffffu, gyr[1][i], 16);
          GX[c][i] = hi ? r1 : gxr[0][i];
          GY[c][i] = hi ? r2 : gyr[0][i];
          GZ[c][i] = hi ? gzr[1][i] : r1;
        }
        __syncwarp();  // the next component's y stage overwrites YB
      }
      // ---- point operator at this lane's two points: fluxes F[c][a] (a = xi, eta, zeta)
      double F[VEC][3][2];
      if constexpr (OPK == OPK_ELAST) {
        const double lam = A.lam, mu = A.mu;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          double Ji[3][3];
#pragma unroll
          for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int a = 0; a < 3; ++a) Ji[k][a] = i ? kf[k * 3 + a].y : kf[k * 3 + a].x;
          const double om = i ? kf[9].y : kf[9].x;
          double Gx[3][3];  // du_c / dx_k
#pragma unroll
          for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int k = 0; k < 3; ++k) Gx[c][k] = Ji[k][0] * GX[c][i] + Ji[k][1] * GY[c][i] + Ji[k][2] * GZ[c][i];
          const double tr = Gx[0][0] + Gx[1][1] + Gx[2][2];
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            double Sr[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) Sr[k] = om * (mu * (Gx[c][k] + Gx[k][c]) + (c == k ? lam * tr : 0.0));
#pragma unroll
            for (int a = 0; a < 3; ++a) F[c][a][i] = Sr[0] * Ji[0][a] + Sr[1] * Ji[1][a] + Sr[2] * Ji[2][a];
          }
        }
      } else {
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const double k0 = i ? kf[0].y : kf[0].x, k1 = i ? kf[1].y : kf[1].x, k2 = i ? kf[2].y : kf[2].x;
          const double k3 = i ? kf[3].y : kf[3].x, k4 = i ? kf[4].y : kf[4].x, k5 = i ? kf[5].y : kf[5].x;
          F[0][0][i] = k0 * GX[0][i] + k1 * GY[0][i] + k2 * GZ[0][i];
          F[0][1][i] = k1 * GX[0][i] + k3 * GY[0][i] + k4 * GZ[0][i];
          F[0][2][i] = k2 * GX[0][i] + k4 * GY[0][i] + k5 * GZ[0][i];
        }
      }
#pragma unroll
      for (int c = 0; c < VEC; ++c) {
        {
          double* fb = RA_ + swz(g & 3, 8 * hh + 2 * t);
          st2(fb, F[c][0][0], F[c][0][1]);
          st2(fb + FC, F[c][1][0], F[c][1][1]);
          st2(fb + 2 * FC, F[c][2][0], F[c][2][1]);
        }
        __syncwarp();
        // ---- backward z: T[channel][i2][n] (rows 0-3 of each product)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const double* fb = RA_ + swz(t, 8 * h + g);
          double a0, a1, b0, b1, c0, c1;
          dmma(a0, a1, azb, fb[0], 0.0, 0.0);        // Nz^T F_xi   -> T_dv
          dmma(b0, b1, azb, fb[FC], 0.0, 0.0);       // Nz^T F_eta  -> T_vd
          dmma(c0, c1, azb2, fb[2 * FC], 0.0, 0.0);  // Nz'^T F_zeta -> T_vv
          if (!hi) {
            double* tb = RB_ + g * T2 + 8 * h + 2 * t;
            st2(tb, a0, a1);
            st2(tb + TC, b0, b1);
            st2(tb + 2 * TC, c0, c1);
          }
        }
        __syncwarp();
        // ---- backward y: columns m = 8h + g -> (q0, i2) = (g & 3, 2h + (g >> 2))
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const double* tb = RB_ + (2 * h + (g >> 2)) * T2 + (g & 3) + 4 * t;
          double v0, v1, d0, d1;
          dmma(v0, v1, ayb2, tb[TC], 0.0, 0.0);   // Ny'^T T_vd
          dmma(v0, v1, ayb, tb[2 * TC], v0, v1);  // + Ny^T T_vv
          dmma(d0, d1, ayb, tb[0], 0.0, 0.0);     // Ny^T T_dv
          if (!hi) {
            double* sb = RA_ + swz(g, 8 * h + 2 * t);
            st2(sb, v0, v1);
            st2(sb + SC, d0, d1);
          }
        }
        __syncwarp();
        // ---- backward x: columns n = 8h + g -> (i1, i2) = (g & 3, 2h + (g >> 2))
        double* cfc = cf + c * fp2 * CF;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const double* sb = RA_ + swz(g & 3, t + 8 * h + 4 * (g >> 2));
          double r0, r1;
          dmma(r0, r1, axb2, sb[SC], 0.0, 0.0);  // Nx'^T S_d
          dmma(r0, r1, axb, sb[0], r0, r1);      // + Nx^T S_v
          if (!hi) {  // res[i0 = g][i1 + 4 i2 = 8h + 2t + i] into the column footprint
#pragma unroll
            for (int i = 0; i < 2; ++i) {
              const int n = 8 * h + 2 * t + i;
              cfc[((offz + (n >> 2)) * P1 + (n & 3)) * P1 + g] += i ? r1 : r0;
            }
          }
        }
        __syncwarp();
      }
    }
  }
  __syncthreads();
  // ---- deterministic gather of the column footprints into the brick footprint
  const int nfoot = fp0 * fp1 * fp2;
  double* out = A.scratch + (size_t)b * VEC * nfoot;
  for (int i = tid; i < VEC * nfoot; i += NT) {
    const int jx = i % fp0;
    const int jy = (i / fp0) % fp1;
    const int jz = (i / (fp0 * fp1)) % fp2;
    const int c = i / nfoot;
    double s = 0.0;
#pragma unroll
    for (int e1 = 0; e1 < TY; ++e1) {
      const int ly = jy - soff[TX + e1];
      if (ly < 0 || ly >= P1) continue;
#pragma unroll
      for (int e0 = 0; e0 < TX; ++e0) {
        const int lx = jx - soff[e0];
        if (lx < 0 || lx >= P1) continue;
        s += colf[(((e1 * TX + e0) * VEC + c) * fp2 + jz) * CF + ly * P1 + lx];
      }
    }
    out[i] = s;
  }
}
