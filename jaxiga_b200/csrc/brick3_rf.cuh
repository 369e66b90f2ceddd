// FP64 tensor-core brick apply at degree 3 with 4 Gauss points per direction,
// scalar operator (Poisson / Darcy) and linear elasticity, polynomial weights,
// with the element data kept in MMA register fragments from the DOF load to
// the residual. Included by apply.cu inside namespace jxb.
//
// The sum factorisation of one element runs in one warp with no shared-memory
// hand-off between stages. It rests on two facts of mma.sync.m8n8k4.f64
// (lane l, g = l >> 2, t = l & 3; A[g][t], B[t][g], D[g][2t + i]):
//   * the two D entries a lane holds, D[g][2t] and D[g][2t+1], are each a
//     valid A fragment (A[g][t]) of an 8 x 4 operand whose k index is t, so a
//     product can feed the next contraction directly when the next contracted
//     index is carried by t (the "column pair" trick), and
//   * a D fragment read as B[t][g] is the transpose of the same trick.
// The stages, per displacement component:
//   forward x  D1_j[(t0,q0)][2 i1 + i] = sum_i0 N^t0_x(q0,i0) u[i0][i1][2j+i]     2 MMAs
//   forward y  D2_i2[(t0,q0)][2 q1 + t1] = sum_i1 D1[(t0,q0)][i1; i2] N^t1_y(q1,i1)  4 MMAs
//   forward z  in the lane: the lane holds D2_i2 for all four i2 at its (q0, q1),
//              so d/dzeta, d/deta (t0 = value lanes) and d/dxi (t0 = derivative
//              lanes) at the four q2 are 32 scalar FMAs; one exchange with the
//              lane 16 away leaves each lane the full gradient at 2 points
//   point operator on those 2 points (factors read straight from HBM)
//   backward z in the lane (the exchange reversed, 32 FMAs)
//   backward y S_i2^T[i1][(t0,q0)] = sum_(t1,q1) N^t1_y(q1,i1) T_i2[(t0,q0)][(t1,q1)]
//              with T as the B operand; two i2 share one accumulator, the
//              first in rows 0-3 and the second in rows 4-7          8 MMAs
//   backward x res[(i2,i1)][i0] by the column pair trick on S^T, the two i2
//              pairs in columns 0-3 and 4-7 of one accumulator     4 MMAs
// so 18 MMAs per component (the staged kernel takes 28) and no shared-memory
// traffic except the z tables (broadcast reads) and the residual's add into
// the column footprint. CTA layout, column footprints and the deterministic
// gather are those of the staged kernel: 16 warps, each owning a column of 8
// elements along z in a 4 x 4 x 8 brick.

namespace brf {
constexpr int P1 = 4, Q = 4, NQE = 64;
constexpr int TX = 4, TY = 4, CZ = 8, NE = TX * TY, NT = NE * 32;
constexpr int ZT = 2 * Q * P1;  // one layer's z tables: [kind (value, d/dzeta)][q2][i2]
constexpr int CF = P1 * P1;     // one z row of a column footprint: [i1][i0]
}  // namespace brf

// 16-byte shared-memory load the compiler may not merge with an earlier load
// of the same address (the z tables are re-read in the backward stages rather
// than held in 64 registers across the point operator).
__device__ __forceinline__ double2 lds2(const double2* p) {
  double2 v;
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];"
               : "=d"(v.x), "=d"(v.y)
               : "r"((unsigned)__cvta_generic_to_shared(p)));
  return v;
}

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// One-shot completion barrier of a bulk copy (count 1: the issuing lane's arrive).
__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}

// Bulk copy (no tensor map, no multicast) of `bytes` from this GPU's global
// memory into this CTA's shared memory, completing on `bar`. Both addresses
// 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // earlier generic reads of dst come first
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Wait for phase `parity` of `bar` to complete, giving up after `limit` polls.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, int limit) {
  for (int i = 0; i < limit; ++i) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// STAGE: each warp's next factor tile is copied into shared memory by the bulk
// copy engine while the warp finishes the current element; otherwise the tile
// is prefetched into L2 and read from there.
template <int OPK, bool STAGE>
static size_t smem3_rf(const Bricks& br) {
  using namespace brf;
  constexpr int VEC = OPK == OPK_ELAST ? 3 : 1;
  constexpr int NG = OPK == OPK_ELAST ? 10 : 6;
  const size_t n = (size_t)CZ * ZT + (STAGE ? (size_t)NE * NG * NQE + NE : 0) + (size_t)NE * VEC * br.fp[2] * CF;
  return n * sizeof(double) + (TX + TY) * sizeof(int) + 64;
}

constexpr int RF_WAIT_LIMIT = 1 << 22;  // polls of a bulk-copy barrier before the kernel reports a stall

template <int OPK, int MINB, bool STAGE>
__global__ void __launch_bounds__(brf::NT, MINB) k_brick3_rf(BrickArgs<double> A) {
  using namespace brf;
  constexpr int VEC = OPK == OPK_ELAST ? 3 : 1;
  constexpr int NG = OPK == OPK_ELAST ? 10 : 6;  // factors per point: J^-1 and w|J| / the symmetric metric
  constexpr unsigned FULL = 0xffffffffu;
  if (A.state && A.state->done) return;
  const Bricks& br = A.br;
  const int fp0 = br.fp[0], fp1 = br.fp[1], fp2 = br.fp[2];

  extern __shared__ __align__(128) unsigned char smem_raw[];
  double* ztab = reinterpret_cast<double*>(smem_raw);  // [CZ][ZT]
  double* fbuf = ztab + CZ * ZT;                        // STAGE: [NE][NG][NQE] factor tiles
  unsigned long long* fbar = reinterpret_cast<unsigned long long*>(fbuf + (STAGE ? NE * NG * NQE : 0));  // [NE]
  double* colf = reinterpret_cast<double*>(fbar + (STAGE ? NE : 0));  // [NE][VEC][fp2][i1][i0] column footprints
  int* soff = reinterpret_cast<int*>(colf + NE * VEC * fp2 * CF);

  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const bool lo = lane < 16;  // t0 = value lanes (g < 4); the others carry t0 = derivative
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
  // the brick's z tables (values and first derivatives, the first 32 of a span's 48)
  for (int i = tid; i < nlayers * ZT; i += NT) {
    const int lz = i / ZT, r = i - lz * ZT;
    ztab[i] = A.tab[2][(size_t)(bz * cz + lz) * 3 * Q * P1 + r];
  }
  double* cf = colf + w * VEC * fp2 * CF;
  for (int i = lane; i < VEC * fp2 * CF; i += 32) cf[i] = 0.0;
  double* fw = fbuf + w * NG * NQE;
  unsigned long long* bar = fbar + w;
  bool stalled = false;
  if constexpr (STAGE) {
    if (lane == 0) mbar_init(bar);
  }
  __syncthreads();

  if (evalid) {
    const double* tx_ = A.tab[0] + (size_t)ex * 3 * Q * P1;
    const double* ty_ = A.tab[1] + (size_t)ey * 3 * Q * P1;
    // forward x, A: N^(g>>2)_x(q0 = g & 3, i0 = t)
    const double ax = tx_[lane];
    // forward y, B[i1 = t][(q1, t1) = (g >> 1, g & 1)]: N^t1_y(q1, i1)
    const double byf = ty_[((g & 1) * Q + (g >> 1)) * P1 + t];
    // backward y, A_j[i1 = g & 3][q1 = t]: N^j_y(q1, i1), rows 0-3 or 4-7 (j = 1 at + Q P1)
    const double* byp = ty_ + t * P1 + (g & 3);
    // backward x, B_i[k = t][i0 = g & 3] for (t0, q0) = (t >> 1, 2 (t & 1) + i), columns 0-3 or 4-7 (i = 1 at + P1)
    const double* bxp = tx_ + ((t >> 1) * Q + 2 * (t & 1)) * P1 + (g & 3);
    // held in registers in the one-CTA-per-SM build, re-read (L1 hits) where registers are scarce
    double byr[2] = {0.0, 0.0}, bxr[2] = {0.0, 0.0};
    if constexpr (MINB == 1) {
      byr[0] = byp[0];
      byr[1] = byp[Q * P1];
      bxr[0] = bxp[0];
      bxr[1] = bxp[P1];
    }
    auto by_tab = [&](int j) { return MINB == 1 ? byr[j] : __ldg(byp + j * Q * P1); };
    auto bx_tab = [&](int i) { return MINB == 1 ? bxr[i] : __ldg(bxp + i * P1); };
    const bool top = g < 4;

    const long long ncx = br.n_cp[0], nxy = (long long)br.n_cp[0] * br.n_cp[1];
    // this lane's input entries (forward-x B fragments): i0 = t, i1 = g >> 1, i2 = 2j + (g & 1)
    const long long cxy = (long long)(br.first[0][ex] + t) + ncx * (br.first[1][ey] + (g >> 1));
    auto load_in = [&](int ez_, double (&u)[VEC][2]) {
      const long long c0 = cxy + nxy * (br.first[2][ez_] + (g & 1));
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
    // this lane's two points: (q0, q1, q2) = (g & 3, t, 2 (lane >> 4) + i), index q0 + 4 q1 + 16 q2
    const int qa = (g & 3) + 4 * t + 32 * (lane >> 4);
    // its residual entries: i0 = 2 (t & 1) + {0, 1}, i1 = g & 3, i2 = 2 (t >> 1) + (g >> 2)
    const int ro = ((2 * (t >> 1) + (g >> 2)) * P1 + (g & 3)) * P1 + 2 * (t & 1);
    if (lane == 0) {
      if constexpr (STAGE)
        bulk_g2s(fw, A.geo + (size_t)(slot_base + w) * NG * NQE, NG * NQE * sizeof(double), bar);
      else
        prefetch_l2(A.geo + (size_t)(slot_base + w) * NG * NQE, NG * NQE * sizeof(double));
    }
    double un[VEC][2];
    load_in(bz * cz, un);
    for (int lz = 0; lz < nlayers; ++lz) {
      const int ez = bz * cz + lz;
      const int offz = br.first[2][ez] - cp0z;
      const long long slot = slot_base + (long long)lz * NE + w;
      if (!STAGE && lane == 0 && lz + 1 < nlayers)
        prefetch_l2(A.geo + (size_t)(slot + NE) * NG * NQE, NG * NQE * sizeof(double));
      double u[VEC][2];
#pragma unroll
      for (int c = 0; c < VEC; ++c) {
        u[c][0] = un[c][0];
        u[c][1] = un[c][1];
      }
      if (lz + 1 < nlayers) load_in(ez + 1, un);
      const double2* zt = reinterpret_cast<const double2*>(ztab + lz * ZT);  // [kind][q2][i2 pair]
      const double* G = STAGE ? fw + qa : A.geo + (size_t)slot * NG * NQE + qa;
      double GX[VEC][2], GY[VEC][2], GZ[VEC][2];
#pragma unroll
      for (int c = 0; c < VEC; ++c) {
        // ---- forward x and y
        double d2[4][2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          double e0, e1;
          dmma(e0, e1, ax, u[c][j], 0.0, 0.0);
          dmma(d2[2 * j][0], d2[2 * j][1], e0, byf, 0.0, 0.0);
          dmma(d2[2 * j + 1][0], d2[2 * j + 1][1], e1, byf, 0.0, 0.0);
        }
        // ---- forward z in the lane: a = N_z . (value lanes: t1 = d, else t1 = v), b = N'_z . (t1 = v)
        double sa[4], a4[4], b4[4];
#pragma unroll
        for (int i2 = 0; i2 < 4; ++i2) sa[i2] = lo ? d2[i2][1] : d2[i2][0];
#pragma unroll
        for (int q2 = 0; q2 < 4; ++q2) {
          const double2 n01 = lds2(zt + q2 * 2), n23 = lds2(zt + q2 * 2 + 1);
          const double2 d01 = lds2(zt + 8 + q2 * 2), d23 = lds2(zt + 8 + q2 * 2 + 1);
          a4[q2] = n01.x * sa[0] + n01.y * sa[1] + n23.x * sa[2] + n23.y * sa[3];
          b4[q2] = d01.x * d2[0][0] + d01.y * d2[1][0] + d23.x * d2[2][0] + d23.y * d2[3][0];
        }
        // value lanes hold d/deta (a) and d/dzeta (b), derivative lanes d/dxi (a), at q2 = 0..3;
        // keep q2 = 0, 1 in the value lanes and q2 = 2, 3 in the others
        const double s0 = __shfl_xor_sync(FULL, lo ? a4[2] : a4[0], 16);
        const double s1 = __shfl_xor_sync(FULL, lo ? a4[3] : a4[1], 16);
        const double s2 = __shfl_xor_sync(FULL, b4[2], 16);
        const double s3 = __shfl_xor_sync(FULL, b4[3], 16);
        GX[c][0] = lo ? s0 : a4[2];
        GX[c][1] = lo ? s1 : a4[3];
        GY[c][0] = lo ? a4[0] : s0;
        GY[c][1] = lo ? a4[1] : s1;
        GZ[c][0] = lo ? b4[0] : s2;
        GZ[c][1] = lo ? b4[1] : s3;
      }
      if constexpr (STAGE) {
        if (!stalled && !mbar_wait(bar, lz & 1, RF_WAIT_LIMIT)) stalled = true;
      }
      auto ld = [&](const double* q) { return STAGE ? *q : __ldg(q); };
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
            for (int a = 0; a < 3; ++a) Ji[k][a] = ld(G + (k * 3 + a) * NQE + 16 * i);
          const double om = ld(G + 9 * NQE + 16 * i);
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
          const double* Gi = G + 16 * i;
          const double k0 = ld(Gi), k1 = ld(Gi + NQE), k2 = ld(Gi + 2 * NQE);
          const double k3 = ld(Gi + 3 * NQE), k4 = ld(Gi + 4 * NQE), k5 = ld(Gi + 5 * NQE);
          F[0][0][i] = k0 * GX[0][i] + k1 * GY[0][i] + k2 * GZ[0][i];
          F[0][1][i] = k1 * GX[0][i] + k3 * GY[0][i] + k4 * GZ[0][i];
          F[0][2][i] = k2 * GX[0][i] + k4 * GY[0][i] + k5 * GZ[0][i];
        }
      }
      // keeps the backward stages' table reads below the point operator: scheduled
      // above it, they would hold 16 more doubles in registers across it. With
      // STAGE, every lane is done with the factor tile here, so the copy of the
      // next layer's tile may overwrite it.
      __syncwarp();
      if constexpr (STAGE) {
        if (lane == 0 && lz + 1 < nlayers && !stalled)
          bulk_g2s(fw, A.geo + (size_t)(slot + NE) * NG * NQE, NG * NQE * sizeof(double), bar);
      }
      double* cfl = cf + offz * CF + ro;
#pragma unroll
      for (int c = 0; c < VEC; ++c) {
        // ---- the exchange reversed: value lanes collect F_eta, F_zeta at q2 = 0..3,
        // derivative lanes F_xi
        const double e0 = __shfl_xor_sync(FULL, lo ? F[c][0][0] : F[c][1][0], 16);
        const double e1 = __shfl_xor_sync(FULL, lo ? F[c][0][1] : F[c][1][1], 16);
        const double e2 = __shfl_xor_sync(FULL, F[c][2][0], 16);
        const double e3 = __shfl_xor_sync(FULL, F[c][2][1], 16);
        const double r4[4] = {lo ? F[c][1][0] : e0, lo ? F[c][1][1] : e1, lo ? e0 : F[c][0][0],
                              lo ? e1 : F[c][0][1]};
        const double p4[4] = {F[c][2][0], F[c][2][1], e2, e3};
        // backward y (T as B) and backward x (column pair trick). The two i2 of a
        // pair land in rows 0-3 and 4-7 and the two pairs in columns 0-3 and 4-7
        // of one result; separate accumulators summed at the end keep the MMA
        // chains two deep.
        double rp[2][2];
#pragma unroll
        for (int p = 0; p < 2; ++p) {
          // ---- backward z in the lane for i2 = 2p, 2p + 1: X = N_z^T r, Y = N'_z^T p
          double X[2] = {0.0, 0.0}, Y[2] = {0.0, 0.0};
#pragma unroll
          for (int q2 = 0; q2 < 4; ++q2) {
            const double2 n = lds2(zt + q2 * 2 + p), d = lds2(zt + 8 + q2 * 2 + p);
            X[0] += n.x * r4[q2];
            X[1] += n.y * r4[q2];
            Y[0] += d.x * p4[q2];
            Y[1] += d.y * p4[q2];
          }
          // T_i2[(t0, q0)][(t1 = v | d, q1)]: value lanes (v,v) = Y, (v,d) = X; derivative lanes (d,v) = X, (d,d) = 0
          const double by0 = by_tab(0), by1 = by_tab(1);
          double sa0, sa1, sb0, sb1;
          dmma(sa0, sa1, top ? by0 : 0.0, lo ? Y[0] : X[0], 0.0, 0.0);
          dmma(sb0, sb1, top ? 0.0 : by0, lo ? Y[1] : X[1], 0.0, 0.0);
          dmma(sa0, sa1, top ? by1 : 0.0, lo ? X[0] : 0.0, sa0, sa1);
          dmma(sb0, sb1, top ? 0.0 : by1, lo ? X[1] : 0.0, sb0, sb1);
          const bool blk = top == (p == 0);
          dmma(rp[p][0], rp[p][1], sa0 + sb0, blk ? bx_tab(0) : 0.0, 0.0, 0.0);
          dmma(rp[p][0], rp[p][1], sa1 + sb1, blk ? bx_tab(1) : 0.0, rp[p][0], rp[p][1]);
        }
        const double r0 = rp[0][0] + rp[1][0], r1 = rp[0][1] + rp[1][1];
        // res[i0 = 2 (t & 1) + {0,1}][i1 = g & 3][i2 = 2 (t >> 1) + (g >> 2)] into the column footprint
        double2* dst = reinterpret_cast<double2*>(cfl + c * fp2 * CF);
        double2 cur = *dst;
        cur.x += r0;
        cur.y += r1;
        *dst = cur;
      }
      __syncwarp();  // the next layer's element overlaps this one's footprint rows
    }
  }
  if constexpr (STAGE) {
    // a copy that did not complete in time: report it, poison this brick's output
    // (so a solve sees a non-finite K.u) and give the copy one more bounded wait
    stalled = __any_sync(FULL, stalled);
    if (stalled) {
      if (lane == 0) {
        atomicExch(A.err, 1);
        mbar_wait(bar, 0, RF_WAIT_LIMIT);
        mbar_wait(bar, 1, RF_WAIT_LIMIT);
      }
      for (int i = lane; i < VEC * fp2 * CF; i += 32) cf[i] = __longlong_as_double(0x7ff8000000000000LL);
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
