// 2D brick kernel (included by apply.cu): TX elements per row, TY rows per brick,
// Q threads per element; x contraction through shared memory, y in registers.
// TX is a template parameter (it sets the thread count and the shared-memory
// layout); TY is the plan's br.te[1], so small problems can take short bricks
// and still fill the GPU.
#pragma once

// Threads of a 2D brick CTA: RG row groups of TX * Q threads, each rounded up
// to whole warps when RG > 1 (a group synchronises on its own named barrier).
constexpr int brick2_group_threads(int tx, int q, int rg) { return rg == 1 ? tx * q : (tx * q + 31) / 32 * 32; }
constexpr int brick2_threads(int tx, int q, int rg) { return rg * brick2_group_threads(tx, q, rg); }

// The body of one brick (element rows [by*TY, +TY) x columns [bx*TX, +TX)).
// The host brick decomposition of the plan must use the same TX. WIDE: the CTA
// may have more than TX * Q threads (the persistent batched kernel). RG: row
// groups working on the brick's rows concurrently (group g takes rows g, g +
// RG, ...), each with its own stage buffers and its own copy of the brick
// footprint; the copies are summed in a fixed order at the end, so the result
// is bitwise reproducible. More rows in flight per CTA hide the latency of the
// stage hand-offs, which bounds this kernel when a brick's rows run one after
// another.
template <typename T, int P, int Q, int OPK, bool RAT, int MODE, int TX, bool WIDE = false, int RG = 1>
__device__ __forceinline__ void brick2_body(const BrickArgs<T>& A, const long long b) {
  constexpr int P1 = P + 1, PP = P1 * P1;
  constexpr int NE = TX, NQE = Q * Q, NT = NE * Q;
  constexpr int VEC = vec_op<OPK>() ? 2 : 1;
  constexpr int NG = GeoCount<OPK, RAT, 2>::value;
  constexpr int E0 = GeoCount<OPK_ELAST, RAT, 2>::elast;  // hyperelastic: start of the state
  constexpr bool HASV = RAT || MODE == MODE_LOAD;
  constexpr bool HESS = OPK == OPK_PLATE;
  constexpr int NK = HESS ? 3 : 2;      // 1D table kinds used
  constexpr int NCH = HESS ? 6 : 3;     // channels (v, g0, g1[, h00, h01, h11])
  constexpr int SX = P1 + 1;            // padded q0 stride
  constexpr int NTP = brick2_group_threads(TX, Q, RG);
  static_assert(RG == 1 || !WIDE, "row groups take the CTA's own thread count");

  if (A.state && A.state->done) return;
  const Bricks& br = A.br;
  const int fp0 = br.fp[0], fp1 = br.fp[1];
  const int TY = br.te[1];

  // A WIDE CTA may have more than NT threads (the persistent batched kernel runs
  // every degree in one CTA shape): cooperative loops stride by the CTA size,
  // and threads past NT own no element.
  const int tid = threadIdx.x, NTH = WIDE ? (int)blockDim.x : RG * NTP;
  const int rg = RG == 1 ? 0 : tid / NTP;   // this thread's row group
  const int tg = RG == 1 ? tid : tid % NTP;  // its thread index in the group
  const int NTG = RG == 1 ? NTH : NTP;       // the group's thread count (cooperative strides)

  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int accn = VEC * fp0 * fp1;
  const int gsz = 3 * Q * P1 + NE * NK * Q * SX + NE * VEC * PP + accn;  // one group's buffers
  T* stx = reinterpret_cast<T*>(smem_raw);   // [TX][3][Q][P1], shared by the groups
  T* sty = stx + TX * 3 * Q * P1 + rg * gsz; // [3][Q][P1]
  T* bufX = sty + 3 * Q * P1;                // [NE][NK][Q][SX]
  T* stage = bufX + NE * NK * Q * SX;        // [NE][VEC][PP]
  T* acc = stage + NE * VEC * PP;            // [VEC][fp1][fp0]
  int* soff = reinterpret_cast<int*>(stx + TX * 3 * Q * P1 + RG * gsz);
  // a barrier of this thread's row group
  auto gsync = [&]() {
    if constexpr (RG == 1)
      __syncthreads();
    else
      asm volatile("bar.sync %0, %1;" ::"r"(1 + rg), "r"(NTP) : "memory");
  };

  const int bx = (int)(b % br.nb[0]);
  const int by = (int)(b / br.nb[0]);
  const int cp0x = br.bcp0[0][bx], cp0y = br.bcp0[1][by];
  const int el = tg / Q, t = tg % Q;
  const int ex = bx * TX + el;
  const bool evalid = (!(WIDE || RG > 1) || el < TX) && ex < br.n_span[0];
  const long long slot_base = b * (long long)TY * NE;
  const int nlayers = min(TY, br.n_span[1] - by * TY);

  // The factors of one row of the brick are one contiguous tile (TX elements x
  // NG x NQE values; TX is a multiple of 16, so the tile is 16-byte aligned and
  // sized). When tiles are small (a few KB, as in batches of small instances,
  // where the kernel waits on latency) the bulk-copy engine brings the first
  // rows into L2 at the start and each row group's next row while it works on
  // the current one. Large tiles are not prefetched: with rows in flight on
  // every SM a prefetch runs tens of MB ahead of its use and is evicted before
  // the demand loads arrive (measured on a B200, plate 256^2, rows of 96 KB:
  // 274-280 MB read from DRAM against 198 MB without the prefetch, and 4-10 %
  // slower).
  constexpr unsigned ROW_BYTES = (unsigned)(NE * NG * NQE * sizeof(T));
  static_assert(ROW_BYTES % 16 == 0, "row tile of whole 16-byte units");
  constexpr bool GEO = MODE != MODE_LOAD && ROW_BYTES <= 32768;
  auto prefetch_row = [&](int ly) {
    prefetch_l2(A.geo + (size_t)(slot_base + (long long)ly * NE) * NG * NQE, ROW_BYTES);
  };
  if constexpr (GEO) {
    if (tid < RG && tid < nlayers) prefetch_row(tid);
  }

  for (int i = tid; i < TX * 3 * Q * P1; i += NTH) {
    int e = i / (3 * Q * P1), r = i % (3 * Q * P1);
    int sp = min(bx * TX + e, br.n_span[0] - 1);
    stx[i] = A.tab[0][(size_t)sp * 3 * Q * P1 + r];
  }
  if (tid < TX) {
    int e = bx * TX + tid;
    soff[tid] = e < br.n_span[0] ? br.first[0][e] - cp0x : -100000;
  }
  for (int i = tg; i < accn; i += NTG) acc[i] = T(0);
  if constexpr (RG > 1) __syncthreads();  // stx and soff, staged by every group, before the groups part
  const T* nx_v = stx + el * 3 * Q * P1;

  for (int ly_ = rg; ly_ < nlayers; ly_ += RG) {
    if constexpr (GEO) {
      if (tg == 0 && ly_ + RG < nlayers) prefetch_row(ly_ + RG);
    }
    const int ey = by * TY + ly_;
    const int fy = br.first[1][ey];
    const int offy = fy - cp0y;
    for (int i = tg; i < 3 * Q * P1; i += NTG) sty[i] = A.tab[1][(size_t)ey * 3 * Q * P1 + i];
    gsync();
    const long long slot = slot_base + (long long)ly_ * NE + el;
    const int fx = evalid ? br.first[0][ex] : 0;
    // this element's factors in the row tile [factor][q1][element][q0]: factor k of
    // point (q0, q1) at Grow[k * GST + q1 * NE * Q + q0]
    constexpr int GST = NE * NQE;
    const T* Grow = A.geo + (size_t)(slot_base + (long long)ly_ * NE) * NG * NQE + (size_t)el * Q;
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
        gsync();
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
        gsync();
      }
      if (evalid) {
#pragma unroll
        for (int q1 = 0; q1 < Q; ++q1) {
          const int q = t + Q * q1;
          const T* G = Grow + (size_t)q1 * (NE * Q) + t;
          if constexpr (OPK == OPK_SCALAR) {
            if constexpr (!RAT) {
              T k0 = G[0], k1 = G[GST], k2 = G[(2) * GST];
              T gx = g[0][1][q1], gy = g[0][2][q1];
              g[0][1][q1] = k0 * gx + k1 * gy;
              g[0][2][q1] = k1 * gx + k2 * gy;
              g[0][0][q1] = 0;
            } else {
              T m[6];
#pragma unroll
              for (int k = 0; k < 6; ++k) m[k] = G[(k) * GST];
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
                T m = G[((k++)) * GST];
                o[i + off] += m * s[j + off];
                if (j != i) o[j + off] += m * s[i + off];
              }
#pragma unroll
            for (int kk = 0; kk < 6; ++kk) g[0][kk][q1] = o[kk];
          } else {  // 2D elasticity
            T Ji[2][2] = {{G[0], G[GST]}, {G[(2) * GST], G[(3) * GST]}};
            T om = G[(4) * GST];
            T iW = 1, gW[2] = {0, 0};
            if constexpr (RAT) {
              iW = G[(5) * GST];
              gW[0] = G[(6) * GST];
              gW[1] = G[(7) * GST];
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
            T Sh[2][2];  // hyperelastic: om dP at the stored state
            if constexpr (OPK == OPK_HYPER) {
              const T M[2][2] = {{G[(E0) * GST], G[((E0 + 1)) * GST]}, {G[((E0 + 2)) * GST], G[((E0 + 3)) * GST]}};
              hyper_dP<T, 2>(M, G[((E0 + 4)) * GST], lam, mu, om, Gx, Sh);
            }
#pragma unroll
            for (int c = 0; c < 2; ++c) {
              T S0 = OPK == OPK_HYPER ? Sh[c][0] : om * (mu * (Gx[c][0] + Gx[0][c]) + (c == 0 ? lam * tr : T(0)));
              T S1 = OPK == OPK_HYPER ? Sh[c][1] : om * (mu * (Gx[c][1] + Gx[1][c]) + (c == 1 ? lam * tr : T(0)));
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
    } else if constexpr (MODE == MODE_RESID) {  // hyperelastic: the stored flux w P J^-T
      if (evalid) {
#pragma unroll
        for (int q1 = 0; q1 < Q; ++q1) {
          const int q = t + Q * q1;
          const T* G = Grow + (size_t)q1 * (NE * Q) + t;
          T iW = 1, gW[2] = {0, 0};
          if constexpr (RAT) {
            iW = G[(5) * GST];
            gW[0] = G[(6) * GST];
            gW[1] = G[(7) * GST];
          }
#pragma unroll
          for (int c = 0; c < VEC; ++c) {
            const T F0 = G[((E0 + 5 + 2 * c)) * GST], F1 = G[((E0 + 6 + 2 * c)) * GST];
#pragma unroll
            for (int k = 0; k < NCH; ++k) g[c][k][q1] = T(0);
            if constexpr (RAT) {
              g[c][0][q1] = -(F0 * gW[0] + F1 * gW[1]) * iW;
              g[c][1][q1] = F0 * iW;
              g[c][2][q1] = F1 * iW;
            } else {
              g[c][1][q1] = F0;
              g[c][2][q1] = F1;
            }
          }
        }
      }
    }

    if constexpr (MODE == MODE_APPLY || MODE == MODE_LOAD || MODE == MODE_RESID) {
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
        gsync();
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
        gsync();
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
            const T* G = Grow + (size_t)q1 * (NE * Q) + q0;
            if constexpr (OPK == OPK_SCALAR || OPK == OPK_PLATE) {
              constexpr int n = OPK == OPK_SCALAR ? (RAT ? 3 : 2) : (RAT ? 6 : 5);
              constexpr int off = RAT ? 0 : 1;
              int k = 0;
              T acc_ = 0;
#pragma unroll
              for (int i = 0; i < n; ++i)
#pragma unroll
                for (int j = i; j < n; ++j) {
                  T m = G[((k++)) * GST];
                  acc_ += (i == j ? T(1) : T(2)) * m * s[i + off] * s[j + off];
                }
              d[0] += acc_;
            } else {
              T Ji[2][2] = {{G[0], G[GST]}, {G[(2) * GST], G[(3) * GST]}};
              T om = G[(4) * GST];
              T gp[2] = {s[1], s[2]};
              if constexpr (RAT) {
                T iW = G[(5) * GST];
                gp[0] = (gp[0] - s[0] * G[(6) * GST]) * iW;
                gp[1] = (gp[1] - s[0] * G[(7) * GST]) * iW;
              }
              T gx[2] = {Ji[0][0] * gp[0] + Ji[0][1] * gp[1], Ji[1][0] * gp[0] + Ji[1][1] * gp[1]};
              T n2 = gx[0] * gx[0] + gx[1] * gx[1];
              if constexpr (OPK == OPK_HYPER) {
                // mu |g|^2 + (c + lambda) (F^-T_c . g)^2 at the stored state
                const T ch = G[((E0 + 4)) * GST] + (T)A.lam;
#pragma unroll
                for (int c = 0; c < VEC; ++c) {
                  const T mg = G[((E0 + 2 * c)) * GST] * gx[0] + G[((E0 + 2 * c + 1)) * GST] * gx[1];
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
            T w = A.wgts[(long long)br.n_cp[0] * (fy + a1) + fx + a0];
            wsq = w * w;
          }
#pragma unroll
          for (int c = 0; c < VEC; ++c) stage[(el * VEC + c) * PP + a0 * P1 + a1] = d[c] * wsq;
        }
      }
      gsync();
    }
    // gather the row into the brick footprint
    {
      const int nfoot = VEC * fp0 * P1;
      for (int i = tg; i < nfoot; i += NTG) {
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
    gsync();
  }
  T* out = A.scratch + (size_t)b * accn;
  if constexpr (RG == 1) {
    for (int i = tid; i < accn; i += NTH) out[i] = acc[i];
  } else {
    __syncthreads();
    const T* acc0 = stx + TX * 3 * Q * P1 + 3 * Q * P1 + NE * NK * Q * SX + NE * VEC * PP;  // group 0's footprint
    for (int i = tid; i < accn; i += NTH) {
      T v = acc0[i];
#pragma unroll
      for (int r = 1; r < RG; ++r) v += acc0[(size_t)r * gsz + i];
      out[i] = v;
    }
  }
}

template <typename T, int P, int Q, int OPK, bool RAT, int MODE, int TX, int RG>
__global__ void __launch_bounds__(brick2_threads(TX, Q, RG)) k_brick2(BrickArgs<T> A) {
  brick2_body<T, P, Q, OPK, RAT, MODE, TX, false, RG>(A, blockIdx.x);
}

// Many instances in one launch: block i processes brick work[i].y of instance
// work[i].x, whose arguments are args[work[i].x]; instances already converged
// (states[inst].done) are skipped.
template <typename T, int P, int Q, int OPK, bool RAT, int MODE, int TX, int RG>
__global__ void __launch_bounds__(brick2_threads(TX, Q, RG))
    k_brick2_batch(const BrickArgs<T>* __restrict__ args, const int2* __restrict__ work,
                   const CgState* __restrict__ states) {
  __shared__ BrickArgs<T> sA;
  const int2 w = work[blockIdx.x];
  if (states && states[w.x].done) return;
  if (threadIdx.x == 0) sA = args[w.x];
  __syncthreads();
  brick2_body<T, P, Q, OPK, RAT, MODE, TX, false, RG>(sA, w.y);
}


// Persistent batched 2D apply. A fixed grid of CTAs takes (instance, brick,
// degree) items off one work list holding the bricks of every instance of every
// degree (sorted by the host: highest degree and largest instance first), so
// one launch covers the whole batch and short instances fill the gaps left by
// long ones. Every instance uses rows of 32 elements; the CTA has 32 x (p_max
// + 1) threads and a degree-p item runs on the first 32 (p + 1) of them.
// The work counter resets itself: each CTA fetches until it draws an index past
// the list, so a launch performs exactly n_work + gridDim.x increments and
// atomicInc wraps the counter back to 0 on the last one.
constexpr int PERSIST_TX = PERSIST2_TX;
constexpr int PERSIST_THREADS = PERSIST_TX * 6;  // degrees 1..5

template <typename T, int OPK, bool RAT, int MODE>
__global__ void __launch_bounds__(PERSIST_THREADS)
    k_brick2_persist(const BrickArgs<T>* __restrict__ args, const int4* __restrict__ work, int n_work,
                     unsigned* __restrict__ next, const CgState* __restrict__ states) {
  __shared__ BrickArgs<T> sA;
  __shared__ int4 item;
  static_assert(sizeof(BrickArgs<T>) % 8 == 0, "BrickArgs copy in 8-byte words");
  for (;;) {
    if (threadIdx.x == 0) {
      const unsigned i = atomicInc(next, (unsigned)n_work + gridDim.x - 1u);
      item = i < (unsigned)n_work ? work[i] : make_int4(-1, 0, 0, 0);
    }
    __syncthreads();
    const int4 it = item;
    if (it.x < 0) break;
    // the instance's arguments, copied by the whole CTA
    {
      const unsigned long long* src = reinterpret_cast<const unsigned long long*>(args + it.x);
      unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sA);
      for (int w = threadIdx.x; w < (int)(sizeof(BrickArgs<T>) / 8); w += blockDim.x) dst[w] = src[w];
    }
    __syncthreads();
    if (!(states && states[it.x].done)) {
      switch (it.z) {
        case 1: brick2_body<T, 1, 2, OPK, RAT, MODE, PERSIST_TX, true>(sA, it.y); break;
        case 2: brick2_body<T, 2, 3, OPK, RAT, MODE, PERSIST_TX, true>(sA, it.y); break;
        case 3: brick2_body<T, 3, 4, OPK, RAT, MODE, PERSIST_TX, true>(sA, it.y); break;
        case 4: brick2_body<T, 4, 5, OPK, RAT, MODE, PERSIST_TX, true>(sA, it.y); break;
        case 5: brick2_body<T, 5, 6, OPK, RAT, MODE, PERSIST_TX, true>(sA, it.y); break;
        default: break;
      }
    }
    __syncthreads();  // item and sA are rewritten by the next fetch
  }
}
