// A 3D convolutional network on the control-point grid, used as a learned
// preconditioner inside flexible CG (the fourth AI-systems form of the
// solver; it has no counterpart in the reference, whose preconditioner is
// Jacobi, src/jaxiga/solvers/linear.py:419-431).
//
// Topology: a U-Net with L levels (2..6) and channels c[0..L-1]; every conv
// is 3x3x3 with zero padding unless marked 1x1, "relu" = rectified output:
//
//   encoder, l = 0..L-2:  x -> c[l] relu;  c[l] -> c[l] relu = s_l;  x = pool(s_l)
//   bottom, level L-1:    x -> c[L-1] relu;  two more c[L-1] -> c[L-1] relu
//   decoder, l = L-2..0:  y = up(y);  m_l = 1x1 c[l+1] -> c[l] (y) + s_l;
//                         y = c[l] -> c[l] relu (m_l)
//   output:               c[0] -> 4 (linear; the first out_ch channels are used)
//
// Level l has ceil(n/2^l) voxels per direction. Pooling averages the (up to
// eight) children of a coarse voxel; upsampling copies a coarse voxel to its
// children. Activations are [channel][z][y][x], FP32.
//
// With input pooling (jxb_cnn_set_input_pooling) the input is pooled once and
// the U-Net runs on the half-resolution grid; its output is interpolated back
// (trilinear: a piecewise-constant correction would carry its block edges into
// the energy norm).
// The network then acts on the smooth part of the residual only, at about an
// eighth of the finest level's cost.
//
// Convolutions (forward and data gradient) use one kernel: a CTA computes a
// 16 x 8 x 4 voxel tile for a block of up to 16 output channels (narrower on
// small grids, so that the grid still fills the GPU, and on the coarsest
// grids with the input channels split over CTAs and the partial sums added in
// a fixed order by a second kernel); each thread
// owns one (x, y) column of 4 voxels along z, so the three z taps reuse
// registers and a warp reads consecutive x from shared memory. Input halos
// and weights are staged in shared memory four input channels at a time.
// Weight gradients are per-tile partials (one thread per input channel and
// tap, the block's output channels in registers) summed over tiles in a
// fixed order, so training is bitwise reproducible run to run.
#include <cuda_bf16.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <string>
#include <vector>

#include "jxb_internal.cuh"

namespace jxb {
namespace cnn {

constexpr int CTX = 16, CTY = 8, CTZ = 4;  // voxel tile of the conv kernels
constexpr int CT = CTX * CTY;              // threads per CTA (one z column of CTZ voxels each)
constexpr int CIB = 4;                     // input channels staged per pass
constexpr int MAXL = 6;
constexpr int MAXC = 64;  // widest supported layer

struct Dims {
  int nx, ny, nz;
  __host__ __device__ long long vox() const { return (long long)nx * ny * nz; }
};

static Dims halve(Dims d) { return {(d.nx + 1) / 2, (d.ny + 1) / 2, (d.nz + 1) / 2}; }
static long long n_tiles(Dims d) {
  return (long long)((d.nx + CTX - 1) / CTX) * ((d.ny + CTY - 1) / CTY) * ((d.nz + CTZ - 1) / CTZ);
}

// out[co] = b[co] + sum_ci sum_k w[co][ci][k] in[ci](v + k)   (+ add[co]) (relu)
// for co in [co0, co0 + COB), co0 = blockIdx.y * COB. K = 3 (27 taps,
// k = dx + 3 dy + 9 dz) or 1. beta: out = beta * out + result.
// Split input channels (small grids): block z sums channels [z cps, (z+1) cps)
// into its own slab out + z * co_n * vox, bias/add/relu/beta left to k_sum_split.
template <int K, int COB>
__global__ void __launch_bounds__(CT) k_conv(Dims d, int ci_n, const float* __restrict__ in, const float* __restrict__ w,
                                            const float* __restrict__ bias, const float* __restrict__ add, int relu,
                                            float beta, float* __restrict__ out, int cps, int co_n) {
  constexpr int R = K / 2, HX = CTX + 2 * R, HY = CTY + 2 * R, HZ = CTZ + 2 * R, KK = K * K * K;
  constexpr int HV = HX * HY * HZ;
  __shared__ __align__(16) float tile[CIB * HV];
  __shared__ __align__(16) float sw[CIB * KK * COB];  // [c][k][co]
  const int tx = threadIdx.x % CTX, ty = threadIdx.x / CTX;
  const int ntx = (d.nx + CTX - 1) / CTX, nty = (d.ny + CTY - 1) / CTY;
  const int bx = blockIdx.x % ntx, by = (blockIdx.x / ntx) % nty, bz = blockIdx.x / (ntx * nty);
  const int co0 = blockIdx.y * COB;
  const long long vox = d.vox();
  const int cb = blockIdx.z * cps, ce = min(ci_n, cb + cps);
  out += (long long)blockIdx.z * co_n * vox;
  float acc[CTZ][COB];
#pragma unroll
  for (int c = 0; c < COB; ++c) {
    const float b0 = bias ? bias[co0 + c] : 0.f;
#pragma unroll
    for (int j = 0; j < CTZ; ++j) acc[j][c] = b0;
  }
  for (int ci0 = cb; ci0 < ce; ci0 += CIB) {
    const int nc = min(CIB, ce - ci0);
    for (int i = threadIdx.x; i < nc * HV; i += CT) {
      const int c = i / HV, r = i % HV;
      const int hx = r % HX, hy = (r / HX) % HY, hz = r / (HX * HY);
      const int gx = bx * CTX + hx - R, gy = by * CTY + hy - R, gz = bz * CTZ + hz - R;
      float v = 0.f;
      if (gx >= 0 && gy >= 0 && gz >= 0 && gx < d.nx && gy < d.ny && gz < d.nz)
        v = in[(long long)(ci0 + c) * vox + ((long long)gz * d.ny + gy) * d.nx + gx];
      tile[i] = v;
    }
    for (int i = threadIdx.x; i < nc * KK * COB; i += CT) {
      const int c = i / (KK * COB), k = (i / COB) % KK, o = i % COB;
      sw[i] = w[((long long)(co0 + o) * ci_n + ci0 + c) * KK + k];
    }
    __syncthreads();
    for (int c = 0; c < nc; ++c) {
      const float* tc = tile + c * HV;
      const float* wc = sw + c * KK * COB;
#pragma unroll
      for (int dy = 0; dy < K; ++dy) {
#pragma unroll
        for (int dx = 0; dx < K; ++dx) {
          float v[HZ];
#pragma unroll
          for (int j = 0; j < HZ; ++j) v[j] = tc[(j * HY + ty + dy) * HX + tx + dx];
#pragma unroll
          for (int dz = 0; dz < K; ++dz) {
            const float4* w4 = reinterpret_cast<const float4*>(wc + ((dz * K + dy) * K + dx) * COB);
#pragma unroll
            for (int c4 = 0; c4 < COB / 4; ++c4) {
              const float4 ww = w4[c4];
#pragma unroll
              for (int j = 0; j < CTZ; ++j) {
                const float a = v[j + dz];
                acc[j][4 * c4 + 0] = fmaf(ww.x, a, acc[j][4 * c4 + 0]);
                acc[j][4 * c4 + 1] = fmaf(ww.y, a, acc[j][4 * c4 + 1]);
                acc[j][4 * c4 + 2] = fmaf(ww.z, a, acc[j][4 * c4 + 2]);
                acc[j][4 * c4 + 3] = fmaf(ww.w, a, acc[j][4 * c4 + 3]);
              }
            }
          }
        }
      }
    }
    __syncthreads();
  }
  const int x = bx * CTX + tx, y = by * CTY + ty;
  if (x >= d.nx || y >= d.ny) return;
#pragma unroll
  for (int j = 0; j < CTZ; ++j) {
    const int z = bz * CTZ + j;
    if (z >= d.nz) break;
    const long long o = ((long long)z * d.ny + y) * d.nx + x;
#pragma unroll
    for (int c = 0; c < COB; ++c) {
      float v = acc[j][c];
      const long long idx = (long long)(co0 + c) * vox + o;
      if (add) v += add[idx];
      if (relu) v = fmaxf(v, 0.f);
      out[idx] = beta != 0.f ? beta * out[idx] + v : v;
    }
  }
}

// out = relu(bias + sum_z part[z] (+ add)) (beta: out = beta * out + result),
// the split-channel slabs summed in a fixed order
__global__ void k_sum_split(long long vox, int co_n, int nsplit, const float* __restrict__ part,
                            const float* __restrict__ bias, const float* __restrict__ add, int relu, float beta,
                            float* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= vox * co_n) return;
  float v = bias ? bias[i / vox] : 0.f;
  for (int z = 0; z < nsplit; ++z) v += part[(long long)z * co_n * vox + i];
  if (add) v += add[i];
  if (relu) v = fmaxf(v, 0.f);
  out[i] = beta != 0.f ? beta * out[i] + v : v;
}

// 1x1 convolution, one thread per voxel and a block of COB output channels:
// out[co](v) = b[co] + sum_ci w[co][ci] in[ci](v) (+ add) (relu), beta as k_conv.
// The input channels are summed in the order k_conv uses, so results match it;
// without a halo to stage, reading straight from global memory is coalesced
// and keeps the kernel at the bandwidth of its reads and writes.
// UP: the input is the coarse grid c and in(v) its upsampled value (the coarse
// voxel holding v), so the decoder never writes the upsampled activation.
template <int COB, bool UP>
__global__ void __launch_bounds__(256) k_conv1(Dims d, Dims c, int ci_n, const float* __restrict__ in,
                                               const float* __restrict__ w, const float* __restrict__ bias,
                                               const float* __restrict__ add, int relu, float beta,
                                               float* __restrict__ out) {
  const long long vox = d.vox();
  __shared__ float sw[64 * COB];  // [ci][co], ci_n <= 64
  const int co0 = blockIdx.y * COB;
  for (int i = threadIdx.x; i < ci_n * COB; i += blockDim.x) sw[i] = w[(long long)(co0 + i % COB) * ci_n + i / COB];
  __syncthreads();
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= vox) return;
  long long src = v, svox = vox;
  if constexpr (UP) {
    const int X = (int)(v % d.nx), Y = (int)((v / d.nx) % d.ny), Z = (int)(v / ((long long)d.nx * d.ny));
    src = ((long long)(Z >> 1) * c.ny + (Y >> 1)) * c.nx + (X >> 1);
    svox = c.vox();
  }
  float acc[COB];
#pragma unroll
  for (int c = 0; c < COB; ++c) acc[c] = bias ? bias[co0 + c] : 0.f;
  for (int ci = 0; ci < ci_n; ++ci) {
    const float a = in[(long long)ci * svox + src];
#pragma unroll
    for (int c = 0; c < COB; ++c) acc[c] = fmaf(sw[ci * COB + c], a, acc[c]);
  }
#pragma unroll
  for (int c = 0; c < COB; ++c) {
    const long long idx = (long long)(co0 + c) * vox + v;
    float r = acc[c];
    if (add) r += add[idx];
    if (relu) r = fmaxf(r, 0.f);
    out[idx] = beta != 0.f ? beta * out[idx] + r : r;
  }
}

// Weight (and bias) gradient partials of one voxel tile:
//   part[tile][co][ci][k] = sum_{v in tile} g[co](v) in[ci](v + k),
//   bpart[tile][co] = sum_{v in tile} g[co](v)   (blockIdx.z == 0 blocks).
// Grid (tiles, co_n / COB, ceil(ci_n / CIB)). Thread t owns the (ci, k) pair
// t % (CIB * KK) and the voxels v = t / (CIB * KK) + j * groups of the tile;
// the groups' sums are added in a fixed order in shared memory.
template <int K, int COB>
__global__ void __launch_bounds__(CT) k_conv_wgrad(Dims d, int ci_n, int co_n, const float* __restrict__ in,
                                                  const float* __restrict__ g, float* __restrict__ part,
                                                  float* __restrict__ bpart) {
  constexpr int R = K / 2, HX = CTX + 2 * R, HY = CTY + 2 * R, HZ = CTZ + 2 * R, KK = K * K * K;
  constexpr int HV = HX * HY * HZ, TV = CTX * CTY * CTZ;
  constexpr int NP = CIB * KK;                      // (ci, k) pairs
  constexpr int GROUPS = NP >= CT ? 1 : CT / NP;    // voxel groups
  constexpr int NPT = (NP + CT - 1) / CT;           // pairs per thread (K=3: 1)
  __shared__ __align__(16) float tile[CIB * HV];
  __shared__ __align__(16) float gt[TV * COB];      // [v][co]
  __shared__ float red[GROUPS > 1 ? CT * COB : 1];
  const int ntx = (d.nx + CTX - 1) / CTX, nty = (d.ny + CTY - 1) / CTY;
  const int t = blockIdx.x;
  const int bx = t % ntx, by = (t / ntx) % nty, bz = t / (ntx * nty);
  const int co0 = blockIdx.y * COB, ci0 = blockIdx.z * CIB;
  const int nc = min(CIB, ci_n - ci0);
  const long long vox = d.vox();
  for (int i = threadIdx.x; i < CIB * HV; i += CT) {
    const int c = i / HV, r = i % HV;
    const int hx = r % HX, hy = (r / HX) % HY, hz = r / (HX * HY);
    const int gx = bx * CTX + hx - R, gy = by * CTY + hy - R, gz = bz * CTZ + hz - R;
    float v = 0.f;
    if (c < nc && gx >= 0 && gy >= 0 && gz >= 0 && gx < d.nx && gy < d.ny && gz < d.nz)
      v = in[(long long)(ci0 + c) * vox + ((long long)gz * d.ny + gy) * d.nx + gx];
    tile[i] = v;
  }
  for (int i = threadIdx.x; i < TV * COB; i += CT) {
    const int o = i / TV, v = i % TV;  // coalesced along x for a fixed channel
    const int vx = v % CTX, vy = (v / CTX) % CTY, vz = v / (CTX * CTY);
    const int x = bx * CTX + vx, y = by * CTY + vy, z = bz * CTZ + vz;
    float gv = 0.f;
    if (x < d.nx && y < d.ny && z < d.nz) gv = g[(long long)(co0 + o) * vox + ((long long)z * d.ny + y) * d.nx + x];
    gt[v * COB + o] = gv;
  }
  __syncthreads();
  const long long nw = (long long)co_n * ci_n * KK;
  float* dst = part + (long long)t * nw;
#pragma unroll
  for (int pp = 0; pp < NPT; ++pp) {
    const int pair = (threadIdx.x % NP) + pp * CT;
    const int grp = GROUPS > 1 ? threadIdx.x / NP : 0;
    const bool active = pair < NP && grp < GROUPS && (NP >= CT || threadIdx.x < GROUPS * NP);
    float acc[COB];
#pragma unroll
    for (int o = 0; o < COB; ++o) acc[o] = 0.f;
    if (active) {
      const int c = pair / KK, k = pair % KK;
      const int dx = k % K, dy = (k / K) % K, dz = k / (K * K);
      const float* tc = tile + c * HV + (dz * HY + dy) * HX + dx;
      for (int v = grp; v < TV; v += GROUPS) {
        const int vx = v % CTX, vy = (v / CTX) % CTY, vz = v / (CTX * CTY);
        const float a = tc[(vz * HY + vy) * HX + vx];
        const float4* g4 = reinterpret_cast<const float4*>(gt + v * COB);
#pragma unroll
        for (int c4 = 0; c4 < COB / 4; ++c4) {
          const float4 gg = g4[c4];
          acc[4 * c4 + 0] = fmaf(gg.x, a, acc[4 * c4 + 0]);
          acc[4 * c4 + 1] = fmaf(gg.y, a, acc[4 * c4 + 1]);
          acc[4 * c4 + 2] = fmaf(gg.z, a, acc[4 * c4 + 2]);
          acc[4 * c4 + 3] = fmaf(gg.w, a, acc[4 * c4 + 3]);
        }
      }
    }
    if (GROUPS > 1) {
      if (active)
#pragma unroll
        for (int o = 0; o < COB; ++o) red[threadIdx.x * COB + o] = acc[o];
      __syncthreads();
      if (threadIdx.x < NP) {
        const int c = threadIdx.x / KK, k = threadIdx.x % KK;
#pragma unroll
        for (int o = 0; o < COB; ++o) {
          float s = 0.f;
          for (int gi = 0; gi < GROUPS; ++gi) s += red[(gi * NP + threadIdx.x) * COB + o];
          if (c < nc) dst[((long long)(co0 + o) * ci_n + ci0 + c) * KK + k] = s;
        }
      }
      __syncthreads();
    } else if (active) {
      const int c = pair / KK, k = pair % KK;
      if (c < nc)
#pragma unroll
        for (int o = 0; o < COB; ++o) dst[((long long)(co0 + o) * ci_n + ci0 + c) * KK + k] = acc[o];
    }
  }
  if (bpart && blockIdx.z == 0 && threadIdx.x < COB) {
    float s = 0.f;
    for (int v = 0; v < TV; ++v) s += gt[v * COB + threadIdx.x];
    bpart[(long long)t * co_n + co0 + threadIdx.x] = s;
  }
}

// grad[i] += sum over tiles of part[tile][i] in a fixed order: one warp per
// parameter, lanes striding over tiles, then a fixed shuffle tree.
__global__ void k_reduce_parts(long long tiles, long long nw, int nb, const float* __restrict__ part,
                               const float* __restrict__ bpart, float* __restrict__ dw, float* __restrict__ db) {
  const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (wid >= nw + nb) return;
  double s = 0.0;
  if (wid < nw) {
    for (long long t = lane; t < tiles; t += 32) s += part[t * nw + wid];
  } else {
    for (long long t = lane; t < tiles; t += 32) s += bpart[t * nb + (wid - nw)];
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) {
    if (wid < nw) dw[wid] += (float)s;
    else db[wid - nw] += (float)s;
  }
}

// wt[ci][co][flip(k)] = w[co][ci][k]: the weights of the data-gradient convolution.
__global__ void k_transpose_w(int co_n, int ci_n, int KK, const float* __restrict__ w, float* __restrict__ wt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= co_n * ci_n * KK) return;
  int k = i % KK, ci = (i / KK) % ci_n, co = i / (KK * ci_n);
  wt[((long long)ci * co_n + co) * KK + (KK - 1 - k)] = w[i];
}

__global__ void k_relu_mask(long long n, const float* __restrict__ act, float* __restrict__ g) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && !(act[i] > 0.f)) g[i] = 0.f;
}

// average of the children (ceil division of odd sizes); activation counts stay below 2^31
__global__ void k_pool(Dims f, Dims c, int ch, const float* __restrict__ in, float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int cv = (int)c.vox(), fv = (int)f.vox();
  if (i >= cv * ch) return;
  const int k = i / cv, o = i - k * cv;
  const int x = o % c.nx, y = (o / c.nx) % c.ny, z = o / (c.nx * c.ny);
  const float* src = in + (long long)k * fv;
  float s = 0.f;
  int n = 0;
  for (int dz = 0; dz < 2; ++dz)
    for (int dy = 0; dy < 2; ++dy)
      for (int dx = 0; dx < 2; ++dx) {
        const int X = 2 * x + dx, Y = 2 * y + dy, Z = 2 * z + dz;
        if (X < f.nx && Y < f.ny && Z < f.nz) {
          s += src[(Z * f.ny + Y) * f.nx + X];
          ++n;
        }
      }
  out[i] = s / n;
}

// backward of k_pool: each fine voxel receives g_coarse / (children of its parent); beta accumulates
__global__ void k_pool_bwd(Dims f, Dims c, int ch, const float* __restrict__ gc, float beta, float* __restrict__ gf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int fv = (int)f.vox(), cv = (int)c.vox();
  if (i >= fv * ch) return;
  const int k = i / fv, o = i - k * fv;
  const int X = o % f.nx, Y = (o / f.nx) % f.ny, Z = o / (f.nx * f.ny);
  const int x = X / 2, y = Y / 2, z = Z / 2;
  const int nxc = min(2, f.nx - 2 * x), nyc = min(2, f.ny - 2 * y), nzc = min(2, f.nz - 2 * z);
  const float v = gc[(long long)k * cv + (z * c.ny + y) * c.nx + x] / (nxc * nyc * nzc);
  gf[i] = beta != 0.f ? beta * gf[i] + v : v;
}

// grid (ceil(nx / 128), ny, nz * ch): one thread per fine voxel along x, no divisions
__global__ void __launch_bounds__(128) k_up(Dims f, Dims c, int ch, const float* __restrict__ in,
                                           float* __restrict__ out) {
  const int X = blockIdx.x * 128 + threadIdx.x;
  if (X >= f.nx) return;
  const int Y = blockIdx.y, Z = blockIdx.z % f.nz, k = blockIdx.z / f.nz;
  out[((long long)k * f.nz + Z) * f.ny * f.nx + (long long)Y * f.nx + X] =
      in[(long long)k * c.vox() + ((long long)(Z >> 1) * c.ny + (Y >> 1)) * c.nx + (X >> 1)];
}

__global__ void k_up_bwd(Dims f, Dims c, int ch, const float* __restrict__ gf, float* __restrict__ gc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int cv = (int)c.vox(), fv = (int)f.vox();
  if (i >= cv * ch) return;
  const int k = i / cv, o = i - k * cv;
  const int x = o % c.nx, y = (o / c.nx) % c.ny, z = o / (c.nx * c.ny);
  const float* src = gf + (long long)k * fv;
  float s = 0.f;
  for (int dz = 0; dz < 2; ++dz)
    for (int dy = 0; dy < 2; ++dy)
      for (int dx = 0; dx < 2; ++dx) {
        const int X = 2 * x + dx, Y = 2 * y + dy, Z = 2 * z + dz;
        if (X < f.nx && Y < f.ny && Z < f.nz) s += src[(Z * f.ny + Y) * f.nx + X];
      }
  gc[i] = s;
}

// Linear prolongation along one direction from nc coarse to nf = 2 nc or
// 2 nc - 1 fine points: fine X = 2c takes coarse c; odd X the mean of its two
// neighbours (X - 1) / 2 and (X + 1) / 2, or the lower one alone past the end.
__device__ __forceinline__ void lin_taps(int X, int nc, int* i0, int* i1, float* w0, float* w1) {
  const int lo = X >> 1;
  if (!(X & 1)) {
    *i0 = *i1 = lo;
    *w0 = 1.f;
    *w1 = 0.f;
  } else if (lo + 1 < nc) {
    *i0 = lo;
    *i1 = lo + 1;
    *w0 = *w1 = 0.5f;
  } else {
    *i0 = *i1 = lo;
    *w0 = 1.f;
    *w1 = 0.f;
  }
}

// weight of coarse c in fine X (the adjoint of lin_taps)
__device__ __forceinline__ float lin_w(int X, int c, int nc) {
  int i0, i1;
  float w0, w1;
  lin_taps(X, nc, &i0, &i1, &w0, &w1);
  return (i0 == c ? w0 : 0.f) + (i1 == c ? w1 : 0.f);
}

// trilinear upsampling of the pooled network's output to the input grid
__global__ void k_up_lin(Dims f, Dims c, int ch, const float* __restrict__ in, float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int fv = (int)f.vox(), cv = (int)c.vox();
  if (i >= fv * ch) return;
  const int k = i / fv, o = i - k * fv;
  const int X = o % f.nx, Y = (o / f.nx) % f.ny, Z = o / (f.nx * f.ny);
  int x[2], y[2], z[2];
  float wx[2], wy[2], wz[2];
  lin_taps(X, c.nx, &x[0], &x[1], &wx[0], &wx[1]);
  lin_taps(Y, c.ny, &y[0], &y[1], &wy[0], &wy[1]);
  lin_taps(Z, c.nz, &z[0], &z[1], &wz[0], &wz[1]);
  const float* src = in + (long long)k * cv;
  float s = 0.f;
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int d = 0; d < 2; ++d) s += wz[a] * wy[b] * wx[d] * src[(z[a] * c.ny + y[b]) * c.nx + x[d]];
  out[i] = s;
}

// adjoint of k_up_lin: each coarse voxel gathers its fine neighbours 2c-1..2c+1 (fixed order)
__global__ void k_up_lin_bwd(Dims f, Dims c, int ch, const float* __restrict__ gf, float* __restrict__ gc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int cv = (int)c.vox(), fv = (int)f.vox();
  if (i >= cv * ch) return;
  const int k = i / cv, o = i - k * cv;
  const int x = o % c.nx, y = (o / c.nx) % c.ny, z = o / (c.nx * c.ny);
  const float* src = gf + (long long)k * fv;
  float s = 0.f;
  for (int dz = -1; dz <= 1; ++dz) {
    const int Z = 2 * z + dz;
    if (Z < 0 || Z >= f.nz) continue;
    const float wz = lin_w(Z, z, c.nz);
    if (wz == 0.f) continue;
    for (int dy = -1; dy <= 1; ++dy) {
      const int Y = 2 * y + dy;
      if (Y < 0 || Y >= f.ny) continue;
      const float wy = lin_w(Y, y, c.ny);
      if (wy == 0.f) continue;
      for (int dx = -1; dx <= 1; ++dx) {
        const int X = 2 * x + dx;
        if (X < 0 || X >= f.nx) continue;
        const float wx = lin_w(X, x, c.nx);
        if (wx != 0.f) s += wz * wy * wx * src[(Z * f.ny + Y) * f.nx + X];
      }
    }
  }
  gc[i] = s;
}

// masked mean squared error: partial sums of mask*(o-t)^2 and mask; g = 2 mask (o - t)
__global__ void __launch_bounds__(256) k_mse(long long n, int ch, const float* __restrict__ o, const float* __restrict__ t,
                                             const float* __restrict__ mask, float* __restrict__ g,
                                             double* __restrict__ part) {
  __shared__ double s1[256], s2[256];
  double a = 0, m = 0;
  long long vox = n;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < vox * ch;
       i += (long long)gridDim.x * blockDim.x) {
    float mk = mask ? mask[i % vox] : 1.f;
    float r = o[i] - t[i];
    a += (double)mk * r * r;
    m += mk;
    g[i] = 2.f * mk * r;
  }
  s1[threadIdx.x] = a;
  s2[threadIdx.x] = m;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st) {
      s1[threadIdx.x] += s1[threadIdx.x + st];
      s2[threadIdx.x] += s2[threadIdx.x + st];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s1[0];
    part[2 * blockIdx.x + 1] = s2[0];
  }
}

__global__ void k_scale(long long n, float s, float* x) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] *= s;
}

__global__ void k_adam(long long n, float lr, float b1, float b2, float eps, float bc1, float bc2, float gscale,
                       float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float gi = g[i] * gscale;
  float mi = b1 * m[i] + (1.f - b1) * gi;
  float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

// deterministic uniform init (splitmix64 hash), U(-a, a)
__global__ void k_init(long long n, unsigned long long seed, float a, float* p) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(i + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  float u = (float)((z >> 11) * (1.0 / 9007199254740992.0));
  p[i] = (2.f * u - 1.f) * a;
}

// ---------------------------------------------------------------------------
// BF16 tensor-core 3x3x3 convolution for inference (the preconditioner's
// forward pass), as an implicit GEMM on mma.sync.m16n8k16 (BF16 operands,
// FP32 accumulation): rows are output voxels, columns output channels, and the
// reduction runs over K = 27 taps x CINP input channels (tap-major, padded to
// a multiple of 16 with zeros). A CTA computes an 8 x 8 x 4 voxel tile: its
// input halo (10 x 10 x 6 voxels) is staged once in shared memory as BF16,
// channel-last, and the layer's weights as BF16 rows [co][k]; each warp owns
// MF row fragments of 16 voxels and every output channel. Row strides are
// padded so that the 32-bit fragment loads are free of bank conflicts
// (stride / 2 = 4 mod 8 words). The epilogue adds bias and skip input, applies
// the ReLU and writes FP32 channel-first activations, as the FP32 kernel does.
// Training keeps the FP32 kernels; this path serves layers of at most 32 input
// and output channels, the fine levels where the network spends its time.
namespace mmaconv {
constexpr int TX = 8, TY = 8, TZ = 4, NV = TX * TY * TZ;  // output tile
constexpr int HX = TX + 2, HY = TY + 2, HZ = TZ + 2, HV = HX * HY * HZ;
__host__ __device__ constexpr int cin_stride(int cinp) { return ((cinp / 2) % 8 == 4) ? cinp : cinp + 8; }
__host__ __device__ constexpr int k_pad(int cinp) { return (27 * cinp + 15) / 16 * 16; }
__host__ __device__ constexpr int k_stride(int cinp) { return k_pad(cinp) + 8; }
__host__ __device__ constexpr int frags(int co) { return co <= 16 ? 4 : 2; }  // row fragments per warp
__host__ __device__ constexpr int warps(int co) { return NV / 16 / frags(co); }
inline size_t smem(int cinp, int co) {
  return (size_t)HV * cin_stride(cinp) * 2 + (size_t)co * k_stride(cinp) * 2;
}
}  // namespace mmaconv

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// wb[co][k] (row stride k_stride) = bf16(w[co][ci][tap]) with k = tap * CINP + ci, zero padding
__global__ void k_weights_bf16(int co_n, int ci_n, int cinp, const float* __restrict__ w, __nv_bfloat16* wb) {
  const int ks = mmaconv::k_stride(cinp);
  const long long n = (long long)co_n * ks;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int co = (int)(i / ks), k = (int)(i % ks);
  const int tap = k / cinp, ci = k % cinp;
  float v = 0.f;
  if (tap < 27 && ci < ci_n) v = w[((long long)co * ci_n + ci) * 27 + tap];
  wb[i] = __float2bfloat16_rn(v);
}

template <int CINP, int CO>
__global__ void __launch_bounds__(32 * mmaconv::warps(CO))
    k_conv_mma(Dims d, int ci_n, const float* __restrict__ in, const __nv_bfloat16* __restrict__ wb,
               const float* __restrict__ bias, const float* __restrict__ add, int relu, float beta,
               float* __restrict__ out) {
  using namespace mmaconv;
  constexpr int CS = cin_stride(CINP), KP = k_pad(CINP), KS = k_stride(CINP), MF = frags(CO), NF = CO / 8;
  constexpr int NT = 32 * warps(CO);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __nv_bfloat16* xs = reinterpret_cast<__nv_bfloat16*>(smem_raw);  // [HV][CS]
  __nv_bfloat16* ws = xs + HV * CS;                                 // [CO][KS]
  const int ntx = (d.nx + TX - 1) / TX, nty = (d.ny + TY - 1) / TY;
  const int bx = blockIdx.x % ntx, by = (blockIdx.x / ntx) % nty, bz = blockIdx.x / (ntx * nty);
  const long long vox = d.vox();
  // stage the halo (channel-last BF16, zero outside the grid and beyond ci_n)
  for (int i = threadIdx.x; i < CINP * HV; i += NT) {
    const int c = i / HV, r = i % HV;
    const int hx = r % HX, hy = (r / HX) % HY, hz = r / (HX * HY);
    const int gx = bx * TX + hx - 1, gy = by * TY + hy - 1, gz = bz * TZ + hz - 1;
    float v = 0.f;
    if (c < ci_n && gx >= 0 && gy >= 0 && gz >= 0 && gx < d.nx && gy < d.ny && gz < d.nz)
      v = in[(long long)c * vox + ((long long)gz * d.ny + gy) * d.nx + gx];
    xs[r * CS + c] = __float2bfloat16_rn(v);
  }
  // stage the weights, 16-byte rows (KS is a multiple of 8 halves)
  {
    const uint4* src = reinterpret_cast<const uint4*>(wb);
    uint4* dst = reinterpret_cast<uint4*>(ws);
    for (int i = threadIdx.x; i < CO * KS / 8; i += NT) dst[i] = src[i];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  float acc[MF][NF][4];
#pragma unroll
  for (int f = 0; f < MF; ++f)
#pragma unroll
    for (int n = 0; n < NF; ++n)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[f][n][j] = 0.f;
  // halo index of this lane's two rows in each fragment (tap offset added per k)
  int hrow[MF][2];
#pragma unroll
  for (int f = 0; f < MF; ++f)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int v = (w * MF + f) * 16 + g + 8 * h;
      const int x = v % TX, y = (v / TX) % TY, z = v / (TX * TY);
      hrow[f][h] = (z * HY + y) * HX + x;
    }
  const uint32_t* xw = reinterpret_cast<const uint32_t*>(xs);
  const uint32_t* ww = reinterpret_cast<const uint32_t*>(ws);
#pragma unroll 2
  for (int kc = 0; kc < KP / 16; ++kc) {
    // A columns 2t, 2t+1 (and +8): (tap, ci) of each pair
    int aoff[2];
    bool aval[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int k = kc * 16 + 2 * t + 8 * h;
      const int tap = k / CINP, ci = k % CINP;
      aval[h] = tap < 27;
      const int tt = aval[h] ? tap : 0;
      const int dx = tt % 3, dy = (tt / 3) % 3, dz = tt / 9;
      aoff[h] = ((dz * HY + dy) * HX + dx) * CS + ci;
    }
    uint32_t b[NF][2];
#pragma unroll
    for (int n = 0; n < NF; ++n) {
      const int row = (n * 8 + g) * KS + kc * 16 + 2 * t;
      b[n][0] = ww[row >> 1];
      b[n][1] = ww[(row + 8) >> 1];
    }
#pragma unroll
    for (int f = 0; f < MF; ++f) {
      const uint32_t a0 = aval[0] ? xw[(hrow[f][0] * CS + aoff[0]) >> 1] : 0u;
      const uint32_t a1 = aval[0] ? xw[(hrow[f][1] * CS + aoff[0]) >> 1] : 0u;
      const uint32_t a2 = aval[1] ? xw[(hrow[f][0] * CS + aoff[1]) >> 1] : 0u;
      const uint32_t a3 = aval[1] ? xw[(hrow[f][1] * CS + aoff[1]) >> 1] : 0u;
#pragma unroll
      for (int n = 0; n < NF; ++n) mma_bf16(acc[f][n], a0, a1, a2, a3, b[n][0], b[n][1]);
    }
  }
  // epilogue: rows g, g + 8 of each fragment; columns 2t, 2t + 1 of each n
#pragma unroll
  for (int f = 0; f < MF; ++f)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int v = (w * MF + f) * 16 + g + 8 * h;
      const int x = bx * TX + v % TX, y = by * TY + (v / TX) % TY, z = bz * TZ + v / (TX * TY);
      if (x >= d.nx || y >= d.ny || z >= d.nz) continue;
      const long long o = ((long long)z * d.ny + y) * d.nx + x;
#pragma unroll
      for (int n = 0; n < NF; ++n)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int co = n * 8 + 2 * t + j;
          float val = acc[f][n][2 * h + j] + (bias ? bias[co] : 0.f);
          const long long idx = (long long)co * vox + o;
          if (add) val += add[idx];
          if (relu) val = fmaxf(val, 0.f);
          out[idx] = beta != 0.f ? beta * out[idx] + val : val;
        }
    }
}

struct Layer {
  int ci, co, k;  // kernel size 1 or 3
  bool relu;
  long long w_off, b_off;  // offsets in the flat parameter vector
};

}  // namespace cnn
}  // namespace jxb

using namespace jxb;
using namespace jxb::cnn;

struct jxb_cnn {
  int in_ch = 0, out_ch = 0, levels = 0, c[MAXL] = {};
  std::vector<Layer> L;  // encoder pairs, bottom triple, decoder pairs, output
  long long n_params = 0;
  float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  long long adam_t = 0;
  // activations, sized for `cap` (level-0 dims)
  Dims cap{0, 0, 0};
  float* arena = nullptr;
  float *A[MAXL] = {}, *S[MAXL] = {}, *P[MAXL] = {}, *U[MAXL] = {}, *M[MAXL] = {}, *D[MAXL] = {}, *GS[MAXL] = {};
  float *B0 = nullptr, *B1 = nullptr, *B2 = nullptr, *OUT = nullptr, *G0 = nullptr, *G1 = nullptr;
  int pool_in = 0;         // run on the pooled input (half resolution), upsample the output
  Dims cap_f{0, 0, 0};     // fine grid of the input-pooling buffers
  float* fine_arena = nullptr;
  float *INC = nullptr, *OUTF = nullptr, *GOF = nullptr;  // pooled input, fine output, fine output gradient
  Dims last{0, 0, 0};      // input grid of the last forward pass
  float* wt = nullptr;     // transposed weights scratch
  float* cpart = nullptr;  // split-channel conv partials
  long long cpart_cap = 0;
  float* part = nullptr;   // weight-gradient partials
  long long part_cap = 0;
  double* red = nullptr;   // loss partials
  int bf16 = 0;            // inference forwards take the BF16 tensor-core convolution where it applies
  int last_bf16 = 0;       // the last forward did (its activations cannot be back-propagated)
  __nv_bfloat16* wbf = nullptr;  // one layer's BF16 weights
  long long wbf_cap = 0;
};

namespace {

inline unsigned nblk(long long n) { return (unsigned)((n + 255) / 256); }

// layer indices
inline int enc_a(int l) { return 2 * l; }
inline int enc_b(int l) { return 2 * l + 1; }
inline int bot(const jxb_cnn* N, int i) { return 2 * (N->levels - 1) + i; }
inline int dec_c(const jxb_cnn* N, int l) { return 2 * (N->levels - 1) + 3 + 2 * (N->levels - 2 - l); }
inline int dec_d(const jxb_cnn* N, int l) { return dec_c(N, l) + 1; }
inline int out_layer(const jxb_cnn* N) { return 4 * N->levels - 1; }

// up_from: for a 1x1 layer, `in` is on that coarse grid and is read upsampled
int conv(jxb_cnn* N, cudaStream_t s, Dims d, const Layer& L, const float* p, const float* in, const float* add,
         float beta, float* out, const Dims* up_from = nullptr) {
  const float* w = p + L.w_off;
  const float* b = L.b_off >= 0 ? p + L.b_off : nullptr;
  const int relu = L.relu ? 1 : 0;
  if (L.k == 1 && L.ci <= 64) {
    const int cob1 = L.co % 16 == 0 ? 16 : (L.co % 8 == 0 ? 8 : 4);
    const dim3 g1((unsigned)((d.vox() + 255) / 256), (unsigned)(L.co / cob1));
    const Dims c = up_from ? *up_from : d;
#define JXB_CONV1(C)                                                                                         \
  if (cob1 == C) {                                                                                           \
    if (up_from) k_conv1<C, true><<<g1, 256, 0, s>>>(d, c, L.ci, in, w, b, add, relu, beta, out);            \
    else k_conv1<C, false><<<g1, 256, 0, s>>>(d, c, L.ci, in, w, b, add, relu, beta, out);                   \
  }
    JXB_CONV1(16) JXB_CONV1(8) JXB_CONV1(4)
#undef JXB_CONV1
    JXB_CUDA(cudaGetLastError());
    return JXB_OK;
  }
  if (up_from) return fail(JXB_ERR_INVALID, "cnn: upsampled input needs a 1x1 layer with at most 64 inputs");
  const long long tiles = n_tiles(d);
  int cob = L.co <= 16 ? L.co : (L.co % 16 == 0 ? 16 : (L.co % 12 == 0 ? 12 : 8));
  // small grids: narrower output-channel blocks until there are two CTAs per SM
  // (every output still sums its inputs in the same order, so results do not change)
  for (const int c : {12, 8, 4})
    if (tiles * (L.co / cob) < 2 * 148 && c < cob && L.co % c == 0) cob = c;
  // fewer than eight CTAs per SM: split the input channels over blocks (each
  // sums a run of whole CIB groups), then sum the slabs in a fixed order. A CTA
  // walks its channel groups one after another, each a staging round trip, so
  // on the coarse levels the split trades a small slab sum for that latency.
  // The partial buffer only grows; its first sizing happens on the forward pass
  // that runs before any graph capture.
  constexpr long long SPLIT_CTAS = 8 * 148;
  int nsplit = 1, cps = L.ci;
  const long long ctas = tiles * (L.co / cob);
  if (ctas < SPLIT_CTAS && L.ci > CIB) {
    const int groups = (L.ci + CIB - 1) / CIB;
    const int want = (int)std::min<long long>(groups, (SPLIT_CTAS + ctas - 1) / ctas);
    cps = ((groups + want - 1) / want) * CIB;
    nsplit = (L.ci + cps - 1) / cps;
  }
  float* dst = out;
  if (nsplit > 1) {
    const long long need = (long long)nsplit * L.co * d.vox();
    if (need > N->cpart_cap) {
      cudaFree(N->cpart);
      N->cpart = nullptr;
      N->cpart_cap = 0;
      JXB_CUDA(cudaMalloc(&N->cpart, need * sizeof(float)));
      N->cpart_cap = need;
    }
    dst = N->cpart;
  }
  const dim3 grid((unsigned)tiles, (unsigned)(L.co / cob), (unsigned)nsplit);
#define JXB_CONV(KS, C)                                                                         \
  if (L.k == KS && cob == C) {                                                                  \
    if (nsplit == 1) {                                                                          \
      k_conv<KS, C><<<grid, CT, 0, s>>>(d, L.ci, in, w, b, add, relu, beta, out, L.ci, L.co);   \
    } else {                                                                                    \
      k_conv<KS, C><<<grid, CT, 0, s>>>(d, L.ci, in, w, nullptr, nullptr, 0, 0.f, dst, cps, L.co); \
      k_sum_split<<<nblk(d.vox() * L.co), 256, 0, s>>>(d.vox(), L.co, nsplit, dst, b, add, relu, beta, out); \
    }                                                                                           \
    JXB_CUDA(cudaGetLastError());                                                               \
    return JXB_OK;                                                                              \
  }
  JXB_CONV(3, 4) JXB_CONV(3, 8) JXB_CONV(3, 12) JXB_CONV(3, 16)
  JXB_CONV(1, 4) JXB_CONV(1, 8) JXB_CONV(1, 12) JXB_CONV(1, 16)
#undef JXB_CONV
  return fail(JXB_ERR_INVALID, "cnn: unsupported output channel count " + std::to_string(L.co));
}

// data gradient of a conv layer: gin = beta*gin + conv^T(g)
int conv_dgrad(jxb_cnn* N, cudaStream_t s, Dims d, const Layer& L, const float* g, float beta, float* gin) {
  int KK = L.k * L.k * L.k;
  int n = L.co * L.ci * KK;
  k_transpose_w<<<(n + 255) / 256, 256, 0, s>>>(L.co, L.ci, KK, N->p + L.w_off, N->wt);
  Layer T{L.co, L.ci, L.k, false, 0, -1};
  return conv(N, s, d, T, N->wt, g, nullptr, beta, gin);
}

int conv_wgrad(jxb_cnn* N, cudaStream_t s, Dims d, const Layer& L, const float* in, const float* g) {
  const long long tiles = n_tiles(d);
  const int KK = L.k * L.k * L.k;
  const long long nw = (long long)L.co * L.ci * KK;
  const long long need = tiles * nw + tiles * L.co;
  if (need > N->part_cap) {
    cudaFree(N->part);
    N->part = nullptr;
    N->part_cap = 0;
    JXB_CUDA(cudaMalloc(&N->part, need * sizeof(float)));
    N->part_cap = need;
  }
  float* bpart = N->part + tiles * nw;
  // at most 12 output channels per block keeps the static shared memory under 48 KB
  const int cob = L.co % 8 == 0 ? 8 : (L.co == 12 ? 12 : 4);
  const dim3 grid((unsigned)tiles, (unsigned)(L.co / cob), (unsigned)((L.ci + CIB - 1) / CIB));
  float* bp = L.b_off >= 0 ? bpart : nullptr;
  bool done = false;
#define JXB_WGRAD(KS, C)                                                                       \
  if (!done && L.k == KS && cob == C) {                                                        \
    k_conv_wgrad<KS, C><<<grid, CT, 0, s>>>(d, L.ci, L.co, in, g, N->part, bp);                \
    done = true;                                                                               \
  }
  JXB_WGRAD(3, 4) JXB_WGRAD(3, 8) JXB_WGRAD(3, 12)
  JXB_WGRAD(1, 4) JXB_WGRAD(1, 8) JXB_WGRAD(1, 12)
#undef JXB_WGRAD
  if (!done) return fail(JXB_ERR_INVALID, "cnn: unsupported output channel count " + std::to_string(L.co));
  JXB_CUDA(cudaGetLastError());
  const int nb = L.b_off >= 0 ? L.co : 0;
  const long long warps = nw + nb;
  k_reduce_parts<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, s>>>(tiles, nw, nb, N->part, bpart, N->g + L.w_off,
                                                                       nb ? N->g + L.b_off : nullptr);
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

int ensure_bufs(jxb_cnn* N, Dims d0) {
  if (d0.nx == N->cap.nx && d0.ny == N->cap.ny && d0.nz == N->cap.nz) return JXB_OK;
  cudaFree(N->arena);
  N->arena = nullptr;
  N->cap = {0, 0, 0};
  const int nl = N->levels;
  Dims d[MAXL];
  d[0] = d0;
  for (int l = 1; l < nl; ++l) d[l] = halve(d[l - 1]);
  // sizes in floats, each rounded up to 64 floats (256 B)
  std::vector<std::pair<float**, long long>> want;
  auto add = [&](float** ptr, long long n) { want.push_back({ptr, (std::max<long long>(n, 1) + 63) / 64 * 64}); };
  long long gmax = (long long)std::max(N->in_ch, 4) * d0.vox();
  if ((long long)64 * d0.vox() >= (1ll << 31)) return fail(JXB_ERR_INVALID, "cnn: grid too large (activation indices are 32-bit)");
  // the upsampling launch maps y and z * channels onto grid dimensions
  if (d0.ny > 65535 || (long long)d0.nz * MAXC > 65535) return fail(JXB_ERR_INVALID, "cnn: grid too large in y or z");
  for (int l = 0; l < nl - 1; ++l) {
    add(&N->A[l], N->c[l] * d[l].vox());
    add(&N->S[l], N->c[l] * d[l].vox());
    add(&N->P[l + 1], N->c[l] * d[l + 1].vox());
    add(&N->U[l], N->c[l + 1] * d[l].vox());
    add(&N->M[l], N->c[l] * d[l].vox());
    add(&N->D[l], N->c[l] * d[l].vox());
    add(&N->GS[l], N->c[l] * d[l].vox());
    gmax = std::max(gmax, (long long)std::max(N->c[l], N->c[l + 1]) * d[l].vox());
  }
  const long long vb = N->c[nl - 1] * d[nl - 1].vox();
  add(&N->B0, vb);
  add(&N->B1, vb);
  add(&N->B2, vb);
  gmax = std::max(gmax, vb);
  add(&N->OUT, 4 * d0.vox());
  add(&N->G0, gmax);
  add(&N->G1, gmax);
  long long total = 0;
  for (auto& w : want) total += w.second;
  JXB_CUDA(cudaMalloc(&N->arena, total * sizeof(float)));
  long long off = 0;
  for (auto& w : want) {
    *w.first = N->arena + off;
    off += w.second;
  }
  N->cap = d0;
  return JXB_OK;
}

// The BF16 tensor-core path for a 3x3x3 layer of at most 32 input and output
// channels (output channels a multiple of 8); 1 when the layer does not
// qualify (the caller then runs the FP32 kernel), else a status.
int conv_mma(jxb_cnn* N, cudaStream_t s, Dims d, const Layer& L, const float* p, const float* in, const float* add,
             float* out) {
  if (L.k != 3 || L.ci > 32 || L.co > 32 || L.co % 8 != 0) return 1;
  const int cinp = (L.ci + 7) / 8 * 8;
  const long long need = (long long)L.co * mmaconv::k_stride(cinp);
  if (need > N->wbf_cap) {
    cudaFree(N->wbf);
    N->wbf = nullptr;
    N->wbf_cap = 0;
    // 32 x k_stride(32) halves: sized for the widest qualifying layer at once
    const long long cap = (long long)32 * mmaconv::k_stride(32);
    JXB_CUDA(cudaMalloc(&N->wbf, cap * sizeof(__nv_bfloat16)));
    N->wbf_cap = cap;
  }
  k_weights_bf16<<<nblk(need), 256, 0, s>>>(L.co, L.ci, cinp, p + L.w_off, N->wbf);
  const float* b = L.b_off >= 0 ? p + L.b_off : nullptr;
  const long long tiles = (long long)((d.nx + 7) / 8) * ((d.ny + 7) / 8) * ((d.nz + 3) / 4);
#define JXB_MMA(CI, C)                                                                                    \
  if (cinp == CI && L.co == C) {                                                                          \
    auto k = k_conv_mma<CI, C>;                                                                           \
    const size_t sm = mmaconv::smem(CI, C);                                                               \
    if (sm > 48 * 1024) JXB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)); \
    k<<<(unsigned)tiles, 32 * mmaconv::warps(C), sm, s>>>(d, L.ci, in, N->wbf, b, add, L.relu ? 1 : 0, 0.f, out); \
    JXB_CUDA(cudaGetLastError());                                                                         \
    return JXB_OK;                                                                                        \
  }
  JXB_MMA(8, 8) JXB_MMA(8, 16) JXB_MMA(8, 24) JXB_MMA(8, 32)
  JXB_MMA(16, 8) JXB_MMA(16, 16) JXB_MMA(16, 24) JXB_MMA(16, 32)
  JXB_MMA(24, 8) JXB_MMA(24, 16) JXB_MMA(24, 24) JXB_MMA(24, 32)
  JXB_MMA(32, 8) JXB_MMA(32, 16) JXB_MMA(32, 24) JXB_MMA(32, 32)
#undef JXB_MMA
  return 1;
}

// a forward layer: the BF16 tensor-core convolution when `mma` and the layer qualifies
int conv_f(jxb_cnn* N, cudaStream_t s, bool mma, Dims d, const Layer& L, const float* p, const float* in,
           const float* add, float* out) {
  if (mma) {
    int rc = conv_mma(N, s, d, L, p, in, add, out);
    if (rc != 1) return rc;
  }
  return conv(N, s, d, L, p, in, add, 0.f, out);
}

int forward(jxb_cnn* N, cudaStream_t s, Dims d0, const float* in, bool infer = false) {
  const bool mma = infer && N->bf16;
  N->last_bf16 = mma ? 1 : 0;
  int rc = ensure_bufs(N, d0);
  if (rc) return rc;
  const int nl = N->levels;
  Dims d[MAXL];
  d[0] = d0;
  for (int l = 1; l < nl; ++l) d[l] = halve(d[l - 1]);
  const float* p = N->p;
  const float* x = in;
  for (int l = 0; l < nl - 1; ++l) {
    if ((rc = conv_f(N, s, mma, d[l], N->L[enc_a(l)], p, x, nullptr, N->A[l]))) return rc;
    if ((rc = conv_f(N, s, mma, d[l], N->L[enc_b(l)], p, N->A[l], nullptr, N->S[l]))) return rc;
    k_pool<<<nblk(d[l + 1].vox() * N->c[l]), 256, 0, s>>>(d[l], d[l + 1], N->c[l], N->S[l], N->P[l + 1]);
    x = N->P[l + 1];
  }
  const Dims db = d[nl - 1];
  if ((rc = conv_f(N, s, mma, db, N->L[bot(N, 0)], p, x, nullptr, N->B0))) return rc;
  if ((rc = conv_f(N, s, mma, db, N->L[bot(N, 1)], p, N->B0, nullptr, N->B1))) return rc;
  if ((rc = conv_f(N, s, mma, db, N->L[bot(N, 2)], p, N->B1, nullptr, N->B2))) return rc;
  const float* y = N->B2;
  for (int l = nl - 2; l >= 0; --l) {
    // the 1x1 layer reads y upsampled; U[l] is only materialised by the backward pass
    if ((rc = conv(N, s, d[l], N->L[dec_c(N, l)], p, y, N->S[l], 0.f, N->M[l], &d[l + 1]))) return rc;
    if ((rc = conv_f(N, s, mma, d[l], N->L[dec_d(N, l)], p, N->M[l], nullptr, N->D[l]))) return rc;
    y = N->D[l];
  }
  // the output layer (4 channels) stays on the FP32 kernel
  if ((rc = conv(N, s, d0, N->L[out_layer(N)], p, y, nullptr, 0.f, N->OUT))) return rc;
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

// Backward through the network for the output gradient in G0 (layout of OUT,
// 4 channels); accumulates parameter gradients into N->g. Needs the
// activations of a forward pass on the same input.
int backward(jxb_cnn* N, cudaStream_t s, Dims d0, const float* in) {
  const int nl = N->levels;
  Dims d[MAXL];
  d[0] = d0;
  for (int l = 1; l < nl; ++l) d[l] = halve(d[l - 1]);
  float *ga = N->G0, *gb = N->G1;
  int rc;
  // output layer
  if ((rc = conv_wgrad(N, s, d0, N->L[out_layer(N)], N->D[0], ga))) return rc;
  if ((rc = conv_dgrad(N, s, d0, N->L[out_layer(N)], ga, 0.f, gb))) return rc;  // dL/dD0
  std::swap(ga, gb);
  // decoder, level 0 upwards: ga = dL/dD_l
  for (int l = 0; l < nl - 1; ++l) {
    const long long n = (long long)N->c[l] * d[l].vox();
    k_relu_mask<<<nblk(n), 256, 0, s>>>(n, N->D[l], ga);
    if ((rc = conv_wgrad(N, s, d[l], N->L[dec_d(N, l)], N->M[l], ga))) return rc;
    if ((rc = conv_dgrad(N, s, d[l], N->L[dec_d(N, l)], ga, 0.f, N->GS[l]))) return rc;  // dL/dM_l = dL/ds_l (skip part)
    const float* yc = l + 1 < nl - 1 ? N->D[l + 1] : N->B2;  // the decoder input below this level
    k_up<<<dim3((d[l].nx + 127) / 128, d[l].ny, d[l].nz * N->c[l + 1]), 128, 0, s>>>(d[l], d[l + 1], N->c[l + 1], yc,
                                                                                   N->U[l]);
    if ((rc = conv_wgrad(N, s, d[l], N->L[dec_c(N, l)], N->U[l], N->GS[l]))) return rc;
    if ((rc = conv_dgrad(N, s, d[l], N->L[dec_c(N, l)], N->GS[l], 0.f, gb))) return rc;  // dL/dU_l
    k_up_bwd<<<nblk((long long)N->c[l + 1] * d[l + 1].vox()), 256, 0, s>>>(d[l], d[l + 1], N->c[l + 1], gb, ga);
  }
  // bottom: ga = dL/dB2
  const Dims db = d[nl - 1];
  const long long nbv = (long long)N->c[nl - 1] * db.vox();
  k_relu_mask<<<nblk(nbv), 256, 0, s>>>(nbv, N->B2, ga);
  if ((rc = conv_wgrad(N, s, db, N->L[bot(N, 2)], N->B1, ga))) return rc;
  if ((rc = conv_dgrad(N, s, db, N->L[bot(N, 2)], ga, 0.f, gb))) return rc;
  k_relu_mask<<<nblk(nbv), 256, 0, s>>>(nbv, N->B1, gb);
  if ((rc = conv_wgrad(N, s, db, N->L[bot(N, 1)], N->B0, gb))) return rc;
  if ((rc = conv_dgrad(N, s, db, N->L[bot(N, 1)], gb, 0.f, ga))) return rc;
  k_relu_mask<<<nblk(nbv), 256, 0, s>>>(nbv, N->B0, ga);
  const float* bot_in = N->P[nl - 1];
  if ((rc = conv_wgrad(N, s, db, N->L[bot(N, 0)], bot_in, ga))) return rc;
  if ((rc = conv_dgrad(N, s, db, N->L[bot(N, 0)], ga, 0.f, gb))) return rc;  // dL/dP_{L-1}
  std::swap(ga, gb);
  // encoder, deepest first: ga = dL/dP_{l+1}
  for (int l = nl - 2; l >= 0; --l) {
    const long long n = (long long)N->c[l] * d[l].vox();
    k_pool_bwd<<<nblk(n), 256, 0, s>>>(d[l], d[l + 1], N->c[l], ga, 1.f, N->GS[l]);  // dL/ds_l
    k_relu_mask<<<nblk(n), 256, 0, s>>>(n, N->S[l], N->GS[l]);
    if ((rc = conv_wgrad(N, s, d[l], N->L[enc_b(l)], N->A[l], N->GS[l]))) return rc;
    if ((rc = conv_dgrad(N, s, d[l], N->L[enc_b(l)], N->GS[l], 0.f, gb))) return rc;  // dL/dA_l
    k_relu_mask<<<nblk(n), 256, 0, s>>>(n, N->A[l], gb);
    const float* xin = l > 0 ? N->P[l] : in;
    if ((rc = conv_wgrad(N, s, d[l], N->L[enc_a(l)], xin, gb))) return rc;
    if (l > 0) {
      if ((rc = conv_dgrad(N, s, d[l], N->L[enc_a(l)], gb, 0.f, ga))) return rc;  // dL/dP_l
    }
  }
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

// The public forward/backward: the U-Net on the input grid, or on the pooled
// input with the output upsampled (input pooling).
int ensure_fine(jxb_cnn* N, Dims df) {
  if (df.nx == N->cap_f.nx && df.ny == N->cap_f.ny && df.nz == N->cap_f.nz) return JXB_OK;
  cudaFree(N->fine_arena);
  N->fine_arena = nullptr;
  N->cap_f = {0, 0, 0};
  if ((long long)64 * df.vox() >= (1ll << 31)) return fail(JXB_ERR_INVALID, "cnn: grid too large (activation indices are 32-bit)");
  const long long a = ((long long)N->in_ch * halve(df).vox() + 63) / 64 * 64, b = (4 * df.vox() + 63) / 64 * 64;
  JXB_CUDA(cudaMalloc(&N->fine_arena, (a + 2 * b) * sizeof(float)));
  N->INC = N->fine_arena;
  N->OUTF = N->INC + a;
  N->GOF = N->OUTF + b;
  N->cap_f = df;
  return JXB_OK;
}

float* out_buf(jxb_cnn* N) { return N->pool_in ? N->OUTF : N->OUT; }
float* gout_buf(jxb_cnn* N) { return N->pool_in ? N->GOF : N->G0; }

int forward_top(jxb_cnn* N, cudaStream_t s, Dims d, const float* in, bool infer = false) {
  N->last = {0, 0, 0};
  if (!N->pool_in) {
    int rc = forward(N, s, d, in, infer);
    if (!rc) N->last = d;
    return rc;
  }
  int rc = ensure_fine(N, d);
  if (rc) return rc;
  const Dims dc = halve(d);
  k_pool<<<nblk(dc.vox() * N->in_ch), 256, 0, s>>>(d, dc, N->in_ch, in, N->INC);
  if ((rc = forward(N, s, dc, N->INC, infer))) return rc;
  k_up_lin<<<nblk(d.vox() * 4), 256, 0, s>>>(d, dc, 4, N->OUT, N->OUTF);
  JXB_CUDA(cudaGetLastError());
  N->last = d;
  return JXB_OK;
}

// backward for the output gradient in gout_buf(N); needs forward_top on the same input
int backward_top(jxb_cnn* N, cudaStream_t s, Dims d, const float* in) {
  if (!N->pool_in) return backward(N, s, d, in);
  const Dims dc = halve(d);
  k_up_lin_bwd<<<nblk(dc.vox() * 4), 256, 0, s>>>(d, dc, 4, N->GOF, N->G0);
  JXB_CUDA(cudaGetLastError());
  return backward(N, s, dc, N->INC);
}

bool supported_co(int c) { return c == 4 || c == 8 || c == 12 || c == 16 || c == 24 || c == 32 || c == 48 || c == 64; }

}  // namespace

namespace jxb {

int cnn_forward(jxb_cnn* N, cudaStream_t s, int nx, int ny, int nz, const float* in, const float** out4, bool infer) {
  int rc = forward_top(N, s, Dims{nx, ny, nz}, in, infer);
  if (rc) return rc;
  if (out4) *out4 = out_buf(N);
  return JXB_OK;
}

float* cnn_grad_out(jxb_cnn* N) { return gout_buf(N); }

int cnn_backward(jxb_cnn* N, cudaStream_t s, int nx, int ny, int nz, const float* in) {
  return backward_top(N, s, Dims{nx, ny, nz}, in);
}

int cnn_out_channels(const jxb_cnn* N) { return N->out_ch; }

}  // namespace jxb

extern "C" int jxb_cnn_create(int in_ch, int out_ch, int levels, const int* channels, uint64_t seed, jxb_cnn** out) {
  if (!out || !channels || in_ch < 1 || in_ch > 8 || out_ch < 1 || out_ch > 3 || levels < 2 || levels > MAXL)
    return fail(JXB_ERR_INVALID, "jxb_cnn_create: bad argument (in_ch 1..8, out_ch 1..3, levels 2..6)");
  for (int i = 0; i < levels; ++i)
    if (!supported_co(channels[i]))
      return fail(JXB_ERR_INVALID, "jxb_cnn_create: channels must be in {4,8,12,16,24,32,48,64}");
  jxb_cnn* N = new jxb_cnn();
  N->in_ch = in_ch;
  N->out_ch = out_ch;
  N->levels = levels;
  for (int i = 0; i < levels; ++i) N->c[i] = channels[i];
  struct Spec { int ci, co, k; bool relu; };
  std::vector<Spec> spec;
  int prev = in_ch;
  for (int l = 0; l < levels - 1; ++l) {
    spec.push_back({prev, channels[l], 3, true});
    spec.push_back({channels[l], channels[l], 3, true});
    prev = channels[l];
  }
  const int cb = channels[levels - 1];
  spec.push_back({prev, cb, 3, true});
  spec.push_back({cb, cb, 3, true});
  spec.push_back({cb, cb, 3, true});
  for (int l = levels - 2; l >= 0; --l) {
    spec.push_back({channels[l + 1], channels[l], 1, false});
    spec.push_back({channels[l], channels[l], 3, true});
  }
  spec.push_back({channels[0], 4, 3, false});  // output padded to 4 channels for the conv kernel
  long long off = 0;
  for (const Spec& sp : spec) {
    Layer L;
    L.ci = sp.ci;
    L.co = sp.co;
    L.k = sp.k;
    L.relu = sp.relu;
    L.w_off = off;
    off += (long long)L.co * L.ci * L.k * L.k * L.k;
    L.b_off = off;
    off += L.co;
    N->L.push_back(L);
  }
  N->n_params = off;
  auto bail = [&](cudaError_t e) {
    int code = cuda_fail(e, "jxb_cnn_create");
    cudaFree(N->p);
    cudaFree(N->g);
    cudaFree(N->m);
    cudaFree(N->v);
    cudaFree(N->wt);
    cudaFree(N->red);
    delete N;
    return code;
  };
  cudaError_t e;
  if ((e = cudaMalloc(&N->p, off * sizeof(float))) != cudaSuccess) return bail(e);
  if ((e = cudaMalloc(&N->g, off * sizeof(float))) != cudaSuccess) return bail(e);
  if ((e = cudaMalloc(&N->m, off * sizeof(float))) != cudaSuccess) return bail(e);
  if ((e = cudaMalloc(&N->v, off * sizeof(float))) != cudaSuccess) return bail(e);
  long long wmax = 0;
  for (const Layer& L : N->L) wmax = std::max(wmax, (long long)L.co * L.ci * 27);
  if ((e = cudaMalloc(&N->wt, wmax * sizeof(float))) != cudaSuccess) return bail(e);
  if ((e = cudaMalloc(&N->red, 2 * JXB_RED_BLOCKS * sizeof(double))) != cudaSuccess) return bail(e);
  cudaMemset(N->g, 0, off * sizeof(float));
  cudaMemset(N->m, 0, off * sizeof(float));
  cudaMemset(N->v, 0, off * sizeof(float));
  // He-uniform weights, zero biases; the output layer starts small
  const int last = out_layer(N);
  for (int i = 0; i <= last; ++i) {
    const Layer& L = N->L[i];
    long long nw = (long long)L.co * L.ci * L.k * L.k * L.k;
    float fan_in = (float)(L.ci * L.k * L.k * L.k);
    float a = sqrtf(6.f / fan_in) * (i == last ? 0.1f : 1.f);
    k_init<<<nblk(nw), 256>>>(nw, seed * 1000003ull + i, a, N->p + L.w_off);
    cudaMemset(N->p + L.b_off, 0, L.co * sizeof(float));
  }
  // zero the padding output channels of the last layer (only out_ch are used)
  {
    const Layer& L = N->L[last];
    long long per = (long long)L.ci * 27;
    if (out_ch < L.co) cudaMemset(N->p + L.w_off + out_ch * per, 0, (L.co - out_ch) * per * sizeof(float));
  }
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return bail(e);
  *out = N;
  return JXB_OK;
}

extern "C" int jxb_cnn_destroy(jxb_cnn* N) {
  if (!N) return JXB_OK;
  cudaDeviceSynchronize();
  cudaFree(N->p);
  cudaFree(N->g);
  cudaFree(N->m);
  cudaFree(N->v);
  cudaFree(N->wt);
  cudaFree(N->part);
  cudaFree(N->cpart);
  cudaFree(N->red);
  cudaFree(N->wbf);
  cudaFree(N->arena);
  cudaFree(N->fine_arena);
  delete N;
  return JXB_OK;
}

extern "C" int jxb_cnn_set_inference_bf16(jxb_cnn* N, int on) {
  if (!N || (on != 0 && on != 1)) return fail(JXB_ERR_INVALID, "jxb_cnn_set_inference_bf16: bad argument");
  N->bf16 = on;
  return JXB_OK;
}

extern "C" int jxb_cnn_set_input_pooling(jxb_cnn* N, int on) {
  if (!N || (on != 0 && on != 1)) return fail(JXB_ERR_INVALID, "jxb_cnn_set_input_pooling: bad argument");
  if (N->pool_in != on) {
    JXB_CUDA(cudaDeviceSynchronize());
    cudaFree(N->arena);
    N->arena = nullptr;
    N->cap = {0, 0, 0};
    N->last = {0, 0, 0};
    N->pool_in = on;
  }
  return JXB_OK;
}

extern "C" int jxb_cnn_params(jxb_cnn* N, float** params, int64_t* n) {
  if (!N || !params || !n) return fail(JXB_ERR_INVALID, "jxb_cnn_params: null argument");
  *params = N->p;
  *n = N->n_params;
  return JXB_OK;
}

extern "C" int jxb_cnn_grads(jxb_cnn* N, float** grads, int64_t* n) {
  if (!N || !grads || !n) return fail(JXB_ERR_INVALID, "jxb_cnn_grads: null argument");
  *grads = N->g;
  *n = N->n_params;
  return JXB_OK;
}

extern "C" int jxb_cnn_forward(jxb_cnn* N, jxb_stream stream, int nx, int ny, int nz, const float* in, float* out) {
  if (!N || !in || !out || nx < 1 || ny < 1 || nz < 1) return fail(JXB_ERR_INVALID, "jxb_cnn_forward: bad argument");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  Dims d{nx, ny, nz};
  int rc = forward_top(N, s, d, in, true);
  if (rc) return rc;
  JXB_CUDA(cudaMemcpyAsync(out, out_buf(N), (size_t)N->out_ch * d.vox() * sizeof(float), cudaMemcpyDeviceToDevice, s));
  return JXB_OK;
}

extern "C" int jxb_cnn_backward(jxb_cnn* N, jxb_stream stream, int nx, int ny, int nz, const float* in,
                                const float* gout) {
  if (!N || !in || !gout || nx < 1 || ny < 1 || nz < 1) return fail(JXB_ERR_INVALID, "jxb_cnn_backward: bad argument");
  if (N->last.nx != nx || N->last.ny != ny || N->last.nz != nz)
    return fail(JXB_ERR_INVALID, "jxb_cnn_backward: no forward pass on these dimensions precedes it");
  if (N->last_bf16)
    return fail(JXB_ERR_INVALID, "jxb_cnn_backward: the preceding forward ran in BF16 inference mode; "
                                 "turn it off (jxb_cnn_set_inference_bf16) before training");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  Dims d{nx, ny, nz};
  const size_t vb = (size_t)d.vox() * sizeof(float);
  float* g0 = gout_buf(N);
  JXB_CUDA(cudaMemcpyAsync(g0, gout, N->out_ch * vb, cudaMemcpyDeviceToDevice, s));
  JXB_CUDA(cudaMemsetAsync(g0 + (size_t)N->out_ch * d.vox(), 0, (4 - N->out_ch) * vb, s));
  return backward_top(N, s, d, in);
}

extern "C" int jxb_cnn_zero_grad(jxb_cnn* N, jxb_stream stream) {
  if (!N) return fail(JXB_ERR_INVALID, "jxb_cnn_zero_grad: null argument");
  JXB_CUDA(cudaMemsetAsync(N->g, 0, N->n_params * sizeof(float), reinterpret_cast<cudaStream_t>(stream)));
  return JXB_OK;
}

extern "C" int jxb_cnn_accumulate(jxb_cnn* N, jxb_stream stream, int nx, int ny, int nz, const float* in,
                                  const float* target, const float* mask, double* loss) {
  if (!N || !in || !target) return fail(JXB_ERR_INVALID, "jxb_cnn_accumulate: null argument");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  Dims d{nx, ny, nz};
  int rc = forward_top(N, s, d, in);
  if (rc) return rc;
  float* g0 = gout_buf(N);
  // loss on the first out_ch channels of the (4-channel padded) output
  k_mse<<<JXB_RED_BLOCKS, 256, 0, s>>>(d.vox(), N->out_ch, out_buf(N), target, mask, g0, N->red);
  JXB_CUDA(cudaMemsetAsync(g0 + (size_t)N->out_ch * d.vox(), 0, (size_t)(4 - N->out_ch) * d.vox() * sizeof(float), s));
  std::vector<double> h(2 * JXB_RED_BLOCKS);
  JXB_CUDA(cudaMemcpyAsync(h.data(), N->red, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  JXB_CUDA(cudaStreamSynchronize(s));
  double a = 0, m = 0;
  for (int i = 0; i < JXB_RED_BLOCKS; ++i) {
    a += h[2 * i];
    m += h[2 * i + 1];
  }
  double denom = m > 0 ? m : 1.0;
  k_scale<<<nblk((long long)N->out_ch * d.vox()), 256, 0, s>>>((long long)N->out_ch * d.vox(), (float)(1.0 / denom), g0);
  rc = backward_top(N, s, d, in);
  if (rc) return rc;
  if (loss) *loss = a / denom;
  return JXB_OK;
}

extern "C" int jxb_cnn_adam(jxb_cnn* N, jxb_stream stream, float lr, float grad_scale) {
  if (!N) return fail(JXB_ERR_INVALID, "jxb_cnn_adam: null argument");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  N->adam_t += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  float bc1 = 1.f - powf(b1, (float)N->adam_t), bc2 = 1.f - powf(b2, (float)N->adam_t);
  k_adam<<<nblk(N->n_params), 256, 0, s>>>(N->n_params, lr, b1, b2, 1e-8f, bc1, bc2, grad_scale, N->p, N->g, N->m, N->v);
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}
