// A small 3D convolutional network on the control-point grid, used as a
// learned preconditioner inside flexible CG (the fourth AI-systems form of
// the solver; it has no counterpart in the reference, whose preconditioner
// is Jacobi, src/jaxiga/solvers/linear.py:419-431).
//
// Topology (channels c0, c1, c2; every conv 3x3x3 with zero padding unless
// marked 1x1; "relu" = rectified output):
//
//   level 0 (n0)          level 1 (n1 = ceil(n0/2))     level 2 (n2 = ceil(n1/2))
//   in  -> c0 relu        pool(s0) -> c1 relu           pool(s1) -> c2 relu
//   c0  -> c0 relu = s0   c1 -> c1 relu = s1            c2 -> c2 relu
//                                                      c2 -> c2 relu
//                         up -> 1x1 c2->c1 (+ s1)
//                         c1 -> c1 relu
//   up -> 1x1 c1->c0 (+ s0)
//   c0 -> c0 relu
//   c0 -> out (linear)
//
// Pooling averages the (up to eight) children of a coarse voxel; upsampling
// copies a coarse voxel to its children. All kernels are FP32 with
// deterministic reductions (fixed partial-sum grids), so training is
// reproducible run to run. Activations are [channel][z][y][x].
#include <math.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "jxb_internal.cuh"

struct jxb_cnn;

namespace jxb {
namespace cnn {

constexpr int TXV = 8, TYV = 8, TZV = 4, TV = TXV * TYV * TZV;  // output tile of the conv kernels
struct Dims {
  int nx, ny, nz;
  __host__ __device__ long long vox() const { return (long long)nx * ny * nz; }
};

static Dims half(Dims d) { return {(d.nx + 1) / 2, (d.ny + 1) / 2, (d.nz + 1) / 2}; }

// out[co] = b[co] + sum_ci sum_k w[co][ci][k] in[ci](v + k)   (+ add[co]) (relu)
// K = 3 (27 taps, zero padding) or K = 1. One thread per output voxel, all
// output channels in registers; input halo tile and weights of one input
// channel at a time in shared memory. beta: out = beta * out + result.
template <int K, int CO>
__global__ void __launch_bounds__(TV) k_conv(Dims d, int ci_n, const float* __restrict__ in, const float* __restrict__ w,
                                            const float* __restrict__ bias, const float* __restrict__ add, int relu,
                                            float beta, float* __restrict__ out) {
  constexpr int R = K / 2, HX = TXV + 2 * R, HY = TYV + 2 * R, HZ = TZV + 2 * R, KK = K * K * K;
  __shared__ __align__(16) float tile[HZ * HY * HX];
  __shared__ __align__(16) float sw[KK * CO];  // [k][co]
  const int tx = threadIdx.x % TXV, ty = (threadIdx.x / TXV) % TYV, tz = threadIdx.x / (TXV * TYV);
  const int ntx = (d.nx + TXV - 1) / TXV, nty = (d.ny + TYV - 1) / TYV;
  const int bx = blockIdx.x % ntx, by = (blockIdx.x / ntx) % nty, bz = blockIdx.x / (ntx * nty);
  const int x = bx * TXV + tx, y = by * TYV + ty, z = bz * TZV + tz;
  const bool valid = x < d.nx && y < d.ny && z < d.nz;
  const long long vox = d.vox();
  float acc[CO];
#pragma unroll
  for (int co = 0; co < CO; ++co) acc[co] = bias ? bias[co] : 0.f;
  for (int ci = 0; ci < ci_n; ++ci) {
    for (int i = threadIdx.x; i < HZ * HY * HX; i += TV) {
      int hx = i % HX, hy = (i / HX) % HY, hz = i / (HX * HY);
      int gx = bx * TXV + hx - R, gy = by * TYV + hy - R, gz = bz * TZV + hz - R;
      float v = 0.f;
      if (gx >= 0 && gy >= 0 && gz >= 0 && gx < d.nx && gy < d.ny && gz < d.nz)
        v = in[(long long)ci * vox + ((long long)gz * d.ny + gy) * d.nx + gx];
      tile[i] = v;
    }
    for (int i = threadIdx.x; i < KK * CO; i += TV) {
      int k = i / CO, co = i % CO;
      sw[i] = w[((long long)co * ci_n + ci) * KK + k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < KK; ++k) {
      const int dx = k % K, dy = (k / K) % K, dz = k / (K * K);
      const float v = tile[((tz + dz) * HY + (ty + dy)) * HX + (tx + dx)];
      const float4* w4 = reinterpret_cast<const float4*>(sw + k * CO);
#pragma unroll
      for (int c4 = 0; c4 < CO / 4; ++c4) {
        float4 ww = w4[c4];
        acc[4 * c4 + 0] += ww.x * v;
        acc[4 * c4 + 1] += ww.y * v;
        acc[4 * c4 + 2] += ww.z * v;
        acc[4 * c4 + 3] += ww.w * v;
      }
    }
    __syncthreads();
  }
  if (!valid) return;
  const long long o = ((long long)z * d.ny + y) * d.nx + x;
#pragma unroll
  for (int co = 0; co < CO; ++co) {
    float v = acc[co];
    if (add) v += add[co * vox + o];
    if (relu) v = fmaxf(v, 0.f);
    float* dst = out + co * vox + o;
    *dst = beta != 0.f ? beta * *dst + v : v;
  }
}

// Weight/bias gradient partials of one tile: dw[co][ci][k] = sum_v g[co](v) in[ci](v+k).
// Grid: (tiles, ci). Each block writes its partial to part[(tile * ci_n + ci) * (co_n*KK)].
// Threads loop over (co, k) pairs; gout tile for all co and the input halo in shared memory.
template <int K>
__global__ void __launch_bounds__(256) k_conv_wgrad(Dims d, int ci_n, int co_n, const float* __restrict__ in,
                                                  const float* __restrict__ g, float* __restrict__ part,
                                                  float* __restrict__ bpart) {
  constexpr int R = K / 2, HX = TXV + 2 * R, HY = TYV + 2 * R, HZ = TZV + 2 * R, KK = K * K * K;
  extern __shared__ float sm[];
  float* tile = sm;                 // [HZ][HY][HX]
  float* gt = sm + HZ * HY * HX;    // [co][TV]
  const int ntx = (d.nx + TXV - 1) / TXV, nty = (d.ny + TYV - 1) / TYV;
  const int t = blockIdx.x, ci = blockIdx.y;
  const int bx = t % ntx, by = (t / ntx) % nty, bz = t / (ntx * nty);
  const long long vox = d.vox();
  for (int i = threadIdx.x; i < HZ * HY * HX; i += blockDim.x) {
    int hx = i % HX, hy = (i / HX) % HY, hz = i / (HX * HY);
    int gx = bx * TXV + hx - R, gy = by * TYV + hy - R, gz = bz * TZV + hz - R;
    float v = 0.f;
    if (gx >= 0 && gy >= 0 && gz >= 0 && gx < d.nx && gy < d.ny && gz < d.nz)
      v = in[(long long)ci * vox + ((long long)gz * d.ny + gy) * d.nx + gx];
    tile[i] = v;
  }
  for (int i = threadIdx.x; i < co_n * TV; i += blockDim.x) {
    int co = i / TV, v = i % TV;
    int tx = v % TXV, ty = (v / TXV) % TYV, tz = v / (TXV * TYV);
    int x = bx * TXV + tx, y = by * TYV + ty, z = bz * TZV + tz;
    float gv = 0.f;
    if (x < d.nx && y < d.ny && z < d.nz) gv = g[(long long)co * vox + ((long long)z * d.ny + y) * d.nx + x];
    gt[i] = gv;
  }
  __syncthreads();
  float* dst = part + ((long long)t * ci_n + ci) * co_n * KK;
  for (int p = threadIdx.x; p < co_n * KK; p += blockDim.x) {
    const int co = p / KK, k = p % KK;
    const int dx = k % K, dy = (k / K) % K, dz = k / (K * K);
    const float* gg = gt + co * TV;
    float s = 0.f;
    for (int v = 0; v < TV; ++v) {
      int tx = v % TXV, ty = (v / TXV) % TYV, tz = v / (TXV * TYV);
      s += gg[v] * tile[((tz + dz) * HY + (ty + dy)) * HX + (tx + dx)];
    }
    dst[p] = s;
  }
  if (ci == 0 && bpart) {
    for (int co = threadIdx.x; co < co_n; co += blockDim.x) {
      float s = 0.f;
      for (int v = 0; v < TV; ++v) s += gt[co * TV + v];
      bpart[(long long)t * co_n + co] = s;
    }
  }
}

// grad[w] += sum over tiles of part (fixed order); one thread per weight.
__global__ void k_reduce_parts(long long n_tiles, int ci_n, int co_n, int KK, const float* __restrict__ part,
                               const float* __restrict__ bpart, float* __restrict__ dw, float* __restrict__ db) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long nw = (long long)co_n * ci_n * KK;
  if (i < nw) {
    int k = (int)(i % KK), ci = (int)((i / KK) % ci_n), co = (int)(i / ((long long)KK * ci_n));
    double s = 0.0;
    for (long long t = 0; t < n_tiles; ++t) s += part[((t * ci_n + ci) * co_n + co) * KK + k];
    dw[i] += (float)s;
  } else if (i < nw + co_n && db) {
    int co = (int)(i - nw);
    double s = 0.0;
    for (long long t = 0; t < n_tiles; ++t) s += bpart[t * co_n + co];
    db[co] += (float)s;
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

// average of the children (ceil division of odd sizes)
__global__ void k_pool(Dims f, Dims c, int ch, const float* __restrict__ in, float* __restrict__ out) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long cv = c.vox();
  if (i >= cv * ch) return;
  long long o = i % cv;
  int k = (int)(i / cv);
  int x = (int)(o % c.nx), y = (int)((o / c.nx) % c.ny), z = (int)(o / ((long long)c.nx * c.ny));
  float s = 0.f;
  int n = 0;
  for (int dz = 0; dz < 2; ++dz)
    for (int dy = 0; dy < 2; ++dy)
      for (int dx = 0; dx < 2; ++dx) {
        int X = 2 * x + dx, Y = 2 * y + dy, Z = 2 * z + dz;
        if (X < f.nx && Y < f.ny && Z < f.nz) {
          s += in[(long long)k * f.vox() + ((long long)Z * f.ny + Y) * f.nx + X];
          ++n;
        }
      }
  out[i] = s / n;
}

// backward of k_pool: each fine voxel receives g_coarse / (children of its parent); beta accumulates
__global__ void k_pool_bwd(Dims f, Dims c, int ch, const float* __restrict__ gc, float beta, float* __restrict__ gf) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long fv = f.vox();
  if (i >= fv * ch) return;
  long long o = i % fv;
  int k = (int)(i / fv);
  int X = (int)(o % f.nx), Y = (int)((o / f.nx) % f.ny), Z = (int)(o / ((long long)f.nx * f.ny));
  int x = X / 2, y = Y / 2, z = Z / 2;
  int nxc = min(2, f.nx - 2 * x), nyc = min(2, f.ny - 2 * y), nzc = min(2, f.nz - 2 * z);
  float v = gc[(long long)k * c.vox() + ((long long)z * c.ny + y) * c.nx + x] / (nxc * nyc * nzc);
  gf[i] = beta != 0.f ? beta * gf[i] + v : v;
}

__global__ void k_up(Dims f, Dims c, int ch, const float* __restrict__ in, float* __restrict__ out) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long fv = f.vox();
  if (i >= fv * ch) return;
  long long o = i % fv;
  int k = (int)(i / fv);
  int X = (int)(o % f.nx), Y = (int)((o / f.nx) % f.ny), Z = (int)(o / ((long long)f.nx * f.ny));
  out[i] = in[(long long)k * c.vox() + ((long long)(Z / 2) * c.ny + Y / 2) * c.nx + X / 2];
}

__global__ void k_up_bwd(Dims f, Dims c, int ch, const float* __restrict__ gf, float* __restrict__ gc) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long cv = c.vox();
  if (i >= cv * ch) return;
  long long o = i % cv;
  int k = (int)(i / cv);
  int x = (int)(o % c.nx), y = (int)((o / c.nx) % c.ny), z = (int)(o / ((long long)c.nx * c.ny));
  float s = 0.f;
  for (int dz = 0; dz < 2; ++dz)
    for (int dy = 0; dy < 2; ++dy)
      for (int dx = 0; dx < 2; ++dx) {
        int X = 2 * x + dx, Y = 2 * y + dy, Z = 2 * z + dz;
        if (X < f.nx && Y < f.ny && Z < f.nz) s += gf[(long long)k * f.vox() + ((long long)Z * f.ny + Y) * f.nx + X];
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

struct Layer {
  int ci, co, k;  // kernel size 1 or 3
  bool relu;
  long long w_off, b_off;  // offsets in the flat parameter vector
};

}  // namespace cnn
}  // namespace jxb

using namespace jxb;
using namespace jxb::cnn;

// layer indices in the fixed topology
enum { L0A, L0B, L1A, L1B, L2A, L2B, L2C, L1C, L1D, L0C, L0D, L0E, NLAYERS };

struct jxb_cnn {
  int in_ch, out_ch, c[3];
  Layer L[NLAYERS];
  long long n_params = 0;
  float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  long long adam_t = 0;
  // activation / gradient buffers sized for `cap` voxels at level 0
  long long cap = 0;
  std::vector<float*> bufs;
  float* wt = nullptr;     // transposed weights scratch
  float* part = nullptr;   // weight-gradient partials
  long long part_cap = 0;
  double* red = nullptr;   // loss partials
  float* h_loss_dummy = nullptr;
};

namespace {

int conv(cudaStream_t s, Dims d, const Layer& L, const float* p, const float* in, const float* add, float beta,
         float* out) {
  long long tiles = (long long)((d.nx + TXV - 1) / TXV) * ((d.ny + TYV - 1) / TYV) * ((d.nz + TZV - 1) / TZV);
  const float* w = p + L.w_off;
  const float* b = L.b_off >= 0 ? p + L.b_off : nullptr;
  int relu = L.relu ? 1 : 0;
#define JXB_CONV(KS, CO)                                                                             \
  if (L.k == KS && L.co == CO) {                                                                     \
    k_conv<KS, CO><<<(unsigned)tiles, TV, 0, s>>>(d, L.ci, in, w, b, add, relu, beta, out);           \
    JXB_CUDA(cudaGetLastError());                                                                    \
    return JXB_OK;                                                                                   \
  }
  JXB_CONV(3, 4) JXB_CONV(3, 8) JXB_CONV(3, 12) JXB_CONV(3, 16) JXB_CONV(3, 24) JXB_CONV(3, 32) JXB_CONV(3, 48)
  JXB_CONV(1, 4) JXB_CONV(1, 8) JXB_CONV(1, 12) JXB_CONV(1, 16) JXB_CONV(1, 24) JXB_CONV(1, 32) JXB_CONV(1, 48)
#undef JXB_CONV
  return fail(JXB_ERR_INVALID, "cnn: unsupported output channel count " + std::to_string(L.co));
}

// data gradient of a conv layer: gin = beta*gin + conv^T(g)
int conv_dgrad(jxb_cnn* N, cudaStream_t s, Dims d, const Layer& L, const float* g, float beta, float* gin) {
  int KK = L.k * L.k * L.k;
  int n = L.co * L.ci * KK;
  k_transpose_w<<<(n + 255) / 256, 256, 0, s>>>(L.co, L.ci, KK, N->p + L.w_off, N->wt);
  Layer T{L.co, L.ci, L.k, false, 0, -1};
  return conv(s, d, T, N->wt, g, nullptr, beta, gin);
}

int conv_wgrad(jxb_cnn* N, cudaStream_t s, Dims d, const Layer& L, const float* in, const float* g) {
  long long tiles = (long long)((d.nx + TXV - 1) / TXV) * ((d.ny + TYV - 1) / TYV) * ((d.nz + TZV - 1) / TZV);
  int KK = L.k * L.k * L.k;
  long long need = tiles * L.ci * L.co * KK + tiles * L.co;
  if (need > N->part_cap) {
    cudaFree(N->part);
    JXB_CUDA(cudaMalloc(&N->part, need * sizeof(float)));
    N->part_cap = need;
  }
  float* bpart = N->part + tiles * L.ci * L.co * KK;
  int R = L.k / 2;
  size_t sm = ((TXV + 2 * R) * (TYV + 2 * R) * (TZV + 2 * R) + (size_t)L.co * TV) * sizeof(float);
  dim3 grid((unsigned)tiles, L.ci);
  if (L.k == 3) {
    if (sm > 48 * 1024) JXB_CUDA(cudaFuncSetAttribute(k_conv_wgrad<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_conv_wgrad<3><<<grid, 256, sm, s>>>(d, L.ci, L.co, in, g, N->part, L.b_off >= 0 ? bpart : nullptr);
  } else {
    if (sm > 48 * 1024) JXB_CUDA(cudaFuncSetAttribute(k_conv_wgrad<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_conv_wgrad<1><<<grid, 256, sm, s>>>(d, L.ci, L.co, in, g, N->part, L.b_off >= 0 ? bpart : nullptr);
  }
  JXB_CUDA(cudaGetLastError());
  long long nw = (long long)L.co * L.ci * KK + (L.b_off >= 0 ? L.co : 0);
  k_reduce_parts<<<(unsigned)((nw + 255) / 256), 256, 0, s>>>(tiles, L.ci, L.co, KK, N->part, bpart, N->g + L.w_off,
                                                             L.b_off >= 0 ? N->g + L.b_off : nullptr);
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

inline unsigned nblk(long long n) { return (unsigned)((n + 255) / 256); }

// buffer indices
enum { A0A, S0, P1, A1A, S1, P2, A2A, A2B, A2C, U1, M1, A1D, U0, M0, A0D, OUT,
       G0, G1, G2, G3, NBUF };

int ensure_bufs(jxb_cnn* N, Dims d0) {
  long long v0 = d0.vox();
  if (v0 <= N->cap) return JXB_OK;
  for (float* b : N->bufs) cudaFree(b);
  N->bufs.assign(NBUF, nullptr);
  Dims d1 = half(d0), d2 = half(d1);
  long long v1 = d1.vox(), v2 = d2.vox();
  int c0 = N->c[0], c1 = N->c[1], c2 = N->c[2];
  long long sizes[NBUF] = {c0 * v0, c0 * v0, c0 * v1, c1 * v1, c1 * v1, c1 * v2, c2 * v2, c2 * v2, c2 * v2,
                           c2 * v1, c1 * v1, c1 * v1, c1 * v0, c0 * v0, c0 * v0, (long long)N->L[L0E].co * v0,
                           0, 0, 0, 0};
  long long gmax = 0;
  for (int i = 0; i < OUT + 1; ++i) gmax = std::max(gmax, sizes[i]);
  gmax = std::max(gmax, (long long)N->in_ch * v0);
  for (int i = G0; i <= G3; ++i) sizes[i] = gmax;
  for (int i = 0; i < NBUF; ++i) JXB_CUDA(cudaMalloc(&N->bufs[i], std::max<long long>(sizes[i], 1) * sizeof(float)));
  N->cap = v0;
  return JXB_OK;
}

int forward(jxb_cnn* N, cudaStream_t s, Dims d0, const float* in, float* out) {
  int rc = ensure_bufs(N, d0);
  if (rc) return rc;
  Dims d1 = half(d0), d2 = half(d1);
  auto& B = N->bufs;
  const float* p = N->p;
  if ((rc = conv(s, d0, N->L[L0A], p, in, nullptr, 0.f, B[A0A]))) return rc;
  if ((rc = conv(s, d0, N->L[L0B], p, B[A0A], nullptr, 0.f, B[S0]))) return rc;
  k_pool<<<nblk(d1.vox() * N->c[0]), 256, 0, s>>>(d0, d1, N->c[0], B[S0], B[P1]);
  if ((rc = conv(s, d1, N->L[L1A], p, B[P1], nullptr, 0.f, B[A1A]))) return rc;
  if ((rc = conv(s, d1, N->L[L1B], p, B[A1A], nullptr, 0.f, B[S1]))) return rc;
  k_pool<<<nblk(d2.vox() * N->c[1]), 256, 0, s>>>(d1, d2, N->c[1], B[S1], B[P2]);
  if ((rc = conv(s, d2, N->L[L2A], p, B[P2], nullptr, 0.f, B[A2A]))) return rc;
  if ((rc = conv(s, d2, N->L[L2B], p, B[A2A], nullptr, 0.f, B[A2B]))) return rc;
  if ((rc = conv(s, d2, N->L[L2C], p, B[A2B], nullptr, 0.f, B[A2C]))) return rc;
  k_up<<<nblk(d1.vox() * N->c[2]), 256, 0, s>>>(d1, d2, N->c[2], B[A2C], B[U1]);
  if ((rc = conv(s, d1, N->L[L1C], p, B[U1], B[S1], 0.f, B[M1]))) return rc;
  if ((rc = conv(s, d1, N->L[L1D], p, B[M1], nullptr, 0.f, B[A1D]))) return rc;
  k_up<<<nblk(d0.vox() * N->c[1]), 256, 0, s>>>(d0, d1, N->c[1], B[A1D], B[U0]);
  if ((rc = conv(s, d0, N->L[L0C], p, B[U0], B[S0], 0.f, B[M0]))) return rc;
  if ((rc = conv(s, d0, N->L[L0D], p, B[M0], nullptr, 0.f, B[A0D]))) return rc;
  if ((rc = conv(s, d0, N->L[L0E], p, B[A0D], nullptr, 0.f, out ? out : B[OUT]))) return rc;
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

// Backward through the network for the output gradient in G0 (layout of OUT);
// accumulates parameter gradients into N->g.
int backward(jxb_cnn* N, cudaStream_t s, Dims d0, const float* in) {
  Dims d1 = half(d0), d2 = half(d1);
  auto& B = N->bufs;
  int c0 = N->c[0], c1 = N->c[1], c2 = N->c[2];
  float *gA = B[G0], *gB = B[G1], *gS0 = B[G2], *gS1 = B[G3];
  int rc;
  // L0E (linear): gA = dL/dOUT
  if ((rc = conv_wgrad(N, s, d0, N->L[L0E], B[A0D], gA))) return rc;
  if ((rc = conv_dgrad(N, s, d0, N->L[L0E], gA, 0.f, gB))) return rc;  // dL/dA0D
  k_relu_mask<<<nblk(c0 * d0.vox()), 256, 0, s>>>(c0 * d0.vox(), B[A0D], gB);
  if ((rc = conv_wgrad(N, s, d0, N->L[L0D], B[M0], gB))) return rc;
  if ((rc = conv_dgrad(N, s, d0, N->L[L0D], gB, 0.f, gA))) return rc;  // dL/dM0 (linear output of L0C + S0)
  // M0 = L0C(U0) + S0: dS0 = gA, dU0 = L0C^T gA
  JXB_CUDA(cudaMemcpyAsync(gS0, gA, c0 * d0.vox() * sizeof(float), cudaMemcpyDeviceToDevice, s));
  if ((rc = conv_wgrad(N, s, d0, N->L[L0C], B[U0], gA))) return rc;
  if ((rc = conv_dgrad(N, s, d0, N->L[L0C], gA, 0.f, gB))) return rc;  // dL/dU0 [c1 @ n0]
  k_up_bwd<<<nblk(c1 * d1.vox()), 256, 0, s>>>(d0, d1, c1, gB, gA);       // dL/dA1D [c1 @ n1]
  k_relu_mask<<<nblk(c1 * d1.vox()), 256, 0, s>>>(c1 * d1.vox(), B[A1D], gA);
  if ((rc = conv_wgrad(N, s, d1, N->L[L1D], B[M1], gA))) return rc;
  if ((rc = conv_dgrad(N, s, d1, N->L[L1D], gA, 0.f, gB))) return rc;  // dL/dM1
  JXB_CUDA(cudaMemcpyAsync(gS1, gB, c1 * d1.vox() * sizeof(float), cudaMemcpyDeviceToDevice, s));
  if ((rc = conv_wgrad(N, s, d1, N->L[L1C], B[U1], gB))) return rc;
  if ((rc = conv_dgrad(N, s, d1, N->L[L1C], gB, 0.f, gA))) return rc;  // dL/dU1 [c2 @ n1]
  k_up_bwd<<<nblk(c2 * d2.vox()), 256, 0, s>>>(d1, d2, c2, gA, gB);       // dL/dA2C
  k_relu_mask<<<nblk(c2 * d2.vox()), 256, 0, s>>>(c2 * d2.vox(), B[A2C], gB);
  if ((rc = conv_wgrad(N, s, d2, N->L[L2C], B[A2B], gB))) return rc;
  if ((rc = conv_dgrad(N, s, d2, N->L[L2C], gB, 0.f, gA))) return rc;
  k_relu_mask<<<nblk(c2 * d2.vox()), 256, 0, s>>>(c2 * d2.vox(), B[A2B], gA);
  if ((rc = conv_wgrad(N, s, d2, N->L[L2B], B[A2A], gA))) return rc;
  if ((rc = conv_dgrad(N, s, d2, N->L[L2B], gA, 0.f, gB))) return rc;
  k_relu_mask<<<nblk(c2 * d2.vox()), 256, 0, s>>>(c2 * d2.vox(), B[A2A], gB);
  if ((rc = conv_wgrad(N, s, d2, N->L[L2A], B[P2], gB))) return rc;
  if ((rc = conv_dgrad(N, s, d2, N->L[L2A], gB, 0.f, gA))) return rc;  // dL/dP2 [c1 @ n2]
  k_pool_bwd<<<nblk(c1 * d1.vox()), 256, 0, s>>>(d1, d2, c1, gA, 1.f, gS1);  // dS1 += pool^T
  k_relu_mask<<<nblk(c1 * d1.vox()), 256, 0, s>>>(c1 * d1.vox(), B[S1], gS1);
  if ((rc = conv_wgrad(N, s, d1, N->L[L1B], B[A1A], gS1))) return rc;
  if ((rc = conv_dgrad(N, s, d1, N->L[L1B], gS1, 0.f, gA))) return rc;
  k_relu_mask<<<nblk(c1 * d1.vox()), 256, 0, s>>>(c1 * d1.vox(), B[A1A], gA);
  if ((rc = conv_wgrad(N, s, d1, N->L[L1A], B[P1], gA))) return rc;
  if ((rc = conv_dgrad(N, s, d1, N->L[L1A], gA, 0.f, gB))) return rc;  // dL/dP1 [c0 @ n1]
  k_pool_bwd<<<nblk(c0 * d0.vox()), 256, 0, s>>>(d0, d1, c0, gB, 1.f, gS0);
  k_relu_mask<<<nblk(c0 * d0.vox()), 256, 0, s>>>(c0 * d0.vox(), B[S0], gS0);
  if ((rc = conv_wgrad(N, s, d0, N->L[L0B], B[A0A], gS0))) return rc;
  if ((rc = conv_dgrad(N, s, d0, N->L[L0B], gS0, 0.f, gA))) return rc;
  k_relu_mask<<<nblk(c0 * d0.vox()), 256, 0, s>>>(c0 * d0.vox(), B[A0A], gA);
  if ((rc = conv_wgrad(N, s, d0, N->L[L0A], in, gA))) return rc;
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

bool supported_co(int c) { return c == 4 || c == 8 || c == 12 || c == 16 || c == 24 || c == 32 || c == 48; }

}  // namespace

extern "C" int jxb_cnn_create(int in_ch, int out_ch, const int* channels, uint64_t seed, jxb_cnn** out) {
  if (!out || !channels || in_ch < 1 || in_ch > 8 || out_ch < 1 || out_ch > 3)
    return fail(JXB_ERR_INVALID, "jxb_cnn_create: bad argument");
  for (int i = 0; i < 3; ++i)
    if (!supported_co(channels[i])) return fail(JXB_ERR_INVALID, "jxb_cnn_create: channels must be in {4,8,12,16,24,32,48}");
  jxb_cnn* N = new jxb_cnn();
  N->in_ch = in_ch;
  N->out_ch = out_ch;
  for (int i = 0; i < 3; ++i) N->c[i] = channels[i];
  int c0 = channels[0], c1 = channels[1], c2 = channels[2];
  // the output layer's channel count must be a multiple of 4 for the conv kernel: pad to 4
  struct Spec { int ci, co, k; bool relu; } spec[NLAYERS] = {
      {in_ch, c0, 3, true}, {c0, c0, 3, true}, {c0, c1, 3, true}, {c1, c1, 3, true}, {c1, c2, 3, true},
      {c2, c2, 3, true},    {c2, c2, 3, true}, {c2, c1, 1, false}, {c1, c1, 3, true}, {c1, c0, 1, false},
      {c0, c0, 3, true},    {c0, 4, 3, false}};
  long long off = 0;
  for (int i = 0; i < NLAYERS; ++i) {
    Layer& L = N->L[i];
    L.ci = spec[i].ci;
    L.co = spec[i].co;
    L.k = spec[i].k;
    L.relu = spec[i].relu;
    L.w_off = off;
    off += (long long)L.co * L.ci * L.k * L.k * L.k;
    L.b_off = off;
    off += L.co;
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
  for (int i = 0; i < NLAYERS; ++i) wmax = std::max(wmax, (long long)N->L[i].co * N->L[i].ci * 27);
  if ((e = cudaMalloc(&N->wt, wmax * sizeof(float))) != cudaSuccess) return bail(e);
  if ((e = cudaMalloc(&N->red, 2 * JXB_RED_BLOCKS * sizeof(double))) != cudaSuccess) return bail(e);
  cudaMemset(N->g, 0, off * sizeof(float));
  cudaMemset(N->m, 0, off * sizeof(float));
  cudaMemset(N->v, 0, off * sizeof(float));
  // He-uniform weights, zero biases; the output layer starts small
  for (int i = 0; i < NLAYERS; ++i) {
    const Layer& L = N->L[i];
    long long nw = (long long)L.co * L.ci * L.k * L.k * L.k;
    float fan_in = (float)(L.ci * L.k * L.k * L.k);
    float a = sqrtf(6.f / fan_in) * (i == L0E ? 0.1f : 1.f);
    k_init<<<nblk(nw), 256>>>(nw, seed * 1000003ull + i, a, N->p + L.w_off);
    cudaMemset(N->p + L.b_off, 0, L.co * sizeof(float));
  }
  // zero the padding output channels of the last layer (only out_ch are used)
  {
    const Layer& L = N->L[L0E];
    long long per = (long long)L.ci * 27;
    if (out_ch < L.co)
      cudaMemset(N->p + L.w_off + out_ch * per, 0, (L.co - out_ch) * per * sizeof(float));
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
  cudaFree(N->red);
  for (float* b : N->bufs) cudaFree(b);
  delete N;
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
  int rc = forward(N, s, d, in, nullptr);
  if (rc) return rc;
  JXB_CUDA(cudaMemcpyAsync(out, N->bufs[OUT], (size_t)N->out_ch * d.vox() * sizeof(float), cudaMemcpyDeviceToDevice, s));
  return JXB_OK;
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
  int rc = forward(N, s, d, in, nullptr);
  if (rc) return rc;
  // loss on the first out_ch channels of the (4-channel padded) output
  k_mse<<<JXB_RED_BLOCKS, 256, 0, s>>>(d.vox(), N->out_ch, N->bufs[OUT], target, mask, N->bufs[G0], N->red);
  JXB_CUDA(cudaMemsetAsync(N->bufs[G0] + (size_t)N->out_ch * d.vox(), 0,
                           (size_t)(N->L[L0E].co - N->out_ch) * d.vox() * sizeof(float), s));
  std::vector<double> h(2 * JXB_RED_BLOCKS);
  JXB_CUDA(cudaMemcpyAsync(h.data(), N->red, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  JXB_CUDA(cudaStreamSynchronize(s));
  double a = 0, m = 0;
  for (int i = 0; i < JXB_RED_BLOCKS; ++i) {
    a += h[2 * i];
    m += h[2 * i + 1];
  }
  double denom = m > 0 ? m : 1.0;
  k_scale<<<nblk((long long)N->out_ch * d.vox()), 256, 0, s>>>((long long)N->out_ch * d.vox(), (float)(1.0 / denom), N->bufs[G0]);
  rc = backward(N, s, d, in);
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
