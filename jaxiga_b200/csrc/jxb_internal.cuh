// Internal declarations shared by the libjxb translation units.
//
// Data layout in HBM (one plan = one single-patch space + one operator):
//   * Elements are grouped into bricks. In 3D a brick is TX x TY elements in
//     (x, y) times CZ element layers in z; in 2D it is TX elements in x times
//     CY element rows in y. One CTA owns one brick, walks its layers in order
//     and accumulates element residuals into a shared-memory copy of the
//     brick's control-point footprint (deterministic, no atomics).
//   * Per-point factors ("geo") are stored element-slot-major in brick order:
//     slot = ((brick * layers + layer) * elems_per_layer + e_in_layer), and
//     per slot [factor k][quadrature point q] with q first-direction fastest.
//     One layer of a brick is therefore one contiguous tile: the apply kernels
//     prefetch the next layer's tile into L2 (cp.async.bulk.prefetch.L2) and
//     read it with coalesced loads.
//   * The brick's footprint partial sums go to a scratch buffer; a combine
//     pass sums, per control point, the (at most JXB_MAXC per direction)
//     bricks that cover it, always in the same order.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/jxb.h"

#define JXB_MAXP 5
#define JXB_MAXQ 6
#define JXB_MAXC 8          // bricks covering one control point, per direction (p + 1 for one-row 2D bricks)
#define JXB_RED_BLOCKS 296  // fixed grid of every deterministic reduction (2 x 148 SMs)
#define JXB_RED_THREADS 256

namespace jxb {

void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define JXB_CUDA(call)                                         \
  do {                                                         \
    cudaError_t _e = (call);                                   \
    if (_e != cudaSuccess) return ::jxb::cuda_fail(_e, #call); \
  } while (0)

// Deterministic reductions: warp shuffle tree, then the warps of a block in
// index order; partials of a fixed JXB_RED_BLOCKS grid summed the same way.
static __device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum returned to every thread (fixed order).
static __device__ double block_sum_all(double v) {
  __shared__ double part[32];
  __shared__ double total;
  v = warp_sum(v);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) part[w] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int i = 0; i < (int)((blockDim.x + 31) >> 5); ++i) s += part[i];
    total = s;
  }
  __syncthreads();
  double r = total;
  __syncthreads();
  return r;
}

// Sum of the JXB_RED_BLOCKS partials in a fixed order, identical in every block.
static __device__ double reduce_partials(const double* part) {
  double v = 0;
  for (int i = threadIdx.x; i < JXB_RED_BLOCKS; i += blockDim.x) v += part[i];
  return block_sum_all(v);
}

// Operator-specific constants handed to kernels by value.
struct Material {
  double lam, mu;  // elasticity (effective plane lambda in 2D)
};

// CUDA events of one solve call (two timing events and one ordering event),
// destroyed on every return path.
struct SolveEvents {
  cudaEvent_t e0 = nullptr, e1 = nullptr, order = nullptr;
  SolveEvents() = default;
  SolveEvents(const SolveEvents&) = delete;
  SolveEvents& operator=(const SolveEvents&) = delete;
  ~SolveEvents() {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (order) cudaEventDestroy(order);
  }
  int create() {
    JXB_CUDA(cudaEventCreate(&e0));
    JXB_CUDA(cudaEventCreate(&e1));
    JXB_CUDA(cudaEventCreateWithFlags(&order, cudaEventDisableTiming));
    return JXB_OK;
  }
};

// Solver state for one Krylov loop, resident in device memory.
struct CgState {
  double gamma;    // r . z
  double rr;       // r . r
  double alpha, beta;
  double bb;       // b . b
  double atol2;    // stopping threshold on r . r
  long long k;     // iterations done
  long long maxiter;
  int done;        // 1 once converged, capped or broken down
  int status;      // JXB_OK, JXB_ERR_NOT_CONVERGED, JXB_ERR_NONFINITE
};

// Device-side description of the brick grid, passed by value.
struct Bricks {
  int dim, vec, p, q;
  int n_span[3], n_cp[3];
  int nb[3];          // bricks per direction
  int te[3];          // elements per brick per direction (tx, ty, layers)
  int fp[3];          // scratch footprint per direction
  const int* first[3];   // per span: first control point
  const int* bcp0[3];    // per brick: first control point of its footprint
  const int* cover[3];   // per control point: JXB_MAXC (brick, offset) pairs
  long long n_bricks;
  long long slots;       // element slots (bricks * elems per brick)
};

// Arguments of one brick launch (one plan), passed by value or, for batched
// launches, read by each CTA from a device array.
template <typename T>
struct BrickArgs {
  Bricks br;
  const T* tab[3];       // per direction [span][3][Q][P+1]: values, d/dxi, d2/dxi2
  const T* geo;          // (slots, ngeo, nqe)
  const double* wq;      // load weights (slots, nqe)
  const T* wgts;         // NURBS weights (rational)
  const uint8_t* keep;   // (n_dofs) 1 = free
  const T* x;            // input DOF vector
  const double* f_qp;    // load: source values, reference order
  T* scratch;            // (n_bricks, vec, fp2, fp1, fp0)
  const CgState* state;  // optional: skip all work once done
  int masked;
  int* err;
  double lam, mu;
};

// 2D brick widths (elements per row TX) the kernels are built for: 32 for every
// operator, 16 and 64 for the scalar one. The rows per brick TY are a runtime
// value in [1, TILE2_MAX_ROWS].
constexpr int N_TILE2 = 3;
constexpr int TILE2X[N_TILE2] = {32, 16, 64};
constexpr int TILE2_MAX_ROWS = 64;
// Row width of every instance of a batch that the persistent batched kernel runs.
constexpr int PERSIST2_TX = 32;

// ---------------------------------------------------------------------------
// Where the per-point factors live. ngeo factors per Gauss point, nqe points
// per element, one geometry slot per element position of a brick.
//   3D: slot-major, [slot][factor][point]: one element layer of a brick (te[0]
//       x te[1] slots) is one contiguous tile.
//   2D: each brick row (te[0] consecutive slots) is one contiguous tile laid
//       out [factor][q1][element][q0], so the threads of a row, one per
//       (element, q0), read consecutive values for every (factor, q1).
// base: offset of factor 0 of point q of `slot`; stride: from one factor to
// the next.
// ---------------------------------------------------------------------------
struct GeoAt {
  size_t base, stride;
};

__host__ __device__ inline GeoAt geo_at(int dim, long long slot, int q, int Q, int ngeo, long long nqe, int te0) {
  if (dim == 3) return {(size_t)slot * ngeo * nqe + q, (size_t)nqe};
  const long long row = slot / te0;
  const int el = (int)(slot - row * te0), q0 = q % Q, q1 = q / Q;
  return {(size_t)row * te0 * ngeo * nqe + ((size_t)q1 * te0 + el) * Q + q0, (size_t)te0 * nqe};
}

// ---------------------------------------------------------------------------
// The combine's sum at one control point: y_i = the sum, over the bricks whose
// footprint holds control point i, of their footprint values -- bricks taken
// in the fixed order (z, then y, then x, each in cover-list order), so the
// result is bitwise reproducible.
//
// The cover table lists per direction and control point up to JXB_MAXC
// (brick, offset) pairs, -1 after the last. Every 3D brick shape and every 2D
// brick of at least p rows puts a control point in at most 2 bricks per
// direction; those points read their 2 x 2 (x 2) bricks with all loads issued
// together, for every component at once. Longer lists (short 2D bricks of high
// degree) take the loop over the tables.
// ---------------------------------------------------------------------------
struct Cover2 {
  int b[2], o[2];
  int n;
  bool longer;
};

__device__ __forceinline__ void cover2(const int* __restrict__ c, Cover2& C) {
  C.b[0] = c[0];
  C.o[0] = c[1];
  C.b[1] = c[2];
  C.o[1] = c[3];
  C.n = (C.b[0] >= 0) + (C.b[1] >= 0);
  C.longer = c[4] >= 0;
}

template <typename T>
__device__ __forceinline__ T cover_sum_long(const Bricks& br, const T* __restrict__ sc, int ix, int iy, int iz) {
  const int dim = br.dim;
  const long long fpz = dim == 3 ? br.fp[2] : 1;
  const int* cx = br.cover[0] + 2 * JXB_MAXC * ix;
  const int* cy = br.cover[1] + 2 * JXB_MAXC * iy;
  const int* cz = dim == 3 ? br.cover[2] + 2 * JXB_MAXC * iz : nullptr;
  T s = 0;
  for (int kz = 0; kz < (dim == 3 ? JXB_MAXC : 1); ++kz) {
    const int bz = dim == 3 ? cz[2 * kz] : 0, oz = dim == 3 ? cz[2 * kz + 1] : 0;
    if (bz < 0) break;
    for (int ky = 0; ky < JXB_MAXC; ++ky) {
      const int by = cy[2 * ky], oy = cy[2 * ky + 1];
      if (by < 0) break;
      for (int kx = 0; kx < JXB_MAXC; ++kx) {
        const int bx = cx[2 * kx], ox = cx[2 * kx + 1];
        if (bx < 0) break;
        const long long brick = bx + (long long)br.nb[0] * (by + (long long)br.nb[1] * bz);
        s += sc[((brick * br.vec * fpz + oz) * br.fp[1] + oy) * br.fp[0] + ox];
      }
    }
  }
  return s;
}

// s[c] = the combine's sum for component c of control point (ix, iy, iz).
// VEC = br.vec and DIM = br.dim.
template <typename T, int VEC, int DIM>
__device__ __forceinline__ void combine_point(const Bricks& br, const T* __restrict__ scratch, int ix, int iy, int iz,
                                              T (&s)[VEC]) {
  const long long layer = (long long)br.fp[0] * br.fp[1];
  const long long comp = (DIM == 3 ? br.fp[2] : 1) * layer;  // one component of one brick's footprint
  const long long S = VEC * comp;                            // one brick's footprint
  Cover2 cx, cy, cz;
  cover2(br.cover[0] + 2 * JXB_MAXC * ix, cx);
  cover2(br.cover[1] + 2 * JXB_MAXC * iy, cy);
  if constexpr (DIM == 3) {
    cover2(br.cover[2] + 2 * JXB_MAXC * iz, cz);
  } else {
    cz.b[0] = 0, cz.o[0] = 0, cz.b[1] = -1, cz.o[1] = 0, cz.n = 1, cz.longer = false;
  }
  if (cx.longer || cy.longer || cz.longer) {
#pragma unroll
    for (int c = 0; c < VEC; ++c) s[c] = cover_sum_long<T>(br, scratch + c * comp, ix, iy, iz);
    return;
  }
  constexpr int KZ = DIM == 3 ? 2 : 1;
  long long X[2], Y[2], Z[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    X[k] = cx.b[k] * S + cx.o[k];
    Y[k] = (long long)cy.b[k] * br.nb[0] * S + (long long)cy.o[k] * br.fp[0];
    Z[k] = (long long)cz.b[k] * br.nb[0] * br.nb[1] * S + cz.o[k] * layer;
  }
  T v[VEC][KZ * 4];
#pragma unroll
  for (int c = 0; c < VEC; ++c)
#pragma unroll
    for (int kz = 0; kz < KZ; ++kz)
#pragma unroll
      for (int ky = 0; ky < 2; ++ky)
#pragma unroll
        for (int kx = 0; kx < 2; ++kx) {
          const bool ok = kz < cz.n && ky < cy.n && kx < cx.n;
          v[c][(kz * 2 + ky) * 2 + kx] = ok ? __ldg(scratch + c * comp + Z[kz] + Y[ky] + X[kx]) : T(0);
        }
#pragma unroll
  for (int c = 0; c < VEC; ++c) {
    T a = 0;
#pragma unroll
    for (int kz = 0; kz < KZ; ++kz)
#pragma unroll
      for (int ky = 0; ky < 2; ++ky)
#pragma unroll
        for (int kx = 0; kx < 2; ++kx)
          if (kz < cz.n && ky < cy.n && kx < cx.n) a += v[c][(kz * 2 + ky) * 2 + kx];
    s[c] = a;
  }
}

}  // namespace jxb

struct jxb_krylov_ws;  // BiCGSTAB workspace (krylov.cu)
struct jxb_mp_data;    // composite multipatch plan (mp.cu)
struct jxb_thb_data;   // padded-element (THB) Poisson plan (thb.cu)

struct jxb_plan {
  int device = 0;  // the CUDA device that was current at creation; its buffers live there
  int dim, vec, p, q, op, rational, order, plane_strain;
  int n_span[3], n_cp[3];
  long long n_elem, n_scalar, n_dofs, n_free, n_qp, nqe;
  int ngeo;
  double coef[4];
  jxb::Material mat;
  jxb::Bricks br;

  // device buffers
  int* d_first[3] = {nullptr, nullptr, nullptr};
  int* d_bcp0[3] = {nullptr, nullptr, nullptr};
  int* d_cover[3] = {nullptr, nullptr, nullptr};
  double* d_tab[3] = {nullptr, nullptr, nullptr};
  double* d_ext[3] = {nullptr, nullptr, nullptr};  // (n_span, p+1, p+1) extraction operators
  double* d_lo[3] = {nullptr, nullptr, nullptr};   // span bounds
  double* d_hi[3] = {nullptr, nullptr, nullptr};
  float* d_tab32[3] = {nullptr, nullptr, nullptr};
  double* d_geo = nullptr;    // (slots, ngeo, nqe)
  float* d_geo32 = nullptr;
  double* d_wq = nullptr;     // (slots, nqe): omega / W, the load-vector weight
  double* d_invW = nullptr;   // (slots, nqe): 1 / W (rational only)
  double* d_cpts = nullptr;   // (n_scalar, dim)
  double* d_wgts = nullptr;   // (n_scalar)
  float* d_wgts32 = nullptr;
  uint8_t* d_keep = nullptr;  // (n_dofs) 1 = free
  double* d_scratch = nullptr;
  float* d_scratch32 = nullptr;
  double* d_red = nullptr;    // reduction partials, 4 x JXB_RED_BLOCKS
  // Krylov workspace (allocated on first solve)
  double *d_x = nullptr, *d_b = nullptr, *d_r = nullptr, *d_z = nullptr, *d_p = nullptr,
         *d_Ap = nullptr, *d_invdiag = nullptr;
  float *d_x32 = nullptr, *d_r32 = nullptr, *d_z32 = nullptr, *d_p32 = nullptr, *d_Ap32 = nullptr,
        *d_invdiag32 = nullptr;
  // true-residual restarts of jxb_pcg: accumulated solution and FP64 residual
  double *d_xacc = nullptr, *d_res = nullptr;
  jxb_krylov_ws* krylov = nullptr;  // allocated by the first jxb_bicgstab
  jxb::CgState* d_state = nullptr;
  jxb::CgState* h_state = nullptr;  // pinned
  bool diag_valid = false;
  // captured CG iteration graphs: [0] FP64, [1] FP32
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  int graph_iters[2] = {0, 0};
  int graph_precond[2] = {-1, -1};
  cudaStream_t graph_stream[2] = {nullptr, nullptr};
  size_t scratch_elems = 0;
  jxb_mp_data* mp = nullptr;  // set on a composite plan over several patch plans
  jxb_thb_data* thb = nullptr;  // set on a plan over a hierarchical (padded-element) space
};

namespace jxb {

// geometry.cu
int build_tables(jxb_plan* plan, const jxb_desc* desc, cudaStream_t s);
int build_factors(jxb_plan* plan, const jxb_desc* desc, cudaStream_t s);
int qp_coords(jxb_plan* plan, cudaStream_t s, double* x);
int interpolate(jxb_plan* plan, cudaStream_t s, const double* coef, int ncomp, double* out);
int interpolate_grad(jxb_plan* plan, cudaStream_t s, const double* coef, int ncomp, double* out);
int hyper_state(jxb_plan* plan, cudaStream_t s, const double* u, double* energy);
int eval_points(jxb_plan* plan, cudaStream_t s, const double* coef, int ncomp, long long n, const long long* elems,
                const double* ref, double* val, double* grad, double* x, double* jac);
int boundary_points(jxb_plan* plan, cudaStream_t s, long long n_faces, int n_q, const long long* elems,
                    const int* sides, const double* ref, const double* wref, double* x, double* normal, double* w);
int boundary_load(jxb_plan* plan, cudaStream_t s, long long n_faces, int n_q, const long long* elems,
                  const double* ref, const double* w, const double* t, long long n_touched, const long long* dof,
                  const long long* ptr, const long long* contrib, double* local, double* F);
int qp_weights(jxb_plan* plan, cudaStream_t s, double* w);

// apply.cu
enum Mode { MODE_APPLY = 0, MODE_LOAD = 1, MODE_DIAG = 2, MODE_RESID = 3 };
template <typename T>
int launch_bricks(jxb_plan* plan, cudaStream_t s, int mode, const T* x, const double* f_qp,
                  const CgState* state, int masked);
template <typename T>
int launch_combine(jxb_plan* plan, cudaStream_t s, T* y, int masked, const T* dot_with,
                   double* partials, const CgState* state);

int tile2_variant(int tx, int ty);
template <typename T>
BrickArgs<T> make_brick_args(jxb_plan* plan, const T* x, const CgState* state, int masked);
// mp.cu: the composite plan's hooks in launch_bricks / launch_combine
int mp_bricks(jxb_plan* plan, cudaStream_t s, int mode, const double* x, const double* f_qp, const CgState* state);
int mp_combine(jxb_plan* plan, cudaStream_t s, double* y, int masked, const double* dot_with, double* partials,
               const CgState* state);
void free_mp(jxb_plan* plan);
// thb.cu: the hierarchical plan's hooks in launch_bricks / launch_combine
int thb_bricks(jxb_plan* plan, cudaStream_t s, int mode, const double* x, const double* f_qp, const CgState* state,
               int masked);
int thb_combine(jxb_plan* plan, cudaStream_t s, double* y, int masked, const double* dot_with, double* partials,
                const CgState* state);
void free_thb(jxb_plan* plan);

size_t smem2_scalar_apply(int p, bool rational, int tx, int fp0, int fp1);
int persist2_grid(bool rational, size_t smem, int* grid);
int launch_bricks2_persist(bool rational, const BrickArgs<double>* d_args, const int4* d_work, int n_work,
                           unsigned* d_next, int grid, size_t smem, const CgState* d_states, cudaStream_t s);
int launch_bricks2_batch(int p, bool rational, int variant, const BrickArgs<double>* d_args, const int2* d_work,
                         long long n_work, int fp0, int fp1, const CgState* d_states, cudaStream_t s);

// pcg.cu
int ensure_workspace(jxb_plan* plan, bool f32);
int compute_invdiag(jxb_plan* plan, cudaStream_t s);
int dot(jxb_plan* plan, cudaStream_t s, const double* a, const double* b, double* out_host);
// ||b - K x|| over free DOFs (FP64, masked); the residual goes to res_out when
// not null; blocks until the norms are on the host
int true_residual(jxb_plan* plan, cudaStream_t s, const double* b, const double* x, double* res_out, double* rnorm,
                  double* bnorm, bool* finite);
// Writes the stats of a finished solve and returns its status:
// JXB_ERR_NONFINITE (nonfinite), JXB_ERR_NOT_CONVERGED (true residual above
// max(tol ||b||, atol)) or JXB_OK.
int finish_solve(const char* who, jxb_stats* stats, long long iters, long long outer, double rn, double bn, bool fin,
                 double tol, double atol, float ms, bool nonfinite);

// krylov.cu
void free_krylov(jxb_plan* plan);

// cnn.cu (the network of the learned preconditioner)
// infer: an inference forward, which takes the BF16 tensor-core convolutions
// when the network is set to (jxb_cnn_set_inference_bf16); training forwards
// pass false
int cnn_forward(jxb_cnn* N, cudaStream_t s, int nx, int ny, int nz, const float* in, const float** out4,
                bool infer = false);
float* cnn_grad_out(jxb_cnn* N);  // the 4-channel output-gradient buffer read by cnn_backward
int cnn_backward(jxb_cnn* N, cudaStream_t s, int nx, int ny, int nz, const float* in);
int cnn_out_channels(const jxb_cnn* N);

}  // namespace jxb
