// Composite plans over several conforming patches (multipatch spaces).
//
// The reference numbers the control points of glued patches globally
// (src/jaxiga/geometry/multipatch.py:441-580) and assembles every element into
// the global matrix (src/jaxiga/methods/galerkin.py:122-148). Here each patch
// keeps its own libjxb plan and the composite plan's K.u is
//   y = mask( sum_p S_p^T K_p S_p x ),
// S_p the gather of patch p's DOFs from the global vector. The gather is one
// kernel over the concatenated patch-local vectors; the sum is one kernel that
// walks, for every global DOF, its patch-local copies in a fixed order (a CSR
// list built on the host), so the result is deterministic and carries the
// CG's p.Ap partials like the single-patch combine. The composite hooks into
// launch_bricks / launch_combine, so jxb_apply, jxb_diag, jxb_load and the CG
// (with its graphs, restarts and diagnostics) run on it unchanged.
#include <algorithm>
#include <vector>

#include "jxb_internal.cuh"

struct jxb_mp_data {
  std::vector<jxb_plan*> subs;  // the patch plans (owned by the caller)
  std::vector<long long> loff;  // offsets of each patch's DOFs in the local concatenation
  std::vector<long long> qoff;  // offsets of each patch's Gauss points (reference element order)
  long long n_local = 0;
  long long* d_gmap = nullptr;  // (n_local) global DOF of each local DOF
  long long* d_sptr = nullptr;  // (n_dofs + 1)
  long long* d_sidx = nullptr;  // (n_local) local DOFs grouped by global DOF
  double* d_xl = nullptr;
  double* d_yl = nullptr;
};

namespace jxb {
namespace {

__global__ void k_mp_gather(const CgState* st, long long n_local, const long long* __restrict__ gmap,
                            const double* __restrict__ x, double* __restrict__ xl) {
  if (st && st->done) return;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n_local;
       k += (long long)gridDim.x * blockDim.x)
    xl[k] = x[gmap[k]];
}

__global__ void __launch_bounds__(JXB_RED_THREADS)
    k_mp_scatter(const CgState* st, long long n, const long long* __restrict__ sptr, const long long* __restrict__ sidx,
                 const double* __restrict__ yl, const uint8_t* __restrict__ keep, int masked, double* __restrict__ y,
                 const double* __restrict__ dot_with, double* __restrict__ partials) {
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

int mp_bricks(jxb_plan* plan, cudaStream_t s, int mode, const double* x, const double* f_qp, const CgState* state) {
  jxb_mp_data* M = plan->mp;
  if (mode == MODE_APPLY) {
    const unsigned nb = (unsigned)std::min<long long>((M->n_local + 255) / 256, 4096);
    k_mp_gather<<<nb, 256, 0, s>>>(state, M->n_local, M->d_gmap, x, M->d_xl);
    JXB_CUDA(cudaGetLastError());
  } else if (mode != MODE_DIAG && mode != MODE_LOAD) {
    return fail(JXB_ERR_INVALID, "multipatch plans apply, load and give the diagonal only");
  }
  for (size_t i = 0; i < M->subs.size(); ++i) {
    jxb_plan* P = M->subs[i];
    const double* xi = mode == MODE_APPLY ? M->d_xl + M->loff[i] : nullptr;
    const double* fi = mode == MODE_LOAD ? f_qp + M->qoff[i] * plan->vec : nullptr;
    int rc = launch_bricks<double>(P, s, mode, xi, fi, state, 0);
    if (rc) return rc;
    rc = launch_combine<double>(P, s, M->d_yl + M->loff[i], 0, nullptr, nullptr, state);
    if (rc) return rc;
  }
  return JXB_OK;
}

int mp_combine(jxb_plan* plan, cudaStream_t s, double* y, int masked, const double* dot_with, double* partials,
               const CgState* state) {
  jxb_mp_data* M = plan->mp;
  k_mp_scatter<<<JXB_RED_BLOCKS, JXB_RED_THREADS, 0, s>>>(state, plan->n_dofs, M->d_sptr, M->d_sidx, M->d_yl,
                                                          plan->d_keep, masked, y, dot_with, partials);
  JXB_CUDA(cudaGetLastError());
  return JXB_OK;
}

void free_mp(jxb_plan* plan) {
  jxb_mp_data* M = plan ? plan->mp : nullptr;
  if (!M) return;
  void* bufs[] = {M->d_gmap, M->d_sptr, M->d_sidx, M->d_xl, M->d_yl};
  for (void* b : bufs) cudaFree(b);
  delete M;
  plan->mp = nullptr;
}

}  // namespace jxb

using namespace jxb;

extern "C" int jxb_mp_create(jxb_plan* const* patches, int n, const int64_t* const* local_to_global,
                             int64_t n_global_scalar, const uint8_t* prescribed, jxb_plan** out) {
  if (!patches || n < 1 || !local_to_global || !out || n_global_scalar < 1)
    return fail(JXB_ERR_INVALID, "jxb_mp_create: bad argument");
  *out = nullptr;
  const jxb_plan* P0 = patches[0];
  for (int i = 0; i < n; ++i) {
    const jxb_plan* P = patches[i];
    if (!P || !local_to_global[i]) return fail(JXB_ERR_INVALID, "jxb_mp_create: null patch plan or map");
    if (P->mp || P->thb) return fail(JXB_ERR_INVALID, "jxb_mp_create: a patch plan is itself composite or hierarchical");
    if (P->dim != P0->dim || P->vec != P0->vec || P->op != P0->op || P->p != P0->p)
      return fail(JXB_ERR_INVALID, "jxb_mp_create: patches differ in dimension, components, operator or degree");
    if (P->op == JXB_OP_HYPERELASTIC) return fail(JXB_ERR_INVALID, "jxb_mp_create: hyperelastic patches are not supported");
    for (long long j = 0; j < P->n_scalar; ++j)
      if (local_to_global[i][j] < 0 || local_to_global[i][j] >= n_global_scalar)
        return fail(JXB_ERR_INVALID, "jxb_mp_create: local_to_global entry out of range");
  }
  int device = 0;
  JXB_CUDA(cudaGetDevice(&device));
  jxb_plan* C = new jxb_plan();
  C->mp = new jxb_mp_data();
  jxb_mp_data* M = C->mp;
  C->device = device;
  C->dim = P0->dim;
  C->vec = P0->vec;
  C->p = P0->p;
  C->q = P0->q;
  C->op = P0->op;
  C->order = P0->order;
  C->plane_strain = P0->plane_strain;
  C->mat = P0->mat;
  for (int i = 0; i < 4; ++i) C->coef[i] = P0->coef[i];
  C->nqe = P0->nqe;
  C->ngeo = P0->ngeo;
  C->n_scalar = n_global_scalar;
  C->n_dofs = n_global_scalar * C->vec;
  const int vec = C->vec;
  M->loff.assign(1, 0);
  M->qoff.assign(1, 0);
  for (int i = 0; i < n; ++i) {
    M->subs.push_back(patches[i]);
    M->loff.push_back(M->loff.back() + patches[i]->n_dofs);
    M->qoff.push_back(M->qoff.back() + patches[i]->n_qp);
    C->rational |= patches[i]->rational;
    C->n_elem += patches[i]->n_elem;
  }
  C->n_qp = M->qoff.back();
  M->n_local = M->loff.back();
  // maps: local DOF (patch i, scalar j, component c) -> global DOF, and the
  // reverse lists in ascending local order (the fixed summation order)
  std::vector<long long> gmap(M->n_local), count(C->n_dofs + 1, 0);
  for (int i = 0; i < n; ++i)
    for (long long j = 0; j < patches[i]->n_scalar; ++j)
      for (int c = 0; c < vec; ++c) {
        const long long k = M->loff[i] + j * vec + c;
        gmap[k] = local_to_global[i][j] * vec + c;
        ++count[gmap[k] + 1];
      }
  for (long long g = 0; g < C->n_dofs; ++g) count[g + 1] += count[g];
  std::vector<long long> sidx(M->n_local), fill(count.begin(), count.end() - 1);
  for (long long k = 0; k < M->n_local; ++k) sidx[fill[gmap[k]]++] = k;
  std::vector<uint8_t> keep(C->n_dofs, 1);
  long long nfree = C->n_dofs;
  if (prescribed)
    for (long long g = 0; g < C->n_dofs; ++g)
      if (prescribed[g]) {
        keep[g] = 0;
        --nfree;
      }
  C->n_free = nfree;
  auto bail = [&](int rc) {
    free_mp(C);
    cudaFree(C->d_keep);
    cudaFree(C->d_red);
    delete C;
    return rc;
  };
  cudaError_t e = cudaSuccess;
  auto al = [&](void** p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, std::max<size_t>(bytes, 8));
  };
  al((void**)&M->d_gmap, M->n_local * sizeof(long long));
  al((void**)&M->d_sidx, M->n_local * sizeof(long long));
  al((void**)&M->d_sptr, (C->n_dofs + 1) * sizeof(long long));
  al((void**)&M->d_xl, M->n_local * sizeof(double));
  al((void**)&M->d_yl, M->n_local * sizeof(double));
  al((void**)&C->d_keep, C->n_dofs);
  al((void**)&C->d_red, (4 * JXB_RED_BLOCKS + 16) * sizeof(double));
  if (e != cudaSuccess) return bail(cuda_fail(e, "jxb_mp_create: cudaMalloc"));
  e = cudaMemcpy(M->d_gmap, gmap.data(), M->n_local * sizeof(long long), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(M->d_sidx, sidx.data(), M->n_local * sizeof(long long), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(M->d_sptr, count.data(), (C->n_dofs + 1) * sizeof(long long), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(C->d_keep, keep.data(), C->n_dofs, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(C->d_red, 0, (4 * JXB_RED_BLOCKS + 16) * sizeof(double));
  if (e != cudaSuccess) return bail(cuda_fail(e, "jxb_mp_create: upload"));
  *out = C;
  return JXB_OK;
}
