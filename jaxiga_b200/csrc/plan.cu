// Plan lifetime and the C-ABI entry points of libjxb.
//
// A plan corresponds to what src/jaxiga/methods/_common.py:163-178
// (build_context) prepares for one linear Galerkin problem on a single
// tensor-product patch: the evaluated basis at the interior Gauss points
// (evaluation.py:305-467), the DOF partition (function_space.py:554-603) and
// the operator constants (library.py / materials.py). Instead of BasisData
// arrays it keeps per-direction extracted 1D tables and per-point factors,
// laid out brick by brick for the sum-factorised kernels.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "jxb_internal.cuh"

namespace jxb {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return JXB_ERR_CUDA;
}

int host_geo_count(int op, int rational, int dim);
void host_brick_shape(int dim, int p, int* te);

__global__ void k_to_f32(long long n, const double* a, float* b) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

template <typename T>
static int upload(T** d, const T* h, size_t n, cudaStream_t s) {
  JXB_CUDA(cudaMalloc(d, std::max<size_t>(n, 1) * sizeof(T)));
  if (n) JXB_CUDA(cudaMemcpyAsync(*d, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
  return JXB_OK;
}

static void free_plan(jxb_plan* p) {
  if (!p) return;
  free_mp(p);
  free_thb(p);
  free_krylov(p);
  for (int d = 0; d < 3; ++d) {
    cudaFree(p->d_first[d]);
    cudaFree(p->d_bcp0[d]);
    cudaFree(p->d_cover[d]);
    cudaFree(p->d_tab[d]);
    cudaFree(p->d_ext[d]);
    cudaFree(p->d_lo[d]);
    cudaFree(p->d_hi[d]);
    cudaFree(p->d_tab32[d]);
  }
  void* bufs[] = {p->d_geo, p->d_geo32, p->d_wq, p->d_invW, p->d_cpts, p->d_wgts, p->d_wgts32,
                  p->d_keep, p->d_scratch, p->d_scratch32, p->d_red, p->d_x, p->d_b, p->d_r,
                  p->d_z, p->d_p, p->d_Ap, p->d_invdiag, p->d_x32, p->d_r32, p->d_z32, p->d_p32,
                  p->d_Ap32, p->d_invdiag32, p->d_xacc, p->d_res, p->d_state};
  for (void* b : bufs) cudaFree(b);
  if (p->h_state) cudaFreeHost(p->h_state);
  for (int i = 0; i < 2; ++i) {
    if (p->graph[i]) cudaGraphExecDestroy(p->graph[i]);
    if (p->graph_stream[i]) cudaStreamDestroy(p->graph_stream[i]);
  }
  delete p;
}

static int validate(const jxb_desc* d) {
  if (!d) return fail(JXB_ERR_INVALID, "desc is NULL");
  if (d->dim != 2 && d->dim != 3) return fail(JXB_ERR_INVALID, "dim must be 2 or 3");
  if (d->degree < 1 || d->degree > JXB_MAXP) return fail(JXB_ERR_INVALID, "degree must be in 1..5");
  if (d->n_quad != d->degree + 1)
    return fail(JXB_ERR_INVALID, "n_quad must equal degree + 1 (the reference's default Gauss rule)");
  if (d->op == JXB_OP_POISSON) {
    if (d->vec != 1) return fail(JXB_ERR_INVALID, "Poisson needs vec == 1");
  } else if (d->op == JXB_OP_ELASTICITY) {
    if (d->vec != d->dim) return fail(JXB_ERR_INVALID, "elasticity needs vec == dim");
  } else if (d->op == JXB_OP_PLATE) {
    if (d->dim != 2 || d->vec != 1) return fail(JXB_ERR_INVALID, "plate needs dim == 2 and vec == 1");
    if (d->degree < 2) return fail(JXB_ERR_INVALID, "plate needs degree >= 2 (C1 continuity)");
  } else if (d->op == JXB_OP_HYPERELASTIC) {
    if (d->vec != d->dim) return fail(JXB_ERR_INVALID, "the hyperelastic operator needs vec == dim");
    if (d->degree > 4) return fail(JXB_ERR_INVALID, "the hyperelastic operator takes degrees 1..4");
    if (d->want_f32) return fail(JXB_ERR_INVALID, "the hyperelastic operator has no FP32 copy");
    if (!(d->coef[0] > 0) || !(d->coef[1] >= 0)) return fail(JXB_ERR_INVALID, "hyperelastic coef = {mu > 0, lambda >= 0}");
  } else {
    return fail(JXB_ERR_INVALID, "unknown operator");
  }
  for (int k = 0; k < d->dim; ++k) {
    if (d->n_span[k] < 1 || d->n_cp[k] < d->degree + 1)
      return fail(JXB_ERR_INVALID, "n_span / n_cp inconsistent with the degree");
    if (!d->first[k] || !d->extraction[k] || !d->span_lo[k] || !d->span_hi[k])
      return fail(JXB_ERR_INVALID, "per-direction arrays must be given");
    for (int e = 0; e < d->n_span[k]; ++e) {
      int f = d->first[k][e];
      if (f < 0 || f + d->degree >= d->n_cp[k]) return fail(JXB_ERR_INVALID, "first index out of range");
      if (e > 0 && f <= d->first[k][e - 1]) return fail(JXB_ERR_INVALID, "first indices must increase");
      if (!(d->span_hi[k][e] > d->span_lo[k][e])) return fail(JXB_ERR_INVALID, "empty span");
    }
  }
  if (!d->cpts || !d->wgts || !d->gauss_nodes || !d->gauss_weights)
    return fail(JXB_ERR_INVALID, "cpts, wgts and the Gauss rule must be given");
  return JXB_OK;
}

}  // namespace jxb

using namespace jxb;

extern "C" const char* jxb_last_error(void) { return g_last_error.c_str(); }
extern "C" int jxb_version(void) { return 1; }

extern "C" int jxb_plan_create(const jxb_desc* desc, jxb_plan** out) {
  if (!out) return fail(JXB_ERR_INVALID, "out is NULL");
  *out = nullptr;
  int rc = validate(desc);
  if (rc) return rc;
  int device = 0;
  JXB_CUDA(cudaGetDevice(&device));
  jxb_plan* P = new jxb_plan();
  P->device = device;
  P->dim = desc->dim;
  P->vec = desc->vec;
  P->p = desc->degree;
  P->q = desc->n_quad;
  P->op = desc->op;
  P->order = desc->op == JXB_OP_PLATE ? 2 : 1;
  P->plane_strain = desc->plane_strain;
  for (int i = 0; i < 4; ++i) P->coef[i] = desc->coef[i];
  P->n_elem = 1;
  P->n_scalar = 1;
  for (int d = 0; d < 3; ++d) {
    P->n_span[d] = d < P->dim ? desc->n_span[d] : 1;
    P->n_cp[d] = d < P->dim ? desc->n_cp[d] : 1;
    P->n_elem *= P->n_span[d];
    P->n_scalar *= P->n_cp[d];
  }
  P->n_dofs = P->n_scalar * P->vec;
  P->nqe = P->dim == 2 ? P->q * P->q : P->q * P->q * P->q;
  P->n_qp = P->n_elem * P->nqe;
  P->rational = 0;
  for (long long i = 0; i < P->n_scalar; ++i)
    if (desc->wgts[i] != 1.0) {
      P->rational = 1;
      break;
    }
  P->ngeo = host_geo_count(P->op, P->rational, P->dim);
  double E = desc->coef[0], nu = desc->coef[1];
  if (P->op == JXB_OP_ELASTICITY) {
    P->mat.mu = E / (2.0 * (1.0 + nu));
    if (P->dim == 3 || P->plane_strain)
      P->mat.lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    else
      P->mat.lam = E * nu / (1.0 - nu * nu);
  } else if (P->op == JXB_OP_HYPERELASTIC) {
    P->mat.mu = desc->coef[0];
    P->mat.lam = desc->coef[1];
  } else {
    P->mat.lam = P->mat.mu = 0.0;
  }

  // ---- brick decomposition (host) ----
  Bricks& br = P->br;
  br.dim = P->dim;
  br.vec = P->vec;
  br.p = P->p;
  br.q = P->q;
  host_brick_shape(P->dim, P->p, br.te);
  if (P->dim == 2 && (desc->tile[0] > 0 || desc->tile[1] > 0)) {
    const int v = tile2_variant(desc->tile[0], desc->tile[1]);
    if (v < 0 || (v != 0 && P->op != JXB_OP_POISSON)) {
      delete P;
      return fail(JXB_ERR_INVALID,
                  "tile: unsupported 2D brick shape (rows of 32 elements, or 16 / 64 for the scalar operator; "
                  "1 to 64 rows per brick)");
    }
    br.te[0] = desc->tile[0];
    br.te[1] = desc->tile[1];
  } else if (P->dim == 3) {
    // the most element layers per brick (up to 8) that still give every SM of a
    // B200 two bricks: the coarse levels of a multigrid hierarchy and other small
    // patches otherwise leave most SMs idle
    const long long nbxy = (long long)((P->n_span[0] + br.te[0] - 1) / br.te[0]) *
                           ((P->n_span[1] + br.te[1] - 1) / br.te[1]);
    while (br.te[2] > 1 && nbxy * ((P->n_span[2] + br.te[2] - 1) / br.te[2]) < 2 * 148) br.te[2] /= 2;
  } else if (P->dim == 2) {
    // rows of 32 elements, and the most rows per brick (up to 8) that still
    // give every SM of a B200 one brick (shorter bricks cost more per element:
    // each loads its tables and writes a footprint of p more rows)
    const long long nbx = (P->n_span[0] + br.te[0] - 1) / br.te[0];
    while (br.te[1] > 1 && nbx * ((P->n_span[1] + br.te[1] - 1) / br.te[1]) < 148) br.te[1] /= 2;
  }
  std::vector<int> cover_h[3], bcp0_h[3];
  long long nb_total = 1;
  for (int d = 0; d < 3; ++d) {
    br.n_span[d] = P->n_span[d];
    br.n_cp[d] = P->n_cp[d];
    if (d >= P->dim) {
      br.nb[d] = 1;
      br.fp[d] = 1;
      br.te[d] = 1;
      bcp0_h[d] = {0};
      cover_h[d].assign(2 * JXB_MAXC, -1);
      cover_h[d][0] = 0;
      cover_h[d][1] = 0;
      continue;
    }
    int te = br.te[d];
    int nb = (P->n_span[d] + te - 1) / te;
    br.nb[d] = nb;
    nb_total *= nb;
    const int32_t* first = desc->first[d];
    std::vector<int> ext(nb);
    int fpmax = 0;
    bcp0_h[d].resize(nb);
    for (int k = 0; k < nb; ++k) {
      int e0 = k * te, e1 = std::min((k + 1) * te, P->n_span[d]) - 1;
      bcp0_h[d][k] = first[e0];
      ext[k] = first[e1] + P->p + 1 - first[e0];
      fpmax = std::max(fpmax, ext[k]);
    }
    br.fp[d] = fpmax;
    cover_h[d].assign((size_t)2 * JXB_MAXC * P->n_cp[d], -1);
    for (int k = 0; k < nb; ++k)
      for (int i = bcp0_h[d][k]; i < bcp0_h[d][k] + ext[k]; ++i) {
        int* c = &cover_h[d][(size_t)2 * JXB_MAXC * i];
        int j = 0;
        while (j < JXB_MAXC && c[2 * j] >= 0) ++j;
        if (j == JXB_MAXC) {
          free_plan(P);
          return fail(JXB_ERR_INVALID, "a control point is covered by too many bricks (knot multiplicities too high)");
        }
        c[2 * j] = k;
        c[2 * j + 1] = i - bcp0_h[d][k];
      }
  }
  br.n_bricks = nb_total;
  br.slots = nb_total * (long long)br.te[0] * br.te[1] * br.te[2];
  if (P->dim == 2) br.te[2] = 1;

  cudaStream_t s;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
    free_plan(P);
    return fail(JXB_ERR_CUDA, "cudaStreamCreate failed");
  }
  auto bail = [&](int code) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    free_plan(P);
    return code;
  };
  for (int d = 0; d < 3; ++d) {
    std::vector<int> first_h(P->n_span[d], 0);
    if (d < P->dim)
      for (int e = 0; e < P->n_span[d]; ++e) first_h[e] = desc->first[d][e];
    if ((rc = upload(&P->d_first[d], first_h.data(), first_h.size(), s))) return bail(rc);
    if ((rc = upload(&P->d_bcp0[d], bcp0_h[d].data(), bcp0_h[d].size(), s))) return bail(rc);
    if ((rc = upload(&P->d_cover[d], cover_h[d].data(), cover_h[d].size(), s))) return bail(rc);
    br.first[d] = P->d_first[d];
    br.bcp0[d] = P->d_bcp0[d];
    br.cover[d] = P->d_cover[d];
  }
  if ((rc = upload(&P->d_cpts, desc->cpts, (size_t)P->n_scalar * P->dim, s))) return bail(rc);
  if ((rc = upload(&P->d_wgts, desc->wgts, (size_t)P->n_scalar, s))) return bail(rc);
  {
    std::vector<uint8_t> keep(P->n_dofs, 1);
    long long nfree = P->n_dofs;
    if (desc->prescribed)
      for (long long i = 0; i < P->n_dofs; ++i)
        if (desc->prescribed[i]) {
          keep[i] = 0;
          --nfree;
        }
    P->n_free = nfree;
    if ((rc = upload(&P->d_keep, keep.data(), keep.size(), s))) return bail(rc);
    JXB_CUDA(cudaStreamSynchronize(s));
  }
  if ((rc = build_tables(P, desc, s))) return bail(rc);

  size_t geo_n = (size_t)br.slots * P->ngeo * P->nqe;
  if (cudaMalloc(&P->d_geo, geo_n * sizeof(double)) != cudaSuccess) return bail(fail(JXB_ERR_NOMEM, "geo allocation failed"));
  if (cudaMalloc(&P->d_wq, (size_t)br.slots * P->nqe * sizeof(double)) != cudaSuccess)
    return bail(fail(JXB_ERR_NOMEM, "weight allocation failed"));
  if (P->rational && cudaMalloc(&P->d_invW, (size_t)br.slots * P->nqe * sizeof(double)) != cudaSuccess)
    return bail(fail(JXB_ERR_NOMEM, "weight allocation failed"));
  if ((rc = build_factors(P, desc, s))) return bail(rc);

  P->scratch_elems = (size_t)br.n_bricks * P->vec * br.fp[0] * br.fp[1] * br.fp[2];
  if (cudaMalloc(&P->d_scratch, P->scratch_elems * sizeof(double)) != cudaSuccess)
    return bail(fail(JXB_ERR_NOMEM, "scratch allocation failed"));
  if (cudaMalloc(&P->d_red, (4 * JXB_RED_BLOCKS + 16) * sizeof(double)) != cudaSuccess)
    return bail(fail(JXB_ERR_NOMEM, "reduction buffer allocation failed"));
  JXB_CUDA(cudaMemsetAsync(P->d_red, 0, (4 * JXB_RED_BLOCKS + 16) * sizeof(double), s));
  if (desc->want_f32) {
    if (cudaMalloc(&P->d_geo32, geo_n * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&P->d_wgts32, P->n_scalar * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&P->d_scratch32, P->scratch_elems * sizeof(float)) != cudaSuccess)
      return bail(fail(JXB_ERR_NOMEM, "FP32 factor allocation failed"));
    k_to_f32<<<(unsigned)((geo_n + 255) / 256), 256, 0, s>>>((long long)geo_n, P->d_geo, P->d_geo32);
    k_to_f32<<<(unsigned)((P->n_scalar + 255) / 256), 256, 0, s>>>(P->n_scalar, P->d_wgts, P->d_wgts32);
  }
  cudaError_t e = cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  if (e != cudaSuccess) {
    free_plan(P);
    return cuda_fail(e, "plan setup");
  }
  *out = P;
  return JXB_OK;
}

extern "C" int jxb_plan_destroy(jxb_plan* plan) {
  if (!plan) return JXB_OK;
  cudaDeviceSynchronize();
  free_plan(plan);
  return JXB_OK;
}

extern "C" int jxb_plan_info(const jxb_plan* P, jxb_info* out) {
  if (!P || !out) return fail(JXB_ERR_INVALID, "jxb_plan_info: null argument");
  out->n_dofs = P->n_dofs;
  out->n_free = P->n_free;
  out->n_elem = P->n_elem;
  out->n_qp = P->n_qp;
  out->n_bricks = P->br.n_bricks;
  out->geo_bytes = (int64_t)P->br.slots * P->ngeo * P->nqe * (int64_t)sizeof(double);
  out->scratch_bytes = (int64_t)P->scratch_elems * (int64_t)sizeof(double);
  out->ngeo = P->ngeo;
  out->rational = P->rational;
  return JXB_OK;
}

extern "C" int jxb_apply(jxb_plan* P, jxb_stream stream, const double* x, double* y, int masked) {
  if (!P || !x || !y) return fail(JXB_ERR_INVALID, "jxb_apply: null argument");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int rc = launch_bricks<double>(P, s, MODE_APPLY, x, nullptr, nullptr, masked);
  if (rc) return rc;
  return launch_combine<double>(P, s, y, masked, nullptr, nullptr, nullptr);
}

extern "C" int jxb_apply_f32(jxb_plan* P, jxb_stream stream, const float* x, float* y) {
  if (P && (P->mp || P->thb)) return fail(JXB_ERR_INVALID, "jxb_apply_f32: not available on a multipatch or hierarchical plan");
  if (!P || !x || !y) return fail(JXB_ERR_INVALID, "jxb_apply_f32: null argument");
  if (!P->d_geo32) return fail(JXB_ERR_INVALID, "jxb_apply_f32: plan was created without want_f32");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int rc = launch_bricks<float>(P, s, MODE_APPLY, x, nullptr, nullptr, 1);
  if (rc) return rc;
  return launch_combine<float>(P, s, y, 1, nullptr, nullptr, nullptr);
}

extern "C" int jxb_diag(jxb_plan* P, jxb_stream stream, double* d) {
  if (!P || !d) return fail(JXB_ERR_INVALID, "jxb_diag: null argument");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int rc = launch_bricks<double>(P, s, MODE_DIAG, nullptr, nullptr, nullptr, 1);
  if (rc) return rc;
  return launch_combine<double>(P, s, d, 1, nullptr, nullptr, nullptr);
}

extern "C" int jxb_hyper_state(jxb_plan* P, jxb_stream stream, const double* u, double* energy) {
  if (P && (P->mp || P->thb)) return fail(JXB_ERR_INVALID, "jxb_hyper_state: not available on a multipatch or hierarchical plan");
  if (!P || !u) return fail(JXB_ERR_INVALID, "jxb_hyper_state: null argument");
  return hyper_state(P, reinterpret_cast<cudaStream_t>(stream), u, energy);
}

extern "C" int jxb_hyper_residual(jxb_plan* P, jxb_stream stream, double* r) {
  if (P && (P->mp || P->thb)) return fail(JXB_ERR_INVALID, "jxb_hyper_residual: not available on a multipatch or hierarchical plan");
  if (!P || !r) return fail(JXB_ERR_INVALID, "jxb_hyper_residual: null argument");
  if (P->op != JXB_OP_HYPERELASTIC) return fail(JXB_ERR_INVALID, "jxb_hyper_residual: not a hyperelastic plan");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int rc = launch_bricks<double>(P, s, MODE_RESID, nullptr, nullptr, nullptr, 0);
  if (rc) return rc;
  return launch_combine<double>(P, s, r, 0, nullptr, nullptr, nullptr);
}

extern "C" int jxb_load(jxb_plan* P, jxb_stream stream, const double* f_qp, double* F) {
  if (!P || !f_qp || !F) return fail(JXB_ERR_INVALID, "jxb_load: null argument");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int rc = launch_bricks<double>(P, s, MODE_LOAD, nullptr, f_qp, nullptr, 0);
  if (rc) return rc;
  return launch_combine<double>(P, s, F, 0, nullptr, nullptr, nullptr);
}

extern "C" int jxb_qp_coords(jxb_plan* P, jxb_stream stream, double* x) {
  if (P && (P->mp || P->thb)) return fail(JXB_ERR_INVALID, "jxb_qp_coords: not available on a multipatch or hierarchical plan");
  if (!P || !x) return fail(JXB_ERR_INVALID, "jxb_qp_coords: null argument");
  return qp_coords(P, reinterpret_cast<cudaStream_t>(stream), x);
}

extern "C" int jxb_interpolate(jxb_plan* P, jxb_stream stream, const double* coef, int ncomp, double* out) {
  if (P && (P->mp || P->thb)) return fail(JXB_ERR_INVALID, "jxb_interpolate: not available on a multipatch or hierarchical plan");
  if (!P || !coef || !out) return fail(JXB_ERR_INVALID, "jxb_interpolate: null argument");
  return interpolate(P, reinterpret_cast<cudaStream_t>(stream), coef, ncomp, out);
}

extern "C" int jxb_interpolate_grad(jxb_plan* P, jxb_stream stream, const double* coef, int ncomp, double* out) {
  if (P && (P->mp || P->thb)) return fail(JXB_ERR_INVALID, "jxb_interpolate_grad: not available on a multipatch or hierarchical plan");
  if (!P || !coef || !out) return fail(JXB_ERR_INVALID, "jxb_interpolate_grad: null argument");
  return interpolate_grad(P, reinterpret_cast<cudaStream_t>(stream), coef, ncomp, out);
}

extern "C" int jxb_eval_points(jxb_plan* P, jxb_stream stream, const double* coef, int ncomp, int64_t n,
                               const int64_t* elems, const double* ref, double* val, double* grad, double* x,
                               double* jac) {
  if (P && (P->mp || P->thb)) return fail(JXB_ERR_INVALID, "jxb_eval_points: not available on a multipatch or hierarchical plan");
  if (!P || (n > 0 && (!elems || !ref))) return fail(JXB_ERR_INVALID, "jxb_eval_points: null argument");
  if (!coef && (val || grad)) return fail(JXB_ERR_INVALID, "jxb_eval_points: values need a coefficient field");
  return eval_points(P, reinterpret_cast<cudaStream_t>(stream), coef, ncomp, n,
                     reinterpret_cast<const long long*>(elems), ref, val, grad, x, jac);
}

extern "C" int jxb_boundary_points(jxb_plan* P, jxb_stream stream, int64_t n_faces, int n_q, const int64_t* elems,
                                   const int32_t* sides, const double* ref, const double* wref, double* x,
                                   double* normal, double* w) {
  if (P && (P->mp || P->thb)) return fail(JXB_ERR_INVALID, "jxb_boundary_points: not available on a multipatch or hierarchical plan");
  if (!P || (n_faces > 0 && (!elems || !sides || !ref || (w && !wref))))
    return fail(JXB_ERR_INVALID, "jxb_boundary_points: null argument");
  return boundary_points(P, reinterpret_cast<cudaStream_t>(stream), n_faces, n_q,
                         reinterpret_cast<const long long*>(elems), sides, ref, wref, x, normal, w);
}

extern "C" int jxb_boundary_load(jxb_plan* P, jxb_stream stream, int64_t n_faces, int n_q, const int64_t* elems,
                                 const double* ref, const double* w, const double* traction, int64_t n_touched,
                                 const int64_t* dofs, const int64_t* ptr, const int64_t* contrib, double* local,
                                 double* F) {
  if (P && (P->mp || P->thb)) return fail(JXB_ERR_INVALID, "jxb_boundary_load: not available on a multipatch or hierarchical plan");
  if (!P || (n_faces > 0 && (!elems || !ref || !w || !traction || !local || !F)) ||
      (n_touched > 0 && (!dofs || !ptr || !contrib)))
    return fail(JXB_ERR_INVALID, "jxb_boundary_load: null argument");
  return boundary_load(P, reinterpret_cast<cudaStream_t>(stream), n_faces, n_q,
                       reinterpret_cast<const long long*>(elems), ref, w, traction, n_touched,
                       reinterpret_cast<const long long*>(dofs), reinterpret_cast<const long long*>(ptr),
                       reinterpret_cast<const long long*>(contrib), local, F);
}

extern "C" int jxb_qp_weights(jxb_plan* P, jxb_stream stream, double* w) {
  if (P && (P->mp || P->thb)) return fail(JXB_ERR_INVALID, "jxb_qp_weights: not available on a multipatch or hierarchical plan");
  if (!P || !w) return fail(JXB_ERR_INVALID, "jxb_qp_weights: null argument");
  return qp_weights(P, reinterpret_cast<cudaStream_t>(stream), w);
}

extern "C" int jxb_profile_apply(jxb_plan* P, jxb_stream stream, const void* x, void* y, int reps, int f32,
                                 double* ms_out) {
  if (P && (P->mp || P->thb)) return fail(JXB_ERR_INVALID, "jxb_profile_apply: not available on a multipatch or hierarchical plan");
  if (!P || !x || !y || !ms_out || reps < 1) return fail(JXB_ERR_INVALID, "jxb_profile_apply: bad argument");
  if (f32 && !P->d_geo32) return fail(JXB_ERR_INVALID, "jxb_profile_apply: plan was created without want_f32");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  std::vector<cudaEvent_t> ev(3 * reps);
  for (auto& e : ev) JXB_CUDA(cudaEventCreate(&e));
  int rc = 0;
  for (int r = 0; r < reps && !rc; ++r) {
    JXB_CUDA(cudaEventRecord(ev[3 * r], s));
    if (f32)
      rc = launch_bricks<float>(P, s, MODE_APPLY, (const float*)x, nullptr, nullptr, 1);
    else
      rc = launch_bricks<double>(P, s, MODE_APPLY, (const double*)x, nullptr, nullptr, 1);
    if (rc) break;
    JXB_CUDA(cudaEventRecord(ev[3 * r + 1], s));
    if (f32)
      rc = launch_combine<float>(P, s, (float*)y, 1, nullptr, nullptr, nullptr);
    else
      rc = launch_combine<double>(P, s, (double*)y, 1, nullptr, nullptr, nullptr);
    JXB_CUDA(cudaEventRecord(ev[3 * r + 2], s));
  }
  if (rc) return rc;
  JXB_CUDA(cudaEventSynchronize(ev[3 * reps - 1]));
  double tb = 0, tc = 0;
  for (int r = 0; r < reps; ++r) {
    float a = 0, b = 0;
    JXB_CUDA(cudaEventElapsedTime(&a, ev[3 * r], ev[3 * r + 1]));
    JXB_CUDA(cudaEventElapsedTime(&b, ev[3 * r + 1], ev[3 * r + 2]));
    tb += a;
    tc += b;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  ms_out[0] = tb / reps;
  ms_out[1] = tc / reps;
  return JXB_OK;
}
