// Discrete adjoint of the 2D DGSEM right-hand side and of SSPRK3 with
// two-level checkpointing (dgsem_adjoint_* in include/dgsem_b200.h).
//
// Forward: SSPRK3 steps with the fused stage kernels; the state is saved at
// the start of every checkpoint segment (every `every` steps).  Reverse:
// for each segment, last to first, the segment's steps are recomputed from
// its checkpoint while their stage states (u^n, u^(1), u^(2)) are kept in
// HBM (the last segment is recorded during the forward pass and not
// recomputed), with Navier-Stokes also the BR1 gradient of each of those
// states as the forward stage computed it (so the reverse VJPs do not
// recompute it), then the adjoint SSPRK3 steps run backwards:
//   lam2 = 2/3 lam + 2/3 dt VJP(u^(2); lam)
//   lam1 = 1/4 lam2 + 1/4 dt VJP(u^(1); lam2)
//   lam  = 1/3 lam + 3/4 lam2 + lam1 + dt VJP(u^n; lam1)
// which is the transpose of SSPRK3::step (time_integrator/SSPRK3.hpp:159-181).
// The objective is the volume-weighted mean kinetic energy
// (analyzer/volume_average_euler.hpp:9-69 with the weights w/|1/J| of
// volume_weighted_analyzer_functor.hpp:80,104).
#include <cuda_runtime.h>

#include <cmath>
#include <memory>
#include <new>
#include <vector>

#include "../../include/dgsem_b200.h"
#include "adjoint_kernel.cuh"
#include "context.hpp"

namespace dgsem {

class AdjointEngineBase {
 public:
  virtual ~AdjointEngineBase() = default;
  // out = x0 X + x1 Y + b w + c (dR/du(u))^T w.  Navier-Stokes: `grad_u` is
  // the forward BR1 gradient of u when the caller kept it from the forward
  // stage; nullptr recomputes it into cfg.grad first.
  virtual cudaError_t vjp(const EngineConfig& cfg, const double* u, const double* grad_u,
                          const double* w, double* out, const double* X, double x0,
                          const double* Y, double x1, double b, double c, double* xy,
                          double* qdir, cudaStream_t s) const = 0;
  virtual int kernels_per_vjp(bool with_gradient) const = 0;
};

template <int N, bool NS>
class AdjointEngine final : public AdjointEngineBase {
 public:
  static constexpr int EPB = (128 / (N * N)) > 0 ? (128 / (N * N)) : 1;

  cudaError_t vjp(const EngineConfig& cfg, const double* u, const double* grad_u,
                  const double* w, double* out, const double* X, double x0, const double* Y,
                  double x1, double b, double c, double* xy, double* qdir,
                  cudaStream_t s) const override {
    AdjArgs<N> a{};
    a.u = u;
    a.w = w;
    a.grad = grad_u ? grad_u : cfg.grad;
    a.xy = xy;
    a.qdir = qdir;
    a.out = out;
    a.X = X;
    a.Y = Y;
    a.x0 = x0;
    a.x1 = x1;
    a.b = b;
    a.c = c;
    a.cells[0] = (int)cfg.cells[0];
    a.cells[1] = (int)cfg.cells[1];
    a.nelem = (int)cfg.nelem;
    a.gamma = cfg.gamma;
    a.inv_gm1 = 1.0 / (cfg.gamma - 1.0);
    a.mu = cfg.mu;
    a.kappa = cfg.gamma / ((cfg.gamma - 1.0) * cfg.prandtl);
    a.tab = cfg.tab;
    fill_basis_const<N>(cfg.basis, &a.basis);
    const unsigned blocks = (unsigned)((cfg.nelem + EPB - 1) / EPB);
    if constexpr (NS) {
      GradArgs<N> ga{};
      ga.u = u;
      ga.grad = cfg.grad;
      for (int i = 0; i < 3; ++i) ga.cells[i] = cfg.cells[i];
      ga.nelem = cfg.nelem;
      ga.gamma = cfg.gamma;
      ga.tab = cfg.tab;
      ga.basis = a.basis;
      ga.periodic[0] = ga.periodic[1] = 1;  // the adjoint covers periodic meshes
      for (int f = 0; f < 4; ++f) ga.bc_kind[f] = 0;
      // programmatic dependent launches: each kernel's blocks are placed while
      // the previous one drains; griddepcontrol.wait orders the memory
      if (!grad_u) launch_stage_kernel(br1_gradient_kernel<N, EPB>, blocks, EPB * N * N, 0, s, ga);
      launch_stage_kernel(adj_viscous_kernel<N, EPB>, blocks, EPB * N * N, 0, s, a);
    }
    launch_stage_kernel(adj_main_kernel<N, NS, EPB>, blocks, EPB * N * N, 0, s, a);
    return cudaGetLastError();
  }
  int kernels_per_vjp(bool with_gradient) const override {
    return NS ? (with_gradient ? 3 : 2) : 1;
  }
};

std::unique_ptr<AdjointEngineBase> make_adjoint_engine(int n, bool ns) {
#define DGSEM_ADJ_CASE(NN)                                      \
  case NN:                                                      \
    if (ns) return std::make_unique<AdjointEngine<NN, true>>(); \
    return std::make_unique<AdjointEngine<NN, false>>();
  switch (n) {
    DGSEM_ADJ_CASE(2)
    DGSEM_ADJ_CASE(3)
    DGSEM_ADJ_CASE(4)
    DGSEM_ADJ_CASE(5)
    DGSEM_ADJ_CASE(6)
    DGSEM_ADJ_CASE(7)
    DGSEM_ADJ_CASE(8)
    default:
      return nullptr;
  }
#undef DGSEM_ADJ_CASE
}

namespace {

constexpr int kKeThreads = 256;

struct KeArgs {
  const double* u;
  int n, nx, nelem, nvars, ndims;
  double w[8];
  DeviceTables tab;
};

// Volume weight of a node, w_i w_j / |1/J| (volume_weighted_analyzer_functor.hpp:80).
__device__ __forceinline__ double ke_weight(const KeArgs& a, int e, int node) {
  const int i = node % a.n, j = node / a.n;
  const int ie = e % a.nx, je = e / a.nx;
  const double inv_j =
      1.0 / (__ldg(a.tab.jdiag[0] + ie * a.n + i) * __ldg(a.tab.jdiag[1] + je * a.n + j));
  return a.w[i] * a.w[j] / fabs(inv_j);
}

__device__ __forceinline__ double ke_node(const KeArgs& a, int e, int node) {
  const int nd = a.n * a.n;
  const double rho = __ldg(a.u + ((int64_t)e * a.nvars + 0) * nd + node);
  double m2 = 0.0;
  for (int d = 0; d < 2; ++d) {
    const double m = __ldg(a.u + ((int64_t)e * a.nvars + 1 + d) * nd + node);
    m2 += m * m;
  }
  return 0.5 * m2 / rho;
}

// Per-block partial sums of (w ke, w): fixed-order tree reduction.
__global__ void __launch_bounds__(kKeThreads) ke_partial_kernel(const KeArgs a, double* partial) {
  __shared__ double s0[kKeThreads], s1[kKeThreads];
  const int nd = a.n * a.n;
  const int64_t idx = (int64_t)blockIdx.x * kKeThreads + threadIdx.x;
  double num = 0.0, den = 0.0;
  if (idx < (int64_t)a.nelem * nd) {
    const int e = (int)(idx / nd), node = (int)(idx % nd);
    const double wt = ke_weight(a, e, node);
    num = wt * ke_node(a, e, node);
    den = wt;
  }
  s0[threadIdx.x] = num;
  s1[threadIdx.x] = den;
  __syncthreads();
  for (int st = kKeThreads / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st) {
      s0[threadIdx.x] += s0[threadIdx.x + st];
      s1[threadIdx.x] += s1[threadIdx.x + st];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = s0[0];
    partial[2 * blockIdx.x + 1] = s1[0];
  }
}

// One block: sums the partials in a fixed order; result[0] = J, result[1] = sum w.
__global__ void __launch_bounds__(kKeThreads) ke_final_kernel(const double* partial, int nblocks,
                                                              double* result) {
  __shared__ double s0[kKeThreads], s1[kKeThreads];
  double num = 0.0, den = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += kKeThreads) {
    num += partial[2 * b];
    den += partial[2 * b + 1];
  }
  s0[threadIdx.x] = num;
  s1[threadIdx.x] = den;
  __syncthreads();
  for (int st = kKeThreads / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st) {
      s0[threadIdx.x] += s0[threadIdx.x + st];
      s1[threadIdx.x] += s1[threadIdx.x + st];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    result[0] = s0[0] / s1[0];
    result[1] = s1[0];
  }
}

// dJ/du = w / sum(w) * d ke / du, ke = |m|^2 / (2 rho).
__global__ void __launch_bounds__(kKeThreads) ke_grad_kernel(const KeArgs a, const double* result,
                                                             double* grad) {
  const int nd = a.n * a.n;
  const int64_t idx = (int64_t)blockIdx.x * kKeThreads + threadIdx.x;
  if (idx >= (int64_t)a.nelem * nd) return;
  const int e = (int)(idx / nd), node = (int)(idx % nd);
  const double s = ke_weight(a, e, node) / result[1];
  const double rho = __ldg(a.u + ((int64_t)e * a.nvars + 0) * nd + node);
  double m2 = 0.0;
  for (int d = 0; d < 2; ++d) {
    const double m = __ldg(a.u + ((int64_t)e * a.nvars + 1 + d) * nd + node);
    m2 += m * m;
    grad[((int64_t)e * a.nvars + 1 + d) * nd + node] = s * m / rho;
  }
  grad[((int64_t)e * a.nvars + 0) * nd + node] = -s * 0.5 * m2 / (rho * rho);
  grad[((int64_t)e * a.nvars + 3) * nd + node] = 0.0;
}

}  // namespace
}  // namespace dgsem

using namespace dgsem;

struct dgsem_adjoint {
  dgsem_ctx* ctx = nullptr;
  std::unique_ptr<AdjointEngineBase> eng;
  int nsteps = 0;
  int every = 0;
  int nsnap = 0;
  int64_t len = 0;
  std::vector<void*> allocations;
  double* snaps = nullptr;  // [nsnap][len]
  double* seg = nullptr;    // [every][3][len]: u^n, u^(1), u^(2) of each step
  // Navier-Stokes: [every][3][glen] forward BR1 gradients of those states,
  // written by the forward stages that consume them (nullptr: Euler)
  double* gseg = nullptr;
  int64_t glen = 0;
  double* work = nullptr;   // forward state
  double* lam = nullptr;
  double* lam2 = nullptr;
  double* lam1 = nullptr;
  double* xy = nullptr;
  double* qdir = nullptr;
  double* partial = nullptr;
  double* result = nullptr;  // J, sum of weights
  int ke_blocks = 0;
  KeArgs ke{};
};

namespace {

dgsem_status st_of(cudaError_t e) { return e == cudaSuccess ? DGSEM_OK : DGSEM_ERR_CUDA; }

double* adj_alloc(dgsem_adjoint* a, size_t count, cudaError_t* err) {
  void* p = nullptr;
  *err = cudaMalloc(&p, count * sizeof(double));
  if (*err != cudaSuccess) return nullptr;
  a->allocations.push_back(p);
  return static_cast<double*>(p);
}

void adj_free(dgsem_adjoint* a) {
  for (void* p : a->allocations) cudaFree(p);
  a->allocations.clear();
}

// Forward stage through the context's engine (same kernels as dgsem_ssprk3_stage).
cudaError_t fwd_stage(dgsem_adjoint* a, int stage, const double* u_n, const double* u_in,
                      double* out, double t, double dt) {
  dgsem_ctx* ctx = a->ctx;
  double ca, cb, cc, ts;
  if (stage == 1) {
    ca = 0.0; cb = 1.0; cc = dt; ts = t;
  } else if (stage == 2) {
    ca = 3.0 / 4.0; cb = 1.0 / 4.0; cc = (1.0 / 4.0) * dt; ts = t + dt;
  } else {
    ca = 1.0 / 3.0; cb = 2.0 / 3.0; cc = (2.0 / 3.0) * dt; ts = t + 0.5 * dt;
  }
  ctx->launches += ctx->engine->kernels_per_stage();
  return ctx->engine->stage(ctx->cfg, u_n, u_in, out, ca, cb, cc, ts, nullptr, nullptr,
                            ctx->stream);
}

double* seg_slot(dgsem_adjoint* a, int r, int k) {
  return a->seg + ((int64_t)r * 3 + k) * a->len;
}

double* grad_slot(dgsem_adjoint* a, int r, int k) {
  return a->gseg ? a->gseg + ((int64_t)r * 3 + k) * a->glen : nullptr;
}

// Forward stage that keeps the BR1 gradient of its input state in `gslot`
// (the engine writes and reads the gradient through cfg.grad).
cudaError_t fwd_stage_keep(dgsem_adjoint* a, int stage, const double* u_n, const double* u_in,
                           double* out, double t, double dt, double* gslot) {
  if (!gslot) return fwd_stage(a, stage, u_n, u_in, out, t, dt);
  double* shared_grad = a->ctx->cfg.grad;
  a->ctx->cfg.grad = gslot;
  const cudaError_t e = fwd_stage(a, stage, u_n, u_in, out, t, dt);
  a->ctx->cfg.grad = shared_grad;
  return e;
}

// Steps [s0, s1) from the state in `state`, recording every step's stage
// states in the segment buffer (slot r = s - s0); the state after s1 is
// written back to `state`.
cudaError_t record_segment(dgsem_adjoint* a, double* state, int s0, int s1, double t0,
                           double dt) {
  cudaStream_t st = a->ctx->stream;
  cudaError_t e = cudaMemcpyAsync(seg_slot(a, 0, 0), state, a->len * sizeof(double),
                                  cudaMemcpyDeviceToDevice, st);
  for (int s = s0; s < s1 && e == cudaSuccess; ++s) {
    const int r = s - s0;
    const double t = t0 + s * dt;
    double* un = seg_slot(a, r, 0);
    double* next = (s + 1 < s1) ? seg_slot(a, r + 1, 0) : state;
    e = fwd_stage_keep(a, 1, nullptr, un, seg_slot(a, r, 1), t, dt, grad_slot(a, r, 0));
    if (e == cudaSuccess)
      e = fwd_stage_keep(a, 2, un, seg_slot(a, r, 1), seg_slot(a, r, 2), t, dt,
                         grad_slot(a, r, 1));
    if (e == cudaSuccess)
      e = fwd_stage_keep(a, 3, un, seg_slot(a, r, 2), next, t, dt, grad_slot(a, r, 2));
  }
  return e;
}

cudaError_t launch_vjp(dgsem_adjoint* a, const double* u, const double* grad_u,
                       const double* w, double* out, const double* X, double x0,
                       const double* Y, double x1, double b, double c) {
  a->ctx->launches += a->eng->kernels_per_vjp(grad_u == nullptr);
  return a->eng->vjp(a->ctx->cfg, u, grad_u, w, out, X, x0, Y, x1, b, c, a->xy, a->qdir,
                     a->ctx->stream);
}

cudaError_t objective(dgsem_adjoint* a, const double* u, double* grad) {
  cudaStream_t st = a->ctx->stream;
  KeArgs k = a->ke;
  k.u = u;
  ke_partial_kernel<<<a->ke_blocks, kKeThreads, 0, st>>>(k, a->partial);
  ke_final_kernel<<<1, kKeThreads, 0, st>>>(a->partial, a->ke_blocks, a->result);
  a->ctx->launches += 2;
  if (grad) {
    ke_grad_kernel<<<a->ke_blocks, kKeThreads, 0, st>>>(k, a->result, grad);
    a->ctx->launches += 1;
  }
  return cudaGetLastError();
}

}  // namespace

extern "C" {

dgsem_status dgsem_adjoint_create(dgsem_ctx* ctx, int nsteps, int checkpoint_every,
                                  dgsem_adjoint** out) {
  if (!out) return DGSEM_ERR_INVALID_ARG;
  *out = nullptr;
  if (!ctx || nsteps < 1 || checkpoint_every < 1) return DGSEM_ERR_INVALID_ARG;
  const dgsem_scheme_desc& s = ctx->scheme;
  if (ctx->mesh.ndims != 2 || s.volume_integral != DGSEM_VI_SPLIT_FORM ||
      s.volume_flux != DGSEM_VF_CHANDRASHEKAR || s.surface_flux != DGSEM_SF_LAX_FRIEDRICHS ||
      (s.equation != DGSEM_EULER_2D && s.equation != DGSEM_NAVIER_STOKES_2D))
    return DGSEM_ERR_UNSUPPORTED;
  for (int f = 0; f < 4; ++f)
    if (s.bc[f] != DGSEM_BC_PERIODIC) return DGSEM_ERR_UNSUPPORTED;
  const bool ns = s.equation == DGSEM_NAVIER_STOKES_2D;
  dgsem_adjoint* a = new (std::nothrow) dgsem_adjoint();
  if (!a) return DGSEM_ERR_ALLOC;
  a->ctx = ctx;
  a->eng = make_adjoint_engine(ctx->cfg.n, ns);
  if (!a->eng) {
    delete a;
    return DGSEM_ERR_UNSUPPORTED;
  }
  a->nsteps = nsteps;
  a->every = checkpoint_every < nsteps ? checkpoint_every : nsteps;
  a->nsnap = (nsteps + a->every - 1) / a->every;
  a->len = ctx->state_len;
  const int64_t nodes = ctx->cfg.nelem * ctx->nodes;
  a->ke_blocks = (int)((nodes + kKeThreads - 1) / kKeThreads);
  cudaError_t err = cudaSuccess;
  a->snaps = adj_alloc(a, (size_t)a->nsnap * a->len, &err);
  if (a->snaps) a->seg = adj_alloc(a, (size_t)a->every * 3 * a->len, &err);
  if (a->seg) a->work = adj_alloc(a, a->len, &err);
  if (a->work) a->lam = adj_alloc(a, a->len, &err);
  if (a->lam) a->lam2 = adj_alloc(a, a->len, &err);
  if (a->lam2) a->lam1 = adj_alloc(a, a->len, &err);
  a->glen = ns ? nodes * 8 : 0;
  if (a->lam1 && ns) a->gseg = adj_alloc(a, (size_t)a->every * 3 * a->glen, &err);
  if (a->lam1 && (!ns || a->gseg)) a->xy = adj_alloc(a, ns ? (size_t)nodes * 8 : 1, &err);
  if (a->xy) a->qdir = adj_alloc(a, ns ? (size_t)nodes * 2 : 1, &err);
  if (a->qdir) a->partial = adj_alloc(a, (size_t)a->ke_blocks * 2, &err);
  if (a->partial) a->result = adj_alloc(a, 2, &err);
  if (!a->result) {
    adj_free(a);
    delete a;
    return DGSEM_ERR_ALLOC;
  }
  KeArgs& k = a->ke;
  k.n = ctx->cfg.n;
  k.nx = (int)ctx->cfg.cells[0];
  k.nelem = (int)ctx->cfg.nelem;
  k.nvars = ctx->nvars;
  k.ndims = 2;
  for (int i = 0; i < 8; ++i) k.w[i] = i < k.n ? ctx->cfg.basis.weights[i] : 0.0;
  k.tab = ctx->cfg.tab;
  *out = a;
  return DGSEM_OK;
}

dgsem_status dgsem_adjoint_destroy(dgsem_adjoint* a) {
  if (!a) return DGSEM_ERR_INVALID_ARG;
  cudaStreamSynchronize(a->ctx->stream);
  adj_free(a);
  delete a;
  return DGSEM_OK;
}

dgsem_status dgsem_adjoint_rhs_vjp(dgsem_adjoint* a, const double* u, const double* w,
                                   double* out) {
  if (!a || !u || !w || !out || out == w) return DGSEM_ERR_INVALID_ARG;
  return st_of(launch_vjp(a, u, nullptr, w, out, nullptr, 0.0, nullptr, 0.0, 0.0, 1.0));
}

dgsem_status dgsem_kinetic_energy(dgsem_adjoint* a, const double* u, double* value,
                                  double* grad) {
  if (!a || !u) return DGSEM_ERR_INVALID_ARG;
  cudaError_t e = objective(a, u, grad);
  if (e == cudaSuccess && value) {
    e = cudaMemcpyAsync(value, a->result, sizeof(double), cudaMemcpyDeviceToHost,
                        a->ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(a->ctx->stream);
  }
  return st_of(e);
}

dgsem_status dgsem_adjoint_gradient(dgsem_adjoint* a, const double* u0, double t0, double dt,
                                    double* value, double* grad_u0) {
  if (!a || !u0 || !grad_u0) return DGSEM_ERR_INVALID_ARG;
  cudaStream_t st = a->ctx->stream;
  const size_t bytes = a->len * sizeof(double);
  const int last = a->nsnap - 1;
  // forward with checkpoints; the last segment is recorded
  cudaError_t e = cudaMemcpyAsync(a->work, u0, bytes, cudaMemcpyDeviceToDevice, st);
  for (int sg = 0; sg < a->nsnap && e == cudaSuccess; ++sg) {
    const int s0 = sg * a->every;
    const int s1 = s0 + a->every < a->nsteps ? s0 + a->every : a->nsteps;
    e = cudaMemcpyAsync(a->snaps + (int64_t)sg * a->len, a->work, bytes,
                        cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) break;
    if (sg == last) {
      e = record_segment(a, a->work, s0, s1, t0, dt);
    } else {
      for (int s = s0; s < s1 && e == cudaSuccess; ++s) {
        const double t = t0 + s * dt;
        e = fwd_stage(a, 1, nullptr, a->work, seg_slot(a, 0, 1), t, dt);
        if (e == cudaSuccess) e = fwd_stage(a, 2, a->work, seg_slot(a, 0, 1), seg_slot(a, 0, 2), t, dt);
        if (e == cudaSuccess) e = fwd_stage(a, 3, a->work, seg_slot(a, 0, 2), a->work, t, dt);
      }
    }
  }
  // objective and its gradient at the final state
  if (e == cudaSuccess) e = objective(a, a->work, a->lam);
  if (e == cudaSuccess && value)
    e = cudaMemcpyAsync(value, a->result, sizeof(double), cudaMemcpyDeviceToHost, st);
  // reverse sweep
  for (int sg = last; sg >= 0 && e == cudaSuccess; --sg) {
    const int s0 = sg * a->every;
    const int s1 = s0 + a->every < a->nsteps ? s0 + a->every : a->nsteps;
    if (sg != last) {
      e = cudaMemcpyAsync(a->work, a->snaps + (int64_t)sg * a->len, bytes,
                          cudaMemcpyDeviceToDevice, st);
      if (e == cudaSuccess) e = record_segment(a, a->work, s0, s1, t0, dt);
    }
    for (int s = s1 - 1; s >= s0 && e == cudaSuccess; --s) {
      const int r = s - s0;
      e = launch_vjp(a, seg_slot(a, r, 2), grad_slot(a, r, 2), a->lam, a->lam2, nullptr, 0.0,
                     nullptr, 0.0, 2.0 / 3.0, (2.0 / 3.0) * dt);
      if (e == cudaSuccess)
        e = launch_vjp(a, seg_slot(a, r, 1), grad_slot(a, r, 1), a->lam2, a->lam1, nullptr,
                       0.0, nullptr, 0.0, 1.0 / 4.0, (1.0 / 4.0) * dt);
      if (e == cudaSuccess)
        e = launch_vjp(a, seg_slot(a, r, 0), grad_slot(a, r, 0), a->lam1, a->lam, a->lam,
                       1.0 / 3.0, a->lam2, 3.0 / 4.0, 1.0, dt);
    }
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(grad_u0, a->lam, bytes, cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return st_of(e);
}

}  // extern "C"
