// C ABI implementation: context lifetime, descriptor validation, device
// tables, and the small auxiliary kernels (indicator, initial conditions,
// layout conversion).  The fused stage kernel lives in stage_kernel.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/dgsem_b200.h"
#include "context.hpp"
#include "engine.cuh"
#include "tables.hpp"

using namespace dgsem;

namespace {

dgsem_status cuda_status(cudaError_t e) {
  return e == cudaSuccess ? DGSEM_OK : DGSEM_ERR_CUDA;
}

void conserved_from_primitive(const double* prim, double gamma, double* cons) {
  // utils/state_conversion.hpp:9-24 (2D)
  cons[0] = prim[0];
  double vsq = 0.0;
  for (int d = 0; d < 2; ++d) {
    cons[d + 1] = prim[0] * prim[d + 1];
    vsq = vsq + prim[d + 1] * prim[d + 1];
  }
  cons[3] = prim[3] / (gamma - 1.0) + 0.5 * prim[0] * vsq;
}

// ---------------------------------------------------------------------------
// auxiliary kernels
// ---------------------------------------------------------------------------

template <int N, int DIM = 2>
__global__ void indicator_kernel(const double* u, int64_t nelem, int ND,
                                 BasisConst<N> basis, double threshold, double s,
                                 double alpha_min, double alpha_max, double atol,
                                 double* alpha, uint8_t* flags) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nelem) return;
  double a;
  if constexpr (DIM == 2)
    a = hg_alpha_2d<N>(u + e * 4 * ND, ND, basis, threshold, s, alpha_min, alpha_max);
  else
    a = hg_alpha_3d<N>(u + e * 5 * ND, ND, basis, threshold, s, alpha_min, alpha_max);
  if (alpha) alpha[e] = a;
  if (flags) flags[e] = (fabs(a - 0.0) > atol) ? 1 : 0;
}

__device__ void ic_state(int kind, int ndims, const double* x,
                         const double* params, double gamma, const BcParams& bc,
                         double* u) {
  const double pi = 3.14159265358979323846;
  if (kind == DGSEM_IC_KELVIN_HELMHOLTZ) {
    const double B = tanh(15.0 * x[1] + 7.5) - tanh(15.0 * x[1] - 7.5);
    const double rho = 0.5 + 0.75 * B;
    const double v1 = 0.5 * (B - 1.0);
    const double v2 = 0.1 * sin(2.0 * pi * x[0]);
    u[0] = rho;
    u[1] = rho * v1;
    u[2] = rho * v2;
    u[3] = 1.0 / (gamma - 1.0) + 0.5 * rho * (v1 * v1 + v2 * v2);
  } else if (kind == DGSEM_IC_DOUBLE_MACH) {
    dmr_state(bc, x[0], x[1], 0.0, u);
  } else if (kind == DGSEM_IC_TAYLOR_GREEN_3D) {
    const double rho = 1.0;
    const double v1 = sin(x[0]) * cos(x[1]) * cos(x[2]);
    const double v2 = -cos(x[0]) * sin(x[1]) * cos(x[2]);
    const double p = 100.0 / 1.4 + 1.0 / 16.0 * (cos(2.0 * x[0]) * cos(2.0 * x[2]) +
                                                 2.0 * cos(2.0 * x[1]) + 2.0 * cos(2.0 * x[0]) +
                                                 cos(2.0 * x[1]) * cos(2.0 * x[2]));
    u[0] = rho;
    u[1] = rho * v1;
    u[2] = rho * v2;
    u[3] = 0.0;
    u[4] = p / (gamma - 1.0) + 0.5 * rho * (v1 * v1 + v2 * v2);
  } else if (kind == DGSEM_IC_TAYLOR_GREEN_2D) {
    const double p0 = params ? params[0] : 1.0 / (gamma * 0.01);
    const double v1 = sin(x[0]) * cos(x[1]);
    const double v2 = -cos(x[0]) * sin(x[1]);
    const double p = p0 + (cos(2.0 * x[0]) + cos(2.0 * x[1])) / 4.0;
    u[0] = 1.0;
    u[1] = v1;
    u[2] = v2;
    u[3] = p / (gamma - 1.0) + 0.5 * (v1 * v1 + v2 * v2);
  } else {  // isentropic vortex (Shu): params = {beta, x0, y0}
    const double beta = params ? params[0] : 5.0;
    const double dx = x[0] - (params ? params[1] : 0.0);
    const double dy = x[1] - (params ? params[2] : 0.0);
    const double r2 = dx * dx + dy * dy;
    const double ex = exp(1.0 - r2);
    const double du = -beta / (2.0 * pi) * exp(0.5 * (1.0 - r2)) * dy;
    const double dvv = beta / (2.0 * pi) * exp(0.5 * (1.0 - r2)) * dx;
    const double T = 1.0 - (gamma - 1.0) * beta * beta / (8.0 * gamma * pi * pi) * ex;
    const double rho = pow(T, 1.0 / (gamma - 1.0));
    const double v1 = 1.0 + du, v2 = dvv;
    u[0] = rho;
    u[1] = rho * v1;
    u[2] = rho * v2;
    u[3] = rho * T / (gamma - 1.0) + 0.5 * rho * (v1 * v1 + v2 * v2);
  }
}

__global__ void initial_kernel(int kind, int ndims, int n, int64_t cells0,
                               int64_t cells1, int64_t nelem, DeviceTables tab,
                               BcParams bc, double gamma, double p0, double p1,
                               double p2, int has_params, double* u) {
  const int ND = ndims == 2 ? n * n : n * n * n;
  const int NV = ndims + 2;
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nelem * ND) return;
  const int64_t e = idx / ND;
  const int node = (int)(idx % ND);
  const int64_t ie = e % cells0;
  const int64_t je = ndims == 2 ? e / cells0 : (e / cells0) % cells1;
  const int64_t ke = ndims == 2 ? 0 : e / (cells0 * cells1);
  double x[3];
  x[0] = tab.coord[0][ie * n + node % n];
  x[1] = tab.coord[1][je * n + (node / n) % n];
  x[2] = ndims == 3 ? tab.coord[2][ke * n + node / (n * n)] : 0.0;
  const double params[3] = {p0, p1, p2};
  double s[5];
  ic_state(kind, ndims, x, has_params ? params : nullptr, gamma, bc, s);
  for (int q = 0; q < NV; ++q) u[(e * NV + q) * ND + node] = s[q];
}

// Device layout [e][var][node] <-> reference LayoutRight (i, j[, k], dof, var)
// where the element's reference offset is ((i * ny + j) * nz + k).
__global__ void layout_kernel(const double* src, double* dst, int ndims,
                              int64_t c0, int64_t c1, int64_t c2, int ND, int NV,
                              int to_reference) {
  const int64_t total = c0 * c1 * c2 * ND * NV;
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  // idx enumerates the device layout
  const int64_t e = idx / (ND * NV);
  const int q = (int)((idx / ND) % NV);
  const int node = (int)(idx % ND);
  const int64_t ie = e % c0;
  const int64_t je = (e / c0) % c1;
  const int64_t ke = e / (c0 * c1);
  const int64_t eref = ndims == 2 ? ie * c1 + je : (ie * c1 + je) * c2 + ke;
  const int64_t ridx = (eref * ND + node) * NV + q;
  if (to_reference) {
    dst[ridx] = src[idx];
  } else {
    dst[idx] = src[ridx];
  }
}

bool is_navier_stokes(int equation) {
  return equation == DGSEM_NAVIER_STOKES_2D || equation == DGSEM_NAVIER_STOKES_3D;
}

dgsem_status validate(const dgsem_mesh_desc* m, const dgsem_scheme_desc* s) {
  if (!m || !s) return DGSEM_ERR_INVALID_ARG;
  if (m->ndims != 2 && m->ndims != 3) return DGSEM_ERR_INVALID_ARG;
  if (m->polydeg < 1 || m->polydeg + 1 > kMaxNodes) return DGSEM_ERR_UNSUPPORTED;
  for (int a = 0; a < m->ndims; ++a) {
    if (m->n_cells[a] < 1 || m->n_cells[a] > (int64_t)1 << 24) return DGSEM_ERR_INVALID_ARG;
    if (!(m->domain_right[a] > m->domain_left[a])) return DGSEM_ERR_INVALID_ARG;
  }
  const bool ns = s->equation == DGSEM_NAVIER_STOKES_2D || s->equation == DGSEM_NAVIER_STOKES_3D;
  const int want_dims =
      s->equation == DGSEM_EULER_3D || s->equation == DGSEM_NAVIER_STOKES_3D ? 3 : 2;
  if (s->equation < 0 || s->equation > 3) return DGSEM_ERR_INVALID_ARG;
  if (want_dims != m->ndims) return DGSEM_ERR_INVALID_ARG;
  if (s->volume_flux < 0 || s->volume_flux > 2) return DGSEM_ERR_INVALID_ARG;
  if (s->surface_flux < 0 || s->surface_flux > 1) return DGSEM_ERR_INVALID_ARG;
  if (s->volume_integral < 0 || s->volume_integral > 1) return DGSEM_ERR_INVALID_ARG;
  if (!(s->gamma > 1.0)) return DGSEM_ERR_INVALID_ARG;
  for (int f = 0; f < 2 * m->ndims; ++f) {
    if (s->bc[f] < 0 || s->bc[f] > 7) return DGSEM_ERR_INVALID_ARG;
    const bool ns_wall = s->bc[f] == DGSEM_BC_NS_NOSLIP_ADIABATIC_WALL ||
                         s->bc[f] == DGSEM_BC_NS_SLIP_ADIABATIC_WALL;
    if (ns_wall && s->equation != DGSEM_NAVIER_STOKES_2D) return DGSEM_ERR_UNSUPPORTED;
    if (m->ndims == 3 && s->bc[f] != DGSEM_BC_PERIODIC) return DGSEM_ERR_UNSUPPORTED;
  }
  for (int d = 0; d < m->ndims; ++d) {
    // a direction is periodic iff both of its faces are periodic
    const bool p0 = s->bc[2 * d] == DGSEM_BC_PERIODIC;
    const bool p1 = s->bc[2 * d + 1] == DGSEM_BC_PERIODIC;
    if (p0 != p1) return DGSEM_ERR_INVALID_ARG;
  }
  if (s->surface_flux == DGSEM_SF_HLLC && m->ndims != 2) return DGSEM_ERR_UNSUPPORTED;
  if (s->volume_integral == DGSEM_VI_SHOCK_CAPTURING_HG) {
    if (!(s->alpha_min >= 0.0 && s->alpha_max >= 0.0)) return DGSEM_ERR_INVALID_ARG;
  }
  if (ns) {
    // shock capturing with the viscous terms in 2D (the reference defines no
    // 3D Navier-Stokes indicator)
    if (s->volume_integral != DGSEM_VI_SPLIT_FORM &&
        (m->ndims != 2 || s->volume_flux != DGSEM_VF_CHANDRASHEKAR ||
         s->surface_flux != DGSEM_SF_LAX_FRIEDRICHS))
      return DGSEM_ERR_UNSUPPORTED;
    // periodic directions or (2D) the Navier-Stokes adiabatic walls; 3D
    // meshes are periodic (checked above)
    for (int f = 0; f < 2 * m->ndims; ++f)
      if (s->bc[f] != DGSEM_BC_PERIODIC && s->bc[f] != DGSEM_BC_NS_NOSLIP_ADIABATIC_WALL &&
          s->bc[f] != DGSEM_BC_NS_SLIP_ADIABATIC_WALL)
        return DGSEM_ERR_UNSUPPORTED;
    if (!(s->mu >= 0.0) || !(s->prandtl > 0.0)) return DGSEM_ERR_INVALID_ARG;
  }
  return DGSEM_OK;
}

// Failure-path testing: with DGSEM_TEST_FAIL_ALLOC_AT=k in the environment
// at context creation, the k-th device allocation of that creation (1-based)
// fails as if cudaMalloc had run out of memory.
int test_fail_alloc_at() {
  const char* v = std::getenv("DGSEM_TEST_FAIL_ALLOC_AT");
  return v ? std::atoi(v) : 0;
}

template <class T>
T* device_alloc(dgsem_ctx* ctx, size_t count, cudaError_t* err) {
  void* p = nullptr;
  if (++ctx->alloc_calls == ctx->fail_alloc_at) {
    *err = cudaErrorMemoryAllocation;
    return nullptr;
  }
  *err = cudaMalloc(&p, count * sizeof(T));
  if (*err != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  ctx->allocations.push_back(p);
  return static_cast<T*>(p);
}

void free_all(dgsem_ctx* ctx) {
  for (void* p : ctx->allocations) cudaFree(p);
  ctx->allocations.clear();
}

}  // namespace

extern "C" {

const char* dgsem_status_string(dgsem_status s) {
  switch (s) {
    case DGSEM_OK: return "ok";
    case DGSEM_ERR_INVALID_ARG: return "invalid argument";
    case DGSEM_ERR_UNSUPPORTED: return "unsupported combination";
    case DGSEM_ERR_CUDA: return "CUDA error";
    case DGSEM_ERR_NONFINITE: return "non-finite value in state";
    case DGSEM_ERR_TIMEOUT: return "device wait timed out";
    case DGSEM_ERR_ALLOC: return "allocation failed";
    case DGSEM_ERR_SCRATCH_LIMIT: return "state larger than the static scratch";
  }
  return "unknown status";
}

dgsem_status dgsem_ctx_create(const dgsem_mesh_desc* mesh,
                              const dgsem_scheme_desc* scheme, void* stream,
                              dgsem_ctx** out) {
  if (!out) return DGSEM_ERR_INVALID_ARG;
  *out = nullptr;
  dgsem_status st = validate(mesh, scheme);
  if (st != DGSEM_OK) return st;
  const int nd = mesh->ndims;
  const int n = mesh->polydeg + 1;
  const bool hg = scheme->volume_integral == DGSEM_VI_SHOCK_CAPTURING_HG;
  std::unique_ptr<EngineBase> engine;
  try {
    engine = make_engine(nd, n, scheme->volume_flux, scheme->surface_flux, hg,
                         is_navier_stokes(scheme->equation));
  } catch (...) {
    return DGSEM_ERR_ALLOC;
  }
  if (!engine) return DGSEM_ERR_UNSUPPORTED;

  dgsem_ctx* ctx = new (std::nothrow) dgsem_ctx();
  if (!ctx) return DGSEM_ERR_ALLOC;
  ctx->mesh = *mesh;
  ctx->scheme = *scheme;
  ctx->stream = static_cast<cudaStream_t>(stream);
  ctx->fail_alloc_at = test_fail_alloc_at();
  cudaGetDevice(&ctx->device);
  ctx->engine = std::move(engine);
  EngineConfig& c = ctx->cfg;
  c.ndims = nd;
  c.n = n;
  c.nelem = 1;
  for (int a = 0; a < 3; ++a) {
    c.cells[a] = a < nd ? mesh->n_cells[a] : 1;
    c.periodic[a] = a < nd ? (scheme->bc[2 * a] == DGSEM_BC_PERIODIC) : 1;
    c.nelem *= c.cells[a];
  }
  // Failure-path testing only: DGSEM_TEST_WAIT_LIMIT_NS bounds the stage
  // kernels' tile-copy waits (default 1 s); DGSEM_TEST_SKIP_TILE_COPY=1 makes
  // the node-parallel kernels arm the u_n barrier without issuing the copy,
  // so the bounded wait runs out (DGSEM_ERR_TIMEOUT from dgsem_check_finite)
  // with no copy in flight.
  if (const char* v = std::getenv("DGSEM_TEST_WAIT_LIMIT_NS"))
    c.wait_limit_ns = std::strtoull(v, nullptr, 10);
  if (const char* v = std::getenv("DGSEM_TEST_SKIP_TILE_COPY")) c.skip_tile_copy = std::atoi(v);
  c.gamma = scheme->gamma;
  c.mu = scheme->mu;
  c.prandtl = scheme->prandtl > 0 ? scheme->prandtl : 0.72;
  c.alpha_max = scheme->alpha_max;
  c.alpha_min = scheme->alpha_min;
  const double eps = std::numeric_limits<double>::epsilon();
  c.atol = std::max(100.0 * eps, std::pow(eps, 0.75));  // volume_flux.hpp:772-773
  // indicator.hpp:367-378
  c.hg_threshold = 0.5 * std::pow(10.0, -1.8 * std::pow((double)n, 0.25));
  c.hg_s = std::log((1.0 - 0.0001) / 0.0001);
  make_basis(mesh->polydeg, &c.basis);
  for (int f = 0; f < 6; ++f) c.bc.kind[f] = f < 2 * nd ? scheme->bc[f] : 0;
  for (int q = 0; q < 4; ++q) c.bc.state[q] = scheme->bc_state[q];
  {
    const double phi = M_PI / 6.0;
    const double post[4] = {8.0, 8.25 * std::cos(phi), -8.25 * std::sin(phi), 116.5};
    const double pre[4] = {1.4, 0.0, 0.0, 1.0};
    conserved_from_primitive(post, scheme->gamma, c.bc.dmr_post);
    conserved_from_primitive(pre, scheme->gamma, c.bc.dmr_pre);
    c.bc.sqrt3 = std::sqrt(3.0);
  }
  ctx->nodes = nd == 2 ? n * n : n * n * n;
  ctx->nvars = nd + 2;
  ctx->state_len = c.nelem * ctx->nodes * ctx->nvars;

  MetricTablesHost mt;
  if (!make_metric_tables(c.basis, nd, c.cells, mesh->domain_left,
                          mesh->domain_right, &mt)) {
    delete ctx;
    return DGSEM_ERR_INVALID_ARG;
  }
  // one device block for all tables
  size_t total = 0;
  auto add = [&](const std::vector<double>& v) { total += v.size(); };
  for (int a = 0; a < nd; ++a) {
    add(mt.coord[a]);
    add(mt.jdiag[a]);
    for (int cc = 0; cc < nd; ++cc) add(mt.ja[a][cc]);
  }
  for (int a = 0; a < nd; ++a)
    for (int cc = 0; cc < nd; ++cc) add(mt.fv[a][cc]);
  cudaError_t err;
  ctx->table_block = device_alloc<double>(ctx, total + 1, &err);
  if (!ctx->table_block) {
    free_all(ctx);
    delete ctx;
    return DGSEM_ERR_ALLOC;
  }
  std::vector<double> host(total + 1, 0.0);
  size_t off = 0;
  auto place = [&](const std::vector<double>& v) -> const double* {
    const double* dptr = ctx->table_block + off;
    std::memcpy(host.data() + off, v.data(), v.size() * sizeof(double));
    off += v.size();
    return dptr;
  };
  std::memset(&c.tab, 0, sizeof(c.tab));
  for (int a = 0; a < nd; ++a) {
    c.tab.coord[a] = place(mt.coord[a]);
    c.tab.jdiag[a] = place(mt.jdiag[a]);
    for (int cc = 0; cc < nd; ++cc) c.tab.ja[a][cc] = place(mt.ja[a][cc]);
  }
  for (int a = 0; a < nd; ++a)
    for (int cc = 0; cc < nd; ++cc) c.tab.fv[a][cc] = place(mt.fv[a][cc]);
  err = cudaMemcpy(ctx->table_block, host.data(), (total + 1) * sizeof(double),
                   cudaMemcpyHostToDevice);
  ctx->tmp1 = device_alloc<double>(ctx, ctx->state_len, &err);
  ctx->tmp2 = ctx->tmp1 ? device_alloc<double>(ctx, ctx->state_len, &err) : nullptr;
  ctx->staging = ctx->tmp2 ? device_alloc<double>(ctx, ctx->state_len, &err) : nullptr;
  ctx->tdev = ctx->staging ? device_alloc<double>(ctx, 1, &err) : nullptr;
  ctx->flag = ctx->tdev ? device_alloc<unsigned int>(ctx, 1, &err) : nullptr;
  c.grad = nullptr;
  if (ctx->flag && is_navier_stokes(scheme->equation)) {
    // four gradient variables x ndims directions per node
    c.grad = device_alloc<double>(ctx, (size_t)c.nelem * 4 * nd * ctx->nodes, &err);
    if (!c.grad) ctx->flag = nullptr;
  }
  // per-element info and -1/J per node, computed once here instead of in
  // every stage launch
  c.elem_info = nullptr;
  c.mij = nullptr;
  int* info_tab = nullptr;
  double* mij_tab = nullptr;
  if (ctx->flag) {
    info_tab = device_alloc<int>(ctx, (size_t)c.nelem * 12, &err);
    mij_tab = info_tab ? device_alloc<double>(ctx, (size_t)c.nelem * ctx->nodes, &err) : nullptr;
    if (!mij_tab) ctx->flag = nullptr;
  }
  if (!ctx->flag) {
    free_all(ctx);
    delete ctx;
    return DGSEM_ERR_ALLOC;
  }
  cudaMemset(ctx->flag, 0, sizeof(unsigned int));
  c.nonfinite = ctx->flag;
  {
    MeshView mv{};
    for (int i = 0; i < 3; ++i) {
      mv.cells[i] = (int)c.cells[i];
      mv.periodic[i] = c.periodic[i];
    }
    mv.nelem = (int)c.nelem;
    mv.tab = c.tab;
    err = ctx->engine->build_mesh_tables(mv, info_tab, mij_tab, nullptr);
  }
  if (err == cudaSuccess) {
    c.elem_info = info_tab;
    c.mij = mij_tab;
  }
  if (err == cudaSuccess) err = cudaDeviceSynchronize();
  if (err != cudaSuccess) {
    free_all(ctx);
    delete ctx;
    return DGSEM_ERR_CUDA;
  }
  *out = ctx;
  return DGSEM_OK;
}

dgsem_status dgsem_ctx_destroy(dgsem_ctx* ctx) {
  if (!ctx) return DGSEM_ERR_INVALID_ARG;
  cudaStreamSynchronize(ctx->stream);
  free_all(ctx);
  delete ctx;
  return DGSEM_OK;
}

dgsem_status dgsem_ctx_set_stream(dgsem_ctx* ctx, void* stream) {
  if (!ctx) return DGSEM_ERR_INVALID_ARG;
  ctx->stream = static_cast<cudaStream_t>(stream);
  return DGSEM_OK;
}

dgsem_status dgsem_get_sizes(const dgsem_ctx* ctx, int64_t* n_elements,
                             int* nodes_per_element, int* nvars,
                             int64_t* state_len) {
  if (!ctx) return DGSEM_ERR_INVALID_ARG;
  if (n_elements) *n_elements = ctx->cfg.nelem;
  if (nodes_per_element) *nodes_per_element = ctx->nodes;
  if (nvars) *nvars = ctx->nvars;
  if (state_len) *state_len = ctx->state_len;
  return DGSEM_OK;
}

dgsem_status dgsem_set_indicator_parameters(dgsem_ctx* ctx, double alpha_max,
                                            double alpha_min, int alpha_smooth) {
  if (!ctx || !(alpha_max >= 0.0) || !(alpha_min >= 0.0)) return DGSEM_ERR_INVALID_ARG;
  ctx->cfg.alpha_max = alpha_max;
  ctx->cfg.alpha_min = alpha_min;
  ctx->scheme.alpha_smooth = alpha_smooth;
  return DGSEM_OK;
}

dgsem_status dgsem_rhs(dgsem_ctx* ctx, const double* u, double* du, double t) {
  if (!ctx || !u || !du || u == du) return DGSEM_ERR_INVALID_ARG;
  ctx->launches += ctx->engine->kernels_per_stage();
  return cuda_status(ctx->engine->stage(ctx->cfg, nullptr, u, du, 0.0, 0.0, 1.0,
                                        t, nullptr, nullptr, ctx->stream));
}

// One SSPRK3 stage (SSPRK3.hpp:162-180).  With t_dev the stage time is
// *t_dev + t + stage offset (graph replay); otherwise t + stage offset.
static dgsem_status launch_stage(dgsem_ctx* ctx, int stage, const double* u_n,
                                 const double* u_in, double* u_out, double t,
                                 double dt, const double* t_dev,
                                 cudaStream_t stream) {
  if (!ctx || !u_in || !u_out || u_out == u_in) return DGSEM_ERR_INVALID_ARG;
  double a, b, c, ts;
  if (stage == 1) {
    a = 0.0; b = 1.0; c = dt; ts = t;
  } else if (stage == 2) {
    a = 3.0 / 4.0; b = 1.0 / 4.0; c = (1.0 / 4.0) * dt; ts = t + dt;
  } else if (stage == 3) {
    a = 1.0 / 3.0; b = 2.0 / 3.0; c = (2.0 / 3.0) * dt; ts = t + 0.5 * dt;
  } else {
    return DGSEM_ERR_INVALID_ARG;
  }
  if (stage > 1 && !u_n) return DGSEM_ERR_INVALID_ARG;
  ctx->launches += ctx->engine->kernels_per_stage();
  // the stage that completes a step also integrates the new state when the
  // fused diagnostics are on
  double* diag = stage == 3 ? ctx->diag_partials : nullptr;
  return cuda_status(ctx->engine->stage(ctx->cfg, u_n, u_in, u_out, a, b, c, ts,
                                        t_dev, nullptr, stream, diag));
}

dgsem_status dgsem_ssprk3_stage(dgsem_ctx* ctx, int stage, const double* u_n,
                                const double* u_in, double* u_out, double t,
                                double dt) {
  if (!ctx) return DGSEM_ERR_INVALID_ARG;
  return launch_stage(ctx, stage, u_n, u_in, u_out, t, dt, nullptr, ctx->stream);
}

dgsem_status dgsem_ssprk3_step(dgsem_ctx* ctx, double* u, double t, double dt) {
  if (!ctx || !u) return DGSEM_ERR_INVALID_ARG;
  dgsem_status st = dgsem_ssprk3_stage(ctx, 1, nullptr, u, ctx->tmp1, t, dt);
  if (st == DGSEM_OK) st = dgsem_ssprk3_stage(ctx, 2, u, ctx->tmp1, ctx->tmp2, t, dt);
  if (st == DGSEM_OK) st = dgsem_ssprk3_stage(ctx, 3, u, ctx->tmp2, u, t, dt);
  return st;
}

dgsem_status dgsem_ssprk3_steps(dgsem_ctx* ctx, double* u, double t0, double dt,
                                int nsteps) {
  if (!ctx || !u || nsteps < 0) return DGSEM_ERR_INVALID_ARG;
  for (int s = 0; s < nsteps; ++s) {
    dgsem_status st = dgsem_ssprk3_step(ctx, u, t0 + s * dt, dt);
    if (st != DGSEM_OK) return st;
  }
  return DGSEM_OK;
}

dgsem_status dgsem_ssprk3_steps_host(dgsem_ctx* ctx, double* u_host, double t0,
                                     double dt, int nsteps) {
  if (!ctx || !u_host || nsteps < 0) return DGSEM_ERR_INVALID_ARG;
  const size_t bytes = (size_t)ctx->state_len * sizeof(double);
  cudaError_t e = cudaMemcpyAsync(ctx->staging, u_host, bytes,
                                  cudaMemcpyHostToDevice, ctx->stream);
  if (e != cudaSuccess) return DGSEM_ERR_CUDA;
  dgsem_status st = dgsem_ssprk3_steps(ctx, ctx->staging, t0, dt, nsteps);
  if (st != DGSEM_OK) return st;
  e = cudaMemcpyAsync(u_host, ctx->staging, bytes, cudaMemcpyDeviceToHost,
                      ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return cuda_status(e);
}

struct dgsem_graph {
  dgsem_ctx* ctx = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int nsteps = 0;
  double dt = 0.0;
};

namespace {
__global__ void set_clock_kernel(double* t_dev, double t) { *t_dev = t; }
}  // namespace

dgsem_status dgsem_graph_create(dgsem_ctx* ctx, double* u, double dt,
                                int nsteps, dgsem_graph** out) {
  if (!ctx || !u || !out || nsteps < 1) return DGSEM_ERR_INVALID_ARG;
  *out = nullptr;
  cudaStream_t cap;
  if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess)
    return DGSEM_ERR_CUDA;
  dgsem_graph* g = new (std::nothrow) dgsem_graph();
  if (!g) {
    cudaStreamDestroy(cap);
    return DGSEM_ERR_ALLOC;
  }
  g->ctx = ctx;
  g->nsteps = nsteps;
  g->dt = dt;
  dgsem_status st = DGSEM_OK;
  cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    for (int s = 0; s < nsteps && st == DGSEM_OK; ++s) {
      const double toff = s * dt;
      st = launch_stage(ctx, 1, nullptr, u, ctx->tmp1, toff, dt, ctx->tdev, cap);
      if (st == DGSEM_OK)
        st = launch_stage(ctx, 2, u, ctx->tmp1, ctx->tmp2, toff, dt, ctx->tdev, cap);
      if (st == DGSEM_OK)
        st = launch_stage(ctx, 3, u, ctx->tmp2, u, toff, dt, ctx->tdev, cap);
    }
    cudaError_t e2 = cudaStreamEndCapture(cap, &g->graph);
    if (e2 != cudaSuccess && st == DGSEM_OK) st = DGSEM_ERR_CUDA;
  } else {
    st = DGSEM_ERR_CUDA;
  }
  if (st == DGSEM_OK &&
      cudaGraphInstantiate(&g->exec, g->graph, 0) != cudaSuccess)
    st = DGSEM_ERR_CUDA;
  cudaStreamDestroy(cap);
  if (st != DGSEM_OK) {
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return st;
  }
  *out = g;
  return DGSEM_OK;
}

dgsem_status dgsem_graph_launch(dgsem_graph* g, double t0) {
  if (!g || !g->exec) return DGSEM_ERR_INVALID_ARG;
  dgsem_ctx* ctx = g->ctx;
  set_clock_kernel<<<1, 1, 0, ctx->stream>>>(ctx->tdev, t0);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaGraphLaunch(g->exec, ctx->stream);
  ctx->launches += 1 + 3 * (int64_t)g->nsteps * ctx->engine->kernels_per_stage();
  return cuda_status(e);
}

dgsem_status dgsem_graph_destroy(dgsem_graph* g) {
  if (!g) return DGSEM_ERR_INVALID_ARG;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return DGSEM_OK;
}

dgsem_status dgsem_indicator(dgsem_ctx* ctx, const double* u, double* alpha,
                             uint8_t* flags) {
  if (!ctx || !u) return DGSEM_ERR_INVALID_ARG;
  if (ctx->scheme.equation == DGSEM_NAVIER_STOKES_3D) return DGSEM_ERR_UNSUPPORTED;
  const EngineConfig& c = ctx->cfg;
  const int threads = 128;
  const unsigned blocks = (unsigned)((c.nelem + threads - 1) / threads);
  if (c.ndims == 3) {
#define DGSEM_IND3(NN)                                                       \
  case NN: {                                                                 \
    BasisConst<NN> b;                                                        \
    fill_basis_const<NN>(c.basis, &b);                                       \
    indicator_kernel<NN, 3><<<blocks, threads, 0, ctx->stream>>>(            \
        u, c.nelem, ctx->nodes, b, c.hg_threshold, c.hg_s, c.alpha_min,      \
        c.alpha_max, c.atol, alpha, flags);                                  \
    break;                                                                   \
  }
    switch (c.n) {
      DGSEM_IND3(2) DGSEM_IND3(3) DGSEM_IND3(4) DGSEM_IND3(5)
      default: return DGSEM_ERR_UNSUPPORTED;
    }
#undef DGSEM_IND3
    ctx->launches++;
    return cuda_status(cudaGetLastError());
  }
#define DGSEM_IND(NN)                                                        \
  case NN: {                                                                 \
    BasisConst<NN> b;                                                        \
    fill_basis_const<NN>(c.basis, &b);                                       \
    indicator_kernel<NN><<<blocks, threads, 0, ctx->stream>>>(               \
        u, c.nelem, ctx->nodes, b, c.hg_threshold, c.hg_s, c.alpha_min,      \
        c.alpha_max, c.atol, alpha, flags);                                  \
    break;                                                                   \
  }
  switch (c.n) {
    DGSEM_IND(2) DGSEM_IND(3) DGSEM_IND(4) DGSEM_IND(5) DGSEM_IND(6)
    DGSEM_IND(7) DGSEM_IND(8)
    default: return DGSEM_ERR_UNSUPPORTED;
  }
#undef DGSEM_IND
  ctx->launches++;
  return cuda_status(cudaGetLastError());
}

}  // extern "C"

namespace dgsem {
cudaError_t launch_initial(int kind, int ndims, int n, const int64_t* cells, int64_t nelem,
                           const DeviceTables& tab, const BcParams& bc, double gamma,
                           const double* params, double* u, cudaStream_t s) {
  const int nodes = ndims == 2 ? n * n : n * n * n;
  const int64_t total = nelem * nodes;
  const int threads = 256;
  initial_kernel<<<(unsigned)((total + threads - 1) / threads), threads, 0, s>>>(
      kind, ndims, n, cells[0], cells[1], nelem, tab, bc, gamma, params ? params[0] : 0.0,
      params ? params[1] : 0.0, params ? params[2] : 0.0, params ? 1 : 0, u);
  return cudaGetLastError();
}
}  // namespace dgsem

extern "C" {

dgsem_status dgsem_initial_condition(dgsem_ctx* ctx, int kind,
                                     const double* params, double* u) {
  if (!ctx || !u || kind < 0 || kind > 4) return DGSEM_ERR_INVALID_ARG;
  const EngineConfig& c = ctx->cfg;
  const bool want3 = kind == DGSEM_IC_TAYLOR_GREEN_3D;
  if (want3 != (c.ndims == 3)) return DGSEM_ERR_INVALID_ARG;
  ctx->launches++;
  return cuda_status(launch_initial(kind, c.ndims, c.n, c.cells, c.nelem, c.tab, c.bc, c.gamma,
                                    params, u, ctx->stream));
}

static dgsem_status layout(dgsem_ctx* ctx, const double* src, double* dst,
                           int to_ref) {
  if (!ctx || !src || !dst || src == dst) return DGSEM_ERR_INVALID_ARG;
  const EngineConfig& c = ctx->cfg;
  const int threads = 256;
  layout_kernel<<<(unsigned)((ctx->state_len + threads - 1) / threads), threads,
                  0, ctx->stream>>>(src, dst, c.ndims, c.cells[0], c.cells[1],
                                    c.cells[2], ctx->nodes, ctx->nvars, to_ref);
  ctx->launches++;
  return cuda_status(cudaGetLastError());
}

dgsem_status dgsem_to_reference_layout(dgsem_ctx* ctx, const double* u,
                                       double* u_ref) {
  return layout(ctx, u, u_ref, 1);
}

dgsem_status dgsem_from_reference_layout(dgsem_ctx* ctx, const double* u_ref,
                                         double* u) {
  return layout(ctx, u_ref, u, 0);
}

dgsem_status dgsem_check_finite(dgsem_ctx* ctx) {
  if (!ctx) return DGSEM_ERR_INVALID_ARG;
  unsigned int h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, ctx->flag, sizeof(h),
                                  cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return DGSEM_ERR_CUDA;
  if (h) {
    cudaMemsetAsync(ctx->flag, 0, sizeof(unsigned int), ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    // bit 1: a pipelined stage kernel gave up waiting for a tile copy
    return (h & 2u) ? DGSEM_ERR_TIMEOUT : DGSEM_ERR_NONFINITE;
  }
  return DGSEM_OK;
}

namespace {
// Second pass of the fused diagnostics: the per-block partials summed in a
// fixed order (each thread a strided subset in index order, then a fixed
// tree), so the result does not depend on block scheduling.
__global__ void diag_reduce_kernel(const double* partials, int64_t nslots, double* out) {
  __shared__ double s[3][256];
  double a[3] = {0.0, 0.0, 0.0};
  for (int64_t i = threadIdx.x; i < nslots; i += 256)
    for (int k = 0; k < 3; ++k) a[k] += partials[3 * i + k];
  for (int k = 0; k < 3; ++k) s[k][threadIdx.x] = a[k];
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int k = 0; k < 3; ++k) s[k][threadIdx.x] += s[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; ++k) out[k] = s[k][0];
}
}  // namespace

dgsem_status dgsem_set_diagnostics(dgsem_ctx* ctx, int enable) {
  if (!ctx) return DGSEM_ERR_INVALID_ARG;
  if (!enable) {
    ctx->diag_partials = nullptr;  // the buffers stay with the context
    return DGSEM_OK;
  }
  if (!ctx->diag_result) {
    cudaError_t err;
    // at most one slot per element (every launch shape has >= 1 element per block)
    double* part = device_alloc<double>(ctx, (size_t)3 * ctx->cfg.nelem, &err);
    if (!part) return DGSEM_ERR_ALLOC;
    double* res = device_alloc<double>(ctx, 3, &err);
    if (!res) return DGSEM_ERR_ALLOC;
    ctx->diag_result = res;
    ctx->diag_store = part;
  }
  ctx->diag_partials = ctx->diag_store;
  return DGSEM_OK;
}

dgsem_status dgsem_diagnostics(dgsem_ctx* ctx, double* volume, double* mean_kinetic_energy,
                               double* mean_entropy) {
  if (!ctx || !ctx->diag_partials) return DGSEM_ERR_INVALID_ARG;
  const int64_t slots = ctx->engine->last_diag_slots();
  if (slots <= 0) return DGSEM_ERR_INVALID_ARG;  // no step since diagnostics were enabled
  diag_reduce_kernel<<<1, 256, 0, ctx->stream>>>(ctx->diag_partials, slots, ctx->diag_result);
  ctx->launches++;
  double h[3];
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h, ctx->diag_result, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return DGSEM_ERR_CUDA;
  if (volume) *volume = h[0];
  if (mean_kinetic_energy) *mean_kinetic_energy = h[1] / h[0];
  if (mean_entropy) *mean_entropy = h[2] / h[0];
  return DGSEM_OK;
}

dgsem_status dgsem_launch_count(const dgsem_ctx* ctx, int64_t* count) {
  if (!ctx || !count) return DGSEM_ERR_INVALID_ARG;
  *count = ctx->launches;
  return DGSEM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Launch-shape autotuner: every engine has kNumVariants launch shapes of the
// same kernel (bitwise-identical results).  Tuning times each on the real mesh
// and state; choices are cached per (scheme, degree, element count) for the
// process and, if DGSEM_TUNING_FILE names a file, persisted there as lines
// "key variant".
// ---------------------------------------------------------------------------
namespace dgsem {
namespace tune_detail {

std::mutex& tune_mutex() {
  static std::mutex m;
  return m;
}

std::map<std::string, int>& tune_cache() {
  static std::map<std::string, int> cache;
  static bool loaded = false;
  if (!loaded) {
    loaded = true;
    if (const char* path = std::getenv("DGSEM_TUNING_FILE")) {
      std::ifstream in(path);
      std::string key;
      int v;
      while (in >> key >> v)
        if (v >= 0 && v < kNumVariants) cache[key] = v;
    }
  }
  return cache;
}

void tune_store(const std::string& key, int v) {
  tune_cache()[key] = v;
  if (const char* path = std::getenv("DGSEM_TUNING_FILE")) {
    std::ofstream out(path, std::ios::app);
    out << key << " " << v << "\n";
  }
}

}  // namespace tune_detail

std::string tune_key(int ndims, int n, int vf, int sf, int hg, int ns, int64_t nelem) {
  std::ostringstream k;
  k << "d" << ndims << "_n" << n << "_vf" << vf << "_sf" << sf << "_hg" << hg << "_ns" << ns
    << "_e" << nelem;
  return k.str();
}

// Times `launch` (one SSPRK3 step on `s`) for each variant of `eng`: one
// warm-up per variant, then `rounds` rounds that each time every variant once,
// starting the round at a different variant so that no variant is always
// timed first or always after the same neighbour (clock and power drift then
// spreads over all variants instead of favouring one).  Each timed launch is
// preceded (outside the timed region) by a write of `flush_bytes` to `flush`
// when given, which evicts L2 so that every timed step streams its states
// from HBM.  Returns the variant with the smallest median time and optionally
// the medians.
template <class Launch>
int time_variants(EngineBase* eng, cudaStream_t s, Launch&& launch, double* times_ms,
                  void* flush, size_t flush_bytes) {
  constexpr int rounds = 7;
  const int nv = eng->num_variants();
  std::vector<cudaEvent_t> ev(2 * rounds * nv);
  for (auto& e : ev) cudaEventCreate(&e);
  for (int v = 0; v < nv; ++v) {
    eng->set_variant(v);
    launch();
  }
  for (int r = 0; r < rounds; ++r)
    for (int k = 0; k < nv; ++k) {
      const int v = (r + k) % nv;
      eng->set_variant(v);
      if (flush) cudaMemsetAsync(flush, (r * nv + k) & 0xff, flush_bytes, s);
      cudaEventRecord(ev[2 * (r * nv + v)], s);
      launch();
      cudaEventRecord(ev[2 * (r * nv + v) + 1], s);
    }
  cudaStreamSynchronize(s);
  int best = 0;
  float best_ms = 1e30f;
  for (int v = 0; v < kNumVariants; ++v) {
    if (v >= nv) {
      if (times_ms) times_ms[v] = 0.0;
      continue;
    }
    float ms[rounds];
    for (int r = 0; r < rounds; ++r) {
      ms[r] = 0.f;
      cudaEventElapsedTime(&ms[r], ev[2 * (r * nv + v)], ev[2 * (r * nv + v) + 1]);
    }
    std::sort(ms, ms + rounds);
    const float med = ms[rounds / 2];
    if (times_ms) times_ms[v] = med;
    if (med < best_ms) {
      best_ms = med;
      best = v;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  return best;
}

}  // namespace dgsem

extern "C" {

dgsem_status dgsem_set_launch_variant(dgsem_ctx* ctx, int variant) {
  if (!ctx || variant < 0 || variant >= ctx->engine->num_variants()) return DGSEM_ERR_INVALID_ARG;
  ctx->engine->set_variant(variant);
  return DGSEM_OK;
}

dgsem_status dgsem_autotune(dgsem_ctx* ctx, const double* u, int* chosen, double* times_ms) {
  using namespace dgsem::tune_detail;
  if (!ctx || !u) return DGSEM_ERR_INVALID_ARG;
  const EngineConfig& c = ctx->cfg;
  const bool warm = std::getenv("DGSEM_AUTOTUNE_WARM") != nullptr;
  const std::string key =
      tune_key(c.ndims, c.n, ctx->scheme.volume_flux, ctx->scheme.surface_flux,
               ctx->scheme.volume_integral, is_navier_stokes(ctx->scheme.equation),
               c.nelem) +
      (warm ? "_warm" : "_cold");
  std::lock_guard<std::mutex> lock(tune_mutex());
  auto it = tune_cache().find(key);
  if (it != tune_cache().end() && !times_ms) {
    ctx->engine->set_variant(it->second);
    if (chosen) *chosen = it->second;
    return DGSEM_OK;
  }
  // L2 eviction buffer (twice the 126 MB L2), released before returning
  void* flush = nullptr;
  const size_t flush_bytes = size_t(256) << 20;
  if (!warm && cudaMalloc(&flush, flush_bytes) != cudaSuccess) {
    cudaGetLastError();
    flush = nullptr;
  }
  // one SSPRK3 step from u into the context temporaries (u is not modified)
  cudaError_t err = cudaSuccess;
  const double dt = 1.0e-6;
  const int best = time_variants(ctx->engine.get(), ctx->stream, [&]() {
    EngineBase* eng = ctx->engine.get();
    cudaError_t e = eng->stage(ctx->cfg, nullptr, u, ctx->tmp1, 0.0, 1.0, dt, 0.0, nullptr,
                               nullptr, ctx->stream);
    if (e == cudaSuccess)
      e = eng->stage(ctx->cfg, u, ctx->tmp1, ctx->tmp2, 3.0 / 4.0, 1.0 / 4.0, dt / 4.0, dt,
                     nullptr, nullptr, ctx->stream);
    if (e == cudaSuccess)
      e = eng->stage(ctx->cfg, u, ctx->tmp2, ctx->tmp1, 1.0 / 3.0, 2.0 / 3.0, 2.0 * dt / 3.0,
                     0.5 * dt, nullptr, nullptr, ctx->stream);
    if (e != cudaSuccess) err = e;
  }, times_ms, flush, flush_bytes);
  if (flush) {
    cudaStreamSynchronize(ctx->stream);
    cudaFree(flush);
  }
  if (err != cudaSuccess) return DGSEM_ERR_CUDA;
  ctx->engine->set_variant(best);
  tune_store(key, best);
  if (chosen) *chosen = best;
  return DGSEM_OK;
}

dgsem_status dgsem_basis_tables_host(int polydeg, double* out) {
  BasisTables b;
  if (!out || !make_basis(polydeg, &b)) return DGSEM_ERR_INVALID_ARG;
  const int n = b.n;
  size_t o = 0;
  for (int i = 0; i < n; ++i) out[o++] = b.nodes[i];
  for (int i = 0; i < n; ++i) out[o++] = b.weights[i];
  for (int i = 0; i < n; ++i) out[o++] = b.inv_weights[i];
  for (int i = 0; i < n; ++i) out[o++] = b.lhat_left[i];
  for (int i = 0; i < n; ++i) out[o++] = b.lhat_right[i];
  for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) out[o++] = b.D[i][j];
  for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) out[o++] = b.Dsplit[i][j];
  for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) out[o++] = b.Dhat[i][j];
  for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) out[o++] = b.Vinv[i][j];
  return DGSEM_OK;
}

dgsem_status dgsem_metrics_host(const dgsem_mesh_desc* mesh, double* ja,
                                double* inv_j) {
  if (!mesh || (mesh->ndims != 2 && mesh->ndims != 3)) return DGSEM_ERR_INVALID_ARG;
  BasisTables b;
  if (!make_basis(mesh->polydeg, &b)) return DGSEM_ERR_INVALID_ARG;
  MetricTablesHost mt;
  int64_t cells[3] = {1, 1, 1};
  for (int a = 0; a < mesh->ndims; ++a) cells[a] = mesh->n_cells[a];
  if (!make_metric_tables(b, mesh->ndims, cells, mesh->domain_left,
                          mesh->domain_right, &mt))
    return DGSEM_ERR_INVALID_ARG;
  const int nd = mesh->ndims;
  const int n = b.n;
  const int ND = nd == 2 ? n * n : n * n * n;
  // reference logical order: cells (i slowest) x dof x a x c
  for (int64_t ie = 0; ie < cells[0]; ++ie)
    for (int64_t je = 0; je < cells[1]; ++je)
      for (int64_t ke = 0; ke < cells[2]; ++ke) {
        const int64_t eref = nd == 2 ? ie * cells[1] + je : (ie * cells[1] + je) * cells[2] + ke;
        int64_t eo[3];
        if (nd == 2) {
          eo[0] = je;
          eo[1] = ie;
        } else {
          eo[0] = je + cells[1] * ke;
          eo[1] = ie + cells[0] * ke;
          eo[2] = ie + cells[0] * je;
        }
        for (int node = 0; node < ND; ++node) {
          const int in = node % n, jn = (node / n) % n, kn = node / (n * n);
          if (ja)
            for (int a = 0; a < nd; ++a)
              for (int c = 0; c < nd; ++c)
                ja[((eref * ND + node) * nd + a) * nd + c] = mt.ja[a][c][eo[c] * ND + node];
          if (inv_j) {
            double det = mt.jdiag[0][ie * n + in];
            if (nd == 2) {
              det = det * mt.jdiag[1][je * n + jn];
            } else {
              det = det * (mt.jdiag[1][je * n + jn] * mt.jdiag[2][ke * n + kn]);
            }
            inv_j[eref * ND + node] = 1.0 / det;
          }
        }
      }
  return DGSEM_OK;
}

dgsem_status dgsem_coordinates_host(const dgsem_mesh_desc* mesh, double* coords) {
  if (!mesh || !coords || (mesh->ndims != 2 && mesh->ndims != 3)) return DGSEM_ERR_INVALID_ARG;
  BasisTables b;
  if (!make_basis(mesh->polydeg, &b)) return DGSEM_ERR_INVALID_ARG;
  MetricTablesHost mt;
  int64_t cells[3] = {1, 1, 1};
  for (int a = 0; a < mesh->ndims; ++a) cells[a] = mesh->n_cells[a];
  if (!make_metric_tables(b, mesh->ndims, cells, mesh->domain_left, mesh->domain_right, &mt))
    return DGSEM_ERR_INVALID_ARG;
  const int nd = mesh->ndims;
  const int n = b.n;
  const int ND = nd == 2 ? n * n : n * n * n;
  // reference logical order: cells (i slowest) x dof x dim
  for (int64_t ie = 0; ie < cells[0]; ++ie)
    for (int64_t je = 0; je < cells[1]; ++je)
      for (int64_t ke = 0; ke < cells[2]; ++ke) {
        const int64_t eref = nd == 2 ? ie * cells[1] + je : (ie * cells[1] + je) * cells[2] + ke;
        const int64_t ev[3] = {ie, je, ke};
        for (int node = 0; node < ND; ++node) {
          const int iv[3] = {node % n, (node / n) % n, node / (n * n)};
          for (int a = 0; a < nd; ++a)
            coords[(eref * ND + node) * nd + a] = mt.coord[a][ev[a] * n + iv[a]];
        }
      }
  return DGSEM_OK;
}

}  // extern "C"
