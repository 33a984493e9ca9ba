// Batched mode: many independent periodic meshes (uneven element counts and
// polynomial degrees) advanced together.  Per stage, the meshes of each degree
// form one tile list and one launch of the fused stage kernel (each block
// reads its mesh view from a device table); the launches of the different
// degrees run concurrently on forked streams, which become parallel branches
// when the step is captured into a CUDA graph.  No reference counterpart
// (the reference advances one mesh per solver instance).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <new>
#include <vector>

#include "../../include/dgsem_b200.h"
#include "batch_persistent.hpp"
#include "engine.cuh"
#include "tables.hpp"

using namespace dgsem;

namespace {

struct Group {
  int n = 0;                      // nodes per direction
  std::unique_ptr<EngineBase> engine;
  EngineConfig cfg{};
  std::vector<int> members;       // mesh indices of this degree
  int ntiles = 0;
  size_t tile_capacity = 0;       // entries of tile_mesh / tile_e0
  int* tile_mesh = nullptr;       // device
  int* tile_e0 = nullptr;         // device
  cudaStream_t stream = nullptr;  // fork stream
  cudaEvent_t done = nullptr;
};

}  // namespace

struct dgsem_batch {
  int nmeshes = 0;
  int ndims = 2;
  dgsem_scheme_desc scheme{};
  std::vector<dgsem_mesh_desc> meshes;
  std::vector<int64_t> offsets;  // state offsets in doubles, nmeshes + 1
  std::vector<int64_t> nelem;
  std::vector<int> nodes;
  std::vector<DeviceTables> tabs;
  // per-mesh element info and -1/J tables of the node-parallel kernels
  std::vector<const int*> minfo;
  std::vector<const double*> mmij;
  std::vector<Group> groups;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<void*> allocations;
  double* tmp1 = nullptr;
  double* tmp2 = nullptr;
  double* tdev = nullptr;
  unsigned int* flag = nullptr;
  MeshView* views = nullptr;  // device [3 stages][nmeshes]
  std::vector<MeshView> views_host;
  const double* views_u = nullptr;  // key of the uploaded views
  std::vector<double> views_dt;
  int64_t launches = 0;
  // persistent mode: one launch per stage over all meshes (2D, LLF)
  bool persistent = false;
  bool persistent_ok = false;
  int* work = nullptr;  // device work list: (n << 24) | tile
  int nwork = 0;
  int* ptile_mesh[7] = {};  // per degree n = k + 2: tile lists of the persistent launch
  int* ptile_e0[7] = {};
  size_t psmem = 0;
  int pgrid = 0;
};

struct dgsem_batch_graph {
  dgsem_batch* batch = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int nsteps = 0;
  bool persistent = false;  // captured in persistent mode
};

namespace {

template <class T>
T* balloc(dgsem_batch* b, size_t count) {
  void* p = nullptr;
  if (cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) return nullptr;
  b->allocations.push_back(p);
  return static_cast<T*>(p);
}

void bfree(dgsem_batch* b) {
  for (Group& g : b->groups) {
    if (g.stream) cudaStreamDestroy(g.stream);
    if (g.done) cudaEventDestroy(g.done);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  for (void* p : b->allocations) cudaFree(p);
  b->allocations.clear();
}

dgsem_status st_of(cudaError_t e) { return e == cudaSuccess ? DGSEM_OK : DGSEM_ERR_CUDA; }

// (Re)builds a group's tile list for its engine's current launch shape.
cudaError_t build_tiles(const dgsem_batch* b, Group& g);

// Per-stage mesh views for state u (stages: u -> tmp1 -> tmp2 -> u) and the
// per-mesh time steps; uploaded only when u or dt changes.
dgsem_status upload_views(dgsem_batch* b, double* u, const double* dt) {
  bool same = b->views_u == u && (int)b->views_dt.size() == b->nmeshes;
  for (int m = 0; same && m < b->nmeshes; ++m) same = b->views_dt[m] == dt[m];
  if (same) return DGSEM_OK;
  const double fac[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};  // SSPRK3.hpp:162-180
  b->views_host.assign(3 * (size_t)b->nmeshes, MeshView{});
  for (int s = 0; s < 3; ++s)
    for (int m = 0; m < b->nmeshes; ++m) {
      MeshView& v = b->views_host[(size_t)s * b->nmeshes + m];
      const int64_t off = b->offsets[m];
      const double* ins[3] = {u, b->tmp1, b->tmp2};
      double* outs[3] = {b->tmp1, b->tmp2, u};
      v.u_in = ins[s] + off;
      v.u_n = u + off;
      v.out = outs[s] + off;
      v.c = fac[s] * dt[m];
      for (int a = 0; a < 3; ++a) {
        v.cells[a] = a < b->ndims ? (int)b->meshes[m].n_cells[a] : 1;
        v.periodic[a] = 1;
      }
      v.nelem = (int)b->nelem[m];
      v.tab = b->tabs[m];
      v.info = b->minfo[m];
      v.mij = b->mmij[m];
    }
  cudaError_t e = cudaMemcpyAsync(b->views, b->views_host.data(),
                                  b->views_host.size() * sizeof(MeshView),
                                  cudaMemcpyHostToDevice, b->stream);
  if (e != cudaSuccess) return DGSEM_ERR_CUDA;
  // the host copy must stay valid until the transfer is done
  e = cudaStreamSynchronize(b->stream);
  b->views_u = u;
  b->views_dt.assign(dt, dt + b->nmeshes);
  return st_of(e);
}

dgsem_status launch_stage(dgsem_batch* b, int stage, double t, const double* t_dev,
                          cudaStream_t main) {
  static const double A[3] = {0.0, 3.0 / 4.0, 1.0 / 3.0};
  static const double B[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
  static const double TOFF[3] = {0.0, 1.0, 0.5};  // fractions of dt (periodic: unused)
  (void)TOFF;
  const MeshView* views = b->views + (size_t)(stage - 1) * b->nmeshes;
  if (b->persistent) {
    PersistentDegree deg[7];
    for (const Group& g : b->groups) {
      PersistentDegree& d = deg[g.n - 2];
      d.cfg = &g.cfg;
      d.meshes = views;
      d.tile_mesh = b->ptile_mesh[g.n - 2];
      d.tile_e0 = b->ptile_e0[g.n - 2];
    }
    cudaError_t e = launch_persistent_stage(b->scheme.volume_flux, deg, b->work, b->nwork,
                                            A[stage - 1], B[stage - 1], t, t_dev, b->pgrid,
                                            b->psmem, main);
    b->launches++;
    return st_of(e);
  }
  if (cudaEventRecord(b->fork, main) != cudaSuccess) return DGSEM_ERR_CUDA;
  for (Group& g : b->groups) {
    if (cudaStreamWaitEvent(g.stream, b->fork, 0) != cudaSuccess) return DGSEM_ERR_CUDA;
    cudaError_t e = g.engine->batch_stage(g.cfg, views, g.tile_mesh, g.tile_e0, g.ntiles,
                                          A[stage - 1], B[stage - 1], t, t_dev, g.stream);
    if (e != cudaSuccess) return DGSEM_ERR_CUDA;
    if (cudaEventRecord(g.done, g.stream) != cudaSuccess) return DGSEM_ERR_CUDA;
    if (cudaStreamWaitEvent(main, g.done, 0) != cudaSuccess) return DGSEM_ERR_CUDA;
    b->launches++;
  }
  return DGSEM_OK;
}

// Work list of the persistent launch: every tile of every degree, higher
// degrees (costlier tiles) first, so that the blocks' round-robin walk ends
// with the cheap tiles.
cudaError_t build_persistent(dgsem_batch* b) {
  b->persistent_ok = persistent_supported(b->ndims, b->scheme.volume_flux,
                                          b->scheme.surface_flux);
  if (!b->persistent_ok) return cudaSuccess;
  std::vector<int> work;
  PersistentDegree deg[7];
  std::vector<Group*> order;
  for (Group& g : b->groups) order.push_back(&g);
  std::sort(order.begin(), order.end(), [](Group* x, Group* y) { return x->n > y->n; });
  for (Group* g : order) {
    const int k = g->n - 2;
    const int epb = persistent_elements_per_tile(g->n);
    std::vector<int> tm, te;
    for (int m : g->members)
      for (int64_t e0 = 0; e0 < b->nelem[m]; e0 += epb) {
        work.push_back((g->n << 24) | (int)tm.size());
        tm.push_back(m);
        te.push_back((int)e0);
      }
    b->ptile_mesh[k] = balloc<int>(b, tm.size());
    b->ptile_e0[k] = balloc<int>(b, te.size());
    if (!b->ptile_mesh[k] || !b->ptile_e0[k]) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMemcpy(b->ptile_mesh[k], tm.data(), tm.size() * sizeof(int),
                               cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(b->ptile_e0[k], te.data(), te.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return e;
    deg[k].cfg = &g->cfg;
  }
  b->nwork = (int)work.size();
  b->work = balloc<int>(b, work.size());
  if (!b->work) return cudaErrorMemoryAllocation;
  cudaError_t e = cudaMemcpy(b->work, work.data(), work.size() * sizeof(int),
                             cudaMemcpyHostToDevice);
  b->psmem = persistent_smem(b->scheme.volume_flux, deg);
  b->pgrid = persistent_grid(b->scheme.volume_flux, b->psmem);
  return e;
}

cudaError_t build_tiles(const dgsem_batch* b, Group& g) {
  const int epb = g.engine->elements_per_block();
  std::vector<int> tm, te;
  for (int m : g.members)
    for (int64_t e0 = 0; e0 < b->nelem[m]; e0 += epb) {
      tm.push_back(m);
      te.push_back((int)e0);
    }
  if (tm.size() > g.tile_capacity) return cudaErrorInvalidValue;
  g.ntiles = (int)tm.size();
  cudaError_t e = cudaMemcpy(g.tile_mesh, tm.data(), tm.size() * sizeof(int),
                             cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(g.tile_e0, te.data(), te.size() * sizeof(int), cudaMemcpyHostToDevice);
  return e;
}

}  // namespace

extern "C" {

dgsem_status dgsem_batch_autotune(dgsem_batch* b, double* u, const double* dt_host,
                                  int* chosen) {
  if (!b || !u || !dt_host) return DGSEM_ERR_INVALID_ARG;
  dgsem_status st = upload_views(b, u, dt_host);
  if (st != DGSEM_OK) return st;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // Rounds that each time every variant once, starting at a different
  // variant per round; the group keeps the variant with the smallest median.
  constexpr int rounds = 5;
  int gi = 0;
  for (Group& g : b->groups) {
    const int nv = g.engine->num_variants();
    std::vector<float> ms((size_t)rounds * nv, 0.f);
    // stage 1 writes tmp1 only, so repeated launches leave u untouched
    auto run = [&]() {
      return g.engine->batch_stage(g.cfg, b->views, g.tile_mesh, g.tile_e0, g.ntiles, 0.0,
                                   1.0, 0.0, nullptr, b->stream);
    };
    for (int r = 0; r < rounds && st == DGSEM_OK; ++r)
      for (int k = 0; k < nv && st == DGSEM_OK; ++k) {
        const int v = (r + k) % nv;
        g.engine->set_variant(v);
        if (build_tiles(b, g) != cudaSuccess || run() != cudaSuccess) {
          st = DGSEM_ERR_CUDA;
          break;
        }
        cudaEventRecord(e0, b->stream);
        for (int q = 0; q < 3 && st == DGSEM_OK; ++q)
          if (run() != cudaSuccess) st = DGSEM_ERR_CUDA;
        cudaEventRecord(e1, b->stream);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms[(size_t)r * nv + v], e0, e1);
      }
    int best = 0;
    float best_ms = 1e30f;
    for (int v = 0; v < nv; ++v) {
      float m[rounds];
      for (int r = 0; r < rounds; ++r) m[r] = ms[(size_t)r * nv + v];
      std::sort(m, m + rounds);
      if (m[rounds / 2] < best_ms) {
        best_ms = m[rounds / 2];
        best = v;
      }
    }
    g.engine->set_variant(best);
    if (st == DGSEM_OK && build_tiles(b, g) != cudaSuccess) st = DGSEM_ERR_CUDA;
    if (chosen) chosen[gi] = best;
    ++gi;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return st;
}

dgsem_status dgsem_batch_set_launch_variant(dgsem_batch* b, int variant) {
  if (!b) return DGSEM_ERR_INVALID_ARG;
  for (const Group& g : b->groups)
    if (variant < 0 || variant >= g.engine->num_variants()) return DGSEM_ERR_INVALID_ARG;
  for (Group& g : b->groups) {
    g.engine->set_variant(variant);
    if (build_tiles(b, g) != cudaSuccess) return DGSEM_ERR_CUDA;
  }
  return DGSEM_OK;
}

dgsem_status dgsem_batch_create(const dgsem_mesh_desc* meshes, int n_meshes,
                                const dgsem_scheme_desc* scheme, void* stream,
                                dgsem_batch** out) {
  if (!out || !meshes || !scheme || n_meshes < 1) return DGSEM_ERR_INVALID_ARG;
  *out = nullptr;
  const int nd = meshes[0].ndims;
  if (nd != 2 && nd != 3) return DGSEM_ERR_INVALID_ARG;
  if (scheme->equation != (nd == 2 ? DGSEM_EULER_2D : DGSEM_EULER_3D)) return DGSEM_ERR_UNSUPPORTED;
  if (scheme->volume_integral != DGSEM_VI_SPLIT_FORM) return DGSEM_ERR_UNSUPPORTED;
  for (int f = 0; f < 2 * nd; ++f)
    if (scheme->bc[f] != DGSEM_BC_PERIODIC) return DGSEM_ERR_UNSUPPORTED;
  if (!(scheme->gamma > 1.0)) return DGSEM_ERR_INVALID_ARG;
  for (int m = 0; m < n_meshes; ++m) {
    const dgsem_mesh_desc& d = meshes[m];
    if (d.ndims != nd) return DGSEM_ERR_INVALID_ARG;
    if (d.polydeg < 1 || d.polydeg + 1 > kMaxNodes) return DGSEM_ERR_UNSUPPORTED;
    int64_t ne = 1;
    for (int a = 0; a < nd; ++a) {
      if (d.n_cells[a] < 1 || !(d.domain_right[a] > d.domain_left[a])) return DGSEM_ERR_INVALID_ARG;
      ne *= d.n_cells[a];
    }
    if (ne > std::numeric_limits<int>::max() / 64) return DGSEM_ERR_INVALID_ARG;
  }
  dgsem_batch* b = new (std::nothrow) dgsem_batch();
  if (!b) return DGSEM_ERR_ALLOC;
  b->nmeshes = n_meshes;
  b->ndims = nd;
  b->scheme = *scheme;
  b->meshes.assign(meshes, meshes + n_meshes);
  b->stream = static_cast<cudaStream_t>(stream);
  // per-mesh sizes, tables and engines grouped by degree
  std::map<int, std::vector<int>> by_n;
  b->offsets.assign(n_meshes + 1, 0);
  std::vector<MetricTablesHost> mts(n_meshes);
  std::map<int, BasisTables> bases;
  size_t table_total = 0;
  for (int m = 0; m < n_meshes; ++m) {
    const dgsem_mesh_desc& d = meshes[m];
    const int n = d.polydeg + 1;
    if (!bases.count(n)) make_basis(d.polydeg, &bases[n]);
    int64_t cells[3] = {1, 1, 1}, ne = 1;
    for (int a = 0; a < nd; ++a) {
      cells[a] = d.n_cells[a];
      ne *= cells[a];
    }
    if (!make_metric_tables(bases[n], nd, cells, d.domain_left, d.domain_right, &mts[m])) {
      delete b;
      return DGSEM_ERR_INVALID_ARG;
    }
    const int nodes = nd == 2 ? n * n : n * n * n;
    b->nelem.push_back(ne);
    b->nodes.push_back(nodes);
    b->offsets[m + 1] = b->offsets[m] + ne * nodes * (nd + 2);
    by_n[n].push_back(m);
    for (int a = 0; a < nd; ++a) {
      table_total += mts[m].coord[a].size() + mts[m].jdiag[a].size();
      for (int c = 0; c < nd; ++c) table_total += mts[m].ja[a][c].size();
    }
  }
  double* tables = balloc<double>(b, table_total);
  const int64_t len = b->offsets[n_meshes];
  b->tmp1 = balloc<double>(b, len);
  b->tmp2 = balloc<double>(b, len);
  b->tdev = balloc<double>(b, 1);
  b->flag = balloc<unsigned int>(b, 1);
  b->views = balloc<MeshView>(b, 3 * (size_t)n_meshes);
  if (!tables || !b->tmp1 || !b->tmp2 || !b->tdev || !b->flag || !b->views) {
    bfree(b);
    delete b;
    return DGSEM_ERR_ALLOC;
  }
  cudaMemset(b->flag, 0, sizeof(unsigned int));
  std::vector<double> host(table_total);
  size_t off = 0;
  b->tabs.assign(n_meshes, DeviceTables{});
  auto place = [&](const std::vector<double>& v) -> const double* {
    const double* dptr = tables + off;
    std::memcpy(host.data() + off, v.data(), v.size() * sizeof(double));
    off += v.size();
    return dptr;
  };
  for (int m = 0; m < n_meshes; ++m)
    for (int a = 0; a < nd; ++a) {
      b->tabs[m].coord[a] = place(mts[m].coord[a]);
      b->tabs[m].jdiag[a] = place(mts[m].jdiag[a]);
      for (int c = 0; c < nd; ++c) b->tabs[m].ja[a][c] = place(mts[m].ja[a][c]);
    }
  cudaError_t e = cudaMemcpy(tables, host.data(), table_total * sizeof(double),
                             cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  const double eps = std::numeric_limits<double>::epsilon();
  for (auto& kv : by_n) {
    Group g;
    g.n = kv.first;
    try {
      g.engine = make_engine(nd, g.n, scheme->volume_flux, scheme->surface_flux, false, false);
    } catch (...) {
      g.engine = nullptr;
    }
    if (!g.engine) {
      bfree(b);
      delete b;
      return DGSEM_ERR_UNSUPPORTED;
    }
    EngineConfig& c = g.cfg;
    c.ndims = nd;
    c.n = g.n;
    c.gamma = scheme->gamma;
    c.mu = 0.0;
    c.prandtl = 0.72;
    c.alpha_max = scheme->alpha_max;
    c.alpha_min = scheme->alpha_min;
    c.atol = std::max(100.0 * eps, std::pow(eps, 0.75));
    c.basis = bases[g.n];
    c.nonfinite = b->flag;
    c.grad = nullptr;
    c.elem_info = nullptr;  // batched launches take the tables from the mesh views
    c.mij = nullptr;
    for (int f = 0; f < 6; ++f) c.bc.kind[f] = 0;
    g.members = kv.second;
    // tile arrays sized for one element per tile (any launch shape fits)
    g.engine->set_variant(0);
    size_t max_tiles = 0;
    for (int m : g.members) max_tiles += (size_t)b->nelem[m];
    g.tile_capacity = max_tiles;
    g.tile_mesh = balloc<int>(b, max_tiles);
    g.tile_e0 = balloc<int>(b, max_tiles);
    if (!g.tile_mesh || !g.tile_e0) {
      bfree(b);
      delete b;
      return DGSEM_ERR_ALLOC;
    }
    if (e == cudaSuccess) e = build_tiles(b, g);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming);
    b->groups.push_back(std::move(g));
  }
  // per-mesh element info and -1/J tables, built by the mesh's degree engine
  if (e == cudaSuccess) {
    int64_t nel_total = 0, nodes_total = 0;
    for (int m = 0; m < n_meshes; ++m) {
      nel_total += b->nelem[m];
      nodes_total += b->nelem[m] * b->nodes[m];
    }
    int* info = balloc<int>(b, (size_t)nel_total * 12);
    double* mij = info ? balloc<double>(b, (size_t)nodes_total) : nullptr;
    if (!mij) {
      bfree(b);
      delete b;
      return DGSEM_ERR_ALLOC;
    }
    b->minfo.assign(n_meshes, nullptr);
    b->mmij.assign(n_meshes, nullptr);
    int64_t io = 0, mo = 0;
    for (const Group& g : b->groups)
      for (int m : g.members) {
        MeshView v{};
        for (int a = 0; a < 3; ++a) {
          v.cells[a] = a < nd ? (int)meshes[m].n_cells[a] : 1;
          v.periodic[a] = 1;
        }
        v.nelem = (int)b->nelem[m];
        v.tab = b->tabs[m];
        if (e == cudaSuccess) e = g.engine->build_mesh_tables(v, info + io, mij + mo, nullptr);
        b->minfo[m] = info + io;
        b->mmij[m] = mij + mo;
        io += b->nelem[m] * 12;
        mo += b->nelem[m] * b->nodes[m];
      }
  }
  if (e == cudaSuccess) e = build_persistent(b);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    bfree(b);
    delete b;
    return DGSEM_ERR_CUDA;
  }
  *out = b;
  return DGSEM_OK;
}

dgsem_status dgsem_batch_destroy(dgsem_batch* b) {
  if (!b) return DGSEM_ERR_INVALID_ARG;
  cudaDeviceSynchronize();
  bfree(b);
  delete b;
  return DGSEM_OK;
}

dgsem_status dgsem_batch_offsets(const dgsem_batch* b, int64_t* offsets) {
  if (!b || !offsets) return DGSEM_ERR_INVALID_ARG;
  for (int m = 0; m <= b->nmeshes; ++m) offsets[m] = b->offsets[m];
  return DGSEM_OK;
}

dgsem_status dgsem_batch_initial_condition(dgsem_batch* b, int kind, const double* params,
                                          double* u) {
  if (!b || !u || kind < 0 || kind > 4) return DGSEM_ERR_INVALID_ARG;
  if ((kind == DGSEM_IC_TAYLOR_GREEN_3D) != (b->ndims == 3)) return DGSEM_ERR_INVALID_ARG;
  BcParams bc{};
  for (int m = 0; m < b->nmeshes; ++m) {
    int64_t cells[3] = {1, 1, 1};
    for (int a = 0; a < b->ndims; ++a) cells[a] = b->meshes[m].n_cells[a];
    cudaError_t e = launch_initial(kind, b->ndims, b->meshes[m].polydeg + 1, cells, b->nelem[m],
                                   b->tabs[m], bc, b->scheme.gamma,
                                   params ? params + 3 * m : nullptr, u + b->offsets[m], b->stream);
    if (e != cudaSuccess) return DGSEM_ERR_CUDA;
  }
  return DGSEM_OK;
}

dgsem_status dgsem_batch_ssprk3_step(dgsem_batch* b, double* u, double t,
                                     const double* dt_host) {
  if (!b || !u || !dt_host) return DGSEM_ERR_INVALID_ARG;
  dgsem_status st = upload_views(b, u, dt_host);
  for (int s = 1; s <= 3 && st == DGSEM_OK; ++s) st = launch_stage(b, s, t, nullptr, b->stream);
  return st;
}

dgsem_status dgsem_batch_graph_create(dgsem_batch* b, double* u, const double* dt_host,
                                      int nsteps, dgsem_batch_graph** out) {
  if (!b || !u || !dt_host || !out || nsteps < 1) return DGSEM_ERR_INVALID_ARG;
  *out = nullptr;
  dgsem_status st = upload_views(b, u, dt_host);
  if (st != DGSEM_OK) return st;
  cudaStream_t cap;
  if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess) return DGSEM_ERR_CUDA;
  dgsem_batch_graph* g = new (std::nothrow) dgsem_batch_graph();
  if (!g) {
    cudaStreamDestroy(cap);
    return DGSEM_ERR_ALLOC;
  }
  g->batch = b;
  g->nsteps = nsteps;
  g->persistent = b->persistent;
  cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    for (int s = 0; s < nsteps && st == DGSEM_OK; ++s)
      for (int k = 1; k <= 3 && st == DGSEM_OK; ++k)
        st = launch_stage(b, k, 0.0, b->tdev, cap);
    cudaError_t e2 = cudaStreamEndCapture(cap, &g->graph);
    if (st == DGSEM_OK && e2 != cudaSuccess) st = DGSEM_ERR_CUDA;
  } else {
    st = DGSEM_ERR_CUDA;
  }
  if (st == DGSEM_OK && cudaGraphInstantiate(&g->exec, g->graph, 0) != cudaSuccess)
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

dgsem_status dgsem_batch_graph_launch(dgsem_batch_graph* g) {
  if (!g || !g->exec) return DGSEM_ERR_INVALID_ARG;
  g->batch->launches +=
      3 * (int64_t)g->nsteps * (g->persistent ? 1 : (int64_t)g->batch->groups.size());
  return st_of(cudaGraphLaunch(g->exec, g->batch->stream));
}

dgsem_status dgsem_batch_graph_destroy(dgsem_batch_graph* g) {
  if (!g) return DGSEM_ERR_INVALID_ARG;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return DGSEM_OK;
}

dgsem_status dgsem_batch_check_finite(dgsem_batch* b) {
  if (!b) return DGSEM_ERR_INVALID_ARG;
  unsigned int h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, b->flag, sizeof(h), cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return DGSEM_ERR_CUDA;
  if (h) {
    cudaMemsetAsync(b->flag, 0, sizeof(unsigned int), b->stream);
    cudaStreamSynchronize(b->stream);
    return DGSEM_ERR_NONFINITE;
  }
  return DGSEM_OK;
}

dgsem_status dgsem_batch_set_persistent(dgsem_batch* b, int enable) {
  if (!b) return DGSEM_ERR_INVALID_ARG;
  if (enable && !b->persistent_ok) return DGSEM_ERR_UNSUPPORTED;
  b->persistent = enable != 0;
  return DGSEM_OK;
}

dgsem_status dgsem_batch_launch_count(const dgsem_batch* b, int64_t* count) {
  if (!b || !count) return DGSEM_ERR_INVALID_ARG;
  *count = b->launches;
  return DGSEM_OK;
}

}  // extern "C"
