// Type-erased solver engine: one instantiation per supported template
// combination (dimension, nodes per direction, volume flux, surface flux,
// shock capturing, Navier-Stokes).  Each engine carries several launch shapes
// of the same fused kernel (elements per block, register cap); they compute
// bitwise-identical results and the autotuner (capi.cu: dgsem_autotune)
// picks the fastest for a mesh.  The C ABI context owns one engine.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <memory>
#include <utility>

#include "br1_kernel.cuh"
#include "stage_kernel.cuh"
#include "stage_node2_kernel.cuh"
#include "stage_node_kernel.cuh"
#include "stage_pipe_kernel.cuh"
#include "tables.hpp"

namespace dgsem {

// Everything an engine needs that does not depend on its template arguments.
struct EngineConfig {
  int ndims;
  int n;
  int64_t cells[3];
  int periodic[3];
  int64_t nelem;
  double gamma;
  double mu, prandtl;
  double alpha_max, alpha_min, atol;
  double hg_threshold, hg_s;
  DeviceTables tab;
  BcParams bc;
  BasisTables basis;
  unsigned int* nonfinite;  // device flag
  double* grad;             // Navier-Stokes lifted gradient [E][4][2][n^2]
  // per-element info (node_element_info layout, 12 ints per element) and
  // -1/J per node [E][n^d], computed once per context (may be null)
  const int* elem_info;
  const double* mij;
  // failure-path testing (StageArgs::wait_limit_ns / skip_tile_copy)
  unsigned long long wait_limit_ns;
  int skip_tile_copy;
};

// Launch-shape variants: 0-2 line-parallel (stage_kernel.cuh), 3-4
// node-parallel (stage_node_kernel.cuh), 5 persistent node-parallel with TMA
// tile streaming (stage_pipe_kernel.cuh; single-mesh launches; split form
// without shock capturing or viscous terms, an even number of doubles per
// element), 6 two nodes per thread (stage_node2_kernel.cuh; 3D, n = 2 or 4,
// split form without shock capturing or viscous terms).
constexpr int kNumVariants = 7;

class EngineBase {
 public:
  virtual ~EngineBase() = default;
  // out = a*u_n + b*u_in + c*RHS(u_in, t); alpha_out optional; diag
  // optional: per-block volume integrals of `out` (StageArgs::diag), as many
  // slots as diag_slots() returns.
  virtual cudaError_t stage(const EngineConfig& cfg, const double* u_n,
                            const double* u_in, double* out, double a, double b,
                            double c, double t, const double* t_dev,
                            double* alpha_out, cudaStream_t s, double* diag = nullptr) = 0;
  // number of diag slots (blocks) the last stage launch with diag wrote
  virtual int64_t last_diag_slots() const = 0;
  // Fills the per-mesh tables of the node-parallel kernels (EngineConfig::
  // elem_info / MeshView::info, 12 ints per element; ::mij, -1/J per node)
  // of the mesh `m` (its cells, periodicity, element count and metric
  // tables) on stream s.
  virtual cudaError_t build_mesh_tables(const MeshView& m, int* info, double* mij,
                                        cudaStream_t s) const = 0;
  // Batched launch over a tile list (mesh index and first element per block)
  // of meshes sharing this engine's scheme and degree; per-mesh data in
  // `meshes` (device array).  Tiles are built with elements_per_block().
  virtual cudaError_t batch_stage(const EngineConfig& cfg, const MeshView* meshes,
                                  const int* tile_mesh, const int* tile_e0, int ntiles,
                                  double a, double b, double t, const double* t_dev,
                                  cudaStream_t s) = 0;
  virtual int kernels_per_stage() const = 0;
  virtual int elements_per_block() const = 0;
  virtual int threads_per_block() const = 0;
  virtual size_t smem_bytes() const = 0;
  // launch-shape variant in [0, num_variants())
  virtual void set_variant(int v) = 0;
  virtual int variant() const = 0;
  virtual int num_variants() const = 0;
};

std::unique_ptr<EngineBase> make_engine(int ndims, int n, int vf, int sf,
                                        bool hg, bool ns);

// Nodal initial condition on one mesh (capi.cu).
cudaError_t launch_initial(int kind, int ndims, int n, const int64_t* cells, int64_t nelem,
                           const DeviceTables& tab, const BcParams& bc, double gamma,
                           const double* params, double* u, cudaStream_t s);

template <int N>
inline void fill_basis_const(const BasisTables& b, BasisConst<N>* out) {
  for (int i = 0; i < N; ++i) {
    for (int j = 0; j < N; ++j) {
      out->Dsplit[i][j] = b.Dsplit[i][j];
      out->Dhat[i][j] = b.Dhat[i][j];
      out->Vinv[i][j] = b.Vinv[i][j];
    }
    out->inv_w[i] = b.inv_weights[i];
    out->w[i] = b.weights[i];
  }
  out->lhat_l0 = b.lhat_left[0];
  out->lhat_rN = b.lhat_right[N - 1];
}

// The arguments of one stage launch that do not depend on the mesh.
template <int N>
inline StageArgs<N> stage_args_common(const EngineConfig& cfg, double a, double b, double t,
                                      const double* t_dev, double* alpha_out) {
  StageArgs<N> args{};
  args.a = a;
  args.b = b;
  args.t = t;
  args.t_dev = t_dev;
  args.gamma = cfg.gamma;
  args.inv_gm1 = 1.0 / (cfg.gamma - 1.0);
  args.alpha_max = cfg.alpha_max;
  args.alpha_min = cfg.alpha_min;
  args.atol = cfg.atol;
  args.hg_threshold = cfg.hg_threshold;
  args.hg_s = cfg.hg_s;
  args.alpha_out = alpha_out;
  args.nonfinite = cfg.nonfinite;
  args.grad = cfg.grad;
  args.mu = cfg.mu;
  args.kappa = cfg.gamma / ((cfg.gamma - 1.0) * cfg.prandtl);
  args.bc = cfg.bc;
  args.wait_limit_ns = cfg.wait_limit_ns;
  args.skip_tile_copy = cfg.skip_tile_copy;
  fill_basis_const<N>(cfg.basis, &args.basis);
  return args;
}

// Launch geometry per (DIM, N, variant): one thread per element line.
//   variant 0: ~128 (2D) / ~96 (3D) threads per block, no register cap
//   variant 1: same block, register cap for one more resident block per SM
//   variant 2: twice the elements per block, no register cap
template <int DIM, int N, int V>
struct LaunchShape {
  static constexpr int NLINE = DIM * ipow(N, DIM - 1);
  static constexpr int TARGET = DIM == 2 ? 128 : 96;
  static constexpr int EPB0 = (TARGET / NLINE) > 0 ? (TARGET / NLINE) : 1;
  static constexpr int EPB = V == 2 ? 2 * EPB0 : EPB0;
  static constexpr int NT = ((EPB * NLINE + 31) / 32) * 32;
  // variant 1 caps registers at 65536 / (MINB * NT) (about 100 per thread);
  // MINB = 0: no cap
  static constexpr int MINB = V == 1 ? (65536 / (NT * 100) > 1 ? 65536 / (NT * 100) : 2) : 0;
};

// Fraction of the lanes of its warps that a block of `threads` threads uses.
constexpr double lane_use(int threads) { return double(threads) / (((threads + 31) / 32) * 32); }

// Elements per block of the node-parallel shapes: 128 / n^d (about 128
// threads), unless that leaves more than 5 % of the block's warp lanes idle
// (n^d = 36, 49 in 2D; 27 in 3D); then the smallest count up to 256 threads
// that fills at least 95 % of them (a partly filled warp costs a whole
// warp's issue slots).
constexpr int node_elements_per_block(int nd) {
  const int e0 = 128 / nd > 0 ? 128 / nd : 1;
  if (lane_use(e0 * nd) >= 0.95) return e0;
  for (int e = e0 + 1; e * nd <= 256; ++e)
    if (lane_use(e * nd) >= 0.95) return e;
  return e0;
}

// Node-parallel variants: one thread per node; variant 3 caps registers at
// ~72 per thread (7 resident blocks of 128 threads), variant 4 leaves them to
// the compiler.
template <int DIM, int N>
struct NodeLaunch {
  static constexpr int ND = ipow(N, DIM);
  static constexpr int EPB = node_elements_per_block(ND);
  static constexpr int NT = EPB * ND;
  static constexpr int MINB = 65536 / (NT * 72) > 1 ? 65536 / (NT * 72) : 1;
};

// Launches a stage kernel with programmatic stream serialization: the GPU
// may schedule its blocks while the previous kernel on `s` drains (hiding the
// launch gap between the three stages of a step); the kernel's first
// instruction, griddepcontrol.wait (stage_dependency_sync), holds every block
// until that kernel has completed and flushed its writes.  After a copy, a
// memset or an event the launch is ordered as usual.
template <class... P, class... A>
void launch_stage_kernel(void (*kernel)(P...), unsigned grid, unsigned block, size_t smem,
                         cudaStream_t s, A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

template <int DIM, int N, int VF, int SF, bool HG, bool NS = false>
class Engine final : public EngineBase {
 public:
  static constexpr int GRAD_EPB = (128 / ipow(N, DIM)) > 0 ? (128 / ipow(N, DIM)) : 1;
  static constexpr bool kBatch = !NS && !HG;
  // the line-parallel shapes 0-2 carry shock capturing or the viscous terms
  // in 2D only (not both); otherwise the node-parallel shapes run (0-2 then
  // run shape 3)
  static constexpr bool kLine = !(DIM == 3 && (HG || NS)) && !(HG && NS);

  template <int V>
  using Sh = StageShape<DIM, N, VF, SF, HG, LaunchShape<DIM, N, V>::EPB, NS>;

  template <int V>
  static auto kernel() {
    using L = LaunchShape<DIM, N, V>;
    if constexpr (L::MINB == 0)
      return stage_kernel<DIM, N, VF, SF, HG, L::EPB, L::NT, NS, false>;
    else
      return stage_kernel_capped<DIM, N, VF, SF, HG, L::EPB, L::NT, NS, false, L::MINB>;
  }
  template <int V>
  static auto batch_kernel() {
    using L = LaunchShape<DIM, N, V>;
    if constexpr (L::MINB == 0)
      return stage_kernel<DIM, N, VF, SF, HG, L::EPB, L::NT, NS, true>;
    else
      return stage_kernel_capped<DIM, N, VF, SF, HG, L::EPB, L::NT, NS, true, L::MINB>;
  }

  template <int V>
  static void set_attributes() {
    if constexpr (kLine)
      cudaFuncSetAttribute(kernel<V>(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)Sh<V>::smem_bytes);
    if constexpr (kBatch)
      cudaFuncSetAttribute(batch_kernel<V>(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)Sh<V>::smem_bytes);
  }

  // node-parallel shapes: split form with shock capturing or with the
  // Navier-Stokes viscous terms; batched node launches with neither
  static constexpr bool kNode = true;
  using NL = NodeLaunch<DIM, N>;
  using NSh = NodeShape<DIM, N, VF, NL::EPB, HG, NS>;
  template <bool B, bool CAP>
  static auto node_kernel() {
    if constexpr (CAP)
      return stage_node_kernel_capped<DIM, N, VF, SF, NL::EPB, B, NL::MINB, HG, NS>;
    else
      return stage_node_kernel<DIM, N, VF, SF, NL::EPB, B, HG, NS>;
  }
  // launches without u_n (a == 0) request the smaller shared-memory size
  static size_t node_smem(const StageArgs<N>& args) {
    return args.a != 0.0 ? NSh::smem_bytes : NSh::smem_bytes_base;
  }
  template <bool CAP>
  void launch_node(const StageArgs<N>& args, int64_t nelem, cudaStream_t s) const {
    if constexpr (kNode) {
      const int64_t blocks = (nelem + NL::EPB - 1) / NL::EPB;
      last_grid_ = blocks;
      launch_stage_kernel(node_kernel<false, CAP>(), (unsigned)blocks, NL::NT, node_smem(args), s,
                          args);
    }
  }
  template <bool CAP>
  void launch_node_batch(const StageArgs<N>& args, int ntiles, cudaStream_t s) const {
    if constexpr (kBatch)
      launch_stage_kernel(node_kernel<true, CAP>(), (unsigned)ntiles, NL::NT, node_smem(args), s,
                          args);
  }

  // shape 6: two nodes per thread (3D, n = 2 or 4, split form)
  static constexpr bool kNode2 = DIM == 3 && (N == 2 || N == 4) && !HG && !NS;
  template <int NN = N>
  static auto node2_kernel() {
    return stage_node2_kernel<NN, VF, SF>;
  }
  void launch_node2(const StageArgs<N>& args, int64_t nelem, cudaStream_t s) const {
    if constexpr (kNode2) {
      using S2 = Node2Shape<N, VF>;
      const int64_t blocks = (nelem + Node2Launch<N>::EPB - 1) / Node2Launch<N>::EPB;
      last_grid_ = blocks;
      launch_stage_kernel(node2_kernel(), (unsigned)blocks, Node2Launch<N>::NT,
                          args.a != 0.0 ? S2::smem_bytes : S2::smem_bytes_base, s, args);
    } else {
      launch_node<true>(args, nelem, s);
    }
  }

  using PSh = PipeShape<DIM, N, VF, NL::EPB>;
  static constexpr bool kPipe = kBatch && PSh::kSupported;
  static auto pipe_kernel() {
    return stage_pipe_kernel<DIM, N, VF, SF, NL::EPB, PSh::MINB>;
  }
  // Persistent launch: as many blocks as fit on the device at once.  Falls
  // back to the node-parallel shape when a state pointer is not 16-byte
  // aligned (bulk copies need it).
  void launch_pipe(const StageArgs<N>& args, int64_t nelem, cudaStream_t s) const {
    if constexpr (kPipe) {
      const uintptr_t al = reinterpret_cast<uintptr_t>(args.mesh.u_in) |
                           reinterpret_cast<uintptr_t>(args.mesh.u_n);
      if (al & 15u) {
        launch_node<true>(args, nelem, s);
        return;
      }
      if (pipe_blocks_ == 0) {
        int dev = 0, nsm = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pipe_kernel(), PSh::NT,
                                                      PSh::smem_bytes);
        pipe_blocks_ = (nsm > 0 ? nsm : 1) * (per_sm > 0 ? per_sm : 1);
      }
      const int64_t ntiles = (nelem + NL::EPB - 1) / NL::EPB;
      const int64_t blocks = ntiles < pipe_blocks_ ? ntiles : pipe_blocks_;
      last_grid_ = blocks;
      launch_stage_kernel(pipe_kernel(), (unsigned)blocks, PSh::NT, PSh::smem_bytes, s, args,
                          (int)ntiles);
    } else {
      launch_node<true>(args, nelem, s);
    }
  }

  Engine() {
    set_attributes<0>();
    set_attributes<1>();
    set_attributes<2>();
    if constexpr (kNode) {
      const int sm = (int)NSh::smem_bytes;
      cudaFuncSetAttribute(node_kernel<false, true>(), cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
      cudaFuncSetAttribute(node_kernel<false, false>(), cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    }
    if constexpr (kBatch) {
      const int sm = (int)NSh::smem_bytes;
      cudaFuncSetAttribute(node_kernel<true, true>(), cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
      cudaFuncSetAttribute(node_kernel<true, false>(), cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    }
    if constexpr (kPipe)
      cudaFuncSetAttribute(pipe_kernel(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)PSh::smem_bytes);
    if constexpr (kNode2)
      cudaFuncSetAttribute(node2_kernel(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)Node2Shape<N, VF>::smem_bytes);
  }

  StageArgs<N> common_args(const EngineConfig& cfg, double a, double b, double t,
                           const double* t_dev, double* alpha_out) const {
    return stage_args_common<N>(cfg, a, b, t, t_dev, alpha_out);
  }

  template <int V>
  void launch(const StageArgs<N>& args, int64_t nelem, cudaStream_t s) const {
    if constexpr (!kLine) {
      launch_node<true>(args, nelem, s);
    } else {
      using L = LaunchShape<DIM, N, V>;
      const int64_t blocks = (nelem + L::EPB - 1) / L::EPB;
      last_grid_ = blocks;
      launch_stage_kernel(kernel<V>(), (unsigned)blocks, L::NT, Sh<V>::smem_bytes, s, args);
    }
  }

  cudaError_t stage(const EngineConfig& cfg, const double* u_n,
                    const double* u_in, double* out, double a, double b,
                    double c, double t, const double* t_dev,
                    double* alpha_out, cudaStream_t s, double* diag = nullptr) override {
    StageArgs<N> args = common_args(cfg, a, b, t, t_dev, alpha_out);
    args.diag = diag;
    args.mesh.u_in = u_in;
    args.mesh.u_n = u_n;
    args.mesh.out = out;
    args.mesh.c = c;
    for (int i = 0; i < 3; ++i) {
      args.mesh.cells[i] = (int)cfg.cells[i];
      args.mesh.periodic[i] = cfg.periodic[i];
    }
    args.mesh.nelem = (int)cfg.nelem;
    args.mesh.tab = cfg.tab;
    args.mesh.info = cfg.elem_info;
    args.mesh.mij = cfg.mij;
    if constexpr (NS) {
      GradArgs<N> ga{};
      ga.u = u_in;
      ga.grad = cfg.grad;
      for (int i = 0; i < 3; ++i) ga.cells[i] = cfg.cells[i];
      ga.nelem = cfg.nelem;
      ga.gamma = cfg.gamma;
      ga.tab = cfg.tab;
      ga.basis = args.basis;
      for (int d = 0; d < DIM; ++d) ga.periodic[d] = cfg.periodic[d];
      for (int f = 0; f < 2 * DIM; ++f) ga.bc_kind[f] = cfg.bc.kind[f];
      const int64_t gblocks = (cfg.nelem + GRAD_EPB - 1) / GRAD_EPB;
      if constexpr (DIM == 2)
        launch_stage_kernel(br1_gradient_kernel<N, GRAD_EPB>, (unsigned)gblocks, GRAD_EPB * N * N,
                            0, s, ga);
      else
        launch_stage_kernel(br1_gradient_kernel_3d<N, GRAD_EPB>, (unsigned)gblocks,
                            GRAD_EPB * N * N * N, 0, s, ga);
    }
    switch (variant_) {
      case 1: launch<1>(args, cfg.nelem, s); break;
      case 2: launch<2>(args, cfg.nelem, s); break;
      case 3: launch_node<true>(args, cfg.nelem, s); break;
      case 4: launch_node<false>(args, cfg.nelem, s); break;
      case 5: launch_pipe(args, cfg.nelem, s); break;
      case 6: launch_node2(args, cfg.nelem, s); break;
      default: launch<0>(args, cfg.nelem, s); break;
    }
    if (diag) last_diag_slots_ = last_grid_;
    return cudaGetLastError();
  }

  template <int V>
  void launch_batch(const StageArgs<N>& args, int ntiles, cudaStream_t s) const {
    if constexpr (kBatch) {
      using L = LaunchShape<DIM, N, V>;
      launch_stage_kernel(batch_kernel<V>(), (unsigned)ntiles, L::NT, Sh<V>::smem_bytes, s, args);
    }
  }

  cudaError_t batch_stage(const EngineConfig& cfg, const MeshView* meshes,
                          const int* tile_mesh, const int* tile_e0, int ntiles,
                          double a, double b, double t, const double* t_dev,
                          cudaStream_t s) override {
    if constexpr (!kBatch) {
      return cudaErrorNotSupported;
    } else {
      StageArgs<N> args = common_args(cfg, a, b, t, t_dev, nullptr);
      args.meshes = meshes;
      args.tile_mesh = tile_mesh;
      args.tile_e0 = tile_e0;
      switch (variant_) {
        case 1: launch_batch<1>(args, ntiles, s); break;
        case 2: launch_batch<2>(args, ntiles, s); break;
        case 3:
        case 5:
        case 6: launch_node_batch<true>(args, ntiles, s); break;
        case 4: launch_node_batch<false>(args, ntiles, s); break;
        default: launch_batch<0>(args, ntiles, s); break;
      }
      return cudaGetLastError();
    }
  }

  cudaError_t build_mesh_tables(const MeshView& m, int* info, double* mij,
                                cudaStream_t s) const override {
    const int64_t nodes = (int64_t)m.nelem * ipow(N, DIM);
    const unsigned blocks = (unsigned)std::min<int64_t>((nodes + 255) / 256, 4096);
    element_tables_kernel<DIM, N, 12><<<blocks, 256, 0, s>>>(m, info, mij);
    return cudaGetLastError();
  }

  int kernels_per_stage() const override { return NS ? 2 : 1; }
  int64_t last_diag_slots() const override { return last_diag_slots_; }
  int elements_per_block() const override {
    if constexpr (kNode2)
      if (variant_ == 6) return Node2Launch<N>::EPB;
    if (variant_ >= 3 || !kLine) return NL::EPB;
    return variant_ == 2 ? LaunchShape<DIM, N, 2>::EPB : LaunchShape<DIM, N, 0>::EPB;
  }
  int threads_per_block() const override {
    if (variant_ >= 3 || !kLine) return NL::NT;
    return variant_ == 2 ? LaunchShape<DIM, N, 2>::NT : LaunchShape<DIM, N, 0>::NT;
  }
  size_t smem_bytes() const override {
    if constexpr (kNode2)
      if (variant_ == 6) return Node2Shape<N, VF>::smem_bytes;
    if (variant_ >= 3 || !kLine) return NSh::smem_bytes;
    return variant_ == 2 ? Sh<2>::smem_bytes : Sh<0>::smem_bytes;
  }
  void set_variant(int v) override { variant_ = (v >= 0 && v < num_variants()) ? v : 0; }
  int variant() const override { return variant_; }
  // shapes 5 and 6 exist for single-mesh launches; batched launches run them as 3
  int num_variants() const override { return kNode2 ? 7 : kPipe ? 6 : kNode ? 5 : 3; }

 private:
  int variant_ = 0;
  mutable int64_t pipe_blocks_ = 0;
  mutable int64_t last_grid_ = 0;  // blocks of the last single-mesh stage launch
  int64_t last_diag_slots_ = 0;
};

}  // namespace dgsem
