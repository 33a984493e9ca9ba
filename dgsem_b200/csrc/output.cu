// On-disk output without VTK: the reference's VTU writer and a binary
// checkpoint / restart of the state.
//
// VTU (replaces VTUOutputObserver::write_vtu_2d/3d,
// observer/vtu_output_observer.hpp:65-235, and write_vtu_lagrange_quad/hex,
// observer/vtu_output_observer_impl.cpp:15-117): a VTK XML UnstructuredGrid
// with one Lagrange quadrilateral (cell type 70) or hexahedron (72) of order
// N per element, the element's nodes in VTK's Lagrange point order, the
// conserved variables and the pressure as point data (names as the
// reference's: rho, rhou, rhov[, rhow], rhoE, pressure), every array in one
// appended raw binary block (the reference's SetDataModeToAppended +
// EncodeAppendedDataOff), little endian, UInt64 block headers.  Elements are
// written in the device order e = ie + nx*(je + ny*ke), as the reference's
// writer does.
//
// Checkpoint: a fixed header (magic, format version, mesh and scheme
// descriptors, time, step, state length) followed by the state in the device
// layout u[e][var][node]; reading checks that the mesh and the state length
// match the context.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "context.hpp"
#include "dgsem_b200.h"
#include "tables.hpp"

namespace {

// VTK's Lagrange point index of node (i, j) of a quadrilateral of order p
// (the published ordering of vtkLagrangeQuadrilateral: vertices, then edge
// nodes edge by edge, then interior nodes row by row).
int vtk_quad_index(int i, int j, int p) {
  const bool ib = (i == 0 || i == p), jb = (j == 0 || j == p);
  const int nb = (ib ? 1 : 0) + (jb ? 1 : 0);
  if (nb == 2) return i ? (j ? 2 : 1) : (j ? 3 : 0);
  int off = 4;
  if (nb == 1) {
    if (!ib) return (i - 1) + (j ? (p - 1) + (p - 1) : 0) + off;
    return (j - 1) + (i ? (p - 1) : 2 * (p - 1) + (p - 1)) + off;
  }
  off += 2 * ((p - 1) + (p - 1));
  return off + (i - 1) + (p - 1) * (j - 1);
}

// VTK's Lagrange point index of node (i, j, k) of a hexahedron of order p
// (vtkLagrangeHexahedron: vertices, edges along i, j at k = 0 and k = p,
// edges along k, faces i = 0, p, j = 0, p, k = 0, p, then the interior).
int vtk_hex_index(int i, int j, int k, int p) {
  const bool ib = (i == 0 || i == p), jb = (j == 0 || j == p), kb = (k == 0 || k == p);
  const int nb = (ib ? 1 : 0) + (jb ? 1 : 0) + (kb ? 1 : 0);
  const int q = p - 1;
  if (nb == 3) return (i ? (j ? 2 : 1) : (j ? 3 : 0)) + (k ? 4 : 0);
  int off = 8;
  if (nb == 2) {
    if (!ib) return (i - 1) + (j ? 2 * q : 0) + (k ? 4 * q : 0) + off;
    if (!jb) return (j - 1) + (i ? q : 3 * q) + (k ? 4 * q : 0) + off;
    off += 8 * q;
    return (k - 1) + q * (i ? (j ? 3 : 1) : (j ? 2 : 0)) + off;
  }
  off += 12 * q;
  if (nb == 1) {
    if (ib) return (j - 1) + q * (k - 1) + (i ? q * q : 0) + off;
    off += 2 * q * q;
    if (jb) return (i - 1) + q * (k - 1) + (j ? q * q : 0) + off;
    off += 2 * q * q;
    return (i - 1) + q * (j - 1) + (k ? q * q : 0) + off;
  }
  off += 6 * q * q;
  return off + (i - 1) + q * ((j - 1) + q * (k - 1));
}

struct Block {
  const void* data;
  uint64_t bytes;
};

bool write_vtu_file(const char* path, int nd, int n, int64_t nelem, const std::vector<double>& pts,
                    const std::vector<std::vector<double>>& fields,
                    const std::vector<std::string>& names) {
  const int ndof = nd == 2 ? n * n : n * n * n;
  const int64_t npts = nelem * ndof;
  std::vector<int64_t> conn(npts), offs(nelem);
  std::vector<uint8_t> types(nelem, nd == 2 ? 70 : 72);
  for (int64_t i = 0; i < npts; ++i) conn[i] = i;
  for (int64_t e = 0; e < nelem; ++e) offs[e] = (e + 1) * ndof;
  std::vector<Block> blocks;
  for (const auto& f : fields) blocks.push_back({f.data(), f.size() * sizeof(double)});
  blocks.push_back({pts.data(), pts.size() * sizeof(double)});
  blocks.push_back({conn.data(), conn.size() * sizeof(int64_t)});
  blocks.push_back({offs.data(), offs.size() * sizeof(int64_t)});
  blocks.push_back({types.data(), types.size()});
  std::vector<uint64_t> at(blocks.size());
  uint64_t o = 0;
  for (size_t b = 0; b < blocks.size(); ++b) {
    at[b] = o;
    o += sizeof(uint64_t) + blocks[b].bytes;
  }
  FILE* fp = std::fopen(path, "wb");
  if (!fp) return false;
  std::string x;
  x += "<?xml version=\"1.0\"?>\n";
  x += "<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\" "
       "header_type=\"UInt64\">\n  <UnstructuredGrid>\n";
  x += "    <Piece NumberOfPoints=\"" + std::to_string(npts) + "\" NumberOfCells=\"" +
       std::to_string(nelem) + "\">\n      <PointData>\n";
  for (size_t f = 0; f < fields.size(); ++f)
    x += "        <DataArray type=\"Float64\" Name=\"" + names[f] +
         "\" format=\"appended\" offset=\"" + std::to_string(at[f]) + "\"/>\n";
  const size_t nf = fields.size();
  x += "      </PointData>\n      <Points>\n";
  x += "        <DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"appended\" "
       "offset=\"" + std::to_string(at[nf]) + "\"/>\n      </Points>\n      <Cells>\n";
  x += "        <DataArray type=\"Int64\" Name=\"connectivity\" format=\"appended\" offset=\"" +
       std::to_string(at[nf + 1]) + "\"/>\n";
  x += "        <DataArray type=\"Int64\" Name=\"offsets\" format=\"appended\" offset=\"" +
       std::to_string(at[nf + 2]) + "\"/>\n";
  x += "        <DataArray type=\"UInt8\" Name=\"types\" format=\"appended\" offset=\"" +
       std::to_string(at[nf + 3]) + "\"/>\n";
  x += "      </Cells>\n    </Piece>\n  </UnstructuredGrid>\n  <AppendedData encoding=\"raw\">\n   _";
  bool ok = std::fwrite(x.data(), 1, x.size(), fp) == x.size();
  for (const Block& b : blocks) {
    ok = ok && std::fwrite(&b.bytes, sizeof(uint64_t), 1, fp) == 1;
    ok = ok && std::fwrite(b.data, 1, b.bytes, fp) == b.bytes;
  }
  const char* tail = "\n  </AppendedData>\n</VTKFile>\n";
  ok = ok && std::fwrite(tail, 1, std::strlen(tail), fp) == std::strlen(tail);
  return std::fclose(fp) == 0 && ok;
}

// Point coordinates and fields of a state in the device layout (host copy).
dgsem_status vtu_from_state(const dgsem_mesh_desc* mesh, double gamma, const double* u,
                            const char* path) {
  using namespace dgsem;
  if (!mesh || !u || !path || (mesh->ndims != 2 && mesh->ndims != 3)) return DGSEM_ERR_INVALID_ARG;
  BasisTables b;
  if (!make_basis(mesh->polydeg, &b)) return DGSEM_ERR_INVALID_ARG;
  const int nd = mesh->ndims, n = b.n, p = n - 1, nv = nd + 2;
  int64_t cells[3] = {1, 1, 1};
  for (int a = 0; a < nd; ++a) cells[a] = mesh->n_cells[a];
  MetricTablesHost mt;
  if (!make_metric_tables(b, nd, cells, mesh->domain_left, mesh->domain_right, &mt))
    return DGSEM_ERR_INVALID_ARG;
  const int ndof = nd == 2 ? n * n : n * n * n;
  const int64_t nelem = cells[0] * cells[1] * cells[2];
  const int64_t npts = nelem * ndof;
  std::vector<double> pts(3 * npts, 0.0);
  std::vector<std::vector<double>> f(nv + 1, std::vector<double>(npts));
  for (int64_t e = 0; e < nelem; ++e) {
    const int64_t ev[3] = {e % cells[0], (e / cells[0]) % cells[1], e / (cells[0] * cells[1])};
    for (int node = 0; node < ndof; ++node) {
      const int iv[3] = {node % n, (node / n) % n, node / (n * n)};
      const int vid = nd == 2 ? vtk_quad_index(iv[0], iv[1], p)
                              : vtk_hex_index(iv[0], iv[1], iv[2], p);
      const int64_t g = e * ndof + vid;
      for (int a = 0; a < nd; ++a) pts[3 * g + a] = mt.coord[a][ev[a] * n + iv[a]];
      double c[5];
      for (int q = 0; q < nv; ++q) {
        c[q] = u[(e * nv + q) * ndof + node];
        f[q][g] = c[q];
      }
      double sq = 0.0;
      for (int d = 0; d < nd; ++d) sq += c[1 + d] * c[1 + d];
      f[nv][g] = (gamma - 1.0) * (c[nv - 1] - 0.5 * sq / c[0]);
    }
  }
  std::vector<std::string> names = nd == 2
      ? std::vector<std::string>{"rho", "rhou", "rhov", "rhoE", "pressure"}
      : std::vector<std::string>{"rho", "rhou", "rhov", "rhow", "rhoE", "pressure"};
  return write_vtu_file(path, nd, n, nelem, pts, f, names) ? DGSEM_OK : DGSEM_ERR_INVALID_ARG;
}

// ---------------------------------------------------------------------------
// checkpoint
// ---------------------------------------------------------------------------
constexpr char kMagic[8] = {'D', 'G', 'S', 'E', 'M', 'C', 'K', 'P'};
constexpr uint32_t kVersion = 1;

struct CheckpointHeader {
  char magic[8];
  uint32_t version;
  uint32_t header_bytes;
  dgsem_mesh_desc mesh;
  dgsem_scheme_desc scheme;
  double time;
  int64_t step;
  int64_t state_len;
};

int64_t state_len_of(const dgsem_mesh_desc* m) {
  const int n = m->polydeg + 1;
  int64_t e = 1;
  for (int a = 0; a < m->ndims; ++a) e *= m->n_cells[a];
  const int64_t nodes = m->ndims == 2 ? n * n : (int64_t)n * n * n;
  return e * nodes * (m->ndims + 2);
}

bool same_mesh(const dgsem_mesh_desc& a, const dgsem_mesh_desc& b) {
  if (a.ndims != b.ndims || a.polydeg != b.polydeg) return false;
  for (int i = 0; i < a.ndims; ++i)
    if (a.n_cells[i] != b.n_cells[i] || a.domain_left[i] != b.domain_left[i] ||
        a.domain_right[i] != b.domain_right[i])
      return false;
  return true;
}

}  // namespace

extern "C" {

dgsem_status dgsem_write_vtu_host(const dgsem_mesh_desc* mesh, double gamma, const double* u_host,
                                  const char* path) {
  if (!(gamma > 1.0)) return DGSEM_ERR_INVALID_ARG;
  return vtu_from_state(mesh, gamma, u_host, path);
}

dgsem_status dgsem_write_vtu(dgsem_ctx* ctx, const double* u, const char* path) {
  if (!ctx || !u || !path) return DGSEM_ERR_INVALID_ARG;
  std::vector<double> h(ctx->state_len);
  cudaError_t e = cudaMemcpyAsync(h.data(), u, h.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                  ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return DGSEM_ERR_CUDA;
  }
  return vtu_from_state(&ctx->mesh, ctx->scheme.gamma, h.data(), path);
}

dgsem_status dgsem_checkpoint_write_host(const dgsem_mesh_desc* mesh,
                                         const dgsem_scheme_desc* scheme, const double* u_host,
                                         double time, int64_t step, const char* path) {
  if (!mesh || !scheme || !u_host || !path) return DGSEM_ERR_INVALID_ARG;
  CheckpointHeader h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, kMagic, 8);
  h.version = kVersion;
  h.header_bytes = sizeof(CheckpointHeader);
  h.mesh = *mesh;
  h.scheme = *scheme;
  h.time = time;
  h.step = step;
  h.state_len = state_len_of(mesh);
  FILE* fp = std::fopen(path, "wb");
  if (!fp) return DGSEM_ERR_INVALID_ARG;
  bool ok = std::fwrite(&h, sizeof(h), 1, fp) == 1;
  ok = ok && std::fwrite(u_host, sizeof(double), h.state_len, fp) == (size_t)h.state_len;
  ok = (std::fclose(fp) == 0) && ok;
  return ok ? DGSEM_OK : DGSEM_ERR_INVALID_ARG;
}

dgsem_status dgsem_checkpoint_read_host(const dgsem_mesh_desc* mesh, double* u_host,
                                        double* time, int64_t* step, const char* path) {
  if (!mesh || !u_host || !path) return DGSEM_ERR_INVALID_ARG;
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return DGSEM_ERR_INVALID_ARG;
  CheckpointHeader h;
  bool ok = std::fread(&h, sizeof(h), 1, fp) == 1 && std::memcmp(h.magic, kMagic, 8) == 0 &&
            h.version == kVersion && h.header_bytes == sizeof(CheckpointHeader) &&
            same_mesh(h.mesh, *mesh) && h.state_len == state_len_of(mesh);
  ok = ok && std::fread(u_host, sizeof(double), h.state_len, fp) == (size_t)h.state_len;
  std::fclose(fp);
  if (!ok) return DGSEM_ERR_INVALID_ARG;
  if (time) *time = h.time;
  if (step) *step = h.step;
  return DGSEM_OK;
}

dgsem_status dgsem_checkpoint_write(dgsem_ctx* ctx, const double* u, double time, int64_t step,
                                    const char* path) {
  if (!ctx || !u || !path) return DGSEM_ERR_INVALID_ARG;
  std::vector<double> h(ctx->state_len);
  cudaError_t e = cudaMemcpyAsync(h.data(), u, h.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                  ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return DGSEM_ERR_CUDA;
  }
  return dgsem_checkpoint_write_host(&ctx->mesh, &ctx->scheme, h.data(), time, step, path);
}

dgsem_status dgsem_checkpoint_read(dgsem_ctx* ctx, double* u, double* time, int64_t* step,
                                   const char* path) {
  if (!ctx || !u || !path) return DGSEM_ERR_INVALID_ARG;
  std::vector<double> h(ctx->state_len);
  dgsem_status st = dgsem_checkpoint_read_host(&ctx->mesh, h.data(), time, step, path);
  if (st != DGSEM_OK) return st;
  cudaError_t e = cudaMemcpyAsync(u, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice,
                                  ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return DGSEM_ERR_CUDA;
  }
  return DGSEM_OK;
}

}  // extern "C"
