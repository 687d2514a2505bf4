// mhy_csr.cu -- explicit cell -> node connectivity at the boundary.
//
// The reference walks Arcane's connectivity: cell -> nodes in the SN_trigo
// local order (cartesian/CartConnectivityCellNode.h:83-94), node -> cells in
// increasing cell id with the node's index in each cell (nodeIndexInCells,
// accenv/AccEnvDefaultService.cc:240-268).  The kernels here take a logically
// Cartesian block and derive every neighbour from (i, j, k), which costs no
// index traffic in HBM.  A caller that holds the mesh as explicit connectivity
// in its own numbering (an Arcane shim reading the mesh's item lists, or a
// mesh file) hands that connectivity over as CSR arrays; mhy_csr_structure
// recovers the block's dimensions and the two numbering maps on the host, and
// a context created with mhy_create_csr keeps the maps in HBM to move state in
// and fields out in the caller's numbering.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <vector>

#include "mhy_kernels.cuh"

namespace mhy {

// out[u] = src[idx[u]] for u < n (cell or node fields); with three
// components per item (xyz interleaved), out[3u + a] = src[3 idx[u] + a].
__global__ void k_gather_index(long long n, int comps, const int32_t* __restrict__ idx,
                               const double* __restrict__ src, double* __restrict__ out) {
  const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (u >= n) return;
  const long long s = idx[u];
  for (int a = 0; a < comps; ++a) out[comps * u + a] = src[comps * s + a];
}

}  // namespace mhy

namespace {

struct I3 { int64_t x, y, z; };
constexpr int kOff[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
constexpr int64_t kUnset = INT64_MIN;

}  // namespace

extern "C" int mhy_csr_structure(int64_t ncells, int64_t nnodes, const int64_t* offsets, const int64_t* cell_nodes,
                                 int32_t dims[3], int32_t* cell_index, int32_t* node_index) {
  if (ncells < 1 || nnodes < 8 || !offsets || !cell_nodes || !dims || !cell_index || !node_index) return MHY_ERR_ARG;
  if (ncells > (int64_t(1) << 31) / 24 || nnodes > (int64_t(1) << 31) / 5) return MHY_ERR_ARG;
  if (offsets[0] != 0) return MHY_ERR_ARG;
  for (int64_t c = 0; c < ncells; ++c)
    if (offsets[c + 1] - offsets[c] != 8) return MHY_ERR_UNSUPPORTED;            // hexahedra only
  for (int64_t e = 0; e < 8 * ncells; ++e)
    if (cell_nodes[e] < 0 || cell_nodes[e] >= nnodes) return MHY_ERR_ARG;
  // node -> cells (CSR)
  std::vector<int64_t> start(nnodes + 1, 0), list(8 * ncells);
  for (int64_t e = 0; e < 8 * ncells; ++e) ++start[cell_nodes[e] + 1];
  for (int64_t n = 0; n < nnodes; ++n) start[n + 1] += start[n];
  {
    std::vector<int64_t> fill(start.begin(), start.end() - 1);
    for (int64_t c = 0; c < ncells; ++c)
      for (int a = 0; a < 8; ++a) list[fill[cell_nodes[8 * c + a]]++] = c;
  }
  // Lattice positions: cell 0 at the origin, then every cell reached through
  // a shared node sits where that node's position minus its local offset
  // says; each cell's 8 nodes must land on its own 8 lattice corners.
  std::vector<I3> org(ncells, I3{kUnset, 0, 0}), pos(nnodes, I3{kUnset, 0, 0});
  std::vector<int64_t> queue;
  queue.reserve(ncells);
  org[0] = I3{0, 0, 0};
  queue.push_back(0);
  for (size_t q = 0; q < queue.size(); ++q) {
    const int64_t c = queue[q];
    for (int a = 0; a < 8; ++a) {
      const int64_t n = cell_nodes[8 * c + a];
      const I3 p{org[c].x + kOff[a][0], org[c].y + kOff[a][1], org[c].z + kOff[a][2]};
      if (pos[n].x == kUnset) pos[n] = p;
      else if (pos[n].x != p.x || pos[n].y != p.y || pos[n].z != p.z) return MHY_ERR_UNSUPPORTED;
      for (int64_t e = start[n]; e < start[n + 1]; ++e) {
        const int64_t d = list[e];
        if (org[d].x != kUnset) continue;
        int b = -1;
        for (int t = 0; t < 8; ++t)
          if (cell_nodes[8 * d + t] == n) { if (b >= 0) return MHY_ERR_UNSUPPORTED; b = t; }
        org[d] = I3{p.x - kOff[b][0], p.y - kOff[b][1], p.z - kOff[b][2]};
        queue.push_back(d);
      }
    }
  }
  if ((int64_t)queue.size() != ncells) return MHY_ERR_UNSUPPORTED;               // not one connected block
  I3 lo{INT64_MAX, INT64_MAX, INT64_MAX}, hi{INT64_MIN, INT64_MIN, INT64_MIN};
  for (int64_t c = 0; c < ncells; ++c) {
    lo.x = std::min(lo.x, org[c].x); lo.y = std::min(lo.y, org[c].y); lo.z = std::min(lo.z, org[c].z);
    hi.x = std::max(hi.x, org[c].x); hi.y = std::max(hi.y, org[c].y); hi.z = std::max(hi.z, org[c].z);
  }
  const int64_t nx = hi.x - lo.x + 1, ny = hi.y - lo.y + 1, nz = hi.z - lo.z + 1;
  if (nx > ncells || ny > ncells || nz > ncells || (double)nx * (double)ny * (double)nz != (double)ncells ||
      (nx + 1) * (ny + 1) * (nz + 1) != nnodes)
    return MHY_ERR_UNSUPPORTED;                                                   // not a full box of cells
  std::vector<char> seen_c(ncells, 0), seen_n(nnodes, 0);
  for (int64_t c = 0; c < ncells; ++c) {
    const int64_t s = (org[c].x - lo.x) + nx * ((org[c].y - lo.y) + ny * (org[c].z - lo.z));
    if (seen_c[s]) return MHY_ERR_UNSUPPORTED;
    seen_c[s] = 1;
    cell_index[c] = (int32_t)s;
  }
  for (int64_t n = 0; n < nnodes; ++n) {
    if (pos[n].x == kUnset) return MHY_ERR_UNSUPPORTED;                         // a node no cell uses
    const int64_t s = (pos[n].x - lo.x) + (nx + 1) * ((pos[n].y - lo.y) + (ny + 1) * (pos[n].z - lo.z));
    if (s < 0 || s >= nnodes || seen_n[s]) return MHY_ERR_UNSUPPORTED;
    seen_n[s] = 1;
    node_index[n] = (int32_t)s;
  }
  dims[0] = (int32_t)nx; dims[1] = (int32_t)ny; dims[2] = (int32_t)nz;
  return MHY_OK;
}
