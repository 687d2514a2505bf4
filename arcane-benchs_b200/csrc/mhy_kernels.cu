// mhy_kernels.cu -- sm_100a initialisation kernels and the CFL dt reduction.
// Layout: structure of arrays in HBM, cells i-fastest, nodes i-fastest, faces
// X then Y then Z.  The cycle kernels are in mhy_cycle.cu.
#include "mhy_kernels.cuh"

namespace mhy {

// ------------------------------------------------------------------ init ----

// Initial geometry: cell centre, corner vectors, volume, characteristic length
// (MahycoAnnexe.cc:102-109, MahycoModule.cc:1054-1262 at t=0, :154-182).
__global__ void k_init_cells(Dims dm, const double* __restrict__ x0, double* __restrict__ xc0,
                             double* __restrict__ cqs, double* __restrict__ vol, double* __restrict__ L,
                             int lc_mode) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= dm.C) return;
  int i, j, k; dm.cijk(c, i, j, k);
  D3 x[8];
  for (int a = 0; a < 8; ++a) {
    long long n = dm.nid(i + kCellNodeOff[a][0], j + kCellNodeOff[a][1], k + kCellNodeOff[a][2]);
    x[a] = d3(x0[n], x0[dm.N + n], x0[2 * dm.N + n]);
  }
  D3 s = d3(0., 0., 0.);
  for (int a = 0; a < 8; ++a) s = s + x[a];
  D3 cc = 0.125 * s;
  if (xc0) { xc0[c] = cc.x; xc0[dm.C + c] = cc.y; xc0[2 * dm.C + c] = cc.z; }
  D3 fc[6], q[8];
  face_centres(x, fc);
  compute_cqs(x, fc, q);
  double v = 0;
  for (int a = 0; a < 8; ++a) {
    v += dot(x[a], q[a]);
    cqs[(a * 3 + 0) * dm.C + c] = q[a].x; cqs[(a * 3 + 1) * dm.C + c] = q[a].y; cqs[(a * 3 + 2) * dm.C + c] = q[a].z;
  }
  v *= 1. / 3;
  vol[c] = v;
  if (lc_mode == 0) L[c] = pow_third(v);
  else {
    double d1 = norm2(fc[0] - fc[3]), d2 = norm2(fc[2] - fc[5]), d3_ = norm2(fc[1] - fc[4]);
    L[c] = (d1 * d2 * d3_) / (d1 * d2 + d1 * d3_ + d2 * d3_);
  }
}

// Face normals and initial face centres, MahycoModule.cc:1013-1040.
__global__ void k_init_faces(Dims dm, const double* __restrict__ x0, double* __restrict__ n0,
                             double* __restrict__ xf0) {
  long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (f >= dm.F) return;
  int d; long long t;
  if (f < dm.Fx) { d = 0; t = f; } else if (f < dm.Fx + dm.Fy) { d = 1; t = f - dm.Fx; } else { d = 2; t = f - dm.Fx - dm.Fy; }
  int i, j, k; dm.fdijk(d, t, i, j, k);
  long long fn[4]; face_node_ids(dm, d, i, j, k, fn);
  D3 x[4];
  for (int a = 0; a < 4; ++a) x[a] = d3(x0[fn[a]], x0[dm.N + fn[a]], x0[2 * dm.N + fn[a]]);
  D3 v1 = x[2] - x[0], v2 = x[3] - x[1];
  D3 nn;
  nn.x = v1.y * v2.z - v1.z * v2.y;
  nn.y = -(v2.x * v1.z - v2.z * v1.x);
  nn.z = v1.x * v2.y - v1.y * v2.x;
  double nr = norm2(nn);
  n0[f] = nn.x / nr; n0[dm.F + f] = nn.y / nr; n0[2 * dm.F + f] = nn.z / nr;
  if (!xf0) return;
  D3 s = d3(0., 0., 0.);
  for (int a = 0; a < 4; ++a) s = s + 0.25 * x[a];
  xf0[f] = s.x; xf0[dm.F + f] = s.y; xf0[2 * dm.F + f] = s.z;
}

// Outer face normals (axis component only, the one the remap uses),
// MahycoModule.cc:1041-1048.  ofn[lf*C + c], local faces z-,x-,y-,z+,x+,y+.
// The initial cell and face centres are recomputed here from the node
// coordinates with the operations of k_init_cells and k_init_faces (the same
// bits), so the set-up needs no temporary arrays.
__global__ void k_init_outer_normals(Dims dm, const double* __restrict__ x0, double* __restrict__ ofn) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= dm.C) return;
  int i, j, k; dm.cijk(c, i, j, k);
  D3 s = d3(0., 0., 0.);
  for (int a = 0; a < 8; ++a) {
    const long long n = dm.nid(i + kCellNodeOff[a][0], j + kCellNodeOff[a][1], k + kCellNodeOff[a][2]);
    s = s + d3(x0[n], x0[dm.N + n], x0[2 * dm.N + n]);
  }
  const D3 cc = 0.125 * s;
  const int fd[6][4] = {{2, i, j, k}, {0, i, j, k}, {1, i, j, k}, {2, i, j, k + 1}, {0, i + 1, j, k}, {1, i, j + 1, k}};
  for (int a = 0; a < 6; ++a) {
    long long fn[4]; face_node_ids(dm, fd[a][0], fd[a][1], fd[a][2], fd[a][3], fn);
    D3 xf = d3(0., 0., 0.);
    for (int b = 0; b < 4; ++b) xf = xf + 0.25 * d3(x0[fn[b]], x0[dm.N + fn[b]], x0[2 * dm.N + fn[b]]);
    const D3 dv = xf - cc;
    const double nr = norm2(dv);
    ofn[a * dm.C + c] = comp(dv, fd[a][0]) / nr;
  }
}

// Initial thermodynamic state of a single-environment mesh: initEOS
// (PerfectGas E:20-32 or StiffenedGas) and ComputeCellMass (MahycoModule.cc:199-225).
__global__ void k_init_state(Dims dm, Phys ph, const double* __restrict__ vol, double* __restrict__ rho,
                             const double* __restrict__ pres, double* __restrict__ e, double* __restrict__ cs,
                             double* __restrict__ mass, double* __restrict__ q) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= dm.C) return;
  double p = pres[c], r = rho[c], ec, cc;
  eos_init(ph.eos, ph.gamma, ph.pinf, r, p, ec, cc);
  e[c] = ec;
  cs[c] = cc;
  mass[c] = r * vol[c];
  q[c] = 0.;
}

// ------------------------------------------------------------ set-up ----

// xyz-interleaved (n x 3) -> three planes (3 x n).
__global__ void k_fill_u32(long long n, uint32_t* __restrict__ a, uint32_t value) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) a[i] = value;
}

__global__ void k_soa3(long long n, const double* __restrict__ aos, double* __restrict__ soa) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  soa[i] = aos[3 * i]; soa[n + i] = aos[3 * i + 1]; soa[2 * n + i] = aos[3 * i + 2];
}

// Three planes (3 x n) -> xyz-interleaved (n x 3); with vh, the Lagrangian
// node coordinates of the last cycle, x0 + old_dt * v_half (MahycoModule.cc:
// 899-901), or x0 before the first cycle.
__global__ void k_aos3(long long n, const double* __restrict__ soa, const double* __restrict__ vh,
                       const Scalars* __restrict__ S, double* __restrict__ aos) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const bool lag = vh != nullptr && S->iteration > 0;
  const double dtu = lag ? S->old_dt : 0.0;
#pragma unroll
  for (int a = 0; a < 3; ++a) aos[3 * i + a] = lag ? soa[a * n + i] + vh[a * n + i] * dtu : soa[a * n + i];
}

// Maximum node coordinate per axis, from -1 as PrepareFaceGroup starts it
// (MahycoAnnexe.cc:189-199): per-block maxima, then one block over them.
// The maximum does not depend on the order in which it is taken.
__global__ void k_max3_partial(long long n, const double* __restrict__ x, double* __restrict__ part) {
  __shared__ double sm[3][256];
  double m[3] = {-1., -1., -1.};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    for (int a = 0; a < 3; ++a) m[a] = (m[a] < x[a * n + i]) ? x[a * n + i] : m[a];
  for (int a = 0; a < 3; ++a) sm[a][threadIdx.x] = m[a];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int a = 0; a < 3; ++a) sm[a][threadIdx.x] = (sm[a][threadIdx.x] < sm[a][threadIdx.x + w]) ? sm[a][threadIdx.x + w] : sm[a][threadIdx.x];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int a = 0; a < 3; ++a) part[3 * blockIdx.x + a] = sm[a][0];
}

// One thread: the maxima over the per-block maxima, in block order (the order
// in which every face thread used to take them), into out[0..2].
__global__ void k_max3_finish(const double* __restrict__ part, int nparts, double* __restrict__ out) {
  double mx[3] = {-1., -1., -1.};
  for (int b = 0; b < nparts; ++b)
    for (int a = 0; a < 3; ++a) mx[a] = (mx[a] < part[3 * b + a]) ? part[3 * b + a] : mx[a];
  for (int a = 0; a < 3; ++a) out[a] = mx[a];
}

// Boundary node groups by coordinate threshold over every face, PrepareFaceGroup
// (MahycoAnnexe.cc:183-251): bit s of grp[n] when the node belongs to a face
// lying on plane s (XMIN..ZMAX).  mx: the per-block maxima of k_max3_partial.
__global__ void k_face_groups(Dims dm, const double* __restrict__ x0, const double* __restrict__ part, int nparts,
                              double thr, unsigned* __restrict__ grp) {
  const long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (f >= dm.F) return;
  double mx[3] = {-1., -1., -1.};
  for (int b = 0; b < nparts; ++b)
    for (int a = 0; a < 3; ++a) mx[a] = (mx[a] < part[3 * b + a]) ? part[3 * b + a] : mx[a];
  int d; long long t;
  if (f < dm.Fx) { d = 0; t = f; } else if (f < dm.Fx + dm.Fy) { d = 1; t = f - dm.Fx; } else { d = 2; t = f - dm.Fx - dm.Fy; }
  int i, j, k; dm.fdijk(d, t, i, j, k);
  long long fn[4]; face_node_ids(dm, d, i, j, k, fn);
  unsigned fl = 0x3f;
  for (int a = 0; a < 4; ++a) {
    const double x = x0[fn[a]], y = x0[dm.N + fn[a]], z = x0[2 * dm.N + fn[a]];
    if (x > thr) fl &= ~(1u << MHY_XMIN);
    if (y > thr) fl &= ~(1u << MHY_YMIN);
    if (z > thr) fl &= ~(1u << MHY_ZMIN);
    if (fabs(x - mx[0]) > thr) fl &= ~(1u << MHY_XMAX);
    if (fabs(y - mx[1]) > thr) fl &= ~(1u << MHY_YMAX);
    if (fabs(z - mx[2]) > thr) fl &= ~(1u << MHY_ZMAX);
  }
  if (fl)
    for (int a = 0; a < 4; ++a) atomicOr(&grp[fn[a]], fl);
}

// bcmask bit b of a node: boundary condition b applies (its surface group holds the node).
__global__ void k_bc_mask(long long n, const unsigned* __restrict__ grp, int nbc, const int* __restrict__ surf,
                          uint16_t* __restrict__ mask) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned m = 0;
  for (int b = 0; b < nbc; ++b)
    if (grp[i] >> surf[b] & 1u) m |= 1u << b;
  mask[i] = (uint16_t)m;
}

// FP64 -> FP32 copy (the initial corner vectors of the mixed form).
__global__ void k_to_f32(long long n, const double* __restrict__ src, float* __restrict__ dst) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (float)src[i];
}

// Node mass = 1/8 sum of the cell masses, increasing cell id (MahycoModule.cc:235-266).
__global__ void k_node_mass(Dims dm, const double* __restrict__ mass, double* __restrict__ nm) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= dm.N) return;
  int i, j, k; dm.nijk(n, i, j, k);
  double s = 0.;
  for (int ck = k - 1; ck <= k; ++ck)
    for (int cj = j - 1; cj <= j; ++cj)
      for (int ci = i - 1; ci <= i; ++ci) {
        if (ci < 0 || cj < 0 || ck < 0 || ci >= dm.nx || cj >= dm.ny || ck >= dm.nz) continue;
        s += mass[dm.cid(ci, cj, ck)];
      }
  nm[n] = .125 * s;
}

// ------------------------------------------------------- conservation ----
// Conserved totals by compensated summation: every addition is Knuth's
// TwoSum (exact rounding error of s + x, accumulated in a second word), with
// a fixed grid and a fixed reduction tree, so the result is deterministic and
// its error does not grow with the number of terms.
struct Comp {
  double s, c;
  __device__ void add(double x) {
    const double t = s + x;
    const double bp = t - s;
    c += (s - (t - bp)) + (x - bp);
    s = t;
  }
  __device__ void merge(const Comp& o) { add(o.s); c += o.c; }
};

// part[6 * block + 2 q + {0, 1}] = (sum, compensation) of quantity q over this
// block's share: q = 0 cell mass, 1 cell internal energy m e, 2 node kinetic
// energy 0.5 m |v|^2.
__global__ void __launch_bounds__(kTotalsThreads) k_totals_partial(Dims dm, const double* __restrict__ mass,
    const double* __restrict__ e, const double* __restrict__ nm, const double* __restrict__ v,
    double* __restrict__ part) {
  __shared__ double sm[kTotalsThreads / 32][6];
  Comp q[3] = {{0., 0.}, {0., 0.}, {0., 0.}};
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < dm.C; c += stride) {
    const double m = mass[c];
    q[0].add(m);
    q[1].add(m * e[c]);
  }
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < dm.N; n += stride) {
    const double vx = v[n], vy = v[dm.N + n], vz = v[2 * dm.N + n];
    q[2].add(0.5 * nm[n] * ((vx * vx + vy * vy) + vz * vz));
  }
  for (int o = 16; o > 0; o >>= 1)
    for (int a = 0; a < 3; ++a) {
      Comp other{__shfl_down_sync(0xffffffffu, q[a].s, o), __shfl_down_sync(0xffffffffu, q[a].c, o)};
      q[a].merge(other);
    }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0)
    for (int a = 0; a < 3; ++a) { sm[w][2 * a] = q[a].s; sm[w][2 * a + 1] = q[a].c; }
  __syncthreads();
  if (threadIdx.x == 0) {
    Comp r[3] = {{0., 0.}, {0., 0.}, {0., 0.}};
    for (int ww = 0; ww < kTotalsThreads / 32; ++ww)
      for (int a = 0; a < 3; ++a) r[a].merge(Comp{sm[ww][2 * a], sm[ww][2 * a + 1]});
    for (int a = 0; a < 3; ++a) { part[6 * blockIdx.x + 2 * a] = r[a].s; part[6 * blockIdx.x + 2 * a + 1] = r[a].c; }
  }
}

// One thread: the block partials in block order; out[q] = sum + compensation.
__global__ void k_totals_finish(const double* __restrict__ part, int nparts, double* __restrict__ out) {
  Comp r[3] = {{0., 0.}, {0., 0.}, {0., 0.}};
  for (int b = 0; b < nparts; ++b)
    for (int a = 0; a < 3; ++a) r[a].merge(Comp{part[6 * b + 2 * a], part[6 * b + 2 * a + 1]});
  for (int a = 0; a < 3; ++a) out[a] = r[a].s + r[a].c;
}

// The dt reduction kernels; their bodies (dt_min_body, dt_finish_body) are in
// mhy_kernels.cuh so that the batched cycle can run them per instance.
__global__ void k_dt_min(Dims dm, Scalars* __restrict__ S, const double* __restrict__ L,
                         const double* __restrict__ cs, const double* __restrict__ vnorm, int linear) {
  dt_min_body(dm, S, L, cs, vnorm, blockIdx.x, linear ? -1 : (int)blockIdx.y, blockIdx.z);
}

__global__ void k_dt_finish(Scalars* S, Phys ph) { dt_finish_body(S, ph); }

// The dt of a slab decomposition: the minimum over all ranks' owned cells
// (combined by the caller) replaces the local one, then computeDeltaT as usual.
__global__ void k_dt_finish_ext(Scalars* S, Phys ph, const unsigned long long* __restrict__ min_bits) {
  S->min_bits = *min_bits;
  dt_finish_body(S, ph);
}

}  // namespace mhy
