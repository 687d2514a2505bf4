// mhy_kernels.cu -- sm_100a kernels of the Lagrange + ADI-remap cycle (single
// environment, plain FP64).  Layout: structure of arrays in HBM, cells
// i-fastest, nodes i-fastest, faces X then Y then Z.  Kernels are launched on
// the context stream by mhy_capi.cu, which also captures one cycle in a CUDA graph.
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
  xc0[c] = cc.x; xc0[dm.C + c] = cc.y; xc0[2 * dm.C + c] = cc.z;
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
  D3 s = d3(0., 0., 0.);
  for (int a = 0; a < 4; ++a) s = s + 0.25 * x[a];
  xf0[f] = s.x; xf0[dm.F + f] = s.y; xf0[2 * dm.F + f] = s.z;
}

// Outer face normals (axis component only, the one the remap uses),
// MahycoModule.cc:1041-1048.  ofn[lf*C + c], local faces z-,x-,y-,z+,x+,y+.
__global__ void k_init_outer_normals(Dims dm, const double* __restrict__ xc0, const double* __restrict__ xf0,
                                     double* __restrict__ ofn) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= dm.C) return;
  int i, j, k; dm.cijk(c, i, j, k);
  const long long cf[6] = {dm.fid(2, i, j, k), dm.fid(0, i, j, k), dm.fid(1, i, j, k),
                           dm.fid(2, i, j, k + 1), dm.fid(0, i + 1, j, k), dm.fid(1, i, j + 1, k)};
  const int ax[6] = {2, 0, 1, 2, 0, 1};
  D3 cc = d3(xc0[c], xc0[dm.C + c], xc0[2 * dm.C + c]);
  for (int a = 0; a < 6; ++a) {
    long long f = cf[a];
    D3 dv = d3(xf0[f], xf0[dm.F + f], xf0[2 * dm.F + f]) - cc;
    double nr = norm2(dv);
    ofn[a * dm.C + c] = comp(dv, ax[a]) / nr;
  }
}

// Initial thermodynamic state of a single-environment mesh: PerfectGas
// initEOS (E:20-32) and ComputeCellMass (MahycoModule.cc:199-225).
__global__ void k_init_state(Dims dm, double gamma, const double* __restrict__ vol, double* __restrict__ rho,
                             const double* __restrict__ pres, double* __restrict__ e, double* __restrict__ cs,
                             double* __restrict__ mass, double* __restrict__ q) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= dm.C) return;
  double p = pres[c], r = rho[c];
  e[c] = p / ((gamma - 1.) * r);
  cs[c] = sqrt(gamma * p / r);
  mass[c] = r * vol[c];
  q[c] = 0.;
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

// ---------------------------------------------------------------- cycle ----

// SaveValuesAtN + UpdateVelocity + ApplyBoundaryCondition + UpdatePosition for
// the nodes (MahycoModule.cc:308-450, 589-665, 936-1004, 870-902), and the
// dual remap variables of PrepareRemap.cc:402-434.
__global__ void k_lagrange_nodes(Dims dm, const Scalars* __restrict__ S, const double* __restrict__ p,
                                 const double* __restrict__ q, const double* __restrict__ cqs,
                                 const double* __restrict__ nm, const double* __restrict__ v,
                                 const double* __restrict__ x0, const uint16_t* __restrict__ bcmask, BCTable bct,
                                 double* __restrict__ vh, double* __restrict__ xl, double* __restrict__ ud,
                                 double* __restrict__ phid) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= dm.N) return;
  int i, j, k; dm.nijk(n, i, j, k);
  const double dt = S->dt;
  const double dtv = 0.5 * (S->old_dt + dt);
  // local index of the node in the cell (i-ci, j-cj, k-ck)
  const int loc[2][2][2] = {{{0, 4}, {3, 7}}, {{1, 5}, {2, 6}}};
  D3 F = d3(0, 0, 0);
  for (int ck = k - 1; ck <= k; ++ck)
    for (int cj = j - 1; cj <= j; ++cj)
      for (int ci = i - 1; ci <= i; ++ci) {
        if (ci < 0 || cj < 0 || ck < 0 || ci >= dm.nx || cj >= dm.ny || ck >= dm.nz) continue;
        long long c = dm.cid(ci, cj, ck);
        int l = loc[i - ci][j - cj][k - ck];
        double pq = p[c] + q[c];
        F = F + pq * d3(cqs[(l * 3 + 0) * dm.C + c], cqs[(l * 3 + 1) * dm.C + c], cqs[(l * 3 + 2) * dm.C + c]);
      }
  const double m = nm[n];
  const double s = dtv / m;
  D3 u = d3(v[n], v[dm.N + n], v[2 * dm.N + n]) + s * F;
  const unsigned mask = bcmask[n];
  for (int b = 0; b < bct.nb; ++b)
    if (mask >> b & 1u) {
      if (bct.type[b] == 0) u.x = bct.value[b];
      else if (bct.type[b] == 1) u.y = bct.value[b];
      else u.z = bct.value[b];
    }
  vh[n] = u.x; vh[dm.N + n] = u.y; vh[2 * dm.N + n] = u.z;
  D3 xx = d3(x0[n], x0[dm.N + n], x0[2 * dm.N + n]) + dt * u;
  xl[n] = xx.x; xl[dm.N + n] = xx.y; xl[2 * dm.N + n] = xx.z;
  const double un = norm2(u);
  ud[n] = m * u.x; ud[dm.N + n] = m * u.y; ud[2 * dm.N + n] = m * u.z; ud[3 * dm.N + n] = m;
  ud[4 * dm.N + n] = 0.5 * m * un;
  phid[n] = u.x; phid[dm.N + n] = u.y; phid[2 * dm.N + n] = u.z; phid[3 * dm.N + n] = 0.5 * un;
}

// ComputeGeometricValues + UpdateDensity + ComputeArtificialViscosity +
// UpdateEnergyAndPressure for single-environment cells, then the cell remap
// variables U = (V, V rho, V rho e, V q) (MahycoModule.cc:1054-1262,
// 1331-1370, 517-528, 1715-1726; PrepareRemap.cc:311-332).
__global__ void k_lagrange_cells(Dims dm, const Scalars* __restrict__ S, Phys ph, const double* __restrict__ xl,
                                 const double* __restrict__ rho, const double* __restrict__ e,
                                 const double* __restrict__ q, const double* __restrict__ p,
                                 const double* __restrict__ cs, const double* __restrict__ mass,
                                 double* __restrict__ cqs, double* __restrict__ xc, double* __restrict__ L,
                                 double* __restrict__ U) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= dm.C) return;
  int i, j, k; dm.cijk(c, i, j, k);
  D3 x[8];
  for (int a = 0; a < 8; ++a) {
    long long n = dm.nid(i + kCellNodeOff[a][0], j + kCellNodeOff[a][1], k + kCellNodeOff[a][2]);
    x[a] = d3(xl[n], xl[dm.N + n], xl[2 * dm.N + n]);
  }
  D3 s = d3(0., 0., 0.);
  for (int a = 0; a < 8; ++a) s = s + x[a];
  D3 cc = .125 * s;
  xc[c] = cc.x; xc[dm.C + c] = cc.y; xc[2 * dm.C + c] = cc.z;
  D3 fc[6], qv[8];
  face_centres(x, fc);
  compute_cqs(x, fc, qv);
  double V = 0;
  for (int a = 0; a < 8; ++a) {
    V += dot(x[a], qv[a]);
    cqs[(a * 3 + 0) * dm.C + c] = qv[a].x; cqs[(a * 3 + 1) * dm.C + c] = qv[a].y; cqs[(a * 3 + 2) * dm.C + c] = qv[a].z;
  }
  V *= 1. / 3;
  double Lc;
  if (ph.lc_mode == 0) Lc = pow_third(V);
  else {
    double d1 = norm2(fc[0] - fc[3]), d2 = norm2(fc[2] - fc[5]), d3_ = norm2(fc[1] - fc[4]);
    Lc = (d1 * d2 * d3_) / (d1 * d2 + d1 * d3_ + d2 * d3_);
  }
  L[c] = Lc;
  const double dt = S->dt;
  const double inv_deltat = 1.0 / dt;
  const double rn = rho[c];
  const double nd = mass[c] / V;
  const double tau = 0.5 * (1.0 / rn + 1.0 / nd);
  const double du = inv_deltat * (1.0 / nd - 1.0 / rn) / tau;
  double qn = 0.;
  const double g = ph.gamma;
  if (du < 0.0) qn = 1. / tau * (-0.5 * Lc * cs[c] * du + (g + 1) / 2.0 * Lc * Lc * du * du);
  const double en = compute_eint(ph.pseudo_centree != 0, g, q[c], qn, rn, nd, p[c], e[c]);
  U[c] = V;
  U[dm.C + c] = V * nd;
  U[2 * dm.C + c] = V * nd * en;
  U[3 * dm.C + c] = V * qn;
}

// Face quantities of the Lagrangian mesh, PrepareRemap.cc:33-55 and :93-117:
// |A| component along the face axis, face centre, normal velocity.
__global__ void k_faces(Dims dm, const double* __restrict__ xl, const double* __restrict__ vh,
                        const double* __restrict__ n0, double* __restrict__ A, double* __restrict__ uf,
                        double* __restrict__ xf) {
  long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (f >= dm.F) return;
  int d; long long t;
  if (f < dm.Fx) { d = 0; t = f; } else if (f < dm.Fx + dm.Fy) { d = 1; t = f - dm.Fx; } else { d = 2; t = f - dm.Fx - dm.Fy; }
  int i, j, k; dm.fdijk(d, t, i, j, k);
  long long fn[4]; face_node_ids(dm, d, i, j, k, fn);
  D3 x[4], w[4];
  for (int a = 0; a < 4; ++a) {
    x[a] = d3(xl[fn[a]], xl[dm.N + fn[a]], xl[2 * dm.N + fn[a]]);
    w[a] = d3(vh[fn[a]], vh[dm.N + fn[a]], vh[2 * dm.N + fn[a]]);
  }
  D3 cr = 0.5 * cross(x[2] - x[0], x[3] - x[1]);
  A[f] = fabs(comp(cr, d));
  D3 vm = d3(0., 0., 0.), fcn = d3(0., 0., 0.);
  for (int a = 0; a < 4; ++a) { fcn = fcn + .25 * x[a]; vm = vm + w[a]; }
  xf[f] = fcn.x; xf[dm.F + f] = fcn.y; xf[2 * dm.F + f] = fcn.z;
  uf[f] = dot(.25 * vm, d3(n0[f], n0[dm.F + f], n0[2 * dm.F + f]));
}

// --- directional sweep d (RemapADIService.cc:91-1040) ---

// computeGradPhiFace on the inner faces of d (R:163-178): dx_f and face gradients
// of Phi = U / sum(U volumes).
__global__ void k_sweep_face_grad(Dims dm, int d, const double* __restrict__ xc, const double* __restrict__ n0,
                                  const double* __restrict__ U, double* __restrict__ dxf, double* __restrict__ gf) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= dm.nfd(d)) return;
  int i, j, k; dm.fdijk(d, t, i, j, k);
  int id = d == 0 ? i : (d == 1 ? j : k);
  if (id == 0 || id == dm.ncd(d)) return;           // boundary face
  long long f = dm.fid(d, i, j, k);
  long long nc = dm.cid(i, j, k);
  long long pc = dm.cid(i - (d == 0), j - (d == 1), k - (d == 2));
  D3 nrm = d3(n0[f], n0[dm.F + f], n0[2 * dm.F + f]);
  D3 xn = d3(xc[nc], xc[dm.C + nc], xc[2 * dm.C + nc]);
  D3 xp = d3(xc[pc], xc[dm.C + pc], xc[2 * dm.C + pc]);
  double dx = dot(xn - xp, nrm);
  dxf[f] = dx;
  const double Dn = U[nc], Dp = U[pc];
  for (int v = 0; v < 4; ++v) gf[v * dm.F + f] = (U[v * dm.C + nc] / Dn - U[v * dm.C + pc] / Dp) / dx;
}

// computeGradPhiCell_PBorn0_LimC (R:472-513): limited cell gradient from the
// back and front face gradients (0 on the boundary faces, never written).
__global__ void k_sweep_cell_grad(Dims dm, int d, int lim, const double* __restrict__ gf, double* __restrict__ G) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= dm.C) return;
  int i, j, k; dm.cijk(c, i, j, k);
  long long bf = dm.fid(d, i, j, k);
  long long ff = dm.fid(d, i + (d == 0), j + (d == 1), k + (d == 2));
  for (int v = 0; v < 4; ++v) {
    double g = 0.;
    double gb = gf[v * dm.F + bf], gfr = gf[v * dm.F + ff];
    if (gb != 0.) g += 0.5 * (limiter(lim, gfr / gb) * gb);
    if (gfr != 0.) g += 0.5 * (limiter(lim, gb / gfr) * gfr);
    G[v * dm.C + c] = g;
  }
}

// computeUpwindFaceQuantitiesForProjection_PBorn0_O2 (R:698-715).
__global__ void k_sweep_face_phi(Dims dm, int d, double order2, const double* __restrict__ xc,
                                 const double* __restrict__ n0, const double* __restrict__ xf,
                                 const double* __restrict__ uf, const double* __restrict__ dxf,
                                 const double* __restrict__ U, const double* __restrict__ G, double* __restrict__ phif) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= dm.nfd(d)) return;
  int i, j, k; dm.fdijk(d, t, i, j, k);
  int id = d == 0 ? i : (d == 1 ? j : k);
  if (id == 0 || id == dm.ncd(d)) return;
  long long f = dm.fid(d, i, j, k);
  long long nc = dm.cid(i, j, k);
  long long pc = dm.cid(i - (d == 0), j - (d == 1), k - (d == 2));
  long long up = (uf[f] * dxf[f] > 0.0) ? pc : nc;
  D3 nrm = d3(n0[f], n0[dm.F + f], n0[2 * dm.F + f]);
  D3 xx = d3(xf[f], xf[dm.F + f], xf[2 * dm.F + f]) - d3(xc[up], xc[dm.C + up], xc[2 * dm.C + up]);
  double dot_xf = dot(xx, nrm);
  const double D = U[up];
  for (int v = 0; v < 4; ++v) phif[v * dm.F + f] = U[v * dm.C + up] / D + order2 * dot_xf * G[v * dm.C + up];
}

// computeUremap_PBorn0 (R:892-988): fluxes through the back and front faces of
// d, U update, clamping, dual mass flux.
__global__ void k_sweep_cell_update(Dims dm, int d, const Scalars* __restrict__ S, const double* __restrict__ n0,
                                    const double* __restrict__ uf, const double* __restrict__ A,
                                    const double* __restrict__ ofn, const double* __restrict__ phif,
                                    double* __restrict__ U, double* __restrict__ dpf) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= dm.C) return;
  int i, j, k; dm.cijk(c, i, j, k);
  const double dt = S->dt;
  long long bf = dm.fid(d, i, j, k);
  long long ff = dm.fid(d, i + (d == 0), j + (d == 1), k + (d == 2));
  const int lb = d == 0 ? 1 : (d == 1 ? 2 : 0), lf = d == 0 ? 4 : (d == 1 ? 5 : 3);
  const bool okb = fabs(n0[d * dm.F + bf]) >= 1.0E-10, okf = fabs(n0[d * dm.F + ff]) >= 1.0E-10;
  const double ob = ofn[lb * dm.C + c], of = ofn[lf * dm.C + c];
  const double ub = uf[bf], uff = uf[ff], Ab = A[bf], Af = A[ff];
  for (int v = 0; v < 4; ++v) {
    double flux_face = 0., dp = 0.;
    if (okb) { double fl = ob * ub * Ab * dt * phif[v * dm.F + bf]; flux_face += fl; dp += 0.5 * fl * ob; }
    if (okf) { double fl = of * uff * Af * dt * phif[v * dm.F + ff]; flux_face += fl; dp += 0.5 * fl * of; }
    double u = U[v * dm.C + c] - flux_face;
    if ((v == 1 || v == 2) && u < 0.) u = 0.;
    U[v * dm.C + c] = u;
    if (v == 1) dpf[c] = dp;
  }
}

// computeDualGradPhi_LimC (D:721-778) on the inner nodes of d.
__global__ void k_sweep_dual_grad(Dims dm, int d, int lim, const double* __restrict__ xl,
                                  const double* __restrict__ phid, double* __restrict__ G) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= dm.N) return;
  int idx[3]; dm.nijk(n, idx[0], idx[1], idx[2]);
  if (idx[d] == 0 || idx[d] == dm.ncd(d)) return;
  long long st = d == 0 ? 1 : (d == 1 ? (dm.nx + 1) : (long long)(dm.nx + 1) * (dm.ny + 1));
  long long bn = n - st, fn = n + st;
  const double xn = xl[d * dm.N + n], xb = xl[d * dm.N + bn], xf = xl[d * dm.N + fn];
  for (int a = 0; a < 3; ++a) {
    double pn = phid[a * dm.N + n];
    double gfr = (phid[a * dm.N + fn] - pn) / (xf - xn);
    double gb = (pn - phid[a * dm.N + bn]) / (xn - xb);
    double g = 0.;
    if (gb != 0.) g += 0.5 * limiter(lim, gfr / gb) * gb;
    if (gfr != 0.) g += 0.5 * limiter(lim, gb / gfr) * gfr;
    G[a * dm.N + n] = g;
  }
}

// Dual remap of the nodes (D:129-523): back/front mass fluxes gathered from the
// 4+4 cells (D:288-341), upwind momentum and kinetic energy (D:372-491),
// filter and Phi_dual (D:507-522).  Phi_dual is double-buffered.
__global__ void k_sweep_dual_update(Dims dm, int d, const Scalars* __restrict__ S, double order2,
                                    const double* __restrict__ xl, const double* __restrict__ dpf,
                                    const double* __restrict__ G, const double* __restrict__ phid,
                                    double* __restrict__ ud, double* __restrict__ phid_out) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= dm.N) return;
  int idx[3]; dm.nijk(n, idx[0], idx[1], idx[2]);
  const bool inner = !(idx[d] == 0 || idx[d] == dm.ncd(d));
  if (!inner) {
    for (int a = 0; a < 4; ++a) phid_out[a * dm.N + n] = phid[a * dm.N + n];
    return;
  }
  const double deltat = S->dt;
  const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
  double bfm = 0., ffm = 0.;
  for (int s1 = -1; s1 <= 0; ++s1)
    for (int s2 = -1; s2 <= 0; ++s2) {
      int ci[3] = {idx[0], idx[1], idx[2]};
      ci[d] -= 1; ci[d1] += s1; ci[d2] += s2;
      if (ci[0] >= 0 && ci[0] < dm.nx && ci[1] >= 0 && ci[1] < dm.ny && ci[2] >= 0 && ci[2] < dm.nz)
        bfm += 0.25 * dpf[dm.cid(ci[0], ci[1], ci[2])];
    }
  for (int s1 = -1; s1 <= 0; ++s1)
    for (int s2 = -1; s2 <= 0; ++s2) {
      int ci[3] = {idx[0], idx[1], idx[2]};
      ci[d1] += s1; ci[d2] += s2;
      if (ci[0] >= 0 && ci[0] < dm.nx && ci[1] >= 0 && ci[1] < dm.ny && ci[2] >= 0 && ci[2] < dm.nz)
        ffm += 0.25 * dpf[dm.cid(ci[0], ci[1], ci[2])];
    }
  long long st = d == 0 ? 1 : (d == 1 ? (dm.nx + 1) : (long long)(dm.nx + 1) * (dm.ny + 1));
  long long bn = n - st, fn = n + st;
  const double xn = xl[d * dm.N + n], xb = xl[d * dm.N + bn], xf = xl[d * dm.N + fn];
  // phi_dual components: 0,1,2 velocity, 3 half |v| (reference index 4)
  double Pn[4], Pb[4], Pf[4], Gn[4], Gb[4], Gf[4];
  for (int a = 0; a < 4; ++a) {
    Pn[a] = phid[a * dm.N + n]; Pb[a] = phid[a * dm.N + bn]; Pf[a] = phid[a * dm.N + fn];
  }
  for (int a = 0; a < 3; ++a) { Gn[a] = G[a * dm.N + n]; Gb[a] = G[a * dm.N + bn]; Gf[a] = G[a * dm.N + fn]; }
  Gn[3] = Gb[3] = Gf[3] = 0.;                      // index 4 of the dual gradient is never set (D:771)
  double u3 = ud[3 * dm.N + n] + (bfm - ffm);
  const double ufront = 0.5 * (Pn[d] + Pn[d]);     // D:391
  const int signfront = (ufront > 0) ? 1 : -1;
  const double uback = 0.5 * (Pb[d] + Pn[d]);
  const int signback = (uback > 0) ? 1 : -1;
  const double* PF = (ffm < 0.) ? Pf : Pn;
  const double* GF = (ffm < 0.) ? Gf : Gn;
  const double* PB = (bfm > 0.) ? Pb : Pn;
  const double* GB = (bfm > 0.) ? Gb : Gn;
  double out[4];
  for (int a = 0; a < 4; ++a) {
    double FV = PF[a] + order2 * (0.5 * GF[a] * (signfront * (xf - xn) - deltat * ufront));
    double BV = PB[a] + order2 * (0.5 * GB[a] * (signback * (xn - xb) - deltat * uback));
    int ua = a < 3 ? a : 4;
    out[a] = ud[ua * dm.N + n] + (bfm * BV - ffm * FV);
  }
  for (int a = 0; a < 3; ++a) if (fabs(out[a]) < 1.e-300) out[a] = 0.;
  ud[0 * dm.N + n] = out[0]; ud[1 * dm.N + n] = out[1]; ud[2 * dm.N + n] = out[2];
  ud[3 * dm.N + n] = u3; ud[4 * dm.N + n] = out[3];
  phid_out[n] = out[0] / u3; phid_out[dm.N + n] = out[1] / u3; phid_out[2 * dm.N + n] = out[2] / u3;
  phid_out[3 * dm.N + n] = out[3] / u3;
}

// --- end of cycle ---

// remapVariables "moy" kernel for single-environment cells (F:446-643), the
// PerfectGas EOS (E:92-106).
__global__ void k_finalize_cells(Dims dm, Phys ph, Scalars* __restrict__ S, const double* __restrict__ U,
                                 const double* __restrict__ Ve, double* __restrict__ rho, double* __restrict__ e,
                                 double* __restrict__ q, double* __restrict__ p, double* __restrict__ cs,
                                 double* __restrict__ mass) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= dm.C) return;
  const double thr = ph.threshold;
  const double U0 = U[c], U1 = U[dm.C + c], U2 = U[2 * dm.C + c], U3 = U[3 * dm.C + c];
  const double vol = Ve[c];
  const double volt = 0. + U0, masset = 0. + U1;
  const double unsurvolt = 1. / volt;
  const double unsurvol = 1. / vol;
  double fvol = U0 * unsurvolt;
  if (fvol < thr) fvol = 0.;
  const double somme_frac = 0. + fvol;
  const double unsursomme_frac = 1. / somme_frac;
  fvol = fvol * unsursomme_frac;
  double mf = 1.;
  if (masset != 0.) {
    const double unsurmasset = 1. / masset;
    mf = U1 * unsurmasset;
    if (fvol < thr) mf = 0.;
    const double fmasset = 0. + mf;
    if (fmasset != 0.) { const double unsurfmasset = 1. / fmasset; mf = mf * unsurfmasset; }
  } else {
    atomicOr(&S->status, MHY_STATUS_ZERO_MASS);
  }
  double de = 0.;
  if (fvol > thr) { const double vn = U0 * vol * unsurvolt; de = U1 / vn; }
  const double density_nplus1 = 0. + fvol * de;
  const double cm = Ve[c] * density_nplus1;
  double ee = 0.;
  if (fvol > thr && U1 != 0.) ee = U2 / U1;
  double energie = 0. + mf * ee;
  const double pv = U3 * unsurvol;
  const double pseudo = 0. + fvol * pv;
  double r = de;
  if (r < 0. || energie < 0.) { energie = 0.; r = 0.; }
  const double g = ph.gamma;
  const double pr = (g - 1.) * r * energie;
  rho[c] = r;
  e[c] = energie;
  q[c] = pseudo;
  mass[c] = mf * cm;
  p[c] = pr;
  cs[c] = sqrt(g * pr / r);
}

// Node velocity v = U_dual / m and node mass (F:660-672, 697-719).
__global__ void k_finalize_nodes(Dims dm, const double* __restrict__ ud, const double* __restrict__ vh,
                                 const double* __restrict__ mass, double* __restrict__ v, double* __restrict__ nm) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= dm.N) return;
  const double m = ud[3 * dm.N + n];
  if (m != 0.) {
    v[n] = ud[n] / m; v[dm.N + n] = ud[dm.N + n] / m; v[2 * dm.N + n] = ud[2 * dm.N + n] / m;
  } else {
    v[n] = vh[n]; v[dm.N + n] = vh[dm.N + n]; v[2 * dm.N + n] = vh[2 * dm.N + n];
  }
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

// computeHydroDeltaT (MahycoModule.cc:2047-2061): min over cells of
// L / (c + max |v|), warp shuffle + block reduction, one atomicMin per block
// on the bit pattern (non-negative doubles order like unsigned integers).
__global__ void k_dt_min(Dims dm, Scalars* __restrict__ S, const double* __restrict__ L,
                         const double* __restrict__ cs, const double* __restrict__ v) {
  __shared__ unsigned long long wmin[32];
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  unsigned long long best = 0x7fefffffffffffffull;  // DBL_MAX
  if (c < dm.C) {
    int i, j, k; dm.cijk(c, i, j, k);
    double vmax = 0.;
    for (int a = 0; a < 8; ++a) {
      long long n = dm.nid(i + kCellNodeOff[a][0], j + kCellNodeOff[a][1], k + kCellNodeOff[a][2]);
      vmax = amax(norm2(d3(v[n], v[dm.N + n], v[2 * dm.N + n])), vmax);
    }
    double dx_sound = L[c] / (cs[c] + vmax);
    if (dx_sound >= 0.) best = (unsigned long long)__double_as_longlong(dx_sound);
    else atomicOr(&S->status, MHY_STATUS_NAN_DT);
  }
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long other = __shfl_down_sync(0xffffffffu, best, o);
    best = other < best ? other : best;
  }
  if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x < 32) {
    best = threadIdx.x < (blockDim.x >> 5) ? wmin[threadIdx.x] : 0x7fefffffffffffffull;
    for (int o = 16; o > 0; o >>= 1) {
      unsigned long long other = __shfl_down_sync(0xffffffffu, best, o);
      best = other < best ? other : best;
    }
    if (threadIdx.x == 0) atomicMin(&S->min_bits, best);
  }
}

// computeDeltaT (MahycoModule.cc:2076-2191): new dt from the reduced minimum.
__global__ void k_dt_finish(Scalars* S, Phys ph) {
  S->time += S->dt;
  const double gold = S->dt;
  S->old_dt = gold;
  const double minimum_aux = __longlong_as_double((long long)S->min_bits);
  double new_dt = ph.cfl * minimum_aux;
  new_dt = amin(new_dt, 1.05 * gold);
  new_dt = amin(new_dt, ph.deltat_max);
  if (new_dt < ph.deltat_min) S->status |= MHY_STATUS_DT_MIN;
  S->dt = new_dt;
  if (S->time > ph.final_time) S->status |= MHY_STATUS_FINAL_TIME;
  S->min_bits = 0x7fefffffffffffffull;
  S->iteration += 1;
}

}  // namespace mhy
