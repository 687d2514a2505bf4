// mhy_oracle.cpp -- CPU ORACLE for MaHyCo's Lagrange + ADI-remap time step.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, in plain C++17 + OpenMP, the
// compiled (accelerator) branches of the reference path so that the CUDA
// implementation can be checked against it.  It is linked only by tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg; the product never
// calls it.
//
// Parity status: UNPINNED by the reference.  MaHyCo ships no golden files and
// its CTest cases compare nothing (CMakeLists.txt:100-101,
// mahyco/launch_test.sh.in:2); the reference needs the Arcane framework, which
// is absent, so it cannot be built or run here.  This restatement follows the
// reference source line by line (citations below, paths relative to the
// reference project root, "M" = mahyco/src/MahycoModule.cc, "P" =
// mahyco/src/PrepareRemap.cc, "R" = mahyco/src/Remap/RemapADIService.cc,
// "D" = mahyco/src/Remap/DualPhaseRemap.cc, "F" = mahyco/src/Remap/RemapADIFinal.cc,
// "E" = mahyco/src/eos/perfectgas/PerfectGasEOSService.cc).
//
// Conventions that live in Arcane (absent) and are fixed here:
//  * cell (i,j,k) id = i + nx*(j + ny*k); node id = i + (nx+1)*(j + (ny+1)*k)
//    (cartesian/CartesianNumberingT.h: i fastest);
//  * cell->node order SN_trigo (cartesian/CartConnectivityCellNode.h:83-94),
//    the order the CQS formula of M:1080-1087,2195-2258 assumes;
//  * faces numbered X-normal, then Y, then Z (cartesian/CartesianGridT.h:49-66);
//    cell->face order = hexahedron local faces (z-,x-,y-,z+,x+,y+), the order
//    of the face centres in M:1080-1087;
//  * face->node order chosen so that the reference's face normal
//    (M:1020-1025, whose y component is the NEGATED cross-product component)
//    points from the previous to the next cell along the face's axis;
//  * node->cell order: increasing cell id.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <vector>
#include <algorithm>
#include <limits>
#include <omp.h>

#include "../arcane-benchs_b200/csrc/mhy_pow_third.h"

namespace {

struct R3 { double x, y, z; };
inline R3 r3(double x, double y, double z) { return R3{x, y, z}; }
inline R3 operator+(R3 a, R3 b) { return R3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline R3 operator-(R3 a, R3 b) { return R3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline R3 operator*(double s, R3 v) { return R3{v.x * s, v.y * s, v.z * s}; }
inline R3& operator+=(R3& a, R3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
inline double dot(R3 a, R3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline R3 cross(R3 u, R3 v) { return R3{u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x}; }
inline double normL2(R3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
inline R3 absolute(R3 a) { return R3{std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
inline R3 divs(R3 a, double s) { return R3{a.x / s, a.y / s, a.z / s}; }
inline double comp(R3 a, int d) { return d == 0 ? a.x : (d == 1 ? a.y : a.z); }
// Arcane math::min/max and std::min/max as written in the reference
inline double amin(double a, double b) { return (a < b) ? a : b; }
inline double amax(double a, double b) { return (a < b) ? b : a; }
inline double smin(double a, double b) { return (b < a) ? b : a; }
inline double smax(double a, double b) { return (a < b) ? b : a; }
inline double produit(double A, double B, double C, double D) { return A * B - C * D; }  // M:2261-2264

// Limiters, mahyco/src/Remap/RemapADIService.h:260-286
inline double limiter(int id, double r) {
  switch (id) {
    case 0: return smax(0.0, smin(1.0, r));                                // MinMod
    case 1: return smax(0.0, smax(smin(2.0 * r, 1.0), smin(r, 2.0)));      // SuperBee
    case 2: return (r <= 0.0 ? 0.0 : 2.0 * r / (1.0 + r));                 // VanLeer
    default: return 0.0;                                                   // DefaultO1
  }
}

// Material variable: global value plus per-environment partial values.  A
// pure cell's environment value IS the global value (Arcane materials); a
// mixed cell's environment values live in the partial slots.
struct MatVar {
  std::vector<double> g;
  std::vector<std::vector<double>> p;
  void init(int K, size_t C) { g.assign(C, 0.0); p.assign(K, std::vector<double>(C, 0.0)); }
};

enum { BC_VX = 0, BC_VY = 1, BC_VZ = 2 };
enum { SURF_XMIN = 0, SURF_XMAX, SURF_YMIN, SURF_YMAX, SURF_ZMIN, SURF_ZMAX };

struct Oracle {
  // mesh
  int nx, ny, nz, NX, NY, NZ;      // cells and nodes per direction
  long C, N, F, Fx, Fy, Fz;
  int K, nvars;
  // options (Mahyco.axl / RemapADI.axl names)
  double cfl, threshold, deltat_init, deltat_min, deltat_max, final_time;
  int lc_mode;          // 0 racine-cubique-volume, 1 faces-opposees
  int pseudo_centree, ordre_projection, limiteur_id, use_project_pow;
  int with_newton = 0;              // Mahyco.axl:308 with-newton
  int schema_csts = 0;              // Mahyco.axl:238 schema-csts
  // RemapADI.axl:155-173: projection-pente-borne, -debar-fix (0, 1, 2),
  // projection-pente-borne-mixte, projection-limiteur-pure-id
  int pente_borne = 0, pb_debar_fix = 0, pb_mixte = 0, limiteur_pure_id = 0;
  int conservation_energie_totale = 0;   // RemapADI.axl:151
  // slabs: the dt minimum over cell layers [dt_k0, dt_k1) only; with ext_dt
  // the cycle stops at the local minimum and orc_dt_finish completes it
  int dt_k0 = 0, dt_k1 = -1, ext_dt = 0;
  double local_min = 0.;
  std::vector<double> gamma;
  std::vector<int> eos;             // per environment: 0 PerfectGas, 1 StiffenedGas
  std::vector<double> pinf;         // StiffenedGas limit-tension (StiffenedGasEOS.axl:104)
  struct BC { int surface, type; double value; std::vector<int> nodes; };
  std::vector<BC> bcs;

  // state
  std::vector<R3> node_coord, node_coord_0, velocity, velocity_n, force;
  std::vector<double> node_mass;
  std::vector<uint32_t> env_mask;  // bit k set: cell belongs to environment k
  std::vector<int> env_id;         // >=0 pure (env id), else -(nbEnv+1)
  MatVar density, internal_energy, pressure, sound_speed, pseudo_viscosity, cell_volume,
      cell_mass, fracvol, mass_fraction, dpde, tau_density, density_n, internal_energy_n,
      pressure_n, cell_volume_n, pseudo_viscosity_n, pseudo_viscosity_nmoins1;
  std::vector<double> div_u, car_len, euler_volume, materiau;
  std::vector<R3> cell_coord, cqs, cqs_n;        // cqs: C*8
  std::vector<R3> face_normal, face_coord, face_length, outer_face_normal;  // ofn: C*6
  std::vector<double> face_normal_velocity, deltax;
  std::vector<double> u_lag, phi_lag, grad_phi, grad_phi_face, phi_face, dual_phi_flux;
  std::vector<double> u_dual, phi_dual, dual_grad_phi;
  std::vector<double> back_flux_mass, front_flux_mass, back_flux_mass_env, front_flux_mass_env;
  std::vector<double> back_flux_contrib_env, front_flux_contrib_env;
  std::vector<int> est_mixte, est_pure;
  std::vector<double> h_cell;                  // cell width along the sweep direction (order 3)
  std::vector<double> delta_phi_face_av, delta_phi_face_ar;   // pente-borne: C*nvars
  double global_deltat = 0, global_old_deltat = 0, old_deltat = 0, global_time = 0;
  int sens_projection = 0;
  long iteration = 0;
  uint32_t status = 0;

  // ---------------- connectivity ----------------
  long cid(int i, int j, int k) const { return i + (long)nx * (j + (long)ny * k); }
  long nid(int i, int j, int k) const { return i + (long)NX * (j + (long)NY * k); }
  void cijk(long c, int& i, int& j, int& k) const { i = (int)(c % nx); long t = c / nx; j = (int)(t % ny); k = (int)(t / ny); }
  void nijk(long n, int& i, int& j, int& k) const { i = (int)(n % NX); long t = n / NX; j = (int)(t % NY); k = (int)(t / NY); }
  int ncell_dir(int d) const { return d == 0 ? nx : (d == 1 ? ny : nz); }
  // SN_trigo, cartesian/CartConnectivityCellNode.h:83-94
  void cell_nodes(long c, long out[8]) const {
    int i, j, k; cijk(c, i, j, k);
    static const int dd[8][3] = {{0,0,0},{1,0,0},{1,1,0},{0,1,0},{0,0,1},{1,0,1},{1,1,1},{0,1,1}};
    for (int a = 0; a < 8; ++a) out[a] = nid(i + dd[a][0], j + dd[a][1], k + dd[a][2]);
  }
  // face id of a d-normal face whose lowest node is (i,j,k)
  long fid(int d, int i, int j, int k) const {
    if (d == 0) return i + (long)(nx + 1) * (j + (long)ny * k);
    if (d == 1) return Fx + i + (long)nx * (j + (long)(ny + 1) * k);
    return Fx + Fy + i + (long)nx * (j + (long)ny * k);
  }
  void fijk(long f, int& d, int& i, int& j, int& k) const {
    long t;
    if (f < Fx) { d = 0; i = (int)(f % (nx + 1)); t = f / (nx + 1); j = (int)(t % ny); k = (int)(t / ny); }
    else if (f < Fx + Fy) { d = 1; f -= Fx; i = (int)(f % nx); t = f / nx; j = (int)(t % (ny + 1)); k = (int)(t / (ny + 1)); }
    else { d = 2; f -= Fx + Fy; i = (int)(f % nx); t = f / nx; j = (int)(t % ny); k = (int)(t / ny); }
  }
  // face -> 4 nodes.  X: (0,0,0),(0,1,0),(0,1,1),(0,0,1); Y: (0,0,0),(1,0,0),(1,0,1),(0,0,1);
  // Z: (0,0,0),(1,0,0),(1,1,0),(0,1,0).  With the reference's normal formula
  // (M:1020-1025) each normal points to +axis.
  void face_nodes(long f, long out[4]) const {
    int d, i, j, k; fijk(f, d, i, j, k);
    if (d == 0) { out[0] = nid(i, j, k); out[1] = nid(i, j + 1, k); out[2] = nid(i, j + 1, k + 1); out[3] = nid(i, j, k + 1); }
    else if (d == 1) { out[0] = nid(i, j, k); out[1] = nid(i + 1, j, k); out[2] = nid(i + 1, j, k + 1); out[3] = nid(i, j, k + 1); }
    else { out[0] = nid(i, j, k); out[1] = nid(i + 1, j, k); out[2] = nid(i + 1, j + 1, k); out[3] = nid(i, j + 1, k); }
  }
  // cell -> 6 faces in hexahedron local order (z-, x-, y-, z+, x+, y+)
  void cell_faces(long c, long out[6]) const {
    int i, j, k; cijk(c, i, j, k);
    out[0] = fid(2, i, j, k); out[1] = fid(0, i, j, k); out[2] = fid(1, i, j, k);
    out[3] = fid(2, i, j, k + 1); out[4] = fid(0, i + 1, j, k); out[5] = fid(1, i, j + 1, k);
  }
  static int back_local_face(int d) { return d == 0 ? 1 : (d == 1 ? 2 : 0); }
  static int front_local_face(int d) { return d == 0 ? 4 : (d == 1 ? 5 : 3); }
  // node -> cells in increasing cell id, with the node's local index in each
  int node_cells(long n, long cells[8], int lidx[8]) const {
    int i, j, k; nijk(n, i, j, k);
    static const int loc[2][2][2] = {{{0, 4}, {3, 7}}, {{1, 5}, {2, 6}}};  // [di][dj][dk]
    int cnt = 0;
    for (int ck = k - 1; ck <= k; ++ck)
      for (int cj = j - 1; cj <= j; ++cj)
        for (int ci = i - 1; ci <= i; ++ci) {
          if (ci < 0 || cj < 0 || ck < 0 || ci >= nx || cj >= ny || ck >= nz) continue;
          cells[cnt] = cid(ci, cj, ck);
          lidx[cnt] = loc[i - ci][j - cj][k - ck];
          ++cnt;
        }
    return cnt;
  }

  // material value accessors (see MatVar)
  int nbEnv(long c) const { return __builtin_popcount(env_mask[c]); }
  double& mv(MatVar& v, int k, long c) { return (nbEnv(c) == 1) ? v.g[c] : v.p[k][c]; }

  void compute_env_id() {  // accenv/AccEnvDefaultService.cc:321-339
    for (long c = 0; c < C; ++c) {
      int n = nbEnv(c);
      env_id[c] = (n == 1) ? __builtin_ctz(env_mask[c]) : -n - 1;
    }
  }

  double pow_third(double v) const { return use_project_pow ? mhy::pow_third(v) : std::pow(v, 1. / 3.); }

  // ---------------- geometry kernels ----------------
  // M:2195-2258
  static void compute_cqs(const R3 x[8], const R3 fc[6], R3 out[8]) {
    const R3 c0 = fc[0], c1 = fc[1], c2 = fc[2], c3 = fc[3], c4 = fc[4], c5 = fc[5];
    const R3 n1a04 = 0.5 * cross(x[0] - c0, x[3] - c0);
    const R3 n1a03 = 0.5 * cross(x[3] - c0, x[2] - c0);
    const R3 n1a02 = 0.5 * cross(x[2] - c0, x[1] - c0);
    const R3 n1a01 = 0.5 * cross(x[1] - c0, x[0] - c0);
    const R3 n2a05 = 0.5 * cross(x[0] - c1, x[4] - c1);
    const R3 n2a12 = 0.5 * cross(x[4] - c1, x[7] - c1);
    const R3 n2a08 = 0.5 * cross(x[7] - c1, x[3] - c1);
    const R3 n2a04 = 0.5 * cross(x[3] - c1, x[0] - c1);
    const R3 n3a01 = 0.5 * cross(x[0] - c2, x[1] - c2);
    const R3 n3a06 = 0.5 * cross(x[1] - c2, x[5] - c2);
    const R3 n3a09 = 0.5 * cross(x[5] - c2, x[4] - c2);
    const R3 n3a05 = 0.5 * cross(x[4] - c2, x[0] - c2);
    const R3 n4a09 = 0.5 * cross(x[4] - c3, x[5] - c3);
    const R3 n4a10 = 0.5 * cross(x[5] - c3, x[6] - c3);
    const R3 n4a11 = 0.5 * cross(x[6] - c3, x[7] - c3);
    const R3 n4a12 = 0.5 * cross(x[7] - c3, x[4] - c3);
    const R3 n5a02 = 0.5 * cross(x[1] - c4, x[2] - c4);
    const R3 n5a07 = 0.5 * cross(x[2] - c4, x[6] - c4);
    const R3 n5a10 = 0.5 * cross(x[6] - c4, x[5] - c4);
    const R3 n5a06 = 0.5 * cross(x[5] - c4, x[1] - c4);
    const R3 n6a03 = 0.5 * cross(x[2] - c5, x[3] - c5);
    const R3 n6a08 = 0.5 * cross(x[3] - c5, x[7] - c5);
    const R3 n6a11 = 0.5 * cross(x[7] - c5, x[6] - c5);
    const R3 n6a07 = 0.5 * cross(x[6] - c5, x[2] - c5);
    const double t = 1. / 12.;
    out[0] = t * (5. * (n1a01 + n1a04 + n2a04 + n2a05 + n3a05 + n3a01) + (n1a02 + n1a03 + n2a08 + n2a12 + n3a06 + n3a09));
    out[1] = t * (5. * (n1a01 + n1a02 + n3a01 + n3a06 + n5a06 + n5a02) + (n1a04 + n1a03 + n3a09 + n3a05 + n5a10 + n5a07));
    out[2] = t * (5. * (n1a02 + n1a03 + n5a07 + n5a02 + n6a07 + n6a03) + (n1a01 + n1a04 + n5a06 + n5a10 + n6a11 + n6a08));
    out[3] = t * (5. * (n1a03 + n1a04 + n2a08 + n2a04 + n6a08 + n6a03) + (n1a01 + n1a02 + n2a05 + n2a12 + n6a07 + n6a11));
    out[4] = t * (5. * (n2a05 + n2a12 + n3a05 + n3a09 + n4a09 + n4a12) + (n2a08 + n2a04 + n3a01 + n3a06 + n4a10 + n4a11));
    out[5] = t * (5. * (n3a06 + n3a09 + n4a09 + n4a10 + n5a10 + n5a06) + (n3a01 + n3a05 + n4a12 + n4a11 + n5a07 + n5a02));
    out[6] = t * (5. * (n4a11 + n4a10 + n5a10 + n5a07 + n6a07 + n6a11) + (n4a12 + n4a09 + n5a06 + n5a02 + n6a03 + n6a08));
    out[7] = t * (5. * (n2a08 + n2a12 + n4a12 + n4a11 + n6a11 + n6a08) + (n2a04 + n2a05 + n4a09 + n4a10 + n6a07 + n6a03));
  }
  static void face_centres(const R3 x[8], R3 fc[6]) {  // M:1080-1087
    fc[0] = 0.25 * (x[0] + x[3] + x[2] + x[1]);
    fc[1] = 0.25 * (x[0] + x[4] + x[7] + x[3]);
    fc[2] = 0.25 * (x[0] + x[1] + x[5] + x[4]);
    fc[3] = 0.25 * (x[4] + x[5] + x[6] + x[7]);
    fc[4] = 0.25 * (x[1] + x[2] + x[6] + x[5]);
    fc[5] = 0.25 * (x[2] + x[3] + x[7] + x[6]);
  }

  // computeGeometricValues, M:1054-1299 (3D, #else branches)
  void computeGeometricValues() {
#pragma omp parallel for schedule(static)
    for (long c = 0; c < C; ++c) {
      long cn[8]; cell_nodes(c, cn);
      R3 x[8], fc[6];
      for (int a = 0; a < 8; ++a) x[a] = node_coord[cn[a]];
      face_centres(x, fc);
      compute_cqs(x, fc, &cqs[8 * c]);
    }
    const double inv_dim = 1. / 3;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < C; ++c) {
      long cn[8]; cell_nodes(c, cn);
      double volume = 0;
      R3 x[8];
      for (int a = 0; a < 8; ++a) { volume += dot(node_coord[cn[a]], cqs[8 * c + a]); x[a] = node_coord[cn[a]]; }
      volume *= inv_dim;
      cell_volume.g[c] = volume;
      if (lc_mode == 0) {
        car_len[c] = pow_third(volume);                                // M:1244-1260
      } else {                                                         // M:1180-1220
        R3 fc[6]; face_centres(x, fc);
        double d1 = normL2(fc[0] - fc[3]), d2 = normL2(fc[2] - fc[5]), d3 = normL2(fc[1] - fc[4]);
        car_len[c] = (d1 * d2 * d3) / (d1 * d2 + d1 * d3 + d2 * d3);
      }
    }
    // mixed cells: V_k = f_k V, M:1274-1295
#pragma omp parallel for schedule(static)
    for (long c = 0; c < C; ++c) {
      if (nbEnv(c) == 1) continue;
      for (int k = 0; k < K; ++k)
        if (env_mask[c] >> k & 1) cell_volume.p[k][c] = fracvol.p[k][c] * cell_volume.g[c];
    }
  }

  // ---------------- init ----------------
  // Init sequence of Mahyco.config:23-29: HydroStartInit (M:48-188),
  // PrepareFaceGroup (MahycoAnnexe.cc:183-251), ComputeCellMass (M:199-225),
  // ComputeNodeMass (M:235-266).  The test-case service (casModel()->initVar)
  // is replaced by the injected state.
  void hydroStartInit(const double* fv, const double* rho, const double* pres, const double* vel) {
    global_deltat = deltat_init;                                        // M:87-88
    // cell centres, MahycoAnnexe.cc:102-109
    for (long c = 0; c < C; ++c) {
      long cn[8]; cell_nodes(c, cn);
      R3 s = r3(0, 0, 0);
      for (int a = 0; a < 8; ++a) s += node_coord[cn[a]];
      cell_coord[c] = 0.125 * s;
    }
    sens_projection = 0;
    // environments from the injected volume fractions (initMat role)
    for (long c = 0; c < C; ++c) {
      uint32_t m = 0;
      for (int k = 0; k < K; ++k) if (fv[(size_t)k * C + c] > 0.0) m |= 1u << k;
      env_mask[c] = m;
    }
    compute_env_id();
    // injected state (initVar role): fractions, density, pressure, velocity
    for (long c = 0; c < C; ++c) {
      if (nbEnv(c) == 1) {
        int k = env_id[c];
        fracvol.g[c] = 1.; mass_fraction.g[c] = 1.;
        density.g[c] = rho[(size_t)k * C + c]; pressure.g[c] = pres[(size_t)k * C + c];
      } else {
        double rg = 0, pg = 0, mt = 0;
        for (int k = 0; k < K; ++k) if (env_mask[c] >> k & 1) {
          double f = fv[(size_t)k * C + c], r = rho[(size_t)k * C + c], p = pres[(size_t)k * C + c];
          fracvol.p[k][c] = f; density.p[k][c] = r; pressure.p[k][c] = p;
          rg += f * r; pg += f * p; mt += f * r;
        }
        for (int k = 0; k < K; ++k) if (env_mask[c] >> k & 1)
          mass_fraction.p[k][c] = fracvol.p[k][c] * density.p[k][c] / mt;
        fracvol.g[c] = 1.; mass_fraction.g[c] = 1.;
        density.g[c] = rg; pressure.g[c] = pg;
      }
    }
    for (long n = 0; n < N; ++n) velocity[n] = r3(vel[3 * n], vel[3 * n + 1], vel[3 * n + 2]);

    computeGeometricValues();                                           // M:96
    prepareFaceGroup();                                                 // M:99-100
    // initEOS per environment: PerfectGas E:20-32, StiffenedGas
    // (eos/stiffenedgas/StiffenedGasEOSService.cc:10-24)
    for (int k = 0; k < K; ++k) {
      const double g = gamma[k], pi = pinf[k];
      for (long c = 0; c < C; ++c) {
        if (!(env_mask[c] >> k & 1)) continue;
        double p = mv(pressure, k, c), r = mv(density, k, c);
        if (eos[k] == 1) {
          mv(internal_energy, k, c) = (p + (g * pi)) / ((g - 1.) * r);
          mv(sound_speed, k, c) = std::sqrt((g / r) * (p + pi));
        } else {
          mv(internal_energy, k, c) = p / ((g - 1.) * r);
          mv(sound_speed, k, c) = std::sqrt(g * p / r);
        }
      }
    }
    // mixed-cell averages, M:116-127
    for (long c = 0; c < C; ++c) {
      if (nbEnv(c) == 1) continue;
      internal_energy.g[c] = 0.;
      for (int k = 0; k < K; ++k) if (env_mask[c] >> k & 1) {
        internal_energy.g[c] += internal_energy.p[k][c] * mass_fraction.p[k][c];
        sound_speed.g[c] = smax(sound_speed.p[k][c], sound_speed.g[c]);
      }
    }
    for (long c = 0; c < C; ++c) euler_volume[c] = cell_volume.g[c];   // M:130-134
    initGeometricValues();                                              // M:150
    // volume again from the CQS, M:154-182 (same formula, same result)
    const double inv_dim = 1. / 3;
    for (long c = 0; c < C; ++c) {
      long cn[8]; cell_nodes(c, cn);
      double volume = 0;
      for (int a = 0; a < 8; ++a) volume += dot(node_coord[cn[a]], cqs[8 * c + a]);
      volume *= inv_dim;
      cell_volume.g[c] = volume;
    }
    prepareFaceGroup();
    // ComputeCellMass, M:199-225
    for (long c = 0; c < C; ++c) cell_mass.g[c] = density.g[c] * cell_volume.g[c];
    for (int k = 0; k < K; ++k)
      for (long c = 0; c < C; ++c) {
        if (!(env_mask[c] >> k & 1)) continue;
        double mf = mv(mass_fraction, k, c);
        mv(cell_mass, k, c) = mf * cell_mass.g[c];
      }
    computeNodeMass();
  }

  void computeNodeMass() {  // M:235-266 and F:712-718
#pragma omp parallel for schedule(static)
    for (long n = 0; n < N; ++n) {
      long cells[8]; int li[8]; int cnt = node_cells(n, cells, li);
      double s = 0.;
      for (int a = 0; a < cnt; ++a) s += cell_mass.g[cells[a]];
      node_mass[n] = .125 * s;
    }
  }

  // InitGeometricValues, M:1008-1050 (3D)
  void initGeometricValues() {
    for (long n = 0; n < N; ++n) node_coord_0[n] = node_coord[n];
    for (long f = 0; f < F; ++f) {
      long fn[4]; face_nodes(f, fn);
      R3 v1 = node_coord[fn[2]] - node_coord[fn[0]];
      R3 v2 = node_coord[fn[3]] - node_coord[fn[1]];
      R3 nn;
      nn.x = produit(v1.y, v2.z, v1.z, v2.y);
      nn.y = -produit(v2.x, v1.z, v2.z, v1.x);
      nn.z = produit(v1.x, v2.y, v1.y, v2.x);
      face_normal[f] = divs(nn, normL2(nn));
    }
    for (long f = 0; f < F; ++f) {
      long fn[4]; face_nodes(f, fn);
      R3 s = r3(0., 0., 0.);
      for (int a = 0; a < 4; ++a) s += .25 * node_coord[fn[a]];
      face_coord[f] = s;
    }
    for (long c = 0; c < C; ++c) {
      long cf[6]; cell_faces(c, cf);
      for (int a = 0; a < 6; ++a) {
        R3 dvec = face_coord[cf[a]] - cell_coord[c];
        outer_face_normal[6 * c + a] = divs(dvec, normL2(dvec));
      }
    }
  }

  // PrepareFaceGroup (MahycoAnnexe.cc:183-251) + _initBoundaryConditionsForAcc (:257-281)
  void prepareFaceGroup() {
    R3 mx = r3(-1., -1., -1.);
    for (long n = 0; n < N; ++n) {
      mx.x = smax(mx.x, node_coord[n].x); mx.y = smax(mx.y, node_coord[n].y); mx.z = smax(mx.z, node_coord[n].z);
    }
    std::vector<std::vector<char>> in_group(6, std::vector<char>(N, 0));
    for (long f = 0; f < F; ++f) {
      long fn[4]; face_nodes(f, fn);
      bool fl[6] = {true, true, true, true, true, true};
      for (int a = 0; a < 4; ++a) {
        R3 x = node_coord[fn[a]];
        if (x.x > threshold) fl[SURF_XMIN] = false;
        if (x.y > threshold) fl[SURF_YMIN] = false;
        if (x.z > threshold) fl[SURF_ZMIN] = false;
        if (std::fabs(x.x - mx.x) > threshold) fl[SURF_XMAX] = false;
        if (std::fabs(x.y - mx.y) > threshold) fl[SURF_YMAX] = false;
        if (std::fabs(x.z - mx.z) > threshold) fl[SURF_ZMAX] = false;
      }
      for (int s = 0; s < 6; ++s) if (fl[s]) for (int a = 0; a < 4; ++a) in_group[s][fn[a]] = 1;
    }
    for (auto& bc : bcs) {
      bc.nodes.clear();
      for (long n = 0; n < N; ++n) if (in_group[bc.surface][n]) bc.nodes.push_back((int)n);
    }
  }

  // ---------------- compute loop (Mahyco.config:30-41) ----------------
  void saveValuesAtN() {  // M:308-450
    global_old_deltat = old_deltat;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < C; ++c) {
      pseudo_viscosity_nmoins1.g[c] = pseudo_viscosity_n.g[c];
      pseudo_viscosity_n.g[c] = pseudo_viscosity.g[c];
      pressure_n.g[c] = pressure.g[c];
      cell_volume_n.g[c] = cell_volume.g[c];
      density_n.g[c] = density.g[c];
      internal_energy_n.g[c] = internal_energy.g[c];
      for (int a = 0; a < 8; ++a) cqs_n[8 * c + a] = cqs[8 * c + a];
      if (nbEnv(c) != 1)
        for (int k = 0; k < K; ++k) if (env_mask[c] >> k & 1) {
          pseudo_viscosity_nmoins1.p[k][c] = pseudo_viscosity_n.p[k][c];
          pseudo_viscosity_n.p[k][c] = pseudo_viscosity.p[k][c];
          pressure_n.p[k][c] = pressure.p[k][c];
          cell_volume_n.p[k][c] = cell_volume.p[k][c];
          density_n.p[k][c] = density.p[k][c];
          internal_energy_n.p[k][c] = internal_energy.p[k][c];
        }
    }
#pragma omp parallel for schedule(static)
    for (long n = 0; n < N; ++n) { velocity_n[n] = velocity[n]; node_coord[n] = node_coord_0[n]; }
  }

  // Nodal force gather of updateForceAndVelocity (M:589-665) from global
  // cell pressures and pseudo-viscosities and the given corner vectors.
  R3 node_force(long n, const MatVar& pres, const MatVar& q, const std::vector<R3>& cq) const {
    long cells[8]; int li[8]; int cnt = node_cells(n, cells, li);
    R3 f = r3(0, 0, 0);
    for (int a = 0; a < cnt; ++a) {
      long c = cells[a];
      f += (pres.g[c] + q.g[c]) * cq[8 * c + li[a]];
    }
    return f;
  }

  void updateVelocity() {  // M:678-731 -> updateForceAndVelocity M:589-665
    const double dt = 0.5 * (global_old_deltat + global_deltat);
#pragma omp parallel for schedule(static)
    for (long n = 0; n < N; ++n) {
      const R3 f = node_force(n, pressure_n, pseudo_viscosity_n, cqs_n);
      force[n] = f;
      // schema-csts with projection: updateVelocityBackward first (M:693,
      // 743-781), v_n from n to n-1/2 with the same force
      if (schema_csts) velocity_n[n] = velocity_n[n] + ((-0.5 * global_old_deltat) / node_mass[n]) * f;
      velocity[n] = velocity_n[n] + (dt / node_mass[n]) * f;
    }
  }

  // updateVelocityForward (PrepareRemap.cc:456, M:792-831): v from n+1/2 to
  // n+1 with the force of this cycle's corner vectors and the current global
  // pressure and pseudo-viscosity; no boundary condition follows.
  void updateVelocityForward() {
    const double dt = 0.5 * global_deltat;
#pragma omp parallel for schedule(static)
    for (long n = 0; n < N; ++n) {
      const R3 f = node_force(n, pressure, pseudo_viscosity, cqs);
      velocity[n] = velocity[n] + (dt / node_mass[n]) * f;
    }
  }

  void applyBoundaryCondition() {  // M:936-1004
    for (auto& bc : bcs)
      for (int n : bc.nodes) {
        if (bc.type == BC_VX) velocity[n].x = bc.value;
        else if (bc.type == BC_VY) velocity[n].y = bc.value;
        else if (bc.type == BC_VZ) velocity[n].z = bc.value;
      }
  }

  void updatePosition() {  // M:870-931
    const double deltat = global_deltat;
#pragma omp parallel for schedule(static)
    for (long n = 0; n < N; ++n) node_coord[n] += deltat * velocity[n];
#pragma omp parallel for schedule(static)
    for (long c = 0; c < C; ++c) {
      long cn[8]; cell_nodes(c, cn);
      R3 s = r3(0., 0., 0.);
      for (int a = 0; a < 8; ++a) s += node_coord[cn[a]];
      cell_coord[c] = .125 * s;
    }
  }

  void updateDensity() {  // M:1331-1426 (compute_density_tau M:1307-1316)
    const double inv_deltat = 1.0 / global_deltat;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < C; ++c) {
      double rn = density_n.g[c];
      double nd = cell_mass.g[c] / cell_volume.g[c];
      double tau = 0.5 * (1.0 / rn + 1.0 / nd);
      density.g[c] = nd;
      tau_density.g[c] = tau;
      div_u[c] = inv_deltat * (1.0 / density.g[c] - 1.0 / rn) / tau_density.g[c];
      if (nbEnv(c) != 1)
        for (int k = 0; k < K; ++k) if (env_mask[c] >> k & 1) {
          double rk = cell_mass.p[k][c] / cell_volume.p[k][c];
          density.p[k][c] = rk;
          tau_density.p[k][c] = 0.5 * (1.0 / density_n.p[k][c] + 1.0 / rk);
        }
    }
  }

  void computeArtificialViscosity() {  // M:454-578 (#else)
#pragma omp parallel for schedule(static)
    for (long c = 0; c < C; ++c) {
      const double L = car_len[c], cs = sound_speed.g[c], du = div_u[c];
      pseudo_viscosity.g[c] = 0.;
      int e = env_id[c];
      if (e >= 0 && du < 0.0) {
        double g = gamma[e];
        pseudo_viscosity.g[c] = 1. / tau_density.g[c] * (-0.5 * L * cs * du + (g + 1) / 2.0 * L * L * du * du);
      }
      if (e < 0)
        for (int k = 0; k < K; ++k) if (env_mask[c] >> k & 1) {
          double g = gamma[k];
          double qk = 0.;
          if (du < 0.0) qk = 1. / tau_density.p[k][c] * (-0.5 * L * cs * du + (g + 1) / 2.0 * L * L * du * du);
          pseudo_viscosity.p[k][c] = qk;
          pseudo_viscosity.g[c] += qk * fracvol.p[k][c];
        }
    }
  }

  static double compute_eint(bool pc, double g, double qn, double q, double rn, double r, double p, double en) {
    double pseudo = 0.;  // M:1630-1654
    if (pc && ((qn + q) * (1.0 / r - 1.0 / rn) < 0.)) pseudo = 0.5 * (q + qn);
    if (!pc && (q * (1.0 / r - 1.0 / rn) < 0.)) pseudo = q;
    double denom = 1 + 0.5 * (g - 1.0) * r * (1.0 / r - 1.0 / rn);
    double numer = en - (0.5 * p + pseudo) * (1.0 / r - 1.0 / rn);
    return numer / denom;
  }

  // updateEnergyAndPressurebyNewton without schema-csts (M:1482-1535):
  // Newton iterations on fvnr(e) = e - en + 0.5 (p + pn + 2 q*) (1/rn1 - 1/rn)
  // with derivative 1 + 0.5 dpde (1/rn1 - 1/rn) (MahycoModule.h:420-429); each
  // iteration sets p and dpde by applyOneCellEOS at the current e and the new
  // density (PerfectGasEOSService.cc:38-45, StiffenedGasEOSService.cc:47-58),
  // and the loop test evaluates fvnr at the updated e with those p, dpde.  The
  // reference makes its first test before any EOS call, with p and dpde not yet
  // set; this restatement always runs the first iteration.  Only e is kept: p
  // and c are recomputed by the EOS after the remap.
  double newton_eint(int k, double qn, double q, double rn, double r, double pn, double en) const {
    const bool pc = pseudo_centree != 0;
    double pseudo = 0.;
    if (pc && ((qn + q) * (1.0 / r - 1.0 / rn) < 0.)) pseudo = 0.5 * (q + qn);
    if (!pc && (q * (1.0 / r - 1.0 / rn) < 0.)) pseudo = q;
    const double g = gamma[k], epsilon = threshold, itermax = 50;
    auto fvnr = [&](double e, double p) { return e - en + 0.5 * (p + pn + 2. * pseudo) * (1. / r - 1. / rn); };
    double e = en, p, dpde;
    int i = 0;
    do {
      if (eos[k] == 1) p = ((g - 1.) * r * e) - (g * pinf[k]);
      else p = (g - 1.) * r * e;
      dpde = (g - 1.) * r;
      const double enew = e - fvnr(e, p) / (1. + 0.5 * dpde * (1. / r - 1. / rn));
      e = enew;
      i++;
    } while (i < itermax && std::fabs(fvnr(e, p)) >= epsilon);
    return e;
  }

  double energy_update(int k, double qn, double q, double rn, double r, double p, double en) const {
    if (with_newton) return newton_eint(k, qn, q, rn, r, p, en);
    return compute_eint(pseudo_centree != 0, gamma[k], qn, q, rn, r, p, en);
  }

  // schema-csts: the four corner-vector sums of a cell (M:1556-1571,
  // 1776-1791): sum over the cell's nodes of v.cqs dt, v.cqs_n dt,
  // (v - v_n).cqs_n (dt - dt_old), v_n.cqs_n dt_old, in node order.
  struct CstsSums { double cn1, cn, cdn, con; };
  CstsSums csts_sums(long c) const {
    long cn[8]; cell_nodes(c, cn);
    CstsSums s{0., 0., 0., 0.};
    for (int a = 0; a < 8; ++a) {
      const R3 v = velocity[cn[a]], vn = velocity_n[cn[a]];
      s.cn1 += dot(v, cqs[8 * c + a]) * global_deltat;
      s.cn += dot(v, cqs_n[8 * c + a]) * global_deltat;
      s.cdn += dot(v - vn, cqs_n[8 * c + a]) * (global_deltat - global_old_deltat);
      s.con += dot(vn, cqs_n[8 * c + a]) * global_old_deltat;
    }
    return s;
  }

  // schema-csts energy of one environment cell, updateEnergyAndPressureforGP
  // (M:1795-1810) or by Newton on f (M:1538-1613, MahycoModule.h:433-445;
  // the first iteration always runs, as in newton_eint).  e = the current
  // energy, m = the environment's mass; qnm1 is the n-1 pseudo-viscosity.
  // Newton leaves p and c of its last EOS call (M:1605-1609), returned in pc.
  double csts_eint(int k, const CstsSums& s, double e0, double r, double m, double pn, double qn, double q,
                   double qnm1, double en, double* pc) const {
    const double g = gamma[k];
    if (!with_newton) {
      const double denom = 1 + 0.5 * (g - 1.0) * r * s.cn1 / m;
      const double numer = e0 - (0.5 * (pn + qn) * s.cn / m) - (0.5 * q * s.cn1 / m) +
                           (0.25 * (pn + qn) * s.cdn / m) - (0.5 * (qn - qnm1) * s.con / m);
      return numer / denom;
    }
    const double cdon = 0., epsilon = threshold, itermax = 50;
    auto f = [&](double e, double p) {
      return e - en + 0.5 * (p + q) * s.cn1 / m + 0.5 * (pn + qn) * s.cn / m - 0.25 * (pn + qn) * s.cdn / m +
             0.5 * (q - qnm1) * cdon / m;
    };
    double e = en, p, c, dpde;
    int i = 0;
    do {
      if (eos[k] == 1) { p = ((g - 1.) * r * e) - (g * pinf[k]); c = std::sqrt((g / r) * (p + pinf[k])); }
      else { p = (g - 1.) * r * e; c = std::sqrt(g * p / r); }
      dpde = (g - 1.) * r;
      const double enew = e - f(e, p) / (1. + 0.5 * dpde * s.cn1 / m);
      e = enew;
      i++;
    } while (i < itermax && std::fabs(f(e, p)) >= epsilon);
    pc[0] = p; pc[1] = c;
    return e;
  }

  void updateEnergyAndPressure() {  // M:1439-1478 -> updateEnergyAndPressureforGP M:1659-1770 (#else)
#pragma omp parallel for schedule(static)
    for (long c = 0; c < C; ++c) {
      const double e_cur = internal_energy.g[c];
      internal_energy.g[c] = 0.;
      int e = env_id[c];
      if (schema_csts) {
        const CstsSums sm = csts_sums(c);
        double pc[2];
        if (e >= 0) {
          const double ee = csts_eint(e, sm, e_cur, density.g[c], cell_mass.g[c], pressure_n.g[c],
                                      pseudo_viscosity_n.g[c], pseudo_viscosity.g[c], pseudo_viscosity_nmoins1.g[c],
                                      internal_energy_n.g[c], pc);
          internal_energy.g[c] = ee;
          if (with_newton) { pressure.g[c] = pc[0]; sound_speed.g[c] = pc[1]; }
        } else {
          for (int k = 0; k < K; ++k) if (env_mask[c] >> k & 1) {
            const double ek = csts_eint(k, sm, internal_energy.p[k][c], density.p[k][c], cell_mass.p[k][c],
                                        pressure_n.p[k][c], pseudo_viscosity_n.p[k][c], pseudo_viscosity.p[k][c],
                                        pseudo_viscosity_nmoins1.p[k][c], internal_energy_n.p[k][c], pc);
            internal_energy.p[k][c] = ek;
            if (with_newton) { pressure.p[k][c] = pc[0]; sound_speed.p[k][c] = pc[1]; }
            internal_energy.g[c] += mass_fraction.p[k][c] * ek;
          }
        }
        continue;
      }
      if (e >= 0) {
        internal_energy.g[c] = energy_update(e, pseudo_viscosity_n.g[c], pseudo_viscosity.g[c],
                                             density_n.g[c], density.g[c], pressure.g[c], internal_energy_n.g[c]);
      } else {
        for (int k = 0; k < K; ++k) if (env_mask[c] >> k & 1) {
          double ek = energy_update(k, pseudo_viscosity_n.p[k][c], pseudo_viscosity.p[k][c],
                                    density_n.p[k][c], density.p[k][c], pressure.p[k][c], internal_energy_n.p[k][c]);
          internal_energy.p[k][c] = ek;
          internal_energy.g[c] += mass_fraction.p[k][c] * ek;
        }
      }
    }
  }

  // ---------------- remap (P:448-563) ----------------
  void computeVariablesForRemap() {  // P:159-245, and its specialisation _PBorn0 P:258-437
    const int ne = K;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < C; ++c) {
      double* U = &u_lag[(size_t)c * nvars];
      for (int v = 0; v < nvars; ++v) U[v] = 0;
      int e = env_id[c];
      if (e >= 0) {
        U[e] = cell_volume.g[c];
        U[ne + e] = cell_volume.g[c] * density.g[c];
        U[2 * ne + e] = cell_volume.g[c] * density.g[c] * internal_energy.g[c];
        U[3 * ne + 0] = 0.; U[3 * ne + 1] = 0.; U[3 * ne + 2] = 0.; U[3 * ne + 3] = 0.;
        U[3 * ne + 4] = cell_volume.g[c] * pseudo_viscosity.g[c];
      } else {
        for (int k = 0; k < K; ++k) if (env_mask[c] >> k & 1) {
          double vk = cell_volume.p[k][c];
          U[k] = vk;
          U[ne + k] = vk * density.p[k][c];
          U[2 * ne + k] = vk * density.p[k][c] * internal_energy.p[k][c];
          U[3 * ne + 0] = 0.; U[3 * ne + 1] = 0.; U[3 * ne + 2] = 0.; U[3 * ne + 3] = 0.;
          U[3 * ne + 4] = vk * pseudo_viscosity.p[k][c];               // last environment wins
        }
      }
      double* P = &phi_lag[(size_t)c * nvars];
      if (pente_borne) {  // P:201-212: volume fraction, density, internal energy, q of each environment
        auto set_phi = [&](int k, double f, double r, double e, double q) {
          P[k] = f; P[ne + k] = r; P[2 * ne + k] = e;
          P[3 * ne + 0] = 0.; P[3 * ne + 1] = 0.; P[3 * ne + 2] = 0.; P[3 * ne + 3] = 0.;
          P[3 * ne + 4] = q;
        };
        if (e >= 0) set_phi(e, fracvol.g[c], density.g[c], internal_energy.g[c], pseudo_viscosity.g[c]);
        else
          for (int k = 0; k < K; ++k) if (env_mask[c] >> k & 1)
            set_phi(k, fracvol.p[k][c], density.p[k][c], internal_energy.p[k][c], pseudo_viscosity.p[k][c]);
      } else {
        for (int v = 0; v < nvars; ++v) P[v] = U[v] / cell_volume.g[c];
      }
    }
#pragma omp parallel for schedule(static)
    for (long n = 0; n < N; ++n) {
      double* Ud = &u_dual[(size_t)n * nvars];
      double* Pd = &phi_dual[(size_t)n * nvars];
      const double m = node_mass[n];
      const R3 v = velocity[n];
      Ud[0] = m * v.x; Ud[1] = m * v.y; Ud[2] = m * v.z; Ud[3] = m;
      Ud[4] = 0.5 * m * normL2(v);
      Pd[0] = v.x; Pd[1] = v.y; Pd[2] = v.z; Pd[3] = m;
      Pd[4] = 0.5 * normL2(v);
    }
  }

  void computeFaceQuantitesForRemap() {  // P:15-123 (3D); schema-csts: P:69-79
    const double one_over_nbnode = .25;
#pragma omp parallel for schedule(static)
    for (long f = 0; f < F; ++f) {
      long fn[4]; face_nodes(f, fn);
      R3 v1 = node_coord[fn[2]] - node_coord[fn[0]];
      R3 v2 = node_coord[fn[3]] - node_coord[fn[1]];
      face_length[f] = absolute(0.5 * cross(v1, v2));
      R3 vm = r3(0., 0., 0.), fc = r3(0., 0., 0.);
      for (int a = 0; a < 4; ++a) {
        fc += one_over_nbnode * node_coord[fn[a]];
        if (schema_csts) vm += 0.5 * (velocity[fn[a]] + velocity_n[fn[a]]);
        else vm += velocity[fn[a]];
      }
      face_coord[f] = fc;
      face_normal_velocity[f] = dot(one_over_nbnode * vm, face_normal[f]);
    }
  }

  // inner faces of direction d: the faces with both a previous and a next cell
  bool face_prev_next(long f, int d, long& pc, long& nc) const {
    int fd, i, j, k; fijk(f, fd, i, j, k);
    int id = d == 0 ? i : (d == 1 ? j : k);
    pc = (id > 0) ? cid(i - (d == 0), j - (d == 1), k - (d == 2)) : -1;
    nc = (id < ncell_dir(d)) ? cid(i, j, k) : -1;
    return pc >= 0 && nc >= 0;
  }
  long face_begin(int d) const { return d == 0 ? 0 : (d == 1 ? Fx : Fx + Fy); }
  long face_end(int d) const { return d == 0 ? Fx : (d == 1 ? Fx + Fy : F); }

  // Order 3 (Remap-ordre-3.cc:7-131), restated with the same operation order.
  static double evaluate_grad(double hm, double h0, double hp, double ym, double y0, double yp) {
    return h0 / (hm + h0 + hp) * ((2. * hm + h0) / (h0 + hp) * (yp - y0) + (h0 + 2. * hp) / (hm + h0) * (y0 - ym));
  }
  static double evaluate_ystar(double hmm, double hm, double hp, double hpp, double ymm, double ym, double yp,
                               double ypp, double gradm, double gradp) {
    const double tmp1 = (2. * hp * hm) / (hm + hp) * ((hmm + hm) / (2. * hm + hp) - (hpp + hp) / (2. * hp + hm)) * (yp - ym);
    const double tmp2 = -hm * (hmm + hm) / (2. * hm + hp) * gradp + hp * (hp + hpp) / (hm + 2. * hp) * gradm;
    return ym + hm / (hm + hp) * (yp - ym) + 1. / (hmm + hm + hp + hpp) * (tmp1 + tmp2);
  }
  static double evaluate_fm(double x, double dx, double up, double du, double u6) {
    return up - 0.5 * x / dx * (du - (1. - 2. / 3. * x / dx) * u6);
  }
  static double evaluate_fp(double x, double dx, double um, double du, double u6) {
    return um + 0.5 * x / dx * (du - (1. - 2. / 3. * x / dx) * u6);
  }
  static double flux_ordre3(double ymmm, double ymm, double ym, double yp, double ypp, double yppp, double hmmm,
                            double hmm, double hm, double hp, double hpp, double hppp, double vdt) {
    const double gradmm = evaluate_grad(hmmm, hmm, hm, ymmm, ymm, ym);
    const double gradm = evaluate_grad(hmm, hm, hp, ymm, ym, yp);
    const double gradp = evaluate_grad(hm, hp, hpp, ym, yp, ypp);
    const double gradpp = evaluate_grad(hp, hpp, hppp, yp, ypp, yppp);
    const double ystarm = evaluate_ystar(hmmm, hmm, hm, hp, ymmm, ymm, ym, yp, gradmm, gradm);
    const double ystar = evaluate_ystar(hmm, hm, hp, hpp, ymm, ym, yp, ypp, gradm, gradp);
    const double ystarp = evaluate_ystar(hm, hp, hpp, hppp, ym, yp, ypp, yppp, gradp, gradpp);
    const double ym_m = ystarm, ym_p = ystar, yp_m = ystar, yp_p = ystarp;
    const double grad_m = ym_p - ym_m, grad_p = yp_p - yp_m;
    const double ym6 = 6. * (ym - 0.5 * (ym_m + ym_p));
    const double yp6 = 6. * (yp - 0.5 * (yp_m + yp_p));
    double flux;
    if (vdt > 0.) flux = evaluate_fm(vdt, hm, ym_p, grad_m, ym6);
    else if (vdt < 0.) flux = evaluate_fp(-vdt, hp, yp_m, grad_p, yp6);
    else return 0.;
    // TVD limitation
    const double num = vdt / hm, nup = vdt / hp;
    const double ym_ym = ym + (1. - num) / num * (ym - ymm);
    const double yp_ym = yp - (1. + nup) / nup * (yp - ypp);
    double i1[2], i2[2], lim[2];
    i1[0] = amin(ym, yp); i1[1] = amax(ym, yp);
    if (vdt >= 0.) { i2[0] = amin(ym, ym_ym); i2[1] = amax(ym, ym_ym); }
    else { i2[0] = amin(yp, yp_ym); i2[1] = amax(yp, yp_ym); }
    if ((i1[1] < i2[0]) || (i2[1] < i1[0])) { lim[0] = 0.; lim[1] = 0.; }
    else { lim[0] = amax(i1[0], i2[0]); lim[1] = amin(i1[1], i2[1]); }
    if (flux < lim[0]) flux = lim[0];
    if (flux > lim[1]) flux = lim[1];
    return flux;
  }

  // fluxLimiterG, UtilesRemap.cc:127-175: the generalised limiters for
  // uneven cell widths (ids of TypesMahyco.h:65-74: 3 minmodG, 4 superBeeG,
  // 5 vanLeerG, 6 arithmeticG, 7 ultrabeeG); std::min / std::max semantics.
  static double flux_limiter_g(int id, double gradplus, double gradmoins, double y0, double yplus, double ymoins,
                               double h0, double hplus, double hmoins) {
    double grady = 0., gradM, gradMplus, gradMmoins;
    if (gradplus * gradmoins < 0.0) return 0.;
    if (id == 3) {
      if ((yplus - ymoins) > 0.) grady = smin(std::fabs(gradplus), std::fabs(gradmoins));
      else grady = -smin(std::fabs(gradplus), std::fabs(gradmoins));
    } else if (id == 4) {
      if ((yplus - ymoins) > 0.) grady = smax(std::fabs(gradplus), std::fabs(gradmoins));
      else grady = -smax(std::fabs(gradplus), std::fabs(gradmoins));
    } else if (id == 5) {
      const double lambdaplus = (h0 / 2. + hplus) / (h0 + hplus + hmoins);
      const double lambdamoins = (h0 / 2. + hmoins) / (h0 + hplus + hmoins);
      if ((lambdaplus * gradplus + lambdamoins * gradmoins) != 0.)
        grady = gradplus * gradmoins / (lambdaplus * gradplus + lambdamoins * gradmoins);
      else grady = 0.;
    } else if (id == 7) {
      grady = (yplus - ymoins) / h0;
    } else if (id == 6) {
      const double lambdaplus = (h0 / 2. + hplus) / (h0 + hplus + hmoins);
      const double lambdamoins = (h0 / 2. + hmoins) / (h0 + hplus + hmoins);
      grady = lambdamoins * gradplus + lambdaplus * gradmoins;
    }
    gradMplus = gradplus * (h0 + hplus) / h0;
    gradMmoins = gradmoins * (h0 + hmoins) / h0;
    gradM = smin(std::fabs(gradMplus), std::fabs(gradMmoins));
    if ((yplus - ymoins) > 0.) grady = smin(std::fabs(gradM), std::fabs(grady));
    else grady = -smin(std::fabs(gradM), std::fabs(grady));
    return grady;
  }

  // ---- pente-borne (projection-pente-borne), UtilesRemap.cc ----
  // INTY, :83-93: integral from -infinity to X of the segment (x0,y0)-(x1,y1)
  double inty(double X, double x0, double y0, double x1, double y1) const {
    double flux = 0.;
    if (std::fabs(x1 - x0) > threshold) {
      const double eta = amin(amax(0., (X - x0) / (x1 - x0)), 1.);
      flux = (y0 + 0.5 * eta * (y1 - y0)) * (x1 - x0) * eta;
    }
    return flux;
  }
  // computeY0, :184-238 (limiter ids of TypesMahyco.h:65-74; 3000 as minmod)
  static void compute_y0(int id, double yplus, double ymoins, double h0, double hplus, double hmoins, double& y0plus,
                         double& y0moins) {
    y0plus = 0.; y0moins = 0.;
    if (id == 3 || id == 0 || id == 3000) {
      y0plus = yplus; y0moins = ymoins;
    } else if (id == 4 || id == 1) {
      y0plus = ((h0 + hmoins) * yplus + h0 * ymoins) / (2 * h0 + hmoins);
      y0moins = ((h0 + hplus) * ymoins + h0 * yplus) / (2 * h0 + hplus);
    } else if (id == 5 || id == 2) {
      const double a = amin(yplus, ymoins), b = amax(yplus, ymoins);
      double xplus = (h0 * h0 + 3 * h0 * hmoins + 2 * hmoins * hmoins) * yplus;
      double xmoins = (h0 * h0 + 3 * h0 * hplus + 2 * hplus * hplus) * ymoins;
      xplus += (h0 * h0 - h0 * hplus - 2 * hplus * hplus + 2 * h0 * hmoins) * ymoins;
      xmoins += (h0 * h0 - h0 * hmoins - 2 * hmoins * hmoins + 2 * h0 * hplus) * yplus;
      xplus /= (2 * h0 * h0 + 5 * h0 * hmoins + 2 * hmoins * hmoins - h0 * hplus - 2 * hplus * hplus);
      xmoins /= (2 * h0 * h0 + 5 * h0 * hplus + 2 * hplus * hplus - h0 * hmoins - 2 * hmoins * hmoins);
      y0plus = amin(amax(xplus, a), b);
      y0moins = amin(amax(xmoins, a), b);
    } else if (id == 7) {
      y0plus = (yplus + ymoins) / 2.;
      y0moins = (yplus + ymoins) / 2.;
    } else if (id == 6) {
      y0plus = ((h0 + hmoins + hplus) * yplus + h0 * ymoins) / (2 * h0 + hmoins + hplus);
      y0moins = ((h0 + hmoins + hplus) * ymoins + h0 * yplus) / (2 * h0 + hmoins + hplus);
    }
  }
  // computeFluxPP / computeFluxPPPure, :406-623 / :628-823: the integral of
  // the three-piece reconstruction (computexgxd :246-266, computeygyd
  // :276-296) over the part of the cell that leaves through the back (type
  // 0) or front (type 1) face in dt; the debar fixes on top.  The reference
  // calls abs() on doubles (the floating-point overload).
  void compute_flux_pp(long c, long fc, long bc, double face_normal_velocity_out, double deltat_n, int type,
                       bool pure, double* Flux) const {
    const int nbmat = K;
    for (int v = 0; v < nvars; ++v) Flux[v] = 0.;
    const double ppv = 0.5 * (face_normal_velocity_out + std::fabs(face_normal_velocity_out)) * deltat_n;
    const int lim_y0 = pure ? limiteur_pure_id : limiteur_id;
    const double* P0 = &phi_lag[(size_t)c * nvars];
    const double* Pf = &phi_lag[(size_t)fc * nvars];
    const double* Pb = &phi_lag[(size_t)bc * nvars];
    const double h0 = h_cell[c], hplus = h_cell[fc], hmoins = h_cell[bc];
    for (int v = 0; v < nvars; ++v) {
      double y0plus, y0moins;
      compute_y0(lim_y0, Pf[v], Pb[v], h0, hplus, hmoins, y0plus, y0moins);
      // computexgxd
      double xplus = 1.;
      if (std::fabs(y0plus - Pf[v]) > threshold) xplus = (P0[v] - Pf[v]) / (y0plus - Pf[v]) - 1. / 2.;
      double xmoins = 1.;
      if (std::fabs(y0moins - Pb[v]) > threshold) xmoins = (P0[v] - Pb[v]) / (y0moins - Pb[v]) - 1. / 2.;
      const double xd = +h0 * amin(amax(xplus, -1. / 2.), 1. / 2.);
      const double xg = -h0 * amin(amax(xmoins, -1. / 2.), 1. / 2.);
      // computeygyd
      const double grady = grad_phi[(size_t)c * nvars + v];
      const double xtd = P0[v] + h0 / 2 * grady;
      const double xtg = P0[v] - h0 / 2 * grady;
      const double ad = amin(Pf[v], 2. * y0moins - Pb[v]), bd = amax(Pf[v], 2. * y0moins - Pb[v]);
      const double ag = amin(Pb[v], 2. * y0plus - Pf[v]), bg = amax(Pb[v], 2. * y0plus - Pf[v]);
      const double yd = amin(amax(xtd, ad), bd);
      const double yg = amin(amax(xtg, ag), bg);
      double flux1, flux2, flux3, flux1m, flux2m, flux3m;
      if (type == 0) {
        flux1m = inty(-h0 / 2. + ppv, -h0 / 2., Pb[v], xg, yg);
        flux1 = inty(-h0 / 2., -h0 / 2., Pb[v], xg, yg);
        flux2m = inty(-h0 / 2. + ppv, xg, yg, xd, yd);
        flux2 = inty(-h0 / 2., xg, yg, xd, yd);
        flux3m = inty(-h0 / 2. + ppv, xd, yd, h0 / 2., Pf[v]);
        flux3 = inty(-h0 / 2., xd, yd, h0 / 2., Pf[v]);
      } else {
        flux1 = inty(h0 / 2. - ppv, -h0 / 2., Pb[v], xg, yg);
        flux1m = inty(h0 / 2., -h0 / 2., Pb[v], xg, yg);
        flux2 = inty(h0 / 2. - ppv, xg, yg, xd, yd);
        flux2m = inty(h0 / 2., xg, yg, xd, yd);
        flux3 = inty(h0 / 2. - ppv, xd, yd, h0 / 2., Pf[v]);
        flux3m = inty(h0 / 2., xd, yd, h0 / 2., Pf[v]);
      }
      Flux[v] = smax(((flux1m - flux1) + (flux2m - flux2) + (flux3m - flux3)), 0.);
      if (((Pf[v] - P0[v]) * (Pb[v] - P0[v])) >= 0.) Flux[v] = P0[v] * ppv;   // formule 16
    }
    if (pb_debar_fix == 1) {
      double somme_flux_masse = 0., somme_flux_volume = 0.;
      for (int m = 0; m < nbmat; m++) somme_flux_volume += Flux[m];
      if (std::fabs(somme_flux_volume) > threshold) {
        for (int m = 0; m < nbmat; m++) {
          if (!pure) Flux[nbmat + m] = (Flux[nbmat + m] / somme_flux_volume) * Flux[m];
          Flux[2 * nbmat + m] = (Flux[2 * nbmat + m] / somme_flux_volume) * Flux[nbmat + m];
          somme_flux_masse += Flux[nbmat + m];
        }
        Flux[3 * nbmat] = (Flux[3 * nbmat] / somme_flux_volume) * somme_flux_masse;
        Flux[3 * nbmat + 1] = (Flux[3 * nbmat + 1] / somme_flux_volume) * somme_flux_masse;
        Flux[3 * nbmat + 2] = (Flux[3 * nbmat + 2] / somme_flux_volume) * somme_flux_masse;
        Flux[3 * nbmat + 3] = P0[3 * nbmat + 3] * somme_flux_volume;
      } else {
        for (int v = 0; v < nvars; ++v) Flux[v] = 0.;
      }
    } else if (pb_debar_fix == 2) {
      double somme_flux_masse = 0., somme_flux_volume = 0.;
      for (int m = 0; m < nbmat; m++) {
        if (!pure) Flux[nbmat + m] = P0[nbmat + m] * Flux[m];
        Flux[2 * nbmat + m] = P0[2 * nbmat + m] * Flux[nbmat + m];
        somme_flux_masse += Flux[nbmat + m];
        somme_flux_volume += Flux[m];
      }
      Flux[3 * nbmat] = P0[3 * nbmat] * somme_flux_masse;
      Flux[3 * nbmat + 1] = P0[3 * nbmat + 1] * somme_flux_masse;
      Flux[3 * nbmat + 2] = P0[3 * nbmat + 2] * somme_flux_masse;
      Flux[3 * nbmat + 3] = P0[3 * nbmat + 3] * somme_flux_volume;
    }
    if (ppv == 0.) for (int v = 0; v < nvars; ++v) Flux[v] = 0.;
  }

  void computeGradPhiFace(int idir) {  // R:91-271 (h_cell by cells, R:225-258; read at order 3 and by the G limiters)
    if (ordre_projection == 3 || limiteur_id >= 3 || pente_borne) {
#pragma omp parallel for schedule(static)
      for (long c = 0; c < C; ++c) {
        long cf[6]; cell_faces(c, cf);
        int ii, jj, kk; cijk(c, ii, jj, kk);
        const int id = idir == 0 ? ii : (idir == 1 ? jj : kk);
        double h = 0;
        if (id > 0) h += std::sqrt(dot(face_coord[cf[back_local_face(idir)]] - cell_coord[c],
                                       face_coord[cf[back_local_face(idir)]] - cell_coord[c]));
        if (id < ncell_dir(idir) - 1)
          h += std::sqrt(dot(face_coord[cf[front_local_face(idir)]] - cell_coord[c],
                             face_coord[cf[front_local_face(idir)]] - cell_coord[c]));
        h_cell[c] = h;
      }
    }
#pragma omp parallel for schedule(static)
    for (long f = face_begin(idir); f < face_end(idir); ++f) {
      long pc, nc;
      if (!face_prev_next(f, idir, pc, nc)) continue;
      deltax[f] = dot(cell_coord[nc] - cell_coord[pc], face_normal[f]);
      for (int v = 0; v < nvars; ++v)
        grad_phi_face[(size_t)f * nvars + v] = (phi_lag[(size_t)nc * nvars + v] - phi_lag[(size_t)pc * nvars + v]) / deltax[f];
    }
  }

  void computeGradPhiCell(int idir) {  // R:283-317 -> computeGradPhiCell_PBorn0_LimC R:447-517
#pragma omp parallel for schedule(static)
    for (long c = 0; c < C; ++c)
      for (int v = 0; v < nvars; ++v) grad_phi[(size_t)c * nvars + v] = 0.;
    if (pente_borne) {  // R:324-326
      std::fill(delta_phi_face_av.begin(), delta_phi_face_av.end(), 0.0);
      std::fill(delta_phi_face_ar.begin(), delta_phi_face_ar.end(), 0.0);
    }
    if (ordre_projection <= 1) return;
    if (limiteur_id >= 3 || pente_borne || pb_mixte) {  // general path R:319-437
      const R3 dirproj = r3(0.5 * (1 - idir) * (2 - idir), 1.0 * idir * (2 - idir), -0.5 * idir * (1 - idir));
      const double deltat = global_deltat;
#pragma omp parallel for schedule(static)
      for (long c = 0; c < C; ++c) {
        long cf[6]; cell_faces(c, cf);
        const int lb = back_local_face(idir), lf = front_local_face(idir);
        long bf = cf[lb], ff = cf[lf];
        const long bc = along(c, idir, -1), fc = along(c, idir, +1);   // the cell itself at the ends
        const bool voisinage_pure = pb_mixte && est_mixte[c] == 0 && est_mixte[fc] == 0 && est_mixte[bc] == 0 &&
                                    est_pure[c] == est_pure[fc] && est_pure[c] == est_pure[bc];
        int lim = limiteur_id;
        if (limiteur_pure_id == 1 && voisinage_pure) lim = limiteur_pure_id;
        // computeAndLimitGradPhi, UtilesRemap.cc:306-333
        for (int v = 0; v < nvars; ++v) {
          const double gf = grad_phi_face[(size_t)ff * nvars + v], gb = grad_phi_face[(size_t)bf * nvars + v];
          double g;
          if (lim < 3) {
            g = 0.;
            if (gb != 0.) g += 0.5 * (limiter(lim, gf / gb) * gb);
            if (gf != 0.) g += 0.5 * (limiter(lim, gb / gf) * gf);
          } else {
            g = flux_limiter_g(lim, gf, gb, phi_lag[(size_t)c * nvars + v], phi_lag[(size_t)fc * nvars + v],
                               phi_lag[(size_t)bc * nvars + v], h_cell[c], h_cell[fc], h_cell[bc]);
          }
          grad_phi[(size_t)c * nvars + v] = g;
        }
        if (!pente_borne) continue;
        // R:380-431: the pente-borne fluxes leaving the cell through its back
        // (type 0) and front (type 1) faces; the dual flux computed there is
        // overwritten by computeUremap (R:752), so it is not formed here
        const double out_ar = dot(outer_face_normal[6 * c + lb], dirproj) * face_normal_velocity[bf];
        const double out_av = dot(outer_face_normal[6 * c + lf], dirproj) * face_normal_velocity[ff];
        compute_flux_pp(c, fc, bc, out_ar, deltat, 0, voisinage_pure, &delta_phi_face_ar[(size_t)c * nvars]);
        compute_flux_pp(c, fc, bc, out_av, deltat, 1, voisinage_pure, &delta_phi_face_av[(size_t)c * nvars]);
      }
      return;
    }
#pragma omp parallel for schedule(static)
    for (long c = 0; c < C; ++c) {
      long cf[6]; cell_faces(c, cf);
      long bf = cf[back_local_face(idir)], ff = cf[front_local_face(idir)];
      for (int v = 0; v < nvars; ++v) {
        double g = 0.;
        double gb = grad_phi_face[(size_t)bf * nvars + v], gf = grad_phi_face[(size_t)ff * nvars + v];
        if (gb != 0.) g += 0.5 * (limiter(limiteur_id, gf / gb) * gb);
        if (gf != 0.) g += 0.5 * (limiter(limiteur_id, gb / gf) * gf);
        grad_phi[(size_t)c * nvars + v] = g;
      }
    }
  }

  // the cell next to c along d in direction s (+1 / -1), or c on the boundary
  long along(long c, int d, int s) const {
    int i, j, k; cijk(c, i, j, k);
    int* id = d == 0 ? &i : (d == 1 ? &j : &k);
    const int t = *id + s;
    if (t < 0 || t >= ncell_dir(d)) return c;
    *id = t;
    return cid(i, j, k);
  }

  void computeUpwindFaceQuantitiesForProjection(int idir) {  // R:530-581, its specialisation _PBorn0_O2 R:658-720
    std::fill(phi_face.begin(), phi_face.end(), 0.0);
    if (ordre_projection == 3) {  // R:583-641
      const double deltat = global_deltat;
      const int nbmat = K;
#pragma omp parallel for schedule(static)
      for (long f = face_begin(idir); f < face_end(idir); ++f) {
        long cb, cf;
        if (!face_prev_next(f, idir, cb, cf)) continue;
        const long cbb = along(cb, idir, -1), cbbb = along(cbb, idir, -1);
        const long cff = along(cf, idir, +1), cfff = along(cff, idir, +1);
        const double vdt = face_normal_velocity[f] * deltat;
        double* pf = &phi_face[(size_t)f * nvars];
        auto ph = [&](long c, int v) { return phi_lag[(size_t)c * nvars + v]; };
        for (int v = 0; v < nvars; ++v)
          pf[v] = flux_ordre3(ph(cbbb, v), ph(cbb, v), ph(cb, v), ph(cf, v), ph(cff, v), ph(cfff, v), h_cell[cbbb],
                              h_cell[cbb], h_cell[cb], h_cell[cf], h_cell[cff], h_cell[cfff], vdt);
        const bool voisinage_pure = (est_mixte[cb] == 0 && est_mixte[cf] == 0 && est_pure[cb] == est_pure[cf]);
        if (!voisinage_pure) {
          for (int imat = 0; imat < nbmat; imat++) {
            if (vdt > 0. && ph(cb, imat) != 0. && ph(cb, nbmat + imat) != 0.) {
              pf[nbmat + imat] = (ph(cb, nbmat + imat) / ph(cb, imat)) * pf[imat];
              pf[2 * nbmat + imat] = (ph(cb, 2 * nbmat + imat) / ph(cb, nbmat + imat)) * pf[nbmat + imat];
            } else if (vdt < 0. && ph(cf, imat) != 0. && ph(cf, nbmat + imat) != 0.) {
              pf[nbmat + imat] = (ph(cf, nbmat + imat) / ph(cf, imat)) * pf[imat];
              pf[2 * nbmat + imat] = (ph(cf, 2 * nbmat + imat) / ph(cf, nbmat + imat)) * pf[nbmat + imat];
            }
          }
        }
      }
      return;
    }
    if (pente_borne) {  // R:574-578: the flux out of the previous cell minus the flux out of the next
#pragma omp parallel for schedule(static)
      for (long f = face_begin(idir); f < face_end(idir); ++f) {
        long cb, cf;
        if (!face_prev_next(f, idir, cb, cf)) continue;
        for (int v = 0; v < nvars; ++v)
          phi_face[(size_t)f * nvars + v] =
              delta_phi_face_av[(size_t)cb * nvars + v] - delta_phi_face_ar[(size_t)cf * nvars + v];
      }
      return;
    }
    const double order2 = (double)(ordre_projection - 1);
#pragma omp parallel for schedule(static)
    for (long f = face_begin(idir); f < face_end(idir); ++f) {
      long pc, nc;
      if (!face_prev_next(f, idir, pc, nc)) continue;
      long up = (face_normal_velocity[f] * deltax[f] > 0.0 ? pc : nc);
      double dot_xf = dot(face_coord[f] - cell_coord[up], face_normal[f]);
      for (int v = 0; v < nvars; ++v)
        phi_face[(size_t)f * nvars + v] = phi_lag[(size_t)up * nvars + v] + order2 * dot_xf * grad_phi[(size_t)up * nvars + v];
    }
  }

  void computeUremap(int idir) {  // R:733-840 (pente-borne), its specialisation computeUremap_PBorn0 R:883-1040
    const double deltat = global_deltat;
    const int nbmat = K;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < C; ++c) {
      long cf[6]; cell_faces(c, cf);
      for (int v = 0; v < nvars; ++v) {
        double& dpf = dual_phi_flux[(size_t)c * nvars + v];
        dpf = 0.;
        double flux = 0., flux_face = 0.;
        for (int a = 0; a < 6; ++a) {
          long f = cf[a];
          if (std::fabs(comp(face_normal[f], idir)) >= 1.0E-10) {
            double u = face_normal_velocity[f];
            double len = comp(face_length[f], idir);
            R3 ofn = outer_face_normal[6 * c + a];
            double od = comp(ofn, idir);
            // pente-borne (R:770-774): Phi_f already holds the integrated flux
            flux = pente_borne ? od * len * phi_face[(size_t)f * nvars + v]
                               : od * u * len * deltat * phi_face[(size_t)f * nvars + v];
            flux_face += flux;
            dpf += 0.5 * flux * comp(ofn, idir);
          }
        }
        u_lag[(size_t)c * nvars + v] = u_lag[(size_t)c * nvars + v] - flux_face;
      }
    }
#pragma omp parallel for schedule(static)
    for (long c = 0; c < C; ++c) {
      double* U = &u_lag[(size_t)c * nvars];
      double* P = &phi_lag[(size_t)c * nvars];
      for (int m = 0; m < nbmat; ++m) {
        if (U[nbmat + m] < 0.) U[nbmat + m] = 0.;
        if (U[2 * nbmat + m] < 0.) U[2 * nbmat + m] = 0.;
      }
      double somme_volume = 0.;
      for (int m = 0; m < nbmat; ++m) somme_volume += U[m];
      if (pente_borne) {  // R:805-834: volume fractions, densities, velocity (x, y), specific energies
        double somme_masse = 0.;
        for (int m = 0; m < nbmat; ++m) {
          P[m] = U[m] / somme_volume;
          if (U[m] != 0.) P[nbmat + m] = U[nbmat + m] / U[m];
          else P[nbmat + m] = 0.;
          somme_masse += U[nbmat + m];
        }
        if (somme_masse != 0) {
          P[3 * nbmat] = U[3 * nbmat] / somme_masse;
          P[3 * nbmat + 1] = U[3 * nbmat + 1] / somme_masse;
        }
        for (int m = 0; m < nbmat; ++m) {
          if (U[nbmat + m] != 0.) P[2 * nbmat + m] = U[2 * nbmat + m] / U[nbmat + m];
          else P[2 * nbmat + m] = 0.;
        }
      } else {
        for (int v = 0; v < nvars; ++v) P[v] = U[v] / somme_volume;
      }
      int imatcell = 0, imatpure = -1;
      for (int m = 0; m < nbmat; ++m) {
        if (P[m] > 0.) { imatcell++; imatpure = m; }
        if (imatcell > 1) { est_mixte[c] = 1; est_pure[c] = -1; } else { est_mixte[c] = 0; est_pure[c] = imatpure; }
      }
    }
  }

  bool node_inner(long n, int d) const {
    int i, j, k; nijk(n, i, j, k);
    int id = d == 0 ? i : (d == 1 ? j : k);
    return id > 0 && id < ncell_dir(d);
  }
  long node_shift(long n, int d, int s) const {  // neighbour along d, -1 if outside
    int i, j, k; nijk(n, i, j, k);
    int idx[3] = {i, j, k};
    idx[d] += s;
    if (idx[d] < 0 || idx[d] > ncell_dir(d)) return -1;
    return nid(idx[0], idx[1], idx[2]);
  }

  void computeDualGradPhi_LimC(int idir) {  // D:700-779
#pragma omp parallel for schedule(static)
    for (long n = 0; n < N; ++n) {
      if (!node_inner(n, idir)) continue;
      long bn = node_shift(n, idir, -1), fn = node_shift(n, idir, +1);
      const double* Pn = &phi_dual[(size_t)n * nvars];
      const double* Pb = &phi_dual[(size_t)bn * nvars];
      const double* Pf = &phi_dual[(size_t)fn * nvars];
      double xn = comp(node_coord[n], idir), xb = comp(node_coord[bn], idir), xf = comp(node_coord[fn], idir);
      double gf[3], gb[3];
      for (int a = 0; a < 3; ++a) { gf[a] = (Pf[a] - Pn[a]) / (xf - xn); gb[a] = (Pn[a] - Pb[a]) / (xn - xb); }
      for (int a = 0; a < 3; ++a) {
        double& G = dual_grad_phi[(size_t)n * nvars + a];
        G = 0.;
        if (gb[a] != 0.) G += 0.5 * limiter(limiteur_id, gf[a] / gb[a]) * gb[a];
        if (gf[a] != 0.) G += 0.5 * limiter(limiteur_id, gb[a] / gf[a]) * gf[a];
      }
    }
  }

  // D:48-64 with computeDualGradPhi (UtilesRemap.cc:15-80) and
  // computeAndLimitGradPhiDual (UtilesRemap.cc:346-377): every gradient
  // zeroed, then the inner nodes' first three components by fluxLimiterG on
  // the dual cell widths.
  void computeDualGradPhi_G(int idir) {
    std::fill(dual_grad_phi.begin(), dual_grad_phi.end(), 0.0);
#pragma omp parallel for schedule(static)
    for (long n = 0; n < N; ++n) {
      if (!node_inner(n, idir)) continue;
      const long bn = node_shift(n, idir, -1), fn = node_shift(n, idir, +1);
      const long bbn = node_shift(bn, idir, -1), ffn = node_shift(fn, idir, +1);
      const double* Pn = &phi_dual[(size_t)n * nvars];
      const double* Pb = &phi_dual[(size_t)bn * nvars];
      const double* Pf = &phi_dual[(size_t)fn * nvars];
      const double xn = comp(node_coord[n], idir), xb = comp(node_coord[bn], idir), xf = comp(node_coord[fn], idir);
      double gf[3], gb[3];
      for (int a = 0; a < 3; ++a) { gf[a] = (Pf[a] - Pn[a]) / (xf - xn); gb[a] = (Pn[a] - Pb[a]) / (xn - xb); }
      const double h0 = 0.5 * (xf - xb);
      double hmoins, hplus;
      if (bbn < 0) { hmoins = 0.; hplus = 0.5 * (comp(node_coord[ffn], idir) - xn); }
      else if (ffn < 0) { hplus = 0.; hmoins = 0.5 * (xn - comp(node_coord[bbn], idir)); }
      else { hmoins = 0.5 * (xn - comp(node_coord[bbn], idir)); hplus = 0.5 * (comp(node_coord[ffn], idir) - xn); }
      for (int a = 0; a < 3; ++a)
        dual_grad_phi[(size_t)n * nvars + a] = flux_limiter_g(limiteur_id, gf[a], gb[a], Pn[a], Pf[a], Pb[a], h0, hplus, hmoins);
    }
  }

  void computeDualUremap(int idir) {  // D:22-676 (#else at :127, #if 1 at :351)
    const double deltat = global_deltat;
    const int nb_env = K;
    if (ordre_projection > 1) {
      if (limiteur_id < 3) computeDualGradPhi_LimC(idir);
      else computeDualGradPhi_G(idir);
    }
    // fcontrib, D:129-189
    const double oneovernbcell = 0.25;
    for (long f = face_begin(idir); f < face_end(idir); ++f) {
      long pc, nc; face_prev_next(f, idir, pc, nc);
      if (pc >= 0) for (int k = 0; k < nb_env; ++k)
        back_flux_contrib_env[(size_t)pc * K + k] = oneovernbcell * dual_phi_flux[(size_t)pc * nvars + nb_env + k];
      if (nc >= 0) for (int k = 0; k < nb_env; ++k)
        front_flux_contrib_env[(size_t)nc * K + k] = oneovernbcell * dual_phi_flux[(size_t)nc * nvars + nb_env + k];
    }
    // ncontrib 3D, D:262-342
    const int dir1 = (idir + 1) % 3, dir2 = (idir + 2) % 3;
#pragma omp parallel for schedule(static)
    for (long n = 0; n < N; ++n) {
      int idx[3]; nijk(n, idx[0], idx[1], idx[2]);
      for (int k = 0; k < nb_env; ++k) { back_flux_mass_env[(size_t)n * K + k] = 0.; front_flux_mass_env[(size_t)n * K + k] = 0.; }
      back_flux_mass[n] = 0.; front_flux_mass[n] = 0.;
      for (int s1 = -1; s1 <= 0; ++s1)
        for (int s2 = -1; s2 <= 0; ++s2) {
          int ci[3] = {idx[0], idx[1], idx[2]};
          ci[idir] -= 1; ci[dir1] += s1; ci[dir2] += s2;
          if (ci[0] >= 0 && ci[0] < nx && ci[1] >= 0 && ci[1] < ny && ci[2] >= 0 && ci[2] < nz) {
            long c = cid(ci[0], ci[1], ci[2]);
            for (int k = 0; k < nb_env; ++k) {
              back_flux_mass_env[(size_t)n * K + k] += back_flux_contrib_env[(size_t)c * K + k];
              back_flux_mass[n] += back_flux_contrib_env[(size_t)c * K + k];
            }
          }
        }
      for (int s1 = -1; s1 <= 0; ++s1)
        for (int s2 = -1; s2 <= 0; ++s2) {
          int ci[3] = {idx[0], idx[1], idx[2]};
          ci[dir1] += s1; ci[dir2] += s2;
          if (ci[0] >= 0 && ci[0] < nx && ci[1] >= 0 && ci[1] < ny && ci[2] >= 0 && ci[2] < nz) {
            long c = cid(ci[0], ci[1], ci[2]);
            for (int k = 0; k < nb_env; ++k) {
              front_flux_mass_env[(size_t)n * K + k] += front_flux_contrib_env[(size_t)c * K + k];
              front_flux_mass[n] += front_flux_contrib_env[(size_t)c * K + k];
            }
          }
        }
    }
    // dual momentum / kinetic-energy update on inner nodes, D:352-492
    const double order2 = (double)(ordre_projection - 1);
#pragma omp parallel for schedule(static)
    for (long n = 0; n < N; ++n) {
      if (!node_inner(n, idir)) continue;
      long bn = node_shift(n, idir, -1), fn = node_shift(n, idir, +1);
      double* Ud = &u_dual[(size_t)n * nvars];
      const double* Pn = &phi_dual[(size_t)n * nvars];
      const double* Pb = &phi_dual[(size_t)bn * nvars];
      const double* Pf = &phi_dual[(size_t)fn * nvars];
      const double* Gn = &dual_grad_phi[(size_t)n * nvars];
      const double* Gb = &dual_grad_phi[(size_t)bn * nvars];
      const double* Gf = &dual_grad_phi[(size_t)fn * nvars];
      const double bfm = back_flux_mass[n], ffm = front_flux_mass[n];
      const double xn = comp(node_coord[n], idir), xb = comp(node_coord[bn], idir), xf = comp(node_coord[fn], idir);
      Ud[3] += bfm - ffm;
      double FV[3], BV[3], FE, BE;
      int signfront;
      double ufront = 0.5 * (Pn[idir] + Pn[idir]);   // D:391, the node's own value twice
      if (ufront > 0) signfront = 1; else signfront = -1;
      const double* PF = (ffm < 0.) ? Pf : Pn;
      const double* GF = (ffm < 0.) ? Gf : Gn;
      for (int a = 0; a < 3; ++a)
        FV[a] = PF[a] + order2 * (0.5 * GF[a] * (signfront * (xf - xn) - deltat * ufront));
      FE = PF[4] + order2 * (0.5 * GF[4] * (signfront * (xf - xn) - deltat * ufront));
      int signback;
      double uback = 0.5 * (Pb[idir] + Pn[idir]);
      if (uback > 0) signback = 1; else signback = -1;
      const double* PB = (bfm > 0.) ? Pb : Pn;
      const double* GB = (bfm > 0.) ? Gb : Gn;
      for (int a = 0; a < 3; ++a)
        BV[a] = PB[a] + order2 * (0.5 * GB[a] * (signback * (xn - xb) - deltat * uback));
      BE = PB[4] + order2 * (0.5 * GB[4] * (signback * (xn - xb) - deltat * uback));
      for (int a = 0; a < 3; ++a) Ud[a] += bfm * BV[a] - ffm * FV[a];
      Ud[4] += bfm * BE - ffm * FE;
    }
    // filter and Phi_dual, D:494-523
    const double thresold = 1.e-300;
#pragma omp parallel for schedule(static)
    for (long n = 0; n < N; ++n) {
      if (!node_inner(n, idir)) continue;
      double* Ud = &u_dual[(size_t)n * nvars];
      double* Pd = &phi_dual[(size_t)n * nvars];
      if (std::fabs(Ud[0]) < thresold) Ud[0] = 0.;
      if (std::fabs(Ud[1]) < thresold) Ud[1] = 0.;
      if (std::fabs(Ud[2]) < thresold) Ud[2] = 0.;
      Pd[0] = Ud[0] / Ud[3]; Pd[1] = Ud[1] / Ud[3]; Pd[2] = Ud[2] / Ud[3];
      Pd[3] = Ud[3];
      Pd[4] = Ud[4] / Ud[3];
    }
  }

  void remapVariables() {  // F:19-778 (#else branches)
    const int nb_env = K;
    // environment add/remove, F:94-226, statuses from the membership before the update
    std::vector<uint32_t> new_mask(env_mask);
    bool changed = false;
    for (int k = 0; k < nb_env; ++k) {
      for (long c = 0; c < C; ++c) {
        const double* U = &u_lag[(size_t)c * nvars];
        double fvol = U[k] / euler_volume[c];
        bool in_env = env_mask[c] >> k & 1;
        int st = 0;
        if (fvol < threshold && in_env) st = -1;
        else if (fvol > threshold && !in_env) {
          double volt = 0.;
          for (int kk = 0; kk < nb_env; ++kk) volt += U[kk];
          double f2 = U[k] / volt;
          if (f2 > threshold && U[nb_env + k] != 0.) st = +1;
        }
        if (st < 0) { new_mask[c] &= ~(1u << k); changed = true; }
        if (st > 0) { new_mask[c] |= 1u << k; changed = true; }
      }
    }
    if (changed) {
      // New partial slots start at zero; every value the step reads later is
      // written first (see the "moy" kernel below and the EOS).
      for (long c = 0; c < C; ++c) {
        if (new_mask[c] == env_mask[c]) continue;
        bool was_pure = nbEnv(c) == 1;
        int old_e = was_pure ? env_id[c] : -1;
        env_mask[c] = new_mask[c];
        bool now_pure = nbEnv(c) == 1;
        if (was_pure && !now_pure) {
          // the old pure environment's values move to its partial slot
          MatVar* vs[] = {&density, &internal_energy, &pressure, &sound_speed, &pseudo_viscosity, &cell_volume,
                          &cell_mass, &fracvol, &mass_fraction, &dpde, &tau_density, &density_n, &internal_energy_n,
                          &pressure_n, &cell_volume_n, &pseudo_viscosity_n, &pseudo_viscosity_nmoins1};
          for (MatVar* v : vs) {
            for (int k = 0; k < K; ++k) v->p[k][c] = 0.;
            if (old_e >= 0 && (env_mask[c] >> old_e & 1)) v->p[old_e][c] = v->g[c];
          }
        } else if (!was_pure && now_pure) {
          int ne = __builtin_ctz(env_mask[c]);
          MatVar* vs[] = {&density, &internal_energy, &pressure, &sound_speed, &pseudo_viscosity, &cell_volume,
                          &cell_mass, &fracvol, &mass_fraction, &dpde, &tau_density, &density_n, &internal_energy_n,
                          &pressure_n, &cell_volume_n, &pseudo_viscosity_n, &pseudo_viscosity_nmoins1};
          for (MatVar* v : vs) v->g[c] = v->p[ne][c];
        } else if (!now_pure) {
          MatVar* vs[] = {&density, &internal_energy, &pressure, &sound_speed, &pseudo_viscosity, &cell_volume,
                          &cell_mass, &fracvol, &mass_fraction, &dpde, &tau_density, &density_n, &internal_energy_n,
                          &pressure_n, &cell_volume_n, &pseudo_viscosity_n, &pseudo_viscosity_nmoins1};
          for (int k = 0; k < K; ++k)
            if ((new_mask[c] >> k & 1) && !(env_mask_prev_bit(c, k)))
              for (MatVar* v : vs) v->p[k][c] = 0.;
        }
      }
      compute_env_id();
    }
    // "moy" kernel, F:406-644
    const double thr = threshold;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < C; ++c) {
      const double* U = &u_lag[(size_t)c * nvars];
      const double vol = euler_volume[c];
      cell_volume.g[c] = vol;
      double volt = 0., masset = 0.;
      for (int k = 0; k < nb_env; ++k) { volt += U[k]; masset += U[nb_env + k]; }
      double volt_normalise = 0.;
      const double unsurvolt = 1. / volt;
      for (int k = 0; k < nb_env; ++k) volt_normalise += U[k] * vol * unsurvolt;
      (void)volt_normalise;
      double somme_frac = 0.;
      const double unsurvol = 1. / vol;
      for (int k = 0; k < K; ++k) if (env_mask[c] >> k & 1) {
        double fvol = U[k] * unsurvolt;
        if (fvol < thr) fvol = 0.;
        mv(fracvol, k, c) = fvol;
        somme_frac += fvol;
      }
      int matcell = 0, imatpure = -1;
      const double unsursomme_frac = 1. / somme_frac;
      for (int k = 0; k < K; ++k) if (env_mask[c] >> k & 1) {
        double fvol = mv(fracvol, k, c) * unsursomme_frac;
        if (fvol > 0.) { matcell++; imatpure = k; }
        mv(fracvol, k, c) = fvol;
      }
      if (matcell > 1) { est_mixte[c] = 1; est_pure[c] = -1; } else { est_mixte[c] = 0; est_pure[c] = imatpure; }
      double fmasset = 0.;
      if (masset != 0.) {
        const double unsurmasset = 1. / masset;
        for (int k = 0; k < K; ++k) if (env_mask[c] >> k & 1) {
          double mf = U[nb_env + k] * unsurmasset;
          if (mv(fracvol, k, c) < thr) mf = 0.;
          fmasset += mf;
          mv(mass_fraction, k, c) = mf;
        }
        if (fmasset != 0.) {
          const double unsurfmasset = 1. / fmasset;
          for (int k = 0; k < K; ++k) if (env_mask[c] >> k & 1) mv(mass_fraction, k, c) = mv(mass_fraction, k, c) * unsurfmasset;
        }
      }
      double density_nplus1 = 0.;
      for (int k = 0; k < K; ++k) if (env_mask[c] >> k & 1) {
        double de = 0.;
        double fvol = mv(fracvol, k, c);
        if (fvol > thr) {
          double vn = U[k] * vol * unsurvolt;
          de = U[nb_env + k] / vn;
        }
        mv(density, k, c) = de;
        density_nplus1 += fvol * de;
      }
      if (est_mixte[c]) density.g[c] = density_nplus1;
      cell_mass.g[c] = euler_volume[c] * density_nplus1;
      double energie_nplus1 = 0., pseudo_nplus1 = 0.;
      for (int k = 0; k < K; ++k) if (env_mask[c] >> k & 1) {
        double fvol = mv(fracvol, k, c);
        double mf = mv(mass_fraction, k, c);
        double ee = 0.;
        if (fvol > thr && U[nb_env + k] != 0.) ee = U[2 * nb_env + k] / U[nb_env + k];
        mv(internal_energy, k, c) = ee;
        energie_nplus1 += mf * ee;
        mv(cell_mass, k, c) = mf * cell_mass.g[c];
        double pv = U[3 * nb_env + 4] * unsurvol;
        mv(pseudo_viscosity, k, c) = pv;
        pseudo_nplus1 += fvol * pv;
      }
      internal_energy.g[c] = energie_nplus1;
      pseudo_viscosity.g[c] = pseudo_nplus1;
      for (int k = 0; k < K; ++k) if (env_mask[c] >> k & 1) {
        if (mv(density, k, c) < 0. || mv(internal_energy, k, c) < 0.) {
          mv(internal_energy, k, c) = 0.; mv(density, k, c) = 0.; mv(fracvol, k, c) = 0.; mv(mass_fraction, k, c) = 0.;
        }
      }
    }
    // node velocity, F:660-672
#pragma omp parallel for schedule(static)
    for (long n = 0; n < N; ++n) {
      const double* Ud = &u_dual[(size_t)n * nvars];
      double m = Ud[3];
      if (m != 0.) velocity[n] = r3(Ud[0] / m, Ud[1] / m, Ud[2] / m);
    }
    computeNodeMass();                                                  // F:697-719
#pragma omp parallel for schedule(static)
    for (long c = 0; c < C; ++c) {                                      // F:721-744
      if (nbEnv(c) == 1) continue;
      for (int k = 0; k < K; ++k) if (env_mask[c] >> k & 1) cell_volume.p[k][c] = fracvol.p[k][c] * cell_volume.g[c];
    }
    // conservation-energie-totale (RemapADI.axl:151), F:751-773: the kinetic
    // energy the dual remap carried (U_dual[4] / U_dual[3]) minus the kinetic
    // energy of the remapped velocity, 0.25 per node over the cell's 8 nodes in
    // cell-node order (only nodes of non-zero mass), floored at 0, goes into
    // the specific internal energy: e_k += x_k delta on every environment cell
    // and, in a mixed cell, the mean e += delta.  U_dual[4] is 0.5 m |v|
    // (PrepareRemap.cc:421), not 0.5 m |v|^2; the reference's quirk is kept.
    if (conservation_energie_totale) {
#pragma omp parallel for schedule(static)
      for (long c = 0; c < C; ++c) {
        long cn[8];
        cell_nodes(c, cn);
        double delta_ec = 0.;
        for (int a = 0; a < 8; ++a) {
          const double* Ud = &u_dual[(size_t)cn[a] * nvars];
          if (Ud[3] != 0.) {
            const double ec_proj = Ud[4] / Ud[3];
            const R3 v = velocity[cn[a]];
            const double ec_reconst = 0.5 * (v.x * v.x + v.y * v.y + v.z * v.z);   // squareNormL2
            delta_ec += 0.25 * (ec_proj - ec_reconst);
          }
        }
        delta_ec = smax(0., delta_ec);                                  // std::max(0., delta_ec)
        for (int k = 0; k < K; ++k) if (env_mask[c] >> k & 1) mv(internal_energy, k, c) += mv(mass_fraction, k, c) * delta_ec;
        if (nbEnv(c) != 1) internal_energy.g[c] += delta_ec;
      }
    }
  }
  std::vector<uint32_t> prev_mask_scratch;
  bool env_mask_prev_bit(long c, int k) const { return !prev_mask_scratch.empty() && (prev_mask_scratch[c] >> k & 1); }

  // applyEOS for every environment: PerfectGas E:50-137, StiffenedGas
  // (eos/stiffenedgas/StiffenedGasEOSService.cc:29-44)
  void applyEOS() {
#pragma omp parallel for schedule(static)
    for (long c = 0; c < C; ++c) {
      for (int k = 0; k < K; ++k) {
        if (!(env_mask[c] >> k & 1)) continue;
        const double g = gamma[k];
        double r = mv(density, k, c), e = mv(internal_energy, k, c);
        if (eos[k] == 1) {
          const double pi = pinf[k];
          double p = ((g - 1.) * r * e) - (g * pi);
          mv(pressure, k, c) = p;
          mv(sound_speed, k, c) = std::sqrt((g / r) * (p + pi));
        } else {
          double p = (g - 1.) * r * e;
          mv(pressure, k, c) = p;
          mv(sound_speed, k, c) = std::sqrt(g * p / r);
        }
        mv(dpde, k, c) = (g - 1.) * r;
      }
    }
  }

  void computePressionMoyenne() {  // M:1836-1915 (#else)
#pragma omp parallel for schedule(static)
    for (long c = 0; c < C; ++c) {
      if (env_id[c] >= 0) continue;
      pressure.g[c] = 0.;
      sound_speed.g[c] = 1.e-20;
      for (int k = 0; k < K; ++k) if (env_mask[c] >> k & 1) {
        pressure.g[c] += fracvol.p[k][c] * pressure.p[k][c];
        sound_speed.g[c] = amax(sound_speed.p[k][c], sound_speed.g[c]);
      }
    }
  }

  void remap() {  // P:448-563
    if (schema_csts) updateVelocityForward();             // P:456
    computeVariablesForRemap();
    computeFaceQuantitesForRemap();
    // IRemap::appliRemap, R:19-60
    for (int i = 0; i < 3; ++i) {
      int idir = (i + sens_projection) % 3;
      computeGradPhiFace(idir);
      computeGradPhiCell(idir);
      computeUpwindFaceQuantitiesForProjection(idir);
      computeUremap(idir);
      computeDualUremap(idir);
    }
    sens_projection = (sens_projection + 1) % 3;
    prev_mask_scratch = env_mask;
    remapVariables();
    prev_mask_scratch.clear();
    // reset of the n-level fields, P:485-550
#pragma omp parallel for schedule(static)
    for (long c = 0; c < C; ++c) {
      pseudo_viscosity_n.g[c] = 0.; pressure_n.g[c] = 0.; cell_volume_n.g[c] = 0.;
      density_n.g[c] = 0.; internal_energy_n.g[c] = 0.; tau_density.g[c] = 0.;
      int e = env_id[c];
      materiau[c] = 0;
      if (e >= 0) materiau[c] = e * fracvol.g[c];
      else
        for (int k = 0; k < K; ++k) if (env_mask[c] >> k & 1) {
          pseudo_viscosity_n.p[k][c] = 0.; pressure_n.p[k][c] = 0.; cell_volume_n.p[k][c] = 0.;
          density_n.p[k][c] = 0.; internal_energy_n.p[k][c] = 0.; tau_density.p[k][c] = 0.;
          materiau[c] += k * fracvol.p[k][c];
        }
    }
    applyEOS();
    computePressionMoyenne();
  }

  // computeHydroDeltaT M:2027-2071 over the cells of layers [dt_k0, dt_k1)
  double hydroDeltaTMin() {
    double minimum_aux = std::numeric_limits<double>::max();
    const long c0 = (long)dt_k0 * nx * ny, c1 = dt_k1 < 0 ? C : (long)dt_k1 * nx * ny;
#pragma omp parallel
    {
      double lmin = std::numeric_limits<double>::max();
#pragma omp for schedule(static)
      for (long c = c0; c < c1; ++c) {
        long cn[8]; cell_nodes(c, cn);
        double vmax = 0.;
        for (int a = 0; a < 8; ++a) vmax = amax(normL2(velocity[cn[a]]), vmax);
        double dx_sound = car_len[c] / (sound_speed.g[c] + vmax);
        lmin = amin(lmin, dx_sound);
      }
#pragma omp critical
      minimum_aux = amin(minimum_aux, lmin);
    }
    return minimum_aux;
  }

  void computeDeltaT() { finishDeltaT(hydroDeltaTMin()); }   // M:2076-2191

  void finishDeltaT(double minimum_aux) {
    global_old_deltat = global_deltat;
    old_deltat = global_old_deltat;
    double new_dt = cfl * minimum_aux;
    new_dt = amin(new_dt, 1.05 * global_old_deltat);
    new_dt = amin(new_dt, deltat_max);
    if (new_dt < deltat_min) status |= 1u;                             // reference: exit(1)
    global_deltat = new_dt;
    if (global_time > final_time) status |= 2u;                        // stopComputeLoop, dt not trimmed
  }

  void cycle() {
    saveValuesAtN();
    updateVelocity();
    applyBoundaryCondition();
    updatePosition();
    computeGeometricValues();
    updateDensity();
    computeArtificialViscosity();
    updateEnergyAndPressure();
    remap();
    global_time += global_deltat;
    if (ext_dt) { local_min = hydroDeltaTMin(); return; }       // orc_dt_finish completes the cycle
    computeDeltaT();
    ++iteration;
  }

  // slabs: the state a cycle starts from for cell layers [clo, chi) and
  // node layers [nlo, nhi), field by field; pack (to buf) or unpack
  template <class F>
  void halo_fields(int clo, int chi, int nlo, int nhi, F&& f) {
    const long cl = (long)nx * ny, nl = (long)NX * NY;
    const long c0 = clo * cl, c1 = chi * cl, n0 = nlo * nl, n1 = nhi * nl;
    MatVar* cv[] = {&density, &internal_energy, &pressure, &sound_speed, &pseudo_viscosity, &cell_mass};
    for (MatVar* v : cv) for (long c = c0; c < c1; ++c) f(v->g[c]);
    for (long c = c0; c < c1; ++c) for (int a = 0; a < 8; ++a) { f(cqs[8 * c + a].x); f(cqs[8 * c + a].y); f(cqs[8 * c + a].z); }
    for (long n = n0; n < n1; ++n) { f(velocity[n].x); f(velocity[n].y); f(velocity[n].z); }
    for (long n = n0; n < n1; ++n) f(node_mass[n]);
    for (long n = n0; n < n1; ++n) for (int v = 0; v < nvars; ++v) f(dual_grad_phi[(size_t)n * nvars + v]);
    if (K > 1) {
      // several environments: membership, every environment's values, the
      // global fractions, the mixed/pure indicators and Phi (the pente-borne
      // Phi of absent environments outlives a cycle); integers travel as
      // doubles, exactly
      for (long c = c0; c < c1; ++c) {
        double m = (double)env_mask[c], e = (double)env_id[c];
        f(m); f(e);
        env_mask[c] = (uint32_t)m; env_id[c] = (int)e;
      }
      MatVar* ev[] = {&fracvol, &mass_fraction, &density, &internal_energy, &pressure, &sound_speed,
                      &pseudo_viscosity, &cell_mass};
      for (MatVar* v : ev) {
        if (v == &fracvol || v == &mass_fraction) for (long c = c0; c < c1; ++c) f(v->g[c]);
        for (int k = 0; k < K; ++k) for (long c = c0; c < c1; ++c) f(v->p[k][c]);
      }
      for (long c = c0; c < c1; ++c) {
        double m = (double)est_mixte[c], e = (double)est_pure[c];
        f(m); f(e);
        est_mixte[c] = (int)m; est_pure[c] = (int)e;
      }
      for (long c = c0; c < c1; ++c) for (int v = 0; v < nvars; ++v) f(phi_lag[(size_t)c * nvars + v]);
    }
  }
};

}  // namespace

// ---------------- C interface for the test harness (ctypes) ----------------
extern "C" {

struct orc_bc { int surface; int type; double value; };

void* orc_create(int nx, int ny, int nz, const double* node_coords, int nenv, const double* gammas,
                 double cfl, double threshold, double deltat_init, double deltat_min, double deltat_max,
                 double final_time, int lc_mode, int pseudo_centree, int ordre_projection, int limiteur_id,
                 int nbc, const orc_bc* bcs, int use_project_pow, const int* eos, const double* pinf,
                 int with_newton, int schema_csts, int pente_borne, int pb_debar_fix, int pb_mixte,
                 int limiteur_pure_id) {
  Oracle* o = new Oracle();
  o->nx = nx; o->ny = ny; o->nz = nz; o->NX = nx + 1; o->NY = ny + 1; o->NZ = nz + 1;
  o->C = (long)nx * ny * nz; o->N = (long)o->NX * o->NY * o->NZ;
  o->Fx = (long)(nx + 1) * ny * nz; o->Fy = (long)nx * (ny + 1) * nz; o->Fz = (long)nx * ny * (nz + 1);
  o->F = o->Fx + o->Fy + o->Fz;
  o->K = nenv; o->nvars = 3 * nenv + 5;
  o->cfl = cfl; o->threshold = threshold; o->deltat_init = deltat_init; o->deltat_min = deltat_min;
  o->deltat_max = deltat_max; o->final_time = final_time; o->lc_mode = lc_mode; o->pseudo_centree = pseudo_centree;
  o->ordre_projection = ordre_projection; o->limiteur_id = limiteur_id; o->use_project_pow = use_project_pow;
  o->with_newton = with_newton;
  o->schema_csts = schema_csts;
  o->pente_borne = pente_borne; o->pb_debar_fix = pb_debar_fix; o->pb_mixte = pb_mixte;
  o->limiteur_pure_id = limiteur_pure_id;
  o->gamma.assign(gammas, gammas + nenv);
  o->eos.assign(nenv, 0);
  o->pinf.assign(nenv, 0.);
  for (int k = 0; k < nenv; ++k) {
    if (eos) o->eos[k] = eos[k];
    if (pinf) o->pinf[k] = pinf[k];
  }
  for (int b = 0; b < nbc; ++b) o->bcs.push_back(Oracle::BC{bcs[b].surface, bcs[b].type, bcs[b].value, {}});
  const long C = o->C, N = o->N, F = o->F; const int K = nenv, nv = o->nvars;
  o->node_coord.resize(N); o->node_coord_0.resize(N); o->velocity.assign(N, r3(0, 0, 0));
  o->velocity_n.assign(N, r3(0, 0, 0)); o->force.assign(N, r3(0, 0, 0)); o->node_mass.assign(N, 0.);
  for (long n = 0; n < N; ++n) o->node_coord[n] = r3(node_coords[3 * n], node_coords[3 * n + 1], node_coords[3 * n + 2]);
  o->env_mask.assign(C, 0); o->env_id.assign(C, 0);
  MatVar* vs[] = {&o->density, &o->internal_energy, &o->pressure, &o->sound_speed, &o->pseudo_viscosity, &o->cell_volume,
                  &o->cell_mass, &o->fracvol, &o->mass_fraction, &o->dpde, &o->tau_density, &o->density_n,
                  &o->internal_energy_n, &o->pressure_n, &o->cell_volume_n, &o->pseudo_viscosity_n,
                  &o->pseudo_viscosity_nmoins1};
  for (MatVar* v : vs) v->init(K, C);
  o->div_u.assign(C, 0.); o->car_len.assign(C, 0.); o->euler_volume.assign(C, 0.); o->materiau.assign(C, 0.);
  o->cell_coord.assign(C, r3(0, 0, 0)); o->cqs.assign(8 * C, r3(0, 0, 0)); o->cqs_n.assign(8 * C, r3(0, 0, 0));
  o->face_normal.assign(F, r3(0, 0, 0)); o->face_coord.assign(F, r3(0, 0, 0)); o->face_length.assign(F, r3(0, 0, 0));
  o->outer_face_normal.assign(6 * C, r3(0, 0, 0));
  o->face_normal_velocity.assign(F, 0.); o->deltax.assign(F, 0.);
  o->u_lag.assign((size_t)C * nv, 0.); o->phi_lag.assign((size_t)C * nv, 0.); o->grad_phi.assign((size_t)C * nv, 0.);
  o->grad_phi_face.assign((size_t)F * nv, 0.); o->phi_face.assign((size_t)F * nv, 0.);
  o->dual_phi_flux.assign((size_t)C * nv, 0.);
  o->u_dual.assign((size_t)N * nv, 0.); o->phi_dual.assign((size_t)N * nv, 0.); o->dual_grad_phi.assign((size_t)N * nv, 0.);
  o->back_flux_mass.assign(N, 0.); o->front_flux_mass.assign(N, 0.);
  o->back_flux_mass_env.assign((size_t)N * K, 0.); o->front_flux_mass_env.assign((size_t)N * K, 0.);
  o->back_flux_contrib_env.assign((size_t)C * K, 0.); o->front_flux_contrib_env.assign((size_t)C * K, 0.);
  o->est_mixte.assign(C, 0); o->est_pure.assign(C, 0); o->h_cell.assign(C, 0.);
  if (pente_borne) { o->delta_phi_face_av.assign((size_t)C * nv, 0.); o->delta_phi_face_ar.assign((size_t)C * nv, 0.); }
  return o;
}

// fracvol, density, pressure: nenv*C arrays (environment-major); velocity: N*3
void orc_init(void* h, const double* fracvol, const double* density, const double* pressure, const double* velocity) {
  static_cast<Oracle*>(h)->hydroStartInit(fracvol, density, pressure, velocity);
}

void orc_step(void* h, int ncycles) {
  Oracle* o = static_cast<Oracle*>(h);
  for (int i = 0; i < ncycles; ++i) o->cycle();
}

void orc_destroy(void* h) { delete static_cast<Oracle*>(h); }

// Slabs (one environment): dt over cell layers [k_lo, k_hi), external finish.
int orc_set_dt_reduction(void* h, int k_lo, int k_hi, int external) {
  Oracle* o = static_cast<Oracle*>(h);
  if (k_lo < 0 || k_hi > o->nz || k_lo >= k_hi) return -1;
  o->dt_k0 = k_lo; o->dt_k1 = k_hi; o->ext_dt = external;
  return 0;
}
double orc_dt_local_min(void* h) { return static_cast<Oracle*>(h)->local_min; }
void orc_dt_finish(void* h, double minimum) {
  Oracle* o = static_cast<Oracle*>(h);
  o->finishDeltaT(minimum);
  ++o->iteration;
}
long orc_halo_count(void* h, int cell_layers, int node_layers) {
  long n = 0;
  static_cast<Oracle*>(h)->halo_fields(0, cell_layers, 0, node_layers, [&](double&) { ++n; });
  return n;
}
int orc_halo_pack(void* h, int clo, int chi, int nlo, int nhi, double* out) {
  Oracle* o = static_cast<Oracle*>(h);
  if (clo < 0 || chi > o->nz || clo > chi || nlo < 0 || nhi > o->nz + 1 || nlo > nhi) return -1;
  long i = 0;
  o->halo_fields(clo, chi, nlo, nhi, [&](double& v) { out[i++] = v; });
  return 0;
}
int orc_halo_unpack(void* h, int clo, int chi, int nlo, int nhi, const double* in) {
  Oracle* o = static_cast<Oracle*>(h);
  if (clo < 0 || chi > o->nz || clo > chi || nlo < 0 || nhi > o->nz + 1 || nlo > nhi) return -1;
  long i = 0;
  o->halo_fields(clo, chi, nlo, nhi, [&](double& v) { v = in[i++]; });
  return 0;
}

// Options beyond orc_create's list, by name; 0 when known, -1 otherwise.
int orc_set_option(void* h, const char* name, int value) {
  Oracle* o = static_cast<Oracle*>(h);
  if (std::strcmp(name, "conservation_energie_totale") == 0) { o->conservation_energie_totale = value; return 0; }
  return -1;
}

void orc_set_threads(int n) { omp_set_num_threads(n); }

// V^(1./3.) as the oracle evaluates it: the project cube root (project != 0)
// or std::pow, the reference's call (MahycoModule.cc:1259).
double orc_pow_third(double v, int project) { return project ? mhy::pow_third(v) : std::pow(v, 1. / 3.); }

// scalars: [dt, old_dt, time, sens, iteration, status]
void orc_get_scalars(void* h, double* out) {
  Oracle* o = static_cast<Oracle*>(h);
  out[0] = o->global_deltat; out[1] = o->global_old_deltat; out[2] = o->global_time;
  out[3] = o->sens_projection; out[4] = (double)o->iteration; out[5] = (double)o->status;
}

// field ids: 0 density, 1 internal energy, 2 pressure, 3 sound speed, 4 pseudo viscosity,
// 5 cell volume, 6 cell mass, 7 characteristic length (cells, global values);
// 10 velocity (N*3), 11 node mass, 12 node coord (N*3);
// 20+k fracvol of env k, 30+k density of env k, 40+k internal energy of env k (C, 0 outside env);
// 50 env mask (as double)
int orc_get_field(void* h, int id, double* out) {
  Oracle* o = static_cast<Oracle*>(h);
  const long C = o->C, N = o->N;
  auto gcopy = [&](const std::vector<double>& v) { std::memcpy(out, v.data(), C * sizeof(double)); };
  switch (id) {
    case 0: gcopy(o->density.g); return 0;
    case 1: gcopy(o->internal_energy.g); return 0;
    case 2: gcopy(o->pressure.g); return 0;
    case 3: gcopy(o->sound_speed.g); return 0;
    case 4: gcopy(o->pseudo_viscosity.g); return 0;
    case 5: gcopy(o->cell_volume.g); return 0;
    case 6: gcopy(o->cell_mass.g); return 0;
    case 7: gcopy(o->car_len); return 0;
    case 10: for (long n = 0; n < N; ++n) { out[3 * n] = o->velocity[n].x; out[3 * n + 1] = o->velocity[n].y; out[3 * n + 2] = o->velocity[n].z; } return 0;
    case 11: std::memcpy(out, o->node_mass.data(), N * sizeof(double)); return 0;
    case 12: for (long n = 0; n < N; ++n) { out[3 * n] = o->node_coord[n].x; out[3 * n + 1] = o->node_coord[n].y; out[3 * n + 2] = o->node_coord[n].z; } return 0;
    case 50: for (long c = 0; c < C; ++c) out[c] = (double)o->env_mask[c]; return 0;
    default: break;
  }
  if (id >= 20 && id < 50) {
    int k = id % 10; int which = id / 10;
    if (k >= o->K) return -1;
    MatVar& v = which == 2 ? o->fracvol : (which == 3 ? o->density : o->internal_energy);
    for (long c = 0; c < C; ++c) out[c] = (o->env_mask[c] >> k & 1) ? o->mv(v, k, c) : 0.;
    return 0;
  }
  return -1;
}

}  // extern "C"
