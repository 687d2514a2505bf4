// mhy_lagrange.cuh -- the Lagrange-phase cell kernel (geometry, corner
// vectors, density, pseudo-viscosity, energy, remap variables and the face
// data of the remap), templated on the number of environments K.
#pragma once

#include "mhy_kernels.cuh"

namespace mhy {

// ------------------------------------------------------------------------
// Lagrange phase, cells: UpdatePosition (cell centre), ComputeGeometricValues,
// UpdateDensity, ComputeArtificialViscosity, UpdateEnergyAndPressure (GP),
// computeVariablesForRemap_PBorn0 and computeFaceQuantitesForRemap for the
// cell's low faces, with the face-only terms of computeGradPhiFace and the
// upwind reconstruction precomputed (dx_f, (x_f - x_c).n0 for both cells).
// (MahycoModule.cc:913-928, 1054-1262, 1331-1370, 517-528, 1715-1726;
// PrepareRemap.cc:33-55, 93-117, 311-332; RemapADIService.cc:171-172, 710.)
__device__ __forceinline__ D3 load_xl(const Dims& dm, const double* __restrict__ x0, const double* __restrict__ vh,
                                      double dt, long long n) {
  return d3(x0[n], x0[dm.N + n], x0[2 * dm.N + n]) + dt * d3(vh[n], vh[dm.N + n], vh[2 * dm.N + n]);
}

// Half cross product 0.5 * (a - c) x (b - c) (MahycoModule.cc:2206-2239).
template <typename T>
__device__ __forceinline__ Vec3<T> half_cross(Vec3<T> a, Vec3<T> b, Vec3<T> c) { return T(0.5) * cross(a - c, b - c); }

// Corner vectors accumulated face by face.  Each corner's two six-term sums
// of MahycoModule.cc:2242-2257 take two consecutive terms from each of its
// three faces, in increasing face order, so adding them as the faces are
// visited keeps the reference's order; a corner is finished as soon as its
// third face is done.
template <typename T> struct CornerAcc { Vec3<T> s1, s2; };
template <typename T>
__device__ __forceinline__ void acc_start(CornerAcc<T>& a, Vec3<T> t1, Vec3<T> t2, Vec3<T> u1, Vec3<T> u2) {
  a.s1 = t1 + t2; a.s2 = u1 + u2;
}
template <typename T>
__device__ __forceinline__ void acc_add(CornerAcc<T>& a, Vec3<T> t1, Vec3<T> t2, Vec3<T> u1, Vec3<T> u2) {
  a.s1 = a.s1 + t1; a.s1 = a.s1 + t2; a.s2 = a.s2 + u1; a.s2 = a.s2 + u2;
}

// The 8 corner vectors of a hexahedron with nodes x (SN_trigo order),
// streamed: finish(a, cqs_a) is called as soon as corner a is complete
// (MahycoModule.cc:2195-2258, face centres as in :1080-1087).  T = double is
// the reference's arithmetic; T = float (mixed form) takes x relative to the
// cell centre, where every term has the size of the cell and nothing cancels.
template <typename T, typename Finish>
__device__ __forceinline__ void corner_vectors(const Vec3<T> x[8], Finish&& finish) {
  const T t12 = T(1.) / T(12.), q = T(0.25);
  auto fin = [&](int a, const CornerAcc<T>& ac) { finish(a, t12 * (T(5.) * ac.s1 + ac.s2)); };
  CornerAcc<T> k0, k1, k2, k3, k4, k5, k6, k7;
  {
    const Vec3<T> c0 = q * (x[0] + x[3] + x[2] + x[1]);
    const Vec3<T> n04 = half_cross(x[0], x[3], c0), n03 = half_cross(x[3], x[2], c0);
    const Vec3<T> n02 = half_cross(x[2], x[1], c0), n01 = half_cross(x[1], x[0], c0);
    acc_start(k0, n01, n04, n02, n03);
    acc_start(k1, n01, n02, n04, n03);
    acc_start(k2, n02, n03, n01, n04);
    acc_start(k3, n03, n04, n01, n02);
  }
  {
    const Vec3<T> c1 = q * (x[0] + x[4] + x[7] + x[3]);
    const Vec3<T> n05 = half_cross(x[0], x[4], c1), n12 = half_cross(x[4], x[7], c1);
    const Vec3<T> n08 = half_cross(x[7], x[3], c1), n04 = half_cross(x[3], x[0], c1);
    acc_add(k0, n04, n05, n08, n12);
    acc_add(k3, n08, n04, n05, n12);
    acc_start(k4, n05, n12, n08, n04);
    acc_start(k7, n08, n12, n04, n05);
  }
  {
    const Vec3<T> c2 = q * (x[0] + x[1] + x[5] + x[4]);
    const Vec3<T> n01 = half_cross(x[0], x[1], c2), n06 = half_cross(x[1], x[5], c2);
    const Vec3<T> n09 = half_cross(x[5], x[4], c2), n05 = half_cross(x[4], x[0], c2);
    acc_add(k0, n05, n01, n06, n09);
    fin(0, k0);
    acc_add(k1, n01, n06, n09, n05);
    acc_add(k4, n05, n09, n01, n06);
    acc_start(k5, n06, n09, n01, n05);
  }
  {
    const Vec3<T> c3 = q * (x[4] + x[5] + x[6] + x[7]);
    const Vec3<T> n09 = half_cross(x[4], x[5], c3), n10 = half_cross(x[5], x[6], c3);
    const Vec3<T> n11 = half_cross(x[6], x[7], c3), n12 = half_cross(x[7], x[4], c3);
    acc_add(k4, n09, n12, n10, n11);
    fin(4, k4);
    acc_add(k5, n09, n10, n12, n11);
    acc_start(k6, n11, n10, n12, n09);
    acc_add(k7, n12, n11, n09, n10);
  }
  {
    const Vec3<T> c4 = q * (x[1] + x[2] + x[6] + x[5]);
    const Vec3<T> n02 = half_cross(x[1], x[2], c4), n07 = half_cross(x[2], x[6], c4);
    const Vec3<T> n10 = half_cross(x[6], x[5], c4), n06 = half_cross(x[5], x[1], c4);
    acc_add(k1, n06, n02, n10, n07);
    fin(1, k1);
    acc_add(k2, n07, n02, n06, n10);
    acc_add(k5, n10, n06, n07, n02);
    fin(5, k5);
    acc_add(k6, n10, n07, n06, n02);
  }
  {
    const Vec3<T> c5 = q * (x[2] + x[3] + x[7] + x[6]);
    const Vec3<T> n03 = half_cross(x[2], x[3], c5), n08 = half_cross(x[3], x[7], c5);
    const Vec3<T> n11 = half_cross(x[7], x[6], c5), n07 = half_cross(x[6], x[2], c5);
    acc_add(k2, n07, n03, n11, n08);
    fin(2, k2);
    acc_add(k3, n08, n03, n07, n11);
    fin(3, k3);
    acc_add(k6, n07, n11, n03, n08);
    fin(6, k6);
    acc_add(k7, n11, n08, n07, n03);
    fin(7, k7);
  }
}

// Remap face data from a cell's nodes (PrepareRemap.cc:41-55, 105-117;
// RemapADIService.cc:710): for the low face of each direction (an inner
// face) |A| along d, u_f and (x_f - x_c).n0 with this cell as the next cell;
// for the high face (an inner face) (x_f - x_c).n0 with this cell as the
// previous one.  Face node order: X (0,3,7,4), Y (0,1,5,4), Z (0,1,2,3) low;
// X (1,2,6,5), Y (3,2,6,7), Z (4,5,6,7) high, in SN_trigo cell-node numbers.
// T = float takes x relative to the cell centre (xc = 0).  HC: also the cell
// widths along each direction into fd.h (order 3 and the generalised limiters).
template <typename T, bool HC = false>
__device__ __forceinline__ void face_data(const Dims& dm, int i, int j, int k, const Vec3<T> x[8], Vec3<T> xc,
                                          const double* __restrict__ n0, const double* __restrict__ vh,
                                          const FaceData& fd) {
  const T q = T(.25);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int id = d == 0 ? i : (d == 1 ? j : k);
    double hsum = 0;            // order 3: cell width along d (RemapADIService.cc:240-257)
    const int lo[3][4] = {{0, 3, 7, 4}, {0, 1, 5, 4}, {0, 1, 2, 3}};
    const int hi[3][4] = {{1, 2, 6, 5}, {3, 2, 6, 7}, {4, 5, 6, 7}};
    const long long off = d == 0 ? 0 : (d == 1 ? dm.Fx : dm.Fx + dm.Fy);
    if (id > 0) {
      const long long f = dm.fid(d, i, j, k);
      const D3 nrm = d3(n0[f], n0[dm.F + f], n0[2 * dm.F + f]);
      const Vec3<T> nr = Vec3<T>{(T)nrm.x, (T)nrm.y, (T)nrm.z};
      const Vec3<T> a0 = x[lo[d][0]], a1 = x[lo[d][1]], a2 = x[lo[d][2]], a3 = x[lo[d][3]];
      Vec3<T> xf = Vec3<T>{0, 0, 0};
      xf = xf + q * a0; xf = xf + q * a1; xf = xf + q * a2; xf = xf + q * a3;
      D3 vs = d3(0., 0., 0.);
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int a = lo[d][b];
        const long long nn = dm.nid(i + kCellNodeOff[a][0], j + kCellNodeOff[a][1], k + kCellNodeOff[a][2]);
        vs = vs + d3(vh[nn], vh[dm.N + nn], vh[2 * dm.N + nn]);
      }
      const Vec3<T> cr = T(0.5) * cross(a2 - a0, a3 - a1);
      double A = fabs((double)comp(cr, d));
      if (!(fabs(comp(nrm, d)) >= 1.0E-10)) A = 0.;   // RemapADIService.cc:925 filter: no flux
      const long long t = f - off;
      fd.A[d][t] = A;
      fd.u[d][t] = dot(.25 * vs, nrm);
      fd.df[d][t] = (double)dot(xf - xc, nr);
      if constexpr (HC) hsum += norm2(xf - xc);
    }
    if (id + 1 < dm.ncd(d)) {
      const long long f = dm.fid(d, i + (d == 0), j + (d == 1), k + (d == 2));
      const Vec3<T> nr = Vec3<T>{(T)n0[f], (T)n0[dm.F + f], (T)n0[2 * dm.F + f]};
      Vec3<T> xf = Vec3<T>{0, 0, 0};
      xf = xf + q * x[hi[d][0]]; xf = xf + q * x[hi[d][1]]; xf = xf + q * x[hi[d][2]]; xf = xf + q * x[hi[d][3]];
      fd.db[d][f - off] = (double)dot(xf - xc, nr);
      if constexpr (HC) hsum += norm2(xf - xc);
    }
    if constexpr (HC) fd.h[d * dm.C + dm.cid(i, j, k)] = hsum;
  }
}

// schema-csts energy of one environment of a cell (MahycoModule.cc:1776-1810,
// updateEnergyAndPressureforGP; or by Newton on f, :1552-1613 with
// MahycoModule.h:433-445, the first iteration always run as in newton_eint).
// cn1, cn, cdn, con: the corner-vector sums v.cqs dt, v.cqs_n dt,
// (v - v_n).cqs_n (dt - dt_old), v_n.cqs_n dt_old.  The n-1 pseudo-viscosity
// is zero: the remap resets the n-level fields (PrepareRemap.cc:485-550)
// before saveValuesAtN copies them into it.  pf gets the pressure that
// updateVelocityForward reads: p_n, or the last Newton EOS value; the
// kernel stores it plus this cycle's pseudo-viscosity.  g, eos, pinf: the
// environment's adiabatic constant, EOS and limit tension.
__device__ __forceinline__ double csts_eint(const Phys& ph, double g, int eos, double pinf, double cn1, double cn,
                                            double cdn, double con, double e0, double r, double m, double pn,
                                            double qn, double q, double& pf) {
  const double qnm1 = 0.;
  if (!ph.with_newton) {
    const double denom = 1 + 0.5 * (g - 1.0) * r * cn1 / m;
    const double numer = e0 - (0.5 * (pn + qn) * cn / m) - (0.5 * q * cn1 / m) + (0.25 * (pn + qn) * cdn / m) -
                         (0.5 * (qn - qnm1) * con / m);
    pf = pn;
    return numer / denom;
  }
  const double cdon = 0., epsilon = ph.threshold, itermax = 50;
  const double en = e0;
  double e = en, pp, dpde;
  int i = 0;
  do {
    if (eos == 1) pp = ((g - 1.) * r * e) - (g * pinf);
    else pp = (g - 1.) * r * e;
    dpde = (g - 1.) * r;
    const double fe = e - en + 0.5 * (pp + q) * cn1 / m + 0.5 * (pn + qn) * cn / m - 0.25 * (pn + qn) * cdn / m +
                      0.5 * (q - qnm1) * cdon / m;
    const double enew = e - fe / (1. + 0.5 * dpde * cn1 / m);
    e = enew;
    i++;
  } while (i < itermax && fabs(e - en + 0.5 * (pp + q) * cn1 / m + 0.5 * (pn + qn) * cn / m -
                                0.25 * (pn + qn) * cdn / m + 0.5 * (q - qnm1) * cdon / m) >= epsilon);
  pf = pp;
  return e;
}

// Lagrange thermodynamics of a mesh with K > 1 environments, then the remap
// variables (MahycoModule.cc:1331-1426 updateDensity, :454-578
// computeArtificialViscosity, :1659-1770 updateEnergyAndPressureforGP,
// PrepareRemap.cc:258-437 computeVariablesForRemap_PBorn0).  Pure cells take
// the single-environment formulas with their environment's gamma; a mixed
// cell works environment by environment on V_k = f_k V (MahycoModule.cc:1274-1295).
// U holds the 3K+1 non-zero remap variables [V_k | V_k rho_k | V_k rho_k e_k |
// V q] as planes; V is kept in Vlag, the divisor of Phi on the first sweep.
// The global density m/V is stored for every cell: the remap keeps it in a
// mixed cell whose fractions leave one environment only (RemapADIFinal.cc:561-562).
// pbphi (pente-borne): Phi of the first sweep for the cell's environments,
// volume fraction, density and internal energy after this step, and q of
// the last of them (PrepareRemap.cc:201-212); the other environments' planes
// are left as they are.  CSTS: each environment's energy by csts_eint from
// the cell's corner-vector sums cssum (cn1, cn, cdn, con), and pf = the
// global p + q the forward step reads (MahycoModule.cc:792-831): a pure
// cell's p_n or Newton pressure plus its q, a mixed cell's mean p_n plus
// sum_k f_k q_k (MahycoModule.cc:454-578).
template <int K, bool CSTS = false>
__device__ __forceinline__ void lagrange_thermo_env(const Phys& ph, const Scalars* S, const EnvState& env, int c,
                                                    int C, double V, double Lc, double* __restrict__ rho,
                                                    const double* __restrict__ e, const double* __restrict__ q,
                                                    const double* __restrict__ p, const double* __restrict__ cs,
                                                    const double* __restrict__ mass, double* __restrict__ U,
                                                    double* __restrict__ Vlag, double* __restrict__ pbphi,
                                                    const double* cssum = nullptr, double* __restrict__ pf = nullptr) {
  constexpr int NV = 3 * K + 1;
  const double inv_deltat = S->inv_dt;
  const double rn = rho[c];
  const double nd = mass[c] / V;
  const double irn = 1.0 / rn, ind = 1.0 / nd;
  const double tau = 0.5 * (irn + ind);
  const double itau = 1. / tau;
  const double du = qdiv(inv_deltat * (ind - irn), tau, itau);
  const uint32_t mk = env.mask[c];
  const bool pc = ph.pseudo_centree != 0;
  double u[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) u[v] = 0.;
  if (__popc(mk) == 1) {
    const int ke = __ffs(mk) - 1;
    const double g = env.gamma[ke];
    double qn = 0.;
    if (du < 0.0) qn = itau * (-0.5 * Lc * cs[c] * du + (g + 1) / 2.0 * Lc * Lc * du * du);
    double en;
    if constexpr (CSTS) {
      double pforward;
      en = csts_eint(ph, g, env.eos[ke], env.pinf[ke], cssum[0], cssum[1], cssum[2], cssum[3], e[c], nd, mass[c],
                     p[c], q[c], qn, pforward);
      pf[c] = pforward + qn;
    } else {
      en = energy_update(ph.with_newton != 0, pc, env.eos[ke], g, env.pinf[ke], ph.threshold, q[c], qn, ind, irn, nd,
                         p[c], e[c]);
    }
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (k == ke) { u[k] = V; u[K + k] = V * nd; u[2 * K + k] = V * nd * en; }
    u[3 * K] = V * qn;
    if (pbphi) {
      pbphi[ke * C + c] = env.fg[c]; pbphi[(K + ke) * C + c] = nd; pbphi[(2 * K + ke) * C + c] = en;
      pbphi[3 * K * C + c] = qn;
    }
  } else {
    const double csc = cs[c];
    double qg = 0.;                                              // the mixed cell's pseudo-viscosity sum_k f_k q_k
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (!(mk >> k & 1)) continue;
      const int o = k * C + c;
      const double vk = env.f[o] * V;
      const double rk = env.m[o] / vk;
      const double irnk = 1.0 / env.rho[o], irk = 1.0 / rk;
      const double tauk = 0.5 * (irnk + irk);
      const double g = env.gamma[k];
      double qk = 0.;
      if (du < 0.0) qk = 1. / tauk * (-0.5 * Lc * csc * du + (g + 1) / 2.0 * Lc * Lc * du * du);
      double ek;
      if constexpr (CSTS) {
        double pk_unused;
        ek = csts_eint(ph, g, env.eos[k], env.pinf[k], cssum[0], cssum[1], cssum[2], cssum[3], env.e[o], rk, env.m[o],
                       env.p[o], env.q[o], qk, pk_unused);
        qg += qk * env.f[o];
      } else {
        ek = energy_update(ph.with_newton != 0, pc, env.eos[k], g, env.pinf[k], ph.threshold, env.q[o], qk, irk, irnk,
                           rk, env.p[o], env.e[o]);
      }
      u[k] = vk;
      u[K + k] = vk * rk;
      u[2 * K + k] = vk * rk * ek;
      u[3 * K] = vk * qk;                                        // the last environment wins (P:318-330)
      if (pbphi) {
        pbphi[o] = env.f[o]; pbphi[K * C + o] = rk; pbphi[2 * K * C + o] = ek; pbphi[3 * K * C + c] = qk;
      }
    }
    if constexpr (CSTS) pf[c] = p[c] + qg;                      // the mean p_n: no EOS runs before the forward step
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) U[v * C + c] = u[v];
  Vlag[c] = V;
  rho[c] = nd;
}


// CSTS (schema-csts, FP64 only): vnb = the backward node velocity of this
// cycle, pf = the pressure plus pseudo-viscosity of the forward step.
template <int K, typename R, bool CSTS = false, bool HC = false>
__device__ __forceinline__ void k_cyc_lagrange_cells_body(Dims dm, const Scalars* __restrict__ S, Phys ph,
    const double* __restrict__ x0, const double* __restrict__ vh, const double* __restrict__ n0,
    double* __restrict__ rho, const double* __restrict__ e, const double* __restrict__ q,
    const double* __restrict__ p, const double* __restrict__ cs, const double* __restrict__ mass,
    double* __restrict__ cqs, float* __restrict__ cqs32, double* __restrict__ L, double* __restrict__ U,
    double* __restrict__ xcs, FaceData fd, EnvState env, double* __restrict__ Vlag,
    int bx_, int by_, int bz_, const double* __restrict__ vnb = nullptr, double* __restrict__ pf = nullptr) {
  static_assert(!CSTS || sizeof(R) == 8, "schema-csts: FP64");
  int i, j, k;
  if (!block_item(dm.nx, dm.ny, dm.nz, bx_, by_, bz_, i, j, k)) return;
  const long long c = dm.cid(i, j, k);
  const long long C = dm.C;
  const double dt = S->dt;
  D3 x[8];
#pragma unroll
  for (int a = 0; a < 8; ++a)
    x[a] = load_xl(dm, x0, vh, dt, dm.nid(i + kCellNodeOff[a][0], j + kCellNodeOff[a][1], k + kCellNodeOff[a][2]));
  D3 sm = d3(0., 0., 0.);
#pragma unroll
  for (int a = 0; a < 8; ++a) sm = sm + x[a];
  const D3 xc = .125 * sm;
  xcs[c] = xc.x; xcs[C + c] = xc.y; xcs[2 * C + c] = xc.z;

  // corner vectors and volume V = 1/3 sum x_a . cqs_a (MahycoModule.cc:1224-1262)
  constexpr bool F32 = sizeof(R) == 4;
  double cs_cn1 = 0., cs_cn = 0., cs_cdn = 0., cs_con = 0.;   // schema-csts sums
  double V = 0;
  F3 xr[8];
  if constexpr (F32) {
    // mixed form: FP32 corner vectors from coordinates relative to the
    // centre (kept in FP32 for the force), volume summed in FP64
#pragma unroll
    for (int a = 0; a < 8; ++a)
      xr[a] = F3{(float)(x[a].x - xc.x), (float)(x[a].y - xc.y), (float)(x[a].z - xc.z)};
    float dv[8];
    corner_vectors<float>(xr, [&](int a, F3 o) {
      cqs32[(a * 3 + 0) * C + c] = o.x; cqs32[(a * 3 + 1) * C + c] = o.y; cqs32[(a * 3 + 2) * C + c] = o.z;
      dv[a] = dot(xr[a], o);
    });
#pragma unroll
    for (int a = 0; a < 8; ++a) V += (double)dv[a];
  } else {
    double dv[8], dv1[8];
    if constexpr (CSTS) {
      // the sums over the previous corner vectors, before they are overwritten
#pragma unroll
      for (int a = 0; a < 8; ++a) {
        const long long nn = dm.nid(i + kCellNodeOff[a][0], j + kCellNodeOff[a][1], k + kCellNodeOff[a][2]);
        const D3 va = d3(vh[nn], vh[dm.N + nn], vh[2 * dm.N + nn]);
        const D3 vb = d3(vnb[nn], vnb[dm.N + nn], vnb[2 * dm.N + nn]);
        const D3 cq = d3(cqs[(a * 3 + 0) * C + c], cqs[(a * 3 + 1) * C + c], cqs[(a * 3 + 2) * C + c]);
        cs_cn += dot(va, cq) * dt;
        cs_cdn += dot(va - vb, cq) * (dt - S->old_dt);
        cs_con += dot(vb, cq) * S->old_dt;
      }
    }
    corner_vectors<double>(x, [&](int a, D3 o) {
      cqs[(a * 3 + 0) * C + c] = o.x; cqs[(a * 3 + 1) * C + c] = o.y; cqs[(a * 3 + 2) * C + c] = o.z;
      dv[a] = dot(x[a], o);
      if constexpr (CSTS) {
        const long long nn = dm.nid(i + kCellNodeOff[a][0], j + kCellNodeOff[a][1], k + kCellNodeOff[a][2]);
        dv1[a] = dot(d3(vh[nn], vh[dm.N + nn], vh[2 * dm.N + nn]), o) * dt;
      }
    });
#pragma unroll
    for (int a = 0; a < 8; ++a) V += dv[a];
    if constexpr (CSTS) {
#pragma unroll
      for (int a = 0; a < 8; ++a) cs_cn1 += dv1[a];
    }
  }
  V *= 1. / 3;
  double Lc;
  // racine-cubique-volume: the project cube root (the reference's bits) in
  // FP64; the mixed form takes CUDA's FP32 cube root of the FP64 volume (L
  // feeds the viscosity and the CFL bound only)
  if (ph.lc_mode == 0) {
    if constexpr (F32) Lc = (double)cbrtf((float)V);
    else Lc = pow_third(V);
  } else {
    D3 fc[6];
    if constexpr (F32) {
      D3 xx[8];
#pragma unroll
      for (int a = 0; a < 8; ++a) xx[a] = d3(xr[a].x, xr[a].y, xr[a].z);
      face_centres(xx, fc);
    } else {
      face_centres(x, fc);
    }
    const double d1 = norm2(fc[0] - fc[3]), d2 = norm2(fc[2] - fc[5]), d3_ = norm2(fc[1] - fc[4]);
    Lc = (d1 * d2 * d3_) / (d1 * d2 + d1 * d3_ + d2 * d3_);
  }
  L[c] = Lc;
  if constexpr (K == 1) {
    const double inv_deltat = S->inv_dt;                        // 1.0 / dt
    const double rn = rho[c];
    const double nd = mass[c] / V;
    const double irn = 1.0 / rn, ind = 1.0 / nd;
    const double tau = 0.5 * (irn + ind);
    const double itau = 1. / tau;
    const double du = qdiv(inv_deltat * (ind - irn), tau, itau);
    double qn = 0.;
    const double g = ph.gamma;
    if (du < 0.0) qn = itau * (-0.5 * Lc * cs[c] * du + (g + 1) / 2.0 * Lc * Lc * du * du);
    double en;
    if constexpr (CSTS) {
      double pforward;
      en = csts_eint(ph, g, ph.eos, ph.pinf, cs_cn1, cs_cn, cs_cdn, cs_con, e[c], nd, mass[c], p[c], q[c], qn,
                     pforward);
      pf[c] = pforward + qn;                                    // the forward force's p + q (q: this cycle's)
    } else {
      en = energy_update(ph.with_newton != 0, ph.pseudo_centree != 0, ph.eos, g, ph.pinf, ph.threshold, q[c], qn, ind,
                         irn, nd, p[c], e[c]);
    }
    U[c] = V;
    U[C + c] = V * nd;
    U[2 * C + c] = V * nd * en;
    U[3 * C + c] = V * qn;
    if (fd.pbphi) { fd.pbphi[c] = nd; fd.pbphi[C + c] = en; fd.pbphi[2 * C + c] = qn; }
  } else {
    const double cssum[4] = {cs_cn1, cs_cn, cs_cdn, cs_con};
    lagrange_thermo_env<K, CSTS>(ph, S, env, (int)c, (int)C, V, Lc, rho, e, q, p, cs, mass, U, Vlag, fd.pbphi, cssum,
                                 pf);
  }
  if constexpr (F32) face_data<float>(dm, i, j, k, xr, F3{0.f, 0.f, 0.f}, n0, vh, fd);
  else face_data<double, HC>(dm, i, j, k, x, xc, n0, vh, fd);
}

template <int K, typename R, bool HC = false>
__global__ void __launch_bounds__(128, sizeof(R) == 4 ? 5 : 3) k_cyc_lagrange_cells(Dims dm,
    const Scalars* __restrict__ S, Phys ph,
    const double* __restrict__ x0, const double* __restrict__ vh, const double* __restrict__ n0,
    double* __restrict__ rho, const double* __restrict__ e, const double* __restrict__ q,
    const double* __restrict__ p, const double* __restrict__ cs, const double* __restrict__ mass,
    double* __restrict__ cqs, float* __restrict__ cqs32, double* __restrict__ L, double* __restrict__ U,
    double* __restrict__ xcs, FaceData fd, EnvState env, double* __restrict__ Vlag, int linear) {
  k_cyc_lagrange_cells_body<K, R, false, HC>(dm, S, ph, x0, vh, n0, rho, e, q, p, cs, mass, cqs, cqs32, L, U, xcs, fd,
                                             env, Vlag, blockIdx.x, linear ? -1 : (int)blockIdx.y, blockIdx.z);
}



}  // namespace mhy
