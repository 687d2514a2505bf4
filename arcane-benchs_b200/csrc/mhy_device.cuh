// mhy_device.cuh -- device helpers shared by the kernels: exact-order vector
// arithmetic, limiters, the energy update, structured indexing.
//
// Every helper evaluates its expression in the same order, with the same
// roundings, as the reference's Arcane Real3 code (sums left to right,
// dot = x*x'+y*y'+z*z', cross as math::vecMul), so that with --fmad=false the
// device produces the same bits as the CPU oracle.
#pragma once

#include <cstdint>
#include "mhy_pow_third.h"

namespace mhy {

// 3-vectors in double (D3) or float (F3, the mixed-precision geometry).
template <typename T> struct Vec3 { T x, y, z; };
using D3 = Vec3<double>;
using F3 = Vec3<float>;
__device__ __forceinline__ D3 d3(double x, double y, double z) { return D3{x, y, z}; }
template <typename T>
__device__ __forceinline__ Vec3<T> operator+(Vec3<T> a, Vec3<T> b) { return Vec3<T>{a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename T>
__device__ __forceinline__ Vec3<T> operator-(Vec3<T> a, Vec3<T> b) { return Vec3<T>{a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename T>
__device__ __forceinline__ Vec3<T> operator*(T s, Vec3<T> v) { return Vec3<T>{v.x * s, v.y * s, v.z * s}; }
template <typename T>
__device__ __forceinline__ T dot(Vec3<T> a, Vec3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T>
__device__ __forceinline__ Vec3<T> cross(Vec3<T> u, Vec3<T> v) {
  return Vec3<T>{u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x};
}
__device__ __forceinline__ double norm2(D3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
template <typename T>
__device__ __forceinline__ T comp(Vec3<T> a, int d) { return d == 0 ? a.x : (d == 1 ? a.y : a.z); }
// x / y with the reciprocal r = 1.0/y already at hand: q0 = RN(x r),
// e = x - y q0 (exact with one fma), q = RN(q0 + e r).  With r the correctly
// rounded reciprocal this is the correctly rounded quotient (P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34(1), 1990), i.e. the same bits as x / y, as
// long as x, y and the quotient stay well inside the normal range; outside
// 2^-960 <= |x|, |q0| <= 2^960 or |y| > 2^960 (zeros, subnormals, huge
// values, inf, NaN; a y above 2^1022 would leave r subnormal) the plain
// division is taken.  Checked against x / y on 3e10 random and
// adversarial operand pairs with no difference.  Used wherever several
// quotients share a denominator.
// A zero numerator over a normal or infinite y is answered by q0 = x r:
// r is then a nonzero finite number or a signed zero with the sign of y, so
// q0 is the zero whose sign is sign(x) xor sign(y), which is IEEE x / y.
// Zeros are the common case on quiescent regions of the mesh (velocity,
// pseudo-viscosity and their differences), and would otherwise pay for a
// full division.
__device__ __forceinline__ double qdiv(double x, double y, double r) {
  const double q0 = x * r;
  if (x == 0.0 && fabs(y) >= 0x1p-1022) return q0;
  const double ax = fabs(x), aq = fabs(q0);
  if (!(ax >= 0x1p-960 && ax <= 0x1p+960 && aq >= 0x1p-960 && aq <= 0x1p+960 && fabs(y) <= 0x1p+960)) return x / y;
  return __fma_rn(__fma_rn(-q0, y, x), r, q0);
}

// The sweeps' speculative form of qdiv: the corrected quotient (or q0 for a
// zero numerator) without a branch, and a flag when it may differ from
// x / y: a zero x over a y that is not a normal number; otherwise x or q0
// outside 2^-960 <= |.| < 2^960 (zeros, subnormals, huge values, inf, NaN)
// or y outside 2^-959 <= |y| < 2^960, all tested on the biased exponents.
// A warp whose lanes raised the flag recomputes its segment with qdiv (the
// sweeps' *_line_exact functions), so the results are x / y bit for bit
// either way.  Measured on Sedov 128^3 FP64: no warp raised the flag in 505
// cycles, and the cycle takes 1.21 ms instead of 1.32 ms with qdiv's
// branches.  (Scaling tiny numerators by 2^200 first, so that a field's
// subnormal tail would stay on the fast path, cost 3 % more and was left out.)
__device__ __forceinline__ double qdiv_spec(double x, double y, double r, unsigned& oor) {
  const double q0 = x * r;
  const double q = __fma_rn(__fma_rn(-q0, y, x), r, q0);
  const unsigned bx = (unsigned)__double2hiint(x) >> 20 & 0x7ffu;
  const unsigned by = (unsigned)__double2hiint(y) >> 20 & 0x7ffu;
  const unsigned bq0 = (unsigned)__double2hiint(q0) >> 20 & 0x7ffu;
  const bool zero = x == 0.0;
  const bool bad = zero ? by - 1u > 2045u : (bx - 63u > 1919u || by - 64u > 1918u || bq0 - 63u > 1919u);
  oor |= bad ? 1u : 0u;
  return zero ? q0 : q;
}

// Quotient x / y with r = 1 / y at hand in the sweeps: FP32 (the mixed form)
// takes the product; FP64 takes qdiv, or its speculative form (SP) with the
// flag in *oor.
template <typename R, bool SP>
__device__ __forceinline__ R dv(R x, R y, R r, unsigned* oor) {
  if constexpr (sizeof(R) == 4) return x * r;
  else if constexpr (SP) return qdiv_spec(x, y, r, *oor);
  else return qdiv(x, y, r);
}

// Arcane math::min / math::max and std::min / std::max, as the reference writes them
__device__ __forceinline__ double amin(double a, double b) { return (a < b) ? a : b; }
__device__ __forceinline__ double amax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }

// Flux limiters, mahyco/src/Remap/RemapADIService.h:260-286
template <typename R> __device__ __forceinline__ R tmin(R a, R b) { return (b < a) ? b : a; }   // std::min
template <typename R> __device__ __forceinline__ R tmax(R a, R b) { return (a < b) ? b : a; }   // std::max
// fluxLimiterG, mahyco/src/Remap/UtilesRemap.cc:127-175: the generalised
// limiters for uneven widths (ids TypesMahyco.h:65-74: 3 minmodG, 4
// superBeeG, 5 vanLeerG, 6 arithmeticG, 7 ultrabeeG), std::min / std::max.
template <typename R>
__device__ __forceinline__ R flux_limiter_g(int id, R gradplus, R gradmoins, R y0, R yplus, R ymoins, R h0, R hplus,
                                            R hmoins) {
  const R zero = R(0), half = R(0.5);
  R grady = zero;
  if (gradplus * gradmoins < zero) return zero;
  if (id == 3) {
    if ((yplus - ymoins) > zero) grady = tmin(fabs(gradplus), fabs(gradmoins));
    else grady = -tmin(fabs(gradplus), fabs(gradmoins));
  } else if (id == 4) {
    if ((yplus - ymoins) > zero) grady = tmax(fabs(gradplus), fabs(gradmoins));
    else grady = -tmax(fabs(gradplus), fabs(gradmoins));
  } else if (id == 5) {
    const R lambdaplus = (h0 / R(2) + hplus) / (h0 + hplus + hmoins);
    const R lambdamoins = (h0 / R(2) + hmoins) / (h0 + hplus + hmoins);
    if ((lambdaplus * gradplus + lambdamoins * gradmoins) != zero)
      grady = gradplus * gradmoins / (lambdaplus * gradplus + lambdamoins * gradmoins);
    else grady = zero;
  } else if (id == 7) {
    grady = (yplus - ymoins) / h0;
  } else if (id == 6) {
    const R lambdaplus = (h0 / R(2) + hplus) / (h0 + hplus + hmoins);
    const R lambdamoins = (h0 / R(2) + hmoins) / (h0 + hplus + hmoins);
    grady = lambdamoins * gradplus + lambdaplus * gradmoins;
  }
  (void)half; (void)y0;
  const R gradMplus = gradplus * (h0 + hplus) / h0;
  const R gradMmoins = gradmoins * (h0 + hmoins) / h0;
  const R gradM = tmin(fabs(gradMplus), fabs(gradMmoins));
  if ((yplus - ymoins) > zero) grady = tmin(fabs(gradM), fabs(grady));
  else grady = -tmin(fabs(gradM), fabs(grady));
  return grady;
}

template <typename R>
__device__ __forceinline__ R limiter(int id, R r) {
  switch (id) {
    case 0: return tmax(R(0), tmin(R(1), r));
    case 1: return tmax(R(0), tmax(tmin(R(2) * r, R(1)), tmin(r, R(2))));
    case 2: return (r <= R(0) ? R(0) : R(2) * r / (R(1) + r));
    default: return R(0);
  }
}

// Arithmetic of the remap evaluation in precision R.  double: the reference's
// operations exactly (qdiv gives x / y bit for bit).  float (the mixed
// precision form): one reciprocal per shared denominator and products.
template <typename R> struct Ar;
template <> struct Ar<double> {
  __device__ static __forceinline__ double rcp(double y) { return 1.0 / y; }
  __device__ static __forceinline__ double div(double x, double y, double r) { return qdiv(x, y, r); }
  __device__ static __forceinline__ double quo(double x, double y) { return x / y; }
};
template <> struct Ar<float> {
  __device__ static __forceinline__ float rcp(float y) { return 1.0f / y; }
  __device__ static __forceinline__ float div(float x, float, float r) { return x * r; }
  __device__ static __forceinline__ float quo(float x, float y) { return __fdividef(x, y); }
};

// Equations of state.  After the remap, p and c from rho and e:
// PerfectGas (eos/perfectgas/PerfectGasEOSService.cc:92-106) and StiffenedGas
// (eos/stiffenedgas/StiffenedGasEOSService.cc:29-44, pinf = limit-tension).
__device__ __forceinline__ void eos_pc(int kind, double g, double pinf, double r, double e, double& p, double& c) {
  if (kind == 1) { p = ((g - 1.) * r * e) - (g * pinf); c = sqrt((g / r) * (p + pinf)); }
  else { p = (g - 1.) * r * e; c = sqrt(g * p / r); }
}
// initEOS: e and c from rho and p (PerfectGasEOSService.cc:20-32,
// StiffenedGasEOSService.cc:10-24).
__device__ __forceinline__ void eos_init(int kind, double g, double pinf, double r, double p, double& e, double& c) {
  if (kind == 1) { e = (p + (g * pinf)) / ((g - 1.) * r); c = sqrt((g / r) * (p + pinf)); }
  else { e = p / ((g - 1.) * r); c = sqrt(g * p / r); }
}

// compute_eint, mahyco/src/MahycoModule.cc:1630-1654; ir = 1.0/r and irn = 1.0/rn given.
__device__ __forceinline__ double compute_eint(bool pc, double g, double qn, double q, double ir, double irn,
                                               double r, double p, double en) {
  double pseudo = 0.;
  if (pc && ((qn + q) * (ir - irn) < 0.)) pseudo = 0.5 * (q + qn);
  if (!pc && (q * (ir - irn) < 0.)) pseudo = q;
  double denom = 1 + 0.5 * (g - 1.0) * r * (ir - irn);
  double numer = en - (0.5 * p + pseudo) * (ir - irn);
  return numer / denom;
}

// updateEnergyAndPressurebyNewton without schema-csts, MahycoModule.cc:1482-1535:
// Newton iterations on fvnr(e) = e - en + 0.5 (p + pn + 2 q*) (1/r - 1/rn),
// derivative 1 + 0.5 dpde (1/r - 1/rn) (MahycoModule.h:420-429), p and dpde
// from the environment's EOS at the current e and the new density
// (applyOneCellEOS); the loop test takes fvnr at the updated e with those p,
// dpde.  The reference makes its first test before any EOS call (p and dpde
// not yet set); here the first iteration always runs.  Only e is kept: p and
// c are recomputed by the EOS after the remap.
__device__ __forceinline__ double newton_eint(bool pc, int kind, double g, double pinf, double epsilon, double qn,
                                              double q, double ir, double irn, double r, double pn, double en) {
  double pseudo = 0.;
  if (pc && ((qn + q) * (ir - irn) < 0.)) pseudo = 0.5 * (q + qn);
  if (!pc && (q * (ir - irn) < 0.)) pseudo = q;
  const double itermax = 50;
  double e = en, p, dpde;
  int i = 0;
  do {
    if (kind == 1) p = ((g - 1.) * r * e) - (g * pinf);
    else p = (g - 1.) * r * e;
    dpde = (g - 1.) * r;
    const double enew = e - (e - en + 0.5 * (p + pn + 2. * pseudo) * (ir - irn)) / (1. + 0.5 * dpde * (ir - irn));
    e = enew;
    i++;
  } while (i < itermax && fabs(e - en + 0.5 * (p + pn + 2. * pseudo) * (ir - irn)) >= epsilon);
  return e;
}

// The Lagrange energy update of one environment cell: the closed form of
// updateEnergyAndPressureforGP, or the Newton iterations when with-newton is set.
__device__ __forceinline__ double energy_update(bool newton, bool pc, int kind, double g, double pinf, double epsilon,
                                                double qn, double q, double ir, double irn, double r, double p,
                                                double en) {
  if (newton) return newton_eint(pc, kind, g, pinf, epsilon, qn, q, ir, irn, r, p, en);
  return compute_eint(pc, g, qn, q, ir, irn, r, p, en);
}

// Corner vectors (CQS) of a hexahedron, mahyco/src/MahycoModule.cc:2195-2258,
// face centres from :1080-1087.  Node order SN_trigo.
__device__ __forceinline__ void face_centres(const D3 x[8], D3 fc[6]) {
  fc[0] = 0.25 * (x[0] + x[3] + x[2] + x[1]);
  fc[1] = 0.25 * (x[0] + x[4] + x[7] + x[3]);
  fc[2] = 0.25 * (x[0] + x[1] + x[5] + x[4]);
  fc[3] = 0.25 * (x[4] + x[5] + x[6] + x[7]);
  fc[4] = 0.25 * (x[1] + x[2] + x[6] + x[5]);
  fc[5] = 0.25 * (x[2] + x[3] + x[7] + x[6]);
}

__device__ __forceinline__ void compute_cqs(const D3 x[8], const D3 fc[6], D3 out[8]) {
  const D3 c0 = fc[0], c1 = fc[1], c2 = fc[2], c3 = fc[3], c4 = fc[4], c5 = fc[5];
  const D3 n1a04 = 0.5 * cross(x[0] - c0, x[3] - c0);
  const D3 n1a03 = 0.5 * cross(x[3] - c0, x[2] - c0);
  const D3 n1a02 = 0.5 * cross(x[2] - c0, x[1] - c0);
  const D3 n1a01 = 0.5 * cross(x[1] - c0, x[0] - c0);
  const D3 n2a05 = 0.5 * cross(x[0] - c1, x[4] - c1);
  const D3 n2a12 = 0.5 * cross(x[4] - c1, x[7] - c1);
  const D3 n2a08 = 0.5 * cross(x[7] - c1, x[3] - c1);
  const D3 n2a04 = 0.5 * cross(x[3] - c1, x[0] - c1);
  const D3 n3a01 = 0.5 * cross(x[0] - c2, x[1] - c2);
  const D3 n3a06 = 0.5 * cross(x[1] - c2, x[5] - c2);
  const D3 n3a09 = 0.5 * cross(x[5] - c2, x[4] - c2);
  const D3 n3a05 = 0.5 * cross(x[4] - c2, x[0] - c2);
  const D3 n4a09 = 0.5 * cross(x[4] - c3, x[5] - c3);
  const D3 n4a10 = 0.5 * cross(x[5] - c3, x[6] - c3);
  const D3 n4a11 = 0.5 * cross(x[6] - c3, x[7] - c3);
  const D3 n4a12 = 0.5 * cross(x[7] - c3, x[4] - c3);
  const D3 n5a02 = 0.5 * cross(x[1] - c4, x[2] - c4);
  const D3 n5a07 = 0.5 * cross(x[2] - c4, x[6] - c4);
  const D3 n5a10 = 0.5 * cross(x[6] - c4, x[5] - c4);
  const D3 n5a06 = 0.5 * cross(x[5] - c4, x[1] - c4);
  const D3 n6a03 = 0.5 * cross(x[2] - c5, x[3] - c5);
  const D3 n6a08 = 0.5 * cross(x[3] - c5, x[7] - c5);
  const D3 n6a11 = 0.5 * cross(x[7] - c5, x[6] - c5);
  const D3 n6a07 = 0.5 * cross(x[6] - c5, x[2] - c5);
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

// Structured mesh dimensions and index maps.
struct Dims {
  int nx, ny, nz;          // cells per direction
  long long C, N, F, Fx, Fy;
  int dt_k0, dt_k1;        // cell layers k the dt reduction covers: [0, nz) unless the mesh is a slab
                           // with ghost layers (mhy_set_dt_reduction)
  __device__ __forceinline__ long long cid(int i, int j, int k) const { return i + (long long)nx * (j + (long long)ny * k); }
  __device__ __forceinline__ long long nid(int i, int j, int k) const { return i + (long long)(nx + 1) * (j + (long long)(ny + 1) * k); }
  __host__ __device__ __forceinline__ int ncd(int d) const { return d == 0 ? nx : (d == 1 ? ny : nz); }
  // face of direction d whose lowest node is (i,j,k)
  __device__ __forceinline__ long long fid(int d, int i, int j, int k) const {
    if (d == 0) return i + (long long)(nx + 1) * (j + (long long)ny * k);
    if (d == 1) return Fx + i + (long long)nx * (j + (long long)(ny + 1) * k);
    return Fx + Fy + i + (long long)nx * (j + (long long)ny * k);
  }
  __device__ __forceinline__ void cijk(long long c, int& i, int& j, int& k) const {
    i = (int)(c % nx); long long t = c / nx; j = (int)(t % ny); k = (int)(t / ny);
  }
  __device__ __forceinline__ void nijk(long long n, int& i, int& j, int& k) const {
    i = (int)(n % (nx + 1)); long long t = n / (nx + 1); j = (int)(t % (ny + 1)); k = (int)(t / (ny + 1));
  }
  // number of faces of direction d, and (i,j,k) of its t-th face
  __device__ __forceinline__ long long nfd(int d) const {
    return d == 0 ? Fx : (d == 1 ? Fy : F - Fx - Fy);
  }
  __device__ __forceinline__ void fdijk(int d, long long t, int& i, int& j, int& k) const {
    int ex = nx + (d == 0), ey = ny + (d == 1);
    i = (int)(t % ex); long long u = t / ex; j = (int)(u % ey); k = (int)(u / ey);
  }
};

// Item (i, j, k) of thread threadIdx.x in block (bx, by, bz) over an
// ex x ey x ez lattice: by >= 0: rows of blockDim.x items along x (block
// (bx, by, bz) = x chunk, y, z); by < 0: blockDim.x consecutive items of the
// whole lattice (block bx), which wastes no thread when ex is not a multiple
// of the block size.  False when the thread has no item.
__device__ __forceinline__ bool block_item(int ex, int ey, int ez, int bx, int by, int bz, int& i, int& j, int& k) {
  if (by >= 0) {
    i = bx * blockDim.x + threadIdx.x; j = by; k = bz;
    return i < ex;
  }
  const int c = bx * blockDim.x + threadIdx.x;
  if (c >= ex * ey * ez) { i = j = k = 0; return false; }
  i = c % ex;
  const int t = c / ex;
  j = t % ey;
  k = t / ey;
  return true;
}

// SN_trigo node offsets of a cell, cartesian/CartConnectivityCellNode.h:83-94
__device__ __constant__ const int kCellNodeOff[8][3] = {{0,0,0},{1,0,0},{1,1,0},{0,1,0},{0,0,1},{1,0,1},{1,1,1},{0,1,1}};

// Face node order: X (0,0,0),(0,1,0),(0,1,1),(0,0,1); Y (0,0,0),(1,0,0),(1,0,1),(0,0,1);
// Z (0,0,0),(1,0,0),(1,1,0),(0,1,0).  With the reference normal formula (whose
// y component is the negated cross-product component) every normal points to +axis.
__device__ __forceinline__ void face_node_ids(const Dims& dm, int d, int i, int j, int k, long long out[4]) {
  if (d == 0) { out[0] = dm.nid(i, j, k); out[1] = dm.nid(i, j + 1, k); out[2] = dm.nid(i, j + 1, k + 1); out[3] = dm.nid(i, j, k + 1); }
  else if (d == 1) { out[0] = dm.nid(i, j, k); out[1] = dm.nid(i + 1, j, k); out[2] = dm.nid(i + 1, j, k + 1); out[3] = dm.nid(i, j, k + 1); }
  else { out[0] = dm.nid(i, j, k); out[1] = dm.nid(i + 1, j, k); out[2] = dm.nid(i + 1, j + 1, k); out[3] = dm.nid(i, j + 1, k); }
}

}  // namespace mhy
