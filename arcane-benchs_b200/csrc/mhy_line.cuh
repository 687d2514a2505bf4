// mhy_line.cuh -- shared pieces of the directional remap sweeps: the line
// layout (a warp per line segment along the sweep direction, neighbours by
// shuffles, y/z tiles staged in shared memory), the per-lane cell and node
// updates, and the node sweep kernels, which serve any number of
// environments K (the dual mass flux of each cell comes in K planes).
#pragma once

#include "mhy_kernels.cuh"

namespace mhy {
// ------------------------------------------------------------------------
// Directional sweeps.  The stencil of the remap runs along one direction d,
// so each line of cells (or nodes) along d is independent.  A warp holds 32
// consecutive items of one line, one per lane, exchanges neighbours with
// shuffles and updates the 28 inner ones; a block holds 8 lines.
//   d = x: the 8 lines are neighbouring rows and a lane's loads and stores
//          are coalesced along x as they are.
//   d = y, z: the 8 lines are 8 consecutive x at one (z or y), and a warp's
//          items are a stride apart in memory.  The block therefore stages
//          its 8 x 32 tile of every input array in shared memory with loads
//          that run along x (8 doubles = 64 contiguous bytes per row), each
//          warp reads its line from there, writes its results back into its
//          own rows, and the block stores them along x again.
// All index arithmetic is 32-bit (mhy_create bounds the mesh so that every
// element offset fits).

constexpr int kLineUpd = 28;    // items updated per warp (32 lanes, 2 halo lanes on each side)
// The sweeps are latency bound (long dependent chains of divisions and
// shuffles per lane); 4 resident blocks (32 warps, 64 registers, a few bytes
// of spill) per SM run them 15 % faster than the 2-3 blocks the compiler's
// own register choice allows (Sedov 128^3 on B200).
constexpr int kLineMinBlocks = 4;
// Row length (doubles) of a staged tile [array][line][position].  Staging
// stores by thread (x = tid % 8, p = tid / 8) hit address 36 x + p, whose
// 8-byte bank pairs (4 x + p) mod 16 cover every pair exactly twice per warp,
// and line reads run along p, so both are free of bank conflicts.
constexpr int kTileLd = 36;
constexpr int kTileArr = kLineWarps * kTileLd;   // doubles per staged array

// The y/z sweeps take the number of lines per block W (8, 16 or 32) as a
// tuning parameter: a block stages W consecutive x of 32 positions, so each
// row of its loads and stores spans W doubles (64, 128 or 256 contiguous
// bytes).  Row length ld: for W = 8 the 36 above; for W >= 16 staging stores
// by thread (x = tid % W, p = tid / W) hit 33 x + p, whose 8-byte bank pairs
// (x + p) mod 16 take every pair twice per warp, and line reads run along p.
// Every W keeps 64 registers a thread: 32 / W resident blocks of 32 W threads.
// A node sweep's cell tile [2][W + 1][cld] is filled with the W + 1 columns
// fastest (coalesced global loads): element (q, xx, p) at ((q (W + 1) + xx)
// cld + p); cld = 41 for W = 8 and 33 otherwise put every warp's 32 stores on
// 16 distinct 8-byte bank pairs twice, the minimum of two wavefronts (a row
// of 32 put the 9 columns of W = 8 on the same pairs: 9 wavefronts).
template <int W> struct TileGeom {
  static_assert(W == 8 || W == 16 || W == 32, "lines per block");
  static constexpr int ld = W == 8 ? kTileLd : 33;
  static constexpr int arr = W * ld;                 // doubles per staged array
  static constexpr int minb = 32 / W;                // resident blocks at 64 registers
  static constexpr int cld = W == 8 ? 41 : 33;       // row length of a node sweep's cell tile
};

// remapVariables "moy" kernel for a single-environment cell and the PerfectGas
// EOS (RemapADIFinal.cc:446-643, PerfectGasEOSService.cc:92-106, with
// PrepareRemap.cc:553-559).  out = rho, e, q, mass, p, c, -, mass fraction
// (0 when the cell was zeroed; conservation-energie-totale scales by it).
template <bool SP = false>
__device__ __forceinline__ void finalize_cell(const Phys& ph, const Scalars* S, double vol, const double u[4],
                                              double out[8], unsigned* oor = nullptr) {
  const double thr = ph.threshold;
  const double U0 = u[0], U1 = u[1], U2 = u[2], U3 = u[3];
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
    atomicOr(&const_cast<Scalars*>(S)->status, MHY_STATUS_ZERO_MASS);
  }
  double de = 0.;
  if (fvol > thr) { const double vn = U0 * vol * unsurvolt; de = U1 / vn; }
  const double density_nplus1 = 0. + fvol * de;
  const double cm = vol * density_nplus1;
  double ee = 0.;
  if (fvol > thr && U1 != 0.) ee = dv<double, SP>(U2, U1, 1. / masset, oor);   // masset = 0 + U1 = U1
  double energie = 0. + mf * ee;
  const double pv = U3 * unsurvol;
  const double pseudo = 0. + fvol * pv;
  double r = de;
  out[7] = mf;
  if (r < 0. || energie < 0.) { energie = 0.; r = 0.; out[7] = 0.; }   // RemapADIFinal.cc:611-626
  double pr, cc;
  eos_pc(ph.eos, ph.gamma, ph.pinf, r, energie, pr, cc);
  out[0] = r;
  out[1] = energie;
  out[2] = pseudo;
  out[3] = mf * cm;
  out[4] = pr;
  out[5] = cc;
}

// The mixed form's end of the remap for one environment: the moy kernel above
// with its volume and mass fractions, which are 1 for a single environment,
// folded in (rho = U1 / V, e = U2 / U1, q = U3 / V in FP64), and the
// PerfectGas EOS evaluated in FP32 (the StiffenedGas EOS, whose p + g pinf
// cancels, stays in FP64).
__device__ __forceinline__ void finalize_cell_mixed(const Phys& ph, const Scalars* S, double vol, const double u[4],
                                                    double out[8]) {
  const double U1 = u[1], U2 = u[2], U3 = u[3];
  if (U1 == 0.) atomicOr(&const_cast<Scalars*>(S)->status, MHY_STATUS_ZERO_MASS);
  const double unsurvol = 1. / vol;
  const double de = U1 * unsurvol;
  double e = U1 != 0. ? U2 / U1 : 0.;
  double r = de;
  out[7] = 1.;
  if (r < 0. || e < 0.) { e = 0.; r = 0.; out[7] = 0.; }
  double pr, cc;
  if (ph.eos == 0) {
    const float g = (float)ph.gamma, rf = (float)r, pf = (g - 1.f) * rf * (float)e;
    pr = pf;
    cc = sqrtf(g * pf / rf);
  } else {
    eos_pc(ph.eos, ph.gamma, ph.pinf, r, e, pr, cc);
  }
  out[0] = r;
  out[1] = e;
  out[2] = U3 * unsurvol;
  out[3] = vol * de;
  out[4] = pr;
  out[5] = cc;
}

// Phi = U / sum of the environment volumes = U / U0 for one environment
// (RemapADIService.cc:962-970, PrepareRemap.cc:394-398); Phi0 = U0/U0 = 1.
template <typename R, bool SP = false>
__device__ __forceinline__ void phi_of(const double U[4], R P[4], unsigned* oor = nullptr) {
  const R U0 = (R)U[0], r = Ar<R>::rcp(U0);
  P[0] = 1;
  P[1] = dv<R, SP>((R)U[1], U0, r, oor); P[2] = dv<R, SP>((R)U[2], U0, r, oor); P[3] = dv<R, SP>((R)U[3], U0, r, oor);
}

// Face gradients (R:174-177) of variables 1..3; variable 0 is zero.
template <typename R, bool SP = false>
__device__ __forceinline__ void face_grad(bool inner, R dx, const R Pn[4], const R Pp[4], R g[4], unsigned* oor = nullptr) {
  g[0] = 0;
  const R r = inner ? Ar<R>::rcp(dx) : R(0);
  unsigned fo = 0u;
#pragma unroll
  for (int v = 1; v < 4; ++v) g[v] = inner ? dv<R, SP>(Pn[v] - Pp[v], dx, r, &fo) : R(0);
  // lane 0's back neighbour is itself (0 / 0): its gradient reaches no updated cell
  if constexpr (SP) { if ((threadIdx.x & 31) != 0) *oor |= fo; }
}

// Limited cell gradient from the back and front face gradients (R:497-506):
//   gc = 0; if (gb != 0) gc += 0.5*(phi(gf/gb)*gb); if (gf != 0) gc += 0.5*(phi(gb/gf)*gf).
// For minmod, phi(r) = max(0, min(1, r)): with finite gb, gf of opposite signs or
// a zero the two terms are signed zeros and gc = +0; with equal signs the ratio
// whose numerator is the smaller magnitude is the only one below 1, the other
// term is exactly 0.5*g.  So one division gives the reference's bits.
template <typename R>
__device__ __forceinline__ R limited_one(int lim, R gb, R gf) {
  const R h = R(0.5), one = R(1), zero = R(0);
  if (lim == 0) {
    if (gb == zero || gf == zero || ((gb > zero) != (gf > zero))) return zero;
    const bool fsmall = fabs(gf) < fabs(gb);
    const R r = fsmall ? Ar<R>::quo(gf, gb) : Ar<R>::quo(gb, gf);
    const R t1 = fsmall ? h * (r * gb) : h * (one * gb);
    const R t2 = fsmall ? h * (one * gf) : h * (r * gf);
    return (zero + t1) + t2;
  }
  R gc = zero;
  if (gb != zero) gc += h * (limiter<R>(lim, Ar<R>::quo(gf, gb)) * gb);
  if (gf != zero) gc += h * (limiter<R>(lim, Ar<R>::quo(gb, gf)) * gf);
  return gc;
}

// Variable 0 (the volume) has Phi = U0/U0 = 1 on every cell of a
// single-environment mesh, so its face gradients are zero and its limited
// gradient is +0; only variables 1..3 are computed.
template <typename R>
__device__ __forceinline__ void limited_grad(int lim, const R gb[4], const R gf[4], R G[4]) {
  G[0] = 0;
#pragma unroll
  for (int v = 1; v < 4; ++v) G[v] = limited_one<R>(lim, gb[v], gf[v]);
}

// Upwind face value (R:707-714): from the previous cell when u_f dx_f > 0.
template <typename R>
__device__ __forceinline__ void face_value(R order2, bool back, R dot_xf, const R Pp[4], const R Gp[4],
                                           const R Pn[4], const R Gn[4], R Pf[4]) {
#pragma unroll
  for (int v = 0; v < 4; ++v) Pf[v] = back ? (Pp[v] + order2 * dot_xf * Gp[v]) : (Pn[v] + order2 * dot_xf * Gn[v]);
}

// ---- pente-borne (projection-pente-borne; FP64, one environment) ----------
// INTY (UtilesRemap.cc:83-93): integral from -infinity to X of the segment
// from (x0, y0) to (x1, y1), zero left of it and constant right of it.
__device__ __forceinline__ double pb_inty(double X, double x0, double y0, double x1, double y1, double thr) {
  double flux = 0.;
  if (fabs(x1 - x0) > thr) {
    const double eta = amin(amax(0., (X - x0) / (x1 - x0)), 1.);
    flux = (y0 + 0.5 * eta * (y1 - y0)) * (x1 - x0) * eta;
  }
  return flux;
}

// computeY0 (UtilesRemap.cc:184-238): the values of the reconstruction at the
// back and front ends of the cell, by limiter (ids of TypesMahyco.h:65-74).
__device__ __forceinline__ void pb_y0(int id, double yplus, double ymoins, double h0, double hplus, double hmoins,
                                      double& y0plus, double& y0moins) {
  y0plus = 0.; y0moins = 0.;
  if (id == 3 || id == 0) {
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

// One variable of computeFluxPP / computeFluxPPPure (UtilesRemap.cc:406-489,
// 628-705) before the debar fix: the integral of the three-piece
// reconstruction (computexgxd :246-266, computeygyd :276-296) over the
// length ppv next to the back (type 0) or front (type 1) face, or
// y0 * ppv where the cell is an extremum (formule 16).
__device__ __forceinline__ double pb_flux_var(int type, int lim_y0, double thr, double ppv, double y0, double yplus,
                                              double ymoins, double h0, double hplus, double hmoins, double grady) {
  double y0plus, y0moins;
  pb_y0(lim_y0, yplus, ymoins, h0, hplus, hmoins, y0plus, y0moins);
  double xplus = 1.;
  if (fabs(y0plus - yplus) > thr) xplus = (y0 - yplus) / (y0plus - yplus) - 1. / 2.;
  double xmoins = 1.;
  if (fabs(y0moins - ymoins) > thr) xmoins = (y0 - ymoins) / (y0moins - ymoins) - 1. / 2.;
  const double xd = +h0 * amin(amax(xplus, -1. / 2.), 1. / 2.);
  const double xg = -h0 * amin(amax(xmoins, -1. / 2.), 1. / 2.);
  const double xtd = y0 + h0 / 2 * grady;
  const double xtg = y0 - h0 / 2 * grady;
  const double ad = amin(yplus, 2. * y0moins - ymoins), bd = amax(yplus, 2. * y0moins - ymoins);
  const double ag = amin(ymoins, 2. * y0plus - yplus), bg = amax(ymoins, 2. * y0plus - yplus);
  const double yd = amin(amax(xtd, ad), bd);
  const double yg = amin(amax(xtg, ag), bg);
  double f1, f2, f3, f1m, f2m, f3m;
  if (type == 0) {
    f1m = pb_inty(-h0 / 2. + ppv, -h0 / 2., ymoins, xg, yg, thr);
    f1 = pb_inty(-h0 / 2., -h0 / 2., ymoins, xg, yg, thr);
    f2m = pb_inty(-h0 / 2. + ppv, xg, yg, xd, yd, thr);
    f2 = pb_inty(-h0 / 2., xg, yg, xd, yd, thr);
    f3m = pb_inty(-h0 / 2. + ppv, xd, yd, h0 / 2., yplus, thr);
    f3 = pb_inty(-h0 / 2., xd, yd, h0 / 2., yplus, thr);
  } else {
    f1 = pb_inty(h0 / 2. - ppv, -h0 / 2., ymoins, xg, yg, thr);
    f1m = pb_inty(h0 / 2., -h0 / 2., ymoins, xg, yg, thr);
    f2 = pb_inty(h0 / 2. - ppv, xg, yg, xd, yd, thr);
    f2m = pb_inty(h0 / 2., xg, yg, xd, yd, thr);
    f3 = pb_inty(h0 / 2. - ppv, xd, yd, h0 / 2., yplus, thr);
    f3m = pb_inty(h0 / 2., xd, yd, h0 / 2., yplus, thr);
  }
  double flux = tmax<double>(((f1m - f1) + (f2m - f2) + (f3m - f3)), 0.);
  if (((yplus - y0) * (ymoins - y0)) >= 0.) flux = y0 * ppv;
  return flux;
}

// The four fluxes (volume, mass, energy, q) leaving the cell through one
// face, debar fix included (UtilesRemap.cc:518-619, 709-819; the momentum and
// kinetic-energy variables have Phi = 0 and move nothing).
__device__ __forceinline__ void pb_fluxes(const Phys& ph, int type, double ppv, const double P[4], const double Pn[4],
                                          const double Pp[4], double h0, double hp, double hm, const double G[4],
                                          double F[4]) {
  const double thr = ph.threshold;
#pragma unroll
  for (int v = 0; v < 4; ++v) F[v] = pb_flux_var(type, ph.pb_lim_y0, thr, ppv, P[v], Pn[v], Pp[v], h0, hp, hm, G[v]);
  if (ph.pb_debar == 1) {
    const double svol = 0. + F[0];
    if (fabs(svol) > thr) {
      if (!ph.pb_pure) F[1] = (F[1] / svol) * F[0];
      F[2] = (F[2] / svol) * F[1];
    } else {
      F[0] = F[1] = F[2] = F[3] = 0.;
    }
  } else if (ph.pb_debar == 2) {
    if (!ph.pb_pure) F[1] = P[1] * F[0];
    F[2] = P[2] * F[1];
  }
  if (ppv == 0.) F[0] = F[1] = F[2] = F[3] = 0.;
}

// Order-3 face value of one variable (Remap-ordre-3.cc:7-131): y and h of
// the six cells bbb, bb, b | f, ff, fff around the face (clamped at the ends
// of the line) and u_f dt.
__device__ __forceinline__ double o3_grad(double hm, double h0, double hp, double ym, double y0, double yp) {
  return h0 / (hm + h0 + hp) * ((2. * hm + h0) / (h0 + hp) * (yp - y0) + (h0 + 2. * hp) / (hm + h0) * (y0 - ym));
}
__device__ __forceinline__ double o3_ystar(double hmm, double hm, double hp, double hpp, double ymm, double ym,
                                           double yp, double ypp, double gradm, double gradp) {
  const double tmp1 = (2. * hp * hm) / (hm + hp) * ((hmm + hm) / (2. * hm + hp) - (hpp + hp) / (2. * hp + hm)) * (yp - ym);
  const double tmp2 = -hm * (hmm + hm) / (2. * hm + hp) * gradp + hp * (hp + hpp) / (hm + 2. * hp) * gradm;
  return ym + hm / (hm + hp) * (yp - ym) + 1. / (hmm + hm + hp + hpp) * (tmp1 + tmp2);
}
__device__ __forceinline__ double o3_flux(const double y[6], const double h[6], double vdt) {
  const double ymmm = y[0], ymm = y[1], ym = y[2], yp = y[3], ypp = y[4], yppp = y[5];
  const double hmmm = h[0], hmm = h[1], hm = h[2], hp = h[3], hpp = h[4], hppp = h[5];
  const double gradmm = o3_grad(hmmm, hmm, hm, ymmm, ymm, ym);
  const double gradm = o3_grad(hmm, hm, hp, ymm, ym, yp);
  const double gradp = o3_grad(hm, hp, hpp, ym, yp, ypp);
  const double gradpp = o3_grad(hp, hpp, hppp, yp, ypp, yppp);
  const double ystarm = o3_ystar(hmmm, hmm, hm, hp, ymmm, ymm, ym, yp, gradmm, gradm);
  const double ystar = o3_ystar(hmm, hm, hp, hpp, ymm, ym, yp, ypp, gradm, gradp);
  const double ystarp = o3_ystar(hm, hp, hpp, hppp, ym, yp, ypp, yppp, gradp, gradpp);
  const double ym_m = ystarm, ym_p = ystar, yp_m = ystar, yp_p = ystarp;
  const double grad_m = ym_p - ym_m, grad_p = yp_p - yp_m;
  const double ym6 = 6. * (ym - 0.5 * (ym_m + ym_p));
  const double yp6 = 6. * (yp - 0.5 * (yp_m + yp_p));
  double flux;
  if (vdt > 0.) { const double x = vdt, dx = hm; flux = ym_p - 0.5 * x / dx * (grad_m - (1. - 2. / 3. * x / dx) * ym6); }
  else if (vdt < 0.) { const double x = -vdt, dx = hp; flux = yp_m + 0.5 * x / dx * (grad_p - (1. - 2. / 3. * x / dx) * yp6); }
  else return 0.;
  const double num = vdt / hm, nup = vdt / hp;
  const double ym_ym = ym + (1. - num) / num * (ym - ymm);
  const double yp_ym = yp - (1. + nup) / nup * (yp - ypp);
  const double i10 = amin(ym, yp), i11 = amax(ym, yp);
  double i20, i21;
  if (vdt >= 0.) { i20 = amin(ym, ym_ym); i21 = amax(ym, ym_ym); }
  else { i20 = amin(yp, yp_ym); i21 = amax(yp, yp_ym); }
  double l0, l1;
  if ((i11 < i20) || (i21 < i10)) { l0 = 0.; l1 = 0.; }
  else { l0 = amax(i10, i20); l1 = amin(i11, i21); }
  if (flux < l0) flux = l0;
  if (flux > l1) flux = l1;
  return flux;
}

// ---- cells ---------------------------------------------------------------
// Inputs of one lane (one cell of a line along d).
struct CellIn {
  double U[4], xc[3];
  double db, df, u, A, n[3];   // low face of the cell along d (inner faces only)
  double ob, of;               // outward-normal component along d of the back and front faces
  double vol;                  // initial cell volume (last sweep only)
  double pf3[4];               // order 3: Phi of the low face from k_o3_faces
  double h;                    // G limiters: cell width along d (RemapADIService.cc:225-258)
  double pb[3];                // pente-borne: rho and e (first sweep only) and the q of the remap's start
};
constexpr int kCellOutLast = 8;   // rho, e, q, mass, p, c, dual mass flux, mass fraction
constexpr int kCellOutMid = 5;    // U0..U3, dual mass flux

// One line step of computeGradPhiFace, computeGradPhiCell, the upwind face
// values and computeUremap_PBorn0 (RemapADIService.cc:91-271, 447-517, 658-720,
// 909-987).  Every lane takes part in the shuffles; lanes with upd set get
// their cell's results in out.  The boundary faces of d carry Phi_f = 0 and
// contribute nothing.  PB: the pente-borne form (R = double): Phi of
// PrepareRemap.cc:201-212 (first sweep) or RemapADIService.cc:805-834, the
// general gradient (R:319-378), face values from the fluxes leaving the two
// cells (R:380-431, 574-578) and fluxes o*A*Phi_f (R:770-774).
template <bool LAST, typename R = double, bool O3 = false, bool GL = false, bool PB = false, bool SP = false>
__device__ __forceinline__ void cell_line(const Phys& ph, double dt, const Scalars* S, bool valid, bool inner,
                                          bool infr, bool upd, const CellIn& in, double* out, unsigned* oor = nullptr) {
  const R order2 = (R)(ph.ordre_projection - 1);
  const int lim = ph.ordre_projection > 1 ? ph.lim_cell : -1;
  R P[4] = {0, 0, 0, 0};
  if constexpr (PB) {
    if (valid) {
      if (ph.pb_first) {
        P[0] = 1.; P[1] = in.pb[0]; P[2] = in.pb[1];      // volume fraction, density, internal energy
      } else {
        P[0] = in.U[0] / (0. + in.U[0]);
        P[1] = in.U[0] != 0. ? in.U[1] / in.U[0] : 0.;
        P[2] = in.U[1] != 0. ? in.U[2] / in.U[1] : 0.;
      }
      P[3] = in.pb[2];
    }
  } else {
    if (valid) phi_of<R, SP>(in.U, P, oor);
  }
  const unsigned full = 0xffffffffu;
  const double xpx = __shfl_up_sync(full, in.xc[0], 1), xpy = __shfl_up_sync(full, in.xc[1], 1),
               xpz = __shfl_up_sync(full, in.xc[2], 1);
  // dx_f = (x_c(next) - x_c(prev)).n0 (RemapADIService.cc:171-172), from the
  // FP64 cell centres in every precision
  const double dx = inner ? dot(d3(in.xc[0], in.xc[1], in.xc[2]) - d3(xpx, xpy, xpz), d3(in.n[0], in.n[1], in.n[2]))
                          : 0.;
  R g[4], gr[4], G[4], Pp[4], Gp[4], Pf[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) Pp[v] = __shfl_up_sync(full, P[v], 1);
  if constexpr (PB) {
    const R r = inner ? Ar<R>::rcp((R)dx) : R(0);
#pragma unroll
    for (int v = 0; v < 4; ++v) g[v] = inner ? Ar<R>::div(P[v] - Pp[v], (R)dx, r) : R(0);
  } else {
    face_grad<R, SP>(inner, (R)dx, P, Pp, g, oor);
  }
#pragma unroll
  for (int v = 0; v < 4; ++v) gr[v] = __shfl_down_sync(full, g[v], 1);
  if constexpr (PB) {
    static_assert(sizeof(R) == 8, "pente-borne is FP64");
    double Pn[4], Pne[4], Ppe[4], ar[4], av[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) Pn[v] = __shfl_down_sync(full, P[v], 1);
    const double hb = __shfl_up_sync(full, in.h, 1), hn = __shfl_down_sync(full, in.h, 1);
    const double h0 = in.h, hm = inner ? hb : in.h, hp = infr ? hn : in.h;   // the cell itself at the ends
#pragma unroll
    for (int v = 0; v < 4; ++v) { Pne[v] = infr ? Pn[v] : P[v]; Ppe[v] = inner ? Pp[v] : P[v]; }
#pragma unroll
    for (int v = 0; v < 4; ++v)
      G[v] = lim < 3 ? limited_one<R>(lim, g[v], gr[v])
                     : flux_limiter_g<R>(lim, gr[v], g[v], P[v], Pne[v], Ppe[v], h0, hp, hm);
    const double un = __shfl_down_sync(full, in.u, 1);
    const double ob = in.ob * in.u, of = in.of * un;                 // outward velocities of the two faces
    pb_fluxes(ph, 0, 0.5 * (ob + fabs(ob)) * dt, P, Pne, Ppe, h0, hp, hm, G, ar);
    pb_fluxes(ph, 1, 0.5 * (of + fabs(of)) * dt, P, Pne, Ppe, h0, hp, hm, G, av);
    // back face: what leaves the previous cell forwards minus what leaves this one backwards
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const double avp = __shfl_up_sync(full, av[v], 1);
      Pf[v] = inner ? avp - ar[v] : 0.;
    }
  } else if constexpr (GL) {
    // generalised limiters (RemapADIService.cc:319-437 -> UtilesRemap.cc:295-330):
    // back and front cells are the cell itself at the ends of the line
    R Pn[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) Pn[v] = __shfl_down_sync(full, P[v], 1);
    const double hb = __shfl_up_sync(full, in.h, 1), hn = __shfl_down_sync(full, in.h, 1);
    const R h0 = (R)in.h, hm = (R)(inner ? hb : in.h), hp = (R)(infr ? hn : in.h);
#pragma unroll
    for (int v = 0; v < 4; ++v)
      G[v] = flux_limiter_g<R>(lim, gr[v], g[v], P[v], infr ? Pn[v] : P[v], inner ? Pp[v] : P[v], h0, hp, hm);
  } else {
    limited_grad<R>(lim, g, gr, G);
  }
#pragma unroll
  for (int v = 0; v < 4; ++v) Gp[v] = __shfl_up_sync(full, G[v], 1);
  if constexpr (PB) {
  } else if (inner) {
    if constexpr (O3) {                                   // order 3: R:583-641, computed per face beforehand
#pragma unroll
      for (int v = 0; v < 4; ++v) Pf[v] = (R)in.pf3[v];
    } else {
      const bool back = in.u * dx > 0.0;
      face_value<R>(order2, back, (R)(back ? in.db : in.df), Pp, Gp, P, G, Pf);
    }
  } else {
#pragma unroll
    for (int v = 0; v < 4; ++v) Pf[v] = 0;
  }
  R Pfn[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) Pfn[v] = __shfl_down_sync(full, Pf[v], 1);
  const double un = __shfl_down_sync(full, in.u, 1), An = __shfl_down_sync(full, in.A, 1);
  if (!upd) return;
  // fluxes o*u*A*dt*Phi_f through the back and front faces, U -= sum, dual
  // mass flux sum 0.5*flux*o, clamping of mass and energy (R:909-987); the
  // sums are FP64 in every precision (each face flux is one rounded value,
  // subtracted from one cell and added to the other)
  const double cb = inner ? (PB ? in.ob * in.A : in.ob * in.u * in.A * dt) : 0.;
  const double cf = infr ? (PB ? in.of * An : in.of * un * An * dt) : 0.;
  double u[4], dpm = 0.;
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    double flux_face = 0., dp = 0.;
    if (inner) { const double fl = (double)((R)cb * Pf[v]); flux_face += fl; dp += 0.5 * fl * in.ob; }
    if (infr) { const double fl = (double)((R)cf * Pfn[v]); flux_face += fl; dp += 0.5 * fl * in.of; }
    u[v] = in.U[v] - flux_face;
    if (v == 1) dpm = dp;
  }
  if (u[1] < 0.) u[1] = 0.;
  if (u[2] < 0.) u[2] = 0.;
  if (!LAST) {
#pragma unroll
    for (int v = 0; v < 4; ++v) out[v] = u[v];
    out[4] = dpm;
  } else {
    if constexpr (sizeof(R) == 4) finalize_cell_mixed(ph, S, in.vol, u, out);
    else finalize_cell<SP>(ph, S, in.vol, u, out, oor);
    out[6] = dpm;
  }
}

// ---- nodes ---------------------------------------------------------------
// Dual update of one inner node (DualPhaseRemap.cc:382-521).
template <typename R>
__device__ __forceinline__ void dual_update(int D, R order2, R dt, double bfm, double ffm,
                                            const R Pm[4], const R Pn[4], const R Pp[4],
                                            const R Gm[3], const R Gn[3], const R Gp[3],
                                            R hb, R hf, double ud[5]) {
  const double u3 = ud[3] + (bfm - ffm);
  const R h = R(0.5), zero = R(0);
  const R pnd = Pn[D];
  const R ufront = h * (pnd + pnd);                            // DualPhaseRemap.cc:391
  const R sfront = (ufront > zero) ? R(1) : R(-1);
  const R uback = h * (Pm[D] + pnd);
  const R sback = (uback > zero) ? R(1) : R(-1);
  const bool fup = ffm < 0., bup = bfm > 0.;
  const R tf = sfront * hf - dt * ufront;                      // hf = x(front) - x, hb = x - x(back)
  const R tb = sback * hb - dt * uback;
  double out[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const R gfa = c < 3 ? (fup ? Gp[c] : Gn[c]) : zero;        // index 4 never set (DualPhaseRemap.cc:771)
    const R gba = c < 3 ? (bup ? Gm[c] : Gn[c]) : zero;
    const R FV = (fup ? Pp[c] : Pn[c]) + order2 * (h * gfa * tf);
    const R BV = (bup ? Pm[c] : Pn[c]) + order2 * (h * gba * tb);
    out[c] = ud[c < 3 ? c : 4] + (bfm * (double)BV - ffm * (double)FV);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) if (fabs(out[c]) < 1.e-300) out[c] = 0.;
  ud[0] = out[0]; ud[1] = out[1]; ud[2] = out[2]; ud[3] = u3; ud[4] = out[3];
}

// One limited nodal gradient component (DualPhaseRemap.cc:736-777) from the
// back and front differences; the terms are (0.5*phi(r))*g here, and the same
// single-division reading of minmod applies.
template <typename R>
__device__ __forceinline__ R dual_limited(int lim, R gb, R gf) {
  const R h = R(0.5), one = R(1), zero = R(0);
  R g = zero;
  if (lim == 0) {
    if (!(gb == zero || gf == zero || ((gb > zero) != (gf > zero)))) {
      const bool fsmall = fabs(gf) < fabs(gb);
      const R r = fsmall ? Ar<R>::quo(gf, gb) : Ar<R>::quo(gb, gf);
      const R t1 = fsmall ? h * r * gb : h * one * gb;
      const R t2 = fsmall ? h * one * gf : h * r * gf;
      g = (zero + t1) + t2;
    }
  } else {
    if (gb != zero) g += h * limiter<R>(lim, Ar<R>::quo(gf, gb)) * gb;
    if (gf != zero) g += h * limiter<R>(lim, Ar<R>::quo(gb, gf)) * gf;
  }
  return g;
}

// Inputs of one lane (one node of a line along d).
struct NodeIn {
  double vh[3];    // Lagrange velocity
  double x0d;      // initial coordinate along d (the Lagrangian one with schema-csts)
  double nm;       // node mass (first sweep)
  double ud[5];    // U_dual (later sweeps)
  double ffm;      // sum of 0.25 * dual mass flux of the 4 cells in front (DualPhaseRemap.cc:299-340)
  double msum;     // sum of the masses of the up to 8 cells around the node (last sweep)
  double x2[2];    // G limiters, halo lanes 1 and 30: the coordinates along d two nodes back / ahead,
                   // which lie outside the warp's segment
};
constexpr int kNodeOut = 5;       // U_dual[0..4], or v.x, v.y, v.z, node mass, |v| on the last sweep
constexpr int kNodeOutLast = 6;   // the last sweep adds the node's conservation-energie-totale term

// One line step of computeDualUremap and computeDualGradPhi_LimC
// (DualPhaseRemap.cc:22-523, 700-778), then remapVariables for the node
// velocity and mass on the last sweep (RemapADIFinal.cc:660-672, 697-719;
// |v| is kept for the dt reduction, MahycoModule.cc:2053).  The state at the
// start of a sweep is PrepareRemap.cc:411-433 on the first sweep or for nodes
// not yet updated this cycle, else U_dual / m.  G holds the node's stale
// gradient on entry and its gradient on return.
template <int D, bool FIRST, bool LAST, typename R = double, bool GL = false, bool SP = false>
__device__ __forceinline__ void node_line(const Phys& ph, double dt, bool valid, bool inner, bool updated,
                                          bool upd, const NodeIn& in, R G[3], double* out, bool xabs = false,
                                          bool bb_ok = true, bool ff_ok = true, unsigned* oor = nullptr) {
  const R order2 = (R)(ph.ordre_projection - 1);
  const int lim = ph.ordre_projection > 1 ? ph.limiteur_id : -1;
  const bool grad_on = ph.ordre_projection > 1;
  double ud[5] = {0., 0., 0., 0., 0.}, x = 0.;
  R P[4] = {0, 0, 0, 0};
  if (valid) {
    const D3 u = d3(in.vh[0], in.vh[1], in.vh[2]);
    if (FIRST) {
      const double m = in.nm;
      const double un = norm2(u);
      ud[0] = m * u.x; ud[1] = m * u.y; ud[2] = m * u.z; ud[3] = m; ud[4] = 0.5 * m * un;
      P[0] = (R)u.x; P[1] = (R)u.y; P[2] = (R)u.z; P[3] = (R)(0.5 * un);
    } else {
#pragma unroll
      for (int c = 0; c < 5; ++c) ud[c] = in.ud[c];
      if (updated) {
        const R m = (R)ud[3], rm = Ar<R>::rcp(m);
        P[0] = dv<R, SP>((R)ud[0], m, rm, oor); P[1] = dv<R, SP>((R)ud[1], m, rm, oor);
        P[2] = dv<R, SP>((R)ud[2], m, rm, oor); P[3] = dv<R, SP>((R)ud[4], m, rm, oor);
      } else {
        P[0] = (R)u.x; P[1] = (R)u.y; P[2] = (R)u.z; P[3] = (R)(0.5 * norm2(u));
      }
    }
    x = xabs ? in.x0d : in.x0d + in.vh[D] * dt;       // xabs: x0d holds the Lagrangian coordinate
  }
  const unsigned full = 0xffffffffu;
  R Pm[4], Pp[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) { Pm[c] = __shfl_up_sync(full, P[c], 1); Pp[c] = __shfl_down_sync(full, P[c], 1); }
  const double xm = __shfl_up_sync(full, x, 1), xp = __shfl_down_sync(full, x, 1);
  if (grad_on) {
    // front difference quotient of this node = back difference quotient of the next
    const R hf = (R)(xp - x), rf = Ar<R>::rcp(hf);
    R gf[3], gb[3];
    // speculative quotients count only where they are used: a valid node
    // whose next node is valid and in this warp (the last lane divides by 0)
    unsigned gfo = 0u;
#pragma unroll
    for (int c = 0; c < 3; ++c) gf[c] = dv<R, SP>(Pp[c] - P[c], hf, rf, &gfo);
    if constexpr (SP) {
      const int next_valid = __shfl_down_sync(full, valid ? 1 : 0, 1);   // every lane takes part
      if (valid && (threadIdx.x & 31) < 31 && next_valid != 0) *oor |= gfo;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) gb[c] = __shfl_up_sync(full, gf[c], 1);
    if constexpr (GL) {
      // generalised limiters (DualPhaseRemap.cc:48-64, UtilesRemap.cc:15-80,
      // 346-377): every gradient zeroed, inner nodes from the dual widths
      const int lane = threadIdx.x & 31;
      double xm2 = __shfl_up_sync(full, x, 2), xp2 = __shfl_down_sync(full, x, 2);
      if (lane == 1) xm2 = in.x2[0];
      if (lane == 30) xp2 = in.x2[1];
#pragma unroll
      for (int c = 0; c < 3; ++c) G[c] = R(0);
      if (valid && inner) {
        const R h0 = (R)(0.5 * (xp - xm));
        R hmo, hpl;
        if (!bb_ok) { hmo = R(0); hpl = (R)(0.5 * (xp2 - x)); }
        else if (!ff_ok) { hpl = R(0); hmo = (R)(0.5 * (x - xm2)); }
        else { hmo = (R)(0.5 * (x - xm2)); hpl = (R)(0.5 * (xp2 - x)); }
#pragma unroll
        for (int c = 0; c < 3; ++c) G[c] = flux_limiter_g<R>(lim, gf[c], gb[c], P[c], Pp[c], Pm[c], h0, hpl, hmo);
      }
    } else if (valid && inner) {
#pragma unroll
      for (int c = 0; c < 3; ++c) G[c] = dual_limited<R>(lim, gb[c], gf[c]);
    }
  }
  R Gm[3], Gp[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) { Gm[c] = __shfl_up_sync(full, G[c], 1); Gp[c] = __shfl_down_sync(full, G[c], 1); }
  const double bfm = __shfl_up_sync(full, in.ffm, 1);  // back cells of node m = front cells of node m-1
  if (!upd) return;
  if (inner) dual_update<R>(D, order2, (R)dt, bfm, in.ffm, Pm, P, Pp, Gm, G, Gp, (R)(x - xm), (R)(xp - x), ud);
  if (!LAST) {
#pragma unroll
    for (int c = 0; c < 5; ++c) out[c] = ud[c];
  } else {
    const double m = ud[3];
    D3 u;
    double rm = 0.;
    if (m != 0.) {
      rm = 1.0 / m;
      u = d3(dv<double, SP>(ud[0], m, rm, oor), dv<double, SP>(ud[1], m, rm, oor), dv<double, SP>(ud[2], m, rm, oor));
    } else {
      u = d3(in.vh[0], in.vh[1], in.vh[2]);
    }
    out[0] = u.x; out[1] = u.y; out[2] = u.z; out[3] = .125 * in.msum; out[4] = norm2(u);
    // conservation-energie-totale (RemapADIFinal.cc:757-764): this node's
    // share 0.25 (ec_proj - ec_reconst) of the kinetic energy the remap lost,
    // ec_proj = U_dual[4] / U_dual[3], ec_reconst = 0.5 |v|^2; nothing for a
    // node of zero mass
    if (ph.cons_ec)
      out[5] = m != 0. ? 0.25 * (dv<double, SP>(ud[4], m, rm, oor) - 0.5 * (u.x * u.x + u.y * u.y + u.z * u.z)) : 0.;
  }
}

// Outputs of one lane's line step, as the sweeps' exact recomputations return them.
template <int NO> struct LineOut { double v[NO]; };
struct NodeLineOut { double v[kNodeOutLast]; double g[3]; };

// inner along an earlier direction of this cycle: Phi_dual = U_dual / m there
__device__ __forceinline__ bool node_updated(const Dims& dm, int D, int prev_inner, const int idx[3]) {
  bool updated = false;
#pragma unroll
  for (int dd = 0; dd < 3; ++dd)
    if (dd != D && (prev_inner >> dd & 1) && idx[dd] > 0 && idx[dd] < dm.ncd(dd)) updated = true;
  return updated;
}

// the node lies on a boundary plane of another direction: its gradient is
// kept for later cycles, where it is read as a stale value
__device__ __forceinline__ bool node_on_plane(const Dims& dm, int D, const int idx[3]) {
  return (D != 0 && (idx[0] == 0 || idx[0] == dm.nx)) || (D != 1 && (idx[1] == 0 || idx[1] == dm.ny)) ||
         (D != 2 && (idx[2] == 0 || idx[2] == dm.nz));
}

// Node sweep along x: lanes run along the rows of nodes.  nodes_x_line is one
// lane's loads and line step.  The body runs it with speculative FP64
// quotients; in a warp where any lane's were out of range it recomputes the
// segment exactly out of line (nodes_x_line_exact reloads the inputs, so
// that none of them stays live across the common path), then stores.
template <bool FIRST, bool LAST, int K, typename R, bool GL, bool SP>
__device__ __forceinline__ void nodes_x_line(const Dims& dm, const Scalars* __restrict__ S, const Phys& ph,
    int prev_inner, const double* __restrict__ x0, const double* __restrict__ xl, const double* __restrict__ vh,
    const double* __restrict__ nm_in, const double* __restrict__ udin, const double* __restrict__ dpf,
    const double* __restrict__ Gd, const double* __restrict__ mass, int bx_, int by_, int bz_, R G[3], double* out,
    unsigned* oor) {
  const int lane = threadIdx.x & 31;
  const int j = by_ * kLineWarps + (threadIdx.x >> 5), k = bz_;
  const int nx = dm.nx, ny = dm.ny, nz = dm.nz, N = (int)dm.N;
  const int m = bx_ * kLineUpd - 2 + lane;      // position of this lane's node along x
  const bool valid = m >= 0 && m <= nx;
  const bool inner = m >= 1 && m <= nx - 1;
  const bool upd = valid && lane >= 2 && lane < 2 + kLineUpd;
  const int idx[3] = {valid ? m : 0, j, k};
  const int n = idx[0] + (nx + 1) * (j + (ny + 1) * k);
  const bool updated = node_updated(dm, 0, prev_inner, idx);
  const bool grad_on = ph.ordre_projection > 1;
  NodeIn in;
  in.vh[0] = in.vh[1] = in.vh[2] = 0.; in.x0d = 0.; in.nm = 0.;
  in.ud[0] = in.ud[1] = in.ud[2] = in.ud[3] = in.ud[4] = 0.; in.ffm = 0.; in.msum = 0.;
  in.x2[0] = in.x2[1] = 0.;
  G[0] = G[1] = G[2] = R(0);
  if (GL && valid && (lane == 1 || lane == 30)) {
    const int q = lane == 1 ? m - 2 : m + 2;           // the node two back (lane 1) or ahead (lane 30)
    if (q >= 0 && q <= nx) {
      const int nq = n + (q - m);
      in.x2[lane == 1 ? 0 : 1] = xl ? xl[nq] : x0[nq] + vh[nq] * S->dt;
    }
  }
  if (valid) {
    in.vh[0] = vh[n]; in.vh[1] = vh[N + n]; in.vh[2] = vh[2 * N + n]; in.x0d = xl ? xl[n] : x0[n];
    if (FIRST) in.nm = nm_in[n];
    else {
#pragma unroll
      for (int c = 0; c < 5; ++c) in.ud[c] = udin[c * N + n];
    }
    // flux of the 4 cells in front (x index m), in the order of DualPhaseRemap.cc:299-340
    // (s1 over y, s2 over z; environments innermost)
    if (m < nx) {
      const int C = (int)dm.C;
      double f = 0.;
#pragma unroll
      for (int s1 = -1; s1 <= 0; ++s1)
#pragma unroll
        for (int s2 = -1; s2 <= 0; ++s2) {
          const int cj = j + s1, ck = k + s2;
          if (cj >= 0 && cj < ny && ck >= 0 && ck < nz) {
            const int c = m + nx * (cj + ny * ck);
#pragma unroll
            for (int e = 0; e < K; ++e) f += 0.25 * dpf[e * C + c];
          }
        }
      in.ffm = f;
    }
    if (!(inner && grad_on)) { G[0] = (R)Gd[n]; G[1] = (R)Gd[N + n]; G[2] = (R)Gd[2 * N + n]; }
    if (LAST && upd) {
      double sm = 0.;
#pragma unroll
      for (int dk = 1; dk >= 0; --dk)
#pragma unroll
        for (int dj = 1; dj >= 0; --dj)
#pragma unroll
          for (int di = 1; di >= 0; --di) {
            const int ci = m - di, cj = j - dj, ck = k - dk;
            if (ci < 0 || cj < 0 || ck < 0 || ci >= nx || cj >= ny || ck >= nz) continue;
            sm += mass[ci + nx * (cj + ny * ck)];
          }
      in.msum = sm;
    }
  }
  node_line<0, FIRST, LAST, R, GL, SP>(ph, S->dt, valid, inner, updated, upd, in, G, out, xl != nullptr, m >= 2,
                                       m + 2 <= nx, oor);
}

template <bool FIRST, bool LAST, int K, typename R, bool GL>
__device__ __noinline__ NodeLineOut nodes_x_line_exact(Dims dm, const Scalars* S, Phys ph, int prev_inner,
    const double* x0, const double* xl, const double* vh, const double* nm_in, const double* udin, const double* dpf,
    const double* Gd, const double* mass, int bx_, int by_, int bz_) {
  NodeLineOut o;
  R G[3];
  nodes_x_line<FIRST, LAST, K, R, GL, false>(dm, S, ph, prev_inner, x0, xl, vh, nm_in, udin, dpf, Gd, mass, bx_, by_,
                                             bz_, G, o.v, nullptr);
  o.g[0] = (double)G[0]; o.g[1] = (double)G[1]; o.g[2] = (double)G[2];
  return o;
}

template <bool FIRST, bool LAST, int K, typename R, bool GL = false>
__device__ __forceinline__ void k_cyc_sweep_nodes_x_body(Dims dm, const Scalars* __restrict__ S,
    Phys ph, int prev_inner, const double* __restrict__ x0, const double* __restrict__ xl, const double* __restrict__ vh,
    const double* __restrict__ nm_in, const double* __restrict__ udin, double* __restrict__ udout,
    const double* __restrict__ dpf, double* __restrict__ Gd, const double* __restrict__ mass,
    double* __restrict__ vout, double* __restrict__ nm_out, double* __restrict__ vnorm,
    int bx_, int by_, int bz_, double* __restrict__ ecn = nullptr) {
  const int lane = threadIdx.x & 31;
  const int j = by_ * kLineWarps + (threadIdx.x >> 5), k = bz_;
  if (j > dm.ny) return;                               // whole warp leaves together
  R G[3];
  double out[LAST ? kNodeOutLast : kNodeOut];
  if constexpr (sizeof(R) == 8) {
    unsigned oor = 0u;
    nodes_x_line<FIRST, LAST, K, R, GL, true>(dm, S, ph, prev_inner, x0, xl, vh, nm_in, udin, dpf, Gd, mass, bx_, by_,
                                              bz_, G, out, &oor);
    if (__any_sync(0xffffffffu, oor != 0u)) {
      const NodeLineOut o = nodes_x_line_exact<FIRST, LAST, K, R, GL>(dm, S, ph, prev_inner, x0, xl, vh, nm_in, udin,
                                                                      dpf, Gd, mass, bx_, by_, bz_);
#pragma unroll
      for (int c = 0; c < (LAST ? kNodeOutLast : kNodeOut); ++c) out[c] = o.v[c];
      G[0] = o.g[0]; G[1] = o.g[1]; G[2] = o.g[2];
    }
  } else {
    nodes_x_line<FIRST, LAST, K, R, GL, false>(dm, S, ph, prev_inner, x0, xl, vh, nm_in, udin, dpf, Gd, mass, bx_, by_,
                                               bz_, G, out, nullptr);
  }
  const int nx = dm.nx, ny = dm.ny, N = (int)dm.N;
  const int m = bx_ * kLineUpd - 2 + lane;
  const bool upd = m >= 0 && m <= nx && lane >= 2 && lane < 2 + kLineUpd;
  const bool inner = m >= 1 && m <= nx - 1;
  const bool grad_on = ph.ordre_projection > 1;
  const int idx[3] = {m, j, k};
  const int n = m + (nx + 1) * (j + (ny + 1) * k);
  if (!upd) return;
  if (inner && grad_on && node_on_plane(dm, 0, idx)) { Gd[n] = (double)G[0]; Gd[N + n] = (double)G[1]; Gd[2 * N + n] = (double)G[2]; }
  if (!LAST) {
#pragma unroll
    for (int c = 0; c < 5; ++c) udout[c * N + n] = out[c];
  } else {
    vout[n] = out[0]; vout[N + n] = out[1]; vout[2 * N + n] = out[2]; nm_out[n] = out[3]; vnorm[n] = out[4];
    if (ecn) ecn[n] = out[5];
  }
}

template <bool FIRST, bool LAST, int K, typename R, bool GL = false>
__global__ void __launch_bounds__(32 * kLineWarps, kLineMinBlocks) k_cyc_sweep_nodes_x(Dims dm, const Scalars* __restrict__ S,
    Phys ph, int prev_inner, const double* __restrict__ x0, const double* __restrict__ xl, const double* __restrict__ vh,
    const double* __restrict__ nm_in, const double* __restrict__ udin, double* __restrict__ udout,
    const double* __restrict__ dpf, double* __restrict__ Gd, const double* __restrict__ mass,
    double* __restrict__ vout, double* __restrict__ nm_out, double* __restrict__ vnorm, double* __restrict__ ecn) {
  k_cyc_sweep_nodes_x_body<FIRST, LAST, K, R, GL>(dm, S, ph, prev_inner, x0, xl, vh, nm_in, udin, udout, dpf, Gd, mass, vout, nm_out, vnorm, blockIdx.x, blockIdx.y, blockIdx.z, ecn);
}

// Node sweep along y (D = 1) or z (D = 2), staged through shared memory.
// Block (bx, by, bz): node x = 8 bx .. 8 bx + 7, positions 28 by - 2 ..
// 28 by + 29 along D, bz = the remaining node coordinate o (z for D = 1, y
// for D = 2).  The cells around those nodes have x = 8 bx - 1 .. 8 bx + 7 and
// o - 1 .. o along the remaining axis: their dual mass fluxes (and masses on
// the last sweep) are staged as [o - 1 + q][x - 8 bx + 1][position], with zero
// for cells outside the mesh (adding +0 to these sums changes no bit).
template <int D, bool FIRST, bool LAST, int K, int W>
struct NodeTileSize {
  static constexpr int NA = FIRST ? 5 : 9;                   // vh x3, x0[D], nm or U_dual x5
  static constexpr int NT = LAST ? K + 1 : K;                // cell tiles: dual mass flux per environment (+ mass)
  static constexpr int CT = 2 * (W + 1) * TileGeom<W>::cld;  // elements of one cell tile
  static constexpr size_t bytes = (size_t)(NA * TileGeom<W>::arr + NT * CT) * sizeof(double);
};

// One lane's line step of a node y/z sweep, from the staged tiles (each warp
// reads only its own tile row and the cell tiles, which no warp writes
// before the stores at the end of the body).
template <int D, bool FIRST, bool LAST, int K, typename R, int W, bool GL, bool SP>
__device__ __forceinline__ void nodes_t_line(const Dims& dm, const Scalars* __restrict__ S, const Phys& ph,
    int prev_inner, const double* __restrict__ x0, const double* __restrict__ xl, const double* __restrict__ vh,
    const double* __restrict__ Gd, int bx_, int by_, int bz_, R G[3], double* out, unsigned* oor) {
  using TS = NodeTileSize<D, FIRST, LAST, K, W>;
  constexpr int NA = TS::NA, CT = TS::CT;
  constexpr int CLd = TileGeom<W>::cld;               // row length of a cell tile
  constexpr int kTileArr = TileGeom<W>::arr, kTileLd = TileGeom<W>::ld;
  extern __shared__ double smem_dyn[];
  const double* tile = smem_dyn;                      // [NA][W][ld]
  const double* ctile = smem_dyn + NA * kTileArr;     // [NT][2][W + 1][cld]
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int i0 = bx_ * W, seg0 = by_ * kLineUpd - 2, o = bz_;
  const int nx = dm.nx, ny = dm.ny, N = (int)dm.N;
  const int nn = dm.ncd(D) + 1;                       // nodes along D
  auto node_id = [&](int i, int m) { return D == 1 ? i + (nx + 1) * (m + (ny + 1) * o) : i + (nx + 1) * (o + (ny + 1) * m); };
  const int m = seg0 + lane;
  const int i = i0 + w;
  const bool valid = i <= nx && m >= 0 && m < nn;
  const bool inner = i <= nx && m >= 1 && m <= nn - 2;
  const bool upd = valid && lane >= 2 && lane < 2 + kLineUpd;
  int idx[3];
  idx[0] = i; idx[D] = m; idx[3 - D] = o;               // D = 1: (i, m, o); D = 2: (i, o, m)
  const bool updated = node_updated(dm, D, prev_inner, idx);
  const bool grad_on = ph.ordre_projection > 1;
  const double* row = tile + w * kTileLd + lane;
  NodeIn in;
  in.vh[0] = row[0]; in.vh[1] = row[kTileArr]; in.vh[2] = row[2 * kTileArr]; in.x0d = row[3 * kTileArr];
  in.nm = FIRST ? row[4 * kTileArr] : 0.;
#pragma unroll
  for (int c = 0; c < 5; ++c) in.ud[c] = FIRST ? 0. : row[(4 + c) * kTileArr];
  // cells in front of the node along D have index m along D; transverse
  // (x - 1, x) = columns (w, w + 1) and (o - 1, o) = tile rows (0, 1)
  const double* cr = ctile + w * CLd + lane;
  constexpr int QS = (W + 1) * CLd;                   // stride between the two tile rows
  // DualPhaseRemap.cc:299-340 order: s1 over d1 = (D+1)%3, s2 over d2 = (D+2)%3,
  // environments innermost.  D = 1: s1 over z (q), s2 over x; D = 2: s1 over
  // x, s2 over y (q).  Tile offsets of the cells (q, dx): q * QS + dx * CLd.
  constexpr int o1 = D == 1 ? CLd : QS, o2 = D == 1 ? QS : CLd;
  double f = 0.;
#pragma unroll
  for (int e = 0; e < K; ++e) f += 0.25 * cr[e * CT];
#pragma unroll
  for (int e = 0; e < K; ++e) f += 0.25 * cr[e * CT + o1];
#pragma unroll
  for (int e = 0; e < K; ++e) f += 0.25 * cr[e * CT + o2];
#pragma unroll
  for (int e = 0; e < K; ++e) f += 0.25 * cr[e * CT + QS + CLd];
  in.ffm = (valid && m < nn - 1) ? f : 0.;
  in.msum = 0.;
  if (LAST) {
    const double* mr = cr + K * CT;
    const double a00 = mr[0], a01 = mr[CLd], a10 = mr[QS], a11 = mr[QS + CLd];   // cells at index m along D
    const unsigned full = 0xffffffffu;
    const double b00 = __shfl_up_sync(full, a00, 1), b01 = __shfl_up_sync(full, a01, 1),
                 b10 = __shfl_up_sync(full, a10, 1), b11 = __shfl_up_sync(full, a11, 1);   // index m - 1
    // increasing cell id: z outer, y, x inner
    double sm = 0.;
    if (D == 1) {   // (x, y=m-1|m, z=o-1|o): q = z
      sm += b00; sm += b01; sm += a00; sm += a01; sm += b10; sm += b11; sm += a10; sm += a11;
    } else {        // (x, y=o-1|o, z=m-1|m): q = y
      sm += b00; sm += b01; sm += b10; sm += b11; sm += a00; sm += a01; sm += a10; sm += a11;
    }
    in.msum = sm;
  }
  in.x2[0] = in.x2[1] = 0.;
  if (GL && valid && (lane == 1 || lane == 30)) {
    const int q = lane == 1 ? m - 2 : m + 2;           // the node two back (lane 1) or ahead (lane 30)
    if (q >= 0 && q < nn) {
      const int nq = node_id(i, q);
      in.x2[lane == 1 ? 0 : 1] = xl ? xl[D * N + nq] : x0[D * N + nq] + vh[D * N + nq] * S->dt;
    }
  }
  G[0] = G[1] = G[2] = R(0);
  const int n = valid ? node_id(i, m) : 0;
  if (valid && !(inner && grad_on)) { G[0] = (R)Gd[n]; G[1] = (R)Gd[N + n]; G[2] = (R)Gd[2 * N + n]; }
  node_line<D, FIRST, LAST, R, GL, SP>(ph, S->dt, valid, inner, updated, upd, in, G, out, xl != nullptr, m >= 2,
                                       m + 2 <= nn - 1, oor);
}

template <int D, bool FIRST, bool LAST, int K, typename R, int W, bool GL>
__device__ __noinline__ NodeLineOut nodes_t_line_exact(Dims dm, const Scalars* S, Phys ph, int prev_inner,
    const double* x0, const double* xl, const double* vh, const double* Gd, int bx_, int by_, int bz_) {
  NodeLineOut o;
  R G[3];
  nodes_t_line<D, FIRST, LAST, K, R, W, GL, false>(dm, S, ph, prev_inner, x0, xl, vh, Gd, bx_, by_, bz_, G, o.v,
                                                   nullptr);
  o.g[0] = (double)G[0]; o.g[1] = (double)G[1]; o.g[2] = (double)G[2];
  return o;
}

template <int D, bool FIRST, bool LAST, int K, typename R, int W = kLineWarps, bool GL = false>
__device__ __forceinline__ void k_cyc_sweep_nodes_t_body(Dims dm, const Scalars* __restrict__ S,
    Phys ph, int prev_inner, const double* __restrict__ x0, const double* __restrict__ xl, const double* __restrict__ vh,
    const double* __restrict__ nm_in, const double* __restrict__ udin, double* __restrict__ udout,
    const double* __restrict__ dpf, double* __restrict__ Gd, const double* __restrict__ mass,
    double* __restrict__ vout, double* __restrict__ nm_out, double* __restrict__ vnorm,
    int bx_, int by_, int bz_, double* __restrict__ ecn = nullptr) {
  using TS = NodeTileSize<D, FIRST, LAST, K, W>;
  constexpr int NA = TS::NA, CT = TS::CT;
  constexpr int CLd = TileGeom<W>::cld;               // row length of a cell tile
  constexpr int kTileArr = TileGeom<W>::arr, kTileLd = TileGeom<W>::ld;
  extern __shared__ double smem_dyn[];
  double* tile = smem_dyn;                            // [NA][W][ld]
  double* ctile = smem_dyn + NA * kTileArr;           // [NT][2][W + 1][cld]
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int i0 = bx_ * W, seg0 = by_ * kLineUpd - 2, o = bz_;
  const int nx = dm.nx, ny = dm.ny, nz = dm.nz, N = (int)dm.N;
  const int nn = dm.ncd(D) + 1, no = D == 1 ? nz : ny;   // cells along D; cells along the remaining axis
  auto node_id = [&](int i, int m) { return D == 1 ? i + (nx + 1) * (m + (ny + 1) * o) : i + (nx + 1) * (o + (ny + 1) * m); };
  const int sx = tid % W, sp = tid / W;
  const int si = i0 + sx, sm_ = seg0 + sp;
  const bool s_valid = si <= nx && sm_ >= 0 && sm_ < nn;
  const int sn = s_valid ? node_id(si, sm_) : 0;
  {
    double v[NA];
#pragma unroll
    for (int a = 0; a < NA; ++a) v[a] = 0.;
    if (s_valid) {
      v[0] = vh[sn]; v[1] = vh[N + sn]; v[2] = vh[2 * N + sn]; v[3] = xl ? xl[D * N + sn] : x0[D * N + sn];
      if (FIRST) v[4] = nm_in[sn];
      else {
#pragma unroll
        for (int c = 0; c < 5; ++c) v[4 + c] = udin[c * N + sn];
      }
    }
#pragma unroll
    for (int a = 0; a < NA; ++a) tile[a * kTileArr + sx * kTileLd + sp] = v[a];
    // cell tiles: element e = (q * 9 + xx) * 32 + p, loaded with xx fastest
    for (int e = tid; e < 2 * (W + 1) * 32; e += 32 * W) {
      const int xx = e % (W + 1), r = e / (W + 1);
      const int p = r & 31, q = r >> 5;
      const int ci = i0 - 1 + xx, cd = seg0 + p, co = o - 1 + q;
      const bool cv = ci >= 0 && ci < nx && cd >= 0 && cd < nn - 1 && co >= 0 && co < no;
      const int c = D == 1 ? ci + nx * (cd + ny * co) : ci + nx * (co + ny * cd);
      const int at = (q * (W + 1) + xx) * CLd + p;
#pragma unroll
      for (int q2 = 0; q2 < K; ++q2) ctile[q2 * CT + at] = cv ? dpf[q2 * (int)dm.C + c] : 0.;
      if (LAST) ctile[K * CT + at] = cv ? mass[c] : 0.;
    }
  }
  __syncthreads();
  R G[3];
  double out[LAST ? kNodeOutLast : kNodeOut];
  if constexpr (sizeof(R) == 8) {
    unsigned oor = 0u;
    nodes_t_line<D, FIRST, LAST, K, R, W, GL, true>(dm, S, ph, prev_inner, x0, xl, vh, Gd, bx_, by_, bz_, G, out, &oor);
    if (__any_sync(0xffffffffu, oor != 0u)) {
      const NodeLineOut o2 = nodes_t_line_exact<D, FIRST, LAST, K, R, W, GL>(dm, S, ph, prev_inner, x0, xl, vh, Gd,
                                                                             bx_, by_, bz_);
#pragma unroll
      for (int c = 0; c < (LAST ? kNodeOutLast : kNodeOut); ++c) out[c] = o2.v[c];
      G[0] = o2.g[0]; G[1] = o2.g[1]; G[2] = o2.g[2];
    }
  } else {
    nodes_t_line<D, FIRST, LAST, K, R, W, GL, false>(dm, S, ph, prev_inner, x0, xl, vh, Gd, bx_, by_, bz_, G, out,
                                                     nullptr);
  }
  const int m = seg0 + lane;
  const int i = i0 + w;
  const bool valid = i <= nx && m >= 0 && m < nn;
  const bool inner = i <= nx && m >= 1 && m <= nn - 2;
  const bool upd = valid && lane >= 2 && lane < 2 + kLineUpd;
  int idx[3];
  idx[0] = i; idx[D] = m; idx[3 - D] = o;               // D = 1: (i, m, o); D = 2: (i, o, m)
  const bool grad_on = ph.ordre_projection > 1;
  double* row = tile + w * kTileLd + lane;
  const int n = valid ? node_id(i, m) : 0;
  if (upd) {
    if (inner && grad_on && node_on_plane(dm, D, idx)) { Gd[n] = (double)G[0]; Gd[N + n] = (double)G[1]; Gd[2 * N + n] = (double)G[2]; }
    // each lane overwrites only the tile column it read itself
#pragma unroll
    for (int c = 0; c < (LAST ? kNodeOutLast : kNodeOut); ++c) row[c * kTileArr] = out[c];
  }
  __syncthreads();
  if (!(s_valid && sp >= 2 && sp < 2 + kLineUpd)) return;
  const double* r = tile + sx * kTileLd + sp;
  if (!LAST) {
#pragma unroll
    for (int c = 0; c < 5; ++c) udout[c * N + sn] = r[c * kTileArr];
  } else {
    vout[sn] = r[0]; vout[N + sn] = r[kTileArr]; vout[2 * N + sn] = r[2 * kTileArr];
    nm_out[sn] = r[3 * kTileArr]; vnorm[sn] = r[4 * kTileArr];
    if (ecn) ecn[sn] = r[5 * kTileArr];
  }
}

template <int D, bool FIRST, bool LAST, int K, typename R, int W, bool GL = false>
__global__ void __launch_bounds__(32 * W, TileGeom<W>::minb) k_cyc_sweep_nodes_t(Dims dm, const Scalars* __restrict__ S,
    Phys ph, int prev_inner, const double* __restrict__ x0, const double* __restrict__ xl, const double* __restrict__ vh,
    const double* __restrict__ nm_in, const double* __restrict__ udin, double* __restrict__ udout,
    const double* __restrict__ dpf, double* __restrict__ Gd, const double* __restrict__ mass,
    double* __restrict__ vout, double* __restrict__ nm_out, double* __restrict__ vnorm, double* __restrict__ ecn) {
  k_cyc_sweep_nodes_t_body<D, FIRST, LAST, K, R, W, GL>(dm, S, ph, prev_inner, x0, xl, vh, nm_in, udin, udout, dpf, Gd, mass, vout, nm_out, vnorm, blockIdx.x, blockIdx.y, blockIdx.z, ecn);
}

// ------------------------------------------------------------------------
// Host-side node sweep launchers.

// Dynamic shared memory above the default 48 KB needs an opt-in per kernel and device.
void smem_opt_in(const void* kernel, size_t bytes);

template <int D, bool FIRST, bool LAST, int K, typename R, int W, bool GL = false>
static void sweep_nodes_launch_w(const CycleArgs& a, int prev, const double* udin, double* udout, cudaStream_t s) {
  const Dims& dm = a.dm;
  const int nseg = (dm.ncd(D) + 1 + kLineUpd - 1) / kLineUpd;
  const dim3 g((dm.nx + 1 + W - 1) / W, nseg, (D == 1 ? dm.nz : dm.ny) + 1);
  const size_t smem = NodeTileSize<D, FIRST, LAST, K, W>::bytes;
  auto kern = k_cyc_sweep_nodes_t<D, FIRST, LAST, K, R, W, GL>;
  smem_opt_in((const void*)kern, smem);
  kern<<<g, 32 * W, smem, s>>>(dm, a.S, a.ph, prev, a.x0, a.xl, a.vh, a.nm, udin, udout, a.dpf, a.Gd, a.st.mass, a.v,
                               a.nm, a.vnorm, a.ecn);
}

template <int D, bool FIRST, bool LAST, int K, typename R>
static void sweep_nodes_launch(const CycleArgs& a, int prev, const double* udin, double* udout, cudaStream_t s) {
  const Dims& dm = a.dm;
  const int nseg = (dm.ncd(D) + 1 + kLineUpd - 1) / kLineUpd;
  const int T = 32 * kLineWarps;
  // the generalised limiters (FP64) have their own kernels
  const bool gl = sizeof(R) == 8 && a.ph.ordre_projection > 1 && a.ph.limiteur_id >= 3;
  if constexpr (D == 0) {
    const dim3 g(nseg, (dm.ny + 1 + kLineWarps - 1) / kLineWarps, dm.nz + 1);
    if (gl)
      k_cyc_sweep_nodes_x<FIRST, LAST, K, R, true><<<g, T, 0, s>>>(dm, a.S, a.ph, prev, a.x0, a.xl, a.vh, a.nm, udin,
                                                                udout, a.dpf, a.Gd, a.st.mass, a.v, a.nm, a.vnorm, a.ecn);
    else
      k_cyc_sweep_nodes_x<FIRST, LAST, K, R><<<g, T, 0, s>>>(dm, a.S, a.ph, prev, a.x0, a.xl, a.vh, a.nm, udin, udout,
                                                       a.dpf, a.Gd, a.st.mass, a.v, a.nm, a.vnorm, a.ecn);
  } else {
    if constexpr (sizeof(R) == 8) {
      if (gl) { sweep_nodes_launch_w<D, FIRST, LAST, K, R, kLineWarps, true>(a, prev, udin, udout, s); return; }
    }
    // lines per block of this sweep (the tuning; K > 1 meshes keep 8)
    const int w = K == 1 ? a.lines[BK_NODES_X + D] : kLineWarps;
    if (w == 32) sweep_nodes_launch_w<D, FIRST, LAST, K, R, 32>(a, prev, udin, udout, s);
    else if (w == 16) sweep_nodes_launch_w<D, FIRST, LAST, K, R, 16>(a, prev, udin, udout, s);
    else sweep_nodes_launch_w<D, FIRST, LAST, K, R, 8>(a, prev, udin, udout, s);
  }
}

// One node sweep along D of a mesh with K environments (dual mass fluxes in K planes).
template <int D, int K, typename R>
static void sweep_nodes_d(const CycleArgs& a, bool first, bool last, int prev, const double* udin, double* udout,
                          cudaStream_t s) {
  if (first) sweep_nodes_launch<D, true, false, K, R>(a, prev, udin, udout, s);
  else if (last) sweep_nodes_launch<D, false, true, K, R>(a, prev, udin, udout, s);
  else sweep_nodes_launch<D, false, false, K, R>(a, prev, udin, udout, s);
}

// R: evaluation precision of the sweep (double, or float in the mixed form).
template <int K, typename R = double>
static void sweep_nodes(const CycleArgs& a, int d, bool first, bool last, int prev, const double* udin,
                        double* udout, cudaStream_t s) {
  if (d == 0) sweep_nodes_d<0, K, R>(a, first, last, prev, udin, udout, s);
  else if (d == 1) sweep_nodes_d<1, K, R>(a, first, last, prev, udin, udout, s);
  else sweep_nodes_d<2, K, R>(a, first, last, prev, udin, udout, s);
}


}  // namespace mhy
