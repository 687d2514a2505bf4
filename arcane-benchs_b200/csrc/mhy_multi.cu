// mhy_multi.cu -- the cycle of a mesh with K = 2..4 environments (materials),
// each an ideal gas with its own adiabatic constant.
//
// Eleven launches per cycle: the Lagrange node kernel (shared with K = 1),
// k_cyc_lagrange_cells<K>, three directional sweeps of cells and of nodes,
// k_env_finalize_cells<K> between the last cell sweep and the last node sweep,
// and the dt reduction.
//   - Remap variables: the 3K+1 non-zero components of U
//     (V_k, V_k rho_k, V_k rho_k e_k for each environment, then V q) as planes
//     of C doubles (PrepareRemap.cc:318-330, 360-372); Phi = U / V on the first
//     sweep and U / sum_k V_k afterwards (PrepareRemap.cc:394-398,
//     RemapADIService.cc:962-970).  No component is constant here, so every
//     one gets gradients, limiters and fluxes.
//   - Dual mass flux: one plane per environment (the mass variables), summed
//     environment by environment by the node sweeps (DualPhaseRemap.cc:299-340).
//   - Environment membership changes (RemapADIFinal.cc:94-226) depend only on
//     the cell's own remapped U, so k_env_finalize_cells decides them cell by
//     cell on the device, with the remapVariables "moy" kernel
//     (RemapADIFinal.cc:406-644), the PerfectGas EOS per environment and the
//     mixed-cell pressure and sound speed (MahycoModule.cc:1836-1915) in the
//     same thread: no host round trip and no list rebuild.
// The operation order is the reference's throughout (the CPU oracle matches
// bit for bit).
#include <mutex>

#include "mhy_lagrange.cuh"
#include "mhy_line.cuh"

namespace mhy {

// The K-environment sweeps carry 3K+1 components per lane; two resident
// blocks (128 registers) per SM keep them from spilling.
constexpr int kEnvMinBlocks = 2;

template <int K>
struct CellInK {
  double U[3 * K + 1], xc[3];
  double db, df, u, A, n[3];   // low face of the cell along d (inner faces only)
  double ob, of;               // outward-normal component along d of the back and front faces
  double den;                  // divisor of Phi on the first sweep: the Lagrangian volume
  double h;                    // G limiters: the cell's width along d (RemapADIService.cc:225-258)
  double pf3[3 * K + 1];       // order 3: Phi of the low face from k_o3_faces_env (inner faces only)
  double pbP[3 * K + 1];       // pente-borne, first sweep: Phi of the cell (FaceData::pbphi)
  double pbq;                  // pente-borne: Phi of q, q at the start of the remap
  uint32_t est;                // first sweep with projection-pente-borne-mixte: the cell's FaceData::est
};

// Face values of a K-environment line at orders 1 and 2
// (RemapADIService.cc:91-271, 447-517, 658-720): Pf of this lane's low face
// and Pfn of its high face, from the lanes' Phi.  lim: this cell's limiter
// (-1 at order 1).  GL: the cell widths are at hand, and limiters 3..7 take
// the generalised form for uneven widths (RemapADIService.cc:319-437 ->
// UtilesRemap.cc:295-330), every component limited alike; at the ends of
// the line the back or front cell is the cell itself.
template <int K, typename R, bool GL, bool SP = false>
__device__ __forceinline__ void face_values_env(const Phys& ph, int lim, bool inner, bool infr, const CellInK<K>& in,
                                                const R P[3 * K + 1], R Pf[3 * K + 1], R Pfn[3 * K + 1],
                                                unsigned* oor = nullptr) {
  constexpr int NV = 3 * K + 1;
  const R order2 = (R)(ph.ordre_projection - 1);
  const unsigned full = 0xffffffffu;
  const double xpx = __shfl_up_sync(full, in.xc[0], 1), xpy = __shfl_up_sync(full, in.xc[1], 1),
               xpz = __shfl_up_sync(full, in.xc[2], 1);
  const double dx = inner ? dot(d3(in.xc[0], in.xc[1], in.xc[2]) - d3(xpx, xpy, xpz), d3(in.n[0], in.n[1], in.n[2]))
                          : 0.;
  const R dxR = (R)dx, rdx = inner ? Ar<R>::rcp(dxR) : R(0);
  R G[NV], Pp[NV];
  R h0 = R(0), hm = R(0), hp = R(0);
  if constexpr (GL) {
    const double hb = __shfl_up_sync(full, in.h, 1), hn = __shfl_down_sync(full, in.h, 1);
    h0 = (R)in.h; hm = (R)(inner ? hb : in.h); hp = (R)(infr ? hn : in.h);
  }
  unsigned fo = 0u;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    Pp[v] = __shfl_up_sync(full, P[v], 1);
    const R g = inner ? dv<R, SP>(P[v] - Pp[v], dxR, rdx, &fo) : R(0);
    const R gr = __shfl_down_sync(full, g, 1);
    if constexpr (GL) {
      const R Pn = __shfl_down_sync(full, P[v], 1);
      G[v] = lim < 3 ? limited_one<R>(lim, g, gr)
                     : flux_limiter_g<R>(lim, gr, g, P[v], infr ? Pn : P[v], inner ? Pp[v] : P[v], h0, hp, hm);
    } else {
      G[v] = limited_one<R>(lim, g, gr);
    }
  }
  // lane 0's back neighbour is itself (0 / 0): its gradient reaches no updated cell
  if constexpr (SP) { if ((threadIdx.x & 31) != 0) *oor |= fo; }
  const bool back = in.u * dx > 0.0;
  const R dot_xf = (R)(back ? in.db : in.df);
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const R Gp = __shfl_up_sync(full, G[v], 1);
    Pf[v] = inner ? (back ? (Pp[v] + order2 * dot_xf * Gp) : (P[v] + order2 * dot_xf * G[v])) : R(0);
    Pfn[v] = __shfl_down_sync(full, Pf[v], 1);
  }
}

// Mixed/pure indicator of a cell from its Phi (RemapADIService.cc:972-988):
// 255 when more than one environment has Phi_k > 0, else 1 + the last such
// environment (0: none), the coding of FaceData::est.
template <int K, typename R>
__device__ __forceinline__ uint32_t est_code(const R* P) {
  int n = 0, e = -1;
#pragma unroll
  for (int k = 0; k < K; ++k)
    if (P[k] > R(0)) { ++n; e = k; }
  return n > 1 ? 255u : (uint32_t)(e + 1);
}

// pente-borne fluxes of the 3K+1 components leaving a K-environment cell
// through one face (UtilesRemap.cc:406-627 computeFluxPP, :628-823
// computeFluxPPPure): the integral of each component's reconstruction, then
// the debar fix over the environments (the mass flux is left alone where the
// neighbourhood is pure).
template <int K>
__device__ __forceinline__ void pb_fluxes_env(const Phys& ph, int type, double ppv, int lim_y0, bool pure,
                                              const double* P, const double* Pn, const double* Pp, double h0,
                                              double hp, double hm, const double* G, double* F) {
  constexpr int NV = 3 * K + 1;
  const double thr = ph.threshold;
#pragma unroll
  for (int v = 0; v < NV; ++v) F[v] = pb_flux_var(type, lim_y0, thr, ppv, P[v], Pn[v], Pp[v], h0, hp, hm, G[v]);
  if (ph.pb_debar == 1) {
    double svol = 0.;
#pragma unroll
    for (int m = 0; m < K; ++m) svol += F[m];
    if (fabs(svol) > thr) {
#pragma unroll
      for (int m = 0; m < K; ++m) {
        if (!pure) F[K + m] = (F[K + m] / svol) * F[m];
        F[2 * K + m] = (F[2 * K + m] / svol) * F[K + m];
      }
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) F[v] = 0.;
    }
  } else if (ph.pb_debar == 2) {
#pragma unroll
    for (int m = 0; m < K; ++m) {
      if (!pure) F[K + m] = P[K + m] * F[m];
      F[2 * K + m] = P[2 * K + m] * F[K + m];
    }
  }
  if (ppv == 0.) {
#pragma unroll
    for (int v = 0; v < NV; ++v) F[v] = 0.;
  }
}

// One line step of the remap of a K-environment cell (RemapADIService.cc:91-271,
// 447-517, 658-720, 883-1040).  out = the 3K+1 updated components, then the
// K dual mass fluxes.  O3: the face values of order 3 (R:583-641), computed
// per face beforehand by k_o3_faces_env; no gradient is formed.  PB:
// projection-pente-borne (FP64): Phi of PrepareRemap.cc:201-212 (first
// sweep) or R:805-834, the general gradient (R:319-378) and the fluxes of
// pb_fluxes_env, face values from the fluxes leaving the two cells
// (R:380-431, 574-578) and fluxes o*A*Phi_f (R:770-774).  With
// projection-pente-borne-mixte the limiter of the gradient and of the
// reconstruction, and the debar fix, follow the cell's neighbourhood
// (R:364-375): pure when the cell and its back and front neighbours (the
// cell itself at the ends of the line) are pure cells of one environment.
template <int K, bool FIRST, typename R, bool GL = false, bool O3 = false, bool PB = false, bool SP = false>
__device__ __forceinline__ void cell_line_env(const Phys& ph, double dt, bool valid, bool inner, bool infr,
                                              bool upd, const CellInK<K>& in, double* out, unsigned* oor = nullptr) {
  constexpr int NV = 3 * K + 1;
  const unsigned full = 0xffffffffu;
  R Pf[NV], Pfn[NV];
  if constexpr (O3) {
    static_assert(sizeof(R) == 8, "order 3 is FP64");
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      Pf[v] = inner ? in.pf3[v] : 0.;
      Pfn[v] = __shfl_down_sync(full, Pf[v], 1);
    }
  } else {
    R P[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) P[v] = 0;
    if (valid) {
      if constexpr (PB) {
        if (FIRST) {
#pragma unroll
          for (int v = 0; v < NV; ++v) P[v] = in.pbP[v];
        } else {
          double sv = 0.;
#pragma unroll
          for (int k = 0; k < K; ++k) sv += in.U[k];
#pragma unroll
          for (int k = 0; k < K; ++k) {
            P[k] = in.U[k] / sv;
            P[K + k] = in.U[k] != 0. ? in.U[K + k] / in.U[k] : 0.;
            P[2 * K + k] = in.U[K + k] != 0. ? in.U[2 * K + k] / in.U[K + k] : 0.;
          }
          P[3 * K] = in.pbq;
        }
      } else {
        double den;
        if (FIRST) den = in.den;
        else {
          den = 0.;
#pragma unroll
          for (int k = 0; k < K; ++k) den += in.U[k];
        }
        const R dR = (R)den, r = Ar<R>::rcp(dR);
#pragma unroll
        for (int v = 0; v < NV; ++v) P[v] = dv<R, SP>((R)in.U[v], dR, r, oor);
      }
    }
    int lim = ph.ordre_projection > 1 ? ph.lim_cell : -1;
    bool pure = false;
    if (ph.pb_mixte) {
      const uint32_t code = FIRST ? in.est : est_code<K>(P);
      const uint32_t cb = __shfl_up_sync(full, code, 1), cf = __shfl_down_sync(full, code, 1);
      pure = code != 255u && code == (inner ? cb : code) && code == (infr ? cf : code);
      if (ph.ordre_projection > 1) lim = (ph.lim_pure == 1 && pure) ? ph.lim_pure : ph.limiteur_id;
    }
    if constexpr (PB) {
      static_assert(sizeof(R) == 8, "pente-borne is FP64");
      const double xpx = __shfl_up_sync(full, in.xc[0], 1), xpy = __shfl_up_sync(full, in.xc[1], 1),
                   xpz = __shfl_up_sync(full, in.xc[2], 1);
      const double dx =
          inner ? dot(d3(in.xc[0], in.xc[1], in.xc[2]) - d3(xpx, xpy, xpz), d3(in.n[0], in.n[1], in.n[2])) : 0.;
      const double rdx = inner ? 1.0 / dx : 0.;
      const double hb = __shfl_up_sync(full, in.h, 1), hn = __shfl_down_sync(full, in.h, 1);
      const double h0 = in.h, hm = inner ? hb : in.h, hp = infr ? hn : in.h;
      double Pne[NV], Ppe[NV], G[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const double Pp = __shfl_up_sync(full, P[v], 1), Pn = __shfl_down_sync(full, P[v], 1);
        Pne[v] = infr ? Pn : P[v]; Ppe[v] = inner ? Pp : P[v];
        const double g = inner ? qdiv(P[v] - Pp, dx, rdx) : 0.;
        const double gr = __shfl_down_sync(full, g, 1);
        G[v] = lim < 3 ? limited_one<double>(lim, g, gr)
                       : flux_limiter_g<double>(lim, gr, g, P[v], Pne[v], Ppe[v], h0, hp, hm);
      }
      const double un = __shfl_down_sync(full, in.u, 1);
      const double ob = in.ob * in.u, of = in.of * un;             // outward velocities of the two faces
      const int lim_y0 = pure ? ph.lim_pure : ph.limiteur_id;
      double ar[NV], av[NV];
      pb_fluxes_env<K>(ph, 0, 0.5 * (ob + fabs(ob)) * dt, lim_y0, pure, P, Pne, Ppe, h0, hp, hm, G, ar);
      pb_fluxes_env<K>(ph, 1, 0.5 * (of + fabs(of)) * dt, lim_y0, pure, P, Pne, Ppe, h0, hp, hm, G, av);
      // back face: what leaves the previous cell forwards minus what leaves this one backwards
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const double avp = __shfl_up_sync(full, av[v], 1);
        Pf[v] = inner ? avp - ar[v] : 0.;
        Pfn[v] = __shfl_down_sync(full, Pf[v], 1);
      }
    } else {
      face_values_env<K, R, GL, SP>(ph, lim, inner, infr, in, P, Pf, Pfn, oor);
    }
  }
  const double un = __shfl_down_sync(full, in.u, 1), An = __shfl_down_sync(full, in.A, 1);
  if (!upd) return;
  // flux sums in FP64 in every precision (each face flux is one rounded value)
  const double cb = inner ? (PB ? in.ob * in.A : in.ob * in.u * in.A * dt) : 0.;
  const double cf = infr ? (PB ? in.of * An : in.of * un * An * dt) : 0.;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double flux_face = 0., dp = 0.;
    if (inner) { const double fl = (double)((R)cb * Pf[v]); flux_face += fl; dp += 0.5 * fl * in.ob; }
    if (infr) { const double fl = (double)((R)cf * Pfn[v]); flux_face += fl; dp += 0.5 * fl * in.of; }
    out[v] = in.U[v] - flux_face;
    if (v >= K && v < 2 * K) out[NV + v - K] = dp;
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    if (out[K + k] < 0.) out[K + k] = 0.;
    if (out[2 * K + k] < 0.) out[2 * K + k] = 0.;
  }
}

// Inputs of a K-environment cell that its own index gives: the cell width
// (GL, PB), the pente-borne Phi and the first sweep's mixed/pure indicator.
template <int K, bool FIRST, bool GL, bool PB>
__device__ __forceinline__ void env_cell_extras(const Phys& ph, const FaceData& fd, int C, int c, int D,
                                                CellInK<K>& in) {
  if constexpr (GL || PB) in.h = fd.h[D * C + c];
  if constexpr (PB) {
    if (FIRST) {
#pragma unroll
      for (int v = 0; v < 3 * K + 1; ++v) in.pbP[v] = fd.pbphi[v * C + c];
    }
    in.pbq = fd.pbphi[3 * K * C + c];
  }
  if (FIRST && ph.pb_mixte) in.est = fd.est[c];
}

// K-environment cell sweep along x (lanes along the rows).
// One lane's inputs and line step of the K-environment x sweep; the body
// below runs it with speculative FP64 quotients and, in a warp where any
// lane's were out of range, recomputes the segment exactly out of line
// (env_x_line_exact reloads the inputs), then stores.
template <int K, bool FIRST, typename R, bool GL, bool O3, bool PB, bool SP>
__device__ __forceinline__ void env_x_line(const Dims& dm, const Scalars* __restrict__ S, const Phys& ph,
    const FaceData& fd, const double* __restrict__ n0, const double* __restrict__ xcs, const double* __restrict__ ofn,
    const double* __restrict__ Uin, const double* __restrict__ Vlag, int bx_, int by_, int bz_, double* out,
    unsigned* oor) {
  constexpr int NV = 3 * K + 1;
  const int lane = threadIdx.x & 31;
  const int j = by_ * kLineWarps + (threadIdx.x >> 5), k = bz_;
  const int nd = dm.nx, C = (int)dm.C, F = (int)dm.F;
  const int s = bx_ * kLineUpd - 2 + lane;
  const bool valid = s >= 0 && s < nd;
  const bool inner = s >= 1 && s <= nd - 1;
  const bool infr = s + 1 <= nd - 1;
  const bool upd = valid && lane >= 2 && lane < 2 + kLineUpd;
  const int c = valid ? s + dm.nx * (j + dm.ny * k) : 0;
  const int t = inner ? s + (dm.nx + 1) * (j + dm.ny * k) : 0;
  CellInK<K> in;
#pragma unroll
  for (int v = 0; v < NV; ++v) in.U[v] = 0.;
  in.xc[0] = in.xc[1] = in.xc[2] = 0.;
  in.db = in.df = in.u = in.A = 0.; in.n[0] = in.n[1] = in.n[2] = 0.; in.ob = in.of = 0.; in.den = 0.; in.h = 0.;
#pragma unroll
  for (int v = 0; v < NV; ++v) in.pbP[v] = 0.;
  in.pbq = 0.; in.est = 0u;
  if (valid) {
#pragma unroll
    for (int v = 0; v < NV; ++v) in.U[v] = Uin[v * C + c];
    in.xc[0] = xcs[c]; in.xc[1] = xcs[C + c]; in.xc[2] = xcs[2 * C + c];
    if (FIRST) in.den = Vlag[c];
    env_cell_extras<K, FIRST, GL, PB>(ph, fd, C, c, 0, in);
    if (PB) { in.ob = ofn[1 * C + c]; in.of = ofn[4 * C + c]; }   // every lane's two faces take part
  }
  if (inner) {
    in.db = fd.db[0][t]; in.df = fd.df[0][t]; in.u = fd.u[0][t]; in.A = fd.A[0][t];
    in.n[0] = n0[t]; in.n[1] = n0[F + t]; in.n[2] = n0[2 * F + t];
  }
  if constexpr (O3) {
    const int Fd = (int)dm.Fx;
#pragma unroll
    for (int v = 0; v < NV; ++v) in.pf3[v] = inner ? fd.phi3[v * Fd + t] : 0.;
  }
  if (upd) { in.ob = ofn[1 * C + c]; in.of = ofn[4 * C + c]; }
  cell_line_env<K, FIRST, R, GL, O3, PB, SP>(ph, S->dt, valid, inner, infr, upd, in, out, oor);
}

template <int K, bool FIRST, typename R, bool GL, bool O3, bool PB>
__device__ __noinline__ LineOut<4 * K + 1> env_x_line_exact(Dims dm, const Scalars* S, Phys ph, FaceData fd,
    const double* n0, const double* xcs, const double* ofn, const double* Uin, const double* Vlag, int bx_, int by_,
    int bz_) {
  LineOut<4 * K + 1> o;
  env_x_line<K, FIRST, R, GL, O3, PB, false>(dm, S, ph, fd, n0, xcs, ofn, Uin, Vlag, bx_, by_, bz_, o.v, nullptr);
  return o;
}

template <int K, bool FIRST, typename R, bool GL = false, bool O3 = false, bool PB = false>
__device__ __forceinline__ void env_sweep_cells_x_body(Dims dm,
    const Scalars* __restrict__ S, Phys ph, FaceData fd, const double* __restrict__ n0,
    const double* __restrict__ xcs, const double* __restrict__ ofn, const double* __restrict__ Uin,
    double* __restrict__ Uout, double* __restrict__ dpf, const double* __restrict__ Vlag, int bx_, int by_, int bz_) {
  constexpr int NV = 3 * K + 1;
  const int lane = threadIdx.x & 31;
  const int j = by_ * kLineWarps + (threadIdx.x >> 5), k = bz_;
  if (j >= dm.ny) return;                              // whole warp leaves together
  double out[NV + K];
  if constexpr (sizeof(R) == 8 && !PB && !O3) {
    unsigned oor = 0u;
    env_x_line<K, FIRST, R, GL, O3, PB, true>(dm, S, ph, fd, n0, xcs, ofn, Uin, Vlag, bx_, by_, bz_, out, &oor);
    if (__any_sync(0xffffffffu, oor != 0u)) {
      const auto o = env_x_line_exact<K, FIRST, R, GL, O3, PB>(dm, S, ph, fd, n0, xcs, ofn, Uin, Vlag, bx_, by_, bz_);
#pragma unroll
      for (int v = 0; v < NV + K; ++v) out[v] = o.v[v];
    }
  } else {
    env_x_line<K, FIRST, R, GL, O3, PB, false>(dm, S, ph, fd, n0, xcs, ofn, Uin, Vlag, bx_, by_, bz_, out, nullptr);
  }
  const int nd = dm.nx, C = (int)dm.C;
  const int s = bx_ * kLineUpd - 2 + lane;
  const bool upd = s >= 0 && s < nd && lane >= 2 && lane < 2 + kLineUpd;
  const int c = s + dm.nx * (j + dm.ny * k);
  if (!upd) return;
#pragma unroll
  for (int v = 0; v < NV; ++v) Uout[v * C + c] = out[v];
#pragma unroll
  for (int e = 0; e < K; ++e) dpf[e * C + c] = out[NV + e];
}

template <int K, bool FIRST, typename R, bool GL = false, bool O3 = false, bool PB = false>
__global__ void __launch_bounds__(32 * kLineWarps, kEnvMinBlocks) k_env_sweep_cells_x(Dims dm,
    const Scalars* __restrict__ S, Phys ph, FaceData fd, const double* __restrict__ n0,
    const double* __restrict__ xcs, const double* __restrict__ ofn, const double* __restrict__ Uin,
    double* __restrict__ Uout, double* __restrict__ dpf, const double* __restrict__ Vlag) {
  env_sweep_cells_x_body<K, FIRST, R, GL, O3, PB>(dm, S, ph, fd, n0, xcs, ofn, Uin, Uout, dpf, Vlag, blockIdx.x,
                                                 blockIdx.y, blockIdx.z);
}

// K-environment cell sweep along y (D = 1) or z (D = 2), staged through
// shared memory exactly as the single-environment one (dynamic shared
// memory: NA * kTileArr doubles).
template <int K, bool FIRST>
__host__ __device__ constexpr int env_cells_staged_arrays() { return 3 * K + 1 + 12 + (FIRST ? 1 : 0); }

// W: lines per block (8 or 16, the tuning; the register budget stays 128).
// One lane's line step of the K-environment y/z sweep, from the staged tile
// (each warp reads only its own tile row, which no other warp writes).
template <int K, int D, bool FIRST, typename R, int W, bool GL, bool O3, bool PB, bool SP>
__device__ __forceinline__ void env_t_line(const Dims& dm, const Scalars* __restrict__ S, const Phys& ph,
    const FaceData& fd, int bx_, int by_, int bz_, double* out, unsigned* oor) {
  constexpr int NV = 3 * K + 1;
  constexpr int AX = NV, AF = NV + 3, AN = NV + 7, AO = NV + 10, AD = NV + 12;   // array offsets
  constexpr int kTileArr = TileGeom<W>::arr, kTileLd = TileGeom<W>::ld;
  extern __shared__ double tile[];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int i0 = bx_ * W, seg0 = by_ * kLineUpd - 2, o = bz_;
  const int nd = dm.ncd(D), C = (int)dm.C;
  const int s = seg0 + lane;
  const bool line_ok = i0 + w < dm.nx;
  const bool valid = line_ok && s >= 0 && s < nd;
  const bool inner = line_ok && s >= 1 && s <= nd - 1;
  const bool infr = s + 1 <= nd - 1;
  const bool upd = valid && lane >= 2 && lane < 2 + kLineUpd;
  const double* row = tile + w * kTileLd + lane;
  CellInK<K> in;
#pragma unroll
  for (int v = 0; v < NV; ++v) in.U[v] = row[v * kTileArr];
  in.xc[0] = row[AX * kTileArr]; in.xc[1] = row[(AX + 1) * kTileArr]; in.xc[2] = row[(AX + 2) * kTileArr];
  in.db = row[AF * kTileArr]; in.df = row[(AF + 1) * kTileArr]; in.u = row[(AF + 2) * kTileArr];
  in.A = row[(AF + 3) * kTileArr];
  in.n[0] = row[AN * kTileArr]; in.n[1] = row[(AN + 1) * kTileArr]; in.n[2] = row[(AN + 2) * kTileArr];
  in.ob = row[AO * kTileArr]; in.of = row[(AO + 1) * kTileArr];
  in.den = FIRST ? row[AD * kTileArr] : 0.;
  in.h = 0.; in.pbq = 0.; in.est = 0u;
#pragma unroll
  for (int v = 0; v < NV; ++v) in.pbP[v] = 0.;
  if (valid) {                                         // the cell's own extras: read directly
    const int ci = i0 + w;
    env_cell_extras<K, FIRST, GL, PB>(ph, fd, C, D == 1 ? ci + dm.nx * (s + dm.ny * o) : ci + dm.nx * (o + dm.ny * s),
                                      D, in);
  }
  if constexpr (O3) {
    // face values in the line layout of k_o3_faces_env: position along D
    // fastest, so the lanes' reads are contiguous
    const int Fd = (int)(D == 1 ? dm.Fy : dm.F - dm.Fx - dm.Fy);
    const int q = s + (nd + 1) * (i0 + w + dm.nx * o);
#pragma unroll
    for (int v = 0; v < NV; ++v) in.pf3[v] = inner ? fd.phi3[v * Fd + q] : 0.;
  }
  cell_line_env<K, FIRST, R, GL, O3, PB, SP>(ph, S->dt, valid, inner, infr, upd, in, out, oor);
}

template <int K, int D, bool FIRST, typename R, int W, bool GL, bool O3, bool PB>
__device__ __noinline__ LineOut<4 * K + 1> env_t_line_exact(Dims dm, const Scalars* S, Phys ph, FaceData fd, int bx_,
                                                            int by_, int bz_) {
  LineOut<4 * K + 1> o;
  env_t_line<K, D, FIRST, R, W, GL, O3, PB, false>(dm, S, ph, fd, bx_, by_, bz_, o.v, nullptr);
  return o;
}

template <int K, int D, bool FIRST, typename R, int W = kLineWarps, bool GL = false, bool O3 = false, bool PB = false>
__device__ __forceinline__ void env_sweep_cells_t_body(Dims dm,
    const Scalars* __restrict__ S, Phys ph, FaceData fd, const double* __restrict__ n0,
    const double* __restrict__ xcs, const double* __restrict__ ofn, const double* __restrict__ Uin,
    double* __restrict__ Uout, double* __restrict__ dpf, const double* __restrict__ Vlag, int bx_, int by_, int bz_) {
  constexpr int NV = 3 * K + 1;
  constexpr int NA = env_cells_staged_arrays<K, FIRST>();
  constexpr int AX = NV, AF = NV + 3, AN = NV + 7, AO = NV + 10, AD = NV + 12;   // array offsets
  constexpr int kTileArr = TileGeom<W>::arr, kTileLd = TileGeom<W>::ld;
  extern __shared__ double tile[];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int i0 = bx_ * W, seg0 = by_ * kLineUpd - 2, o = bz_;
  const int nd = dm.ncd(D), C = (int)dm.C, F = (int)dm.F;
  const int foff = D == 1 ? (int)dm.Fx : (int)(dm.Fx + dm.Fy);
  const int lb = D == 1 ? 2 : 0, lf = D == 1 ? 5 : 3;
  const int sx = tid % W, sp = tid / W;
  const int si = i0 + sx, ss = seg0 + sp;
  const bool s_valid = si < dm.nx && ss >= 0 && ss < nd;
  const int sc = D == 1 ? si + dm.nx * (ss + dm.ny * o) : si + dm.nx * (o + dm.ny * ss);
  {
    const bool s_inner = si < dm.nx && ss >= 1 && ss <= nd - 1;
    const int st_ = D == 1 ? si + dm.nx * (ss + (dm.ny + 1) * o) : sc;
    double* wr = tile + sx * kTileLd + sp;
#pragma unroll
    for (int v = 0; v < NV; ++v) wr[v * kTileArr] = s_valid ? Uin[v * C + sc] : 0.;
    wr[(AX + 0) * kTileArr] = s_valid ? xcs[sc] : 0.;
    wr[(AX + 1) * kTileArr] = s_valid ? xcs[C + sc] : 0.;
    wr[(AX + 2) * kTileArr] = s_valid ? xcs[2 * C + sc] : 0.;
    wr[(AF + 0) * kTileArr] = s_inner ? fd.db[D][st_] : 0.;
    wr[(AF + 1) * kTileArr] = s_inner ? fd.df[D][st_] : 0.;
    wr[(AF + 2) * kTileArr] = s_inner ? fd.u[D][st_] : 0.;
    wr[(AF + 3) * kTileArr] = s_inner ? fd.A[D][st_] : 0.;
    const int f = foff + st_;
    wr[(AN + 0) * kTileArr] = s_inner ? n0[f] : 0.;
    wr[(AN + 1) * kTileArr] = s_inner ? n0[F + f] : 0.;
    wr[(AN + 2) * kTileArr] = s_inner ? n0[2 * F + f] : 0.;
    wr[(AO + 0) * kTileArr] = s_valid ? ofn[lb * C + sc] : 0.;
    wr[(AO + 1) * kTileArr] = s_valid ? ofn[lf * C + sc] : 0.;
    if (FIRST) wr[AD * kTileArr] = s_valid ? Vlag[sc] : 0.;
  }
  __syncthreads();
  constexpr int NO = NV + K;
  static_assert(NO <= NA, "outputs reuse the staged rows");
  double out[NO];
  if constexpr (sizeof(R) == 8 && !PB && !O3) {
    unsigned oor = 0u;
    env_t_line<K, D, FIRST, R, W, GL, O3, PB, true>(dm, S, ph, fd, bx_, by_, bz_, out, &oor);
    if (__any_sync(0xffffffffu, oor != 0u)) {
      const auto o2 = env_t_line_exact<K, D, FIRST, R, W, GL, O3, PB>(dm, S, ph, fd, bx_, by_, bz_);
#pragma unroll
      for (int v = 0; v < NO; ++v) out[v] = o2.v[v];
    }
  } else {
    env_t_line<K, D, FIRST, R, W, GL, O3, PB, false>(dm, S, ph, fd, bx_, by_, bz_, out, nullptr);
  }
  const int s = seg0 + lane;
  const bool upd = i0 + w < dm.nx && s >= 0 && s < nd && lane >= 2 && lane < 2 + kLineUpd;
  double* row = tile + w * kTileLd + lane;
  if (upd) {
#pragma unroll
    for (int a = 0; a < NO; ++a) row[a * kTileArr] = out[a];
  }
  __syncthreads();
  if (!(s_valid && sp >= 2 && sp < 2 + kLineUpd)) return;
  const double* r = tile + sx * kTileLd + sp;
#pragma unroll
  for (int v = 0; v < NV; ++v) Uout[v * C + sc] = r[v * kTileArr];
#pragma unroll
  for (int e = 0; e < K; ++e) dpf[e * C + sc] = r[(NV + e) * kTileArr];
}

template <int K, int D, bool FIRST, typename R, int W = kLineWarps, bool GL = false, bool O3 = false, bool PB = false>
__global__ void __launch_bounds__(32 * W, kEnvMinBlocks * kLineWarps / W) k_env_sweep_cells_t(Dims dm,
    const Scalars* __restrict__ S, Phys ph, FaceData fd, const double* __restrict__ n0,
    const double* __restrict__ xcs, const double* __restrict__ ofn, const double* __restrict__ Uin,
    double* __restrict__ Uout, double* __restrict__ dpf, const double* __restrict__ Vlag) {
  env_sweep_cells_t_body<K, D, FIRST, R, W, GL, O3, PB>(dm, S, ph, fd, n0, xcs, ofn, Uin, Uout, dpf, Vlag, blockIdx.x,
                                                       blockIdx.y, blockIdx.z);
}

// Order-3 face values of direction D for K environments
// (RemapADIService.cc:583-641, Remap-ordre-3.cc:7-131), one thread per face.
// Phi of the six cells around an inner face (clamped at the ends of the
// line) as the sweeps form it (U over the Lagrangian volume on the first
// sweep, over the sum of the environment volumes afterwards), o3_flux per
// component; then, unless the two cells are pure cells of one environment,
// each environment's density and energy face values are rescaled by the
// upwind cell's ratios (R:623-641).  A cell is mixed when more than one
// environment has Phi_k > 0, else pure in the last such environment
// (R:972-988 after every sweep, RemapADIFinal.cc:495-507 after the remap):
// within a remap that is a function of the Phi the sweep starts from; the
// first sweep reads the indicator the previous remap left (FaceData::est;
// before the run's first remap both indicators are zero, every face pure).
// Faces are written in line order: the position along D fastest, then x,
// then the remaining axis (for D = 0 the usual face order).
template <int D, int K, bool FIRST>
__device__ __forceinline__ void o3_faces_env_item(const Dims& dm, const Scalars* __restrict__ S,
    const double* __restrict__ Uin, const FaceData& fd, const double* __restrict__ Vlag, long long t) {
  constexpr int NV = 3 * K + 1;
  const long long Fd = dm.nfd(D);
  if (t >= Fd) return;
  const int n = dm.ncd(D);
  const int id = (int)(t % (n + 1));
  const long long line = t / (n + 1);
  if (id <= 0 || id >= n) return;                     // boundary faces carry no flux
  int i, j, k;
  if (D == 0) { i = id; j = (int)(line % dm.ny); k = (int)(line / dm.ny); }
  else if (D == 1) { i = (int)(line % dm.nx); j = id; k = (int)(line / dm.nx); }
  else { i = (int)(line % dm.nx); j = (int)(line / dm.nx); k = id; }
  int pos[6];
  pos[2] = id - 1; pos[1] = pos[2] > 0 ? pos[2] - 1 : pos[2]; pos[0] = pos[1] > 0 ? pos[1] - 1 : pos[1];
  pos[3] = id; pos[4] = pos[3] + 1 < n ? pos[3] + 1 : pos[3]; pos[5] = pos[4] + 1 < n ? pos[4] + 1 : pos[4];
  const long long C = dm.C;
  long long cc[6];
  double den[6], rden[6], h[6];
#pragma unroll
  for (int a = 0; a < 6; ++a) {
    cc[a] = D == 0 ? dm.cid(pos[a], j, k) : (D == 1 ? dm.cid(i, pos[a], k) : dm.cid(i, j, pos[a]));
    if (FIRST) den[a] = Vlag[cc[a]];
    else {
      double sv = 0.;
#pragma unroll
      for (int e = 0; e < K; ++e) sv += Uin[e * C + cc[a]];
      den[a] = sv;
    }
    rden[a] = 1.0 / den[a];
    h[a] = fd.h[D * C + cc[a]];
  }
  const long long tf = dm.fid(D, i, j, k) - (D == 0 ? 0 : (D == 1 ? dm.Fx : dm.Fx + dm.Fy));
  const double vdt = fd.u[D][tf] * S->dt;
  double pf[NV];
  double pb[NV], pn[NV];                              // Phi of the two cells of the face
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double y[6];
#pragma unroll
    for (int a = 0; a < 6; ++a) y[a] = qdiv(Uin[v * C + cc[a]], den[a], rden[a]);
    pb[v] = y[2]; pn[v] = y[3];
    pf[v] = o3_flux(y, h, vdt);
  }
  const uint32_t codeb = FIRST ? fd.est[cc[2]] : est_code<K>(pb);
  const uint32_t codef = FIRST ? fd.est[cc[3]] : est_code<K>(pn);
  const bool pure = codeb != 255u && codeb == codef;
  if (!pure) {
#pragma unroll
    for (int e = 0; e < K; ++e) {
      if (vdt > 0. && pb[e] != 0. && pb[K + e] != 0.) {
        pf[K + e] = (pb[K + e] / pb[e]) * pf[e];
        pf[2 * K + e] = (pb[2 * K + e] / pb[K + e]) * pf[K + e];
      } else if (vdt < 0. && pn[e] != 0. && pn[K + e] != 0.) {
        pf[K + e] = (pn[K + e] / pn[e]) * pf[e];
        pf[2 * K + e] = (pn[2 * K + e] / pn[K + e]) * pf[K + e];
      }
    }
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) fd.phi3[v * Fd + t] = pf[v];
}

template <int D, int K, bool FIRST>
__global__ void __launch_bounds__(128) k_o3_faces_env(Dims dm, const Scalars* __restrict__ S,
    const double* __restrict__ Uin, FaceData fd, const double* __restrict__ Vlag) {
  o3_faces_env_item<D, K, FIRST>(dm, S, Uin, fd, Vlag, blockIdx.x * (long long)blockDim.x + threadIdx.x);
}

// The same over the face work table of D (instance, chunk of 128 faces), the
// sweep's input U[it & 1].
template <int D, int K, bool FIRST>
__global__ void __launch_bounds__(128) k_bat_o3_faces_env(const CycleArgs* __restrict__ A, const int4* __restrict__ W,
                                                          int nw, int it) {
  for (int w = blockIdx.x; w < nw; w += gridDim.x) {
    const int4 t = W[w];
    const CycleArgs& a = A[t.x];
    o3_faces_env_item<D, K, FIRST>(a.dm, a.S, a.U[it & 1], a.fd, a.Vlag, (long long)t.y * 128 + threadIdx.x);
  }
}

// ---- end of the remap, per cell ----------------------------------------
// Environment add/remove (RemapADIFinal.cc:94-226, decided from the
// membership before the update), the "moy" kernel (RemapADIFinal.cc:406-644),
// PerfectGas EOS per environment (PerfectGasEOSService.cc:72-136) and the
// mixed-cell averages (MahycoModule.cc:1836-1915).  When a cell changes
// membership the values of the environments involved move between the global
// and the partial slots as Arcane's material modifier moves them; of those
// only the mass fraction can outlive this kernel (it is kept when the cell's
// mass is exactly zero), so only it is moved.
// fd.est: the cell's mixed/pure indicator of RemapADIFinal.cc:495-507.
// fd.pbphi (pente-borne): the Phi of this last sweep for every environment
// (RemapADIService.cc:805-834); the next Lagrange step overwrites the cell's
// environments, and the others keep these values into the next remap.
template <int K>
__device__ __forceinline__ void env_finalize_cell(const Dims& dm, Scalars* __restrict__ S, const Phys& ph,
                                                  const EnvState& env, const double* __restrict__ U,
                                                  const CellState& st, const FaceData& fd, int c) {
  constexpr int NV = 3 * K + 1;
  const int C = (int)dm.C;
  double u[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) u[v] = U[v * C + c];
  if (fd.pbphi) {
    double sv = 0.;
#pragma unroll
    for (int k = 0; k < K; ++k) sv += u[k];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      fd.pbphi[k * C + c] = u[k] / sv;
      fd.pbphi[(K + k) * C + c] = u[k] != 0. ? u[K + k] / u[k] : 0.;
      fd.pbphi[(2 * K + k) * C + c] = u[K + k] != 0. ? u[2 * K + k] / u[K + k] : 0.;
    }
  }
  const double vol = st.Ve[c];
  const double thr = ph.threshold;
  uint32_t mask = env.mask[c];
  // membership changes (RemapADIFinal.cc:94-148)
  uint32_t nmask = mask;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const double fv = u[k] / vol;
    const bool in_env = mask >> k & 1;
    if (fv < thr && in_env) nmask &= ~(1u << k);
    else if (fv > thr && !in_env) {
      double volt = 0.;
#pragma unroll
      for (int kk = 0; kk < K; ++kk) volt += u[kk];
      const double f2 = u[k] / volt;
      if (f2 > thr && u[K + k] != 0.) nmask |= 1u << k;
    }
  }
  if (nmask != mask) {
    const bool was_pure = __popc(mask) == 1, now_pure = __popc(nmask) == 1;
    if (was_pure && !now_pure) {
      const int oe = __ffs(mask) - 1;
#pragma unroll
      for (int k = 0; k < K; ++k) env.x[k * C + c] = (k == oe && (nmask >> oe & 1)) ? env.xg[c] : 0.;
    } else if (!was_pure && now_pure) {
      env.xg[c] = env.x[(__ffs(nmask) - 1) * C + c];
    } else if (!now_pure) {
#pragma unroll
      for (int k = 0; k < K; ++k)
        if ((nmask >> k & 1) && !(mask >> k & 1)) env.x[k * C + c] = 0.;
    }
    mask = nmask;
    env.mask[c] = nmask;
  }
  const bool pure = __popc(mask) == 1;
  const int ke = pure ? __ffs(mask) - 1 : -1;
  // "moy" kernel
  double volt = 0., masset = 0.;
#pragma unroll
  for (int k = 0; k < K; ++k) { volt += u[k]; masset += u[K + k]; }
  const double unsurvolt = 1. / volt;
  const double unsurvol = 1. / vol;
  double f[K], x[K], r[K], e[K], q[K], m[K];
  double somme_frac = 0.;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    f[k] = x[k] = r[k] = e[k] = q[k] = m[k] = 0.;
    if (!(mask >> k & 1)) continue;
    double fvol = u[k] * unsurvolt;
    if (fvol < thr) fvol = 0.;
    f[k] = fvol;
    somme_frac += fvol;
  }
  const double unsursomme_frac = 1. / somme_frac;
  int matcell = 0, imatpure = -1;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    if (!(mask >> k & 1)) continue;
    const double fvol = f[k] * unsursomme_frac;
    if (fvol > 0.) { matcell++; imatpure = k; }
    f[k] = fvol;
  }
  const bool est_mixte = matcell > 1;
  if (fd.est) fd.est[c] = est_mixte ? 255u : (uint32_t)(imatpure + 1);
#pragma unroll
  for (int k = 0; k < K; ++k)
    if (mask >> k & 1) x[k] = pure ? env.xg[c] : env.x[k * C + c];
  if (masset != 0.) {
    const double unsurmasset = 1. / masset;
    double fmasset = 0.;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (!(mask >> k & 1)) continue;
      double mf = u[K + k] * unsurmasset;
      if (f[k] < thr) mf = 0.;
      fmasset += mf;
      x[k] = mf;
    }
    if (fmasset != 0.) {
      const double unsurfmasset = 1. / fmasset;
#pragma unroll
      for (int k = 0; k < K; ++k)
        if (mask >> k & 1) x[k] = x[k] * unsurfmasset;
    }
  } else {
    atomicOr(&S->status, MHY_STATUS_ZERO_MASS);
  }
  double density_nplus1 = 0.;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    if (!(mask >> k & 1)) continue;
    double de = 0.;
    if (f[k] > thr) {
      const double vn = u[k] * vol * unsurvolt;
      de = u[K + k] / vn;
    }
    r[k] = de;
    density_nplus1 += f[k] * de;
  }
  const double cell_mass = vol * density_nplus1;
  double energie_nplus1 = 0., pseudo_nplus1 = 0.;
  const double pv = u[3 * K] * unsurvol;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    if (!(mask >> k & 1)) continue;
    double ee = 0.;
    if (f[k] > thr && u[K + k] != 0.) ee = u[2 * K + k] / u[K + k];
    e[k] = ee;
    energie_nplus1 += x[k] * ee;
    m[k] = x[k] * cell_mass;
    q[k] = pv;
    pseudo_nplus1 += f[k] * pv;
  }
  // A pure cell's environment value is its global value, so the global
  // energy and pseudo-viscosity written after the loop are its values too.
  if (pure) { e[ke] = energie_nplus1; q[ke] = pseudo_nplus1; }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    if (!(mask >> k & 1)) continue;
    if (r[k] < 0. || e[k] < 0.) { e[k] = 0.; r[k] = 0.; f[k] = 0.; x[k] = 0.; }
  }
  // conservation-energie-totale: the energies change once the node terms are
  // known (k_env_cons_ec, after the last node sweep), which then applies the EOS
  const bool eos_now = !ph.cons_ec;
  double pk[K], ck[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    pk[k] = ck[k] = 0.;
    if (!(mask >> k & 1) || !eos_now) continue;
    eos_pc(env.eos[k], env.gamma[k], env.pinf[k], r[k], e[k], pk[k], ck[k]);
  }
  if (pure) {
    st.rho[c] = r[ke]; st.e[c] = e[ke]; st.q[c] = q[ke]; st.mass[c] = m[ke];
    if (eos_now) { st.p[c] = pk[ke]; st.cs[c] = ck[ke]; }
    env.fg[c] = f[ke]; env.xg[c] = x[ke];
  } else {
    double pm = 0., cm = 1.e-20;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (!(mask >> k & 1)) continue;
      const int o = k * C + c;
      env.f[o] = f[k]; env.x[o] = x[k]; env.rho[o] = r[k]; env.e[o] = e[k]; env.q[o] = q[k]; env.m[o] = m[k];
      env.p[o] = pk[k]; env.cs[o] = ck[k];
      pm += f[k] * pk[k];
      cm = amax(ck[k], cm);
    }
    if (est_mixte) st.rho[c] = density_nplus1;
    st.e[c] = energie_nplus1; st.q[c] = pseudo_nplus1; st.mass[c] = cell_mass;
    if (eos_now) { st.p[c] = pm; st.cs[c] = cm; }
  }
}

template <int K>
__global__ void __launch_bounds__(256) k_env_finalize_cells(Dims dm, Scalars* __restrict__ S, Phys ph,
                                                            EnvState env, const double* __restrict__ U,
                                                            CellState st, FaceData fd) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= (int)dm.C) return;
  env_finalize_cell<K>(dm, S, ph, env, U, st, fd, c);
}

// conservation-energie-totale with K environments (RemapADIFinal.cc:751-773,
// then PerfectGasEOSService.cc:72-136 and MahycoModule.cc:1836-1915): the
// kinetic energy the dual remap lost, summed over the cell's 8 nodes in
// cell-node order (each node's 0.25 (U_dual[4]/U_dual[3] - 0.5 |v|^2) from
// the last node sweep), floored at 0, added as x_k delta to every
// environment's specific energy and as delta to a mixed cell's mean; then the
// EOS of every environment and the mixed-cell pressure and sound speed.  A
// pure cell's environment values are its global values.
template <int K>
__device__ __forceinline__ void env_cons_ec_cell(const Dims& dm, const EnvState& env, const CellState& st,
                                                 const double* __restrict__ ecn, int i, int j, int k) {
  const int C = (int)dm.C;
  const int c = (int)dm.cid(i, j, k);
  double delta_ec = 0.;
#pragma unroll
  for (int a = 0; a < 8; ++a)
    delta_ec += ecn[dm.nid(i + kCellNodeOff[a][0], j + kCellNodeOff[a][1], k + kCellNodeOff[a][2])];
  delta_ec = smax(0., delta_ec);
  const uint32_t mask = env.mask[c];
  if (__popc(mask) == 1) {
    const int ke = __ffs(mask) - 1;
    const double en = st.e[c] + env.xg[c] * delta_ec;
    double pr, cc;
    eos_pc(env.eos[ke], env.gamma[ke], env.pinf[ke], st.rho[c], en, pr, cc);
    st.e[c] = en; st.p[c] = pr; st.cs[c] = cc;
    return;
  }
  double pm = 0., cm = 1.e-20;
#pragma unroll
  for (int kk = 0; kk < K; ++kk) {
    if (!(mask >> kk & 1)) continue;
    const int o = kk * C + c;
    const double ek = env.e[o] + env.x[o] * delta_ec;
    double pr, cc;
    eos_pc(env.eos[kk], env.gamma[kk], env.pinf[kk], env.rho[o], ek, pr, cc);
    env.e[o] = ek; env.p[o] = pr; env.cs[o] = cc;
    pm += env.f[o] * pr;
    cm = amax(cc, cm);
  }
  st.e[c] += delta_ec;
  st.p[c] = pm; st.cs[c] = cm;
}

template <int K>
__global__ void __launch_bounds__(128) k_env_cons_ec(Dims dm, Phys ph, EnvState env, CellState st,
                                                     const double* __restrict__ ecn, int linear) {
  int i, j, k;
  if (!block_item(dm.nx, dm.ny, dm.nz, blockIdx.x, linear ? -1 : (int)blockIdx.y, blockIdx.z, i, j, k)) return;
  env_cons_ec_cell<K>(dm, env, st, ecn, i, j, k);
}

void launch_cons_ec_env(const CycleArgs& a, cudaStream_t s) {
  int linear;
  const dim3 nbc = cell_grid(a.dm, linear);
  if (a.K == 2) k_env_cons_ec<2><<<nbc, 128, 0, s>>>(a.dm, a.ph, a.env, a.st, a.ecn, linear);
  else if (a.K == 3) k_env_cons_ec<3><<<nbc, 128, 0, s>>>(a.dm, a.ph, a.env, a.st, a.ecn, linear);
  else k_env_cons_ec<4><<<nbc, 128, 0, s>>>(a.dm, a.ph, a.env, a.st, a.ecn, linear);
}

// Initial thermodynamic state of a K-environment mesh, after the initial
// geometry: initEOS per environment (PerfectGas E:20-32 or StiffenedGas), the mixed-cell
// energy and sound speed (MahycoModule.cc:116-127) and ComputeCellMass
// (MahycoModule.cc:199-225).  Fractions, partial densities and pressures,
// mass fractions and the global density and pressure come from the host.
template <int K>
__global__ void k_env_init_state(Dims dm, EnvState env, CellState st) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int C = (int)dm.C;
  if (c >= C) return;
  const uint32_t mask = env.mask[c];
  const double V = st.Ve[c];
  st.q[c] = 0.;
  if (__popc(mask) == 1) {
    const int ke = __ffs(mask) - 1;
    double ec, cc;
    eos_init(env.eos[ke], env.gamma[ke], env.pinf[ke], st.rho[c], st.p[c], ec, cc);
    st.e[c] = ec;
    st.cs[c] = cc;
    const double r = st.rho[c];
    st.mass[c] = r * V;
    env.fg[c] = 1.; env.xg[c] = 1.;
    return;
  }
  double eg = 0., cg = 0.;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    if (!(mask >> k & 1)) continue;
    const int o = k * C + c;
    double ek, ck;
    eos_init(env.eos[k], env.gamma[k], env.pinf[k], env.rho[o], env.p[o], ek, ck);
    env.e[o] = ek; env.cs[o] = ck; env.q[o] = 0.;
    eg += ek * env.x[o];
    cg = smax(ck, cg);
  }
  st.e[c] = eg;
  st.cs[c] = cg;
  const double mg = st.rho[c] * V;
  st.mass[c] = mg;
#pragma unroll
  for (int k = 0; k < K; ++k)
    if (mask >> k & 1) env.m[k * C + c] = env.x[k * C + c] * mg;
  env.fg[c] = 1.; env.xg[c] = 1.;
}

// ------------------------------------------------------------------------
// Host-side launchers.
// the generalised limiters (FP64): the cell sweeps' GL kernels (with
// projection-pente-borne-mixte some cells may take the pure limiter instead)
static bool env_gl(const CycleArgs& a) { return a.ph.ordre_projection > 1 && a.ph.limiteur_id >= 3; }
// projection-pente-borne (FP64): the PB kernels, which read the cell widths themselves
static bool env_pb(const CycleArgs& a) { return a.ph.pb != 0; }

// order 3 (FP64): the sweeps read the face values of k_o3_faces_env
static bool env_o3(const CycleArgs& a) { return a.ph.ordre_projection == 3; }

template <int K, int D, bool FIRST, typename R, int W, bool GL = false, bool O3 = false, bool PB = false>
static void env_cells_staged_w(const CycleArgs& a, const double* Uin, double* Uout, cudaStream_t s) {
  const Dims& dm = a.dm;
  const int nseg = (dm.ncd(D) + kLineUpd - 1) / kLineUpd;
  const dim3 g((dm.nx + W - 1) / W, nseg, D == 1 ? dm.nz : dm.ny);
  const size_t smem = (size_t)env_cells_staged_arrays<K, FIRST>() * TileGeom<W>::arr * sizeof(double);
  auto kern = k_env_sweep_cells_t<K, D, FIRST, R, W, GL, O3, PB>;
  smem_opt_in((const void*)kern, smem);
  kern<<<g, 32 * W, smem, s>>>(dm, a.S, a.ph, a.fd, a.n0, a.xc, a.ofn, Uin, Uout, a.dpf, a.Vlag);
}

// lines per block of this sweep: the tuning's (8 or 16)
template <int K, int D, bool FIRST, typename R>
static void env_cells_staged(const CycleArgs& a, const double* Uin, double* Uout, cudaStream_t s) {
  if constexpr (sizeof(R) == 8) {
    if (env_pb(a)) { env_cells_staged_w<K, D, FIRST, R, kLineWarps, false, false, true>(a, Uin, Uout, s); return; }
    if (env_o3(a)) { env_cells_staged_w<K, D, FIRST, R, kLineWarps, false, true>(a, Uin, Uout, s); return; }
    if (env_gl(a)) { env_cells_staged_w<K, D, FIRST, R, kLineWarps, true>(a, Uin, Uout, s); return; }
  }
  if (a.lines[BK_CELLS_X + D] == 16) env_cells_staged_w<K, D, FIRST, R, 16>(a, Uin, Uout, s);
  else env_cells_staged_w<K, D, FIRST, R, kLineWarps>(a, Uin, Uout, s);
}

template <int K, bool FIRST, typename R>
static void env_cells(const CycleArgs& a, int d, const double* Uin, double* Uout, cudaStream_t s) {
  const Dims& dm = a.dm;
  if (d == 0) {
    const int nseg = (dm.nx + kLineUpd - 1) / kLineUpd;
    const dim3 g(nseg, (dm.ny + kLineWarps - 1) / kLineWarps, dm.nz);
    auto kern = k_env_sweep_cells_x<K, FIRST, R>;
    if constexpr (sizeof(R) == 8) {
      if (env_pb(a)) kern = k_env_sweep_cells_x<K, FIRST, R, false, false, true>;
      else if (env_o3(a)) kern = k_env_sweep_cells_x<K, FIRST, R, false, true>;
      else if (env_gl(a)) kern = k_env_sweep_cells_x<K, FIRST, R, true>;
    }
    kern<<<g, 32 * kLineWarps, 0, s>>>(dm, a.S, a.ph, a.fd, a.n0, a.xc, a.ofn, Uin, Uout, a.dpf, a.Vlag);
  } else if (d == 1) {
    env_cells_staged<K, 1, FIRST, R>(a, Uin, Uout, s);
  } else {
    env_cells_staged<K, 2, FIRST, R>(a, Uin, Uout, s);
  }
}

// R: evaluation type of the sweeps (double, or float in the mixed form).
template <int K, typename R>
static void remap_env(const CycleArgs& a, int sens, cudaStream_t s, KernelMarks* m) {
  int prev = 0;
  for (int it = 0; it < 3; ++it) {
    const int d = (it + sens) % 3;
    const bool first = it == 0, last = it == 2;
    const double* uin = a.U[it & 1];
    double* uout = a.U[(it + 1) & 1];
    const double* udin = a.ud[(it + 1) & 1];
    double* udout = a.ud[it & 1];
    if (sizeof(R) == 8 && env_o3(a)) {
      const long long Fd = d == 0 ? a.dm.Fx : (d == 1 ? a.dm.Fy : a.dm.F - a.dm.Fx - a.dm.Fy);
      const unsigned nb = (unsigned)((Fd + 127) / 128);
      auto kern = first ? (d == 0 ? k_o3_faces_env<0, K, true> : (d == 1 ? k_o3_faces_env<1, K, true> : k_o3_faces_env<2, K, true>))
                        : (d == 0 ? k_o3_faces_env<0, K, false> : (d == 1 ? k_o3_faces_env<1, K, false> : k_o3_faces_env<2, K, false>));
      kern<<<nb, 128, 0, s>>>(a.dm, a.S, uin, a.fd, a.Vlag);
    }
    if (first) env_cells<K, true, R>(a, d, uin, uout, s);
    else env_cells<K, false, R>(a, d, uin, uout, s);
    if (last) {
      const unsigned nb = (unsigned)((a.dm.C + 255) / 256);
      k_env_finalize_cells<K><<<nb, 256, 0, s>>>(a.dm, a.S, a.ph, a.env, uout, a.st, a.fd);
    }
    mark(m, BK_CELLS_X + d, s);
    sweep_nodes<K, R>(a, d, first, last, prev, udin, udout, s);
    mark(m, BK_NODES_X + d, s);
    prev |= 1 << d;
  }
}

template <int K, typename R>
static void set_env_attributes_r() {
  const int mx = (int)(env_cells_staged_arrays<K, true>() * kTileArr * sizeof(double));
  cudaFuncSetAttribute(k_env_sweep_cells_t<K, 1, true, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_env_sweep_cells_t<K, 2, true, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_env_sweep_cells_t<K, 1, false, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_env_sweep_cells_t<K, 2, false, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  if constexpr (sizeof(R) == 8) {
    cudaFuncSetAttribute(k_env_sweep_cells_t<K, 1, true, R, kLineWarps, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
    cudaFuncSetAttribute(k_env_sweep_cells_t<K, 2, true, R, kLineWarps, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
    cudaFuncSetAttribute(k_env_sweep_cells_t<K, 1, false, R, kLineWarps, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
    cudaFuncSetAttribute(k_env_sweep_cells_t<K, 2, false, R, kLineWarps, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
    cudaFuncSetAttribute(k_env_sweep_cells_t<K, 1, true, R, kLineWarps, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
    cudaFuncSetAttribute(k_env_sweep_cells_t<K, 2, true, R, kLineWarps, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
    cudaFuncSetAttribute(k_env_sweep_cells_t<K, 1, false, R, kLineWarps, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
    cudaFuncSetAttribute(k_env_sweep_cells_t<K, 2, false, R, kLineWarps, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
    cudaFuncSetAttribute(k_env_sweep_cells_t<K, 1, true, R, kLineWarps, false, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
    cudaFuncSetAttribute(k_env_sweep_cells_t<K, 2, true, R, kLineWarps, false, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
    cudaFuncSetAttribute(k_env_sweep_cells_t<K, 1, false, R, kLineWarps, false, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
    cudaFuncSetAttribute(k_env_sweep_cells_t<K, 2, false, R, kLineWarps, false, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  }
}

template <int K>
static void set_env_attributes() {
  set_env_attributes_r<K, double>();
  set_env_attributes_r<K, float>();
}

template <int K, typename R>
static void lagrange_cells_env(const CycleArgs& a, const dim3 nbc, int linear, cudaStream_t s) {
  auto kern = k_cyc_lagrange_cells<K, R>;
  if constexpr (sizeof(R) == 8)
    if (a.fd.h) kern = k_cyc_lagrange_cells<K, R, true>;   // cell widths: order 3 and the generalised limiters
  kern<<<nbc, 128, 0, s>>>(a.dm, a.S, a.ph, a.x0, a.vh, a.n0, a.st.rho, a.st.e, a.st.q, a.st.p, a.st.cs, a.st.mass,
                           a.cqs, a.cqs32, a.L, a.U[0], a.xc, a.fd, a.env, a.Vlag, linear);
}

void launch_lagrange_cells_env(const CycleArgs& a, cudaStream_t s) {
  if (a.ph.csts) { launch_lagrange_cells_csts_env(a, s); return; }
  int linear;
  const dim3 nbc = cell_grid(a.dm, linear);
  if (a.ph.precision) {
    if (a.K == 2) lagrange_cells_env<2, float>(a, nbc, linear, s);
    else if (a.K == 3) lagrange_cells_env<3, float>(a, nbc, linear, s);
    else lagrange_cells_env<4, float>(a, nbc, linear, s);
  } else {
    if (a.K == 2) lagrange_cells_env<2, double>(a, nbc, linear, s);
    else if (a.K == 3) lagrange_cells_env<3, double>(a, nbc, linear, s);
    else lagrange_cells_env<4, double>(a, nbc, linear, s);
  }
}

void launch_remap_env(const CycleArgs& a0, int sens, cudaStream_t s, KernelMarks* m) {
  // schema-csts: the remap starts from the forward velocity (U_dual,
  // Phi_dual, PrepareRemap.cc:411-433) on the Lagrangian coordinates
  CycleArgs a = a0;
  if (a.ph.csts) a.vh = a.vf;
  if (a.ph.precision) {
    if (a.K == 2) remap_env<2, float>(a, sens, s, m);
    else if (a.K == 3) remap_env<3, float>(a, sens, s, m);
    else remap_env<4, float>(a, sens, s, m);
  } else {
    if (a.K == 2) remap_env<2, double>(a, sens, s, m);
    else if (a.K == 3) remap_env<3, double>(a, sens, s, m);
    else remap_env<4, double>(a, sens, s, m);
  }
}

// ------------------------------------------------------------------------
// Batched cycle of instances with K environments each: the same bodies as the
// single-context kernels, driven by the batch's work tables over persistent
// grids (as the one-environment batch in mhy_cycle.cu).  The cell y/z sweeps
// take 8 or 16 lines per block, the node y/z sweeps 8, as in one context.

template <int K, typename R, bool HC, bool CSTS = false>
__global__ void __launch_bounds__(128, sizeof(R) == 4 ? 5 : 3) k_bat_env_lagrange_cells(
    const CycleArgs* __restrict__ D, const int4* __restrict__ W, int nw) {
  for (int w = blockIdx.x; w < nw; w += gridDim.x) {
    const int4 t = W[w];
    const CycleArgs& a = D[t.x];
    k_cyc_lagrange_cells_body<K, R, CSTS, HC>(a.dm, a.S, a.ph, a.x0, a.vh, a.n0, a.st.rho, a.st.e, a.st.q, a.st.p,
                                              a.st.cs, a.st.mass, a.cqs, CSTS ? nullptr : a.cqs32, a.L, a.U[0], a.xc,
                                              a.fd, a.env, a.Vlag, t.y, t.z, t.w, a.vnb, a.pf);
  }
}

template <int K, bool FIRST, typename R, bool GL, bool PB = false, bool O3 = false>
__global__ void __launch_bounds__(32 * kLineWarps, kEnvMinBlocks) k_bat_env_cells_x(
    const CycleArgs* __restrict__ D, const int4* __restrict__ W, int nw, int it) {
  for (int w = blockIdx.x; w < nw; w += gridDim.x) {
    const int4 t = W[w];
    const CycleArgs& a = D[t.x];
    env_sweep_cells_x_body<K, FIRST, R, GL, O3, PB>(a.dm, a.S, a.ph, a.fd, a.n0, a.xc, a.ofn, a.U[it & 1], a.U[(it + 1) & 1],
                                        a.dpf, a.Vlag, t.y, t.z, t.w);
  }
}

template <int K, int DD, bool FIRST, typename R, int LW, bool GL, bool PB = false, bool O3 = false>
__global__ void __launch_bounds__(32 * LW, kEnvMinBlocks * kLineWarps / LW) k_bat_env_cells_t(
    const CycleArgs* __restrict__ D, const int4* __restrict__ W, int nw, int it) {
  for (int w = blockIdx.x; w < nw; w += gridDim.x) {
    const int4 t = W[w];
    const CycleArgs& a = D[t.x];
    __syncthreads();                                   // the previous item's tile reads are done
    env_sweep_cells_t_body<K, DD, FIRST, R, LW, GL, O3, PB>(a.dm, a.S, a.ph, a.fd, a.n0, a.xc, a.ofn, a.U[it & 1],
                                                a.U[(it + 1) & 1], a.dpf, a.Vlag, t.y, t.z, t.w);
  }
}

// the end of the remap, per cell, over the Lagrange cell kernel's tiles; the
// last cell sweep (it = 2) wrote U[1]
template <int K>
__global__ void __launch_bounds__(128) k_bat_env_finalize(const CycleArgs* __restrict__ D, const int4* __restrict__ W,
                                                          int nw) {
  for (int w = blockIdx.x; w < nw; w += gridDim.x) {
    const int4 t = W[w];
    const CycleArgs& a = D[t.x];
    int i, j, k;
    if (block_item(a.dm.nx, a.dm.ny, a.dm.nz, t.y, t.z, t.w, i, j, k))
      env_finalize_cell<K>(a.dm, a.S, a.ph, a.env, a.U[1], a.st, a.fd, (int)a.dm.cid(i, j, k));
  }
}

template <bool FIRST, bool LAST, int K, typename R, bool GL>
__global__ void __launch_bounds__(32 * kLineWarps, kLineMinBlocks) k_bat_env_nodes_x(
    const CycleArgs* __restrict__ D, const int4* __restrict__ W, int nw, int it, int prev) {
  for (int w = blockIdx.x; w < nw; w += gridDim.x) {
    const int4 t = W[w];
    const CycleArgs& a = D[t.x];
    // schema-csts: the forward velocity on the Lagrangian coordinates (xl is null otherwise)
    k_cyc_sweep_nodes_x_body<FIRST, LAST, K, R, GL>(a.dm, a.S, a.ph, prev, a.x0, a.xl, a.ph.csts ? a.vf : a.vh, a.nm,
                                                 a.ud[(it + 1) & 1], a.ud[it & 1], a.dpf, a.Gd, a.st.mass, a.v, a.nm,
                                                 a.vnorm, t.y, t.z, t.w, a.ecn);
  }
}

template <int DD, bool FIRST, bool LAST, int K, typename R, bool GL>
__global__ void __launch_bounds__(32 * kLineWarps, TileGeom<kLineWarps>::minb) k_bat_env_nodes_t(
    const CycleArgs* __restrict__ D, const int4* __restrict__ W, int nw, int it, int prev) {
  for (int w = blockIdx.x; w < nw; w += gridDim.x) {
    const int4 t = W[w];
    const CycleArgs& a = D[t.x];
    __syncthreads();
    k_cyc_sweep_nodes_t_body<DD, FIRST, LAST, K, R, kLineWarps, GL>(a.dm, a.S, a.ph, prev, a.x0, a.xl,
                                                                    a.ph.csts ? a.vf : a.vh,
                                                                    a.nm, a.ud[(it + 1) & 1], a.ud[it & 1], a.dpf,
                                                                    a.Gd, a.st.mass, a.v, a.nm, a.vnorm, t.y, t.z,
                                                                    t.w, a.ecn);
  }
}

template <class Kern, class... Args>
static void bat_env_launch(Kern kernel, int threads, size_t smem, const BatchPlan& P, int kind, int tk, cudaStream_t s,
                           KernelMarks* m, Args... args) {
  const int nwork = P.nwork[kind];
  smem_opt_in((const void*)kernel, smem);
  if (nwork > 0)
    kernel<<<persistent_grid((const void*)kernel, threads, smem, nwork, P.occ_pct[tk]), threads, smem, s>>>(args...);
  mark(m, tk, s);
}

template <int K, int DD, bool FIRST, typename R, bool GL>
static void bat_env_cells(const BatchPlan& P, int it, cudaStream_t s, KernelMarks* m) {
  const int kind = BK_CELLS_X + DD;
  if constexpr (sizeof(R) == 8) {
    if (P.o3) {   // order 3: the face values first, then the O3 cell sweeps (no gradient), 8 lines
      auto fk = k_bat_o3_faces_env<DD, K, FIRST>;
      if (P.o3nwork[DD] > 0)
        fk<<<persistent_grid((const void*)fk, 128, 0, P.o3nwork[DD], 100), 128, 0, s>>>(P.descs, P.o3work[DD],
                                                                                   P.o3nwork[DD], it);
      if constexpr (DD == 0)
        bat_env_launch(k_bat_env_cells_x<K, FIRST, R, false, false, true>, 32 * kLineWarps, 0, P, kind, kind, s,
                       nullptr, P.descs, P.work[kind], P.nwork[kind], it);
      else
        bat_env_launch(k_bat_env_cells_t<K, DD, FIRST, R, kLineWarps, false, false, true>, 32 * kLineWarps,
                       (size_t)env_cells_staged_arrays<K, FIRST>() * TileGeom<kLineWarps>::arr * sizeof(double), P,
                       kind, kind, s, nullptr, P.descs, P.work[kind], P.nwork[kind], it);
      return;
    }
    if (P.pb) {   // pente-borne: its own cell sweeps, 8 lines
      if constexpr (DD == 0)
        bat_env_launch(k_bat_env_cells_x<K, FIRST, R, false, true>, 32 * kLineWarps, 0, P, kind, kind, s, nullptr,
                       P.descs, P.work[kind], P.nwork[kind], it);
      else
        bat_env_launch(k_bat_env_cells_t<K, DD, FIRST, R, kLineWarps, false, true>, 32 * kLineWarps,
                       (size_t)env_cells_staged_arrays<K, FIRST>() * TileGeom<kLineWarps>::arr * sizeof(double), P,
                       kind, kind, s, nullptr, P.descs, P.work[kind], P.nwork[kind], it);
      return;
    }
  }
  if constexpr (DD == 0) {
    bat_env_launch(k_bat_env_cells_x<K, FIRST, R, GL>, 32 * kLineWarps, 0, P, kind, kind, s, nullptr, P.descs,
                   P.work[kind], P.nwork[kind], it);
  } else if (!GL && P.lines[kind] == 16) {
    bat_env_launch(k_bat_env_cells_t<K, DD, FIRST, R, 16, false>, 32 * 16,
                   (size_t)env_cells_staged_arrays<K, FIRST>() * TileGeom<16>::arr * sizeof(double), P, kind, kind, s,
                   nullptr, P.descs, P.work[kind], P.nwork[kind], it);
  } else {
    bat_env_launch(k_bat_env_cells_t<K, DD, FIRST, R, kLineWarps, GL>, 32 * kLineWarps,
                   (size_t)env_cells_staged_arrays<K, FIRST>() * TileGeom<kLineWarps>::arr * sizeof(double), P, kind,
                   kind, s, nullptr, P.descs, P.work[kind], P.nwork[kind], it);
  }
}

template <int K, int DD, bool FIRST, bool LAST, typename R, bool GL>
static void bat_env_nodes(const BatchPlan& P, int it, int prev, cudaStream_t s, KernelMarks* m) {
  const int kind = BK_NODES_X + DD;
  if constexpr (DD == 0)
    bat_env_launch(k_bat_env_nodes_x<FIRST, LAST, K, R, GL>, 32 * kLineWarps, 0, P, kind, kind, s, m, P.descs,
                   P.work[kind], P.nwork[kind], it, prev);
  else
    bat_env_launch(k_bat_env_nodes_t<DD, FIRST, LAST, K, R, GL>, 32 * kLineWarps,
                   NodeTileSize<DD, FIRST, LAST, K, kLineWarps>::bytes, P, kind, kind, s, m, P.descs, P.work[kind],
                   P.nwork[kind], it, prev);
}

template <int K, int DD, typename R, bool GL>
static void bat_env_sweep(const BatchPlan& P, int it, int prev, cudaStream_t s, KernelMarks* m) {
  const bool first = it == 0, last = it == 2;
  if (first) bat_env_cells<K, DD, true, R, GL>(P, it, s, m);
  else bat_env_cells<K, DD, false, R, GL>(P, it, s, m);
  if (last)   // the end of the remap per cell, between the last cell and node sweeps
    bat_env_launch(k_bat_env_finalize<K>, 128, 0, P, BK_LCELLS, BK_CELLS_X + DD, s, nullptr, P.descs,
                   P.work[BK_LCELLS], P.nwork[BK_LCELLS]);
  else
    mark(m, BK_CELLS_X + DD, s);
  if (first) bat_env_nodes<K, DD, true, false, R, GL>(P, it, prev, s, m);
  else if (last) bat_env_nodes<K, DD, false, true, R, GL>(P, it, prev, s, m);
  else bat_env_nodes<K, DD, false, false, R, GL>(P, it, prev, s, m);
}

// conservation-energie-totale of the instances that have it, over the Lagrange
// cell kernel's tiles, after the last node sweep
template <int K>
__global__ void __launch_bounds__(128) k_bat_env_cons_ec(const CycleArgs* __restrict__ D, const int4* __restrict__ W,
                                                         int nw) {
  for (int w = blockIdx.x; w < nw; w += gridDim.x) {
    const int4 t = W[w];
    const CycleArgs& a = D[t.x];
    if (!a.ph.cons_ec) continue;
    int i, j, k;
    if (block_item(a.dm.nx, a.dm.ny, a.dm.nz, t.y, t.z, t.w, i, j, k))
      env_cons_ec_cell<K>(a.dm, a.env, a.st, a.ecn, i, j, k);
  }
}

template <int K, typename R, bool GL, bool HC>
static void batch_cycle_env(const BatchPlan& P, int sens, cudaStream_t s, KernelMarks* m) {
  launch_bat_lagrange_nodes(P, s, m);
  bool done = false;
  if constexpr (sizeof(R) == 8) {
    if (P.csts) {   // schema-csts: the cell kernel's CSTS form, then the forward step and the face velocities
      bat_env_launch(k_bat_env_lagrange_cells<K, R, HC, true>, 128, 0, P, BK_LCELLS, BK_LCELLS, s, m, P.descs,
                     P.work[BK_LCELLS], P.nwork[BK_LCELLS]);
      launch_bat_csts_forward(P, s);
      done = true;
    }
  }
  if (!done)
    bat_env_launch(k_bat_env_lagrange_cells<K, R, HC>, 128, 0, P, BK_LCELLS, BK_LCELLS, s, m, P.descs,
                   P.work[BK_LCELLS], P.nwork[BK_LCELLS]);
  int prev = 0;
  for (int it = 0; it < 3; ++it) {
    const int d = (it + sens) % 3;
    if (d == 0) bat_env_sweep<K, 0, R, GL>(P, it, prev, s, m);
    else if (d == 1) bat_env_sweep<K, 1, R, GL>(P, it, prev, s, m);
    else bat_env_sweep<K, 2, R, GL>(P, it, prev, s, m);
    prev |= 1 << d;
  }
  if (P.cons_ec)
    bat_env_launch(k_bat_env_cons_ec<K>, 128, 0, P, BK_LCELLS, BK_LCELLS, s, nullptr, P.descs, P.work[BK_LCELLS],
                   P.nwork[BK_LCELLS]);
  launch_bat_dt(P, s, m);
}

template <int K>
static void batch_cycle_env_k(const BatchPlan& P, int sens, cudaStream_t s, KernelMarks* m) {
  // HC: the cell widths (the G limiters, pente-borne, order 3); GL: the G limiters' sweeps
  if (P.precision) batch_cycle_env<K, float, false, false>(P, sens, s, m);
  else if (P.gl) batch_cycle_env<K, double, true, true>(P, sens, s, m);
  else if (P.pb || P.o3) batch_cycle_env<K, double, false, true>(P, sens, s, m);
  else batch_cycle_env<K, double, false, false>(P, sens, s, m);
}

void launch_batch_cycle_env(const BatchPlan& P, int sens, cudaStream_t s, KernelMarks* m) {
  if (P.K == 2) batch_cycle_env_k<2>(P, sens, s, m);
  else if (P.K == 3) batch_cycle_env_k<3>(P, sens, s, m);
  else batch_cycle_env_k<4>(P, sens, s, m);
}

// Called once per context before any cycle (and so before any graph capture).
void launch_init_env(const CycleArgs& a, cudaStream_t s) {
  static std::once_flag once[kMaxEnvDevice + 1];
  const unsigned nb = (unsigned)((a.dm.C + 255) / 256);
  if (a.K == 2) { std::call_once(once[2], set_env_attributes<2>); k_env_init_state<2><<<nb, 256, 0, s>>>(a.dm, a.env, a.st); }
  else if (a.K == 3) { std::call_once(once[3], set_env_attributes<3>); k_env_init_state<3><<<nb, 256, 0, s>>>(a.dm, a.env, a.st); }
  else { std::call_once(once[4], set_env_attributes<4>); k_env_init_state<4><<<nb, 256, 0, s>>>(a.dm, a.env, a.st); }
}

}  // namespace mhy
