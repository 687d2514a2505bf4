// mhy_kernels.cuh -- kernel declarations and the small structs passed to them.
#pragma once

#include <cstdint>
#include "mhy_device.cuh"
#include "../../include/mhy.h"

namespace mhy {

// Device-resident time-step scalars: dt of the current cycle (m_global_deltat),
// dt of the previous cycle (m_old_deltat), time, the dt-reduction slot and the
// status word.  Read by every kernel, so a captured cycle needs no host value.
struct Scalars {
  double dt;
  double old_dt;
  double inv_dt;       // 1.0 / dt
  double time;
  unsigned long long min_bits;
  unsigned int status;
  unsigned int pad;
  long long iteration;
};

struct Phys {
  double gamma, threshold, cfl, deltat_min, deltat_max, final_time;
  int lc_mode, pseudo_centree, ordre_projection, limiteur_id;
};

struct BCTable {
  int nb;
  int type[MHY_MAX_BC];
  double value[MHY_MAX_BC];
};

// Per-cycle data of the inner faces of each direction d (index = face index
// within direction d): (x_f - x_c(prev)).n0, (x_f - x_c(next)).n0, |A_f|
// along d, normal velocity u_f.
struct FaceData {
  double* db[3];
  double* df[3];
  double* A[3];
  double* u[3];
};

// Persistent cell state (global values of a single-environment mesh).
struct CellState {
  double *rho, *e, *q, *p, *cs, *mass;
  const double* Ve;
};

// Environments (materials) of a mesh with K > 1 of them.  A cell that
// belongs to one environment only keeps that environment's values in the
// global cell arrays (CellState); a cell that belongs to several ("mixed")
// keeps each environment's values in the [K][C] planes below (Arcane's
// partial values, accenv/MultiEnvUtils.h:303-442) and the mixed averages in
// the global arrays.  fg and xg are the global volume and mass fractions.
struct EnvState {
  uint32_t* mask;       // bit k set: the cell belongs to environment k
  double *f, *x;        // [K][C] volume fraction, mass fraction
  double *rho, *e, *p, *cs, *q, *m;   // [K][C] density, specific internal energy, pressure, sound speed,
                                      // pseudo-viscosity, mass
  double *fg, *xg;      // [C]
  double gamma[MHY_MAX_ENV];
};

struct CycleArgs {
  Dims dm;
  Scalars* S;
  Phys ph;
  BCTable bct;
  const uint16_t* bcmask;
  const double *x0, *n0, *ofn;
  double *v, *vh, *nm, *cqs, *L, *dpf, *Gd, *xc, *vnorm;
  double* U[2];
  double* ud[2];
  FaceData fd;
  CellState st;
  int K;                // number of environments
  EnvState env;         // K > 1 only
  double* Vlag;         // Lagrangian cell volume (K > 1: divisor of Phi on the first sweep)
};

void launch_lagrange_nodes(const CycleArgs& a, cudaStream_t s);
void launch_lagrange_cells(const CycleArgs& a, cudaStream_t s);
void launch_remap(const CycleArgs& a, int sens, cudaStream_t s);
void launch_delta_t(const CycleArgs& a, cudaStream_t s);
constexpr int kKernelsPerCycle = 10;
// meshes with 2..kMaxEnvDevice environments (mhy_multi.cu)
constexpr int kMaxEnvDevice = 4;
void launch_lagrange_cells_env(const CycleArgs& a, cudaStream_t s);
void launch_remap_env(const CycleArgs& a, int sens, cudaStream_t s);
void launch_init_env(const CycleArgs& a, cudaStream_t s);
constexpr int kKernelsPerCycleEnv = 11;

__global__ void k_init_cells(Dims dm, const double* x0, double* xc0, double* cqs, double* vol, double* L, int lc_mode);
__global__ void k_init_faces(Dims dm, const double* x0, double* n0, double* xf0);
__global__ void k_init_outer_normals(Dims dm, const double* xc0, const double* xf0, double* ofn);
__global__ void k_init_state(Dims dm, double gamma, const double* vol, double* rho, const double* pres, double* e,
                             double* cs, double* mass, double* q);
__global__ void k_node_mass(Dims dm, const double* mass, double* nm);
__global__ void k_dt_min(Dims dm, Scalars* S, const double* L, const double* cs, const double* vnorm);
__global__ void k_dt_finish(Scalars* S, Phys ph);

}  // namespace mhy
