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
  int precision;        // 0: FP64; 1: mixed (FP32 evaluation of the remap, FP64 state and sums)
  int eos;              // environment 0: 0 PerfectGas, 1 StiffenedGas
  double pinf;          // its limit-tension
  int with_newton;      // Lagrange energy update by Newton iterations
  int csts;             // schema-csts time scheme (FP64)
  int lim_cell;         // limiter of the cell gradients: limiteur_id, or the pure-cell limiter when
                        // projection-pente-borne-mixte and projection-limiteur-pure-id 1 (RemapADIService.cc:369-375)
  // projection-pente-borne (FP64, order 2): the flux variant
  // (0: computeFluxPP, 1: computeFluxPPPure), its debar fix, the limiter of its
  // reconstruction (computeY0), and whether the sweep is the first of the cycle
  int pb, pb_pure, pb_debar, pb_lim_y0, pb_first;
  int cons_ec;          // conservation-energie-totale (RemapADI.axl:151; FP64)
  int ext_dt;           // slabs: the cycle ends with the local dt minimum; the caller combines the
                        // ranks' minima and finishes the dt (mhy_dt_finish)
  // several environments: projection-pente-borne-mixte and projection-limiteur-pure-id, applied
  // cell by cell where the neighbourhood is pure (RemapADIService.cc:364-375, UtilesRemap.cc:406-409)
  int pb_mixte, lim_pure;
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
  double* h;      // order 3: cell widths along each direction, 3 planes of C (RemapADIService.cc:225-258)
  double* phi3;   // order 3: face values of the current sweep, [4][faces of its direction]
  double* pbphi;  // pente-borne: rho, e and q after the Lagrange step, 3 planes of C (Phi of the first
                  // sweep, PrepareRemap.cc:201-212; q stays the Phi of q in every sweep).  Several
                  // environments: the 3K+1 planes of Phi for the first sweep (volume fraction, density,
                  // internal energy of each environment, then q); an environment absent from a cell
                  // keeps the Phi of the previous remap's last sweep (PrepareRemap.cc:201-212 sets only
                  // the cell's environments), zero before the first remap
  uint32_t* est;  // several environments with order 3 or projection-pente-borne-mixte: each cell's
                  // mixed/pure indicator after the last remap (m_est_mixte, m_est_pure,
                  // RemapADIFinal.cc:495-507) as 255 (mixed) or 1 + the pure environment (0: none);
                  // 1 (both indicators zero) before the first remap
};

// Persistent cell state (global values of a single-environment mesh).
struct CellState {
  double *rho, *e, *q, *p, *cs, *mass;
  const double* Ve;
  double* mf;           // conservation-energie-totale: the cell's mass fraction out of the last
                        // cell sweep (0 where the remap zeroed the cell); null otherwise
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
  int eos[MHY_MAX_ENV];           // 0 PerfectGas, 1 StiffenedGas
  double pinf[MHY_MAX_ENV];       // StiffenedGas limit-tension
};

struct CycleArgs {
  Dims dm;
  Scalars* S;
  Phys ph;
  BCTable bct;
  const uint16_t* bcmask;
  const double *x0, *n0, *ofn;
  double *v, *vh, *nm, *cqs, *L, *dpf, *Gd, *xc, *vnorm;
  float* cqs32;         // corner vectors of the mixed form (FP32)
  double* U[2];
  double* ud[2];
  FaceData fd;
  CellState st;
  int K;                // number of environments
  EnvState env;         // K > 1 only
  double* Vlag;         // Lagrangian cell volume (K > 1: divisor of Phi on the first sweep)
  int lines[8];         // lines per block of each sweep (indexed like BatchKernel; y/z sweeps of K = 1: 8, 16, 32)
  double *vnb, *vf, *xl;  // schema-csts: backward v_n, forward v, Lagrangian node coordinates (3N each)
  double* pf;             // schema-csts: p + q of the forward step (C)
  double* ecn;            // conservation-energie-totale: each node's kinetic-energy term out of the
                          // last node sweep (N); null otherwise
};

void launch_lagrange_nodes(const CycleArgs& a, cudaStream_t s);
void launch_csts_forward(const CycleArgs& a, cudaStream_t s);
void launch_lagrange_cells(const CycleArgs& a, cudaStream_t s);
struct KernelMarks;
void launch_remap(const CycleArgs& a, int sens, cudaStream_t s, KernelMarks* marks = nullptr);
void launch_delta_t(const CycleArgs& a, cudaStream_t s);
void launch_cons_ec(const CycleArgs& a, cudaStream_t s);
void launch_cons_ec_env(const CycleArgs& a, cudaStream_t s);
void launch_lagrange_cells_csts_env(const CycleArgs& a, cudaStream_t s);
constexpr int kKernelsPerCycle = 10;
// meshes with 2..kMaxEnvDevice environments (mhy_multi.cu)
constexpr int kMaxEnvDevice = 4;
void launch_lagrange_cells_env(const CycleArgs& a, cudaStream_t s);
void launch_remap_env(const CycleArgs& a, int sens, cudaStream_t s, KernelMarks* m = nullptr);
void launch_init_env(const CycleArgs& a, cudaStream_t s);
constexpr int kKernelsPerCycleEnv = 11;

// Batched cycle of many independent meshes (the same K in each).  Each kernel
// type has a work table: one (instance, bx, by, bz) entry per block of the
// instance's own grid; a persistent grid of resident blocks walks the table.
// The arguments of instance i are descs[i] in device memory.
constexpr int kLineWarps = 8;                   // warps (lines) per block of the sweeps (default)
constexpr int kLineOptions[3] = {8, 16, 32};    // the y/z sweeps' tunable lines per block
enum BatchKernel { BK_LNODES = 0, BK_LCELLS, BK_CELLS_X, BK_CELLS_Y, BK_CELLS_Z, BK_NODES_X, BK_NODES_Y, BK_NODES_Z,
                   BK_COUNT,
                   BK_DT_MIN = BK_COUNT,      // tuning slots beyond the work tables: the dt reduction (cell
                   BK_DT_FINISH,              // tiles of BK_LCELLS) and the per-instance dt finish
                   BK_TUNE_SLOTS };
struct BatchPlan {
  const CycleArgs* descs;       // device, one per instance
  int ninst;
  const int4* work[BK_COUNT];   // device work tables
  int nwork[BK_COUNT];
  int precision;                // all instances share it
  int occ_pct[BK_TUNE_SLOTS];   // persistent grid of each slot: % of the resident-block capacity
  int lines[BK_COUNT];          // lines per block of the y/z sweeps (8, 16, 32); the work shapes follow it
  int K;                        // environments of every instance
  int gl;                       // every instance takes the G limiters (FP64): the GL sweeps and cell widths
  int pb;                       // every instance takes projection-pente-borne (FP64): the PB cell sweeps
  int o3;                       // every instance takes order 3 (FP64): face values, then the O3 cell sweeps
  int csts;                     // every instance takes schema-csts (FP64)
  const int4* fwork;            // schema-csts: face work table (instance, chunk of 128 faces of all directions)
  int nfwork;
  const int4* o3work[3];        // order 3: face work tables (instance, chunk of 128 faces) per direction
  int o3nwork[3];
  int cons_ec;                  // some instance has conservation-energie-totale
};
// Events recorded after each launch of a cycle (autotuning), with the tuning
// slot of each launch.
struct KernelMarks {
  static constexpr int kMax = 16;
  cudaEvent_t ev[kMax];
  int kind[kMax];
  int n;
};
void batch_work_shape(const Dims& dm, int kind, int lines, int& gx, int& gy, int& gz);
// Records an event after a launch (autotuning): slot `kind` of the marks.
void mark(KernelMarks* m, int kind, cudaStream_t s);
// Batched cycle helpers: the resident-block grid of a persistent kernel, the
// Lagrange node kernel and the dt reduction of a batch (any K), and the
// batched cycle of instances with K > 1 environments.
int persistent_grid(const void* kernel, int threads, size_t smem, int nwork, int pct);
void launch_bat_lagrange_nodes(const BatchPlan& P, cudaStream_t s, KernelMarks* m);
void launch_bat_dt(const BatchPlan& P, cudaStream_t s, KernelMarks* m);
void launch_bat_csts_forward(const BatchPlan& P, cudaStream_t s);
void launch_batch_cycle_env(const BatchPlan& P, int sens, cudaStream_t s, KernelMarks* m);
void launch_bat_cons_ec(const BatchPlan& P, cudaStream_t s);
void launch_batch_cycle(const BatchPlan& plan, int sens, cudaStream_t s, KernelMarks* marks = nullptr);
constexpr int kKernelsPerCycleBatch = 10;

__global__ void k_init_cells(Dims dm, const double* x0, double* xc0, double* cqs, double* vol, double* L, int lc_mode);
__global__ void k_init_faces(Dims dm, const double* x0, double* n0, double* xf0);
__global__ void k_init_outer_normals(Dims dm, const double* x0, double* ofn);
constexpr int kTotalsThreads = 256;
constexpr int kTotalsBlocks = 148;   // one per SM; partials: 6 doubles per block
__global__ void k_totals_partial(Dims dm, const double* mass, const double* e, const double* nm, const double* v,
                                 double* part);
__global__ void k_totals_finish(const double* part, int nparts, double* out);
__global__ void k_max3_finish(const double* part, int nparts, double* out);
__global__ void k_init_state(Dims dm, Phys ph, const double* vol, double* rho, const double* pres, double* e,
                             double* cs, double* mass, double* q);
__global__ void k_node_mass(Dims dm, const double* mass, double* nm);
__global__ void k_to_f32(long long n, const double* src, float* dst);
__global__ void k_soa3(long long n, const double* aos, double* soa);
__global__ void k_fill_u32(long long n, uint32_t* a, uint32_t value);
__global__ void k_gather_index(long long n, int comps, const int32_t* idx, const double* src, double* out);
__global__ void k_aos3(long long n, const double* soa, const double* vh, const Scalars* S, double* aos);
__global__ void k_max3_partial(long long n, const double* x, double* part);
__global__ void k_face_groups(Dims dm, const double* x0, const double* part, int nparts, double thr, unsigned* grp);
__global__ void k_bc_mask(long long n, const unsigned* grp, int nbc, const int* surf, uint16_t* mask);
__global__ void k_dt_min(Dims dm, Scalars* S, const double* L, const double* cs, const double* vnorm, int linear);
dim3 cell_grid(const Dims& dm, int& linear);
__global__ void k_dt_finish(Scalars* S, Phys ph);
__global__ void k_dt_finish_ext(Scalars* S, Phys ph, const unsigned long long* min_bits);

// computeHydroDeltaT (MahycoModule.cc:2047-2061): min over cells of
// L / (c + max |v|) (|v| per node precomputed), warp shuffle + block
// reduction, one atomicMin per block on the bit pattern (non-negative doubles
// order like unsigned integers).
__device__ __forceinline__ void dt_min_body(Dims dm, Scalars* __restrict__ S, const double* __restrict__ L,
                                            const double* __restrict__ cs, const double* __restrict__ vnorm,
                                            int bx_, int by_, int bz_) {
  __shared__ unsigned long long wmin[32];
  int i, j, k;
  const bool has = block_item(dm.nx, dm.ny, dm.nz, bx_, by_, bz_, i, j, k) && k >= dm.dt_k0 && k < dm.dt_k1;
  unsigned long long best = 0x7fefffffffffffffull;  // DBL_MAX
  if (has) {
    const long long c = dm.cid(i, j, k);
    double vmax = 0.;
    for (int a = 0; a < 8; ++a) {
      long long n = dm.nid(i + kCellNodeOff[a][0], j + kCellNodeOff[a][1], k + kCellNodeOff[a][2]);
      vmax = amax(vnorm[n], vmax);
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
    // the running minimum only decreases, so a block whose minimum is not
    // below a value read from it would leave it unchanged: skip that atomic
    // (one block per 128 cells would otherwise queue ~16k atomics on one
    // address per Sedov 128^3 cycle)
    if (threadIdx.x == 0 && best < __ldcg(&S->min_bits)) atomicMin(&S->min_bits, best);
  }
}

// computeDeltaT (MahycoModule.cc:2076-2191): new dt from the reduced minimum.
__device__ __forceinline__ void dt_finish_body(Scalars* S, const Phys& ph) {
  S->time += S->dt;
  const double gold = S->dt;
  S->old_dt = gold;
  const double minimum_aux = __longlong_as_double((long long)S->min_bits);
  double new_dt = ph.cfl * minimum_aux;
  new_dt = amin(new_dt, 1.05 * gold);
  new_dt = amin(new_dt, ph.deltat_max);
  if (new_dt < ph.deltat_min) S->status |= MHY_STATUS_DT_MIN;
  S->dt = new_dt;
  S->inv_dt = 1.0 / new_dt;
  if (S->time > ph.final_time) S->status |= MHY_STATUS_FINAL_TIME;
  S->min_bits = 0x7fefffffffffffffull;
  S->iteration += 1;
}

}  // namespace mhy
