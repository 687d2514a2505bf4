/* mhy.h -- C ABI of the B200 implementation of MaHyCo's Lagrange + ADI-remap step.
 *
 * Every entry point returns 0 (MHY_OK) or a negative MHY_ERR_* code; nothing
 * throws across this boundary and nothing calls exit().  A context owns its
 * device memory and one CUDA stream; all work is ordered on that stream.  One
 * context per host thread.  The caller owns every host buffer it passes.
 *
 * Reference interfaces replaced (paths relative to the reference project root):
 *   - the Arcane module entry points of mahyco/src/Mahyco.axl:150-168, called in
 *     the order of mahyco/src/Mahyco.config:18-41 (MahycoModule.cc);
 *   - the remap service interface IRemap, mahyco/src/Remap/IRemap.h:32-65
 *     (appliRemap + remapVariables, called from mahyco/src/PrepareRemap.cc:462);
 *   - the equation-of-state interface IEquationOfState,
 *     mahyco/src/eos/IEquationOfState.h:32-65 (PerfectGas, applied after the remap,
 *     mahyco/src/PrepareRemap.cc:553-558).
 */
#ifndef MHY_H
#define MHY_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define MHY_OK                 0
#define MHY_ERR_ARG           -1   /* bad argument or size */
#define MHY_ERR_CUDA          -2   /* a CUDA call failed (message: mhy_last_error) */
#define MHY_ERR_OOM           -3   /* device allocation failed */
#define MHY_ERR_UNSUPPORTED   -4   /* option or configuration not implemented */
#define MHY_ERR_ORDER         -5   /* entry point called out of the time-loop order */
#define MHY_ERR_DT_MIN        -6   /* new dt < deltat-min (reference: exit(1), MahycoModule.cc:2152-2159) */
#define MHY_ERR_NUMERIC       -7   /* NaN / non-positive volume detected on the device */
#define MHY_ERR_STATE         -8   /* context not initialised / state missing */

/* ---- device status bits (mhy_get_status) ---- */
#define MHY_STATUS_DT_MIN       0x1u  /* dt fell below deltat-min */
#define MHY_STATUS_FINAL_TIME   0x2u  /* time passed final-time (reference stopComputeLoop) */
#define MHY_STATUS_NAN_DT       0x4u  /* a cell's dx/(c+|v|) was NaN or negative */
#define MHY_STATUS_ZERO_MASS    0x8u  /* a cell's remapped mass was exactly 0 (unsupported) */

/* ---- boundary conditions (TypesMahyco.h:9-18, MahycoAnnexe.cc:183-281) ---- */
enum { MHY_XMIN = 0, MHY_XMAX, MHY_YMIN, MHY_YMAX, MHY_ZMIN, MHY_ZMAX };
enum { MHY_VX = 0, MHY_VY = 1, MHY_VZ = 2 };

typedef struct mhy_bc {
  int32_t surface;   /* MHY_XMIN .. MHY_ZMAX: nodes of the faces lying on that plane */
  int32_t type;      /* MHY_VX / MHY_VY / MHY_VZ: velocity component imposed */
  double value;
} mhy_bc;

#define MHY_MAX_BC  16
#define MHY_MAX_ENV 8

/* Options, with the names of Mahyco.axl:170-340 and Remap/RemapADI.axl:139-177.
 * mhy_options_default() gives the reference defaults plus the values of the
 * decks in mahyco/data/Data.1.arc:59-104. */
typedef struct mhy_options {
  double cfl;                        /* 0.3 */
  double threshold;                  /* 1e-10 */
  double deltat_init;                /* 1e-5 */
  double deltat_min;                 /* 1e-8 */
  double deltat_max;                 /* 0.01 */
  double final_time;                 /* 0.2 */
  int32_t longueur_caracteristique;  /* 0 "racine-cubique-volume", 1 "faces-opposees" */
  int32_t pseudo_centree;            /* 0 */
  int32_t ordre_projection;          /* 2 (1, 2, and 3 in FP64 for one to four environments: Remap-ordre-3.cc) */
  int32_t projection_limiteur_id;    /* 0 minmod, 1 superBee, 2 vanLeer; the generalised limiters for uneven
                                        widths 3 minmodG, 4 superBeeG, 5 vanLeerG, 6 arithmeticG, 7 ultrabeeG
                                        (UtilesRemap.cc:127-175; FP64, one to four environments, >= 3 cells a
                                        direction) */
  int32_t nb_bc;
  mhy_bc bc[MHY_MAX_BC];             /* default: walls on the six planes */
  int32_t nb_env;                    /* number of environments (one ideal gas each; 1..4 on the device) */
  double adiabatic_cst[MHY_MAX_ENV]; /* PerfectGas adiabatic-cst per environment */
  int32_t precision;                 /* 0: plain FP64 (bit for bit the reference's arithmetic);
                                        1: mixed: the remap's Phi, gradients, limiters, face values and
                                        flux terms in FP32; state, coordinates, volumes, conserved sums
                                        and the dt reduction in FP64 */
  int32_t eos[MHY_MAX_ENV];           /* per environment: 0 PerfectGas (eos/perfectgas), 1 StiffenedGas
                                        (eos/stiffenedgas/StiffenedGasEOSService.cc) */
  double limit_tension[MHY_MAX_ENV]; /* StiffenedGas limit-tension (StiffenedGasEOS.axl:104, default 0.01) */
  int32_t with_newton;               /* 0; 1: Lagrange energy update by Newton iterations on the EOS
                                        (Mahyco.axl:308, MahycoModule.cc:1482-1535; schema-csts false) */
  int32_t schema_csts;               /* 0; 1: the CSTS time scheme (Mahyco.axl:238): velocity taken back to n-1/2
                                        before the Lagrange step and forward to n+1 before the remap, energy from
                                        the corner vectors of n and n+1 (MahycoModule.cc:693-831, 1776-1810,
                                        PrepareRemap.cc:69-79, 456); precision 0 */
  int32_t projection_pente_borne;    /* 0; 1: the pente-borne remap (RemapADI.axl:167; RemapADIService.cc:319-437,
                                        530-581, 745-840; UtilesRemap.cc:73-93, 184-296, 406-823): fluxes
                                        integrated from a three-piece reconstruction; precision 0,
                                        ordre-projection 2, one to four environments */
  int32_t pente_borne_debar_fix;     /* 0, 1 or 2: projection-pente-borne-debar-fix (RemapADI.axl:171) */
  int32_t pente_borne_mixte;         /* 0; 1: projection-pente-borne-mixte (RemapADI.axl:155): where a cell and
                                        its two neighbours along the sweep are pure cells of one environment
                                        (with one environment: everywhere) the pure-cell fluxes
                                        (computeFluxPPPure) and limiter apply; precision 0 */
  int32_t limiteur_pure_id;          /* 0..7: projection-limiteur-pure-id (RemapADI.axl:163), the reconstruction's
                                        limiter in pure neighbourhoods, and the gradient's when it is 1 */
  int32_t conservation_energie_totale; /* 0; 1: conservation-energie-totale (RemapADI.axl:151;
                                        RemapADIFinal.cc:751-773): after the remap each cell's specific
                                        internal energy gains max(0, sum over its 8 nodes of
                                        0.25 (U_dual[4]/U_dual[3] - 0.5 |v|^2)) times its mass fraction,
                                        with U_dual[4] = 0.5 m |v| as the reference builds it (each
                                        environment's energy gains x_k delta, a mixed cell's mean delta);
                                        precision 0, not batched */
} mhy_options;

/* Structured hexahedral mesh: (nx+1)(ny+1)(nz+1) nodes, node (i,j,k) at
 * index i + (nx+1)*(j + (ny+1)*k), coordinates xyz interleaved (copied). */
typedef struct mhy_mesh_desc {
  int32_t nx, ny, nz;
  const double* node_coords;
} mhy_mesh_desc;

/* Explicit connectivity, in the caller's own numbering of cells and nodes:
 * cell c has the 8 nodes cell_nodes[cell_node_offsets[c] .. +8) in the
 * SN_trigo local order of Arcane's Cartesian cells
 * (cartesian/CartConnectivityCellNode.h:83-94), offsets every 8 from 0;
 * node coordinates xyz interleaved.  This is the cell -> node table the
 * reference reads from Arcane (accenv/AccEnvDefaultService.cc:240-268 builds
 * its node -> cell counterpart from it). */
typedef struct mhy_csr_mesh {
  int64_t ncells, nnodes;
  const int64_t* cell_node_offsets;   /* ncells + 1 */
  const int64_t* cell_nodes;          /* 8 * ncells node ids */
  const double* node_coords;          /* nnodes x 3 */
} mhy_csr_mesh;

/* Recognises a logically Cartesian block of hexahedra in explicit
 * connectivity (any numbering, every cell in the SN_trigo local order):
 * dims = cells along x, y, z; cell_index[c] / node_index[n] = the structured
 * id (i + nx (j + ny k), nodes with nx+1, ny+1) of the caller's cell c / node
 * n.  Host only, no GPU needed.  MHY_ERR_UNSUPPORTED when the connectivity is
 * not one full box of cells with consistently ordered nodes, MHY_ERR_ARG on
 * bad arrays. */
int mhy_csr_structure(int64_t ncells, int64_t nnodes, const int64_t* cell_node_offsets, const int64_t* cell_nodes,
                      int32_t dims[3], int32_t* cell_index, int32_t* node_index);

/* Initial state, the role of the test-case service initVar + the EOS initEOS
 * (casTest/IInitialisations.h:32-50, eos/IEquationOfState.h): per environment
 * volume fraction, density and pressure of every cell (nb_env x ncells,
 * environment-major; a cell belongs to environment k when fracvol > 0), and
 * the node velocity (nnodes x 3 interleaved). */
typedef struct mhy_state {
  const double* fracvol;
  const double* density;
  const double* pressure;
  const double* velocity;
} mhy_state;

/* Fields readable with mhy_get_field (global cell values; velocity/coords as xyz) */
typedef enum mhy_field {
  MHY_FIELD_DENSITY = 0, MHY_FIELD_INTERNAL_ENERGY = 1, MHY_FIELD_PRESSURE = 2,
  MHY_FIELD_SOUND_SPEED = 3, MHY_FIELD_PSEUDO_VISCOSITY = 4, MHY_FIELD_CELL_VOLUME = 5,
  MHY_FIELD_CELL_MASS = 6, MHY_FIELD_CARACTERISTIC_LENGTH = 7,
  MHY_FIELD_VELOCITY = 10, MHY_FIELD_NODE_MASS = 11, MHY_FIELD_NODE_COORD = 12
} mhy_field;

typedef struct mhy_ctx mhy_ctx;

void mhy_options_default(mhy_options* opt);

/* Mesh + options -> context (MahycoModule::accBuild, MahycoModule.cc:34-43, and
 * the mesh/connectivity part of AccEnvDefaultService::initMesh,
 * accenv/AccEnvDefaultService.cc:274-302). device < 0: current device. */
int mhy_create(const mhy_mesh_desc* mesh, const mhy_options* opt, int device, mhy_ctx** out);

/* The same from explicit connectivity (the mesh part of
 * AccEnvDefaultService::initMesh, accenv/AccEnvDefaultService.cc:240-302,
 * from Arcane's item lists): the block is recognised with mhy_csr_structure
 * and the two numbering maps are kept in device memory.  Every cell and node
 * array the context exchanges with the caller (mhy_set_state, mhy_get_field,
 * mhy_get_env_field, mhy_get_env_mask) is then in the caller's numbering; the
 * kernels run on the structured layout.  Results equal those of mhy_create on
 * the same block bit for bit. */
int mhy_create_csr(const mhy_csr_mesh* mesh, const mhy_options* opt, int device, mhy_ctx** out);

/* Initial state (casModel()->initVar, MahycoModule.cc:104). */
int mhy_set_state(mhy_ctx* ctx, const mhy_state* st);

/* Init entry points of Mahyco.config:23-29 in one call: HydroStartInit
 * (MahycoModule.cc:48-188), PrepareFaceGroup (MahycoAnnexe.cc:183-251),
 * ComputeCellMass (MahycoModule.cc:199-225), ComputeNodeMass (:235-266). */
int mhy_hydro_start_init(mhy_ctx* ctx);

/* Compute-loop entry points, Mahyco.config:30-41, to be called in this order
 * once per cycle.  The work is fused into fewer kernels, so a function may do
 * the work of the next ones (e.g. mhy_update_velocity also applies the
 * boundary conditions and moves the nodes); fields are only defined at cycle
 * boundaries.  Out-of-order calls return MHY_ERR_ORDER. */
int mhy_save_values_at_n(mhy_ctx* ctx);             /* MahycoModule.cc:308-450 */
int mhy_update_velocity(mhy_ctx* ctx);              /* MahycoModule.cc:678-731 */
int mhy_apply_boundary_condition(mhy_ctx* ctx);     /* MahycoModule.cc:936-1004 */
int mhy_update_position(mhy_ctx* ctx);              /* MahycoModule.cc:870-931 */
int mhy_compute_geometric_values(mhy_ctx* ctx);     /* MahycoModule.cc:1054-1299 */
int mhy_update_density(mhy_ctx* ctx);               /* MahycoModule.cc:1331-1426 */
int mhy_compute_artificial_viscosity(mhy_ctx* ctx); /* MahycoModule.cc:454-578 */
int mhy_update_energy_and_pressure(mhy_ctx* ctx);   /* MahycoModule.cc:1439-1478 */
int mhy_remap(mhy_ctx* ctx);                        /* PrepareRemap.cc:448-563 = IRemap::appliRemap
                                                       + remapVariables + IEquationOfState::applyEOS */
int mhy_compute_delta_t(mhy_ctx* ctx);              /* MahycoModule.cc:2076-2191 */

/* ncycles complete cycles (all entry points above), replayed from a CUDA graph. */
int mhy_step(mhy_ctx* ctx, int ncycles);

/* Wait for the context's stream; returns MHY_ERR_DT_MIN / MHY_ERR_NUMERIC when
 * the device raised the matching status bit. */
int mhy_synchronize(mhy_ctx* ctx);

/* Copy one field to host memory (pinned memory copies at full bus speed):
 * ncells or nnodes doubles, or nnodes x 3 interleaved for the velocity and
 * the node coordinates (interleaved on the device, then one copy).  Waits
 * for the work recorded so far; MHY_ERR_ARG when bytes is too small. */
int mhy_get_field(mhy_ctx* ctx, int field, void* dst, size_t bytes);
/* Per-environment cell values (Arcane's environment views, e.g. the
 * EnvCellVariableRealRef fields of Mahyco.axl read through an IMeshEnvironment):
 * for every cell, the value of environment `env` when the cell belongs to it
 * (the cell's own value for a pure cell), else 0.  ncells doubles. */
typedef enum mhy_env_field {
  MHY_ENV_FRACVOL = 0, MHY_ENV_DENSITY = 1, MHY_ENV_INTERNAL_ENERGY = 2, MHY_ENV_PRESSURE = 3,
  MHY_ENV_SOUND_SPEED = 4, MHY_ENV_MASS_FRACTION = 5, MHY_ENV_CELL_MASS = 6
} mhy_env_field;
int mhy_get_env_field(mhy_ctx* ctx, int field, int env, void* dst, size_t bytes);
/* Environment membership: bit k of dst[c] set when cell c belongs to
 * environment k (ncells uint32). */
int mhy_get_env_mask(mhy_ctx* ctx, uint32_t* dst, size_t bytes);
/* dt of the next cycle (m_global_deltat), dt of the last cycle (m_old_deltat) */
int mhy_get_dt(mhy_ctx* ctx, double* dt, double* dt_old);
int mhy_get_time(mhy_ctx* ctx, double* time, int64_t* iteration);
int mhy_get_status(mhy_ctx* ctx, uint32_t* flags);
int mhy_get_sizes(mhy_ctx* ctx, int64_t* ncells, int64_t* nnodes, int64_t* nfaces);
/* Conserved totals at the current cycle boundary, summed on the device with
 * compensated (TwoSum) additions in a fixed order: out[0] = total mass
 * sum_c m_c, out[1] = internal energy sum_c m_c e_c, out[2] = kinetic energy
 * sum_n 0.5 m_n |v_n|^2 (node mass as remapVariables sets it,
 * RemapADIFinal.cc:712-718).  Total energy = out[1] + out[2]. */
int mhy_get_totals(mhy_ctx* ctx, double out[3]);
/* The context's CUDA stream (cudaStream_t), for callers that order their own work after it. */
void* mhy_get_stream(mhy_ctx* ctx);
/* Number of kernels one cycle launches. */
int mhy_kernels_per_cycle(mhy_ctx* ctx);
const char* mhy_last_error(void);
void mhy_destroy(mhy_ctx* ctx);

/* ---- restart dump (checkpoint / resume) ----
 * The state a cycle starts from, as one host buffer: dt, old dt, time,
 * iteration, remap direction, and the cell and node variables the reference
 * dumps for a restart (Mahyco.axl variables with dump="true": Density,
 * InternalEnergy, Pressure, SoundSpeed, PseudoViscosity, CellMass, Velocity,
 * NodeMass, CellCQS, DualGradPhi, and the per-environment values), in a
 * self-describing layout (header, named field records, arrays).  Save between
 * cycles; load into a context created with the same mesh and options (in
 * place of mhy_set_state + mhy_hydro_start_init: the "continue-init"
 * entry point hydroContinueInit, MahycoModule.cc:269-305, Mahyco.axl:153).  The continued run equals the uninterrupted one bit for
 * bit. */
int mhy_checkpoint_size(mhy_ctx* ctx, size_t* bytes);
int mhy_checkpoint_save(mhy_ctx* ctx, void* dst, size_t bytes);
int mhy_checkpoint_load(mhy_ctx* ctx, const void* src, size_t bytes);

/* ---- slabs: one mesh split along z over several contexts (GPUs) ----
 * The reference splits its mesh into MPI subdomains with ghost layers
 * (MahycoModule.cc:62-75) and reduces dt over all of them once a cycle
 * (ReducerMin, MahycoModule.cc:2067).  Here each rank holds a context on its
 * own z-slab plus `ghost` layers of the neighbours' cells and nodes on each
 * inner side, deeper than one cycle's dependency reach along z (at most 5
 * layers: Lagrange 1, cell sweep 2, node sweep and its mass fluxes 2), so the
 * owned layers of every rank come out of a cycle exactly as in the unsplit
 * run.  A cycle is: mhy_step(ctx, 1) (ending with the dt minimum over the
 * owned cell layers only), mhy_dt_local_min, a minimum over the ranks done by
 * the caller (e.g. an NCCL all-reduce on the 64-bit pattern: non-negative
 * doubles order like unsigned integers), mhy_dt_finish, then the ghost
 * layers refreshed from the neighbours with mhy_halo_pack / mhy_halo_unpack
 * (every restart-dump field, contiguous per component and layer range; the
 * caller moves the buffers, e.g. with NCCL send/recv).  Any number of
 * environments: the restart state holds every environment plane. */
/* dt reduced over cell layers [k_lo, k_hi) of this context; external = 1:
 * the cycle stops after the local minimum (mhy_dt_local_min / mhy_dt_finish). */
int mhy_set_dt_reduction(mhy_ctx* ctx, int32_t k_lo, int32_t k_hi, int32_t external);
/* copies the local minimum (uint64 bit pattern) to device memory, on the context's stream */
int mhy_dt_local_min(mhy_ctx* ctx, void* dev_min_bits);
/* the new dt from the combined minimum (device uint64), on the context's stream */
int mhy_dt_finish(mhy_ctx* ctx, const void* dev_min_bits);
/* bytes of the state of `cell_layers` cell layers and `node_layers` node layers */
int mhy_halo_bytes(mhy_ctx* ctx, int32_t cell_layers, int32_t node_layers, size_t* bytes);
/* state of cell layers [cell_lo, cell_hi) and node layers [node_lo, node_hi) to / from a
 * device buffer, on the context's stream */
int mhy_halo_pack(mhy_ctx* ctx, int32_t cell_lo, int32_t cell_hi, int32_t node_lo, int32_t node_hi, void* dev_dst,
                  size_t bytes);
int mhy_halo_unpack(mhy_ctx* ctx, int32_t cell_lo, int32_t cell_hi, int32_t node_lo, int32_t node_hi,
                    const void* dev_src, size_t bytes);

/* ---- batches: many independent meshes on one GPU ----
 * No counterpart in the reference (one Arcane process runs one mesh): a batch
 * advances n instances of uneven sizes, options and initial states together,
 * each kernel of the cycle launched once for all instances (persistent grids
 * walking a per-instance work table), each instance with its own dt on the
 * device; the whole cycle is replayed from a CUDA graph.  Instance i is set up
 * exactly as a context (mesh i, options i, state i) and its results equal a
 * context's bit for bit.  Every instance has the same nb_env (1..4) and the same
 * precision; the G limiters (projection_limiteur_id 3..7),
 * projection_pente_borne, ordre_projection 3 and schema_csts are in every
 * instance or in none (MHY_ERR_UNSUPPORTED otherwise). */
typedef struct mhy_batch mhy_batch;
int mhy_batch_create(int n, const mhy_mesh_desc* meshes, const mhy_options* opts, int device, mhy_batch** out);
int mhy_batch_set_state(mhy_batch* b, int i, const mhy_state* st);
int mhy_batch_hydro_start_init(mhy_batch* b);          /* all instances */
int mhy_batch_step(mhy_batch* b, int ncycles);         /* ncycles cycles of every instance */
int mhy_batch_synchronize(mhy_batch* b);               /* MHY_ERR_DT_MIN / MHY_ERR_NUMERIC if any instance raised it */
int mhy_batch_get_field(mhy_batch* b, int i, int field, void* dst, size_t bytes);
int mhy_batch_get_dt(mhy_batch* b, int i, double* dt, double* dt_old);
int mhy_batch_get_status(mhy_batch* b, int i, uint32_t* flags);
int mhy_batch_get_totals(mhy_batch* b, int i, double out[3]);

/* Tuning of the cycle: per kernel slot, the lines per block of the staged
 * y/z sweeps and, in a batch, the order of the work table and the size of the
 * persistent grid.  Slots: 0 Lagrange nodes, 1 Lagrange cells, 2-4 cell
 * sweeps x/y/z, 5-7 node sweeps x/y/z, 8 dt reduction (walks the work table
 * of slot 1, so its order is slot 1's), 9 dt finish (nothing to tune).
 * Results do not depend on the tuning: every work item computes the same
 * values whatever its tile shape, its order or the grid that runs it. */
#define MHY_TUNE_SLOTS 10
typedef struct mhy_tuning {
  int32_t order[MHY_TUNE_SLOTS];           /* batch: 0 instance-major (default), 1 largest instance first,
                                              2 instances interleaved 16 tiles at a time */
  int32_t occupancy_pct[MHY_TUNE_SLOTS];   /* batch: persistent grid as % of the resident-block capacity,
                                              1..100 (100) */
  int32_t lines_per_block[MHY_TUNE_SLOTS]; /* slots 3, 4, 6, 7 (y/z sweeps) of one-environment meshes: 8 (default),
                                              16 or 32 lines of 32 positions per block, i.e. rows of 64, 128 or
                                              256 contiguous bytes in the staged loads; other slots 8 */
  double ms_default[MHY_TUNE_SLOTS];       /* autotune: measured ms per cycle of each slot with the defaults ... */
  double ms_tuned[MHY_TUNE_SLOTS];         /* ... and with the chosen settings */
  int32_t from_cache;                      /* 1: taken from the in-process cache (keyed on the mesh sizes, the
                                              number of environments and the precision) without trials */
  int32_t trials;                          /* settings tried */
} mhy_tuning;

/* Autotuner: times every candidate setting on the context's (batch's) own
 * state for `cycles` cycles each (1..20, after mhy_hydro_start_init), keeps
 * per slot the fastest (a setting must beat the default by 2 %) and restores
 * the state bit for bit afterwards (device snapshot: needs free device memory
 * the size of the state).  Candidates: lines per block 8/16/32 on the y/z
 * sweeps; in a batch also 3 work orders x occupancy 100/75/50 %.  The choice
 * is cached for the process per set of mesh sizes. */
int mhy_autotune(mhy_ctx* ctx, int cycles, mhy_tuning* out);
int mhy_set_tuning(mhy_ctx* ctx, const mhy_tuning* t);
int mhy_get_tuning(mhy_ctx* ctx, mhy_tuning* out);
int mhy_batch_autotune(mhy_batch* b, int cycles, mhy_tuning* out);
int mhy_batch_set_tuning(mhy_batch* b, const mhy_tuning* t);
int mhy_batch_get_tuning(mhy_batch* b, mhy_tuning* out);
int mhy_batch_size(mhy_batch* b);
int mhy_batch_kernels_per_cycle(mhy_batch* b);
void* mhy_batch_get_stream(mhy_batch* b);
void mhy_batch_destroy(mhy_batch* b);

/* CFL time step from device-resident fields, for callers that cannot allocate
 * device memory (a host framework that owns all device allocations, or code
 * recording into a stream capture).  No counterpart in the reference: it is the
 * dt reduction of mhy_compute_delta_t with its scratch in a fixed 64 KiB
 * __device__ array instead of context memory.  Inputs (device pointers):
 * characteristic length L and sound speed cs per cell, node velocity v as
 * three planes (x[N], y[N], z[N]).  Output (device pointer, 2 doubles):
 * out[0] = min over cells of L/(cs + max |v| over the cell's nodes),
 * out[1] = min(cfl*out[0], 1.05*dt_old, deltat_max).  When any cell's
 * L/(cs + max |v|) is NaN or negative (an inverted cell, a NaN field), the
 * call writes out[0] = NaN and out[1] = 0: a dt below any positive deltat_min,
 * so a caller that checks the new dt against deltat_min stops the run as the
 * reference does (the context's reduction raises MHY_STATUS_NAN_DT instead).
 * Work is queued on `stream` (a cudaStream_t, NULL for the default stream);
 * nothing is allocated.  Meshes above 134217728 cells are rejected with
 * MHY_ERR_ARG.  All calls on a device share the scratch: calls that overlap
 * on the GPU race and must be serialised by the caller.  The first call on a
 * device, and the first call after the device's context was reset
 * (cudaDeviceReset), resolve the scratch address; make them before any
 * stream capture. */
int mhy_compute_hydro_dt_noalloc(int32_t nx, int32_t ny, int32_t nz, const double* L, const double* cs,
                                 const double* v, double cfl, double dt_old, double deltat_max,
                                 double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* MHY_H */
