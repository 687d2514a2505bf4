// mhy_capi.cu -- the C ABI of include/mhy.h: context, device memory, init,
// per-entry-point calls, CUDA-graph replay of whole cycles.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <algorithm>
#include <array>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "mhy_kernels.cuh"

using namespace mhy;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define MHY_CUDA(call)                                                                        \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return fail(e_ == cudaErrorMemoryAllocation ? MHY_ERR_OOM : MHY_ERR_CUDA,               \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                        \
  } while (0)

constexpr int kThreads = 256;
inline unsigned blocks(long long n) { return (unsigned)((n + kThreads - 1) / kThreads); }

// Makes a context's (or batch's) device current for the duration of an entry
// point and gives the caller back its own current device afterwards, so a
// context may be driven from a thread whose current device is another GPU.
struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int dev) {
    int cur = 0;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != dev && cudaSetDevice(dev) == cudaSuccess) prev = cur;
  }
  ~DeviceScope() { if (prev >= 0) cudaSetDevice(prev); }
  DeviceScope(const DeviceScope&) = delete;
  DeviceScope& operator=(const DeviceScope&) = delete;
};

enum Phase {
  PH_SAVE = 0, PH_VELOCITY, PH_BC, PH_POSITION, PH_GEOMETRY, PH_DENSITY, PH_VISCOSITY, PH_ENERGY,
  PH_REMAP, PH_DELTA_T
};

}  // namespace

struct mhy_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  Dims dm{};
  Phys ph{};
  BCTable bct{};
  mhy_options opt{};
  std::vector<void*> allocs;
  std::vector<size_t> alloc_bytes;               // size of each allocation (device state snapshots)
  std::vector<std::pair<void**, size_t>> plan;   // arena requests (pointer, bytes)
  double* setup = nullptr;                       // 1024 doubles of set-up scratch
  // nodes
  double *x0 = nullptr, *v = nullptr, *vh = nullptr, *nm = nullptr, *Gd = nullptr, *vnorm = nullptr;
  double *ud[2] = {nullptr, nullptr};
  uint16_t* bcmask = nullptr;
  // cells
  double *rho = nullptr, *e = nullptr, *q = nullptr, *p = nullptr, *cs = nullptr, *mass = nullptr;
  double *L = nullptr, *Ve = nullptr, *dpf = nullptr, *cqs = nullptr, *ofn = nullptr, *xc = nullptr;
  float* cqs32 = nullptr;
  double *vnb = nullptr, *vf = nullptr, *xl = nullptr, *pf = nullptr;   // schema-csts
  double *mfc = nullptr, *ecn = nullptr;   // conservation-energie-totale: cell mass fraction, node term
  // explicit connectivity (mhy_create_csr): the structured id of each of the
  // caller's cells and nodes, on the host and in HBM; empty for mhy_create
  std::vector<int32_t> cell_index, node_index;
  int32_t *d_cell_index = nullptr, *d_node_index = nullptr;
  double *U[2] = {nullptr, nullptr};
  // environments (K > 1)
  int K = 1;
  EnvState env{};
  double* Vlag = nullptr;
  // faces
  double* n0 = nullptr;
  FaceData fd{};
  Scalars* S = nullptr;
  int sens = 0;
  int phase = PH_SAVE;
  bool state_set = false, initialized = false;
  cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};
  int kernels_per_cycle = 0;
  int lines[BK_COUNT] = {kLineWarps, kLineWarps, kLineWarps, kLineWarps, kLineWarps, kLineWarps, kLineWarps,
                         kLineWarps};                  // lines per block of the sweeps (the tuning)
  // Entry points record their work and launch it late: at mhy_compute_delta_t a
  // whole recorded cycle becomes one launch of the cycle graph; any call that
  // reads or waits on the device launches what is pending first.
  int pend = 0;                                  // bit 0 velocity, 1 geometry, 2 remap
  int pend_sens = 0;                             // direction rotation of the pending remap
  mhy_tuning tuning{};

  // Device arrays come from one allocation: alloc() records a request,
  // commit() allocates the sum (256-byte aligned pieces) and sets the pointers.
  template <class T>
  int alloc(T** ptr, size_t count) {
    plan.emplace_back(reinterpret_cast<void**>(ptr), count * sizeof(T));
    return MHY_OK;
  }
  int commit() {
    size_t total = 0;
    for (auto& r : plan) total += (r.second + 255) & ~size_t(255);
    void* base = nullptr;
    cudaError_t err = cudaMalloc(&base, total + 256);
    if (err != cudaSuccess) return fail(MHY_ERR_OOM, "cudaMalloc failed: " + std::string(cudaGetErrorString(err)));
    allocs.push_back(base);
    alloc_bytes.push_back(total + 256);
    char* p_ = static_cast<char*>(base);
    for (auto& r : plan) {
      *r.first = p_;
      p_ += (r.second + 255) & ~size_t(255);
    }
    plan.clear();
    return MHY_OK;
  }

  CycleArgs args() const {
    CycleArgs a{};
    a.dm = dm; a.S = S; a.ph = ph; a.bct = bct; a.bcmask = bcmask;
    a.x0 = x0; a.n0 = n0; a.ofn = ofn;
    a.v = v; a.vh = vh; a.nm = nm; a.cqs = cqs; a.cqs32 = cqs32; a.L = L; a.dpf = dpf; a.Gd = Gd; a.xc = xc; a.vnorm = vnorm;
    a.U[0] = U[0]; a.U[1] = U[1]; a.ud[0] = ud[0]; a.ud[1] = ud[1];
    a.fd = fd;
    a.st.rho = rho; a.st.e = e; a.st.q = q; a.st.p = p; a.st.cs = cs; a.st.mass = mass; a.st.Ve = Ve;
    a.K = K; a.env = env; a.Vlag = Vlag;
    for (int k = 0; k < BK_COUNT; ++k) a.lines[k] = lines[k];
    a.vnb = vnb; a.vf = vf; a.xl = xl; a.pf = pf;
    a.st.mf = mfc; a.ecn = ecn;
    return a;
  }
};

extern "C" {

const char* mhy_last_error(void) { return g_last_error.c_str(); }

void mhy_options_default(mhy_options* o) {
  std::memset(o, 0, sizeof(*o));
  o->cfl = 0.3;
  o->threshold = 1.e-10;
  o->deltat_init = 1.e-5;
  o->deltat_min = 1.e-8;
  o->deltat_max = 0.01;
  o->final_time = 0.2;
  o->longueur_caracteristique = 0;
  o->pseudo_centree = 0;
  o->ordre_projection = 2;
  o->projection_limiteur_id = 0;
  o->nb_bc = 6;
  const int surf[6] = {MHY_XMIN, MHY_XMAX, MHY_YMIN, MHY_YMAX, MHY_ZMIN, MHY_ZMAX};
  const int typ[6] = {MHY_VX, MHY_VX, MHY_VY, MHY_VY, MHY_VZ, MHY_VZ};
  for (int b = 0; b < 6; ++b) { o->bc[b].surface = surf[b]; o->bc[b].type = typ[b]; o->bc[b].value = 0.; }
  o->nb_env = 1;
  o->adiabatic_cst[0] = 1.4;
  o->precision = 0;
  for (int k = 0; k < MHY_MAX_ENV; ++k) o->limit_tension[k] = 0.01;   // StiffenedGasEOS.axl:104
}

int mhy_create(const mhy_mesh_desc* mesh, const mhy_options* opt, int device, mhy_ctx** out) {
  if (!mesh || !opt || !out || !mesh->node_coords) return fail(MHY_ERR_ARG, "null argument");
  *out = nullptr;
  if (mesh->nx < 2 || mesh->ny < 2 || mesh->nz < 2) return fail(MHY_ERR_ARG, "need at least 2 cells per direction");
  {
    // The sweep kernels index elements with 32-bit offsets; the largest is
    // 24 C (the corner vectors) or 3 F (the face normals).
    const long long nx = mesh->nx, ny = mesh->ny, nz = mesh->nz;
    const long long C = nx * ny * nz, N = (nx + 1) * (ny + 1) * (nz + 1);
    const long long F = (nx + 1) * ny * nz + nx * (ny + 1) * nz + nx * ny * (nz + 1);
    if (nx > 65535 || ny > 65535 || nz > 65535 || 24 * C >= (1LL << 31) || 5 * N >= (1LL << 31) ||
        3 * F >= (1LL << 31))
      return fail(MHY_ERR_ARG, "mesh too large for one context (at most 89 million cells)");
  }
  if (opt->nb_env < 1 || opt->nb_env > kMaxEnvDevice)
    return fail(MHY_ERR_UNSUPPORTED, "nb_env must be 1.." + std::to_string(kMaxEnvDevice) + " on the device");
  for (int k = 0; k < opt->nb_env; ++k) {
    if (!(opt->adiabatic_cst[k] > 1.)) return fail(MHY_ERR_ARG, "adiabatic-cst must be > 1");
    if (opt->eos[k] < 0 || opt->eos[k] > 1) return fail(MHY_ERR_ARG, "eos must be 0 (PerfectGas) or 1 (StiffenedGas)");
  }
  if (opt->with_newton != 0 && opt->with_newton != 1) return fail(MHY_ERR_ARG, "with_newton must be 0 or 1");
  if (opt->ordre_projection < 1 || opt->ordre_projection > 3)
    return fail(MHY_ERR_UNSUPPORTED, "ordre-projection must be 1, 2 or 3");
  if (opt->ordre_projection == 3 && opt->precision != 0)
    return fail(MHY_ERR_UNSUPPORTED, "ordre-projection 3: FP64 on the device");
  if (opt->projection_limiteur_id < 0 || opt->projection_limiteur_id > 7)
    return fail(MHY_ERR_UNSUPPORTED, "projection-limiteur-id must be 0..7 (TypesMahyco.h:65-74)");
  if (opt->projection_limiteur_id >= 3 && opt->precision != 0)
    return fail(MHY_ERR_UNSUPPORTED, "the generalised (G) limiters: FP64 on the device");
  if (opt->projection_limiteur_id >= 3 && (mesh->nx < 3 || mesh->ny < 3 || mesh->nz < 3))
    return fail(MHY_ERR_UNSUPPORTED, "the generalised (G) limiters need 3 cells or more along every direction");
  if (opt->nb_bc < 0 || opt->nb_bc > MHY_MAX_BC) return fail(MHY_ERR_ARG, "nb_bc out of range");
  if (!(opt->cfl > 0.) || !(opt->deltat_init > 0.) || !(opt->deltat_max > 0.) || !(opt->deltat_min >= 0.) ||
      !(opt->threshold >= 0.) || !(opt->final_time > 0.))
    return fail(MHY_ERR_ARG, "cfl, deltat-init, deltat-max and final-time must be > 0, deltat-min and threshold >= 0");
  if (opt->precision < 0 || opt->precision > 1) return fail(MHY_ERR_ARG, "precision must be 0 (FP64) or 1 (mixed)");
  if (opt->schema_csts != 0 && opt->schema_csts != 1) return fail(MHY_ERR_ARG, "schema_csts must be 0 or 1");
  if (opt->schema_csts && opt->precision != 0)
    return fail(MHY_ERR_UNSUPPORTED, "schema-csts: FP64 on the device");
  if (opt->projection_pente_borne != 0 && opt->projection_pente_borne != 1)
    return fail(MHY_ERR_ARG, "projection_pente_borne must be 0 or 1");
  if (opt->pente_borne_mixte != 0 && opt->pente_borne_mixte != 1)
    return fail(MHY_ERR_ARG, "pente_borne_mixte must be 0 or 1");
  if (opt->pente_borne_debar_fix < 0 || opt->pente_borne_debar_fix > 2)
    return fail(MHY_ERR_ARG, "pente_borne_debar_fix must be 0, 1 or 2");
  if (opt->limiteur_pure_id < 0 || opt->limiteur_pure_id > 7)
    return fail(MHY_ERR_ARG, "limiteur_pure_id must be 0..7 (TypesMahyco.h:65-74)");
  if ((opt->projection_pente_borne || opt->pente_borne_mixte) && opt->precision != 0)
    return fail(MHY_ERR_UNSUPPORTED, "pente-borne: FP64 on the device");
  if (opt->projection_pente_borne && opt->ordre_projection != 2)
    return fail(MHY_ERR_UNSUPPORTED, "pente-borne: ordre-projection 2 on the device");
  for (int b = 0; b < opt->nb_bc; ++b)
    if (opt->bc[b].surface < 0 || opt->bc[b].surface > 5 || opt->bc[b].type < 0 || opt->bc[b].type > 2)
      return fail(MHY_ERR_ARG, "bad boundary condition");
  if (opt->conservation_energie_totale != 0 && opt->conservation_energie_totale != 1)
    return fail(MHY_ERR_ARG, "conservation_energie_totale must be 0 or 1");
  if (opt->conservation_energie_totale && opt->precision != 0)
    return fail(MHY_ERR_UNSUPPORTED, "conservation-energie-totale: FP64 on the device");

  mhy_ctx* c = new mhy_ctx();
  for (int k = 0; k < MHY_TUNE_SLOTS; ++k) {
    c->tuning.order[k] = 0; c->tuning.occupancy_pct[k] = 100; c->tuning.lines_per_block[k] = kLineWarps;
  }
  c->opt = *opt;
  if (device >= 0) {
    cudaError_t err = cudaSetDevice(device);
    if (err != cudaSuccess) { delete c; return fail(MHY_ERR_CUDA, cudaGetErrorString(err)); }
  }
  cudaGetDevice(&c->device);
  Dims& dm = c->dm;
  dm.nx = mesh->nx; dm.ny = mesh->ny; dm.nz = mesh->nz;
  dm.C = (long long)dm.nx * dm.ny * dm.nz;
  dm.N = (long long)(dm.nx + 1) * (dm.ny + 1) * (dm.nz + 1);
  dm.Fx = (long long)(dm.nx + 1) * dm.ny * dm.nz;
  dm.Fy = (long long)dm.nx * (dm.ny + 1) * dm.nz;
  dm.F = dm.Fx + dm.Fy + (long long)dm.nx * dm.ny * (dm.nz + 1);
  dm.dt_k0 = 0; dm.dt_k1 = dm.nz;
  Phys& ph = c->ph;
  ph.gamma = opt->adiabatic_cst[0];
  c->K = opt->nb_env;
  for (int k = 0; k < c->K; ++k) {
    c->env.gamma[k] = opt->adiabatic_cst[k];
    c->env.eos[k] = opt->eos[k];
    c->env.pinf[k] = opt->limit_tension[k];
  }
  ph.with_newton = opt->with_newton;
  ph.eos = opt->eos[0];
  ph.pinf = opt->limit_tension[0];
  ph.threshold = opt->threshold; ph.cfl = opt->cfl;
  ph.deltat_min = opt->deltat_min; ph.deltat_max = opt->deltat_max; ph.final_time = opt->final_time;
  ph.lc_mode = opt->longueur_caracteristique; ph.pseudo_centree = opt->pseudo_centree;
  ph.ordre_projection = opt->ordre_projection; ph.limiteur_id = opt->projection_limiteur_id;
  ph.precision = opt->precision;
  ph.csts = opt->schema_csts;
  // with one environment every cell and its neighbours are pure, so
  // projection-pente-borne-mixte selects the pure-cell forms everywhere
  // (voisinage_pure, RemapADIService.cc:369-375)
  ph.lim_cell = (opt->pente_borne_mixte && opt->limiteur_pure_id == 1) ? 1 : opt->projection_limiteur_id;
  ph.pb = opt->projection_pente_borne;
  ph.pb_pure = opt->pente_borne_mixte;
  ph.pb_debar = opt->pente_borne_debar_fix;
  ph.pb_lim_y0 = opt->pente_borne_mixte ? opt->limiteur_pure_id : opt->projection_limiteur_id;
  ph.pb_mixte = opt->pente_borne_mixte;
  ph.lim_pure = opt->limiteur_pure_id;
  ph.pb_first = 0;
  ph.cons_ec = opt->conservation_energie_totale;
  c->bct.nb = opt->nb_bc;
  for (int b = 0; b < opt->nb_bc; ++b) { c->bct.type[b] = opt->bc[b].type; c->bct.value[b] = opt->bc[b].value; }

  int rc = MHY_OK;
  auto A_ = [&](double** pp, long long n) { if (rc == MHY_OK) rc = c->alloc(pp, (size_t)n); };
  const long long C = dm.C, N = dm.N, F = dm.F;
  A_(&c->x0, 3 * N); A_(&c->v, 3 * N); A_(&c->vh, 3 * N); A_(&c->nm, N); A_(&c->Gd, 3 * N); A_(&c->vnorm, N);
  A_(&c->ud[0], 5 * N); A_(&c->ud[1], 5 * N);
  A_(&c->rho, C); A_(&c->e, C); A_(&c->q, C); A_(&c->p, C); A_(&c->cs, C); A_(&c->mass, C); A_(&c->L, C);
  const int K = c->K, NV = 3 * K + 1;
  A_(&c->Ve, C); A_(&c->dpf, K * C); A_(&c->xc, 3 * C); A_(&c->ofn, 6 * C);
  // corner vectors: FP64, and FP32 in the mixed form (hydro_start_init
  // converts the FP64 ones of t = 0)
  A_(&c->cqs, 24 * C);
  if (opt->precision == 1 && rc == MHY_OK) rc = c->alloc(&c->cqs32, (size_t)(24 * C));
  if (opt->schema_csts && rc == MHY_OK) {           // backward / forward velocities, coordinates, pressure
    rc = c->alloc(&c->vnb, (size_t)(3 * N));
    if (rc == MHY_OK) rc = c->alloc(&c->vf, (size_t)(3 * N));
    if (rc == MHY_OK) rc = c->alloc(&c->xl, (size_t)(3 * N));
    if (rc == MHY_OK) rc = c->alloc(&c->pf, (size_t)C);
  }
  A_(&c->U[0], NV * C); A_(&c->U[1], NV * C);
  if (opt->conservation_energie_totale) { A_(&c->mfc, C); A_(&c->ecn, N); }
  if (K > 1) {
    EnvState& ev = c->env;
    A_(&ev.f, K * C); A_(&ev.x, K * C); A_(&ev.rho, K * C); A_(&ev.e, K * C); A_(&ev.p, K * C);
    A_(&ev.cs, K * C); A_(&ev.q, K * C); A_(&ev.m, K * C); A_(&ev.fg, C); A_(&ev.xg, C); A_(&c->Vlag, C);
    if (rc == MHY_OK) rc = c->alloc(&ev.mask, (size_t)C);
  }
  A_(&c->n0, 3 * F);
  {
    const long long nf[3] = {dm.Fx, dm.Fy, dm.F - dm.Fx - dm.Fy};
    for (int d = 0; d < 3; ++d) {
      A_(&c->fd.db[d], nf[d]); A_(&c->fd.df[d], nf[d]); A_(&c->fd.A[d], nf[d]);
      A_(&c->fd.u[d], nf[d]);
    }
    if (opt->ordre_projection == 3 || opt->projection_limiteur_id >= 3 || opt->projection_pente_borne)
      A_(&c->fd.h, 3 * C);                                                                      // cell widths
    if (opt->projection_pente_borne) A_(&c->fd.pbphi, (K == 1 ? 3 : 3 * K + 1) * C);
    if (K > 1 && (opt->ordre_projection == 3 || opt->pente_borne_mixte) && rc == MHY_OK)
      rc = c->alloc(&c->fd.est, (size_t)C);                                                   // mixed/pure indicators
    if (opt->ordre_projection == 3)   // face values of the current sweep: 4 (one environment) or 3K+1 components
      A_(&c->fd.phi3, (K == 1 ? 4 : 3 * K + 1) * std::max(nf[0], std::max(nf[1], nf[2])));
  }
  if (rc == MHY_OK) rc = c->alloc(&c->bcmask, (size_t)N);
  if (rc == MHY_OK) rc = c->alloc(&c->S, 1);
  static_assert(6 * kTotalsBlocks + 3 <= 1024, "set-up scratch holds the totals partials");
  static_assert(3 * 256 + 64 + 3 <= 1024 && MHY_MAX_BC <= 128, "set-up scratch holds the coordinate maxima");
  if (rc == MHY_OK) rc = c->alloc(&c->setup, 1024);
  if (rc == MHY_OK) rc = c->commit();
  if (rc != MHY_OK) { mhy_destroy(c); return rc; }
  cudaError_t err = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (err != cudaSuccess) { mhy_destroy(c); return fail(MHY_ERR_CUDA, cudaGetErrorString(err)); }

  // Set-up on the device: the interleaved coordinates are staged in ud[0]
  // (5N doubles) and the node groups in vh, arrays the first cycle
  // overwrites; the per-block coordinate maxima and the BC surfaces go to
  // the set-up scratch.
  {
    const long long nb = (N + 255) / 256;
    const int nparts = 256;
    err = cudaMemcpyAsync(c->ud[0], mesh->node_coords, 3 * N * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (err == cudaSuccess) {
      k_soa3<<<(unsigned)nb, 256, 0, c->stream>>>(N, c->ud[0], c->x0);
      // dual gradients of nodes never inner so far read 0 (the reference's variables start at zero)
      cudaMemsetAsync(c->Gd, 0, 3 * N * sizeof(double), c->stream);
      // several environments: pente-borne Phi of environments absent so far read 0, and both
      // mixed/pure indicators start at zero (code 1), as the reference's variables do
      if (K > 1 && c->fd.pbphi) cudaMemsetAsync(c->fd.pbphi, 0, (size_t)(3 * K + 1) * C * sizeof(double), c->stream);
      if (c->fd.est) k_fill_u32<<<(unsigned)((C + 255) / 256), 256, 0, c->stream>>>(C, c->fd.est, 1u);
      k_max3_partial<<<nparts, 256, 0, c->stream>>>(N, c->x0, c->setup);
      unsigned* grp = reinterpret_cast<unsigned*>(c->vh);
      cudaMemsetAsync(grp, 0, N * sizeof(unsigned), c->stream);
      double* mx = c->setup + 3 * nparts + 64;           // after the partials and the BC surfaces
      k_max3_finish<<<1, 1, 0, c->stream>>>(c->setup, nparts, mx);
      k_face_groups<<<(unsigned)((F + 255) / 256), 256, 0, c->stream>>>(dm, c->x0, mx, 1, opt->threshold, grp);
      int* surf = reinterpret_cast<int*>(c->setup + 3 * nparts);
      int hs[MHY_MAX_BC] = {};
      for (int b = 0; b < opt->nb_bc; ++b) hs[b] = opt->bc[b].surface;
      err = cudaMemcpyAsync(surf, hs, sizeof(hs), cudaMemcpyHostToDevice, c->stream);
      k_bc_mask<<<(unsigned)nb, 256, 0, c->stream>>>(N, grp, opt->nb_bc, surf, c->bcmask);
      if (err == cudaSuccess) err = cudaGetLastError();
    }
    if (err != cudaSuccess) { mhy_destroy(c); return fail(MHY_ERR_CUDA, cudaGetErrorString(err)); }
  }
  // one wait at the end: the caller's coordinates may be pinned memory it frees on return
  Scalars s0{};
  s0.dt = opt->deltat_init; s0.old_dt = 0.; s0.time = 0.; s0.inv_dt = 1.0 / opt->deltat_init; s0.min_bits = 0x7fefffffffffffffull;
  err = cudaMemcpyAsync(c->S, &s0, sizeof(s0), cudaMemcpyHostToDevice, c->stream);
  if (err == cudaSuccess) err = cudaStreamSynchronize(c->stream);
  if (err != cudaSuccess) { mhy_destroy(c); return fail(MHY_ERR_CUDA, cudaGetErrorString(err)); }
  c->kernels_per_cycle = K > 1 ? kKernelsPerCycleEnv + (opt->ordre_projection == 3 ? 3 : 0) +
                                     (opt->conservation_energie_totale ? 1 : 0) + (opt->schema_csts ? 2 : 0)
                               : kKernelsPerCycle + (opt->schema_csts ? 2 : 0) + (opt->ordre_projection == 3 ? 3 : 0) +
                                     (opt->conservation_energie_totale ? 1 : 0);
  *out = c;
  return MHY_OK;
}

int mhy_create_csr(const mhy_csr_mesh* mesh, const mhy_options* opt, int device, mhy_ctx** out) {
  if (!mesh || !opt || !out || !mesh->cell_node_offsets || !mesh->cell_nodes || !mesh->node_coords)
    return fail(MHY_ERR_ARG, "null argument");
  *out = nullptr;
  if (mesh->ncells < 8 || mesh->nnodes < 27) return fail(MHY_ERR_ARG, "need at least 2 cells per direction");
  std::vector<int32_t> ci((size_t)mesh->ncells), ni((size_t)mesh->nnodes);
  int32_t dims[3] = {0, 0, 0};
  int rc = mhy_csr_structure(mesh->ncells, mesh->nnodes, mesh->cell_node_offsets, mesh->cell_nodes, dims, ci.data(),
                             ni.data());
  if (rc != MHY_OK)
    return fail(rc, rc == MHY_ERR_ARG ? "bad connectivity arrays (offsets, node ids or sizes)"
                                      : "connectivity is not one logically Cartesian block of hexahedra with the "
                                        "SN_trigo local node order (CartConnectivityCellNode.h:83-94)");
  std::vector<double> xs((size_t)3 * mesh->nnodes);
  for (int64_t u = 0; u < mesh->nnodes; ++u)
    for (int a = 0; a < 3; ++a) xs[3 * (size_t)ni[u] + a] = mesh->node_coords[3 * u + a];
  const mhy_mesh_desc md{dims[0], dims[1], dims[2], xs.data()};
  mhy_ctx* c = nullptr;
  rc = mhy_create(&md, opt, device, &c);
  if (rc != MHY_OK) return rc;
  DeviceScope on_dev(c->device);
  const size_t bc = ci.size() * sizeof(int32_t), bn = ni.size() * sizeof(int32_t);
  void* d = nullptr;
  cudaError_t err = cudaMalloc(&d, bc + bn + 256);
  if (err != cudaSuccess) { mhy_destroy(c); return fail(MHY_ERR_OOM, cudaGetErrorString(err)); }
  c->allocs.push_back(d);
  c->alloc_bytes.push_back(bc + bn + 256);
  c->d_cell_index = static_cast<int32_t*>(d);
  c->d_node_index = reinterpret_cast<int32_t*>(static_cast<char*>(d) + ((bc + 255) & ~size_t(255)));
  err = cudaMemcpy(c->d_cell_index, ci.data(), bc, cudaMemcpyHostToDevice);
  if (err == cudaSuccess) err = cudaMemcpy(c->d_node_index, ni.data(), bn, cudaMemcpyHostToDevice);
  if (err != cudaSuccess) { mhy_destroy(c); return fail(MHY_ERR_CUDA, cudaGetErrorString(err)); }
  c->cell_index = std::move(ci);
  c->node_index = std::move(ni);
  *out = c;
  return MHY_OK;
}

int mhy_set_state(mhy_ctx* c, const mhy_state* st) {
  if (!c || !st || !st->fracvol || !st->density || !st->pressure || !st->velocity) return fail(MHY_ERR_ARG, "null argument");
  DeviceScope on_dev(c->device);
  const long long C = c->dm.C, N = c->dm.N;
  const int K = c->K;
  std::vector<double> pfv, pde, ppr, pve;
  mhy_state perm{};
  if (!c->cell_index.empty()) {
    // the caller's numbering -> the structured one
    pfv.resize((size_t)K * C); pde.resize((size_t)K * C); ppr.resize((size_t)K * C); pve.resize((size_t)3 * N);
    for (int k = 0; k < K; ++k)
      for (long long u = 0; u < C; ++u) {
        const size_t d = (size_t)k * C + c->cell_index[u], o = (size_t)k * C + u;
        pfv[d] = st->fracvol[o]; pde[d] = st->density[o]; ppr[d] = st->pressure[o];
      }
    for (long long u = 0; u < N; ++u)
      for (int a = 0; a < 3; ++a) pve[3 * (size_t)c->node_index[u] + a] = st->velocity[3 * u + a];
    perm = mhy_state{pfv.data(), pde.data(), ppr.data(), pve.data()};
    st = &perm;
  }
  if (K == 1) {
    // the copies run while the host checks the volume fractions; a refused
    // state leaves the context without a state (state_set stays false)
    MHY_CUDA(cudaMemcpyAsync(c->rho, st->density, C * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    MHY_CUDA(cudaMemcpyAsync(c->p, st->pressure, C * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    MHY_CUDA(cudaMemcpyAsync(c->ud[0], st->velocity, 3 * N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    bool ok = true;
    for (long long i = 0; i < C; ++i) ok &= st->fracvol[i] > 0.;
    if (!ok) {
      cudaStreamSynchronize(c->stream);               // the caller may free its buffers on return
      c->state_set = false;
      return fail(MHY_ERR_UNSUPPORTED, "single-environment context: every cell needs fracvol > 0");
    }
  } else {
    // Environments from the volume fractions and the initial per-environment
    // state, as HydroStartInit sets them up on the host (MahycoModule.cc:48-127
    // with the test case's initMat/initVar): a pure cell takes its
    // environment's density and pressure as global values; a mixed cell keeps
    // f_k, rho_k, p_k per environment, the mass fractions f_k rho_k / sum f rho,
    // and the averages sum f_k rho_k, sum f_k p_k as global values.
    std::vector<uint32_t> mask(C, 0);
    std::vector<double> rho(C, 0.), pg(C, 0.), f((size_t)K * C, 0.), x((size_t)K * C, 0.), r((size_t)K * C, 0.),
        pk((size_t)K * C, 0.);
    for (long long i = 0; i < C; ++i) {
      uint32_t m = 0;
      for (int k = 0; k < K; ++k) if (st->fracvol[(size_t)k * C + i] > 0.) m |= 1u << k;
      if (!m) return fail(MHY_ERR_ARG, "a cell belongs to no environment (all fracvol <= 0)");
      mask[i] = m;
      if (__builtin_popcount(m) == 1) {
        const int e = __builtin_ctz(m);
        rho[i] = st->density[(size_t)e * C + i]; pg[i] = st->pressure[(size_t)e * C + i];
      } else {
        double rg = 0., pp = 0., mt = 0.;
        for (int k = 0; k < K; ++k) if (m >> k & 1) {
          const size_t o = (size_t)k * C + i;
          const double fk = st->fracvol[o], rk = st->density[o], pk_ = st->pressure[o];
          f[o] = fk; r[o] = rk; pk[o] = pk_;
          rg += fk * rk; pp += fk * pk_; mt += fk * rk;
        }
        for (int k = 0; k < K; ++k) if (m >> k & 1) {
          const size_t o = (size_t)k * C + i;
          x[o] = f[o] * r[o] / mt;
        }
        rho[i] = rg; pg[i] = pp;
      }
    }
    const EnvState& ev = c->env;
    MHY_CUDA(cudaMemcpyAsync(ev.mask, mask.data(), C * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
    MHY_CUDA(cudaMemcpyAsync(c->rho, rho.data(), C * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    MHY_CUDA(cudaMemcpyAsync(c->p, pg.data(), C * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    MHY_CUDA(cudaMemcpyAsync(ev.f, f.data(), (size_t)K * C * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    MHY_CUDA(cudaMemcpyAsync(ev.x, x.data(), (size_t)K * C * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    MHY_CUDA(cudaMemcpyAsync(ev.rho, r.data(), (size_t)K * C * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    MHY_CUDA(cudaMemcpyAsync(ev.p, pk.data(), (size_t)K * C * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  }
  // interleaved velocity staged in ud[0] (unused until the first cycle), then planes
  if (K > 1)
    MHY_CUDA(cudaMemcpyAsync(c->ud[0], st->velocity, 3 * N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  k_soa3<<<(unsigned)((N + 255) / 256), 256, 0, c->stream>>>(N, c->ud[0], c->v);
  MHY_CUDA(cudaGetLastError());
  MHY_CUDA(cudaStreamSynchronize(c->stream));
  c->state_set = true;
  return MHY_OK;
}

}  // extern "C"

namespace {

// Initial geometry from the mesh: cell centres and corner vectors, Eulerian
// volumes and lengths, face normals, outward face normals
// (MahycoAnnexe.cc:102-109, MahycoModule.cc:1008-1050, 1054-1262 at t = 0).
int init_geometry(mhy_ctx* c) {
  const Dims& dm = c->dm;
  cudaStream_t s = c->stream;
  k_init_cells<<<blocks(dm.C), kThreads, 0, s>>>(dm, c->x0, nullptr, c->cqs, c->Ve, c->L, c->ph.lc_mode);
  k_init_faces<<<blocks(dm.F), kThreads, 0, s>>>(dm, c->x0, c->n0, nullptr);
  k_init_outer_normals<<<blocks(dm.C), kThreads, 0, s>>>(dm, c->x0, c->ofn);
  MHY_CUDA(cudaGetLastError());
  return MHY_OK;
}

}  // namespace

extern "C" {

int mhy_hydro_start_init(mhy_ctx* c) {
  if (!c) return fail(MHY_ERR_ARG, "null context");
  if (!c->state_set) return fail(MHY_ERR_STATE, "mhy_set_state must come first");
  DeviceScope on_dev(c->device);
  const Dims& dm = c->dm;
  cudaStream_t s = c->stream;
  const int rc = init_geometry(c);
  if (rc != MHY_OK) return rc;
  if (c->K == 1) k_init_state<<<blocks(dm.C), kThreads, 0, s>>>(dm, c->ph, c->Ve, c->rho, c->p, c->e, c->cs, c->mass, c->q);
  else launch_init_env(c->args(), s);
  k_node_mass<<<blocks(dm.N), kThreads, 0, s>>>(dm, c->mass, c->nm);
  if (c->cqs32) k_to_f32<<<blocks(24 * dm.C), kThreads, 0, s>>>(24 * dm.C, c->cqs, c->cqs32);
  MHY_CUDA(cudaGetLastError());
  MHY_CUDA(cudaStreamSynchronize(s));
  c->initialized = true;
  c->phase = PH_SAVE;
  return MHY_OK;
}

}  // extern "C"

namespace {

int launch_velocity(mhy_ctx* c) { launch_lagrange_nodes(c->args(), c->stream); return MHY_OK; }
int launch_geometry(mhy_ctx* c) {
  if (c->K == 1) launch_lagrange_cells(c->args(), c->stream);
  else launch_lagrange_cells_env(c->args(), c->stream);
  return MHY_OK;
}
int launch_remap_(mhy_ctx* c, int sens, KernelMarks* m = nullptr) {
  if (c->K == 1) {
    if (c->ph.csts) launch_csts_forward(c->args(), c->stream);   // PrepareRemap.cc:456, then the face velocities
    launch_remap(c->args(), sens, c->stream, m);
    if (c->ph.cons_ec) launch_cons_ec(c->args(), c->stream);   // after the last node sweep, before dt
  } else {
    if (c->ph.csts) launch_csts_forward(c->args(), c->stream);   // PrepareRemap.cc:456, then the face velocities
    launch_remap_env(c->args(), sens, c->stream, m);
    if (c->ph.cons_ec) launch_cons_ec_env(c->args(), c->stream);   // after the last node sweep, before dt
  }
  return MHY_OK;
}
int launch_delta_t_(mhy_ctx* c) { launch_delta_t(c->args(), c->stream); return MHY_OK; }

int launch_cycle(mhy_ctx* c, int sens) {
  launch_velocity(c);
  launch_geometry(c);
  launch_remap_(c, sens);
  launch_delta_t_(c);
  return MHY_OK;
}

// The cycle graph of direction rotation s (captured once).
int cycle_graph(mhy_ctx* c, int s) {
  if (c->graph[s]) return MHY_OK;
  cudaGraph_t g = nullptr;
  MHY_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  launch_cycle(c, s);
  cudaError_t le = cudaGetLastError();
  cudaError_t ee = cudaStreamEndCapture(c->stream, &g);
  if (le != cudaSuccess || ee != cudaSuccess)
    return fail(MHY_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(le != cudaSuccess ? le : ee));
  cudaError_t ie = cudaGraphInstantiate(&c->graph[s], g, 0);
  cudaGraphDestroy(g);
  if (ie != cudaSuccess) { c->graph[s] = nullptr; return fail(MHY_ERR_CUDA, cudaGetErrorString(ie)); }
  return MHY_OK;
}

// Launches the entry-point work recorded so far, in order.
int flush(mhy_ctx* c) {
  if (!c || !c->pend) return MHY_OK;
  if (c->pend & 1) launch_velocity(c);
  if (c->pend & 2) launch_geometry(c);
  if (c->pend & 4) launch_remap_(c, c->pend_sens);
  c->pend = 0;
  MHY_CUDA(cudaGetLastError());
  return MHY_OK;
}

#define MHY_FLUSH(c)                  \
  do {                                \
    const int frc_ = flush(c);        \
    if (frc_ != MHY_OK) return frc_;  \
  } while (0)

int check_phase(mhy_ctx* c, int expected) {
  if (!c) return fail(MHY_ERR_ARG, "null context");
  if (!c->initialized) return fail(MHY_ERR_STATE, "mhy_hydro_start_init must come first");
  if (c->phase != expected) return fail(MHY_ERR_ORDER, "entry point called out of the time-loop order");
  return MHY_OK;
}

}  // namespace

extern "C" {

int mhy_save_values_at_n(mhy_ctx* c) {
  int rc = check_phase(c, PH_SAVE); if (rc) return rc;
  c->phase = PH_VELOCITY; return MHY_OK;
}
int mhy_update_velocity(mhy_ctx* c) {
  int rc = check_phase(c, PH_VELOCITY); if (rc) return rc;
  c->pend |= 1;
  c->phase = PH_BC; return MHY_OK;
}
int mhy_apply_boundary_condition(mhy_ctx* c) {
  int rc = check_phase(c, PH_BC); if (rc) return rc;
  c->phase = PH_POSITION; return MHY_OK;
}
int mhy_update_position(mhy_ctx* c) {
  int rc = check_phase(c, PH_POSITION); if (rc) return rc;
  c->phase = PH_GEOMETRY; return MHY_OK;
}
int mhy_compute_geometric_values(mhy_ctx* c) {
  int rc = check_phase(c, PH_GEOMETRY); if (rc) return rc;
  c->pend |= 2;
  c->phase = PH_DENSITY; return MHY_OK;
}
int mhy_update_density(mhy_ctx* c) {
  int rc = check_phase(c, PH_DENSITY); if (rc) return rc;
  c->phase = PH_VISCOSITY; return MHY_OK;
}
int mhy_compute_artificial_viscosity(mhy_ctx* c) {
  int rc = check_phase(c, PH_VISCOSITY); if (rc) return rc;
  c->phase = PH_ENERGY; return MHY_OK;
}
int mhy_update_energy_and_pressure(mhy_ctx* c) {
  int rc = check_phase(c, PH_ENERGY); if (rc) return rc;
  c->phase = PH_REMAP; return MHY_OK;
}
int mhy_remap(mhy_ctx* c) {
  int rc = check_phase(c, PH_REMAP); if (rc) return rc;
  c->pend |= 4;
  c->pend_sens = c->sens;
  c->sens = (c->sens + 1) % 3;
  c->phase = PH_DELTA_T; return MHY_OK;
}
int mhy_compute_delta_t(mhy_ctx* c) {
  int rc = check_phase(c, PH_DELTA_T); if (rc) return rc;
  DeviceScope on_dev(c->device);
  if (c->pend == 7) {                                // a whole cycle recorded: one graph launch
    rc = cycle_graph(c, c->pend_sens);
    if (rc != MHY_OK) return rc;
    MHY_CUDA(cudaGraphLaunch(c->graph[c->pend_sens], c->stream));
    c->pend = 0;
  } else {
    MHY_FLUSH(c);
    launch_delta_t_(c); MHY_CUDA(cudaGetLastError());
  }
  c->phase = PH_SAVE; return MHY_OK;
}

int mhy_step(mhy_ctx* c, int ncycles) {
  int rc = check_phase(c, PH_SAVE); if (rc) return rc;
  if (ncycles < 0) return fail(MHY_ERR_ARG, "ncycles < 0");
  DeviceScope on_dev(c->device);
  for (int it = 0; it < ncycles; ++it) {
    const int s = c->sens;
    rc = cycle_graph(c, s);
    if (rc != MHY_OK) return rc;
    MHY_CUDA(cudaGraphLaunch(c->graph[s], c->stream));
    c->sens = (s + 1) % 3;
  }
  return MHY_OK;
}

int mhy_synchronize(mhy_ctx* c) {
  if (!c) return fail(MHY_ERR_ARG, "null context");
  DeviceScope on_dev(c->device);
  MHY_FLUSH(c);
  MHY_CUDA(cudaStreamSynchronize(c->stream));
  Scalars h{};
  MHY_CUDA(cudaMemcpy(&h, c->S, sizeof(h), cudaMemcpyDeviceToHost));
  if (h.status & MHY_STATUS_DT_MIN) return fail(MHY_ERR_DT_MIN, "dt fell below deltat-min");
  if (h.status & (MHY_STATUS_NAN_DT | MHY_STATUS_ZERO_MASS)) return fail(MHY_ERR_NUMERIC, "numeric status raised on the device");
  return MHY_OK;
}

// ---- batches ---------------------------------------------------------------
}  // extern "C"

struct mhy_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<mhy_ctx*> inst;
  CycleArgs* d_descs = nullptr;
  int4* d_work[BK_COUNT] = {};
  int4* d_o3work[3] = {};                       // order 3: face work tables per direction
  int4* d_fwork = nullptr;                      // schema-csts: face work table (all directions)
  int order[BK_COUNT] = {};                     // work-table order of each kind (mhy_tuning.order)
  BatchPlan plan{};
  int sens = 0;
  bool initialized = false;
  cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};
  mhy_tuning tuning{};
};

namespace {

// Work table of one kernel kind: every block of every instance's grid, in
// one of three orders (mhy_tuning.order), for the given lines per block.
std::vector<int4> build_work(const std::vector<mhy_ctx*>& inst, int kind, int order, int lines) {
  const int n = (int)inst.size();
  std::vector<int> ids(n);
  std::iota(ids.begin(), ids.end(), 0);
  if (order == 1)
    std::stable_sort(ids.begin(), ids.end(), [&](int a, int b) { return inst[a]->dm.C > inst[b]->dm.C; });
  std::vector<std::vector<int4>> per(n);
  for (int i = 0; i < n; ++i) {
    int gx, gy, gz;
    batch_work_shape(inst[i]->dm, kind, lines, gx, gy, gz);
    if (gy < 0) {                               // linear chunks of consecutive items
      for (int x = 0; x < gx; ++x) per[i].push_back(make_int4(i, x, -1, 0));
      continue;
    }
    for (int z = 0; z < gz; ++z)
      for (int y = 0; y < gy; ++y)
        for (int x = 0; x < gx; ++x) per[i].push_back(make_int4(i, x, y, z));
  }
  std::vector<int4> w;
  if (order == 2) {                             // instances interleaved, 16 consecutive tiles at a time
    constexpr size_t kChunk = 16;
    for (size_t off = 0;; off += kChunk) {
      bool any = false;
      for (int i : ids)
        for (size_t t = off; t < std::min(off + kChunk, per[i].size()); ++t) { w.push_back(per[i][t]); any = true; }
      if (!any) break;
    }
  } else {
    for (int i : ids) w.insert(w.end(), per[i].begin(), per[i].end());
  }
  return w;
}

}  // namespace

extern "C" {

void mhy_batch_destroy(mhy_batch* b) {
  if (!b) return;
  DeviceScope on_dev(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (int s = 0; s < 3; ++s) if (b->graph[s]) cudaGraphExecDestroy(b->graph[s]);
  for (int k = 0; k < BK_COUNT; ++k) if (b->d_work[k]) cudaFree(b->d_work[k]);
  for (int d = 0; d < 3; ++d) if (b->d_o3work[d]) cudaFree(b->d_o3work[d]);
  if (b->d_fwork) cudaFree(b->d_fwork);
  if (b->d_descs) cudaFree(b->d_descs);
  for (mhy_ctx* c : b->inst) mhy_destroy(c);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

int mhy_batch_create(int n, const mhy_mesh_desc* meshes, const mhy_options* opts, int device, mhy_batch** out) {
  if (!meshes || !opts || !out || n <= 0) return fail(MHY_ERR_ARG, "null argument or empty batch");
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    if (opts[i].nb_env != opts[0].nb_env)
      return fail(MHY_ERR_UNSUPPORTED, "batched instances share one number of environments");
    if ((opts[i].schema_csts != 0) != (opts[0].schema_csts != 0))
      return fail(MHY_ERR_UNSUPPORTED, "batched instances: schema-csts in every instance or in none");
    if ((opts[i].ordre_projection == 3) != (opts[0].ordre_projection == 3))
      return fail(MHY_ERR_UNSUPPORTED, "batched instances: order 3 in every instance or in none");
    if ((opts[i].projection_limiteur_id >= 3) != (opts[0].projection_limiteur_id >= 3))
      return fail(MHY_ERR_UNSUPPORTED, "batched instances: the G limiters (ids 3..7) in every instance or in none");
    if ((opts[i].projection_pente_borne != 0) != (opts[0].projection_pente_borne != 0))
      return fail(MHY_ERR_UNSUPPORTED, "batched instances: pente-borne in every instance or in none");
    if (opts[i].precision != opts[0].precision) return fail(MHY_ERR_ARG, "batched instances share one precision");
  }
  mhy_batch* b = new mhy_batch();
  for (int i = 0; i < n; ++i) {
    mhy_ctx* c = nullptr;
    const int rc = mhy_create(&meshes[i], &opts[i], device, &c);
    if (rc != MHY_OK) { mhy_batch_destroy(b); return rc; }
    b->inst.push_back(c);
  }
  b->device = b->inst[0]->device;
  cudaError_t err = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (err != cudaSuccess) { mhy_batch_destroy(b); return fail(MHY_ERR_CUDA, cudaGetErrorString(err)); }
  // work tables: every block of every instance's grid, instance-major
  for (int k = 0; k < BK_COUNT; ++k) {
    // capacity for the largest table any tuning builds (8 lines per block)
    size_t cap = 0;
    for (int lw : kLineOptions) cap = std::max(cap, build_work(b->inst, k, 0, lw).size());
    const std::vector<int4> w = build_work(b->inst, k, 0, kLineWarps);
    err = cudaMalloc(&b->d_work[k], cap * sizeof(int4));
    if (err == cudaSuccess) err = cudaMemcpy(b->d_work[k], w.data(), w.size() * sizeof(int4), cudaMemcpyHostToDevice);
    if (err != cudaSuccess) { mhy_batch_destroy(b); return fail(MHY_ERR_OOM, cudaGetErrorString(err)); }
    b->plan.work[k] = b->d_work[k];
    b->plan.nwork[k] = (int)w.size();
  }
  err = cudaMalloc(&b->d_descs, n * sizeof(CycleArgs));
  if (err != cudaSuccess) { mhy_batch_destroy(b); return fail(MHY_ERR_OOM, cudaGetErrorString(err)); }
  b->plan.descs = b->d_descs;
  b->plan.ninst = n;
  b->plan.precision = opts[0].precision;
  b->plan.K = opts[0].nb_env;
  b->plan.gl = opts[0].projection_limiteur_id >= 3;   // the same in every instance (checked above)
  b->plan.pb = opts[0].projection_pente_borne != 0;
  b->plan.o3 = opts[0].ordre_projection == 3;
  b->plan.csts = opts[0].schema_csts != 0;
  if (b->plan.csts) {
    // face work table: (instance, chunk of 128 consecutive faces of all directions), instance-major
    std::vector<int4> w;
    for (int i = 0; i < n; ++i)
      for (long long x = 0; x < (b->inst[i]->dm.F + 127) / 128; ++x) w.push_back(make_int4(i, (int)x, 0, 0));
    err = cudaMalloc(&b->d_fwork, w.size() * sizeof(int4));
    if (err == cudaSuccess) err = cudaMemcpy(b->d_fwork, w.data(), w.size() * sizeof(int4), cudaMemcpyHostToDevice);
    if (err != cudaSuccess) { mhy_batch_destroy(b); return fail(MHY_ERR_OOM, cudaGetErrorString(err)); }
    b->plan.fwork = b->d_fwork;
    b->plan.nfwork = (int)w.size();
  }
  if (b->plan.o3) {
    // face work tables: (instance, chunk of 128 consecutive faces of direction d), instance-major
    for (int d = 0; d < 3; ++d) {
      std::vector<int4> w;
      for (int i = 0; i < n; ++i) {
        const Dims& dm = b->inst[i]->dm;
        const long long Fd = d == 0 ? dm.Fx : (d == 1 ? dm.Fy : dm.F - dm.Fx - dm.Fy);
        for (long long x = 0; x < (Fd + 127) / 128; ++x) w.push_back(make_int4(i, (int)x, 0, 0));
      }
      err = cudaMalloc(&b->d_o3work[d], w.size() * sizeof(int4));
      if (err == cudaSuccess) err = cudaMemcpy(b->d_o3work[d], w.data(), w.size() * sizeof(int4), cudaMemcpyHostToDevice);
      if (err != cudaSuccess) { mhy_batch_destroy(b); return fail(MHY_ERR_OOM, cudaGetErrorString(err)); }
      b->plan.o3work[d] = b->d_o3work[d];
      b->plan.o3nwork[d] = (int)w.size();
    }
  }
  for (int i = 0; i < n; ++i) b->plan.cons_ec |= opts[i].conservation_energie_totale;
  for (int k = 0; k < BK_TUNE_SLOTS; ++k) {
    b->plan.occ_pct[k] = 100;
    b->tuning.occupancy_pct[k] = 100;
    b->tuning.order[k] = 0;
    b->tuning.lines_per_block[k] = kLineWarps;
  }
  for (int k = 0; k < BK_COUNT; ++k) b->plan.lines[k] = kLineWarps;
  *out = b;
  return MHY_OK;
}

int mhy_batch_set_state(mhy_batch* b, int i, const mhy_state* st) {
  if (!b || i < 0 || i >= (int)b->inst.size()) return fail(MHY_ERR_ARG, "bad batch or instance index");
  return mhy_set_state(b->inst[i], st);
}

int mhy_batch_hydro_start_init(mhy_batch* b) {
  if (!b) return fail(MHY_ERR_ARG, "null batch");
  DeviceScope on_dev(b->device);
  std::vector<CycleArgs> d;
  for (mhy_ctx* c : b->inst) {
    const int rc = mhy_hydro_start_init(c);
    if (rc != MHY_OK) return rc;
    d.push_back(c->args());
  }
  MHY_CUDA(cudaMemcpy(b->d_descs, d.data(), d.size() * sizeof(CycleArgs), cudaMemcpyHostToDevice));
  b->initialized = true;
  return MHY_OK;
}

int mhy_batch_step(mhy_batch* b, int ncycles) {
  if (!b) return fail(MHY_ERR_ARG, "null batch");
  if (!b->initialized) return fail(MHY_ERR_STATE, "mhy_batch_hydro_start_init must come first");
  if (ncycles < 0) return fail(MHY_ERR_ARG, "ncycles < 0");
  DeviceScope on_dev(b->device);
  for (int it = 0; it < ncycles; ++it) {
    const int s = b->sens;
    if (!b->graph[s]) {
      cudaGraph_t g = nullptr;
      MHY_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      launch_batch_cycle(b->plan, s, b->stream);
      cudaError_t le = cudaGetLastError();
      cudaError_t ee = cudaStreamEndCapture(b->stream, &g);
      if (le != cudaSuccess || ee != cudaSuccess)
        return fail(MHY_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(le != cudaSuccess ? le : ee));
      cudaError_t ie = cudaGraphInstantiate(&b->graph[s], g, 0);
      cudaGraphDestroy(g);
      if (ie != cudaSuccess) { b->graph[s] = nullptr; return fail(MHY_ERR_CUDA, cudaGetErrorString(ie)); }
    }
    MHY_CUDA(cudaGraphLaunch(b->graph[s], b->stream));
    b->sens = (s + 1) % 3;
  }
  for (mhy_ctx* c : b->inst) c->sens = b->sens;
  return MHY_OK;
}

int mhy_batch_synchronize(mhy_batch* b) {
  if (!b) return fail(MHY_ERR_ARG, "null batch");
  DeviceScope on_dev(b->device);
  MHY_CUDA(cudaStreamSynchronize(b->stream));
  for (mhy_ctx* c : b->inst) {
    const int rc = mhy_synchronize(c);
    if (rc != MHY_OK) return rc;
  }
  return MHY_OK;
}

int mhy_batch_get_field(mhy_batch* b, int i, int field, void* dst, size_t bytes) {
  if (!b || i < 0 || i >= (int)b->inst.size()) return fail(MHY_ERR_ARG, "bad batch or instance index");
  MHY_CUDA(cudaStreamSynchronize(b->stream));
  return mhy_get_field(b->inst[i], field, dst, bytes);
}

int mhy_batch_get_dt(mhy_batch* b, int i, double* dt, double* dt_old) {
  if (!b || i < 0 || i >= (int)b->inst.size()) return fail(MHY_ERR_ARG, "bad batch or instance index");
  MHY_CUDA(cudaStreamSynchronize(b->stream));
  return mhy_get_dt(b->inst[i], dt, dt_old);
}

int mhy_batch_get_status(mhy_batch* b, int i, uint32_t* flags) {
  if (!b || i < 0 || i >= (int)b->inst.size()) return fail(MHY_ERR_ARG, "bad batch or instance index");
  MHY_CUDA(cudaStreamSynchronize(b->stream));
  return mhy_get_status(b->inst[i], flags);
}

int mhy_batch_get_totals(mhy_batch* b, int i, double* out) {
  if (!b || i < 0 || i >= (int)b->inst.size()) return fail(MHY_ERR_ARG, "bad batch or instance index");
  MHY_CUDA(cudaStreamSynchronize(b->stream));
  return mhy_get_totals(b->inst[i], out);
}

int mhy_batch_size(mhy_batch* b) { return b ? (int)b->inst.size() : 0; }

}  // extern "C"

namespace {

static_assert(MHY_TUNE_SLOTS == BK_TUNE_SLOTS, "tuning slots of the ABI and the batch plan");
constexpr int kTuneOrders = 3;
constexpr int kTunePcts[] = {100, 75, 50};
constexpr int kNP = sizeof(kTunePcts) / sizeof(kTunePcts[0]);
constexpr int kNL = sizeof(kLineOptions) / sizeof(kLineOptions[0]);
inline bool line_slot(int k) {
  return k == BK_CELLS_Y || k == BK_CELLS_Z || k == BK_NODES_Y || k == BK_NODES_Z;
}

// The line counts a batch's sweeps are built for: any on one environment; with
// several, 8 or 16 on the cell y/z sweeps and 8 on the node y/z sweeps; 8
// everywhere with the G limiters or pente-borne.
bool batch_tunable_lines(const mhy_batch* b, int k, int w) {
  if (!line_slot(k) || b->plan.gl || b->plan.pb || b->plan.o3) return w == kLineWarps;   // these sweeps keep 8 lines
  if (b->plan.K > 1) return w == kLineWarps || ((k == BK_CELLS_Y || k == BK_CELLS_Z) && w == 16);
  return true;
}

// The line counts a context's sweeps are built for: 8, 16 or 32 on the y/z
// sweeps of one environment at order 1 or 2 with the classic limiters; 8 or 16
// on the cell y/z sweeps of several environments (their node sweeps keep 8);
// 8 everywhere at order 3, with the G limiters or with pente-borne.
bool tunable_lines(const mhy_ctx* c, int k, int w) {
  if (!line_slot(k)) return w == kLineWarps;
  if (c->ph.ordre_projection == 3 || c->ph.limiteur_id >= 3 || c->ph.pb) return w == kLineWarps;
  if (c->K > 1) return w == kLineWarps || ((k == BK_CELLS_Y || k == BK_CELLS_Z) && w == 16);
  return true;
}

mhy_tuning default_tuning() {
  mhy_tuning t{};
  for (int k = 0; k < BK_TUNE_SLOTS; ++k) { t.order[k] = 0; t.occupancy_pct[k] = 100; t.lines_per_block[k] = kLineWarps; }
  return t;
}

int check_tuning(const mhy_tuning& t) {
  for (int k = 0; k < BK_TUNE_SLOTS; ++k) {
    if (t.order[k] < 0 || t.order[k] >= kTuneOrders) return fail(MHY_ERR_ARG, "tuning order must be 0, 1 or 2");
    if (t.occupancy_pct[k] < 1 || t.occupancy_pct[k] > 100) return fail(MHY_ERR_ARG, "occupancy_pct must be 1..100");
    const int w = t.lines_per_block[k];
    if (w != 8 && w != 16 && w != 32) return fail(MHY_ERR_ARG, "lines_per_block must be 8, 16 or 32");
    if (w != kLineWarps && !line_slot(k)) return fail(MHY_ERR_ARG, "lines_per_block applies to the y/z sweeps only");
  }
  return MHY_OK;
}

// The tuning of a batch: work tables (order and shape) and grid sizes; the
// cycle graphs are re-captured at the next step.
int apply_tuning(mhy_batch* b, const mhy_tuning& t) {
  for (int k = 0; k < BK_COUNT; ++k) {
    if (t.order[k] == b->order[k] && t.lines_per_block[k] == b->plan.lines[k]) continue;
    const std::vector<int4> w = build_work(b->inst, k, t.order[k], t.lines_per_block[k]);
    MHY_CUDA(cudaMemcpyAsync(b->d_work[k], w.data(), w.size() * sizeof(int4), cudaMemcpyHostToDevice, b->stream));
    MHY_CUDA(cudaStreamSynchronize(b->stream));                 // w is a host temporary
    b->order[k] = t.order[k];
    b->plan.lines[k] = t.lines_per_block[k];
    b->plan.nwork[k] = (int)w.size();
  }
  for (int k = 0; k < BK_TUNE_SLOTS; ++k) b->plan.occ_pct[k] = t.occupancy_pct[k];
  for (int s = 0; s < 3; ++s)
    if (b->graph[s]) { cudaGraphExecDestroy(b->graph[s]); b->graph[s] = nullptr; }
  return MHY_OK;
}

// The tuning of a context: lines per block; the graphs are re-captured.
int apply_tuning(mhy_ctx* c, const mhy_tuning& t) {
  for (int k = 0; k < BK_COUNT; ++k) c->lines[k] = t.lines_per_block[k];
  for (int s = 0; s < 3; ++s)
    if (c->graph[s]) { cudaGraphExecDestroy(c->graph[s]); c->graph[s] = nullptr; }
  return MHY_OK;
}

// Cache key: the precision, the number of environments, the options that
// change which kernels a cycle launches or what they cost (schema-csts adds
// kernels and sweeps on the Lagrangian coordinates; Newton, the EOS kinds,
// the order, the limiter and the length mode change the work per item) and
// the sorted mesh sizes (with each instance's own options in a batch).
std::string tune_key(const std::vector<mhy_ctx*>& inst, const char* kind) {
  auto opts = [](const mhy_ctx* c) {
    std::string s = "c" + std::to_string(c->ph.csts) + "n" + std::to_string(c->ph.with_newton) + "o" +
                    std::to_string(c->ph.ordre_projection) + "l" + std::to_string(c->ph.limiteur_id) + "L" +
                    std::to_string(c->ph.lc_mode) + "e";
    for (int k = 0; k < c->K; ++k) s += std::to_string(c->env.eos[k]);
    return s;
  };
  std::vector<std::string> sz;
  for (const mhy_ctx* c : inst)
    sz.push_back(std::to_string(c->dm.nx) + "x" + std::to_string(c->dm.ny) + "x" + std::to_string(c->dm.nz) + "/" +
                 opts(c));
  std::sort(sz.begin(), sz.end());
  std::string key = std::string(kind) + ":p" + std::to_string(inst[0]->ph.precision) + ":k" +
                    std::to_string(inst[0]->K);
  for (const auto& x : sz) key += ":" + x;
  return key;
}

std::mutex g_tune_mu;
std::map<std::string, mhy_tuning> g_tune_cache;

// Device snapshot of the state (every allocation) of some contexts.
struct Snapshot {
  char* buf = nullptr;
  int save(const std::vector<mhy_ctx*>& inst, cudaStream_t s) {
    size_t total = 0;
    for (const mhy_ctx* c : inst)
      for (size_t x : c->alloc_bytes) total += (x + 255) & ~size_t(255);
    if (cudaMalloc(&buf, total) != cudaSuccess) {
      cudaGetLastError();
      buf = nullptr;
      return fail(MHY_ERR_OOM, "autotune: no device memory for the state snapshot");
    }
    return copy(inst, s, true);
  }
  int copy(const std::vector<mhy_ctx*>& inst, cudaStream_t s, bool to_snap) {
    size_t off = 0;
    for (const mhy_ctx* c : inst)
      for (size_t a = 0; a < c->allocs.size(); ++a) {
        char* dev = static_cast<char*>(c->allocs[a]);
        const cudaError_t e = cudaMemcpyAsync(to_snap ? buf + off : dev, to_snap ? dev : buf + off, c->alloc_bytes[a],
                                              cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return fail(MHY_ERR_CUDA, cudaGetErrorString(e));
        off += (c->alloc_bytes[a] + 255) & ~size_t(255);
      }
    const cudaError_t e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? MHY_OK : fail(MHY_ERR_CUDA, cudaGetErrorString(e));
  }
  ~Snapshot() { if (buf) cudaFree(buf); }
};

// Per-slot GPU time of `cycles` eager cycles (after one untimed cycle);
// launch(marks) enqueues one cycle and advances the direction rotation.
template <class Launch>
int time_cycles(cudaStream_t stream, int cycles, Launch&& launch, double ms[BK_TUNE_SLOTS]) {
  for (int k = 0; k < BK_TUNE_SLOTS; ++k) ms[k] = 0.;
  KernelMarks m{};
  cudaEvent_t start = nullptr;
  if (cudaEventCreate(&start) != cudaSuccess) return fail(MHY_ERR_CUDA, "event");
  int made = 0;
  for (; made < KernelMarks::kMax; ++made)
    if (cudaEventCreate(&m.ev[made]) != cudaSuccess) break;
  int rc = made == KernelMarks::kMax ? MHY_OK : fail(MHY_ERR_CUDA, "event");
  if (rc == MHY_OK) launch(nullptr);
  for (int c = 0; c < cycles && rc == MHY_OK; ++c) {
    m.n = 0;
    cudaEventRecord(start, stream);
    launch(&m);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(stream) != cudaSuccess) {
      rc = fail(MHY_ERR_CUDA, "autotune cycle failed");
      break;
    }
    cudaEvent_t prev = start;
    for (int i = 0; i < m.n; ++i) {
      float t = 0.f;
      cudaEventElapsedTime(&t, prev, m.ev[i]);
      ms[m.kind[i]] += t;
      prev = m.ev[i];
    }
  }
  for (int i = 0; i < made; ++i) cudaEventDestroy(m.ev[i]);
  cudaEventDestroy(start);
  if (rc == MHY_OK)
    for (int k = 0; k < BK_TUNE_SLOTS; ++k) ms[k] /= cycles;
  return rc;
}

// Best setting per slot: the trials are grouped by the slot's own setting
// (order, occupancy, lines) and each group's times averaged, since trials
// that differ only in other slots time the same kernel; trial 0 is the
// default, and another setting must be 2 % faster.  allowed(k, i) restricts
// the trials of slot k.
template <class Allowed>
void pick(const std::vector<mhy_tuning>& tr, const std::vector<std::array<double, BK_TUNE_SLOTS>>& ms, Allowed&& allowed,
          mhy_tuning& best) {
  for (int k = 0; k < BK_TUNE_SLOTS; ++k) {
    auto same = [&](int a, int b) {
      return tr[a].order[k] == tr[b].order[k] && tr[a].occupancy_pct[k] == tr[b].occupancy_pct[k] &&
             tr[a].lines_per_block[k] == tr[b].lines_per_block[k];
    };
    auto mean = [&](int a) {
      double sum = 0.;
      int n = 0;
      for (int i = 0; i < (int)tr.size(); ++i)
        if (allowed(k, i) && same(i, a)) { sum += ms[i][k]; ++n; }
      return n ? sum / n : ms[a][k];
    };
    int bi = -1;
    double bt = 0.;
    for (int i = 0; i < (int)tr.size(); ++i) {
      if (!allowed(k, i)) continue;
      bool first = true;                       // first trial of its group
      for (int j = 0; j < i && first; ++j) first = !(allowed(k, j) && same(j, i));
      if (!first) continue;
      const double t = mean(i);
      if (bi < 0 || t < 0.98 * bt) { bi = i; bt = t; }
    }
    if (bi < 0) { bi = 0; bt = ms[0][k]; }
    best.order[k] = tr[bi].order[k];
    best.occupancy_pct[k] = tr[bi].occupancy_pct[k];
    best.lines_per_block[k] = tr[bi].lines_per_block[k];
    best.ms_default[k] = mean(0);
    best.ms_tuned[k] = bt;
  }
  best.trials = (int)tr.size();
  best.from_cache = 0;
}

}  // namespace

extern "C" {

int mhy_get_tuning(mhy_ctx* c, mhy_tuning* out) {
  if (!c || !out) return fail(MHY_ERR_ARG, "null argument");
  *out = c->tuning;
  return MHY_OK;
}

int mhy_set_tuning(mhy_ctx* c, const mhy_tuning* t) {
  if (!c || !t) return fail(MHY_ERR_ARG, "null argument");
  DeviceScope on_dev(c->device);
  MHY_FLUSH(c);
  mhy_tuning u = *t;
  for (int k = 0; k < BK_TUNE_SLOTS; ++k) { u.order[k] = 0; u.occupancy_pct[k] = 100; }
  int rc = check_tuning(u);
  if (rc != MHY_OK) return rc;
  for (int k = 0; k < BK_TUNE_SLOTS; ++k)
    if (u.lines_per_block[k] != kLineWarps && !tunable_lines(c, k, u.lines_per_block[k]))
      return fail(MHY_ERR_UNSUPPORTED,
                  "lines_per_block: 8 or 16 on the cell y/z sweeps of several environments; 8 with order 3, "
                  "the G limiters or pente-borne");
  apply_tuning(c, u);
  c->tuning = u;
  return MHY_OK;
}

int mhy_autotune(mhy_ctx* c, int cycles, mhy_tuning* out) {
  if (!c) return fail(MHY_ERR_ARG, "null context");
  DeviceScope on_dev(c->device);
  MHY_FLUSH(c);
  if (!c->initialized) return fail(MHY_ERR_STATE, "mhy_hydro_start_init must come first");
  if (c->phase != PH_SAVE) return fail(MHY_ERR_ORDER, "autotune runs between cycles");
  if (cycles < 1 || cycles > 20) return fail(MHY_ERR_ARG, "cycles must be 1..20");
  if (c->ph.ordre_projection == 3 || c->ph.limiteur_id >= 3 || c->ph.pb) {   // these sweeps keep 8 lines
    c->tuning = default_tuning();
    if (out) *out = c->tuning;
    return MHY_OK;
  }
  const std::vector<mhy_ctx*> inst{c};
  const std::string key = tune_key(inst, "ctx");
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      mhy_tuning t = it->second;
      t.from_cache = 1;
      apply_tuning(c, t);
      c->tuning = t;
      if (out) *out = t;
      return MHY_OK;
    }
  }
  Snapshot snap;
  int rc = snap.save(inst, c->stream);
  if (rc != MHY_OK) return rc;
  const int sens0 = c->sens;
  std::vector<mhy_tuning> tr;
  for (int l = 0; l < kNL; ++l) {
    mhy_tuning t = default_tuning();
    bool any = false;
    for (int k = 0; k < BK_TUNE_SLOTS; ++k)
      if (line_slot(k) && tunable_lines(c, k, kLineOptions[l])) { t.lines_per_block[k] = kLineOptions[l]; any = true; }
    if (l == 0 || any) tr.push_back(t);
  }
  std::vector<std::array<double, BK_TUNE_SLOTS>> ms(tr.size());
  for (size_t i = 0; i < tr.size() && rc == MHY_OK; ++i) {
    apply_tuning(c, tr[i]);
    rc = time_cycles(c->stream, cycles, [&](KernelMarks* m) {
      launch_velocity(c);
      mark(m, BK_LNODES, c->stream);
      launch_geometry(c);
      mark(m, BK_LCELLS, c->stream);
      launch_remap_(c, c->sens, m);
      launch_delta_t_(c);
      mark(m, BK_DT_FINISH, c->stream);
      c->sens = (c->sens + 1) % 3;
    }, ms[i].data());
  }
  const int rr = snap.copy(inst, c->stream, false);
  c->sens = sens0;
  if (rc == MHY_OK) rc = rr;
  if (rc != MHY_OK) {
    apply_tuning(c, c->tuning);
    return rc;
  }
  mhy_tuning best = default_tuning();
  pick(tr, ms, [](int, int) { return true; }, best);
  apply_tuning(c, best);
  c->tuning = best;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = best;
  }
  if (out) *out = best;
  return MHY_OK;
}

int mhy_batch_get_tuning(mhy_batch* b, mhy_tuning* out) {
  if (!b || !out) return fail(MHY_ERR_ARG, "null argument");
  *out = b->tuning;
  return MHY_OK;
}

int mhy_batch_set_tuning(mhy_batch* b, const mhy_tuning* t) {
  if (!b || !t) return fail(MHY_ERR_ARG, "null argument");
  mhy_tuning u = *t;
  u.order[BK_DT_MIN] = u.order[BK_LCELLS];
  u.order[BK_DT_FINISH] = 0;
  u.occupancy_pct[BK_DT_FINISH] = 100;
  DeviceScope on_dev(b->device);
  int rc = check_tuning(u);
  for (int k = 0; k < BK_TUNE_SLOTS && rc == MHY_OK; ++k)
    if (!batch_tunable_lines(b, k, u.lines_per_block[k]))
      rc = fail(MHY_ERR_ARG, "lines_per_block: 8 or 16 on the cell y/z sweeps and 8 on the node y/z sweeps of a batch "
                             "with several environments");
  if (rc == MHY_OK) rc = apply_tuning(b, u);
  if (rc == MHY_OK) b->tuning = u;
  return rc;
}

int mhy_batch_autotune(mhy_batch* b, int cycles, mhy_tuning* out) {
  if (!b) return fail(MHY_ERR_ARG, "null batch");
  if (!b->initialized) return fail(MHY_ERR_STATE, "mhy_batch_hydro_start_init must come first");
  if (cycles < 1 || cycles > 20) return fail(MHY_ERR_ARG, "cycles must be 1..20");
  DeviceScope on_dev(b->device);
  const std::string key = tune_key(b->inst, "batch");
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      mhy_tuning t = it->second;
      t.from_cache = 1;
      int rc = apply_tuning(b, t);
      if (rc != MHY_OK) return rc;
      b->tuning = t;
      if (out) *out = t;
      return MHY_OK;
    }
  }
  MHY_CUDA(cudaStreamSynchronize(b->stream));
  Snapshot snap;
  int rc = snap.save(b->inst, b->stream);
  if (rc != MHY_OK) return rc;
  const int sens0 = b->sens;
  const mhy_tuning before = b->tuning;
  // trials: every (order, occupancy, lines) setting on every slot at once
  std::vector<mhy_tuning> tr;
  for (int o = 0; o < kTuneOrders; ++o)
    for (int q = 0; q < kNP; ++q)
      for (int l = 0; l < kNL; ++l) {
        mhy_tuning t = default_tuning();
        for (int k = 0; k < BK_TUNE_SLOTS; ++k) {
          if (k != BK_DT_FINISH) { t.order[k] = o; t.occupancy_pct[k] = kTunePcts[q]; }
          if (line_slot(k)) t.lines_per_block[k] = batch_tunable_lines(b, k, kLineOptions[l]) ? kLineOptions[l] : kLineWarps;
        }
        tr.push_back(t);
      }
  std::vector<std::array<double, BK_TUNE_SLOTS>> ms(tr.size());
  for (size_t i = 0; i < tr.size() && rc == MHY_OK; ++i) {
    rc = apply_tuning(b, tr[i]);
    if (rc == MHY_OK)
      rc = time_cycles(b->stream, cycles, [&](KernelMarks* m) {
        launch_batch_cycle(b->plan, b->sens, b->stream, m);
        b->sens = (b->sens + 1) % 3;
      }, ms[i].data());
  }
  const int rr = snap.copy(b->inst, b->stream, false);
  b->sens = sens0;
  for (mhy_ctx* c : b->inst) c->sens = b->sens;
  if (rc == MHY_OK) rc = rr;
  if (rc != MHY_OK) {
    apply_tuning(b, before);
    return rc;
  }
  mhy_tuning best = default_tuning();
  // slots 0-7 pick freely; the dt reduction only among the trials that ran
  // slot 1's chosen order (it walks that table); the dt finish keeps the default
  pick(tr, ms, [&](int k, int i) {
    if (k == BK_DT_FINISH) return i == 0;
    if (k == BK_DT_MIN) return tr[i].order[BK_LCELLS] == tr[0].order[BK_LCELLS];
    return true;
  }, best);
  {
    // the dt reduction walks slot 1's table: among the trials with slot 1's
    // chosen order, its best occupancy
    mhy_tuning dt = default_tuning();
    const int o1 = best.order[BK_LCELLS];
    pick(tr, ms, [&](int k, int i) { return k != BK_DT_MIN || tr[i].order[BK_LCELLS] == o1; }, dt);
    best.order[BK_DT_MIN] = o1;
    best.occupancy_pct[BK_DT_MIN] = dt.occupancy_pct[BK_DT_MIN];
    best.ms_tuned[BK_DT_MIN] = dt.ms_tuned[BK_DT_MIN];
  }
  rc = apply_tuning(b, best);
  if (rc != MHY_OK) return rc;
  b->tuning = best;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = best;
  }
  if (out) *out = best;
  return MHY_OK;
}
int mhy_batch_kernels_per_cycle(mhy_batch* b) {
  // several environments: the end-of-remap kernel; conservation-energie-totale: its kernel
  // order 3: the face kernel of each direction; schema-csts: the forward step and the face velocities
  return b ? kKernelsPerCycleBatch + (b->plan.K > 1 ? 1 : 0) + (b->plan.cons_ec ? 1 : 0) + (b->plan.o3 ? 3 : 0) +
                 (b->plan.csts ? 2 : 0)
           : 0;
}
void* mhy_batch_get_stream(mhy_batch* b) { return b ? (void*)b->stream : nullptr; }

int mhy_get_field(mhy_ctx* c, int field, void* dst, size_t bytes) {
  if (!c || !dst) return fail(MHY_ERR_ARG, "null argument");
  DeviceScope on_dev(c->device);
  MHY_FLUSH(c);
  const long long C = c->dm.C, N = c->dm.N;
  const double* src = nullptr;
  bool vec = false;
  long long n = C;
  switch (field) {
    case MHY_FIELD_DENSITY: src = c->rho; break;
    case MHY_FIELD_INTERNAL_ENERGY: src = c->e; break;
    case MHY_FIELD_PRESSURE: src = c->p; break;
    case MHY_FIELD_SOUND_SPEED: src = c->cs; break;
    case MHY_FIELD_PSEUDO_VISCOSITY: src = c->q; break;
    case MHY_FIELD_CELL_VOLUME: src = c->Ve; break;
    case MHY_FIELD_CELL_MASS: src = c->mass; break;
    case MHY_FIELD_CARACTERISTIC_LENGTH: src = c->L; break;
    case MHY_FIELD_VELOCITY: src = c->v; vec = true; n = N; break;
    case MHY_FIELD_NODE_MASS: src = c->nm; n = N; break;
    case MHY_FIELD_NODE_COORD: src = c->x0; vec = true; n = N; break;   // x0 + dt * v_half, MahycoModule.cc:899-901
    default: return fail(MHY_ERR_ARG, "unknown field");
  }
  const size_t need = (size_t)n * (vec ? 3 : 1) * sizeof(double);
  if (bytes < need) return fail(MHY_ERR_ARG, "destination too small");
  if (vec) {
    // xyz interleaving on the device, into the dual remap variables (5N
    // doubles), which hold nothing between entry-point calls
    const bool coord = field == MHY_FIELD_NODE_COORD;
    k_aos3<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(n, src, coord ? c->vh : nullptr, c->S, c->ud[0]);
    MHY_CUDA(cudaGetLastError());
    src = c->ud[0];
  }
  if (c->d_cell_index) {
    // into the caller's numbering, in the other dual remap buffer (5N doubles)
    const int32_t* idx = n == N ? c->d_node_index : c->d_cell_index;
    k_gather_index<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(n, vec ? 3 : 1, idx, src, c->ud[1]);
    MHY_CUDA(cudaGetLastError());
    src = c->ud[1];
  }
  MHY_CUDA(cudaMemcpyAsync(dst, src, need, cudaMemcpyDeviceToHost, c->stream));
  MHY_CUDA(cudaStreamSynchronize(c->stream));
  return MHY_OK;
}

// ---- restart dump ------------------------------------------------------------
}  // extern "C"

namespace {

// Layout of a restart dump: CkptHeader, nfields CkptField records, then the
// arrays (each at its record's offset from the start of the dump, 64-byte
// aligned).  Field names are the reference's variable names (Mahyco.axl).
struct CkptHeader {
  char magic[8];
  int32_t version, nx, ny, nz, nenv, precision, nfields, sens;
  double dt, old_dt, time;
  int64_t iteration;
  uint32_t status, pad;
  uint64_t options_hash;   // options_hash() of the context that saved the dump
};
constexpr int32_t kCkptVersion = 2;

// FNV-1a hash of every option that changes the computed state (all of
// mhy_options but deltat-init, whose effect the dump's dt replaces): a dump
// only loads into a context that will continue with the same physics.
uint64_t options_hash(const mhy_options& o) {
  uint64_t h = 0xcbf29ce484222325ull;
  auto add = [&](const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; ++i) { h ^= b[i]; h *= 0x100000001b3ull; }
  };
  auto d = [&](double x) { add(&x, sizeof(x)); };
  auto i = [&](int32_t x) { add(&x, sizeof(x)); };
  d(o.cfl); d(o.threshold); d(o.deltat_min); d(o.deltat_max); d(o.final_time);
  i(o.longueur_caracteristique); i(o.pseudo_centree); i(o.ordre_projection); i(o.projection_limiteur_id);
  i(o.nb_bc);
  for (int b = 0; b < o.nb_bc && b < MHY_MAX_BC; ++b) { i(o.bc[b].surface); i(o.bc[b].type); d(o.bc[b].value); }
  i(o.nb_env);
  for (int k = 0; k < o.nb_env && k < MHY_MAX_ENV; ++k) { d(o.adiabatic_cst[k]); i(o.eos[k]); d(o.limit_tension[k]); }
  i(o.precision); i(o.with_newton); i(o.schema_csts); i(o.projection_pente_borne); i(o.pente_borne_debar_fix);
  i(o.pente_borne_mixte); i(o.limiteur_pure_id); i(o.conservation_energie_totale);
  return h;
}
struct CkptField {
  char name[40];
  int32_t dtype;        // 0 double, 1 float, 2 uint32
  int32_t pad;
  int64_t count, offset;
};
constexpr char kCkptMagic[8] = {'M', 'H', 'Y', 'C', 'K', 'P', 'T', '1'};

struct CkField { const char* name; void* dev; int dtype; long long count; };

// The state a cycle starts from: everything a kernel reads before writing it.
std::vector<CkField> ckpt_fields(mhy_ctx* c) {
  const long long C = c->dm.C, N = c->dm.N;
  const int K = c->K;
  std::vector<CkField> f = {
      {"Density", c->rho, 0, C}, {"InternalEnergy", c->e, 0, C}, {"Pressure", c->p, 0, C},
      {"SoundSpeed", c->cs, 0, C}, {"PseudoViscosity", c->q, 0, C}, {"CellMass", c->mass, 0, C},
      {"Velocity", c->v, 0, 3 * N}, {"NodeMass", c->nm, 0, N}, {"DualGradPhi", c->Gd, 0, 3 * N}};
  if (c->cqs32) f.push_back({"CellCQS", c->cqs32, 1, 24 * C});
  else f.push_back({"CellCQS", c->cqs, 0, 24 * C});
  if (K > 1) {
    const EnvState& ev = c->env;
    f.push_back({"EnvMask", ev.mask, 2, C});
    f.push_back({"FracVol.env", ev.f, 0, K * C}); f.push_back({"MassFraction.env", ev.x, 0, K * C});
    f.push_back({"Density.env", ev.rho, 0, K * C}); f.push_back({"InternalEnergy.env", ev.e, 0, K * C});
    f.push_back({"Pressure.env", ev.p, 0, K * C}); f.push_back({"SoundSpeed.env", ev.cs, 0, K * C});
    f.push_back({"PseudoViscosity.env", ev.q, 0, K * C}); f.push_back({"CellMass.env", ev.m, 0, K * C});
    f.push_back({"FracVol", ev.fg, 0, C}); f.push_back({"MassFraction", ev.xg, 0, C});
    if (c->fd.est) f.push_back({"EstMixtePure", c->fd.est, 2, C});
    if (c->fd.pbphi) f.push_back({"PenteBornePhi", c->fd.pbphi, 0, (3 * K + 1) * C});
  }
  return f;
}

size_t ckpt_elem(int dtype) { return dtype == 0 ? 8 : 4; }

size_t ckpt_layout(const std::vector<CkField>& f, std::vector<int64_t>& offsets) {
  size_t off = sizeof(CkptHeader) + f.size() * sizeof(CkptField);
  offsets.clear();
  for (const CkField& x : f) {
    off = (off + 63) & ~size_t(63);
    offsets.push_back((int64_t)off);
    off += (size_t)x.count * ckpt_elem(x.dtype);
  }
  return off;
}

}  // namespace

extern "C" {

int mhy_checkpoint_size(mhy_ctx* c, size_t* bytes) {
  if (!c || !bytes) return fail(MHY_ERR_ARG, "null argument");
  DeviceScope on_dev(c->device);
  MHY_FLUSH(c);
  std::vector<int64_t> off;
  *bytes = ckpt_layout(ckpt_fields(c), off);
  return MHY_OK;
}

int mhy_checkpoint_save(mhy_ctx* c, void* dst, size_t bytes) {
  if (!c || !dst) return fail(MHY_ERR_ARG, "null argument");
  DeviceScope on_dev(c->device);
  MHY_FLUSH(c);
  if (!c->initialized) return fail(MHY_ERR_STATE, "mhy_hydro_start_init must come first");
  if (c->phase != PH_SAVE) return fail(MHY_ERR_ORDER, "a restart dump is taken between cycles");
  const std::vector<CkField> f = ckpt_fields(c);
  std::vector<int64_t> off;
  const size_t need = ckpt_layout(f, off);
  if (bytes < need) return fail(MHY_ERR_ARG, "destination too small (mhy_checkpoint_size)");
  MHY_CUDA(cudaStreamSynchronize(c->stream));
  Scalars h{};
  MHY_CUDA(cudaMemcpy(&h, c->S, sizeof(h), cudaMemcpyDeviceToHost));
  char* base = static_cast<char*>(dst);
  std::memset(base, 0, sizeof(CkptHeader) + f.size() * sizeof(CkptField));
  CkptHeader hd{};
  std::memcpy(hd.magic, kCkptMagic, 8);
  hd.version = kCkptVersion; hd.nx = c->dm.nx; hd.ny = c->dm.ny; hd.nz = c->dm.nz; hd.nenv = c->K;
  hd.precision = c->ph.precision; hd.nfields = (int32_t)f.size(); hd.sens = c->sens;
  hd.options_hash = options_hash(c->opt);
  hd.dt = h.dt; hd.old_dt = h.old_dt; hd.time = h.time; hd.iteration = h.iteration; hd.status = h.status;
  std::memcpy(base, &hd, sizeof(hd));
  for (size_t i = 0; i < f.size(); ++i) {
    CkptField r{};
    std::strncpy(r.name, f[i].name, sizeof(r.name) - 1);
    r.dtype = f[i].dtype; r.count = f[i].count; r.offset = off[i];
    std::memcpy(base + sizeof(CkptHeader) + i * sizeof(CkptField), &r, sizeof(r));
    MHY_CUDA(cudaMemcpy(base + off[i], f[i].dev, (size_t)f[i].count * ckpt_elem(f[i].dtype), cudaMemcpyDeviceToHost));
  }
  return MHY_OK;
}

int mhy_checkpoint_load(mhy_ctx* c, const void* src, size_t bytes) {
  if (!c || !src) return fail(MHY_ERR_ARG, "null argument");
  DeviceScope on_dev(c->device);
  MHY_FLUSH(c);
  if (bytes < sizeof(CkptHeader)) return fail(MHY_ERR_ARG, "not a restart dump");
  const char* base = static_cast<const char*>(src);
  CkptHeader hd;
  std::memcpy(&hd, base, sizeof(hd));
  if (std::memcmp(hd.magic, kCkptMagic, 8) != 0 || hd.version != kCkptVersion)
    return fail(MHY_ERR_ARG, "not a restart dump");
  if (hd.nx != c->dm.nx || hd.ny != c->dm.ny || hd.nz != c->dm.nz || hd.nenv != c->K ||
      hd.precision != c->ph.precision)
    return fail(MHY_ERR_ARG, "restart dump of another mesh, environment count or precision");
  if (hd.options_hash != options_hash(c->opt))
    return fail(MHY_ERR_ARG, "restart dump taken with other options (EOS, gamma, limiter, order, schemes, BCs, ...)");
  if (hd.sens < 0 || hd.sens > 2) return fail(MHY_ERR_ARG, "corrupt restart dump");
  const std::vector<CkField> f = ckpt_fields(c);
  if (hd.nfields != (int32_t)f.size() || bytes < sizeof(CkptHeader) + f.size() * sizeof(CkptField))
    return fail(MHY_ERR_ARG, "restart dump field list does not match this context");
  // geometry of t = 0 from the mesh, then the dumped state over it (the
  // copies below are synchronous on another stream: wait for the geometry)
  const int rc = init_geometry(c);
  if (rc != MHY_OK) return rc;
  MHY_CUDA(cudaStreamSynchronize(c->stream));
  for (size_t i = 0; i < f.size(); ++i) {
    CkptField r;
    std::memcpy(&r, base + sizeof(CkptHeader) + i * sizeof(CkptField), sizeof(r));
    r.name[sizeof(r.name) - 1] = 0;
    const size_t nb = (size_t)f[i].count * ckpt_elem(f[i].dtype);
    if (std::strcmp(r.name, f[i].name) != 0 || r.dtype != f[i].dtype || r.count != f[i].count || r.offset < 0 ||
        (size_t)r.offset + nb > bytes)
      return fail(MHY_ERR_ARG, std::string("restart dump field mismatch: ") + f[i].name);
    MHY_CUDA(cudaMemcpy(f[i].dev, base + r.offset, nb, cudaMemcpyHostToDevice));
  }
  Scalars h{};
  h.dt = hd.dt; h.old_dt = hd.old_dt; h.inv_dt = 1.0 / hd.dt; h.time = hd.time;
  h.min_bits = 0x7fefffffffffffffull; h.status = hd.status; h.iteration = hd.iteration;
  MHY_CUDA(cudaMemcpy(c->S, &h, sizeof(h), cudaMemcpyHostToDevice));
  c->sens = hd.sens;
  c->state_set = true;
  c->initialized = true;
  c->phase = PH_SAVE;
  return MHY_OK;
}

int mhy_get_env_mask(mhy_ctx* c, uint32_t* dst, size_t bytes) {
  if (!c || !dst) return fail(MHY_ERR_ARG, "null argument");
  DeviceScope on_dev(c->device);
  MHY_FLUSH(c);
  const long long C = c->dm.C;
  if (bytes < (size_t)C * sizeof(uint32_t)) return fail(MHY_ERR_ARG, "destination too small");
  MHY_CUDA(cudaStreamSynchronize(c->stream));
  if (c->K == 1) {
    for (long long i = 0; i < C; ++i) dst[i] = 1u;
    return MHY_OK;
  }
  MHY_CUDA(cudaMemcpy(dst, c->env.mask, C * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  if (!c->cell_index.empty()) {
    const std::vector<uint32_t> t(dst, dst + C);
    for (long long u = 0; u < C; ++u) dst[u] = t[c->cell_index[u]];
  }
  return MHY_OK;
}

int mhy_get_env_field(mhy_ctx* c, int field, int env, void* dst, size_t bytes) {
  if (!c || !dst) return fail(MHY_ERR_ARG, "null argument");
  DeviceScope on_dev(c->device);
  MHY_FLUSH(c);
  if (env < 0 || env >= c->K) return fail(MHY_ERR_ARG, "environment index out of range");
  const long long C = c->dm.C;
  if (bytes < (size_t)C * sizeof(double)) return fail(MHY_ERR_ARG, "destination too small");
  const EnvState& ev = c->env;
  const double *glob = nullptr, *part = nullptr;
  switch (field) {
    case MHY_ENV_FRACVOL: glob = ev.fg; part = ev.f; break;
    case MHY_ENV_DENSITY: glob = c->rho; part = ev.rho; break;
    case MHY_ENV_INTERNAL_ENERGY: glob = c->e; part = ev.e; break;
    case MHY_ENV_PRESSURE: glob = c->p; part = ev.p; break;
    case MHY_ENV_SOUND_SPEED: glob = c->cs; part = ev.cs; break;
    case MHY_ENV_MASS_FRACTION: glob = ev.xg; part = ev.x; break;
    case MHY_ENV_CELL_MASS: glob = c->mass; part = ev.m; break;
    default: return fail(MHY_ERR_ARG, "unknown environment field");
  }
  MHY_CUDA(cudaStreamSynchronize(c->stream));
  double* o = static_cast<double*>(dst);
  auto to_caller = [&]() {                         // the structured numbering -> the caller's
    if (c->cell_index.empty()) return;
    const std::vector<double> t(o, o + C);
    for (long long u = 0; u < C; ++u) o[u] = t[c->cell_index[u]];
  };
  if (c->K == 1) {
    if (field == MHY_ENV_FRACVOL || field == MHY_ENV_MASS_FRACTION) {
      for (long long i = 0; i < C; ++i) o[i] = 1.;
      return MHY_OK;
    }
    MHY_CUDA(cudaMemcpy(o, glob, C * sizeof(double), cudaMemcpyDeviceToHost));
    to_caller();
    return MHY_OK;
  }
  std::vector<uint32_t> mask(C);
  std::vector<double> g(C), pt(C);
  MHY_CUDA(cudaMemcpy(mask.data(), ev.mask, C * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  MHY_CUDA(cudaMemcpy(g.data(), glob, C * sizeof(double), cudaMemcpyDeviceToHost));
  MHY_CUDA(cudaMemcpy(pt.data(), part + (size_t)env * C, C * sizeof(double), cudaMemcpyDeviceToHost));
  for (long long i = 0; i < C; ++i) {
    const uint32_t m = mask[i];
    o[i] = !(m >> env & 1) ? 0. : (__builtin_popcount(m) == 1 ? g[i] : pt[i]);
  }
  to_caller();
  return MHY_OK;
}

int mhy_get_dt(mhy_ctx* c, double* dt, double* dt_old) {
  if (!c) return fail(MHY_ERR_ARG, "null context");
  DeviceScope on_dev(c->device);
  MHY_FLUSH(c);
  Scalars h{};
  MHY_CUDA(cudaStreamSynchronize(c->stream));
  MHY_CUDA(cudaMemcpy(&h, c->S, sizeof(h), cudaMemcpyDeviceToHost));
  if (dt) *dt = h.dt;
  if (dt_old) *dt_old = h.old_dt;
  return MHY_OK;
}

int mhy_get_time(mhy_ctx* c, double* time, int64_t* iteration) {
  if (!c) return fail(MHY_ERR_ARG, "null context");
  DeviceScope on_dev(c->device);
  MHY_FLUSH(c);
  Scalars h{};
  MHY_CUDA(cudaStreamSynchronize(c->stream));
  MHY_CUDA(cudaMemcpy(&h, c->S, sizeof(h), cudaMemcpyDeviceToHost));
  if (time) *time = h.time;
  if (iteration) *iteration = h.iteration;
  return MHY_OK;
}

int mhy_get_status(mhy_ctx* c, uint32_t* flags) {
  if (!c || !flags) return fail(MHY_ERR_ARG, "null argument");
  DeviceScope on_dev(c->device);
  MHY_FLUSH(c);
  Scalars h{};
  MHY_CUDA(cudaStreamSynchronize(c->stream));
  MHY_CUDA(cudaMemcpy(&h, c->S, sizeof(h), cudaMemcpyDeviceToHost));
  *flags = h.status;
  return MHY_OK;
}

int mhy_get_sizes(mhy_ctx* c, int64_t* ncells, int64_t* nnodes, int64_t* nfaces) {
  if (!c) return fail(MHY_ERR_ARG, "null context");
  if (ncells) *ncells = c->dm.C;
  if (nnodes) *nnodes = c->dm.N;
  if (nfaces) *nfaces = c->dm.F;
  return MHY_OK;
}

int mhy_get_totals(mhy_ctx* c, double* out) {
  if (!c || !out) return fail(MHY_ERR_ARG, "null argument");
  DeviceScope on_dev(c->device);
  MHY_FLUSH(c);
  if (!c->initialized) return fail(MHY_ERR_ORDER, "mhy_hydro_start_init has not run");
  double* part = c->setup;                       // 6 x kTotalsBlocks partials, then the 3 totals
  double* res = c->setup + 6 * kTotalsBlocks;
  k_totals_partial<<<kTotalsBlocks, kTotalsThreads, 0, c->stream>>>(c->dm, c->mass, c->e, c->nm, c->v, part);
  k_totals_finish<<<1, 1, 0, c->stream>>>(part, kTotalsBlocks, res);
  MHY_CUDA(cudaGetLastError());
  MHY_CUDA(cudaMemcpyAsync(out, res, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  MHY_CUDA(cudaStreamSynchronize(c->stream));
  return MHY_OK;
}

void* mhy_get_stream(mhy_ctx* c) {
  if (!c) return nullptr;
  DeviceScope on_dev(c->device);
  flush(c);                                        // work the caller enqueues follows the entry points
  return (void*)c->stream;
}

int mhy_kernels_per_cycle(mhy_ctx* c) { return c ? c->kernels_per_cycle : 0; }

// ---- slabs: one mesh split along z over several contexts ----------------------
int mhy_set_dt_reduction(mhy_ctx* c, int32_t k_lo, int32_t k_hi, int32_t external) {
  if (!c) return fail(MHY_ERR_ARG, "null context");
  if (k_lo < 0 || k_hi > c->dm.nz || k_lo >= k_hi || (external != 0 && external != 1))
    return fail(MHY_ERR_ARG, "need 0 <= k_lo < k_hi <= nz and external 0 or 1");
  DeviceScope on_dev(c->device);
  MHY_FLUSH(c);
  c->dm.dt_k0 = k_lo;
  c->dm.dt_k1 = k_hi;
  c->ph.ext_dt = external;
  for (int s = 0; s < 3; ++s)
    if (c->graph[s]) { cudaGraphExecDestroy(c->graph[s]); c->graph[s] = nullptr; }
  return MHY_OK;
}

int mhy_dt_local_min(mhy_ctx* c, void* dev_min_bits) {
  if (!c || !dev_min_bits) return fail(MHY_ERR_ARG, "null argument");
  if (!c->ph.ext_dt) return fail(MHY_ERR_STATE, "mhy_set_dt_reduction(..., external = 1) must come first");
  DeviceScope on_dev(c->device);
  MHY_FLUSH(c);
  MHY_CUDA(cudaMemcpyAsync(dev_min_bits, &c->S->min_bits, sizeof(unsigned long long), cudaMemcpyDeviceToDevice,
                           c->stream));
  return MHY_OK;
}

int mhy_dt_finish(mhy_ctx* c, const void* dev_min_bits) {
  if (!c || !dev_min_bits) return fail(MHY_ERR_ARG, "null argument");
  if (!c->ph.ext_dt) return fail(MHY_ERR_STATE, "mhy_set_dt_reduction(..., external = 1) must come first");
  DeviceScope on_dev(c->device);
  MHY_FLUSH(c);
  k_dt_finish_ext<<<1, 1, 0, c->stream>>>(c->S, c->ph, static_cast<const unsigned long long*>(dev_min_bits));
  MHY_CUDA(cudaGetLastError());
  return MHY_OK;
}

}  // extern "C"

namespace {

// The persistent state of layers [lo, hi) of cells and [nlo, nhi) of nodes, as
// (device pointer, bytes) pieces in a fixed order: every restart-dump field,
// each component plane's slice of those layers (contiguous, k is outermost).
int halo_pieces(mhy_ctx* c, int lo, int hi, int nlo, int nhi, std::vector<std::pair<char*, size_t>>& out) {
  const Dims& dm = c->dm;
  if (lo < 0 || hi > dm.nz || lo > hi || nlo < 0 || nhi > dm.nz + 1 || nlo > nhi)
    return fail(MHY_ERR_ARG, "layer range outside the mesh");
  const long long cl = (long long)dm.nx * dm.ny, nl = (long long)(dm.nx + 1) * (dm.ny + 1);
  out.clear();
  for (const CkField& f : ckpt_fields(c)) {
    const size_t el = ckpt_elem(f.dtype);
    const bool cell = std::strcmp(f.name, "Velocity") != 0 && std::strcmp(f.name, "NodeMass") != 0 &&
                      std::strcmp(f.name, "DualGradPhi") != 0;   // the node fields of ckpt_fields
    const long long items = cell ? dm.C : dm.N, comps = f.count / items, per = cell ? cl : nl;
    const int a = cell ? lo : nlo, b = cell ? hi : nhi;
    for (long long q = 0; q < comps; ++q)
      out.emplace_back(static_cast<char*>(f.dev) + ((size_t)q * items + (size_t)a * per) * el, (size_t)(b - a) * per * el);
  }
  return MHY_OK;
}

int halo_copy(mhy_ctx* c, int lo, int hi, int nlo, int nhi, char* buf, size_t bytes, bool pack) {
  std::vector<std::pair<char*, size_t>> pc;
  int rc = halo_pieces(c, lo, hi, nlo, nhi, pc);
  if (rc != MHY_OK) return rc;
  size_t need = 0;
  for (auto& x : pc) need += x.second;
  if (bytes < need) return fail(MHY_ERR_ARG, "halo buffer too small (mhy_halo_bytes)");
  size_t off = 0;
  for (auto& x : pc) {
    if (x.second)
      MHY_CUDA(cudaMemcpyAsync(pack ? buf + off : x.first, pack ? x.first : buf + off, x.second,
                               cudaMemcpyDeviceToDevice, c->stream));
    off += x.second;
  }
  return MHY_OK;
}

}  // namespace

extern "C" {

int mhy_halo_bytes(mhy_ctx* c, int32_t cell_layers, int32_t node_layers, size_t* bytes) {
  if (!c || !bytes) return fail(MHY_ERR_ARG, "null argument");
  std::vector<std::pair<char*, size_t>> pc;
  const int rc = halo_pieces(c, 0, cell_layers, 0, node_layers, pc);
  if (rc != MHY_OK) return rc;
  size_t need = 0;
  for (auto& x : pc) need += x.second;
  *bytes = need;
  return MHY_OK;
}

int mhy_halo_pack(mhy_ctx* c, int32_t cell_lo, int32_t cell_hi, int32_t node_lo, int32_t node_hi, void* dev_dst,
                  size_t bytes) {
  if (!c || !dev_dst) return fail(MHY_ERR_ARG, "null argument");
  DeviceScope on_dev(c->device);
  MHY_FLUSH(c);
  return halo_copy(c, cell_lo, cell_hi, node_lo, node_hi, static_cast<char*>(dev_dst), bytes, true);
}

int mhy_halo_unpack(mhy_ctx* c, int32_t cell_lo, int32_t cell_hi, int32_t node_lo, int32_t node_hi,
                    const void* dev_src, size_t bytes) {
  if (!c || !dev_src) return fail(MHY_ERR_ARG, "null argument");
  DeviceScope on_dev(c->device);
  MHY_FLUSH(c);
  return halo_copy(c, cell_lo, cell_hi, node_lo, node_hi, const_cast<char*>(static_cast<const char*>(dev_src)), bytes,
                   false);
}

void mhy_destroy(mhy_ctx* c) {
  if (!c) return;
  DeviceScope on_dev(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (int s = 0; s < 3; ++s) if (c->graph[s]) cudaGraphExecDestroy(c->graph[s]);
  for (void* p_ : c->allocs) cudaFree(p_);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

}  // extern "C"
