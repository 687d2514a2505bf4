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

__global__ void k_init_cells(Dims dm, const double* x0, double* xc0, double* cqs, double* vol, double* L, int lc_mode);
__global__ void k_init_faces(Dims dm, const double* x0, double* n0, double* xf0);
__global__ void k_init_outer_normals(Dims dm, const double* xc0, const double* xf0, double* ofn);
__global__ void k_init_state(Dims dm, double gamma, const double* vol, double* rho, const double* pres, double* e,
                             double* cs, double* mass, double* q);
__global__ void k_node_mass(Dims dm, const double* mass, double* nm);
__global__ void k_lagrange_nodes(Dims dm, const Scalars* S, const double* p, const double* q, const double* cqs,
                                 const double* nm, const double* v, const double* x0, const uint16_t* bcmask,
                                 BCTable bct, double* vh, double* xl, double* ud, double* phid);
__global__ void k_lagrange_cells(Dims dm, const Scalars* S, Phys ph, const double* xl, const double* rho,
                                 const double* e, const double* q, const double* p, const double* cs,
                                 const double* mass, double* cqs, double* xc, double* L, double* U);
__global__ void k_faces(Dims dm, const double* xl, const double* vh, const double* n0, double* A, double* uf,
                        double* xf);
__global__ void k_sweep_face_grad(Dims dm, int d, const double* xc, const double* n0, const double* U, double* dxf,
                                  double* gf);
__global__ void k_sweep_cell_grad(Dims dm, int d, int lim, const double* gf, double* G);
__global__ void k_sweep_face_phi(Dims dm, int d, double order2, const double* xc, const double* n0,
                                 const double* xf, const double* uf, const double* dxf, const double* U,
                                 const double* G, double* phif);
__global__ void k_sweep_cell_update(Dims dm, int d, const Scalars* S, const double* n0, const double* uf,
                                    const double* A, const double* ofn, const double* phif, double* U, double* dpf);
__global__ void k_sweep_dual_grad(Dims dm, int d, int lim, const double* xl, const double* phid, double* G);
__global__ void k_sweep_dual_update(Dims dm, int d, const Scalars* S, double order2, const double* xl,
                                    const double* dpf, const double* G, const double* phid, double* ud,
                                    double* phid_out);
__global__ void k_finalize_cells(Dims dm, Phys ph, Scalars* S, const double* U, const double* Ve, double* rho,
                                 double* e, double* q, double* p, double* cs, double* mass);
__global__ void k_finalize_nodes(Dims dm, const double* ud, const double* vh, const double* mass, double* v,
                                 double* nm);
__global__ void k_dt_min(Dims dm, Scalars* S, const double* L, const double* cs, const double* v);
__global__ void k_dt_finish(Scalars* S, Phys ph);

}  // namespace mhy
