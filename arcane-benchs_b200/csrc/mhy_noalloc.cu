// mhy_noalloc.cu -- the CFL time-step reduction for callers that cannot
// allocate device memory.
//
// Who needs it: a host framework that owns every device allocation (Arcane
// hands out its variables from its own allocator and unified memory; a plugin
// is not supposed to call cudaMalloc behind its back), and code that records
// its work into a stream capture, where cudaMalloc is not a legal call.  Such a
// caller already holds the mesh fields on the device and only needs the time
// step computed from them.
//
// The reduction needs scratch memory (one partial minimum per block of the
// first pass).  Here that scratch is a file-scope __device__ array, so the
// entry point allocates nothing: it issues two kernel launches on the caller's
// stream and returns.
//
// Limits and sharing, stated for users:
//  * the scratch holds kNoAllocBlocks partial minima (64 KiB per GPU, kept by
//    every GPU that loads this library until the process exits);
//  * the first pass uses at most kNoAllocBlocks blocks of 256 threads and each
//    thread takes at most kNoAllocCellsPerThread cells, so meshes are limited
//    to kNoAllocMaxCells cells; larger meshes are rejected with MHY_ERR_ARG;
//  * every call on a device shares the same scratch and leaves its partial
//    minima there; each call writes every slot it reads before reading it, so
//    nothing has to be cleared, but calls that overlap on the GPU (different
//    streams, or different host threads on one device) race on the scratch and
//    must be serialised by the caller;
//  * the first call on a device looks up the scratch's device address with
//    cudaGetSymbolAddress (with that device current); make that first call
//    before any stream capture.  The address is kept per device together with
//    the identity of the device's current CUDA context, and looked up again
//    when that context has changed (after cudaDeviceReset, for instance), so
//    the first call after such a reset must also come before any capture;
//  * a cell whose L / (c + max |v|) is NaN or negative (an inverted cell, a NaN
//    field) is not skipped: the call then writes out[0] = NaN and out[1] = 0,
//    a time step below any positive deltat-min, so a caller that checks the
//    new dt against deltat-min stops as the reference does (MahycoModule.cc:
//    2152-2159).  The context's own reduction raises MHY_STATUS_NAN_DT for the
//    same cells.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "mhy_kernels.cuh"

namespace mhy {
namespace {

constexpr int kNoAllocBlocks = 8192;
constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocCellsPerThread = 64;
constexpr long long kNoAllocMaxCells = (long long)kNoAllocBlocks * kNoAllocThreads * kNoAllocCellsPerThread;
constexpr unsigned long long kDblMaxBits = 0x7fefffffffffffffull;
// A block's partial minimum is the bit pattern of a non-negative double (bit
// 63 clear); bit 63 set records that the block met an invalid cell.
constexpr unsigned long long kInvalidBit = 0x8000000000000000ull;

static __device__ __align__(256) unsigned long long g_dt_scratch[kNoAllocBlocks];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
struct ScratchAddr {
  unsigned long long* addr = nullptr;
  unsigned long long ctx_id = 0;   // CUDA context the address belongs to (0: unknown)
};
ScratchAddr g_scratch[kMaxDevices];

// Identity of the calling thread's current CUDA context (cuCtxGetId through
// the runtime's driver entry points, so the library does not link libcuda);
// 0 when there is none or the driver cannot say.
unsigned long long current_ctx_id() {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {             // under g_mutex
    void* f1 = nullptr;
    void* f2 = nullptr;
    cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
        q1 == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f1);
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
        q2 == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f2);
    cudaGetLastError();
    looked_up = true;
  }
  if (!get_current || !get_id) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

__device__ __forceinline__ unsigned long long block_min(unsigned long long best, unsigned long long* wmin) {
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long other = __shfl_down_sync(0xffffffffu, best, o);
    best = other < best ? other : best;
  }
  if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = best;
  __syncthreads();
  best = kDblMaxBits;
  if (threadIdx.x < 32) {
    best = threadIdx.x < (blockDim.x >> 5) ? wmin[threadIdx.x] : kDblMaxBits;
    for (int o = 16; o > 0; o >>= 1) {
      unsigned long long other = __shfl_down_sync(0xffffffffu, best, o);
      best = other < best ? other : best;
    }
  }
  return best;  // valid in thread 0
}

// First pass: dx_sound = L / (c + max over the cell's nodes of |v|), as in
// computeHydroDeltaT (mahyco/src/MahycoModule.cc:2047-2060); one partial
// minimum per block (bit patterns of non-negative doubles order like
// integers), with kInvalidBit set when the block met a NaN or negative value.
__global__ void k_dt_partial_noalloc(Dims dm, const double* __restrict__ L, const double* __restrict__ cs,
                                     const double* __restrict__ v, unsigned long long* __restrict__ scratch) {
  __shared__ unsigned long long wmin[32];
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  unsigned long long best = kDblMaxBits;
  bool invalid = false;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < dm.C;
       c += (long long)gridDim.x * blockDim.x) {
    int i, j, k; dm.cijk(c, i, j, k);
    double vmax = 0.;
    for (int a = 0; a < 8; ++a) {
      long long n = dm.nid(i + kCellNodeOff[a][0], j + kCellNodeOff[a][1], k + kCellNodeOff[a][2]);
      vmax = amax(norm2(d3(v[n], v[dm.N + n], v[2 * dm.N + n])), vmax);
    }
    double dx_sound = L[c] / (cs[c] + vmax);
    if (dx_sound >= 0.) {
      unsigned long long b = (unsigned long long)__double_as_longlong(dx_sound);
      best = b < best ? b : best;
    } else {
      invalid = true;                               // NaN or negative
    }
  }
  if (invalid) bad = 1;                             // benign race: every writer stores 1
  best = block_min(best, wmin);                     // its barrier also orders the writes to `bad`
  if (threadIdx.x == 0) scratch[blockIdx.x] = best | (bad ? kInvalidBit : 0ull);
}

// Second pass: minimum of the partial minima, then the new dt of
// computeDeltaT (MahycoModule.cc:2144-2150): min(cfl * min, 1.05 * dt_old, deltat_max);
// NaN and 0 when any block met an invalid cell.
__global__ void k_dt_final_noalloc(const unsigned long long* __restrict__ scratch, int nparts, double cfl,
                                   double dt_old, double deltat_max, double* __restrict__ out) {
  __shared__ unsigned long long wmin[32];
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  unsigned long long best = kDblMaxBits;
  bool invalid = false;
  for (int t = threadIdx.x; t < nparts; t += blockDim.x) {
    const unsigned long long s = scratch[t];
    if (s & kInvalidBit) invalid = true;
    const unsigned long long b = s & ~kInvalidBit;
    best = b < best ? b : best;
  }
  if (invalid) bad = 1;
  best = block_min(best, wmin);
  if (threadIdx.x == 0) {
    if (bad) {
      out[0] = __longlong_as_double(0x7ff8000000000000ll);   // quiet NaN: no valid minimum
      out[1] = 0.;
      return;
    }
    const double minimum_aux = __longlong_as_double((long long)best);
    double new_dt = cfl * minimum_aux;
    new_dt = amin(new_dt, 1.05 * dt_old);
    new_dt = amin(new_dt, deltat_max);
    out[0] = minimum_aux;
    out[1] = new_dt;
  }
}

}  // namespace
}  // namespace mhy

extern "C" int mhy_compute_hydro_dt_noalloc(int32_t nx, int32_t ny, int32_t nz, const double* L, const double* cs,
                                            const double* v, double cfl, double dt_old, double deltat_max,
                                            double* out, void* stream) {
  using namespace mhy;
  if (nx < 1 || ny < 1 || nz < 1 || !L || !cs || !v || !out) return MHY_ERR_ARG;
  Dims dm{};
  dm.nx = nx; dm.ny = ny; dm.nz = nz;
  dm.C = (long long)nx * ny * nz;
  dm.N = (long long)(nx + 1) * (ny + 1) * (nz + 1);
  if (dm.C > kNoAllocMaxCells) return MHY_ERR_ARG;  // beyond the scratch's capacity
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return MHY_ERR_CUDA;
  unsigned long long* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    ScratchAddr& sa = g_scratch[dev];
    const unsigned long long id = current_ctx_id();
    if (!sa.addr || id == 0 || id != sa.ctx_id) {
      // set-up of this device (or of its new context): the scratch's device address
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_dt_scratch) != cudaSuccess || !p) {
        cudaGetLastError();
        sa = ScratchAddr{};
        return MHY_ERR_CUDA;
      }
      sa.addr = static_cast<unsigned long long*>(p);
      sa.ctx_id = current_ctx_id();                 // the lookup has made the context current
    }
    scratch = sa.addr;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  long long want = (dm.C + kNoAllocThreads - 1) / kNoAllocThreads;
  const int nblocks = (int)(want < kNoAllocBlocks ? want : kNoAllocBlocks);
  k_dt_partial_noalloc<<<nblocks, kNoAllocThreads, 0, s>>>(dm, L, cs, v, scratch);
  k_dt_final_noalloc<<<1, 1024, 0, s>>>(scratch, nblocks, cfl, dt_old, deltat_max, out);
  if (cudaGetLastError() != cudaSuccess) return MHY_ERR_CUDA;
  return MHY_OK;
}
