// Fragment-memory forces through an entry point that allocates nothing.
//
// Who needs it: callers that may not call cudaMalloc at force time -- a host
// MD code that owns all device memory through its own pool, a step already
// being recorded into a CUDA graph by the caller, or a real-time pipeline
// that forbids allocation after start-up.  They pass device buffers for the
// positions and the outputs; the fixed-point force accumulator this kernel
// needs lives in a file-scope __device__ array of fixed size instead of a
// buffer allocated by the engine.
//
// Limits and sharing: the array holds AWSEM_NOALLOC_MAX_ATOMS atoms (per
// GPU that loads the library, held until exit).  Every call on a device
// uses the same array and leaves its contents behind; each call clears the
// part it uses first.  Two calls whose kernels overlap on the GPU (different
// streams, or different host threads) race on the array and give wrong
// forces: serialise them.
#include <cuda_runtime.h>

#include <mutex>
#include <stdexcept>
#include <string>

#include "awsem_device.cuh"
#include "awsem_fragmem.cuh"
#include "awsem_gpu.h"

namespace awsem {
namespace noalloc {

// fixed-point (2^-32) force accumulator [atoms][3], then one slot for the
// fixed-point energy (padded to keep the array a multiple of 256 bytes)
constexpr int kEnergySlot = AWSEM_NOALLOC_MAX_ATOMS * 3;
static __device__ __align__(256) unsigned long long g_facc[AWSEM_NOALLOC_MAX_ATOMS * 3 + 32];

constexpr int kMaxDevices = 64;
struct ScratchAddr {
  void *ctx = nullptr;                // the CUDA context the address belongs to
  unsigned long long *addr = nullptr;
};
static ScratchAddr g_facc_addr[kMaxDevices];
static std::mutex g_mutex;

// The driver's cuCtxGetCurrent, found through the runtime (no link-time
// dependency on the driver library); CUcontext is an opaque pointer.
typedef int (*CtxGetCurrentFn)(void **);
static CtxGetCurrentFn ctx_get_current()
{
  static CtxGetCurrentFn fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return (CtxGetCurrentFn) p;
  }();
  return fn;
}

// Device address of g_facc on `device` (the current device).  In host code
// the array's name is only a host-side stand-in; the address comes from the
// runtime: at the first call on the device, and again whenever the device's
// context has changed since (after a cudaDeviceReset the old address is
// gone).
static unsigned long long *scratch(int device)
{
  if (device < 0 || device >= kMaxDevices) throw std::invalid_argument("device index out of range");
  std::lock_guard<std::mutex> lock(g_mutex);
  void *ctx = nullptr;
  if (CtxGetCurrentFn get = ctx_get_current()) {
    if (get(&ctx) != 0) ctx = nullptr;
  }
  ScratchAddr &c = g_facc_addr[device];
  if (!c.addr || ctx != c.ctx) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_facc);
    if (e != cudaSuccess) throw std::runtime_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    c.addr = (unsigned long long *) p;
    c.ctx = ctx;
  }
  return c.addr;
}

__global__ void k_clear(unsigned long long *facc, int n)
{
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) facc[k] = 0ull;
  if (k == 0) facc[kEnergySlot] = 0ull;
}

struct SigmaTable {
  double v[64];  // |i-j|^(2 * fm_sigma_exp) by sequence separation
};

// Positions from the caller's [atoms][3] array (per residue CA, CB/H-beta, O)
struct CallerPos {
  const double *x;
  __device__ __forceinline__ dev::V3<double> operator()(int r, int b) const
  {
    const double *q = x + ((size_t) 3 * r + b) * 3;
    return {q[0], q[1], q[2]};
  }
};

// The engine's fragment-memory warp routine on the caller's positions, so
// both entry points give the same forces bit for bit.
template <typename R>
__global__ void __launch_bounds__(128) k_fragmem(const double *x, int n_res, dev::FMSlices<R> t, SigmaTable sig,
                                                 unsigned long long *facc)
{
  const CallerPos pos{x};
  dev::fragmem_warp(t, sig.v, n_res, pos, facc, facc + kEnergySlot, 0);
}

__global__ void k_unfix(const unsigned long long *facc, int n, double *f, double *energy)
{
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) f[k] = (double) (long long) facc[k] * dev::F_UNSCALE;
  if (k == 0) *energy = (double) (long long) facc[kEnergySlot] * dev::F_UNSCALE;
}

template <typename R> dev::FMSlices<R> slices(const FMView &v)
{
  dev::FMSlices<R> t;
  t.soff = v.soff;
  t.slen = v.slen;
  t.rf = (const R *) v.rf;
  t.coef = (const R *) v.coef;
  t.uniform = v.uniform;
  t.nd = v.nd;
  t.min_sep = v.min_sep;
  t.groups = v.groups;
  t.dsplit = v.dsplit;
  t.wait_limit = dev::kFmWaitLimit;  // the register-load path used here has no waits
  t.hold_tx = 0;
  return t;
}

}  // namespace noalloc

// Called by the C ABI with the handle's device current.
void fragmem_noalloc(int device, const FMView &v, const double *d_x, double *d_f, double *d_energy,
                     cudaStream_t stream)
{
  using namespace noalloc;
  const int n_atoms = 3 * v.n_res;
  if (n_atoms > AWSEM_NOALLOC_MAX_ATOMS)
    throw std::invalid_argument("awsem_fragmem_noalloc: " + std::to_string(n_atoms) + " atoms exceed the " +
                                std::to_string(AWSEM_NOALLOC_MAX_ATOMS) + "-atom scratch of this entry point");
  SigmaTable sig;
  for (int k = 0; k < 64; k++) sig.v[k] = v.sigma_sq[k];
  unsigned long long *facc = scratch(device);
  int n3 = 3 * n_atoms, tb = 256;
  k_clear<<<(n3 + tb - 1) / tb, tb, 0, stream>>>(facc, n3);
  if (v.nd > 0) {
    int blocks = (v.groups * v.dsplit * 32 + 127) / 128;
    if (v.is_double)
      k_fragmem<double><<<blocks, 128, 0, stream>>>(d_x, v.n_res, slices<double>(v), sig, facc);
    else
      k_fragmem<float><<<blocks, 128, 0, stream>>>(d_x, v.n_res, slices<float>(v), sig, facc);
  }
  k_unfix<<<(n3 + tb - 1) / tb, tb, 0, stream>>>(facc, n3, d_f, d_energy);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw std::runtime_error(std::string("awsem_fragmem_noalloc: ") + cudaGetErrorString(e));
}

}  // namespace awsem
