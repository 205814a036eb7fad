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
#include "awsem_gpu.h"

namespace awsem {
namespace noalloc {

// fixed-point (2^-32) force accumulator, [atoms][3]
static __device__ __align__(256) unsigned long long g_facc[AWSEM_NOALLOC_MAX_ATOMS * 3];

constexpr int kMaxDevices = 64;
static unsigned long long *g_facc_addr[kMaxDevices];
static std::mutex g_mutex;

// Device address of g_facc on `device` (the current device).  In host code
// the array's name is only a host-side stand-in; the address comes from the
// runtime, once per device.
static unsigned long long *scratch(int device)
{
  if (device < 0 || device >= kMaxDevices) throw std::invalid_argument("device index out of range");
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_facc_addr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_facc);
    if (e != cudaSuccess) throw std::runtime_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_facc_addr[device] = (unsigned long long *) p;
  }
  return g_facc_addr[device];
}

__global__ void k_clear(unsigned long long *facc, int n, double *energy)
{
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) facc[k] = 0ull;
  if (k == 0) *energy = 0.0;
}

// Warp per target residue i; same arithmetic as the engine's fragment-memory
// kernel (fix_backbone.cpp:4079-4177 in pair-major form), positions read
// from the caller's [atoms][3] array (per residue CA, CB/H-beta, O).
struct SigmaTable {
  double v[64];  // |i-j|^(2 * fm_sigma_exp) by sequence separation
};

template <typename R>
__global__ void k_fragmem(const double *x, int n_res, const int *row, const R *rf, const R *coef, double uniform,
                          int nd, int min_sep, SigmaTable sigma_sq, unsigned long long *facc, double *energy)
{
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (i >= n_res) return;
  int k = lane & 3;
  const int ib = (k < 2) ? 0 : 1, jb = (k & 1) ? 1 : 0;
  const double *pi = x + ((size_t) 3 * i + ib) * 3;
  long long Fi[3] = {0, 0, 0};
  double e_tot = 0.0;
  for (int dd = 0; dd < nd; dd++) {
    int r0 = row[i * nd + dd], r1 = row[i * nd + dd + 1];
    if (r1 == r0) continue;
    int j = i + min_sep + dd;
    const double *pj = x + ((size_t) 3 * j + jb) * 3;
    dev::V3<R> d = {(R) (pi[0] - pj[0]), (R) (pi[1] - pj[1]), (R) (pi[2] - pj[2])};
    R r = dev::m_sqrt(dev::norm2(d));
    R s2 = R(sigma_sq.v[min_sep + dd]);
    R inv2s = R(1) / (R(2) * s2);
    R esum = 0, fsum = 0;
    const R *t = rf + (size_t) r0 * 4;
    int nrec4 = (r1 - r0) * 4;
    for (int e = lane; e < nrec4; e += 32) {
      R dr = r - t[e];
      R c = coef ? coef[r0 + (e >> 2)] : R(uniform);
      R g = c * dev::m_fastexp(-dr * dr * inv2s);
      esum -= g;
      fsum -= g * dr;
    }
    for (int o = 4; o < 32; o <<= 1) {
      esum += __shfl_xor_sync(0xffffffffu, esum, o);
      fsum += __shfl_xor_sync(0xffffffffu, fsum, o);
    }
    double erow = (double) esum;
    erow += __shfl_xor_sync(0xffffffffu, erow, 1);
    erow += __shfl_xor_sync(0xffffffffu, erow, 2);
    e_tot += erow;
    if (lane < 4 && fsum != R(0)) {
      R fc = fsum / (s2 * r);
      long long fx = dev::fix_force((double) (fc * d.x)), fy = dev::fix_force((double) (fc * d.y)),
                fz = dev::fix_force((double) (fc * d.z));
      Fi[0] += fx;
      Fi[1] += fy;
      Fi[2] += fz;
      unsigned long long *fj = facc + ((size_t) 3 * j + jb) * 3;
      atomicAdd(fj + 0, (unsigned long long) (-fx));
      atomicAdd(fj + 1, (unsigned long long) (-fy));
      atomicAdd(fj + 2, (unsigned long long) (-fz));
    }
  }
  for (int c = 0; c < 3; c++) Fi[c] += __shfl_xor_sync(0xffffffffu, Fi[c], 1);
  if (lane == 0 || lane == 2) {
    unsigned long long *fi = facc + ((size_t) 3 * i + ib) * 3;
    for (int c = 0; c < 3; c++)
      if (Fi[c]) atomicAdd(fi + c, (unsigned long long) Fi[c]);
  }
  if (lane == 0 && e_tot != 0.0) atomicAdd(energy, e_tot);
}

__global__ void k_unfix(const unsigned long long *facc, int n, double *f)
{
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) f[k] = (double) (long long) facc[k] * dev::F_UNSCALE;
}

}  // namespace noalloc

// Called by the C ABI with the handle's device current.
void fragmem_noalloc(int device, int n_res, const int *row, const void *rf, const void *coef, double uniform, int nd,
                     int min_sep, const double *sigma_sq, int is_double, const double *d_x, double *d_f,
                     double *d_energy, cudaStream_t stream)
{
  using namespace noalloc;
  SigmaTable sig;
  for (int k = 0; k < 64; k++) sig.v[k] = sigma_sq[k];
  const int n_atoms = 3 * n_res;
  if (n_atoms > AWSEM_NOALLOC_MAX_ATOMS)
    throw std::invalid_argument("awsem_fragmem_noalloc: " + std::to_string(n_atoms) + " atoms exceed the " +
                                std::to_string(AWSEM_NOALLOC_MAX_ATOMS) + "-atom scratch of this entry point");
  unsigned long long *facc = scratch(device);
  int n3 = 3 * n_atoms, tb = 256;
  k_clear<<<(n3 + tb - 1) / tb, tb, 0, stream>>>(facc, n3, d_energy);
  if (nd > 0) {
    int wb = (n_res * 32 + 127) / 128;
    if (is_double)
      k_fragmem<double><<<wb, 128, 0, stream>>>(d_x, n_res, row, (const double *) rf, (const double *) coef, uniform,
                                                nd, min_sep, sig, facc, d_energy);
    else
      k_fragmem<float><<<wb, 128, 0, stream>>>(d_x, n_res, row, (const float *) rf, (const float *) coef, uniform, nd,
                                               min_sep, sig, facc, d_energy);
  }
  k_unfix<<<(n3 + tb - 1) / tb, tb, 0, stream>>>(facc, n3, d_f);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw std::runtime_error(std::string("awsem_fragmem_noalloc: ") + cudaGetErrorString(e));
}

}  // namespace awsem
