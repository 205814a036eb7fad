// Fragment-memory term (fix_backbone.cpp:4079-4177, fragment_memory.cpp:
// 190-202) on a sliced, lane-interleaved memory table.
//
// Table layout.  A row is one target pair (i, j = i + min_sep + d) with the
// records of every memory covering it; a record holds the four memory
// distances of the atom pairs CA-CA, CA-CB, CB-CA, CB-CB.  Residues are
// taken 32 at a time (group g = residues 32g .. 32g+31).  Block (g, d) holds
// the rows (32g + l, d) of the group's 32 residues as `len` stripes; stripe
// m carries record m of each of the 32 rows side by side, lane l's record
// at [stripe][l].  Rows shorter than `len` are padded with records whose
// distances are 1e30 and whose coefficient is 0: their Gaussian is exactly
// zero, so padding never changes a sum.  Blocks are stored g-major
// (block = g * nd + d), so the data of one group is contiguous.
//
// Kernel mapping.  One warp per (group, chunk of separations); lane l owns
// residue i = 32g + l and streams its rows stripe by stripe: every load of
// the warp is 32 consecutive records (512 B FP32, 1 KiB FP64) and each lane
// keeps its own sums, so no cross-lane reduction is needed.  Forces are
// converted to 64-bit fixed point (2^-32) per (row, atom pair) and added to
// the accumulator of j with integer atomics; i's forces are summed in
// registers over the chunk first.  Everything is order independent, so a
// residue's result does not depend on its group mates or on the chunking.
#pragma once

#include "awsem_device.cuh"

namespace awsem {
namespace dev {

template <typename R> struct FMSlices {
  const int *soff;  // [G * nd] first stripe of block (g, d)
  const int *slen;  // [G * nd] stripes of block (g, d)
  const R *rf;      // [stripes][32][4] memory distances
  const R *coef;    // [stripes][32] eps * k_fm * weight * gamma, or nullptr when all equal `uniform`
  double uniform;
  int nd, min_sep;  // separations min_sep .. min_sep + nd - 1
  int groups;       // G = ceil(n_res / 32)
  int dsplit;       // separation chunks per group (warps per group)
};

// One memory record: 16 bytes (FP32) or 32 bytes (FP64)
__device__ __forceinline__ void load_record(const float *rf, size_t rec, float m[4])
{
  float4 v = __ldg(reinterpret_cast<const float4 *>(rf) + rec);
  m[0] = v.x, m[1] = v.y, m[2] = v.z, m[3] = v.w;
}
__device__ __forceinline__ void load_record(const double *rf, size_t rec, double m[4])
{
  const double2 *q = reinterpret_cast<const double2 *>(rf) + 2 * rec;
  double2 u = __ldg(q), v = __ldg(q + 1);
  m[0] = u.x, m[1] = u.y, m[2] = v.x, m[3] = v.y;
}

__device__ __forceinline__ void red_add3(unsigned long long *p, const long long f[3])
{
#pragma unroll
  for (int c = 0; c < 3; c++)
    if (f[c]) atomicAdd(p + c, (unsigned long long) f[c]);
}

// The warp's share of the fragment-memory term.  `pos(r, b)` returns the FP64
// position of residue r's CA (b = 0) or CB (b = 1); forces go to `facc`
// ([atom][3], atom = 3 r + b, fixed point).  Energies are added in fixed
// point to e_acc[i * e_stride] (per residue with e_stride = 1; one total
// with e_stride = 0).  sig[s] is the Gaussian variance of sequence
// separation s, |s|^(2 * sigma_exp) (fix_backbone.cpp:4126).
template <typename R, class Pos>
__device__ __forceinline__ void fragmem_warp(const FMSlices<R> &t, const double *sig, int n, const Pos &pos,
                                             unsigned long long *facc, unsigned long long *e_acc, int e_stride)
{
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= t.groups * t.dsplit) return;
  const int g = w / t.dsplit, c = w - g * t.dsplit;
  const int d0 = c * t.nd / t.dsplit, d1 = (c + 1) * t.nd / t.dsplit;
  const int i = g * 32 + lane;
  const bool live = i < n;
  const int ii = live ? i : n - 1;
  const V3<double> ca_i = pos(ii, 0), cb_i = pos(ii, 1);
  long long fca[3] = {0, 0, 0}, fcb[3] = {0, 0, 0};
  double e = 0.0;
  const R cu = R(t.uniform);
  for (int d = d0; d < d1; d++) {
    const int blk = g * t.nd + d;
    const int len = t.slen[blk];
    if (len == 0) continue;
    const size_t base = (size_t) t.soff[blk] * 32 + lane;
    // rows past the end carry padding only; any valid partner index will do
    const int j = min(ii + t.min_sep + d, n - 1);
    const V3<double> ca_j = pos(j, 0), cb_j = pos(j, 1);
    const V3<R> dv[4] = {diff<R>(ca_i, ca_j), diff<R>(ca_i, cb_j), diff<R>(cb_i, ca_j), diff<R>(cb_i, cb_j)};
    R r[4];
#pragma unroll
    for (int k = 0; k < 4; k++) r[k] = m_sqrt(norm2(dv[k]));
    const R s2 = R(sig[t.min_sep + d]);
    const R inv2s = R(1) / (R(2) * s2);
    R es = 0, fs[4] = {0, 0, 0, 0};
#pragma unroll 4
    for (int m = 0; m < len; m++) {
      const size_t at = base + (size_t) m * 32;
      R rec[4];
      load_record(t.rf, at, rec);
      const R cc = t.coef ? t.coef[at] : cu;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const R dr = r[k] - rec[k];
        const R gk = cc * m_fastexp(-dr * dr * inv2s);
        es -= gk;
        fs[k] -= gk * dr;
      }
    }
    e += (double) es;
    // atom pair k acts on CA(i) (k < 2) or CB(i), and on CA(j) (k even) or CB(j)
    long long fja[3] = {0, 0, 0}, fjb[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const R fc = fs[k] != R(0) ? fs[k] / (s2 * r[k]) : R(0);
      const long long v[3] = {fix_force((double) (fc * dv[k].x)), fix_force((double) (fc * dv[k].y)),
                              fix_force((double) (fc * dv[k].z))};
#pragma unroll
      for (int q = 0; q < 3; q++) {
        if (k < 2)
          fca[q] += v[q];
        else
          fcb[q] += v[q];
        if (k & 1)
          fjb[q] -= v[q];
        else
          fja[q] -= v[q];
      }
    }
    red_add3(facc + (size_t) 9 * j, fja);
    red_add3(facc + (size_t) 9 * j + 3, fjb);
  }
  if (live) {
    red_add3(facc + (size_t) 9 * i, fca);
    red_add3(facc + (size_t) 9 * i + 3, fcb);
  }
  long long ef = live ? fix_force(e) : 0;
  if (e_stride) {
    if (ef) atomicAdd(e_acc + (size_t) i * e_stride, (unsigned long long) ef);
  } else {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ef += __shfl_xor_sync(0xffffffffu, ef, o);
    if (lane == 0 && ef) atomicAdd(e_acc, (unsigned long long) ef);
  }
}

}  // namespace dev

// A handle's resident fragment-memory table, for entry points outside the
// engine: the slices with the element type erased, plus the variance table.
struct FMView {
  const int *soff, *slen;
  const void *rf, *coef;  // double (FP64 form) or float (mixed form) elements
  double uniform;
  int nd, min_sep, groups, dsplit, n_res, is_double;
  const double *sigma_sq;  // host table [64]
};

}  // namespace awsem
