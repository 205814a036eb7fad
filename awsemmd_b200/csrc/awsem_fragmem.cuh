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
// zero, so padding never changes a sum.  Block lengths are even, so every
// block starts on an even stripe.  Blocks are stored g-major (block =
// g * nd + d), so the data of one group is contiguous.
//
// Kernel mapping.  One warp per (group, chunk of separations); lane l owns
// residue i = 32g + l and streams its rows stripe by stripe: every load of
// the warp is 32 consecutive records (512 B FP32, 1 KiB FP64) and each lane
// keeps its own sums, so no cross-lane reduction is needed.  A row's even
// and odd records go to two sets of sums, added at the row's end: two
// independent dependency chains per lane, and the same sums in every path
// that reads the table (the records pair up the same way in each).  Forces are
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
  long long wait_limit;  // SM clock cycles a warp waits for one stage's copies before it gives up
  unsigned hold_tx;      // bytes each stage expects beyond its copies: 0, or (tests of the give-up
                         // path) 16, which never arrive, so every stage wait runs out
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

// Per-record arithmetic, shared by both load paths (so they agree bit for
// bit).  The Gaussian of a row with variance s^2 is exp(-dr^2 / (2 s^2)):
// FP32 evaluates it as 2^(k2 dr^2) with k2 = -log2(e) / (2 s^2) on the ex2
// unit, FP64 as exp(k2 dr^2) with k2 = -1 / (2 s^2).
__device__ __forceinline__ float fm_gauss(float x)
{
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ double fm_gauss(double x) { return exp(x); }
__device__ __forceinline__ float fm_k2(float s2) { return -1.4426950408889634f / (2.f * s2); }
__device__ __forceinline__ double fm_k2(double s2) { return -1.0 / (2.0 * s2); }

// One record's four Gaussians g_k (times the record's coefficient when the
// coefficients are not uniform): es += sum g_k, fs_k += g_k dr_k.  The row's
// energy and radial force sums are scale * es and scale * fs_k, with scale =
// -coefficient (uniform) or -1.
// FP32 operand pairs for Blackwell's paired FP32 instructions (f32x2): each
// element is rounded as the scalar operation rounds it.
__device__ __forceinline__ unsigned long long f2_pack(float a, float b)
{
  unsigned long long d;
  asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(a), "f"(b));
  return d;
}
__device__ __forceinline__ void f2_unpack(unsigned long long d, float &a, float &b)
{
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(d));
}
__device__ __forceinline__ unsigned long long f2_sub(unsigned long long a, unsigned long long b)
{
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ unsigned long long f2_mul(unsigned long long a, unsigned long long b)
{
  unsigned long long d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ unsigned long long f2_fma(unsigned long long a, unsigned long long b, unsigned long long c)
{
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

template <bool COEF, typename R>
__device__ __forceinline__ void fm_record(const R rec[4], R cc, const R r[4], R k2, R &es, R fs[4])
{
  if constexpr (sizeof(R) == 4) {
    // atom pairs (0, 1) and (2, 3) as f32x2 pairs: the same operations in
    // the same order as the scalar loop below, half the instructions
    const unsigned long long k22 = f2_pack(k2, k2);
#pragma unroll
    for (int h = 0; h < 4; h += 2) {
      const unsigned long long dr = f2_sub(f2_pack(r[h], r[h + 1]), f2_pack(rec[h], rec[h + 1]));
      float x0, x1;
      f2_unpack(f2_mul(f2_mul(dr, dr), k22), x0, x1);
      float g0 = fm_gauss(x0), g1 = fm_gauss(x1);
      if (COEF) f2_unpack(f2_mul(f2_pack(g0, g1), f2_pack(cc, cc)), g0, g1);
      es = es + g0;
      es = es + g1;
      f2_unpack(f2_fma(f2_pack(g0, g1), dr, f2_pack(fs[h], fs[h + 1])), fs[h], fs[h + 1]);
    }
  } else {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const R dr = r[k] - rec[k];
      R g = fm_gauss(dr * dr * k2);
      if (COEF) g = g * cc;
      es = es + g;
      fs[k] = madd(g, dr, fs[k]);
    }
  }
}

// Work unit w (group g, chunk c of its separations) of the fragment-memory
// term, records loaded into registers.  `pos(r, b)` returns the FP64
// position of residue r's CA (b = 0) or CB (b = 1); forces go to `facc`
// ([atom][3], atom = 3 r + b, fixed point).  Energies are added in fixed
// point to e_acc[i * e_stride] (per residue with e_stride = 1; one total
// with e_stride = 0).  sig[s] is the Gaussian variance of sequence
// separation s, |s|^(2 * sigma_exp) (fix_backbone.cpp:4126).
template <bool COEF, typename R, class Pos>
__device__ __forceinline__ void fragmem_unit_reg_t(int w, const FMSlices<R> &t, const double *sig, int n,
                                                   const Pos &pos, unsigned long long *facc,
                                                   unsigned long long *e_acc, int e_stride)
{
  const int lane = threadIdx.x & 31;
  const int g = w / t.dsplit, c = w - g * t.dsplit;
  const int d0 = c * t.nd / t.dsplit, d1 = (c + 1) * t.nd / t.dsplit;
  const int i = g * 32 + lane;
  const bool live = i < n;
  const int ii = live ? i : n - 1;
  const V3<double> ca_i = pos(ii, 0), cb_i = pos(ii, 1);
  long long fca[3] = {0, 0, 0}, fcb[3] = {0, 0, 0};
  double e = 0.0;
  const R scale = COEF ? R(-1) : -R(t.uniform);
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
    const R k2 = fm_k2(s2);
    R es = 0, fs[4] = {0, 0, 0, 0}, es1 = 0, fs1[4] = {0, 0, 0, 0};
#pragma unroll 2
    for (int m = 0; m < len; m += 2) {  // len is even
      const size_t at = base + (size_t) m * 32;
      R rec[4], rec1[4];
      load_record(t.rf, at, rec);
      load_record(t.rf, at + 32, rec1);
      fm_record<COEF>(rec, COEF ? t.coef[at] : R(1), r, k2, es, fs);
      fm_record<COEF>(rec1, COEF ? t.coef[at + 32] : R(1), r, k2, es1, fs1);
    }
    es = es + es1;
#pragma unroll
    for (int k = 0; k < 4; k++) fs[k] = fs[k] + fs1[k];
    e += (double) (scale * es);
    // atom pair k acts on CA(i) (k < 2) or CB(i), and on CA(j) (k even) or CB(j)
    long long fja[3] = {0, 0, 0}, fjb[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const R fc = fs[k] != R(0) ? (scale * fs[k]) / (s2 * r[k]) : R(0);
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

template <typename R, class Pos>
__device__ __forceinline__ void fragmem_unit_reg(int w, const FMSlices<R> &t, const double *sig, int n, const Pos &pos,
                                                 unsigned long long *facc, unsigned long long *e_acc, int e_stride)
{
  if (t.coef)
    fragmem_unit_reg_t<true>(w, t, sig, n, pos, facc, e_acc, e_stride);
  else
    fragmem_unit_reg_t<false>(w, t, sig, n, pos, facc, e_acc, e_stride);
}

// one warp per work unit
template <typename R, class Pos>
__device__ __forceinline__ void fragmem_warp(const FMSlices<R> &t, const double *sig, int n, const Pos &pos,
                                             unsigned long long *facc, unsigned long long *e_acc, int e_stride)
{
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w < t.groups * t.dsplit) fragmem_unit_reg(w, t, sig, n, pos, facc, e_acc, e_stride);
}


// ---------------------------------------------------------------------------
// Bulk-copy pipeline.  A group's blocks are contiguous stripes, so a warp's
// whole share is one contiguous run of stripes: lane 0 streams it into a
// ring of kFmStages shared-memory stages of kFmStripes stripes with 1-D bulk
// copies (cp.async.bulk, the TMA engine) completing on one mbarrier per
// stage, and the 32 lanes read their records from shared memory.  Up to
// kFmStages stages are in flight per warp with no register cost, which is
// what the register-load version lacks at full size.  Per lane the records
// are consumed in the same order, so the sums equal the register version's
// bit for bit.
constexpr int kFmStages = 3, kFmStripes = 8;

template <typename R> __host__ __device__ constexpr int fm_stage_bytes(bool coef)
{
  return kFmStripes * 32 * (int) sizeof(R) * (coef ? 5 : 4);
}
// shared memory of one warp: 128 bytes of mbarriers, then the stages
template <typename R> __host__ __device__ constexpr int fm_warp_smem(bool coef)
{
  return 128 + kFmStages * fm_stage_bytes<R>(coef);
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t) __cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect(uint32_t bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// Wait for phase `parity` of an mbarrier, giving up after `limit` clock
// cycles (false: timed out).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit)
{
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > limit) return false;
  }
}

constexpr long long kFmWaitLimit = 4000000000LL;  // about two seconds at 2 GHz

__device__ __forceinline__ void load_record_shared(const float *rf, int rec, float m[4])
{
  const float4 v = reinterpret_cast<const float4 *>(rf)[rec];
  m[0] = v.x, m[1] = v.y, m[2] = v.z, m[3] = v.w;
}
__device__ __forceinline__ void load_record_shared(const double *rf, int rec, double m[4])
{
  const double2 *q = reinterpret_cast<const double2 *>(rf) + 2 * rec;
  const double2 u = q[0], v = q[1];
  m[0] = u.x, m[1] = u.y, m[2] = v.x, m[3] = v.y;
}

// One work unit (group g, chunk c of its separations) of a warp.  The warp's
// mbarriers keep counting phases across its units: chunk k of this unit is
// the warp's chunk kbase + k (stage (kbase + k) % kFmStages).  Returns false
// when a wait gave up.
template <bool COEF, typename R, class Pos>
__device__ __forceinline__ bool fragmem_unit_bulk_t(int w, const FMSlices<R> &t, const double *sig, int n,
                                                    const Pos &pos, unsigned long long *facc,
                                                    unsigned long long *e_acc, int e_stride, int *timed_out,
                                                    unsigned char *wsm, unsigned &kbase)
{
  const int lane = threadIdx.x & 31;
  const int g = w / t.dsplit, c = w - g * t.dsplit;
  const int d0 = c * t.nd / t.dsplit, d1 = (c + 1) * t.nd / t.dsplit;
  const int i = g * 32 + lane;
  const bool live = i < n;
  const int ii = live ? i : n - 1;
  const bool coef = COEF;
  const int stage_bytes = fm_stage_bytes<R>(coef);
  const uint32_t bars = smem_addr(wsm), data = bars + 128;
  // the warp's run of stripes: its non-empty blocks, contiguous from the first
  int first = -1, total = 0;
  for (int dd = d0; dd < d1; dd++) {
    const int len = t.slen[g * t.nd + dd];
    if (len > 0 && first < 0) first = t.soff[g * t.nd + dd];
    total += len;
  }
  if (total <= 0) return true;
  const int last = first + total, nchunks = (total + kFmStripes - 1) / kFmStripes;
  auto issue = [&](int k) {  // lane 0: chunk k into stage (kbase + k) % kFmStages
    const int st = (kbase + k) % kFmStages, s0 = first + k * kFmStripes, ns = min(kFmStripes, last - s0);
    const uint32_t bar = bars + 8 * st, dst = data + st * stage_bytes;
    const uint32_t rb = ns * 32 * 4 * sizeof(R), cb = coef ? ns * 32 * sizeof(R) : 0;
    // the stage was last read through the generic proxy: order that before the async-proxy write
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect(bar, rb + cb + t.hold_tx);
    bulk_load(dst, t.rf + (size_t) s0 * 32 * 4, rb, bar);
    if (coef) bulk_load(dst + kFmStripes * 32 * 4 * sizeof(R), t.coef + (size_t) s0 * 32, cb, bar);
  };
  if (lane == 0)
    for (int k = 0; k < kFmStages && k < nchunks; k++) issue(k);

  const V3<double> ca_i = pos(ii, 0), cb_i = pos(ii, 1);
  long long fca[3] = {0, 0, 0}, fcb[3] = {0, 0, 0};
  double e = 0.0;
  const R scale = COEF ? R(-1) : -R(t.uniform);
  // current row (block d): geometry and sums
  int d = d0, blk_end = 0, j = 0;
  V3<R> dv[4];
  R r[4], s2 = 1, k2 = -1, es = 0, fs[4] = {0, 0, 0, 0}, es1 = 0, fs1[4] = {0, 0, 0, 0};
  auto begin_row = [&]() {  // d: the next non-empty block at or after d
    while (d < d1 && t.slen[g * t.nd + d] == 0) d++;
    if (d >= d1) return;
    blk_end = t.soff[g * t.nd + d] - first + t.slen[g * t.nd + d];
    j = min(ii + t.min_sep + d, n - 1);
    const V3<double> ca_j = pos(j, 0), cb_j = pos(j, 1);
    dv[0] = diff<R>(ca_i, ca_j);
    dv[1] = diff<R>(ca_i, cb_j);
    dv[2] = diff<R>(cb_i, ca_j);
    dv[3] = diff<R>(cb_i, cb_j);
#pragma unroll
    for (int k = 0; k < 4; k++) r[k] = m_sqrt(norm2(dv[k]));
    s2 = R(sig[t.min_sep + d]);
    k2 = fm_k2(s2);
    es = es1 = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) fs[k] = fs1[k] = 0;
  };
  auto end_row = [&]() {
    es = es + es1;
#pragma unroll
    for (int k = 0; k < 4; k++) fs[k] = fs[k] + fs1[k];
    e += (double) (scale * es);
    long long fja[3] = {0, 0, 0}, fjb[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const R fc = fs[k] != R(0) ? (scale * fs[k]) / (s2 * r[k]) : R(0);
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
    d++;
  };
  begin_row();
  bool ok = true;
  int fail_k = 0;
  for (int k = 0; k < nchunks; k++) {
    const int st = (kbase + k) % kFmStages;
    // the warp gives up together (every lane polls the same barrier)
    if (!__all_sync(0xffffffffu, mbar_wait(bars + 8 * st, ((kbase + k) / kFmStages) & 1, t.wait_limit))) {
      ok = false;
      fail_k = k;
      break;
    }
    const unsigned char *sd = wsm + 128 + st * stage_bytes;
    const R *srf = reinterpret_cast<const R *>(sd);
    const R *scf = reinterpret_cast<const R *>(sd + kFmStripes * 32 * 4 * sizeof(R));
    const int s0 = k * kFmStripes, ns = min(kFmStripes, total - s0);
    for (int q = 0; q < ns;) {
      while (s0 + q >= blk_end && d < d1) {  // rows end on stripe boundaries
        end_row();
        begin_row();
      }
      // the stripes of this chunk that belong to the current row (rows,
      // chunks and their ends fall on even stripes: records pair up as in
      // the register path)
      const int run = max(q + 2, min(ns, blk_end - s0));
#pragma unroll(sizeof(R) == 4 ? 2 : 1)
      for (; q < run; q += 2) {
        R rec[4], rec1[4];
        load_record_shared(srf, q * 32 + lane, rec);
        load_record_shared(srf, (q + 1) * 32 + lane, rec1);
        fm_record<COEF>(rec, COEF ? scf[q * 32 + lane] : R(1), r, k2, es, fs);
        fm_record<COEF>(rec1, COEF ? scf[(q + 1) * 32 + lane] : R(1), r, k2, es1, fs1);
      }
    }
    __syncwarp();  // every lane has read the stage
    if (lane == 0 && k + kFmStages < nchunks) issue(k + kFmStages);
  }
  if (!ok) {
    // record the failure, let the copies in flight land (bounded), skip the sums
    if (lane == 0) atomicExch(timed_out, 1);
    for (int k = fail_k; k < nchunks && k < fail_k + kFmStages; k++)
      mbar_wait(bars + 8 * ((kbase + k) % kFmStages), ((kbase + k) / kFmStages) & 1, kFmWaitLimit / 8);
    return false;
  }
  kbase += nchunks;
  end_row();
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
  return true;
}

template <typename R, class Pos>
__device__ __forceinline__ bool fragmem_unit_bulk(int w, const FMSlices<R> &t, const double *sig, int n,
                                                  const Pos &pos, unsigned long long *facc,
                                                  unsigned long long *e_acc, int e_stride, int *timed_out,
                                                  unsigned char *wsm, unsigned &kbase)
{
  return t.coef ? fragmem_unit_bulk_t<true>(w, t, sig, n, pos, facc, e_acc, e_stride, timed_out, wsm, kbase)
                : fragmem_unit_bulk_t<false>(w, t, sig, n, pos, facc, e_acc, e_stride, timed_out, wsm, kbase);
}

// A warp's copy ring: its stage mbarriers, initialised once (the phase
// count then runs on across the warp's units through kbase).
__device__ __forceinline__ void fragmem_ring_init(unsigned char *wsm)
{
  const uint32_t bars = smem_addr(wsm);
  if ((threadIdx.x & 31) == 0)
    for (int s = 0; s < kFmStages; s++) mbar_init(bars + 8 * s, 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncwarp();
}

// The kernel body: each warp takes work units one at a time from a counter
// (zero at launch), so a grid smaller than the number of units (a few blocks
// per SM) still streams at full bandwidth and leaves the rest of each SM to
// the concurrent pair passes; warps that get more of their SM take more
// units, and the launch ends within one unit of balance.
template <typename R, class Pos>
__device__ __forceinline__ void fragmem_warp_take(const FMSlices<R> &t, const double *sig, int n, const Pos &pos,
                                                  unsigned long long *facc, unsigned long long *e_acc,
                                                  int e_stride, int *timed_out, unsigned char *wsm, int *next)
{
  const int units = t.groups * t.dsplit, lane = threadIdx.x & 31;
  fragmem_ring_init(wsm);
  unsigned kbase = 0;
  while (true) {
    int u = 0;
    if (lane == 0) u = atomicAdd(next, 1);
    u = __shfl_sync(0xffffffffu, u, 0);
    if (u >= units) return;
    if (!fragmem_unit_bulk(u, t, sig, n, pos, facc, e_acc, e_stride, timed_out, wsm, kbase)) return;
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
