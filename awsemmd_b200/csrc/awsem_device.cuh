// Device-side AWSEM term evaluation (sm_100a).
//
// Every function here is templated on the geometry type R: double for the
// plain FP64 form, float for the mixed form (FP32 pair geometry, Gaussians
// and switching functions; FP64 densities, energies and integration).
//
// Accumulation that feeds the dynamics is exact and order independent:
// every force contribution is converted to 64-bit fixed point (2^-32 kcal/mol/A)
// before it is added (registers, warp shuffles or global atomics), and the
// density / xi sums use 2^-40.  Results are therefore bitwise identical no
// matter how residues are mapped to warps or which other systems share the
// launch.
//
// Formulas follow the reference fix_backbone.cpp; each function cites the
// lines it restates.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include "awsem_model.h"

namespace awsem {
namespace dev {

constexpr double F_SCALE = 4294967296.0;        // forces: 2^32
constexpr double F_UNSCALE = 1.0 / 4294967296.0;
constexpr double D_SCALE = 1099511627776.0;     // densities, xi: 2^40
constexpr double D_UNSCALE = 1.0 / 1099511627776.0;

enum Bead { B_CA = 0, B_CB = 1, B_O = 2, B_N = 3, B_H = 4, B_CP = 5, N_BEADS = 6 };

template <typename R> struct R4;
template <> struct R4<double> { typedef double4 T; };
template <> struct R4<float> { typedef float4 T; };

template <typename R> struct V3 {
  R x, y, z;
};

template <typename R> __device__ __forceinline__ V3<R> sub(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }

// r^2 without FMA contraction in FP64, so threshold tests see the same value
// as the reference's `dx0*dx0 + dx1*dx1 + dx2*dx2` on x86-64.
__device__ __forceinline__ double norm2(V3<double> d)
{
  return __dadd_rn(__dadd_rn(__dmul_rn(d.x, d.x), __dmul_rn(d.y, d.y)), __dmul_rn(d.z, d.z));
}
// FP32: the multiply-adds are spelled out, so every kernel that inlines this
// (the per-pass kernels and the persistent step kernel) rounds identically.
__device__ __forceinline__ float norm2(V3<float> d)
{
  return __fmaf_rn(d.z, d.z, __fmaf_rn(d.y, d.y, __fmul_rn(d.x, d.x)));
}

__device__ __forceinline__ double dot(V3<double> a, V3<double> b)
{
  return __dadd_rn(__dadd_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)), __dmul_rn(a.z, b.z));
}
__device__ __forceinline__ float dot(V3<float> a, V3<float> b)
{
  return __fmaf_rn(a.z, b.z, __fmaf_rn(a.y, b.y, __fmul_rn(a.x, b.x)));
}

// c + a * b with one rounding, in either form: accumulations whose
// contraction would otherwise be left to the compiler
__device__ __forceinline__ double madd(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float madd(float a, float b, float c) { return __fmaf_rn(a, b, c); }

template <typename R> __device__ __forceinline__ V3<R> cross(V3<R> a, V3<R> b)
{
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

__device__ __forceinline__ double m_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float m_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double m_exp(double x) { return exp(x); }
__device__ __forceinline__ float m_exp(float x) { return expf(x); }
__device__ __forceinline__ double m_fastexp(double x) { return exp(x); }
__device__ __forceinline__ float m_fastexp(float x) { return __expf(x); }
__device__ __forceinline__ double m_tanh(double x) { return tanh(x); }
__device__ __forceinline__ float m_tanh(float x) { return tanhf(x); }
__device__ __forceinline__ double m_cos(double x) { return cos(x); }
__device__ __forceinline__ float m_cos(float x) { return cosf(x); }
__device__ __forceinline__ double m_sin(double x) { return sin(x); }
__device__ __forceinline__ float m_sin(float x) { return sinf(x); }
__device__ __forceinline__ double m_atan2(double y, double x) { return atan2(y, x); }
__device__ __forceinline__ float m_atan2(float y, float x) { return atan2f(y, x); }

__device__ __forceinline__ long long fix_force(double v) { return __double2ll_rn(v * F_SCALE); }
__device__ __forceinline__ long long fix_dens(double v) { return __double2ll_rn(v * D_SCALE); }

// Device views of one system batch.  Residues are numbered globally; chain
// boundaries (res_flags, chain_start/end) keep index arithmetic inside a
// chain, and `res_chain` is globally unique so different systems never
// match as "same chain".
// A block's shared-memory force accumulator over residues [r0, r0 + n) in
// the facc layout ([residue][bead][3], 2^-32 fixed point); n == 0: none.
struct ForceWindow {
  uint32_t addr;  // shared-state-space address
  int r0, n;
};

template <typename R> struct DevSys {
  int n_res;
  const int *res_type, *res_flags, *res_chain, *chain_start, *chain_end;
  const double *aps;    // [12][n_res]
  const double *tables; // TB_SIZE
  const double4 *pos;            // [n_res][6] working coordinates (FP64 in both forms)
  const double4 *cpos;           // [n_res] contact bead (CB, CA for glycine), a copy k_prepare writes
  unsigned long long *facc;      // [n_res*3][3] fixed-point forces
  ForceWindow win;               // residues whose forces the block sums in shared memory first
};

// The same system viewed with FP64 geometry (the storage is type independent).
template <typename R> __device__ __forceinline__ DevSys<double> widen(const DevSys<R> &s)
{
  DevSys<double> d;
  d.n_res = s.n_res;
  d.res_type = s.res_type;
  d.res_flags = s.res_flags;
  d.res_chain = s.res_chain;
  d.chain_start = s.chain_start;
  d.chain_end = s.chain_end;
  d.aps = s.aps;
  d.tables = s.tables;
  d.pos = s.pos;
  d.cpos = s.cpos;
  d.facc = s.facc;
  d.win = s.win;
  return d;
}

template <typename R> __device__ __forceinline__ V3<double> bead(const DevSys<R> &s, int r, int b)
{
  double4 q = s.pos[(size_t) r * N_BEADS + b];
  return {q.x, q.y, q.z};
}

// Bead-pair difference: formed in FP64 (exact for nearby beads), then
// rounded once to the geometry type.  The mixed form's FP32 arithmetic
// starts here, so its error does not grow with the absolute coordinates.
template <typename R> __device__ __forceinline__ V3<R> diff(V3<double> a, V3<double> b)
{
  return {(R) (a.x - b.x), (R) (a.y - b.y), (R) (a.z - b.z)};
}

// Add a force to bead b of residue r: converted to fixed point first, then
// summed in the block's shared-memory window when r lies in it (flushed to
// facc by the block), else added to facc directly.
template <typename R> __device__ __forceinline__ void scatter(const DevSys<R> &s, int r, int b, R fx, R fy, R fz)
{
  const long long v[3] = {fix_force((double) fx), fix_force((double) fy), fix_force((double) fz)};
  if ((unsigned) (r - s.win.r0) < (unsigned) s.win.n) {
    const uint32_t q = s.win.addr + (uint32_t) (((r - s.win.r0) * 3 + b) * 3) * 8u;
#pragma unroll
    for (int c = 0; c < 3; c++)
      if (v[c]) asm volatile("red.shared.add.u64 [%0], %1;" ::"r"(q + 8u * c), "l"(v[c]) : "memory");
    return;
  }
  unsigned long long *p = s.facc + ((size_t) 3 * r + b) * 3;
#pragma unroll
  for (int c = 0; c < 3; c++)
    if (v[c]) atomicAdd(p + c, (unsigned long long) v[c]);
}

template <typename R> __device__ __forceinline__ void scatter(const DevSys<R> &s, int r, int b, V3<R> f)
{
  scatter(s, r, b, f.x, f.y, f.z);
}

// Density-well theta and d(theta)/dr / r (cWell::compute_theta_pair,
// smart_matrix_lib.h:612-628).
template <typename R>
__device__ __forceinline__ void well_theta(R r, R rmin_th, R rmax_th, R kappa, R rmin, R rmax, R &theta, R &prd)
{
  if (r < rmin_th || r > rmax_th) {
    theta = prd = R(0);
    return;
  }
  R t_min = m_tanh(kappa * (r - rmin));
  R t_max = m_tanh(kappa * (rmax - r));
  theta = R(0.25) * (R(1) + t_min) * (R(1) + t_max);
  prd = kappa * theta * (t_max - t_min) / r;
}
// FP32 (mixed form) from two exponentials instead of two tanh.  With
// e_a = exp(-2 kappa (r - rmin)) and e_b = exp(-2 kappa (rmax - r)), the
// identity 1 + tanh(x) = 2 / (1 + exp(-2x)) gives
//   theta = 1 / ((1 + e_a)(1 + e_b)),
//   tanh(kappa (rmax - r)) - tanh(kappa (r - rmin)) = 2 (e_a - e_b) theta,
//   prd = kappa theta (t_max - t_min) / r = 2 kappa theta^2 (e_a - e_b) / r.
// Inside the support (|kappa (r - edge)| <= 8 ln 10) the exponentials stay
// below 1e17.  Hardware 2^x and reciprocal (relative error ~1e-7); every
// operation spelled out, no contraction left to the compiler.
__device__ __forceinline__ float fast_exp2(float x)
{
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float fast_rcp(float x)
{
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
template <>
__device__ __forceinline__ void well_theta(float r, float rmin_th, float rmax_th, float kappa, float rmin, float rmax,
                                           float &theta, float &prd)
{
  if (r < rmin_th || r > rmax_th) {
    theta = prd = 0.f;
    return;
  }
  const float c = __fmul_rn(-2.8853900817779268f, kappa);  // -2 kappa log2(e)
  const float ea = fast_exp2(__fmul_rn(c, __fsub_rn(r, rmin)));
  const float eb = fast_exp2(__fmul_rn(c, __fsub_rn(rmax, r)));
  theta = fast_rcp(__fmul_rn(__fadd_rn(1.f, ea), __fadd_rn(1.f, eb)));
  prd = __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(2.f, kappa), __fmul_rn(theta, theta)), __fsub_rn(ea, eb)),
                  fast_rcp(r));
}

// compute_chain_potential(i), fix_backbone.cpp:2062-2170
template <typename R> __device__ R chain_term(const DevSys<R> &s, const FFParams &p, int i)
{
  int fl = s.res_flags[i];
  R E = 0;
  V3<double> n = bead(s, i, B_N), cb = bead(s, i, B_CB), cpv = bead(s, i, B_CP);
  const R an = p.an, bn = p.bn, cn = p.cn, ap = p.ap, bp = p.bp, cp = p.cp;
  if (!(fl & R_FIRST) && !(fl & R_GLY)) {
    V3<R> d = diff<R>(n, cb);
    R r = m_sqrt(norm2(d)), dr = r - R(p.r_ncb0);
    R f = R(2) * R(p.k_chain[0]) * dr / r;
    E += R(p.k_chain[0]) * dr * dr;
    scatter(s, i - 1, B_CA, -an * d.x * f, -an * d.y * f, -an * d.z * f);
    scatter(s, i - 1, B_O, -cn * d.x * f, -cn * d.y * f, -cn * d.z * f);
    scatter(s, i, B_CA, -bn * d.x * f, -bn * d.y * f, -bn * d.z * f);
    scatter(s, i, B_CB, d.x * f, d.y * f, d.z * f);
  }
  if (!(fl & R_LAST) && !(fl & R_GLY)) {
    V3<R> d = diff<R>(cpv, cb);
    R r = m_sqrt(norm2(d)), dr = r - R(p.r_cpcb0);
    R f = R(2) * R(p.k_chain[1]) * dr / r;
    E += R(p.k_chain[1]) * dr * dr;
    scatter(s, i + 1, B_CA, -bp * d.x * f, -bp * d.y * f, -bp * d.z * f);
    scatter(s, i, B_CA, -ap * d.x * f, -ap * d.y * f, -ap * d.z * f);
    scatter(s, i, B_O, -cp * d.x * f, -cp * d.y * f, -cp * d.z * f);
    scatter(s, i, B_CB, d.x * f, d.y * f, d.z * f);
  }
  if (!(fl & R_FIRST) && !(fl & R_LAST)) {
    V3<R> d = diff<R>(n, cpv);
    R r = m_sqrt(norm2(d)), dr = r - R(p.r_ncp0);
    R f = R(2) * R(p.k_chain[2]) * dr / r;
    E += R(p.k_chain[2]) * dr * dr;
    scatter(s, i - 1, B_CA, -an * d.x * f, -an * d.y * f, -an * d.z * f);
    scatter(s, i - 1, B_O, -cn * d.x * f, -cn * d.y * f, -cn * d.z * f);
    scatter(s, i + 1, B_CA, bp * d.x * f, bp * d.y * f, bp * d.z * f);
    R q = bn - ap;
    scatter(s, i, B_CA, -q * d.x * f, -q * d.y * f, -q * d.z * f);
    scatter(s, i, B_O, cp * d.x * f, cp * d.y * f, cp * d.z * f);
  }
  return E;
}

// compute_chi_potential(i), fix_backbone.cpp:2239-2339
template <typename R> __device__ R chi_term(const DevSys<R> &s, const FFParams &p, int i)
{
  V3<double> ca = bead(s, i, B_CA);
  V3<R> a = diff<R>(bead(s, i, B_CP), ca), b = diff<R>(ca, bead(s, i, B_N)), c = diff<R>(ca, bead(s, i, B_CB));
  R arv = R(1) / dot(a, a), brv = R(1) / dot(b, b), crv = R(1) / dot(c, c);
  R norm = m_sqrt(arv * brv * crv);
  V3<R> axb = cross(a, b), cxa = cross(c, a), bxc = cross(b, c);
  R chi = dot(axb, c) * norm;
  V3<R> ap_ = {norm * bxc.x - arv * chi * a.x, norm * bxc.y - arv * chi * a.y, norm * bxc.z - arv * chi * a.z};
  V3<R> bp_ = {norm * cxa.x - brv * chi * b.x, norm * cxa.y - brv * chi * b.y, norm * cxa.z - brv * chi * b.z};
  V3<R> cp_ = {norm * axb.x - crv * chi * c.x, norm * axb.y - crv * chi * c.y, norm * axb.z - crv * chi * c.z};
  R dchi = chi - R(p.chi0);
  R f = R(2) * R(p.k_chi) * dchi;
  const R an = p.an, bn = p.bn, cn = p.cn, ap = p.ap, bp = p.bp, cp = p.cp;
  scatter(s, i - 1, B_CA, an * bp_.x * f, an * bp_.y * f, an * bp_.z * f);
  scatter(s, i - 1, B_O, cn * bp_.x * f, cn * bp_.y * f, cn * bp_.z * f);
  scatter(s, i + 1, B_CA, -bp * ap_.x * f, -bp * ap_.y * f, -bp * ap_.z * f);
  scatter(s, i, B_CA, -(cp_.x + (R(1) - bn) * bp_.x + (ap - R(1)) * ap_.x) * f,
          -(cp_.y + (R(1) - bn) * bp_.y + (ap - R(1)) * ap_.y) * f,
          -(cp_.z + (R(1) - bn) * bp_.z + (ap - R(1)) * ap_.z) * f);
  scatter(s, i, B_O, -cp * ap_.x * f, -cp * ap_.y * f, -cp * ap_.z * f);
  scatter(s, i, B_CB, cp_.x * f, cp_.y * f, cp_.z * f);
  return R(p.k_chi) * dchi * dchi;
}

// calcDihedralAndSlopes, fix_backbone.cpp:2341-2453.  Slopes of the five
// real atoms CA(i-1), CA(i), CA(i+1), O(i-1), O(i), y and x parts summed.
// The angle is atan2(Y, X); it is returned as its cosine X / |(X, Y)| and
// sine Y / |(X, Y)| (cos 0 = 1, sin 0 = 0 when X = Y = 0, as atan2(0, 0) = 0).
template <typename R>
__device__ void dihedral(const DevSys<R> &s, const FFParams &p, int i, int phi, R &cang, R &sang, V3<R> sl[5])
{
  V3<R> a, b, c;
  V3<double> ca = bead(s, i, B_CA), n = bead(s, i, B_N), cpv = bead(s, i, B_CP);
  if (phi) {
    a = diff<R>(cpv, ca);
    b = diff<R>(ca, n);
    c = diff<R>(n, bead(s, i - 1, B_CP));
  } else {
    a = diff<R>(bead(s, i + 1, B_N), cpv);
    b = diff<R>(cpv, ca);
    c = diff<R>(ca, n);
  }
  R adb = dot(a, b), bdc = dot(b, c), adc = dot(a, c), b2 = dot(b, b), bm = m_sqrt(b2);
  V3<R> bxa = cross(b, a), cxa = cross(c, a), cxb = cross(c, b);
  R cdbxa = dot(c, bxa);
  R Y = bm * cdbxa, X = adb * bdc - b2 * adc;
  const R h2 = X * X + Y * Y;
  if (h2 > R(0)) {
    const R h = m_sqrt(h2);
    cang = X / h;
    sang = Y / h;
  } else {
    cang = R(1);
    sang = R(0);
  }
  R inv = R(1) / h2;
  R dy = X * inv, dx = -Y * inv;
  b2 *= dx;
  adb *= dx;
  adc *= dx;
  bdc *= dx;
  cdbxa *= dy / bm;
  bm *= dy;
  const R an = p.an, bn = p.bn, cn = p.cn, ap = p.ap, bp = p.bp, cp = p.cp;
  R A[3] = {a.x, a.y, a.z}, Bv[3] = {b.x, b.y, b.z}, C[3] = {c.x, c.y, c.z};
  R BXA[3] = {bxa.x, bxa.y, bxa.z}, CXA[3] = {cxa.x, cxa.y, cxa.z}, CXB[3] = {cxb.x, cxb.y, cxb.z};
  R out[5][3];
  for (int l = 0; l < 3; l++) {
    R h1, h2, h3, h4, y0, y1, y2, y3, y4;
    if (phi) {
      h1 = CXB[l] * bm;
      h2 = CXA[l] * bm;
      h3 = BXA[l] * bm;
      h4 = Bv[l] * cdbxa;
      y0 = -an * h4 + (an - ap) * h3 + an * h2;
      y1 = (R(1) - bn) * h4 + (bn - bp) * h3 + (ap - R(1)) * h1 - (R(1) - bn) * h2;
      y2 = bp * h1;
      y3 = -cn * h4 + (cn - cp) * h3 + cn * h2;
      y4 = cp * h1;
      h1 = Bv[l] * bdc - C[l] * b2;
      h2 = A[l] * bdc - R(2) * Bv[l] * adc + C[l] * adb;
      h3 = Bv[l] * adb - A[l] * b2;
      out[0][l] = y0 + (-an * h2 + (an - ap) * h3);
      out[1][l] = y1 + ((ap - R(1)) * h1 + (R(1) - bn) * h2 + (bn - bp) * h3);
      out[2][l] = y2 + bp * h1;
      out[3][l] = y3 + (-cn * h2 + (cn - cp) * h3);
      out[4][l] = y4 + cp * h1;
    } else {
      h1 = BXA[l] * bm;
      h2 = CXB[l] * bm;
      h3 = CXA[l] * bm;
      h4 = Bv[l] * cdbxa;
      y0 = -an * h1;
      y1 = (ap - R(1)) * h4 + (R(1) - bn) * h1 + (an - ap) * h2 - (ap - R(1)) * h3;
      y2 = bp * h4 + (bn - bp) * h2 - bp * h3;
      y3 = -cn * h1;
      y4 = cp * h4 + (cn - cp) * h2 - cp * h3;
      h1 = Bv[l] * bdc - C[l] * b2;
      h2 = A[l] * bdc - R(2) * Bv[l] * adc + C[l] * adb;
      h3 = Bv[l] * adb - A[l] * b2;
      out[0][l] = y0 + (-an * h3);
      out[1][l] = y1 + ((an - ap) * h1 + (ap - R(1)) * h2 + (R(1) - bn) * h3);
      out[2][l] = y2 + ((bn - bp) * h1 + bp * h2);
      out[3][l] = y3 + (-cn * h3);
      out[4][l] = y4 + ((cn - cp) * h1 + cp * h2);
    }
  }
  for (int k = 0; k < 5; k++) sl[k] = {out[k][0], out[k][1], out[k][2]};
}

// compute_rama_potential + compute_rama_force, fix_backbone.cpp:2455-2546
// cos(phi + phi0) and sin(phi + phi0) by the angle-sum identities from the
// dihedral's own cosine and sine and the well's constant cos / sin phi0,
// instead of an atan2 and four trigonometric calls per well.
template <typename R> __device__ R rama_term(const DevSys<R> &s, const FFParams &p, int i)
{
  R cf, sf, cs, ss;
  V3<R> sphi[5], spsi[5];
  dihedral(s, p, i, 1, cf, sf, sphi);
  dihedral(s, p, i, 0, cs, ss, spsi);
  int j0 = 0, j1 = p.n_rama;
  if ((s.res_flags[i] & R_PRO) && (p.terms & T_RAMA_P)) {
    j0 = 6;
    j1 = 6 + p.n_rama_p;
  }
  R E = 0, g0 = 0, g1 = 0;
  for (int j = j0; j < j1; j++) {
    double aps = s.aps[(size_t) j * s.n_res + i];
    if (p.ssweight[j] && aps == 0.0) continue;
    const R c0 = R(p.cphi0[j]), s0 = R(p.sphi0[j]), c1 = R(p.cpsi0[j]), s1 = R(p.spsi0[j]);
    R cphi = (cf * c0 - sf * s0) - R(1);
    R cpsi = (cs * c1 - ss * s1) - R(1);
    R pc = R(p.phiw[j]) * cphi, sc = R(p.psiw[j]) * cpsi;
    R V = R(p.w[j]) * m_exp(-cphi * pc - cpsi * sc);
    if (p.ssweight[j]) V *= R(aps);
    R f = R(2) * V;
    g0 += f * pc * (sf * c0 + cf * s0);
    g1 += f * sc * (ss * c1 + cs * s1);
    E += -V;
  }
  if (g0 != R(0) || g1 != R(0)) {
    const int rr[5] = {i - 1, i, i + 1, i - 1, i};
    const int bb[5] = {B_CA, B_CA, B_CA, B_O, B_O};
    for (int k = 0; k < 5; k++)
      scatter(s, rr[k], bb[k], g0 * sphi[k].x + g1 * spsi[k].x, g0 * sphi[k].y + g1 * spsi[k].y,
              g0 * sphi[k].z + g1 * spsi[k].z);
  }
  return E;
}

// compute_helix_dtheta_pair(i, j = i + helix_i_diff), fix_backbone.cpp:3706-3785.
// Returns the energy; writes the density-derivative coefficients xi1, xi2.
template <typename R>
__device__ R helix_pair(const DevSys<R> &s, const FFParams &p, int i, int j, double sh_i, double shp_i, double sh_j,
                        double shp_j, double &xi1, double &xi2, unsigned *gate = nullptr)
{
  V3<double> oi = bead(s, i, B_O);
  V3<R> xNO = diff<R>(oi, bead(s, j, B_N)), xHO = diff<R>(oi, bead(s, j, B_H));
  R R_NO = m_sqrt(norm2(xNO));
  if (R_NO > R(p.helix_cutoff)) return R(0);
  if (gate) *gate = 1u;
  R R_HO = m_sqrt(norm2(xHO));
  const double *T = s.tables;
  (void) T;
  int ti = s.res_type[i], tj = s.res_type[j];
  R h4i = R(p.h4prob[ti]);
  if ((s.res_flags[i] & R_PRO) && p.pro_acc_flag) h4i = R(p.h4prob_pro);
  R prob_sum = h4i + R(p.h4prob[tj]);
  R dNO = R_NO - R(p.helix_NO_zero), dHO = R_HO - R(p.helix_HO_zero);
  R dNOs = dNO * R(p.helix_sigma_NO_sqinv), dHOs = dHO * R(p.helix_sigma_HO_sqinv);
  R pair_theta = -R(p.k_helix) * prob_sum * m_exp(R(-0.5) * (dNO * dNOs + dHO * dHOs));
  R prd0 = -dNOs / R_NO, prd1 = -dHOs / R_HO;
  double gw = p.helix_gamma_w - p.helix_gamma_p;
  R sigma_gamma = R(p.helix_gamma_p + gw * sh_i * sh_j);
  xi1 = gw * (double) pair_theta * shp_i * sh_j;
  xi2 = gw * (double) pair_theta * sh_i * shp_j;
  R V = sigma_gamma * pair_theta;
  const R an = p.an, bn = p.bn, cn = p.cn, ah = p.ah, bh = p.bh, ch = p.ch;
  scatter(s, j - 1, B_CA, V * (an * prd0 * xNO.x + ah * prd1 * xHO.x), V * (an * prd0 * xNO.y + ah * prd1 * xHO.y),
          V * (an * prd0 * xNO.z + ah * prd1 * xHO.z));
  scatter(s, j, B_CA, V * (bn * prd0 * xNO.x + bh * prd1 * xHO.x), V * (bn * prd0 * xNO.y + bh * prd1 * xHO.y),
          V * (bn * prd0 * xNO.z + bh * prd1 * xHO.z));
  scatter(s, j - 1, B_O, V * (cn * prd0 * xNO.x + ch * prd1 * xHO.x), V * (cn * prd0 * xNO.y + ch * prd1 * xHO.y),
          V * (cn * prd0 * xNO.z + ch * prd1 * xHO.z));
  scatter(s, i, B_O, -V * (prd0 * xNO.x + prd1 * xHO.x), -V * (prd0 * xNO.y + prd1 * xHO.y),
          -V * (prd0 * xNO.z + prd1 * xHO.z));
  return V;
}

// compute_dssp_hdrgn(i, j): O of residue i, N-H of residue j.
// fix_backbone.cpp:2902-3277.  Returns the energy and scatters the forces;
// *gate (optional) receives the gates passed: bit 0 r_NO <= cutoff (:2904),
// bit 1 both nu switches >= 1e-4 (:3052).
template <typename R> __device__ R dssp_term(const DevSys<R> &s, const FFParams &p, int i, int j,
                                             unsigned *gate = nullptr)
{
  V3<double> oi = bead(s, i, B_O);
  R rno = m_sqrt(norm2(diff<R>(oi, bead(s, j, B_N))));
  if (rno > R(p.dssp_cut)) return R(0);
  if (gate) *gate = 1u;
  const int *fl = s.res_flags, *ty = s.res_type;
  int ic = s.res_chain[i], jc = s.res_chain[j];
  int i_start = s.chain_start[ic], i_end = s.chain_end[ic];
  int j_start = s.chain_start[jc], j_end = s.chain_end[jc];
  bool jlast = fl[j] & R_LAST;
  bool i_rep = !(jlast || (fl[j + 1] & R_PRO));
  bool i_AP = !((fl[i] & R_FIRST) || jlast || (fl[i] & R_PRO));
  // reference: i_resno >= i_ch_end-2 with a 1-based chain end
  bool i_P = !(i >= i_end - 1 || jlast || (fl[i + 2] & R_PRO));
  const double *T = s.tables;
  auto aHB = [&](int a, int b, int k) { return T[TB_ANTI_HB + (ty[a] * 20 + ty[b]) * 2 + k]; };
  auto aNHB = [&](int a, int b, int k) { return T[TB_ANTI_NHB + (ty[a] * 20 + ty[b]) * 2 + k]; };
  auto pHB = [&](int a, int b, int k) { return T[TB_PARA_HB + (ty[a] * 20 + ty[b]) * 2 + k]; };
  auto p1 = [&](int a) { return T[TB_PARA_ONE + ty[a]]; };
  auto a1 = [&](int a) { return T[TB_ANTI_ONE + ty[a]]; };
  double tsa[2] = {0, 0}, tsn[2] = {0, 0}, tsp[2] = {0, 0};
  for (int k = 0; k < 2; k++) {
    if (i_AP) {
      tsa[k] = 0.5 * aHB(i, j, k);
      tsn[k] = 0.25 * (aNHB(i + 1, j - 1, k) + aNHB(i - 1, j + 1, k));
    }
    if (i_P) tsp[k] = pHB(i + 1, j, k);
  }
  double lam[4];
  int hb_class;
  int dij = abs(j - i);
  if (ic == jc && dij < 45) {
    if (dij < 4) {
      lam[0] = -p.hbscl[0][0];
      lam[1] = -p.hbscl[0][1];
      lam[2] = lam[3] = 0.0;
      hb_class = 1;
    } else if (dij < 18) {
      const double *beta = s.aps + (size_t) (p.n_rama - 1) * s.n_res;
      if (p.n_rama > 0 && beta[i] == 1.0 && beta[j] == 1.0) {
        lam[0] = -p.hbscl[1][0];
        lam[1] = -p.hbscl[1][1];
        lam[2] = -p.hbscl[1][2] - p.hbscl[1][3] * tsa[0] - p.hbscl[1][4] * tsn[0] - p.hbscl[1][5] * (a1(i) + a1(j));
        lam[3] = -p.hbscl[1][6];
      } else {
        lam[0] = 0.0;
        lam[1] = -p.hbscl[1][1];
        lam[2] = lam[3] = 0.0;
      }
      hb_class = 2;
    } else {
      lam[0] = -p.hbscl[2][0];
      lam[1] = -p.hbscl[2][1];
      lam[2] = -p.hbscl[2][2] - p.hbscl[2][3] * tsa[1] - p.hbscl[2][4] * tsn[1] - p.hbscl[2][5] * (a1(i) + a1(j));
      lam[3] = -p.hbscl[2][6] - p.hbscl[2][7] * tsp[1] - p.hbscl[2][8] * (p1(i + 1) + p1(j));
      hb_class = 3;
    }
  } else {
    lam[0] = -p.hbscl[3][0];
    lam[1] = -p.hbscl[3][1];
    lam[2] = -p.hbscl[3][2] - p.hbscl[3][3] * tsa[1] - p.hbscl[3][4] * tsn[1] - p.hbscl[3][5] * (a1(i) + a1(j));
    lam[3] = -p.hbscl[3][6] - p.hbscl[3][7] * tsp[1] - p.hbscl[3][8] * (p1(i + 1) + p1(j));
    hb_class = 4;
  }
  // nu switches on CA(c-2)..CA(c+2); reference bounds use 1-based chain ends
  bool use_nu[2] = {i - 2 >= i_start && i + 2 <= i_end && hb_class != 2,
                    j - 2 >= j_start && j + 2 <= j_end && hb_class != 2};
  R nu[2], prdnu[2];
  V3<R> dxnu[2];
  int cen[2] = {i, j};
  for (int q = 0; q < 2; q++) {
    nu[q] = prdnu[q] = R(0);
    if (use_nu[q]) {
      int c = cen[q];
      dxnu[q] = diff<R>(bead(s, c + 2, B_CA), bead(s, c - 2, B_CA));
      R rn = norm2(dxnu[q]);
      if (rn > R(p.nu_cut_sq[q])) {
        rn = m_sqrt(rn);
        R th = m_tanh(R(p.pref[q]) * (rn - R(p.d_nu0)));
        nu[q] = R(0.5) * (R(1) + th);
        prdnu[q] = R(p.pref[q]) * nu[q] * (R(1) - th) / rn;
      }
    } else {
      nu[q] = R(1);
    }
  }
  if (nu[0] < R(1e-4) || nu[1] < R(1e-4)) return R(0);
  if (gate) *gate = 3u;
  bool on[4] = {true, i_rep, i_AP, i_P};
  const int acc[4] = {i, i, j, j}, don[4] = {j, j + 1, i, i + 2};
  R theta[4], prd[4][2];
  V3<R> xNO[4], xHO[4];
  for (int k = 0; k < 4; k++) {
    theta[k] = prd[k][0] = prd[k][1] = R(0);
    if (!on[k]) continue;
    V3<double> o = bead(s, acc[k], B_O);
    xNO[k] = diff<R>(o, bead(s, don[k], B_N));
    xHO[k] = diff<R>(o, bead(s, don[k], B_H));
    R rn = m_sqrt(norm2(xNO[k])), rh = m_sqrt(norm2(xHO[k]));
    R dn = (rn - R(p.NO_zero)) * R(p.sigma_NO_sqinv), dh = (rh - R(p.HO_zero)) * R(p.sigma_HO_sqinv);
    theta[k] = m_exp(R(-0.5) * ((rn - R(p.NO_zero)) * dn + (rh - R(p.HO_zero)) * dh));
    prd[k][0] = -dn / rn;
    prd[k][1] = -dh / rh;
  }
  R ff1 = R(p.k_dssp) * theta[0];
  R V[4] = {R(lam[0]), R(lam[1]) * theta[1], R(lam[2]) * theta[2], R(lam[3]) * theta[3]};
  R theta_sum = ff1 * (V[0] + V[1] + V[2] + V[3]);
  ff1 *= nu[0] * nu[1];
  for (int k = 0; k < 4; k++) V[k] *= ff1;
  R VT = V[0] + V[1] + V[2] + V[3];
  // Beads that several contributions reach are summed here first, in this
  // fixed order, and scattered once: O(i) (acceptor of k = 0, 1), O(j)
  // (O(d - 1) of k = 1, acceptor of k = 2, 3), CA(j) (CA(d) of k = 0,
  // CA(d - 1) of k = 1) and CA(i + 2) (CA(d) of k = 3, the nu switch of i).
  V3<R> fOi = {R(0), R(0), R(0)}, fOj = fOi, fCAj = fOi, fCAi2 = fOi;
  auto add = [](V3<R> &t, R x, R y, R z) { t = {t.x + x, t.y + y, t.z + z}; };
  for (int q = 0; q < 2; q++) {
    if (!use_nu[q]) continue;
    R g = q == 0 ? theta_sum * prdnu[0] * nu[1] : theta_sum * nu[0] * prdnu[1];
    int c = cen[q];
    scatter(s, c - 2, B_CA, g * dxnu[q].x, g * dxnu[q].y, g * dxnu[q].z);
    if (q == 0)
      add(fCAi2, -g * dxnu[q].x, -g * dxnu[q].y, -g * dxnu[q].z);
    else
      scatter(s, c + 2, B_CA, -g * dxnu[q].x, -g * dxnu[q].y, -g * dxnu[q].z);
  }
  const R an = p.an, bn = p.bn, cn = p.cn, ah = p.ah, bh = p.bh, ch = p.ch;
  for (int k = 0; k < 4; k++) {
    if (!on[k]) continue;
    R sc = k == 0 ? VT : V[k];
    R q0 = prd[k][0] * sc, q1 = prd[k][1] * sc;
    V3<R> a = xNO[k], h = xHO[k];
    int d = don[k];
    const R ox = -(q0 * a.x + q1 * h.x), oy = -(q0 * a.y + q1 * h.y), oz = -(q0 * a.z + q1 * h.z);
    const R px = an * q0 * a.x + ah * q1 * h.x, py = an * q0 * a.y + ah * q1 * h.y, pz = an * q0 * a.z + ah * q1 * h.z;
    const R cx = bn * q0 * a.x + bh * q1 * h.x, cy = bn * q0 * a.y + bh * q1 * h.y, cz = bn * q0 * a.z + bh * q1 * h.z;
    const R wx = cn * q0 * a.x + ch * q1 * h.x, wy = cn * q0 * a.y + ch * q1 * h.y, wz = cn * q0 * a.z + ch * q1 * h.z;
    add(k < 2 ? fOi : fOj, ox, oy, oz);  // O of the acceptor (i for k < 2, j otherwise)
    if (k == 1)
      add(fCAj, px, py, pz);  // CA(d - 1) = CA(j)
    else
      scatter(s, d - 1, B_CA, px, py, pz);
    if (k == 0)
      add(fCAj, cx, cy, cz);  // CA(d) = CA(j)
    else if (k == 3)
      add(fCAi2, cx, cy, cz);  // CA(d) = CA(i + 2)
    else
      scatter(s, d, B_CA, cx, cy, cz);
    if (k == 1)
      add(fOj, wx, wy, wz);  // O(d - 1) = O(j)
    else
      scatter(s, d - 1, B_O, wx, wy, wz);
  }
  scatter(s, i, B_O, fOi);
  scatter(s, j, B_O, fOj);
  scatter(s, j, B_CA, fCAj);
  if (use_nu[0] || on[3]) scatter(s, i + 2, B_CA, fCAi2);
  return VT;
}

// cP_AP::compute, smart_matrix_lib.h:178-203
template <typename R> __device__ __forceinline__ void pap_nu(const DevSys<R> &s, const FFParams &p, int i, int j, R &nu, R &prd, V3<R> &d)
{
  d = diff<R>(bead(s, i, B_CA), bead(s, j, B_CA));
  R drsq = norm2(d);
  if (drsq > R(p.pap_drmax_sq)) {
    nu = prd = R(0);
  } else if (drsq < R(p.pap_drmin_sq)) {
    nu = R(1);
    prd = R(0);
  } else {
    R dr = m_sqrt(drsq);
    R th = m_tanh(R(p.pap_pref) * (R(p.pap_cut) - dr));
    nu = R(0.5) * (R(1) + th);
    prd = R(0.5) * R(p.pap_pref) * (R(1) - th * th) / dr;
  }
}

// compute_P_AP_potential(i, j) with i < j, fix_backbone.cpp:3279-3383.
// *gate (optional): bit 0 nu(i, j) >= 1e-12 (:3281), bits 1-3 the classes
// antiparallel medium, antiparallel long, parallel (:3290-3295).
template <typename R> __device__ R pap_term(const DevSys<R> &s, const FFParams &p, int i, int j,
                                            unsigned *gate = nullptr)
{
  R nu_ij, prd_ij;
  V3<R> d0;
  pap_nu(s, p, i, j, nu_ij, prd_ij, d0);
  if (nu_ij < R(1e-12)) return R(0);
  int ic = s.res_chain[i], jc = s.res_chain[j], dd = p.i_diff_pap;
  // reference chain ends are 1-based: i_ch_end = last index + 1
  int ie = s.chain_end[ic] + 1, je = s.chain_end[jc] + 1;
  bool same = ic == jc;
  bool ap_med = same && i < ie - (p.i_med_min + 2 * dd) && j >= i + (p.i_med_min + 2 * dd) &&
                j <= min(i + p.i_med_max + 2 * dd, ie - 1);
  bool ap_long = (same && i < ie - (p.i_med_max + 2 * dd + 1) && j >= i + (p.i_med_max + 2 * dd + 1) && j < je) ||
                 (!same && i + dd < s.n_res && j - dd >= 0 && s.res_chain[i + dd] == ic && s.res_chain[j - dd] == jc);
  bool par = (same && i < ie - (p.i_med_max + 1 + dd) && j >= i + (p.i_med_max + 1) && j < ie - dd) ||
             (!same && i + dd < s.n_res && j + dd < s.n_res && s.res_chain[i + dd] == ic && s.res_chain[j + dd] == jc);
  if (gate) *gate = 1u | (ap_med ? 2u : 0u) | (ap_long ? 4u : 0u) | (par ? 8u : 0u);
  const double *beta = s.aps + (size_t) (p.n_rama - 1) * s.n_res;
  bool bp = p.n_rama > 0 && beta[i] == 1.0 && beta[j] == 1.0;
  R E = 0;
  auto apply = [&](double K, int i2, int j2) {
    R nu2, prd2;
    V3<R> d1;
    pap_nu(s, p, i2, j2, nu2, prd2, d1);
    R kk = R(p.k_global_pap * K);
    E += -R(p.k_global_pap) * R(K) * nu_ij * nu2;
    R f0 = kk * prd_ij * nu2, f1 = kk * nu_ij * prd2;
    scatter(s, i, B_CA, -f0 * d0.x, -f0 * d0.y, -f0 * d0.z);
    scatter(s, j, B_CA, f0 * d0.x, f0 * d0.y, f0 * d0.z);
    scatter(s, i2, B_CA, -f1 * d1.x, -f1 * d1.y, -f1 * d1.z);
    scatter(s, j2, B_CA, f1 * d1.x, f1 * d1.y, f1 * d1.z);
  };
  if (ap_med || ap_long) {
    double K = bp ? (ap_med ? p.k_pap[0] : 0.0) + (ap_long ? p.k_pap[1] * p.k_betapred_pap : 0.0)
                  : (ap_med ? p.k_pap[0] : 0.0) + (ap_long ? p.k_pap[1] : 0.0);
    apply(K, i + dd, j - dd);
  }
  if (par) apply(bp ? p.k_pap[2] * p.k_betapred_pap : p.k_pap[2], i + dd, j + dd);
  return E;
}

template <typename T> __device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace dev
}  // namespace awsem
