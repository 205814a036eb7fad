// Per-step kernels of the AWSEM engine (sm_100a).
//
// One MD step is this chain of launches (captured into a CUDA graph):
//   prepare      thread/residue: CA, CB, O -> working copy + virtual N, H, C'
//                (fix_backbone.cpp:7067-7138); zero forces; list-check data
//   nl_decide    1 thread: rebuild decision for the residue pair list
//   nl_build     warp/residue: contact-bead pairs within the list radius
//   density      warp/residue: rho_water, rho_helix (DL1, :7728-7791)
//   residue      thread/residue: switching functions, burial (SL, :7795-7841),
//                helical (i,i+4) pairs (:7843-7868), chain/chi/rama
//   water_xi     warp/residue: xi_water (DL2, :7877-7954)
//   pair         warp/residue: water/burial/helix radial forces, excluded
//                volume (DL3, :7956-8134); queues DSSP and P_AP pairs
//   hbond        thread/queued pair: DSSP hydrogen bonds, P_AP
//   fragmem      warp/32 residues, lane/residue row: fragment-memory
//                Gaussians (:4079-4177), on a second stream
//   bonds        thread/residue: harmonic bonds
//   finish       thread/residue: fixed-point -> FP64 forces, Langevin,
//                velocity-Verlet half kicks and drift
// Residue-owned quantities are written by their owner without atomics;
// forces scattered to other residues' beads use 64-bit integer atomics.
#pragma once

#include "awsem_device.cuh"
#include "awsem_fragmem.cuh"

namespace awsem {
namespace dev {

struct NLState {
  float d2max;        // max contact-bead displacement^2 since the last build
  float bO, bN, bCA, bAll;  // max bead offsets from the contact bead
  float r_list;       // list radius of the current list
  int rebuild;        // decision for this step
  int steps_since;    // steps since the last build
  int every;          // forced rebuild period (0: displacement check only)
  int nbuilds;
  int overflow;       // max neighbour count seen when it exceeded capacity
  float skin;
  float r_contact, r_dssp, r_pap, r_ev;  // term cutoffs on the bead pairs they test
  float bCAx;         // max distance of a residue's CB or O from its own CA (this step)
  float ev_pre_sq;    // CA-CA distance^2 beyond which no bead pair of two residues is in excluded-volume range
  int n_dssp, n_pap;  // hydrogen-bond queue lengths of the current evaluation
};

template <typename R> struct StepArgs {
  DevSys<R> s;
  int n_atoms;
  const double *x;  // [n_atoms][3]
  double *v;
  const double *mass;
  const int *atom_tag;
  // per-residue pair-pass intermediates
  double *rho_w, *rho_h, *sig_w, *sigp_w, *sig_h, *sigp_h, *xi_w, *xi1, *xi2, *bur;
  double *e_res;  // [E_SLOTS][n_res]
  // residue pair list
  int *nbr, *ncount, cap;
  double4 *cb_build;
  NLState *nl;
  // hydrogen-bond work queues: list slots (residue * cap + k) of the DSSP
  // candidates in [0, n_res*cap) and of the P_AP candidates after them
  int *hbq;
  // energies summed by several threads per residue, in 2^-32 fixed point
  // (sums independent of order): [0] DSSP, [1] P_AP, [2] fragment memory
  long long *e_fix;
  // excluded volume
  int ntypes, ev_p;
  const double *ev_pref, *ev_cs, *ev_cl;
  const int *atom_type;
  const unsigned *excl_self, *excl_next;
  // bonds grouped by the residue of their first atom
  const int *bond_start, *bond_i, *bond_j;
  const double *bond_k, *bond_r0;
  // fragment memory
  FMSlices<R> fm;
  int groups;       // AWSEM_TERMS_* bits: 1 fix backbone, 2 pair vexcluded, 4 bonds
  long long *step;   // device step counter (advanced by k_nl_decide)
  // replicas: residue -> replica, replica residue ranges, Langevin seeds
  const int *res_sys, *sys_begin, *sys_end;
  const unsigned long long *sys_seed;
};

enum Group { G_FIX = 1, G_PAIR = 2, G_BOND = 4 };

__device__ __forceinline__ void atomic_max_f(float *addr, float v)
{
  // non-negative floats order like their bit patterns
  atomicMax((int *) addr, __float_as_int(v));
}

template <typename R> __global__ void k_prepare(StepArgs<R> a, FFParams p)
{
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  float d2 = 0.f, oO = 0.f, oN = 0.f, oCA = 0.f, oAll = 0.f, oX = 0.f;
  if (r < a.s.n_res) {
    const double *x = a.x;
    int fl = a.s.res_flags[r];
    double ca[3], cb[3], o[3], n[3] = {0, 0, 0}, h[3] = {0, 0, 0}, cp[3] = {0, 0, 0};
    for (int k = 0; k < 3; k++) {
      ca[k] = x[(3 * r + 0) * 3 + k];
      cb[k] = x[(3 * r + 1) * 3 + k];
      o[k] = x[(3 * r + 2) * 3 + k];
    }
    if (!(fl & R_FIRST)) {
      for (int k = 0; k < 3; k++) {
        double ca0 = x[(3 * (r - 1) + 0) * 3 + k], o0 = x[(3 * (r - 1) + 2) * 3 + k];
        n[k] = __dadd_rn(__dadd_rn(__dmul_rn(p.an, ca0), __dmul_rn(p.bn, ca[k])), __dmul_rn(p.cn, o0));
        h[k] = __dadd_rn(__dadd_rn(__dmul_rn(p.ah, ca0), __dmul_rn(p.bh, ca[k])), __dmul_rn(p.ch, o0));
      }
    }
    if (!(fl & R_LAST)) {
      for (int k = 0; k < 3; k++) {
        double ca1 = x[(3 * (r + 1) + 0) * 3 + k];
        cp[k] = __dadd_rn(__dadd_rn(__dmul_rn(p.ap, ca[k]), __dmul_rn(p.bp, ca1)), __dmul_rn(p.cp, o[k]));
      }
    }
    double4 *w = const_cast<double4 *>(a.s.pos) + (size_t) r * N_BEADS;
    w[B_CA] = make_double4(ca[0], ca[1], ca[2], 0.0);
    w[B_CB] = make_double4(cb[0], cb[1], cb[2], 0.0);
    w[B_O] = make_double4(o[0], o[1], o[2], 0.0);
    w[B_N] = make_double4(n[0], n[1], n[2], 0.0);
    w[B_H] = make_double4(h[0], h[1], h[2], 0.0);
    w[B_CP] = make_double4(cp[0], cp[1], cp[2], 0.0);
    unsigned long long *f = a.s.facc + (size_t) 9 * r;
    for (int k = 0; k < 9; k++) f[k] = 0ull;
    for (int k = 0; k < 3; k++) a.e_fix[(size_t) k * a.s.n_res + r] = 0;
    {
      // reach of the residue's beads around its CA (excluded-volume prefilter)
      double ux = cb[0] - ca[0], uy = cb[1] - ca[1], uz = cb[2] - ca[2];
      double wx = o[0] - ca[0], wy = o[1] - ca[1], wz = o[2] - ca[2];
      oX = (float) sqrt(fmax(ux * ux + uy * uy + uz * uz, wx * wx + wy * wy + wz * wz));
    }
    // list-validity data: contact-bead displacement and bead offsets
    const double *c = (fl & R_GLY) ? ca : cb;
    double4 b0 = a.cb_build[r];
    double dx = c[0] - b0.x, dy = c[1] - b0.y, dz = c[2] - b0.z;
    d2 = (float) (dx * dx + dy * dy + dz * dz);
    auto off = [&](const double *q) {
      double ex = q[0] - c[0], ey = q[1] - c[1], ez = q[2] - c[2];
      return (float) sqrt(ex * ex + ey * ey + ez * ez);
    };
    oO = off(o);
    oCA = off(ca);
    oAll = fmaxf(fmaxf(off(ca), off(cb)), off(o));
    if (!(fl & R_FIRST)) oN = off(n);
  }
  // block max, then one atomic per block
  for (int s = 16; s > 0; s >>= 1) {
    d2 = fmaxf(d2, __shfl_xor_sync(0xffffffffu, d2, s));
    oO = fmaxf(oO, __shfl_xor_sync(0xffffffffu, oO, s));
    oN = fmaxf(oN, __shfl_xor_sync(0xffffffffu, oN, s));
    oCA = fmaxf(oCA, __shfl_xor_sync(0xffffffffu, oCA, s));
    oAll = fmaxf(oAll, __shfl_xor_sync(0xffffffffu, oAll, s));
    oX = fmaxf(oX, __shfl_xor_sync(0xffffffffu, oX, s));
  }
  if ((threadIdx.x & 31) == 0) {
    atomic_max_f(&a.nl->d2max, d2);
    atomic_max_f(&a.nl->bO, oO);
    atomic_max_f(&a.nl->bN, oN);
    atomic_max_f(&a.nl->bCA, oCA);
    atomic_max_f(&a.nl->bAll, oAll);
    atomic_max_f(&a.nl->bCAx, oX);
  }
}

// Pair-list rebuild decision.  A residue pair is needed when one of its
// tested bead pairs is inside that term's cutoff; in contact-bead distance
// that is at most R_need = max(r_contact, r_dssp + bO + bN, r_pap + 2 bCA,
// r_ev + 2 bAll).  The list built at t0 with radius R_need(t0) + skin stays
// complete while R_need(t) + 2 * max displacement <= radius.
__global__ void k_nl_decide(NLState *nl, int force, long long *step)
{
  if (step) (*step)++;
  NLState &s = *nl;
  float need = fmaxf(fmaxf(s.r_contact, s.r_dssp + s.bO + s.bN), fmaxf(s.r_pap + 2.f * s.bCA, s.r_ev + 2.f * s.bAll));
  float disp = sqrtf(s.d2max);
  bool rb = force || s.r_list <= 0.f || need + 2.f * disp > s.r_list || (s.every > 0 && s.steps_since + 1 >= s.every);
  if (rb) {
    s.r_list = need + s.skin;
    s.steps_since = 0;
    s.nbuilds++;
  } else {
    s.steps_since++;
  }
  s.rebuild = rb;
  // two residues whose CAs are farther apart than r_ev + 2 * reach have no
  // bead pair inside any excluded-volume cutoff (0.01 A covers rounding)
  float pre = s.r_ev + 2.f * s.bCAx + 0.01f;
  s.ev_pre_sq = pre * pre;
  s.d2max = s.bO = s.bN = s.bCA = s.bAll = s.bCAx = 0.f;
  s.n_dssp = s.n_pap = 0;
}

template <typename R> __device__ __forceinline__ V3<double> contact(const DevSys<R> &s, int r)
{
  return bead(s, r, (s.res_flags[r] & R_GLY) ? B_CA : B_CB);
}

// Full residue pair list (both directions) over contact beads within r_list,
// written in ascending j.  Brute force over the residue's own replica, one
// warp per residue.
template <typename R> __global__ void k_nl_build(StepArgs<R> a)
{
  if (!a.nl->rebuild) return;
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  int i = warp;
  if (i >= a.s.n_res) return;
  int rep = a.res_sys[i];
  const int sys_begin = a.sys_begin[rep], sys_end = a.sys_end[rep];
  const DevSys<R> &s = a.s;
  V3<double> ci = contact(s, i);
  R rl = (R) a.nl->r_list, rl2 = rl * rl;
  int count = 0;
  int *out = a.nbr + (size_t) i * a.cap;
  for (int j0 = sys_begin; j0 < sys_end; j0 += 32) {
    int j = j0 + lane;
    bool take = false;
    if (j < sys_end && j != i) {
      V3<R> d = diff<R>(ci, contact(s, j));
      take = norm2(d) < rl2;
    }
    unsigned m = __ballot_sync(0xffffffffu, take);
    int at = count + __popc(m & ((1u << lane) - 1u));
    if (take && at < a.cap) out[at] = j;
    count += __popc(m);
  }
  if (lane == 0) {
    a.ncount[i] = min(count, a.cap);
    if (count > a.cap) atomicMax(&a.nl->overflow, count);
    a.cb_build[i] = make_double4(ci.x, ci.y, ci.z, 0.0);
  }
}

// DL1: local densities of contact beads (fix_backbone.cpp:7728-7791)
template <typename R> __global__ void k_density(StepArgs<R> a, FFParams p)
{
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  const DevSys<R> &s = a.s;
  if (i >= s.n_res) return;
  V3<double> ci = contact(s, i);
  int chi = s.res_chain[i];
  long long aw = 0, ah = 0;
  const bool fix = a.groups & G_FIX;
  int cnt = fix ? a.ncount[i] : 0;
  const int *nb = a.nbr + (size_t) i * a.cap;
  bool water = p.terms & T_WATER, helix = p.terms & T_HELIX;
  // FP64 in both forms: the densities feed the burial and switching
  // functions, and the well selection is then the reference's exactly
  for (int k = lane; k < cnt; k += 32) {
    int j = nb[k];
    if (s.res_chain[j] == chi && abs(i - j) <= 1) continue;
    V3<double> d = diff<double>(ci, contact(s, j));
    double rsq = norm2(d);
    if (water && rsq > p.w_rmin_sq[0] && rsq < p.w_rmax_sq[0]) {
      double th, pr;
      well_theta(sqrt(rsq), p.w_rmin_th[0], p.w_rmax_th[0], p.water_kappa, p.well_rmin[0], p.well_rmax[0], th, pr);
      aw += fix_dens(th);
    }
    if (helix && rsq > p.h_rmin_sq && rsq < p.h_rmax_sq) {
      double th, pr;
      well_theta(sqrt(rsq), p.h_rmin_th, p.h_rmax_th, p.helix_kappa, p.helix_rmin, p.helix_rmax, th, pr);
      ah += fix_dens(th);
    }
  }
  aw = warp_sum(aw);
  ah = warp_sum(ah);
  if (lane == 0) {
    a.rho_w[i] = (double) aw * D_UNSCALE;
    a.rho_h[i] = (double) ah * D_UNSCALE;
  }
}

__device__ __forceinline__ void switching(double rho, double kappa_sigma, double thr, double &sig, double &sigp)
{
  double th = tanh(kappa_sigma * (rho - thr));
  sig = 0.5 * (1.0 - th);
  sigp = -kappa_sigma * sig * (1.0 + th);
}

// Excluded volume between beads (PairExcludedVolume::compute,
// pair_excluded_volume.cpp:50-138).  Returns the pair energy and the force
// on bead a (the force on b is its negative).
template <typename R>
__device__ __forceinline__ R ev_pair(const StepArgs<R> &a, int ta, int tb, bool short_range, V3<R> d, V3<R> &f)
{
  int N = a.ntypes + 1;
  double pref = a.ev_pref[ta * N + tb];
  f = {R(0), R(0), R(0)};
  if (pref == 0.0) return R(0);
  R rc = (R) (short_range ? a.ev_cs[ta * N + tb] : a.ev_cl[ta * N + tb]);
  R r = m_sqrt(norm2(d));
  if (!(r < rc)) return R(0);
  R dr = r - rc;
  R pw = R(1);
  for (int k = 1; k < a.ev_p; k++) pw *= dr;  // dr^(p-1)
  R pr = R(pref) * pw;
  R fp = r > R(0) ? -pr * R(a.ev_p) / r : R(0);
  f = {d.x * fp, d.y * fp, d.z * fp};
  return pr * dr;
}

// SL and the per-residue backbone terms
template <typename R> __global__ void k_residue(StepArgs<R> a, FFParams p)
{
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  const DevSys<R> &s = a.s;
  if (i >= s.n_res) return;
  // the per-residue backbone terms (chain, chi, rama, helical pair) are a
  // small share of the work and some are sums of steep Gaussians: FP64 in
  // both forms
  const DevSys<double> sd = widen(s);
  int n = s.n_res, fl = s.res_flags[i];
  double *E = a.e_res;
  const bool fix = a.groups & G_FIX;
  bool water = fix && (p.terms & T_WATER), helix = fix && (p.terms & T_HELIX);
  double sw = 0, swp = 0, sh = 0, shp = 0;
  if (water) switching(a.rho_w[i], p.water_kappa_sigma, p.treshold, sw, swp);
  if (helix) switching(a.rho_h[i], p.helix_kappa_sigma, p.helix_treshold, sh, shp);
  a.sig_w[i] = sw;
  a.sigp_w[i] = swp;
  a.sig_h[i] = sh;
  a.sigp_h[i] = shp;
  double eb = 0.0, bc = 0.0;
  if (fix && (p.terms & T_BURIAL)) {
    double rho = a.rho_w[i];
    const double *g = s.tables + TB_BURIAL + 3 * s.res_type[i];
    double t[3][2];
    for (int k = 0; k < 3; k++) {
      t[k][0] = tanh(p.burial_kappa * (rho - p.burial_ro_min[k]));
      t[k][1] = tanh(p.burial_kappa * (p.burial_ro_max[k] - rho));
      eb += -0.5 * p.k_burial * g[k] * (t[k][0] + t[k][1]);
    }
    bc = g[0] * (t[0][1] * t[0][1] - t[0][0] * t[0][0]);
    bc += g[1] * (t[1][1] * t[1][1] - t[1][0] * t[1][0]);
    bc += g[2] * (t[2][1] * t[2][1] - t[2][0] * t[2][0]);
    bc *= 0.5 * p.k_burial * p.burial_kappa;
  }
  a.bur[i] = bc;
  E[(size_t) E_BURIAL * n + i] = eb;
  // helical (i, i+d) pair; sigma of the partner is recomputed from its density
  double x1 = 0.0, x2 = 0.0, eh = 0.0;
  int j = i + p.helix_i_diff;
  if (helix && j < n && s.res_chain[j] == s.res_chain[i]) {
    V3<R> d = diff<R>(bead(s, i, B_O), bead(s, j, B_N));
    if (norm2(d) < R(p.helix_cutoff_sq)) {
      double shj, shpj;
      switching(a.rho_h[j], p.helix_kappa_sigma, p.helix_treshold, shj, shpj);
      eh = (double) helix_pair(sd, p, i, j, sh, shp, shj, shpj, x1, x2);
    }
  }
  a.xi1[i] = x1;
  a.xi2[i] = x2;
  E[(size_t) E_HELIX * n + i] = eh;
  double ec = 0.0, ex = 0.0, er = 0.0;
  if (fix && (p.terms & T_CHAIN)) ec = (double) chain_term(sd, p, i);
  bool inner = fix && !(fl & (R_FIRST | R_LAST | R_GLY));
  if (inner && (p.terms & T_CHI)) ex = (double) chi_term(sd, p, i);
  if (inner && (p.terms & T_RAMA)) er = (double) rama_term(sd, p, i);
  E[(size_t) E_CHAIN * n + i] = ec;
  E[(size_t) E_CHI * n + i] = ex;
  E[(size_t) E_RAMA * n + i] = er;
  // excluded volume inside the residue (1-3 pairs; 1-2 pairs are excluded)
  double ev = 0.0;
  unsigned ex_self = (a.groups & G_PAIR) ? a.excl_self[i] : 0x1ffu;
  for (int b0 = 0; b0 < 3; b0++)
    for (int b1 = b0 + 1; b1 < 3; b1++) {
      if (ex_self & (1u << (b0 * 3 + b1))) continue;
      V3<R> f;
      R e = ev_pair(a, a.atom_type[3 * i + b0], a.atom_type[3 * i + b1], true,
                    diff<R>(bead(s, i, b0), bead(s, i, b1)), f);
      if (e != R(0) || f.x != R(0) || f.y != R(0) || f.z != R(0)) {
        ev += (double) e;
        scatter(s, i, b0, f);
        scatter(s, i, b1, -f.x, -f.y, -f.z);
      }
    }
  E[(size_t) E_PAIR * n + i] = ev;
}

// DL2: water-mediated density derivative coefficients (fix_backbone.cpp:7877-7954)
template <typename R> __global__ void k_water_xi(StepArgs<R> a, FFParams p)
{
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  const DevSys<R> &s = a.s;
  if (i >= s.n_res) return;
  if (!(p.terms & T_WATER) || !(a.groups & G_FIX)) {
    if (lane == 0) a.xi_w[i] = 0.0;
    return;
  }
  V3<double> ci = contact(s, i);
  int chi = s.res_chain[i], ti = s.res_type[i];
  long long acc = 0;
  int cnt = a.ncount[i];
  const int *nb = a.nbr + (size_t) i * a.cap;
  const double *WG = s.tables + TB_WATER;
  for (int k = lane; k < cnt; k += 32) {
    int j = nb[k];
    if (s.res_chain[j] == chi && abs(i - j) < p.contact_cutoff) continue;
    V3<R> d = diff<R>(ci, contact(s, j));
    R rsq = norm2(d);
    int tj = s.res_type[j];
    for (int w = 0; w < p.n_wells; w++) {
      if (!p.well_flag[w]) continue;
      double g0 = WG[w * 800 + (ti * 20 + tj) * 2], g1 = WG[w * 800 + (ti * 20 + tj) * 2 + 1];
      // the reference's `!fabs(g0 - g1) < delta` holds exactly when g0 != g1
      if (g0 != g1 && rsq > R(p.w_rmin_sq[w]) && rsq < R(p.w_rmax_sq[w])) {
        R th, pr;
        well_theta(m_sqrt(rsq), R(p.w_rmin_th[w]), R(p.w_rmax_th[w]), R(p.water_kappa), R(p.well_rmin[w]),
                   R(p.well_rmax[w]), th, pr);
        acc += fix_dens((g1 - g0) * (double) th * a.sig_w[j]);
      }
    }
  }
  acc = warp_sum(acc);
  if (lane == 0) a.xi_w[i] = (double) acc * D_UNSCALE * a.sigp_w[i];
}

// DL3: main pair loop (fix_backbone.cpp:7956-8134) plus excluded volume
// between residues.  Radial contact forces and excluded volume act on the
// owner's beads only (each pair is visited from both sides).  DSSP and P_AP
// pairs are only detected here (cheap distance and index tests) and queued;
// k_hbond evaluates them one thread per pair, so their long, branchy bodies
// neither serialise this warp nor inflate its register count.
template <typename R> __global__ void __launch_bounds__(128) k_pair(StepArgs<R> a, FFParams p)
{
  int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  const DevSys<R> &s = a.s;
  if (i >= s.n_res) return;
  int n = s.n_res, fli = s.res_flags[i], chi = s.res_chain[i], ti = s.res_type[i];
  // (arrays below are only indexed by unrolled constants: they stay in registers)
  const bool gly_i = fli & R_GLY;
  V3<double> bi[3] = {bead(s, i, B_CA), bead(s, i, B_CB), bead(s, i, B_O)};
  V3<double> ci = gly_i ? bi[0] : bi[1];
  V3<double> oi = bi[2];
  int tat[3] = {a.atom_type[3 * i], a.atom_type[3 * i + 1], a.atom_type[3 * i + 2]};
  double xi_i = a.xi_w[i], bur_i = a.bur[i], x1_i = a.xi1[i];
  int dh = p.helix_i_diff;
  double x2_i = i - dh >= 0 ? a.xi2[i - dh] : 0.0;
  double sw_i = a.sig_w[i];
  long long F[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  long long Fc[3] = {0, 0, 0};  // contact-bead radial forces
  double e_water = 0.0, e_ev = 0.0;
  const double *WG = s.tables + TB_WATER;
  const bool fix = a.groups & G_FIX, evon = a.groups & G_PAIR;
  uint32_t T = fix ? p.terms : 0u;
  int cnt = a.ncount[i];
  const int *nb = a.nbr + (size_t) i * a.cap;
  const R ev_pre_sq = R(a.nl->ev_pre_sq);
  // smallest same-chain separation of any P_AP class (fix_backbone.cpp:3279-3383)
  const int pap_sep = min(p.i_med_min + 2 * p.i_diff_pap, p.i_med_max + 1);
  const bool dssp_i = (T & T_DSSP) && !(fli & R_LAST);
  const size_t qcap = (size_t) n * a.cap;
  for (int k0 = 0; k0 < cnt; k0 += 32) {
    const int k = k0 + lane;
    bool q_dssp = false, q_pap = false;
    if (k < cnt) {
    int j = nb[k];
    int flj = s.res_flags[j];
    bool other = s.res_chain[j] != chi;
    int dij = abs(i - j);
    bool upper = j > i;
    // contact-bead radial terms
    if (fix && (other || dij > 1)) {
      V3<R> d = diff<R>(ci, contact(s, j));
      R rsq = norm2(d);
      R r = m_sqrt(rsq);
      R force = 0;
      bool in0 = rsq > R(p.w_rmin_sq[0]) && rsq < R(p.w_rmax_sq[0]);
      R th0 = 0, pr0 = 0;
      if ((T & (T_WATER | T_BURIAL)) && in0)
        well_theta(r, R(p.w_rmin_th[0]), R(p.w_rmax_th[0]), R(p.water_kappa), R(p.well_rmin[0]), R(p.well_rmax[0]),
                   th0, pr0);
      if (T & T_WATER) {
        int tj = s.res_type[j];
        bool sep = other || dij >= p.contact_cutoff;
        for (int w = 0; w < p.n_wells; w++) {
          if (!p.well_flag[w]) continue;
          if (sep && rsq > R(p.w_rmin_sq[w]) && rsq < R(p.w_rmax_sq[w])) {
            double g0 = WG[w * 800 + (ti * 20 + tj) * 2], g1 = WG[w * 800 + (ti * 20 + tj) * 2 + 1];
            double sg = fabs(g0 - g1) < 1e-5 ? 0.5 * (g0 + g1) : g0 + (g1 - g0) * sw_i * a.sig_w[j];
            R th, pr;
            if (w == 0) {
              th = th0;
              pr = pr0;
            } else {
              well_theta(r, R(p.w_rmin_th[w]), R(p.w_rmax_th[w]), R(p.water_kappa), R(p.well_rmin[w]),
                         R(p.well_rmax[w]), th, pr);
            }
            if (upper) e_water += -sg * (double) th;
            force += R(sg) * pr;
          }
        }
        if (in0) {
          double xj = a.xi_w[j];
          if (fabs(xi_i) > 1e-8) force += pr0 * R(xi_i);
          if (fabs(xj) > 1e-8) force += pr0 * R(xj);
        }
      }
      if ((T & T_BURIAL) && in0) force += R(bur_i + a.bur[j]) * pr0;
      if ((T & T_HELIX) && rsq > R(p.h_rmin_sq) && rsq < R(p.h_rmax_sq)) {
        double fac = x1_i + a.xi1[j] + x2_i;
        if (j - dh >= 0) fac += a.xi2[j - dh];
        if (fabs(fac) > 1e-6) {
          R th, pr;
          well_theta(r, R(p.h_rmin_th), R(p.h_rmax_th), R(p.helix_kappa), R(p.helix_rmin), R(p.helix_rmax), th, pr);
          force += -R(fac) * pr;
        }
      }
      if (force != R(0)) {
        Fc[0] += fix_force((double) (force * d.x));
        Fc[1] += fix_force((double) (force * d.y));
        Fc[2] += fix_force((double) (force * d.z));
      }
    }
    const R rca2 = (evon || (T & T_PAP)) ? norm2(diff<R>(bi[0], bead(s, j, B_CA))) : R(0);
    // excluded volume between beads of i and j (1-2 bonded pairs removed)
    if (evon && rca2 < ev_pre_sq) {
      unsigned excl = 0;
      if (j == i + 1) excl = a.excl_next[i];
      bool prev = j == i - 1;
      unsigned exclp = prev ? a.excl_next[j] : 0u;
      bool shortr = !other && dij < 5;
#pragma unroll
      for (int b1 = 0; b1 < 3; b1++) {
        V3<double> bj = bead(s, j, b1);
        int tb = a.atom_type[3 * j + b1];
#pragma unroll
        for (int b0 = 0; b0 < 3; b0++) {
          if (excl & (1u << (b0 * 3 + b1))) continue;
          if (exclp & (1u << (b1 * 3 + b0))) continue;
          V3<R> f;
          R e = ev_pair(a, tat[b0], tb, shortr, diff<R>(bi[b0], bj), f);
          if (e == R(0) && f.x == R(0) && f.y == R(0) && f.z == R(0)) continue;
          if (upper) e_ev += (double) e;
          F[b0][0] += fix_force((double) f.x);
          F[b0][1] += fix_force((double) f.y);
          F[b0][2] += fix_force((double) f.z);
        }
      }
    }
    // DSSP with O(i) as acceptor and N-H(j) as donor (fix_backbone.cpp:8064-8079)
    if (dssp_i && (other || dij > 2) && !(flj & R_PRO) && !(flj & R_FIRST))
      q_dssp = norm2(diff<R>(oi, bead(s, j, B_N))) < R(p.dssp_cut_sq);
    // P_AP on CA pairs, visited from the lower residue (fix_backbone.cpp:8096-8103)
    if ((T & T_PAP) && upper && (other || j - i >= pap_sep)) q_pap = rca2 < R(p.pap_cutoff_sq);
    }
    // append this round's candidates to the queues (one atomic per warp and kind)
    const unsigned md = __ballot_sync(0xffffffffu, q_dssp), mp = __ballot_sync(0xffffffffu, q_pap);
    if (md | mp) {
      int bd = 0, bp = 0;
      if (lane == 0) {
        if (md) bd = atomicAdd(&a.nl->n_dssp, __popc(md));
        if (mp) bp = atomicAdd(&a.nl->n_pap, __popc(mp));
      }
      bd = __shfl_sync(0xffffffffu, bd, 0);
      bp = __shfl_sync(0xffffffffu, bp, 0);
      const unsigned below = (1u << lane) - 1u;
      const int slot = i * a.cap + k;
      if (q_dssp) a.hbq[bd + __popc(md & below)] = slot;
      if (q_pap) a.hbq[qcap + bp + __popc(mp & below)] = slot;
    }
  }
#pragma unroll
  for (int c = 0; c < 3; c++) {
    F[0][c] += gly_i ? Fc[c] : 0ll;
    F[1][c] += gly_i ? 0ll : Fc[c];
  }
#pragma unroll
  for (int b = 0; b < 3; b++)
#pragma unroll
    for (int c = 0; c < 3; c++) F[b][c] = warp_sum(F[b][c]);
  e_water = warp_sum(e_water);
  e_ev = warp_sum(e_ev);
  if (lane == 0) {
    unsigned long long *f = s.facc + (size_t) 9 * i;
#pragma unroll
    for (int b = 0; b < 3; b++)
#pragma unroll
      for (int c = 0; c < 3; c++)
        if (F[b][c]) atomicAdd(f + 3 * b + c, (unsigned long long) F[b][c]);
    double *E = a.e_res;
    E[(size_t) E_WATER * n + i] = e_water;
    E[(size_t) E_PAIR * n + i] += e_ev;
  }
}

// DSSP hydrogen bonds and P_AP of the queued pairs, one thread per pair
// (grid-stride over both queues).  Forces scatter with fixed-point atomics;
// each pair's energy goes to its first residue in fixed point, so the sums
// do not depend on the queue order.
template <typename R> __global__ void __launch_bounds__(128) k_hbond(StepArgs<R> a, FFParams p)
{
  const DevSys<R> &s = a.s;
  const int nd = a.nl->n_dssp, np = a.nl->n_pap, n = s.n_res;
  const size_t qcap = (size_t) n * a.cap;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nd + np; t += gridDim.x * blockDim.x) {
    const bool d = t < nd;
    const int slot = d ? a.hbq[t] : a.hbq[qcap + (t - nd)];
    const int i = slot / a.cap, j = a.nbr[slot];
    R e = d ? dssp_term(s, p, i, j) : pap_term(s, p, i, j);
    if (e != R(0))
      atomicAdd((unsigned long long *) (a.e_fix + (d ? 0 : (size_t) n) + i), (unsigned long long) fix_force((double) e));
  }
}

// Fragment memory: sliced lane-interleaved table, lane per residue row
// (awsem_fragmem.cuh)
template <typename R> struct BeadPos {
  const DevSys<R> *s;
  __device__ __forceinline__ V3<double> operator()(int r, int b) const { return bead(*s, r, b ? B_CB : B_CA); }
};

template <typename R> __global__ void __launch_bounds__(128) k_fragmem(StepArgs<R> a, FFParams p)
{
  const BeadPos<R> pos{&a.s};
  fragmem_warp(a.fm, p.fm_sigma_sq, a.s.n_res, pos, a.s.facc,
               (unsigned long long *) (a.e_fix + (size_t) 2 * a.s.n_res), 1);
}

// bond_style harmonic, bonds grouped by the residue of their first atom
template <typename R> __global__ void k_bonds(StepArgs<R> a)
{
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  const DevSys<R> &s = a.s;
  if (r >= s.n_res) return;
  double e = 0.0;
  for (int b = a.bond_start[r]; b < a.bond_start[r + 1]; b++) {
    int ai = a.bond_i[b], aj = a.bond_j[b];
    V3<R> d = diff<R>(bead(s, ai / 3, ai % 3), bead(s, aj / 3, aj % 3));
    R rr = m_sqrt(norm2(d));
    R dr = rr - R(a.bond_r0[b]);
    R rk = R(a.bond_k[b]) * dr;
    R fb = rr > R(0) ? R(-2) * rk / rr : R(0);
    e += (double) (rk * dr);
    scatter(s, ai / 3, ai % 3, d.x * fb, d.y * fb, d.z * fb);
    scatter(s, aj / 3, aj % 3, -d.x * fb, -d.y * fb, -d.z * fb);
  }
  a.e_res[(size_t) E_BOND * s.n_res + r] = e;
}

__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

// Uniform in [0,1) keyed by (seed, step, atom id, component): the Langevin
// noise stream shared with the CPU oracle.
__device__ __forceinline__ double uniform01(uint64_t seed, long long step, long long tag, int comp)
{
  uint64_t key = mix64(seed ^ mix64((uint64_t) step));
  uint64_t r = mix64(key ^ ((uint64_t) tag * 4ULL + (uint64_t) comp));
  return (double) (r >> 11) * (1.0 / 9007199254740992.0);
}

struct Integrator {
  double dt, dtf;           // dtf = 0.5 * dt * ftm2v
  int langevin;
  double t_start, t_stop;   // thermostat ramp over [begin, end]
  long long begin, end;
  double damp;
  unsigned long long seed;
};

// Total force (fixed point -> FP64, plus Langevin at `step`), then
// final_integrate of `step` (half kick) and, if `next`, initial_integrate of
// step+1 (half kick + drift) -- LAMMPS fix nve / fix langevin order.
template <typename R>
__global__ void k_finish(StepArgs<R> a, const Integrator *inp, const double *g1, const double *g2, double *ftot,
                         double *x_out)
{
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= a.s.n_res) return;
  const Integrator in = *inp;
  const long long step = *a.step;
  const bool final_kick = step > in.begin, next = step < in.end;
  const unsigned long long seed = a.sys_seed[a.res_sys[r]];
  double tsqrt = 0.0;
  if (in.langevin) {
    double delta = in.end != in.begin ? (double) (step - in.begin) / (double) (in.end - in.begin) : 0.0;
    tsqrt = sqrt(in.t_start + delta * (in.t_stop - in.t_start));
  }
  double ke = 0.0;
  for (int b = 0; b < 3; b++) {
    int at = 3 * r + b;
    double m = a.mass[at];
    double dtfm = in.dtf / m;
    const unsigned long long *fa = a.s.facc + (size_t) 3 * at;
    for (int c = 0; c < 3; c++) {
      double f = (double) (long long) fa[c] * F_UNSCALE;
      double v = a.v[3 * at + c];
      if (in.langevin) f += g1[at] * v + g2[at] * tsqrt * (uniform01(seed, step, a.atom_tag[at], c) - 0.5);
      if (ftot) ftot[3 * at + c] = f;
      if (final_kick) v += dtfm * f;
      ke += m * v * v;
      if (next) {
        v += dtfm * f;
        x_out[3 * at + c] += in.dt * v;
      }
      a.v[3 * at + c] = v;
    }
  }
  // kinetic energy after the final half kick (thermo output of the step)
  a.e_res[(size_t) E_KIN * a.s.n_res + r] = 0.5 * 48.88821291 * 48.88821291 * ke;
}

// Conservative total force of the last evaluation in FP64 (no Langevin)
template <typename R> __global__ void k_total_force(StepArgs<R> a, double *ftot)
{
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 3 * a.n_atoms) return;
  ftot[k] = (double) (long long) a.s.facc[k] * F_UNSCALE;
}

// Thermo row of the current step: [fix total, vexcluded, bonds, kinetic],
// residue sums in a fixed tree order (one block of 256 threads).
__global__ void k_thermo(const double *e_res, const long long *e_fix, int n_res, const long long *step,
                         const Integrator *inp, const int *sys_begin, const int *sys_end, long long nrows, double *rows)
{
  const long long begin = inp->begin;
  const int rep = blockIdx.x;
  __shared__ double sh[4][256];
  double acc[4] = {0, 0, 0, 0};
  for (int r = sys_begin[rep] + threadIdx.x; r < sys_end[rep]; r += blockDim.x) {
    double fx = 0.0;
    for (int t = 1; t < E_FIX_TERMS; t++) fx += e_res[(size_t) t * n_res + r];
    fx += (double) (e_fix[r] + e_fix[(size_t) n_res + r] + e_fix[(size_t) 2 * n_res + r]) * F_UNSCALE;
    acc[0] += fx;
    acc[1] += e_res[(size_t) E_PAIR * n_res + r];
    acc[2] += e_res[(size_t) E_BOND * n_res + r];
    acc[3] += e_res[(size_t) E_KIN * n_res + r];
  }
  for (int c = 0; c < 4; c++) sh[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int c = 0; c < 4; c++) sh[c][threadIdx.x] += sh[c][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    long long row = *step - begin;
    for (int c = 0; c < 4; c++) rows[((size_t) rep * nrows + row) * 4 + c] = sh[c][0];
  }
}

// Per-term sums of each replica's residues in a fixed tree order
// (block (t, rep) sums energy slot t of replica rep)
__global__ void k_energy_reduce(const double *e_res, const long long *e_fix, int n_res, const int *sys_begin,
                                const int *sys_end, double *out)
{
  const int t = blockIdx.x, rep = blockIdx.y;
  __shared__ double sh[256];
  double acc = 0.0;
  // DSSP, P_AP and fragment-memory energies are kept in fixed point
  const long long *fx = t == E_DSSP ? e_fix : t == E_PAP ? e_fix + n_res : t == E_FRAGMEM ? e_fix + 2 * (size_t) n_res : nullptr;
  for (int r = sys_begin[rep] + threadIdx.x; r < sys_end[rep]; r += blockDim.x)
    acc += fx ? (double) fx[r] * F_UNSCALE : e_res[(size_t) t * n_res + r];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[(size_t) rep * E_SLOTS + t] = sh[0];
}

}  // namespace dev
}  // namespace awsem
