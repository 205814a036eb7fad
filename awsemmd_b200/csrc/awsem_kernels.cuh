// Per-step kernels of the AWSEM engine (sm_100a).
//
// One MD step is this set of launches (captured into a CUDA graph), on three
// streams joined before `finish`:
//   prepare      thread/residue: CA, CB, O -> working copy + virtual N, H, C'
//                (fix_backbone.cpp:7067-7138) and the contact-bead copy;
//                zero forces; list-check data
//   nl_decide    1 thread: rebuild decision for the residue pair list
//   nl_build     warp/residue: pairs i < j of contact beads within the list
//                radius, appended to a flat pair array
// first stream:
//   density      warp/list segment: rho_water, rho_helix (DL1, :7728-7791);
//                writes the near list
//   residue      thread/residue: switching functions, burial (SL,
//                :7795-7841), helical (i,i+4) pairs (:7843-7868), harmonic
//                bonds, excluded volume inside the residue
//   water_xi     thread/near pair: xi_water (DL2, :7877-7954)
//   radial       thread/near pair: water/burial/helix radial forces (DL3,
//                :7956-8057)
// third stream:
//   backbone     thread/residue: chain, chi, rama (:2062-2546)
//   pair         thread/near pair: DSSP and P_AP detection into queues,
//                excluded volume between residues (DL3, :8064-8103)
//   hbond        thread/queued pair: DSSP hydrogen bonds, P_AP
// second stream:
//   fragmem      warp/32 residues, lane/residue row: fragment-memory
//                Gaussians (:4079-4177)
// then
//   finish       thread/component: fixed-point -> FP64 forces, Langevin,
//                velocity-Verlet half kicks and drift
// Residue-owned quantities are written by their owner without atomics;
// sums over pairs (forces, densities, pair energies) use 64-bit integer
// atomics on fixed-point accumulators, which makes them exact and order
// independent.
#pragma once

#include "awsem_device.cuh"
#include "awsem_fragmem.cuh"
#include "awsem_gpu.h"

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
  float bCBx, bOx;    // the same for CB and for O alone (this step, reduced by k_prepare)
  float ev_pre_sq;    // CA-CA distance^2 beyond which no bead pair of two residues is in excluded-volume range
  // Excluded volume by bead kind (0 CA, 1 CB, 2 O): the largest cutoff of
  // any type pair found at those positions (short range [0], long range
  // [1]; 0 when no such pair interacts; set by the host), and this step's
  // reach of each kind from its residue's CA (0 for CA itself).
  float ev_cutk[2][3][3];
  float ev_reach[3];
  float bNCA;         // max distance of a residue's virtual N from its own CA (this step)
  float dssp_pre_sq;  // CA-CA distance^2 beyond which neither O-N pair of two residues is within the DSSP cutoff
  int npairs;         // pairs in the residue pair list (may exceed its capacity: overflow)
  int fm_timeout;     // a fragment-memory stream wait gave up (results invalid)
  int tb_error;       // table fragment memory: 1 a distance outside the table's range, 2 a grid index outside it
  // The reference fix reads LAMMPS's neighbour lists, whose membership is
  // fixed at each list build.  Terms that use list membership itself (AMH-Go;
  // Debye-Hueckel and the solvent barrier on the CA pairs of the half list)
  // follow LAMMPS's rebuild rule, emulated per replica (k_list_decide).
  double lst_skin;    // neighbor skin (A)
  int lst_delay, lst_every, lst_check;  // neigh_modify delay / every / check
  int lst_force;      // host: the next evaluation is a run setup (the lists are built)
  int lst_setup;      // this evaluation is a run setup
  int lst_host;       // the host decides the builds (awsem_compute): lst_setup alone
  float lst_pair_cut; // CA-CA reach of the half list (pair-list cutoff + skin) the
                      // CA-pair terms need covered by the residue pair list (0: none)
  float lst_d2max;    // max CA displacement^2 since the last emulated build (this step)
  int bad_x;          // a position was not finite (results invalid; the host reports and clears it)
  float need;         // R_need of this step: no term reaches a pair whose contact beads are farther apart
  // The near list (the listed pairs whose contact beads are within `need`)
  // is written by the density pass in segments: warp w of that pass scans
  // the listed pairs [w seg_len, (w + 1) seg_len) and writes its near pairs,
  // in list order, to the start of the same range of cpairs; seg_n[w] holds
  // their count.  No shared counter: every warp owns its range.
  int seg_len;        // pairs per segment (a multiple of 32)
  int nseg;           // segments
  // Counters updated with atomics during a pass, each on its own cache line:
  // reads of a line that other threads are updating atomically wait for
  // those atomics
  alignas(128) int n_dssp;  // hydrogen-bond queue lengths of the current evaluation
  alignas(128) int n_pap;
  alignas(128) int fm_next;  // fragment-memory work units handed out (k_fragmem), zeroed by the list decision
  alignas(128) int end_pad;
};

// Run window of one replica: integrated over steps begin..end (the
// evaluation at `begin` is its setup evaluation), thermostat ramp t_start ->
// t_stop over the window, Langevin noise keyed by step - step0.
struct SlotRun {
  long long begin, end, step0;
  double t_start, t_stop;
};

// What the radial pass reads of a residue, packed into one 64-byte record
// (written by the residue pass): three cache lines per residue of a pair
// (this record, the contact bead, the water-xi sum) instead of ten arrays.
struct __align__(64) RadRec {
  double sw, bur, x1, x2, sigp;  // sigma_water, burial coefficient, helix xi1, xi2 of residue r - helix_i_diff, sigma_water'
  double pad0;
  int type, flags, chain, pad;
};
static_assert(sizeof(RadRec) == 64 && offsetof(RadRec, type) == 48, "RadRec layout");

template <typename R> struct StepArgs {
  DevSys<R> s;
  int n_run;  // residues the per-residue passes cover: a prefix of s.n_res (the used part of a serving handle)
  int n_atoms;
  const double *x;  // [n_atoms][3]
  double *v;
  const double *mass;
  const int *atom_tag;
  // per-residue pair-pass intermediates
  double *rho_w, *rho_h, *sig_w, *sigp_w, *sig_h, *sigp_h, *xi_w, *xi1, *xi2, *bur;
  RadRec *rrec;  // [n_res]
  double *e_res;  // [E_SLOTS][n_res]
  // residue pair list: pairs (i, j), i < j, capacity pcap; per-residue counts.
  // cpairs: the near list of this evaluation (the listed pairs whose contact
  // beads are within NLState::need), written by the density pass in segments
  // (seg_n: near pairs per segment, capacity pcap / 32 + 2) and walked by the
  // water-xi, pair and hydrogen-bond passes (capacity pcap)
  int2 *pairs, *cpairs;
  int *seg_n;
  int *ncount, pcap;
  double4 *cb_build;
  NLState *nl;
  // hydrogen-bond work queues (pair indices): DSSP in [0, 2 pcap) (q: O(i)
  // acceptor, ~q: O(j) acceptor), P_AP in [2 pcap, 3 pcap)
  int *hbq;
  // energies summed over pairs, in 2^-32 fixed point (sums independent of
  // order): [0] DSSP, [1] P_AP, [2] fragment memory, [3] water, [4] excluded
  // volume between residues; [5][n_res]
  long long *e_fix;
  // density sums in 2^-40 fixed point: [0] water, [1] helix, [2] raw xi_water; [3][n_res]
  long long *dacc;
  // excluded volume
  int ntypes, ev_p;
  const double *ev_pref, *ev_cs, *ev_cl;
  const int *atom_type;
  const unsigned *excl_self, *excl_next;
  // bonds in bond_cap slots per residue of their first atom ([n_res][bond_cap],
  // internal atom indices; bond_i < 0 ends a residue's slots)
  int bond_cap;
  const int *bond_i, *bond_j;
  const double *bond_k, *bond_r0;
  // fragment memory
  FMSlices<R> fm;
  // table fragment memory: [n_res][tb_nbrs][4][tb_size] (energy, force) and the tables present
  const double2 *tb_data;
  const unsigned char *tb_present;
  // AMH-Go native contacts per CA / CB atom slot 2 r + b ([2 n_res + 1] offsets), per residue normalisation
  const int *go_start, *go_partner;
  const double *go_rnat, *go_gamma, *go_sig_sq, *go_norm;
  unsigned char *go_in;          // per AMH-Go contact: in the list since the last build
  double *lst_x0;                // [9 n]: positions at the replica's last list build
  int *lst_ago, *lst_over;       // per replica: steps since the build; an atom moved over half the skin
  const int *lst_build;          // per replica: this evaluation builds the lists
  // Debye-Hueckel, solvent barrier, contact restraints (k_pair_extra)
  const double *charge;          // [n]: charge of the residue
  const int *cr_start, *cr_j;    // contact restraints of residue i (i < j): [cr_start[i], cr_start[i+1])
  const double *cr_w, *cr_r0;
  int efix_slots;                // fixed-point energy slots in use (5, or 8 with the pair terms above)
  const int *zim;                // [n]: membrane zone (1, 2, 3) of the residue
  const int *vfm_start, *vfm_j;  // vector fragment memory records of residue i (i < j)
  const double *vfm_angle;
  int groups;       // AWSEM_TERMS_* bits: 1 fix backbone, 2 pair vexcluded, 4 bonds
  long long *step;   // device step counter (advanced by k_nl_decide)
  // replicas: residue -> replica, replica residue ranges, Langevin seeds
  // (res_sys < 0: residue of no replica, skipped)
  const int *res_sys, *sys_begin, *sys_end;
  const unsigned long long *sys_seed;
  const SlotRun *slot_run;
  // selection records (awsem_debug_selections; null in steps): keys, count, capacity
  unsigned long long *sel, *sel_n;
  long long sel_cap;
};

enum Group { G_FIX = 1, G_PAIR = 2, G_BOND = 4 };

// The threads of a pass: thread t of nthr, grid-stride over the pass's items.
// A standalone kernel gives a pass its whole grid; the persistent step
// kernel (awsem_step.cuh) gives it the threads it reserves for the pass.
struct Span {
  int t, nthr;
};
__device__ __forceinline__ Span grid_span()
{
  return Span{(int) (blockIdx.x * blockDim.x + threadIdx.x), (int) (gridDim.x * blockDim.x)};
}

// one selection record (AWSEM_SEL_* key, awsem_gpu.h).  The passes take SEL
// as a template flag: the per-step kernels are compiled without recording
// (SEL false), the diagnostic kernels of awsem_debug_selections with it.
template <bool SEL, typename R>
__device__ __forceinline__ void sel_rec(const StepArgs<R> &a, int kind, int aux, int i, int j)
{
  if (!SEL || !a.sel) return;
  const unsigned long long k = atomicAdd(a.sel_n, 1ull);
  if (k < (unsigned long long) a.sel_cap)
    a.sel[k] = (unsigned long long) kind << 56 | (unsigned long long) aux << 44 | (unsigned long long) i << 22 |
               (unsigned long long) j;
}

__device__ __forceinline__ void atomic_max_f(float *addr, float v)
{
  // non-negative floats order like their bit patterns
  atomicMax((int *) addr, __float_as_int(v));
}

template <typename R> __device__ __forceinline__ void prepare_pass(const StepArgs<R> &a, const FFParams &p, Span sp)
{
  float d2 = 0.f, dl = 0.f;
  // squared bead offsets, maximised over this thread's residues; the square
  // root of the maximum is the maximum of the square roots (both roundings
  // are monotonic), so one root per thread gives the same maxima
  double qO = 0.0, qN = 0.0, qCA = 0.0, qAll = 0.0, qB = 0.0, qX = 0.0, qNCA = 0.0;
  const int lane = threadIdx.x & 31;
  // warp-uniform trip count: the maxima are reduced across the warp below
  for (int r0 = sp.t - lane; r0 < a.n_run; r0 += sp.nthr) {
  const int r = r0 + lane;
  if (r < a.n_run) {
    unsigned long long *f = a.s.facc + (size_t) 9 * r;
    for (int k = 0; k < 9; k++) f[k] = 0ull;
    for (int k = 0; k < a.efix_slots; k++) a.e_fix[(size_t) k * a.s.n_res + r] = 0;
    for (int k = 0; k < 3; k++) a.dacc[(size_t) k * a.s.n_res + r] = 0;
  }
  if (r < a.n_run && a.res_sys[r] >= 0) {
    const double *x = a.x;
    int fl = a.s.res_flags[r];
    double ca[3], cb[3], o[3], n[3] = {0, 0, 0}, h[3] = {0, 0, 0}, cp[3] = {0, 0, 0};
    bool finite = true;
    for (int k = 0; k < 3; k++) {
      ca[k] = x[(3 * r + 0) * 3 + k];
      cb[k] = x[(3 * r + 1) * 3 + k];
      o[k] = x[(3 * r + 2) * 3 + k];
      finite = finite && isfinite(ca[k]) && isfinite(cb[k]) && isfinite(o[k]);
    }
    if (!finite) a.nl->bad_x = 1;
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
    if (a.lst_x0) {
      // LAMMPS check_distance for the emulated lists: an atom farther than
      // half the skin from where it was at the last build
      const double trig = 0.25 * a.nl->lst_skin * a.nl->lst_skin;
      const double *h = a.lst_x0 + (size_t) 9 * r;
      bool over = false;
      for (int b = 0; b < 3; b++) {
        const double *q = b == 0 ? ca : b == 1 ? cb : o;
        const double dx = q[0] - h[3 * b], dy = q[1] - h[3 * b + 1], dz = q[2] - h[3 * b + 2];
        const double d2b = dx * dx + dy * dy + dz * dz;
        if (d2b > trig) over = true;
        if (b == 0) dl = fmaxf(dl, (float) d2b * 1.0001f);
      }
      if (over) a.lst_over[a.res_sys[r]] = 1;
    }
    double4 *w = const_cast<double4 *>(a.s.pos) + (size_t) r * N_BEADS;
    w[B_CA] = make_double4(ca[0], ca[1], ca[2], 0.0);
    w[B_CB] = make_double4(cb[0], cb[1], cb[2], 0.0);
    w[B_O] = make_double4(o[0], o[1], o[2], 0.0);
    w[B_N] = make_double4(n[0], n[1], n[2], 0.0);
    w[B_H] = make_double4(h[0], h[1], h[2], 0.0);
    w[B_CP] = make_double4(cp[0], cp[1], cp[2], 0.0);
    {
      const double *cc = (fl & R_GLY) ? ca : cb;
      const_cast<double4 *>(a.s.cpos)[r] = make_double4(cc[0], cc[1], cc[2], 0.0);
    }
    {
      // reach of the residue's beads around its CA (excluded-volume prefilter)
      double ux = cb[0] - ca[0], uy = cb[1] - ca[1], uz = cb[2] - ca[2];
      double wx = o[0] - ca[0], wy = o[1] - ca[1], wz = o[2] - ca[2];
      qB = fmax(qB, ux * ux + uy * uy + uz * uz);
      qX = fmax(qX, wx * wx + wy * wy + wz * wz);
    }
    // list-validity data: contact-bead displacement and bead offsets
    const double *c = (fl & R_GLY) ? ca : cb;
    double4 b0 = a.cb_build[r];
    double dx = c[0] - b0.x, dy = c[1] - b0.y, dz = c[2] - b0.z;
    d2 = fmaxf(d2, (float) (dx * dx + dy * dy + dz * dz));
    auto off2 = [&](const double *q) {
      double ex = q[0] - c[0], ey = q[1] - c[1], ez = q[2] - c[2];
      return ex * ex + ey * ey + ez * ez;
    };
    const double o_o = off2(o), o_ca = off2(ca);
    qO = fmax(qO, o_o);
    qCA = fmax(qCA, o_ca);
    qAll = fmax(qAll, fmax(fmax(o_ca, off2(cb)), o_o));
    if (!(fl & R_FIRST)) {
      qN = fmax(qN, off2(n));
      const double ex = n[0] - ca[0], ey = n[1] - ca[1], ez = n[2] - ca[2];
      qNCA = fmax(qNCA, ex * ex + ey * ey + ez * ez);
    }
  }
  }
  float oO = (float) sqrt(qO), oN = (float) sqrt(qN), oCA = (float) sqrt(qCA), oAll = (float) sqrt(qAll);
  float oB = (float) sqrt(qB), oX = (float) sqrt(qX), oNCA = (float) sqrt(qNCA);
  // warp max, block max, then one atomic per block and quantity (every
  // thread of the block calls this pass)
  for (int s = 16; s > 0; s >>= 1) {
    d2 = fmaxf(d2, __shfl_xor_sync(0xffffffffu, d2, s));
    oO = fmaxf(oO, __shfl_xor_sync(0xffffffffu, oO, s));
    oN = fmaxf(oN, __shfl_xor_sync(0xffffffffu, oN, s));
    oCA = fmaxf(oCA, __shfl_xor_sync(0xffffffffu, oCA, s));
    oAll = fmaxf(oAll, __shfl_xor_sync(0xffffffffu, oAll, s));
    oB = fmaxf(oB, __shfl_xor_sync(0xffffffffu, oB, s));
    oX = fmaxf(oX, __shfl_xor_sync(0xffffffffu, oX, s));
    oNCA = fmaxf(oNCA, __shfl_xor_sync(0xffffffffu, oNCA, s));
    dl = fmaxf(dl, __shfl_xor_sync(0xffffffffu, dl, s));
  }
  __shared__ float red[9][32];
  if (lane == 0) {
    const int w = threadIdx.x >> 5;
    red[0][w] = d2, red[1][w] = oO, red[2][w] = oN, red[3][w] = oCA, red[4][w] = oAll, red[5][w] = oX;
    red[6][w] = oNCA, red[7][w] = dl, red[8][w] = oB;
  }
  __syncthreads();
  if (threadIdx.x < 9) {
    const int k = threadIdx.x;
    float m = 0.f;
    for (int w = 0; w < (int) (blockDim.x >> 5); w++) m = fmaxf(m, red[k][w]);
    float *dst = k == 0 ? &a.nl->d2max : k == 1 ? &a.nl->bO : k == 2 ? &a.nl->bN : k == 3 ? &a.nl->bCA
               : k == 4 ? &a.nl->bAll : k == 5 ? &a.nl->bOx : k == 6 ? &a.nl->bNCA : k == 7 ? &a.nl->lst_d2max
               : &a.nl->bCBx;
    if (m > 0.f) atomic_max_f(dst, m);  // the maxima start each step at 0
  }
}

template <typename R> __global__ void k_prepare(StepArgs<R> a, FFParams p) { prepare_pass(a, p, grid_span()); }

// Pair-list rebuild decision.  A residue pair is needed when one of its
// tested bead pairs is inside that term's cutoff; in contact-bead distance
// that is at most R_need = max(r_contact, r_dssp + bO + bN, r_pap + 2 bCA,
// r_ev + 2 bAll).  The list built at t0 with radius R_need(t0) + skin stays
// complete while R_need(t) + 2 * max displacement <= radius.
__device__ __forceinline__ void nl_decide(NLState *nl, int force, long long *step)
{
  if (step) (*step)++;
  NLState &s = *nl;
  float need = fmaxf(fmaxf(s.r_contact, s.r_dssp + s.bO + s.bN), fmaxf(s.r_pap + 2.f * s.bCA, s.r_ev + 2.f * s.bAll));
  // residue pairs whose CAs were within the half list's reach at the last
  // emulated build: their contact beads are at most that reach + twice the
  // CA displacement since then + twice the CA-to-contact-bead offset apart
  if (s.lst_pair_cut > 0.f) need = fmaxf(need, s.lst_pair_cut + 2.f * sqrtf(s.lst_d2max) + 2.f * s.bCA + 0.01f);
  float disp = sqrtf(s.d2max);
  bool rb = force || s.r_list <= 0.f || need + 2.f * disp > s.r_list || (s.every > 0 && s.steps_since + 1 >= s.every);
  if (rb) {
    s.npairs = 0;  // k_nl_build appends
    s.r_list = need + s.skin;
    s.steps_since = 0;
    s.nbuilds++;
  } else {
    s.steps_since++;
  }
  s.rebuild = rb;
  s.need = need;
  s.fm_next = 0;
  s.bCAx = fmaxf(s.bCBx, s.bOx);
  // |b(i) - b'(j)| >= |CA(i) - CA(j)| - reach(b) - reach(b'): two residues
  // whose CAs are farther apart than the largest cutoff + reaches of any
  // interacting bead kinds have no bead pair in excluded-volume range
  // (0.01 A covers rounding)
  s.ev_reach[0] = 0.f;
  s.ev_reach[1] = s.bCBx;
  s.ev_reach[2] = s.bOx;
  float pre = 0.f;
  for (int r = 0; r < 2; r++)
    for (int b0 = 0; b0 < 3; b0++)
      for (int b1 = 0; b1 < 3; b1++)
        if (s.ev_cutk[r][b0][b1] > 0.f) pre = fmaxf(pre, s.ev_cutk[r][b0][b1] + s.ev_reach[b0] + s.ev_reach[b1]);
  pre += 0.01f;
  s.ev_pre_sq = pre * pre;
  // |O(i) - N(j)| >= |CA(i) - CA(j)| - |O(i) - CA(i)| - |N(j) - CA(j)|, and bCAx bounds |O - CA|
  const float dpre = s.r_dssp + s.bCAx + s.bNCA + 0.01f;
  s.dssp_pre_sq = dpre * dpre;
  s.d2max = s.bO = s.bN = s.bCA = s.bAll = s.bCBx = s.bOx = s.bNCA = 0.f;
  s.n_dssp = s.n_pap = 0;
  s.lst_setup = s.lst_force;
  s.lst_force = 0;
  s.lst_d2max = 0.f;
}

__global__ void k_nl_decide(NLState *nl, int force, long long *step) { nl_decide(nl, force, step); }

// contact bead of residue r (one load, no dependence on the residue's flags)
template <typename R> __device__ __forceinline__ V3<double> contact(const DevSys<R> &s, int r)
{
  const double4 q = s.cpos[r];
  return {q.x, q.y, q.z};
}

// Cell grids for large replicas (more than kGridMin residues): each such
// replica gets a uniform grid over the bounding box of its contact beads at
// every list build, cells no smaller than the list radius (grown when the
// box would need more cells than the replica's cell budget), and residues
// sorted by cell; its residues then scan the 27 surrounding cells instead of
// the whole replica.  Smaller replicas scan all their higher residues.
constexpr int kGridMin = 2048;

struct GridDesc {
  float ox, oy, oz, inv_cell;
  int nx, ny, nz;
  int cell0, cap;  // first cell in the shared cell arrays, cells budgeted
};

struct GridArgs {
  int nbig;
  const int *big_rep;   // [nbig] replica of each gridded replica
  const int *big_of;    // [n_sys] gridded index of a replica, -1 when scanned directly
  GridDesc *desc;       // [nbig]
  int *cell_count, *cell_start, *cell_fill;  // [total cells]
  int *res_cell;        // [n_res] cell of a gridded residue
  int *sorted;          // [n_res] residues of each gridded replica, by cell, at the replica's residue range
};

// one block per gridded replica: bounding box, grid shape, cleared counts
template <typename R> __global__ void k_grid_setup(StepArgs<R> a, GridArgs g)
{
  if (!a.nl->rebuild) return;
  const int b = blockIdx.x, rep = g.big_rep[b];
  const int r0 = a.sys_begin[rep], r1 = a.sys_end[rep];
  float lo[3] = {3e38f, 3e38f, 3e38f}, hi[3] = {-3e38f, -3e38f, -3e38f};
  for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    const V3<double> c = contact(a.s, r);
    const float p[3] = {(float) c.x, (float) c.y, (float) c.z};
    for (int k = 0; k < 3; k++) {
      lo[k] = fminf(lo[k], p[k]);
      hi[k] = fmaxf(hi[k], p[k]);
    }
  }
  __shared__ float sl[3][32], sh[3][32];
  for (int k = 0; k < 3; k++) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
      hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
    }
    if ((threadIdx.x & 31) == 0) {
      sl[k][threadIdx.x >> 5] = lo[k];
      sh[k][threadIdx.x >> 5] = hi[k];
    }
  }
  __syncthreads();
  GridDesc &d = g.desc[b];
  if (threadIdx.x == 0) {
    for (int k = 0; k < 3; k++)
      for (int w = 1; w < (int) (blockDim.x >> 5); w++) {
        sl[k][0] = fminf(sl[k][0], sl[k][w]);
        sh[k][0] = fmaxf(sh[k][0], sh[k][w]);
      }
    // cells at least the list radius (plus rounding room) wide
    float cell = a.nl->r_list * 1.0001f + 1e-3f;
    int n[3];
    for (int it = 0; it < 64; it++) {
      long long tot = 1;
      for (int k = 0; k < 3; k++) {
        n[k] = max(1, (int) ((sh[k][0] - sl[k][0]) / cell) + 1);
        tot *= n[k];
      }
      if (tot <= d.cap) break;
      cell *= 1.26f;
    }
    d.ox = sl[0][0];
    d.oy = sl[1][0];
    d.oz = sl[2][0];
    d.inv_cell = 1.f / cell;
    d.nx = n[0];
    d.ny = n[1];
    d.nz = n[2];
  }
  __syncthreads();
  for (int c = threadIdx.x; c < d.cap; c += blockDim.x) {
    g.cell_count[d.cell0 + c] = 0;
    g.cell_fill[d.cell0 + c] = 0;
  }
}

__device__ __forceinline__ int grid_coord(float p, float o, float inv, int n)
{
  return min(n - 1, max(0, (int) ((p - o) * inv)));
}

// thread per residue of a gridded replica: its cell, and the cell counts
template <typename R> __global__ void k_grid_count(StepArgs<R> a, GridArgs g)
{
  if (!a.nl->rebuild) return;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= a.s.n_res || a.res_sys[r] < 0) return;
  const int b = g.big_of[a.res_sys[r]];
  if (b < 0) return;
  const GridDesc d = g.desc[b];
  const V3<double> c = contact(a.s, r);
  const int cx = grid_coord((float) c.x, d.ox, d.inv_cell, d.nx), cy = grid_coord((float) c.y, d.oy, d.inv_cell, d.ny),
            cz = grid_coord((float) c.z, d.oz, d.inv_cell, d.nz);
  const int cell = d.cell0 + (cz * d.ny + cy) * d.nx + cx;
  g.res_cell[r] = cell;
  atomicAdd(&g.cell_count[cell], 1);
}

// one block per gridded replica: cell starts (exclusive scan, offset by the
// replica's first residue) in chunks of blockDim.x cells
template <typename R> __global__ void k_grid_scan(StepArgs<R> a, GridArgs g)
{
  if (!a.nl->rebuild) return;
  const int b = blockIdx.x;
  const GridDesc d = g.desc[b];
  const int ncell = d.nx * d.ny * d.nz;
  __shared__ int part[1024];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = a.sys_begin[g.big_rep[b]];
  __syncthreads();
  for (int c0 = 0; c0 < ncell; c0 += blockDim.x) {
    const int c = c0 + threadIdx.x;
    const int v = c < ncell ? g.cell_count[d.cell0 + c] : 0;
    part[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < (int) blockDim.x; o <<= 1) {  // inclusive Hillis-Steele scan
      const int add = threadIdx.x >= (unsigned) o ? part[threadIdx.x - o] : 0;
      __syncthreads();
      part[threadIdx.x] += add;
      __syncthreads();
    }
    if (c < ncell) g.cell_start[d.cell0 + c] = carry + part[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry += part[threadIdx.x];
    __syncthreads();
  }
}

// thread per residue of a gridded replica: place it in its cell's range
template <typename R> __global__ void k_grid_fill(StepArgs<R> a, GridArgs g)
{
  if (!a.nl->rebuild) return;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= a.s.n_res || a.res_sys[r] < 0 || g.big_of[a.res_sys[r]] < 0) return;
  const int cell = g.res_cell[r];
  g.sorted[g.cell_start[cell] + atomicAdd(&g.cell_fill[cell], 1)] = r;
}

// Residue pair list: every pair i < j of one replica whose contact beads are
// closer than r_list, as (i, j) in a flat array.  One warp per residue scans
// the candidates twice (count, then write after one atomic reservation), so
// a residue's pairs are contiguous.  Candidates: the higher residues of its
// replica, or for a gridded replica the residues of the 27 cells around its
// own.  Every pair pass below runs one thread per listed (or near) pair and
// scatters to both residues with fixed-point atomics: each pair is evaluated
// once, as in the reference's half neighbour list.
template <typename R> __device__ __forceinline__ void nl_build_one(const StepArgs<R> &a, const GridArgs &g, int i,
                                                               int lane)
{
  if (a.res_sys[i] < 0) {
    if (lane == 0) a.ncount[i] = 0;
    return;
  }
  const int rep = a.res_sys[i], sys_end = a.sys_end[rep];
  const int b = g.nbig ? g.big_of[rep] : -1;
  const DevSys<R> &s = a.s;
  const V3<double> ci = contact(s, i);
  const R rl = (R) a.nl->r_list, rl2 = rl * rl;
  // candidate ranges: [lo, hi) of residue indices, or of sorted positions (gridded)
  GridDesc d{};
  int cx = 0, cy = 0, cz = 0;
  if (b >= 0) {
    d = g.desc[b];
    const int cell = g.res_cell[i] - d.cell0;
    cx = cell % d.nx;
    cy = (cell / d.nx) % d.ny;
    cz = cell / (d.nx * d.ny);
  }
  auto scan = [&](auto &&visit) {  // visit(j, take) for every candidate, warp-uniform trip counts
    if (b < 0) {
      for (int j0 = i + 1; j0 < sys_end; j0 += 32) {
        const int j = j0 + lane;
        visit(j, j < sys_end && norm2(diff<R>(ci, contact(s, j))) < rl2);
      }
      return;
    }
    for (int z = max(0, cz - 1); z <= min(d.nz - 1, cz + 1); z++)
      for (int y = max(0, cy - 1); y <= min(d.ny - 1, cy + 1); y++)
        for (int x = max(0, cx - 1); x <= min(d.nx - 1, cx + 1); x++) {
          const int c = d.cell0 + (z * d.ny + y) * d.nx + x;
          const int k0 = g.cell_start[c], k1 = k0 + g.cell_count[c];
          for (int kb = k0; kb < k1; kb += 32) {
            const int k = kb + lane;
            const int j = k < k1 ? g.sorted[k] : -1;
            visit(j, j > i && norm2(diff<R>(ci, contact(s, j))) < rl2);
          }
        }
  };
  int count = 0;
  scan([&](int, bool take) { count += __popc(__ballot_sync(0xffffffffu, take)); });
  int base = 0;
  if (lane == 0 && count) base = atomicAdd(&a.nl->npairs, count);
  base = __shfl_sync(0xffffffffu, base, 0);
  if (lane == 0) {
    if (base + count > a.pcap) atomicMax(&a.nl->overflow, base + count);
    a.ncount[i] = count;
    a.cb_build[i] = make_double4(ci.x, ci.y, ci.z, 0.0);
  }
  int at = base;
  if (count)
    scan([&](int j, bool take) {
      const unsigned m = __ballot_sync(0xffffffffu, take);
      const int k = at + __popc(m & ((1u << lane) - 1u));
      if (take && k < a.pcap) a.pairs[k] = make_int2(i, j);
      at += __popc(m);
    });
}

// a fixed grid of warps loops over the residues, so the launch costs little
// on the steps that do not rebuild
template <typename R>
__device__ __forceinline__ void nl_build_pass(const StepArgs<R> &a, const GridArgs &g, int n_launch, Span sp)
{
  const int lane = threadIdx.x & 31;
  for (int i = sp.t >> 5; i < n_launch; i += sp.nthr >> 5) nl_build_one(a, g, i, lane);
}

template <typename R> __global__ void k_nl_build(StepArgs<R> a, GridArgs g, int n_launch)
{
  if (!a.nl->rebuild) return;
  nl_build_pass(a, g, n_launch, grid_span());
}

// Pairs of the list, grid-stride (the count is known only on the device)
#define FOR_EACH_PAIR(a, p, sp) \
  for (int p = (sp).t, np_ = min((a).nl->npairs, (a).pcap); p < np_; p += (sp).nthr)
// Pairs of the near list (written by the density pass of this evaluation):
// index p is entry p % seg_len of segment p / seg_len, present when below
// that segment's count
#define FOR_EACH_NEAR_PAIR(a, p, sp)                                                                     \
  for (int p = (sp).t, S_ = (a).nl->seg_len, end_ = (a).nl->nseg * S_; p < end_; p += (sp).nthr)      \
    if (p - (p / S_) * S_ < (a).seg_n[p / S_])

// Density well value (FP64 in both forms).  The plain FP64 form evaluates
// the reference's 0.25 (1 + tanh(kappa (r - rmin))) (1 + tanh(kappa (rmax -
// r))); the mixed form the same from two exponentials,
// 1 / ((1 + e^(-2 kappa (r - rmin))) (1 + e^(-2 kappa (rmax - r)))), one
// division instead of the two inside two tanh (equal to about 1e-16).
template <typename R>
__device__ __forceinline__ double density_well(double r, double rmin_th, double rmax_th, double kappa, double rmin,
                                               double rmax)
{
  if constexpr (sizeof(R) == 4) {
    if (r < rmin_th || r > rmax_th) return 0.0;
    const double ea = exp(-2.0 * kappa * (r - rmin)), eb = exp(-2.0 * kappa * (rmax - r));
    return 1.0 / ((1.0 + ea) * (1.0 + eb));
  } else {
    double th, pr;
    well_theta(r, rmin_th, rmax_th, kappa, rmin, rmax, th, pr);
    return th;
  }
}

// DL1: local densities of contact beads (fix_backbone.cpp:7728-7791).  FP64
// in both forms: the densities feed the burial and switching functions (an
// FP32 well value here put the helix term of configuration 1 at 3e-5 of its
// small magnitude), and the well selection is the reference's exactly.  Sums
// in 2^-40 fixed point (dacc[0], dacc[1]).
template <typename R, bool SEL = false> __device__ __forceinline__ void density_pass(const StepArgs<R> &a, const FFParams &p, Span sp)
{
  const DevSys<R> &s = a.s;
  const int n = s.n_res;
  const bool fix = a.groups & G_FIX;
  const bool water = fix && (p.terms & T_WATER), helix = fix && (p.terms & T_HELIX);
  unsigned long long *aw = (unsigned long long *) a.dacc, *ah = aw + n;
  // the near list: the listed pairs some term can reach at this step (the
  // bound the list's validity check uses; the margin covers its rounding)
  const double need_sq = (double) a.nl->need * (double) a.nl->need * 1.00001;
  const int lane = threadIdx.x & 31, w = sp.t >> 5, nw = sp.nthr >> 5;
  const int np = min(a.nl->npairs, a.pcap);
  // one contiguous segment of the list per warp
  const int seg = max(32, ((np + nw - 1) / nw + 31) & ~31), nseg = (np + seg - 1) / seg;
  if (sp.t == 0) {
    a.nl->seg_len = seg;
    a.nl->nseg = nseg;
  }
  if (w >= nseg) return;
  const int lo = w * seg, hi = min(lo + seg, np);
  int cnt = 0;  // near pairs written so far (warp-uniform)
  for (int base = lo; base < hi; base += 32) {
    const int q = base + lane;
    int2 ij = {0, 0};
    double rsq = 0.0;
    bool near = false;
    if (q < hi) {
      ij = a.pairs[q];
      rsq = norm2(diff<double>(contact(s, ij.x), contact(s, ij.y)));
      near = rsq < need_sq;
    }
    const unsigned m = __ballot_sync(0xffffffffu, near);
    if (near) a.cpairs[lo + cnt + __popc(m & ((1u << lane) - 1u))] = ij;
    cnt += __popc(m);
    const int i = ij.x, j = ij.y;
    if (q >= hi || (s.res_chain[j] == s.res_chain[i] && j - i <= 1)) continue;
    const double r = sqrt(rsq);
    if (water && rsq > p.w_rmin_sq[0] && rsq < p.w_rmax_sq[0]) {
      const double th = density_well<R>(r, p.w_rmin_th[0], p.w_rmax_th[0], p.water_kappa, p.well_rmin[0], p.well_rmax[0]);
      const unsigned long long v = (unsigned long long) fix_dens(th);
      atomicAdd(aw + i, v);
      atomicAdd(aw + j, v);
      sel_rec<SEL>(a, AWSEM_SEL_DENS_WATER, 0, i, j);
    }
    if (helix && rsq > p.h_rmin_sq && rsq < p.h_rmax_sq) {
      const double th = density_well<R>(r, p.h_rmin_th, p.h_rmax_th, p.helix_kappa, p.helix_rmin, p.helix_rmax);
      const unsigned long long v = (unsigned long long) fix_dens(th);
      atomicAdd(ah + i, v);
      atomicAdd(ah + j, v);
      sel_rec<SEL>(a, AWSEM_SEL_DENS_HELIX, 0, i, j);
    }
  }
  if (lane == 0) a.seg_n[w] = cnt;
}

template <typename R> __global__ void k_density(StepArgs<R> a, FFParams p) { density_pass(a, p, grid_span()); }
template <typename R> __global__ void k_density_sel(StepArgs<R> a, FFParams p)
{
  density_pass<R, true>(a, p, grid_span());
}

// density sums -> values: k = 0 water density, 1 helix density
template <typename R> __device__ __forceinline__ double density(const StepArgs<R> &a, int k, int r)
{
  return (double) a.dacc[(size_t) k * a.s.n_res + r] * D_UNSCALE;
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
__device__ __forceinline__ R ev_pair(const StepArgs<R> &a, int ta, int tb, bool short_range, V3<R> d, V3<R> &f,
                                     bool *hit = nullptr)
{
  int N = a.ntypes + 1;
  double pref = a.ev_pref[ta * N + tb];
  f = {R(0), R(0), R(0)};
  if (pref == 0.0) return R(0);
  R rc = (R) (short_range ? a.ev_cs[ta * N + tb] : a.ev_cl[ta * N + tb]);
  R r = m_sqrt(norm2(d));
  if (!(r < rc)) return R(0);
  if (hit) *hit = true;
  R dr = r - rc;
  R pw = R(1);
  for (int k = 1; k < a.ev_p; k++) pw *= dr;  // dr^(p-1)
  R pr = R(pref) * pw;
  R fp = r > R(0) ? -pr * R(a.ev_p) / r : R(0);
  f = {d.x * fp, d.y * fp, d.z * fp};
  return pr * dr;
}

// bond_style harmonic, the bonds whose first atom is in residue r (run by
// k_residue's thread of that residue).  FP64 in both forms: a bond's energy
// k (r - r0)^2 is a small difference near equilibrium, and FP32 geometry put
// the bond energy of configuration 3 at 5e-6 relative.
template <typename R, typename Q>
__device__ __forceinline__ void bonds_of(const StepArgs<R> &a, const DevSys<Q> &s, int r)
{
  double e = 0.0;
  for (int b = r * a.bond_cap; b < (r + 1) * a.bond_cap && a.bond_i[b] >= 0; b++) {
    int ai = a.bond_i[b], aj = a.bond_j[b];
    V3<Q> d = diff<Q>(bead(s, ai / 3, ai % 3), bead(s, aj / 3, aj % 3));
    Q rr = m_sqrt(norm2(d));
    Q dr = rr - Q(a.bond_r0[b]);
    Q rk = Q(a.bond_k[b]) * dr;
    Q fb = rr > Q(0) ? Q(-2) * rk / rr : Q(0);
    e = __dadd_rn(e, (double) mul_rn(rk, dr));
    scatter(s, ai / 3, ai % 3, d.x * fb, d.y * fb, d.z * fb);
    scatter(s, aj / 3, aj % 3, -d.x * fb, -d.y * fb, -d.z * fb);
  }
  a.e_res[(size_t) E_BOND * s.n_res + r] = e;
}

// Parts of the per-residue pass: the density-dependent terms (switching,
// burial, helical pair), the excluded volume inside the residue and the
// bonds (RES_SL), and the backbone terms chain, chi and rama (RES_BB), which
// need only the positions and run as their own kernel beside the pair
// passes.
constexpr int RES_SL = 1, RES_BB = 2, RES_ALL = 3;

// SL and the per-residue backbone terms
template <typename R, bool SEL = false, int PART = RES_ALL>
__device__ __forceinline__ void residue_one(const StepArgs<R> &a, const FFParams &p, int i, ForceWindow win = {})
{
  DevSys<R> s = a.s;
  s.win = win;
  // the per-residue backbone terms (chain, chi, rama, helical pair) are a
  // small share of the work and some are sums of steep Gaussians: FP64 in
  // both forms
  const DevSys<double> sd = widen(s);
  int n = s.n_res, fl = s.res_flags[i];
  double *E = a.e_res;
  const bool fix = a.groups & G_FIX;
  if constexpr (PART & RES_SL) {
  bool water = fix && (p.terms & T_WATER), helix = fix && (p.terms & T_HELIX);
  double sw = 0, swp = 0, sh = 0, shp = 0;
  const double rw = density(a, 0, i), rh = density(a, 1, i);
  a.rho_w[i] = rw;
  a.rho_h[i] = rh;
  if (water) switching(rw, p.water_kappa_sigma, p.treshold, sw, swp);
  if (helix) switching(rh, p.helix_kappa_sigma, p.helix_treshold, sh, shp);
  a.sig_w[i] = sw;
  a.sigp_w[i] = swp;
  a.sig_h[i] = sh;
  a.sigp_h[i] = shp;
  double eb = 0.0, bc = 0.0;
  if (fix && (p.terms & T_BURIAL)) {
    double rho = rw;
    // a phosphorylated residue takes glutamate's burial gammas (fix_backbone.cpp:2887-2899)
    const double *g = s.tables + TB_BURIAL + 3 * ((fl & R_PHOSPH) ? 6 : s.res_type[i]);
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
      switching(density(a, 1, j), p.helix_kappa_sigma, p.helix_treshold, shj, shpj);
      unsigned gate = 0;
      eh = (double) helix_pair(sd, p, i, j, sh, shp, shj, shpj, x1, x2, SEL ? &gate : nullptr);
      sel_rec<SEL>(a, AWSEM_SEL_HELIX_PAIR, (int) gate, i, j);
    }
  }
  a.xi1[i] = x1;
  a.xi2[i] = x2;
  {
    RadRec &rr = a.rrec[i];
    rr.sw = sw;
    rr.bur = bc;
    rr.x1 = x1;
    rr.sigp = swp;
    rr.type = s.res_type[i];
    rr.flags = fl;
    rr.chain = s.res_chain[i];
    // xi2 is read at residue r + helix_i_diff: stored with that residue's
    // record; a record whose residue r - helix_i_diff is not integrated (no
    // residue, or a free residue of a serving handle) holds 0
    if (i + p.helix_i_diff < n) a.rrec[i + p.helix_i_diff].x2 = x2;
    if (i < p.helix_i_diff || a.res_sys[i - p.helix_i_diff] < 0) rr.x2 = 0.0;
  }
  E[(size_t) E_HELIX * n + i] = eh;
  }
  if constexpr (PART & RES_BB) {
  double ec = 0.0, ex = 0.0, er = 0.0;
  if (fix && (p.terms & T_CHAIN)) ec = (double) chain_term(sd, p, i);
  bool inner = fix && !(fl & (R_FIRST | R_LAST | R_GLY));
  if (inner && (p.terms & T_CHI)) ex = (double) chi_term(sd, p, i);
  if (inner && (p.terms & T_RAMA)) er = (double) rama_term(sd, p, i);
  E[(size_t) E_CHAIN * n + i] = ec;
  E[(size_t) E_CHI * n + i] = ex;
  E[(size_t) E_RAMA * n + i] = er;
  }
  if constexpr (PART & RES_SL) {
  // excluded volume inside the residue (1-3 pairs; 1-2 pairs are excluded)
  double ev = 0.0;
  unsigned ex_self = (a.groups & G_PAIR) ? a.excl_self[i] : 0x1ffu;
  for (int b0 = 0; b0 < 3; b0++)
    for (int b1 = b0 + 1; b1 < 3; b1++) {
      if (ex_self & (1u << (b0 * 3 + b1))) continue;
      V3<R> f;
      bool hit = false;
      R e = ev_pair(a, a.atom_type[3 * i + b0], a.atom_type[3 * i + b1], true,
                    diff<R>(bead(s, i, b0), bead(s, i, b1)), f, SEL ? &hit : nullptr);
      if (hit) sel_rec<SEL>(a, AWSEM_SEL_EV, 3 * b0 + b1, i, i);
      if (e != R(0) || f.x != R(0) || f.y != R(0) || f.z != R(0)) {
        ev += (double) e;
        scatter(s, i, b0, f);
        scatter(s, i, b1, -f.x, -f.y, -f.z);
      }
    }
  E[(size_t) E_PAIR * n + i] = ev;
  if (a.groups & G_BOND) bonds_of(a, sd, i);
  }
}

template <typename R, bool SEL = false> __device__ __forceinline__ void residue_pass(const StepArgs<R> &a, const FFParams &p, Span sp)
{
  for (int i = sp.t; i < a.n_run; i += sp.nthr)
    if (a.res_sys[i] >= 0) residue_one<R, SEL>(a, p, i);
}

// The standalone residue kernel: 128 residues per block and iteration; the
// forces its terms push to residues r0 - 1 .. r0 + 127 + helix_i_diff (the
// helical pair reaches i + 4) are summed in shared memory and flushed with
// one global atomic per non-zero component.  Each contribution is converted
// to fixed point before it is summed, so the result is the direct scatter's
// bit for bit.
constexpr int kResBlock = 128, kResHalo = 5, kResWin = kResBlock + kResHalo;
template <typename R, bool SEL, int PART> __device__ __forceinline__ void residue_pass_window(const StepArgs<R> &a, const FFParams &p)
{
  __shared__ unsigned long long acc[kResWin * 9];
  const uint32_t addr = (uint32_t) __cvta_generic_to_shared(acc);
  for (int r0 = blockIdx.x * kResBlock; r0 < a.n_run; r0 += gridDim.x * kResBlock) {
    for (int k = threadIdx.x; k < kResWin * 9; k += kResBlock) acc[k] = 0ull;
    __syncthreads();
    const int i = r0 + threadIdx.x;
    if (i < a.n_run && a.res_sys[i] >= 0) residue_one<R, SEL, PART>(a, p, i, ForceWindow{addr, r0 - 1, kResWin});
    __syncthreads();
    for (int k = threadIdx.x; k < kResWin * 9; k += kResBlock) {
      const unsigned long long v = acc[k];
      const int r = r0 - 1 + k / 9;
      if (v && r >= 0 && r < a.s.n_res) atomicAdd(a.s.facc + (size_t) 9 * r + k % 9, v);
    }
    __syncthreads();
  }
}
template <typename R> __global__ void __launch_bounds__(kResBlock, 4) k_residue(StepArgs<R> a, FFParams p)
{
  residue_pass_window<R, false, RES_SL>(a, p);
}
template <typename R> __global__ void __launch_bounds__(kResBlock, 4) k_backbone(StepArgs<R> a, FFParams p)
{
  residue_pass_window<R, false, RES_BB>(a, p);
}
template <typename R> __global__ void __launch_bounds__(kResBlock) k_residue_sel(StepArgs<R> a, FFParams p)
{
  residue_pass_window<R, true, RES_ALL>(a, p);
}

// DL2: water-mediated density derivative coefficients (fix_backbone.cpp:
// 7877-7954): raw sums in dacc[2] (2^-40 fixed point); xi_water(i) is that
// sum times sigma_water'(i) (water_xi below).
template <typename R, bool SEL = false> __device__ __forceinline__ void water_xi_pass(const StepArgs<R> &a, const FFParams &p, Span sp)
{
  const DevSys<R> &s = a.s;
  if (!(p.terms & T_WATER) || !(a.groups & G_FIX)) return;
  unsigned long long *acc = (unsigned long long *) a.dacc + (size_t) 2 * s.n_res;
  const double *WG = s.tables + TB_WATER;
  FOR_EACH_NEAR_PAIR(a, q, sp)
  {
    const int2 ij = a.cpairs[q];
    const int i = ij.x, j = ij.y;
    // the residues' packed records (written by the residue pass) and contact beads
    const RadRec ri = a.rrec[i], rj = a.rrec[j];
    if (rj.chain == ri.chain && j - i < p.contact_cutoff) continue;
    const R rsq = norm2(diff<R>(contact(s, i), contact(s, j)));
    const int ti = ri.type, tj = rj.type;
    // pairs with a phosphorylated residue use the phosphorylation gammas (fix_backbone.cpp:2872-2885)
    const double *W = ((p.terms & T_PHOSPH) && ((ri.flags | rj.flags) & R_PHOSPH)) ? s.tables + TB_WATER_PHOSPH : WG;
    for (int w = 0; w < p.n_wells; w++) {
      if (!p.well_flag[w]) continue;
      const double g0 = W[w * 800 + (ti * 20 + tj) * 2], g1 = W[w * 800 + (ti * 20 + tj) * 2 + 1];
      // the reference's `!fabs(g0 - g1) < delta` holds exactly when g0 != g1
      if (g0 != g1 && rsq > R(p.w_rmin_sq[w]) && rsq < R(p.w_rmax_sq[w])) {
        sel_rec<SEL>(a, AWSEM_SEL_XI_WATER, w, i, j);
        R th, pr;
        well_theta(m_sqrt(rsq), R(p.w_rmin_th[w]), R(p.w_rmax_th[w]), R(p.water_kappa), R(p.well_rmin[w]),
                   R(p.well_rmax[w]), th, pr);
        const double tg = (g1 - g0) * (double) th;
        atomicAdd(acc + i, (unsigned long long) fix_dens(tg * rj.sw));
        atomicAdd(acc + j, (unsigned long long) fix_dens(tg * ri.sw));
      }
    }
  }
}

template <typename R> __global__ void k_water_xi(StepArgs<R> a, FFParams p) { water_xi_pass(a, p, grid_span()); }
template <typename R> __global__ void k_water_xi_sel(StepArgs<R> a, FFParams p)
{
  water_xi_pass<R, true>(a, p, grid_span());
}

template <typename R> __device__ __forceinline__ double water_xi(const StepArgs<R> &a, int r)
{
  return (double) a.dacc[(size_t) 2 * a.s.n_res + r] * D_UNSCALE * a.sigp_w[r];
}

template <typename R> __device__ __forceinline__ void scatter_fix(const DevSys<R> &s, int r, int b, const long long f[3])
{
  unsigned long long *q = s.facc + ((size_t) 3 * r + b) * 3;
#pragma unroll
  for (int c = 0; c < 3; c++)
    if (f[c]) atomicAdd(q + c, (unsigned long long) f[c]);
}

// DL3 radial terms (fix_backbone.cpp:7956-8057, :8116-8128): the water,
// burial and helix wells of the contact beads of every near pair, one thread
// per pair; the radial force goes to both residues.
template <typename R, bool SEL = false> __device__ __forceinline__ void radial_pass(const StepArgs<R> &a, const FFParams &p, Span sp)
{
  const DevSys<R> &s = a.s;
  const bool fix = a.groups & G_FIX;
  if (!fix) return;
  const int n = s.n_res;
  const double *WG = s.tables + TB_WATER;
  const uint32_t T = p.terms;
  const int dh = p.helix_i_diff;
  unsigned long long *e_water = (unsigned long long *) a.e_fix + (size_t) 3 * n;
  FOR_EACH_NEAR_PAIR(a, q, sp)
  {
    const int2 ij = a.cpairs[q];
    const int i = ij.x, j = ij.y;
    // every per-residue input of the pair, loaded up front and without
    // conditions, so that the gathers are in flight together
    const RadRec ri = a.rrec[i], rj = a.rrec[j];
    const V3<double> c_i = contact(s, i), c_j = contact(s, j);
    const double ui = (double) a.dacc[(size_t) 2 * n + i], uj = (double) a.dacc[(size_t) 2 * n + j];
    const int fli = ri.flags, flj = rj.flags, ti = ri.type, tj = rj.type;
    const bool other = rj.chain != ri.chain;
    const double sw_i = ri.sw, sw_j = rj.sw, bur_i = ri.bur, bur_j = rj.bur;
    const double xi_i = ui * D_UNSCALE * ri.sigp, xi_j = uj * D_UNSCALE * rj.sigp;  // water_xi
    const double x1_i = ri.x1, x1_j = rj.x1, x2_i = ri.x2, x2_j = rj.x2;
    const int dij = j - i;
    // contact-bead radial terms
    if (other || dij > 1) {
      const bool gi = fli & R_GLY, gj = flj & R_GLY;
      const V3<R> d = diff<R>(c_i, c_j);
      const R rsq = norm2(d);
      const R r = m_sqrt(rsq);
      R force = 0;
      double ew = 0.0;
      const bool in0 = rsq > R(p.w_rmin_sq[0]) && rsq < R(p.w_rmax_sq[0]);
      R th0 = 0, pr0 = 0;
      if ((T & (T_WATER | T_BURIAL)) && in0)
        well_theta(r, R(p.w_rmin_th[0]), R(p.w_rmax_th[0]), R(p.water_kappa), R(p.well_rmin[0]), R(p.well_rmax[0]),
                   th0, pr0);
      if (T & T_WATER) {
        const bool sep = other || dij >= p.contact_cutoff;
        const double *W = ((fli | flj) & R_PHOSPH) ? s.tables + TB_WATER_PHOSPH : WG;
        for (int w = 0; w < p.n_wells; w++) {
          if (!p.well_flag[w]) continue;
          if (sep && rsq > R(p.w_rmin_sq[w]) && rsq < R(p.w_rmax_sq[w])) {
            sel_rec<SEL>(a, AWSEM_SEL_WATER, w, i, j);
            const double g0 = W[w * 800 + (ti * 20 + tj) * 2], g1 = W[w * 800 + (ti * 20 + tj) * 2 + 1];
            const double sg = fabs(g0 - g1) < 1e-5 ? 0.5 * (g0 + g1) : g0 + (g1 - g0) * sw_i * sw_j;
            R th, pr;
            if (w == 0) {
              th = th0;
              pr = pr0;
            } else {
              well_theta(r, R(p.w_rmin_th[w]), R(p.w_rmax_th[w]), R(p.water_kappa), R(p.well_rmin[w]),
                         R(p.well_rmax[w]), th, pr);
            }
            ew = madd(-sg, (double) th, ew);
            force = madd(R(sg), pr, force);
          }
        }
        if (in0) {
          const int on = (fabs(xi_i) > 1e-8 ? 1 : 0) | (fabs(xi_j) > 1e-8 ? 2 : 0);
          if (on & 1) force = madd(pr0, R(xi_i), force);
          if (on & 2) force = madd(pr0, R(xi_j), force);
          if (on) sel_rec<SEL>(a, AWSEM_SEL_XI_FORCE, on, i, j);
        }
      }
      if ((T & T_BURIAL) && in0) force = madd(R(bur_i + bur_j), pr0, force);
      if ((T & T_HELIX) && rsq > R(p.h_rmin_sq) && rsq < R(p.h_rmax_sq)) {
        double fac = x1_i + x1_j;
        if (i - dh >= 0) fac += x2_i;
        if (j - dh >= 0) fac += x2_j;
        if (fabs(fac) > 1e-6) {
          sel_rec<SEL>(a, AWSEM_SEL_HELIX_FORCE, 0, i, j);
          R th, pr;
          well_theta(r, R(p.h_rmin_th), R(p.h_rmax_th), R(p.helix_kappa), R(p.helix_rmin), R(p.helix_rmax), th, pr);
          force = madd(-R(fac), pr, force);
        }
      }
      if (ew != 0.0) atomicAdd(e_water + i, (unsigned long long) fix_force(ew));
      if (force != R(0)) {
        const long long f[3] = {fix_force((double) (force * d.x)), fix_force((double) (force * d.y)),
                                fix_force((double) (force * d.z))};
        const long long g[3] = {-f[0], -f[1], -f[2]};
        scatter_fix(s, i, gi ? B_CA : B_CB, f);
        scatter_fix(s, j, gj ? B_CA : B_CB, g);
      }
    }
  }
}

// blocks per SM the radial and detection passes are compiled for (the
// passes are latency bound: 8 blocks of 4 warps in FP32 fit in 64 registers
// without spills; the FP64 form holds twice the data)
template <typename R> constexpr int kPairMinBlocks = sizeof(R) == 4 ? 8 : 5;
template <typename R> __global__ void __launch_bounds__(128, kPairMinBlocks<R>) k_radial(StepArgs<R> a, FFParams p)
{
  radial_pass(a, p, grid_span());
}
template <typename R> __global__ void __launch_bounds__(128) k_radial_sel(StepArgs<R> a, FFParams p)
{
  radial_pass<R, true>(a, p, grid_span());
}

// DL3 pair detection (fix_backbone.cpp:8064-8103) and excluded volume
// between residues, one thread per near pair i < j.  DSSP and P_AP pairs
// are only detected here (cheap distance and index tests) and queued:
// k_hbond evaluates them, so their long, branchy bodies do not slow this
// pass.  Excluded volume is applied to both residues.
template <typename R, bool SEL = false> __device__ __forceinline__ void pair_pass(const StepArgs<R> &a, const FFParams &p, Span sp)
{
  const DevSys<R> &s = a.s;
  const int n = s.n_res;
  const bool fix = a.groups & G_FIX, evon = a.groups & G_PAIR;
  const uint32_t T = fix ? p.terms : 0u;
  const R ev_pre_sq = R(a.nl->ev_pre_sq), dssp_pre_sq = R(a.nl->dssp_pre_sq);
  // the largest excluded-volume cutoff, squared, with room for its rounding
  // to float and for the rounding of the bead distance
  const R ev_max_sq = R(a.nl->r_ev) * R(a.nl->r_ev) * R(1.0001);
  // smallest same-chain separation of any P_AP class (fix_backbone.cpp:3279-3383)
  const int pap_sep = min(p.i_med_min + 2 * p.i_diff_pap, p.i_med_max + 1);
  const size_t qd = 0, qp = (size_t) 2 * a.pcap;  // queue regions: DSSP (both orientations), P_AP
  unsigned long long *e_ev = (unsigned long long *) a.e_fix + (size_t) 4 * n;
  const int lane = threadIdx.x & 31, seg = a.nl->seg_len, np = a.nl->nseg * seg;
  // Queue entries are staged per warp in shared memory and written out 32 at
  // a time with one atomic reservation: one counter update per 32 entries
  // instead of one per warp iteration (same-address atomics serialise in L2).
  constexpr int kStageWarps = 8;  // warps per block of any caller
  __shared__ int stage_d[kStageWarps][96], stage_p[kStageWarps][64], stage_e[kStageWarps][64];
  int *const sd = stage_d[threadIdx.x >> 5], *const spp = stage_p[threadIdx.x >> 5];
  int *const se = stage_e[threadIdx.x >> 5];
  int nsd = 0, nsp = 0, nse = 0;  // staged entries (warp-uniform)
  // write the first `count` staged entries (count <= 32) to the queue at `region`, move the rest down
  auto flush = [&](int *buf, int &cnt, int count, int *counter, size_t region) {
    int at = 0;
    if (lane == 0) at = atomicAdd(counter, count);
    at = __shfl_sync(0xffffffffu, at, 0);
    if (lane < count) a.hbq[region + at + lane] = buf[lane];
    const int v1 = lane + 32 < cnt ? buf[lane + 32] : 0, v2 = lane + 64 < cnt ? buf[lane + 64] : 0;
    __syncwarp();
    buf[lane] = v1;
    buf[lane + 32] = v2;  // index < 64: inside both buffers
    __syncwarp();
    cnt -= count;
  };
  // Excluded volume between the beads of the staged pairs, in two steps.
  // First a lane per pair: which of its nine bead pairs (bead kinds CA, CB,
  // O = 0, 1, 2) can be in range -- not excluded (1-2 bonded pairs), a
  // type pair that interacts at those kinds, and |CA(i) - CA(j)| at most
  // the kinds' cutoff plus their reach from the CA.  Then a lane per
  // surviving bead pair, 32 at a time, so that the bead loads of a batch
  // are independent of one another.  Each bead pair's force and energy go
  // to fixed point and are added as they are found.
  // this step's bead-kind cutoffs (lanes 0-17: [short / long][b0][b1]) and
  // reaches (lanes 18-20), read once: the list state shares cache lines with
  // the queue counters this pass updates atomically, and reads of those
  // lines during the pass wait for the atomics
  const float tab = lane < 18 ? (&a.nl->ev_cutk[0][0][0])[lane] : lane < 21 ? a.nl->ev_reach[lane - 18] : 0.f;
  __shared__ int ev_item[kStageWarps][9 * 32];
  __shared__ int ev_pi[kStageWarps][32], ev_pj[kStageWarps][32];
  int *const items = ev_item[threadIdx.x >> 5], *const pi = ev_pi[threadIdx.x >> 5], *const pj = ev_pj[threadIdx.x >> 5];
  // run the first `count` staged EV pairs (count <= 32); move the rest down
  auto ev_batch = [&](int count) {
    const int q = lane < count ? se[lane] : -1;
    const int v1 = lane + 32 < nse ? se[lane + 32] : 0;
    __syncwarp();
    se[lane] = v1;
    __syncwarp();
    nse -= count;
    unsigned mask = 0u;  // bead pairs c = 3 b0 + b1 that may be in range
    int i = 0, j = 0, sh = 9;
    float dca = 0.f;
    if (q >= 0) {
      const int2 ij = a.cpairs[q];
      i = ij.x, j = ij.y;
      const bool shortr = s.res_chain[j] == s.res_chain[i] && j - i < 5;
      sh = shortr ? 0 : 9;
      const unsigned excl = j == i + 1 ? a.excl_next[i] : 0u;
      dca = sqrtf((float) norm2(diff<R>(bead(s, i, B_CA), bead(s, j, B_CA))));
      mask = ~excl & 0x1ffu;
    }
#pragma unroll
    for (int c = 0; c < 9; c++) {
      const float ck = __shfl_sync(0xffffffffu, tab, sh + c);
      const float r0 = __shfl_sync(0xffffffffu, tab, 18 + c / 3), r1 = __shfl_sync(0xffffffffu, tab, 18 + c % 3);
      if (!(ck > 0.f) || dca > ck + r0 + r1 + 0.01f) mask &= ~(1u << c);
    }
    pi[lane] = i;
    pj[lane] = j | (sh ? 0 : 1 << 30);  // bit 30: short range
    // exclusive prefix of the survivors over the lanes
    const int cnt = __popc(mask);
    int off = cnt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, off, d);
      if (lane >= d) off += t;
    }
    const int total = __shfl_sync(0xffffffffu, off, 31);
    off -= cnt;
    for (unsigned m = mask; m; m &= m - 1u) items[off++] = lane << 4 | (__ffs(m) - 1);
    __syncwarp();
    for (int b = 0; b < total; b += 32) {
      if (b + lane < total) {
        const int it = items[b + lane], src = it >> 4, c = it & 15, b0 = c / 3, b1 = c - 3 * b0;
        const int ii = pi[src], jw = pj[src], jj = jw & ((1 << 30) - 1);
        const bool shortr = jw >> 30;
        const V3<R> dd = diff<R>(bead(s, ii, b0), bead(s, jj, b1));
        if (norm2(dd) <= ev_max_sq) {  // beyond every cutoff: no table lookups
          V3<R> f;
          bool hit = false;
          const R e = ev_pair(a, a.atom_type[3 * ii + b0], a.atom_type[3 * jj + b1], shortr, dd, f, SEL ? &hit : nullptr);
          if (hit) sel_rec<SEL>(a, AWSEM_SEL_EV, c, ii, jj);
          if (e != R(0) || f.x != R(0) || f.y != R(0) || f.z != R(0)) {
            const long long v[3] = {fix_force((double) f.x), fix_force((double) f.y), fix_force((double) f.z)};
            const long long w[3] = {-v[0], -v[1], -v[2]};
            scatter_fix(s, ii, b0, v);
            scatter_fix(s, jj, b1, w);
            const long long ef = fix_force((double) e);
            if (ef) atomicAdd(e_ev + ii, (unsigned long long) ef);
          }
        }
      }
    }
    __syncwarp();
  };
  // warp-uniform trip count: the queue appends below are warp collectives
  // (a warp's 32 indices lie in one near-list segment: segments are multiples of 32 long)
  for (int base = sp.t - lane; base < np; base += sp.nthr) {
    const int q = base + lane, sg = base / seg, have = a.seg_n[sg] - (base - sg * seg);
    if (have <= 0) continue;  // warp-uniform: past this segment's near pairs
    bool q_d0 = false, q_d1 = false, q_p = false, q_e = false;  // queue: DSSP O(i), DSSP O(j), P_AP; stage: EV
    if (lane < have) {
    const int2 ij = a.cpairs[q];
    const int i = ij.x, j = ij.y;
    // (the topology arrays, not the residue pass's records: this pass runs
    // beside the residue pass)
    const int fli = s.res_flags[i], flj = s.res_flags[j];
    const bool other = s.res_chain[j] != s.res_chain[i];
    const V3<double> ca_i = bead(s, i, B_CA), ca_j = bead(s, j, B_CA);
    const int dij = j - i;
    const R rca2 = norm2(diff<R>(ca_i, ca_j));
    // excluded volume between beads of i and j: staged (below), so that the
    // few pairs this close run their 3 x 3 bead loop with full warps
    q_e = evon && rca2 < ev_pre_sq;
    // DSSP (fix_backbone.cpp:8064-8094): O(i) with N-H(j), and O(j) with N-H(i)
    if ((T & T_DSSP) && (other || dij > 2) && rca2 < dssp_pre_sq) {
      q_d0 = !(flj & (R_PRO | R_FIRST)) && !(fli & R_LAST) &&
             norm2(diff<R>(bead(s, i, B_O), bead(s, j, B_N))) < R(p.dssp_cut_sq);
      q_d1 = !(fli & (R_PRO | R_FIRST)) && !(flj & R_LAST) &&
             norm2(diff<R>(bead(s, j, B_O), bead(s, i, B_N))) < R(p.dssp_cut_sq);
    }
    // P_AP on CA pairs (fix_backbone.cpp:8096-8103)
    q_p = (T & T_PAP) && (other || dij >= pap_sep) && rca2 < R(p.pap_cutoff_sq);
    }
    // stage this iteration's queue entries (at most 64 DSSP and 32 P_AP)
    const unsigned m0 = __ballot_sync(0xffffffffu, q_d0), m1 = __ballot_sync(0xffffffffu, q_d1),
                   mp = __ballot_sync(0xffffffffu, q_p), me = __ballot_sync(0xffffffffu, q_e);
    const unsigned below = (1u << lane) - 1u;
    if (q_d0) sd[nsd + __popc(m0 & below)] = q;
    if (q_d1) sd[nsd + __popc(m0) + __popc(m1 & below)] = ~q;
    if (q_p) spp[nsp + __popc(mp & below)] = q;
    if (q_e) se[nse + __popc(me & below)] = q;
    nsd += __popc(m0) + __popc(m1);
    nsp += __popc(mp);
    nse += __popc(me);
    __syncwarp();
    while (nsd >= 32) flush(sd, nsd, 32, &a.nl->n_dssp, qd);
    if (nsp >= 32) flush(spp, nsp, 32, &a.nl->n_pap, qp);
    if (nse >= 32) ev_batch(32);
  }
  if (nsd > 0) flush(sd, nsd, nsd, &a.nl->n_dssp, qd);
  if (nsp > 0) flush(spp, nsp, nsp, &a.nl->n_pap, qp);
  if (nse > 0) ev_batch(nse);
}

template <typename R> __global__ void __launch_bounds__(128, kPairMinBlocks<R>) k_pair(StepArgs<R> a, FFParams p)
{
  pair_pass(a, p, grid_span());
}
template <typename R> __global__ void __launch_bounds__(128) k_pair_sel(StepArgs<R> a, FFParams p)
{
  pair_pass<R, true>(a, p, grid_span());
}

// DSSP hydrogen bonds and P_AP of the queued pairs, one thread per entry
// (grid-stride over both queues).  A DSSP entry q >= 0 is pair q with O(i)
// as acceptor; ~q is the same pair with O(j).  Forces scatter with
// fixed-point atomics; each pair's energy goes to its acceptor (DSSP) or
// lower residue (P_AP) in fixed point, so sums do not depend on the order.
template <typename R, bool SEL = false> __device__ __forceinline__ void hbond_pass(const StepArgs<R> &a, const FFParams &p, Span sp)
{
  const DevSys<R> &s = a.s;
  const int nd = a.nl->n_dssp, np = a.nl->n_pap, n = s.n_res;
  for (int t = sp.t; t < nd + np; t += sp.nthr) {
    const bool d = t < nd;
    const int q = d ? a.hbq[t] : a.hbq[(size_t) 2 * a.pcap + (t - nd)];
    const int2 ij = a.cpairs[q < 0 ? ~q : q];
    const int i = q < 0 ? ij.y : ij.x, j = q < 0 ? ij.x : ij.y;
    unsigned gate = 0;
    const R e = d ? dssp_term(s, p, i, j, SEL ? &gate : nullptr) : pap_term(s, p, i, j, SEL ? &gate : nullptr);
    sel_rec<SEL>(a, d ? AWSEM_SEL_DSSP : AWSEM_SEL_PAP, (int) gate, i, j);
    if (e != R(0))
      atomicAdd((unsigned long long *) (a.e_fix + (d ? 0 : (size_t) n) + i), (unsigned long long) fix_force((double) e));
  }
}

// blocks per SM the hydrogen-bond pass is compiled for (the FP64 form needs
// the registers of 4 blocks to keep its terms out of local memory)
template <typename R> constexpr int kHbondMinBlocks = sizeof(R) == 4 ? 6 : 4;
template <typename R> __global__ void __launch_bounds__(128, kHbondMinBlocks<R>) k_hbond(StepArgs<R> a, FFParams p)
{
  hbond_pass(a, p, grid_span());
}
template <typename R> __global__ void __launch_bounds__(128) k_hbond_sel(StepArgs<R> a, FFParams p)
{
  hbond_pass<R, true>(a, p, grid_span());
}

// Fragment memory: sliced lane-interleaved table, lane per residue row
// (awsem_fragmem.cuh)
template <typename R> struct BeadPos {
  const DevSys<R> *s;
  __device__ __forceinline__ V3<double> operator()(int r, int b) const { return bead(*s, r, b ? B_CB : B_CA); }
};

// 128 threads, fm_warp_smem<R>(coef) bytes of dynamic shared memory per warp
template <typename R> __global__ void __launch_bounds__(128) k_fragmem(StepArgs<R> a, FFParams p)
{
  extern __shared__ __align__(128) unsigned char fm_smem[];
  const BeadPos<R> pos{&a.s};
  unsigned char *wsm = fm_smem + (threadIdx.x >> 5) * fm_warp_smem<R>(a.fm.coef != nullptr);
  fragmem_warp_take(a.fm, p.fm_sigma_sq, a.s.n_res, pos, a.s.facc,
                    (unsigned long long *) (a.e_fix + (size_t) 2 * a.s.n_res), 1, &a.nl->fm_timeout, wsm,
                    &a.nl->fm_next);
}

// Table fragment memory of residue i and separation slot jo
// (FixBackbone::table_fragment_memory, fix_backbone.cpp:4325-4429, called
// for j = i + min_sep .. min(i + max_sep, the chain's last residue) at
// :7513-7527): energy and force factor interpolated linearly between the two
// grid points around r, for the atom pairs CA-CA, CA-CB, CB-CA, CB-CB in that
// order.  As in the reference, a pair without a CA-CA table is skipped, the
// first atom pair without a table ends the pair, and a distance outside the
// table's range is an error (flagged; the host reports it).  FP64 in both
// forms; energy and forces to fixed point.
template <typename R> __device__ __forceinline__ void fm_table_pair(const StepArgs<R> &a, const FFParams &p, int i, int jo)
{
  const DevSys<R> &s = a.s;
  const int j = i + p.fm_min_sep + jo;
  if (a.res_sys[i] < 0 || j > s.chain_end[s.res_chain[i]]) return;
  const size_t t0 = ((size_t) i * p.tb_nbrs + jo) * 4;
  if (!a.tb_present[t0]) return;
  const bool gi = s.res_flags[i] & R_GLY, gj = s.res_flags[j] & R_GLY;
  double e = 0.0;
  long long fi[2][3] = {{0, 0, 0}, {0, 0, 0}}, fj[2][3] = {{0, 0, 0}, {0, 0, 0}};
  for (int k = 0; k < 4; k++) {
    const int bi = k >= 2 ? 1 : 0, bj = k & 1;  // 0 CA, 1 CB
    if ((bi && gi) || (bj && gj)) continue;
    const V3<double> xi = bead(s, i, bi ? B_CB : B_CA), xj = bead(s, j, bj ? B_CB : B_CA);
    const V3<double> dx = {xi.x - xj.x, xi.y - xj.y, xi.z - xj.z};
    const double r = sqrt(norm2(dx));
    if (!(r >= p.tb_rmin && r <= p.tb_rmax)) {
      atomicMax(&a.nl->tb_error, 1);
      break;
    }
    const int ir = (int) ((r - p.tb_rmin) / p.tb_dr);
    if (!a.tb_present[t0 + k]) break;
    if (ir < 0 || ir + 1 >= p.tb_size) {
      atomicMax(&a.nl->tb_error, 2);
      break;
    }
    const double r1 = p.tb_rmin + (double) ir * p.tb_dr, r2 = p.tb_rmin + (double) (ir + 1) * p.tb_dr;
    const double2 *T = a.tb_data + (t0 + k) * p.tb_size;
    const double2 q1 = T[ir], q2 = T[ir + 1];
    e += ((q2.x - q1.x) * r + q1.x * r2 - q2.x * r1) / (r2 - r1);
    const double ff = ((q2.y - q1.y) * r + q1.y * r2 - q2.y * r1) / (r2 - r1);
    const long long v[3] = {fix_force(ff * dx.x), fix_force(ff * dx.y), fix_force(ff * dx.z)};
#pragma unroll
    for (int c = 0; c < 3; c++) {
      fi[bi][c] += v[c];
      fj[bj][c] -= v[c];
    }
  }
  scatter_fix(s, i, B_CA, fi[0]);
  if (!gi) scatter_fix(s, i, B_CB, fi[1]);
  scatter_fix(s, j, B_CA, fj[0]);
  if (!gj) scatter_fix(s, j, B_CB, fj[1]);
  if (e != 0.0) atomicAdd((unsigned long long *) (a.e_fix + (size_t) 2 * s.n_res + i), (unsigned long long) fix_force(e));
}

template <typename R> __device__ __forceinline__ void fm_table_pass(const StepArgs<R> &a, const FFParams &p, Span sp)
{
  const long long items = (long long) a.n_run * p.tb_nbrs;
  for (long long t = sp.t; t < items; t += sp.nthr) fm_table_pair(a, p, (int) (t / p.tb_nbrs), (int) (t % p.tb_nbrs));
}

template <typename R> __global__ void k_fm_table(StepArgs<R> a, FFParams p) { fm_table_pass(a, p, grid_span()); }

// LAMMPS Neighbor::decide() per replica, for the emulated lists: built at a
// run setup; otherwise `ago` counts the steps since the last build and the
// lists are rebuilt once ago >= delay and ago % every == 0, unconditionally
// without check, with check only if an atom has moved more than half the
// skin since that build (lst_over, set by the prepare pass).  On a handle
// driven by awsem_compute the host decides (lst_setup alone).  Runs between
// the prepare pass and the passes that read lst_build; the finish pass then
// records the positions of a build.
__device__ __forceinline__ void list_decide_one(const NLState &nl, int *ago, int *over, int *built, int rep)
{
  bool b;
  if (nl.lst_setup) {
    b = true;
  } else if (nl.lst_host) {
    b = false;
  } else {
    const int g = ago[rep] + 1;
    b = g >= nl.lst_delay && g % nl.lst_every == 0 && (!nl.lst_check || over[rep] != 0);
  }
  built[rep] = b;
  ago[rep] = b ? 0 : ago[rep] + 1;
  over[rep] = 0;
}

__global__ void k_list_decide(const NLState *nl, int n_sys, int *ago, int *over, int *built)
{
  const int rep = blockIdx.x * blockDim.x + threadIdx.x;
  if (rep < n_sys) list_decide_one(*nl, ago, over, built, rep);
}

// awsem_compute has no finish pass: record the positions of a build here
template <typename R> __global__ void k_list_hold(StepArgs<R> a)
{
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= a.n_run || a.res_sys[r] < 0 || !a.lst_build[a.res_sys[r]]) return;
  for (int k = 0; k < 9; k++) a.lst_x0[(size_t) 9 * r + k] = a.x[(size_t) 9 * r + k];
}

// Terms of the reference's DL3 loop (fix_backbone.cpp:7956-8134) that the
// benchmark force field leaves off, one thread per listed residue pair i < j,
// on the second stream beside the pair passes:
//   contact restraints (:8058-8060, :8152-8177) on the contact beads, for
//     restrained pairs closer than the global cutoff that are in the fix's
//     half list (contact beads within the pair-list cutoff plus the skin at
//     the last list build);
//   solvent-separated barrier (:8109-8110, :6237-6305) and Debye-Hueckel
//     (:8112-8113, :6307-6363), evaluated for every CA pair of the fix's half
//     list -- CAs within the pair-list cutoff plus the skin at the replica's
//     last list build, 1-2 bonded pairs removed -- on the contact beads.
// Forces to the fixed-point accumulators; energies to fixed-point slots 5-7.
template <typename R> __device__ __forceinline__ void pair_extra_pass(const StepArgs<R> &a, const FFParams &p, Span sp)
{
  const DevSys<R> &s = a.s;
  const int n = s.n_res;
  if (!(a.groups & G_FIX)) return;
  const uint32_t T = p.terms;
  unsigned long long *e_ssb = (unsigned long long *) a.e_fix + (size_t) 5 * n;
  unsigned long long *e_dh = (unsigned long long *) a.e_fix + (size_t) 6 * n;
  unsigned long long *e_cr = (unsigned long long *) a.e_fix + (size_t) 7 * n;
  const double cut = p.pair_list_cutoff + a.nl->lst_skin, cutsq = cut * cut;
  const int np = min(a.nl->npairs, a.pcap);
  for (int q = sp.t; q < np; q += sp.nthr) {
    const int2 ij = a.pairs[q];
    const int i = ij.x, j = ij.y;
    const bool other = s.res_chain[j] != s.res_chain[i];
    const int dij = j - i;
    if (!other && dij <= 1) continue;  // the contact-bead branch and every CA-pair term need more
    const bool gi = s.res_flags[i] & R_GLY, gj = s.res_flags[j] & R_GLY;
    const V3<double> ci = bead(s, i, gi ? B_CA : B_CB), cj = bead(s, j, gj ? B_CA : B_CB);
    const V3<double> d = {ci.x - cj.x, ci.y - cj.y, ci.z - cj.z};
    const double rsq = norm2(d);
    double force = 0.0;
    const bool build = a.lst_build[a.res_sys[i]];
    const double *h = a.lst_x0;
    // contact restraints: the restraint listed for (i, j), if any
    bool cr_on = (T & T_CONTREST) && a.cr_start[i] < a.cr_start[i + 1] && rsq < p.cr_cut_sq;
    if (cr_on && !build) {  // on a build step the bead pair is within reach (rsq < cr_cut_sq <= cutsq)
      const int bi = 9 * i + 3 * (gi ? 0 : 1), bj = 9 * j + 3 * (gj ? 0 : 1);
      cr_on = norm2(V3<double>{h[bi] - h[bj], h[bi + 1] - h[bj + 1], h[bi + 2] - h[bj + 2]}) < cutsq;
    }
    if (cr_on) {
      for (int k = a.cr_start[i]; k < a.cr_start[i + 1]; k++) {
        if (a.cr_j[k] != j) continue;
        const double r = sqrt(rsq), dr = r - a.cr_r0[k];
        if (fabs(dr) < p.cr_dr_cut) {
          const double V = -a.cr_w[k] * exp(-0.5 * (dr * dr) * p.cr_sigma_sq_inv);
          force += V * dr * p.cr_sigma_sq_inv / r;
          atomicAdd(e_cr + i, (unsigned long long) fix_force(V));
        }
        break;
      }
    }
    // CA pair of the fix's half list?
    if (T & (T_SSB | T_DH)) {
      const double *c = build ? a.x : h;
      bool in_list = norm2(V3<double>{c[9 * i] - c[9 * j], c[9 * i + 1] - c[9 * j + 1], c[9 * i + 2] - c[9 * j + 2]}) < cutsq;
      if (in_list && dij == 1 && (a.excl_next[i] & 1u)) in_list = false;  // CA(i)-CA(i+1) bonded
      if (in_list) {
        const double r = sqrt(rsq);
        if ((T & T_SSB) && (other || dij >= p.ssb_ij_sep)) {
          double rmin1 = p.ssb_rmin1, rmax1 = p.ssb_rmax1, rmin2 = p.ssb_rmin2, rmax2 = p.ssb_rmax2;
          if (p.ssb_rad_cor) {
            const double sh = p.ssb_rshift[s.res_type[i]] + p.ssb_rshift[s.res_type[j]];
            rmin1 += sh;
            rmax1 += sh;
            rmin2 += sh;
            rmax2 += sh;
          }
          if (!(r > rmax1 + 10 / p.ssb_kappa && r > rmax2 + 10 / p.ssb_kappa)) {
            const double tn1 = tanh(p.ssb_kappa * (r - rmin1)), tx1 = tanh(p.ssb_kappa * (rmax1 - r));
            const double tn2 = tanh(p.ssb_kappa * (r - rmin2)), tx2 = tanh(p.ssb_kappa * (rmax2 - r));
            const double th1 = 0.5 * (tn1 + tx1), th2 = 0.5 * (tn2 + tx2);
            const double e = p.epsilon * p.k_ssb1 * th1 + p.epsilon * p.k_ssb2 * th2;
            atomicAdd(e_ssb + i, (unsigned long long) fix_force(e));
            force += -p.epsilon * p.k_ssb1 * p.ssb_kappa * th1 * (tx1 - tn1) / r;
            force += -p.epsilon * p.k_ssb2 * p.ssb_kappa * th2 * (tx2 - tn2) / r;
          }
        }
        if ((T & T_DH) && dij > 1 && dij >= p.dh_min_sep) {
          const double qi = a.charge[i], qj = a.charge[j];
          double qq = 0.0;
          if (qi > 0.0 && qj > 0.0) qq = p.k_plusplus * qi * qj / r;
          else if (qi < 0.0 && qj < 0.0) qq = p.k_minusminus * qi * qj / r;
          else if ((qi < 0.0 && qj > 0.0) || (qi > 0.0 && qj < 0.0)) qq = p.k_plusminus * qi * qj / r;
          if (qq != 0.0) {
            const double e = p.epsilon * qq * exp(-p.k_screening * r / p.screening_length);
            atomicAdd(e_dh + i, (unsigned long long) fix_force(e));
            force += (e / r) * (1.0 / r + p.k_screening / p.screening_length);
          }
        }
      }
    }
    if (force != 0.0) {
      const long long f[3] = {fix_force(force * d.x), fix_force(force * d.y), fix_force(force * d.z)};
      const long long g[3] = {-f[0], -f[1], -f[2]};
      scatter_fix(s, i, gi ? B_CA : B_CB, f);
      scatter_fix(s, j, gj ? B_CA : B_CB, g);
    }
  }
}

template <typename R> __global__ void k_pair_extra(StepArgs<R> a, FFParams p) { pair_extra_pass(a, p, grid_span()); }

// Per-residue terms the benchmark force field leaves off, thread per residue,
// FP64 in both forms, on the second stream: Shake (compute_shake,
// fix_backbone.cpp:2172-2237) and the membrane potential
// (compute_membrane_potential, :6107-6235) on the contact bead.
template <typename R> __device__ __forceinline__ void residue_extra_one(const StepArgs<R> &a, const FFParams &p, int i)
{
  const DevSys<R> &s = a.s;
  const int n = s.n_res, fl = s.res_flags[i];
  if (p.terms & T_SHAKE) {
    // harmonic CA(i)-CA(i+1), CA(i)-O(i), O(i)-CA(i+1) (the first and last not at a chain end)
    double e = 0.0;
    long long fca[3] = {0, 0, 0}, fo[3] = {0, 0, 0}, fnx[3] = {0, 0, 0};
    const V3<double> ca = bead(s, i, B_CA), o = bead(s, i, B_O);
    auto spring = [&](V3<double> u, V3<double> v, double r0, long long *fu, long long *fv) {
      const double dx[3] = {u.x - v.x, u.y - v.y, u.z - v.z};
      const double r = sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]), dr = r - r0;
      const double force = 2 * p.epsilon * p.k_shake * dr / r;
      e += p.epsilon * p.k_shake * dr * dr;
      for (int c = 0; c < 3; c++) {
        fu[c] += fix_force(-dx[c] * force);
        fv[c] += fix_force(dx[c] * force);
      }
    };
    const bool last = fl & R_LAST;
    V3<double> ca1{0, 0, 0};
    if (!last) {
      ca1 = bead(s, i + 1, B_CA);
      spring(ca, ca1, p.r_sh1, fca, fnx);
    }
    spring(ca, o, p.r_sh2, fca, fo);
    if (!last) spring(o, ca1, p.r_sh3, fo, fnx);
    scatter_fix(s, i, B_CA, fca);
    scatter_fix(s, i, B_O, fo);
    if (!last) scatter_fix(s, i + 1, B_CA, fnx);
    a.e_res[(size_t) E_SHAKE * n + i] = e;
  }
  if (p.terms & T_MEMB) {
    const bool gly = fl & R_GLY;
    const V3<double> xi = bead(s, i, gly ? B_CA : B_CB);
    const double dx = xi.x - p.memb_xo[0], dy = xi.y - p.memb_xo[1], dz = xi.z - p.memb_xo[2];
    const double ma = p.rho0_distor * p.rho0_max, mb = p.memb_len / 2;
    const double rho = sqrt(dx * dx + dy * dy);
    const double rho0 = (p.rho0_max - ma) + (ma / p.memb_len) * (dz + mb);
    const double kb = p.k_bin;
    const double t_per = tanh(kb * (dz - mb)), t_m1 = tanh(kb * (dz + mb)), t_m2 = tanh(kb * (mb - dz));
    const double t_cyt = tanh(kb * (-mb - dz)), t_por = tanh(kb * (rho - rho0));
    const double s_per = 0.5 * (1 + t_per), s_mem = 0.5 * (t_m1 + t_m2), s_cyt = 0.5 * (1 + t_cyt);
    const double s_por = 0.5 * (1 - t_por), s_nopor = 1 - s_por;
    const double dz_per = 0.5 * kb * (1 - t_per * t_per);
    const double dz_mem = -0.5 * kb * (t_m1 * t_m1) + 0.5 * kb * (t_m2 * t_m2);
    const double dz_cyt = -0.5 * kb * (1 - t_cyt * t_cyt);
    const double dr1_dz = ma / p.memb_len;
    const double dz_s_por = 0.5 * kb * (1 - t_por * t_por) * dr1_dz;
    const double dx_s_por = ((-0.5 * kb * dx) / rho) * (1 - t_por * t_por);
    const double dy_s_por = ((-0.5 * kb * dy) / rho) * (1 - t_por * t_por);
    const double dz_s_por_smem = s_mem * dz_s_por + dz_mem * s_por;
    const double dz_s_nopor_smem = s_mem * -dz_s_por + dz_mem * s_nopor;
    // zones 1 and 3 share one sign pattern, zone 2 the opposite one
    const int z = a.zim[i] - 1;
    const double *g = p.g_memb[z];
    const double sg = z == 1 ? -1.0 : 1.0;
    const double V = sg * ((-g[0] * s_per) + (-g[1] * s_cyt) + (g[2] * s_mem * s_nopor) + (-g[3] * s_mem * s_por));
    const double dVx = sg * (g[2] * s_mem * -dx_s_por + (-g[3]) * s_mem * dx_s_por);
    const double dVy = sg * (g[2] * s_mem * -dy_s_por + (-g[3]) * s_mem * dy_s_por);
    const double dVz = sg * (-g[0] * dz_per + (-g[1]) * dz_cyt + g[2] * dz_s_nopor_smem + (-g[3]) * dz_s_por_smem);
    const double k = p.epsilon * p.k_overall_memb;
    const long long f[3] = {fix_force(-k * dVx), fix_force(-k * dVy), fix_force(-k * dVz)};
    scatter_fix(s, i, gly ? B_CA : B_CB, f);
    a.e_res[(size_t) E_MEMB * n + i] = k * V;
  }
}

// Vector fragment memory (compute_vector_fragment_memory_potential,
// fix_backbone.cpp:3994-4077) of residue i: per record (partner j, the
// memory's CA->CB angle), V = -eps k exp(-(theta - theta_mem)^2 / 2 sigma^2)
// with theta the angle between the CA->CB vectors of i and j.
template <typename R> __device__ __forceinline__ void vfm_one(const StepArgs<R> &a, const FFParams &p, int i)
{
  const DevSys<R> &s = a.s;
  const int c0 = a.vfm_start[i], c1 = a.vfm_start[i + 1];
  double E = 0.0;
  if (c0 < c1) {
    const V3<double> cai = bead(s, i, B_CA), cbi = bead(s, i, B_CB);
    const double vi[3] = {cbi.x - cai.x, cbi.y - cai.y, cbi.z - cai.z};
    const double vmsqi = vi[0] * vi[0] + vi[1] * vi[1] + vi[2] * vi[2], vmi = sqrt(vmsqi);
    const double ek = p.epsilon * p.k_vfm;
    long long fi[3] = {0, 0, 0};
    for (int c = c0; c < c1; c++) {
      const int j = a.vfm_j[c];
      const V3<double> caj = bead(s, j, B_CA), cbj = bead(s, j, B_CB);
      const double vj[3] = {cbj.x - caj.x, cbj.y - caj.y, cbj.z - caj.z};
      const double vmsqj = vj[0] * vj[0] + vj[1] * vj[1] + vj[2] * vj[2], vmj = sqrt(vmsqj);
      const double vp = vi[0] * vj[0] + vi[1] * vj[1] + vi[2] * vj[2];
      const double vpn = vp / (vmi * vmj);
      const double dg = acos(vpn) - a.vfm_angle[c];
      const double V = -ek * exp(-dg * dg / (2 * p.vfm_sigma_sq));
      E += V;
      const double force = -V * dg / (p.vfm_sigma_sq * vmi * vmj * sqrt(1 - vpn * vpn));
      long long fj[3], mfj[3];
      for (int k = 0; k < 3; k++) {
        const long long v = fix_force(force * (vj[k] - vi[k] * vp / vmsqi));
        fi[k] += v;
        fj[k] = fix_force(force * (vi[k] - vj[k] * vp / vmsqj));
        mfj[k] = -fj[k];
      }
      scatter_fix(s, j, B_CA, mfj);
      scatter_fix(s, j, B_CB, fj);
    }
    const long long mfi[3] = {-fi[0], -fi[1], -fi[2]};
    scatter_fix(s, i, B_CA, mfi);
    scatter_fix(s, i, B_CB, fi);
  }
  a.e_res[(size_t) E_VFRAGMEM * s.n_res + i] = E;
}

template <typename R> __device__ __forceinline__ void residue_extra_pass(const StepArgs<R> &a, const FFParams &p, Span sp)
{
  if (!(a.groups & G_FIX)) return;
  for (int r = sp.t; r < a.n_run; r += sp.nthr)
    if (a.res_sys[r] >= 0) {
      if (p.terms & (T_SHAKE | T_MEMB)) residue_extra_one(a, p, r);
      if (p.terms & T_VFM) vfm_one(a, p, r);
    }
}

template <typename R> __global__ void k_residue_extra(StepArgs<R> a, FFParams p) { residue_extra_pass(a, p, grid_span()); }

// AMH-Go (FixBackbone::compute_amh_go_model, fix_backbone.cpp:3856-3992) of
// residue r's CA and CB: over each atom's native contacts (the full-list
// partners with a native distance below rc) that are in the fix's full
// neighbour list -- pairs within the pair-list cutoff plus the skin at the
// list's last build (k_list_decide), which a build step records -- and whose deviation passes
// dr^2 < 27.6 sigma^2, E_i = sum gamma exp(-dr^2 / 2 sigma^2); the atom's
// energy is -k E_i^p / (2 a) and each contact's force is scaled by
// -k p E_i^(p-1) / (2 a) (a: the normalisation).  FP64 in both forms; forces
// to fixed point, the energy to the residue's slot.
template <typename R> __device__ __forceinline__ void amh_go_residue(const StepArgs<R> &a, const FFParams &p, int r)
{
  const DevSys<R> &s = a.s;
  const bool build = a.lst_build[a.res_sys[r]];
  const double cut = p.pair_list_cutoff + a.nl->lst_skin, cutsq = cut * cut;
  double E = 0.0;
  for (int b = 0; b < 2; b++) {
    const int c0 = a.go_start[2 * r + b], c1 = a.go_start[2 * r + b + 1];
    if (c0 == c1) continue;
    const V3<double> xi = bead(s, r, b ? B_CB : B_CA);
    double Ei = 0.0;
    for (int c = c0; c < c1; c++) {
      const int q = a.go_partner[c];
      const V3<double> xj = bead(s, q / 3, (q % 3) ? B_CB : B_CA);
      const V3<double> dx = {xi.x - xj.x, xi.y - xj.y, xi.z - xj.z};
      const double rsq = norm2(dx);
      if (build) a.go_in[c] = rsq < cutsq;
      if (!a.go_in[c]) continue;
      const double dr = sqrt(rsq) - a.go_rnat[c], drsq = dr * dr, sig_sq = a.go_sig_sq[c];
      if (drsq < 27.6 * sig_sq) Ei += a.go_gamma[c] * exp(-drsq / (2.0 * sig_sq));
    }
    const double factor = -0.5 * p.k_amh_go * p.amh_go_p * pow(Ei, p.amh_go_p - 1) / a.go_norm[r];
    double fi[3] = {0.0, 0.0, 0.0};
    for (int c = c0; c < c1; c++) {
      if (!a.go_in[c]) continue;
      const int q = a.go_partner[c];
      const V3<double> xj = bead(s, q / 3, (q % 3) ? B_CB : B_CA);
      const V3<double> dx = {xi.x - xj.x, xi.y - xj.y, xi.z - xj.z};
      const double rr = sqrt(norm2(dx)), dr = rr - a.go_rnat[c], drsq = dr * dr, sig_sq = a.go_sig_sq[c];
      if (!(drsq < 27.6 * sig_sq)) continue;
      const double Eij = a.go_gamma[c] * exp(-drsq / (2.0 * sig_sq));
      const double force = Eij * dr / (sig_sq * rr);
      fi[0] += force * dx.x;
      fi[1] += force * dx.y;
      fi[2] += force * dx.z;
      const long long fj[3] = {fix_force(factor * (-force * dx.x)), fix_force(factor * (-force * dx.y)),
                               fix_force(factor * (-force * dx.z))};
      scatter_fix(s, q / 3, (q % 3) ? B_CB : B_CA, fj);
    }
    const long long fq[3] = {fix_force(factor * fi[0]), fix_force(factor * fi[1]), fix_force(factor * fi[2])};
    scatter_fix(s, r, b ? B_CB : B_CA, fq);
    E += -0.5 * p.k_amh_go * pow(Ei, p.amh_go_p) / a.go_norm[r];
  }
  a.e_res[(size_t) E_AMHGO * s.n_res + r] = E;
}

template <typename R> __device__ __forceinline__ void amh_go_pass(const StepArgs<R> &a, const FFParams &p, Span sp)
{
  for (int r = sp.t; r < a.n_run; r += sp.nthr)
    if (a.res_sys[r] >= 0) amh_go_residue(a, p, r);
}

template <typename R> __global__ void k_amh_go(StepArgs<R> a, FFParams p) { amh_go_pass(a, p, grid_span()); }

__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

// Uniform in [0,1) keyed by (seed, step, atom id, component): the Langevin
// noise stream shared with the CPU oracle.
// the stream's key for (seed, step), and the uniform of (key, atom id, component)
__device__ __forceinline__ uint64_t uniform_key(uint64_t seed, long long step)
{
  return mix64(seed ^ mix64((uint64_t) step));
}
__device__ __forceinline__ double uniform01_k(uint64_t key, long long tag, int comp)
{
  uint64_t r = mix64(key ^ ((uint64_t) tag * 4ULL + (uint64_t) comp));
  return (double) (r >> 11) * (1.0 / 9007199254740992.0);
}
__device__ __forceinline__ double uniform01(uint64_t seed, long long step, long long tag, int comp)
{
  return uniform01_k(uniform_key(seed, step), tag, comp);
}

struct Integrator {
  double dt, dtf;           // dtf = 0.5 * dt * ftm2v
  int langevin;
  double damp;
  long long begin;          // first evaluated step of the current call (thermo row 0)
  long long stop;           // last step of the current call: its state stays at the full step (no drift after it)
};

// Total force (fixed point -> FP64, plus Langevin at `step`), then
// final_integrate of `step` (half kick) and, if `next`, initial_integrate of
// step+1 (half kick + drift) -- LAMMPS fix nve / fix langevin order.  Each
// replica follows its own run window (SlotRun); outside it the replica is
// frozen, and residues of no replica are skipped.
//
// Whether residue r is integrated at `step`, and its run-window values:
// the thermostat temperature's square root and the Langevin stream's key
// (the replica's own step count keys its noise).
template <typename R>
__device__ __forceinline__ bool finish_residue(const StepArgs<R> &a, const Integrator &in, long long step, int r,
                                               double *tsqrt, uint64_t *nkey)
{
  const int rep = a.res_sys[r];
  if (rep < 0) return false;
  const SlotRun sr = a.slot_run[rep];
  if (step < sr.begin || step > sr.end) return false;
  if (in.langevin) {
    // every multiply and add rounded on its own, as the x86-64 CPU build
    // computes fix langevin
    const double delta = sr.end != sr.begin ? (double) (step - sr.begin) / (double) (sr.end - sr.begin) : 0.0;
    *tsqrt = sqrt(__dadd_rn(sr.t_start, __dmul_rn(delta, __dsub_rn(sr.t_stop, sr.t_start))));
    *nkey = uniform_key(a.sys_seed[rep], step - sr.step0);
  } else {
    *tsqrt = 0.0;
    *nkey = 0ull;
  }
  return true;
}

// One component k = 3 b + c (bead b, axis c) of an integrated residue r,
// given its atom's dtfm = dtf / m and the residue's window values; writes
// its kinetic-energy term m v^2 (after the final half kick) to *ke.
template <typename R>
__device__ __forceinline__ void finish_comp(const StepArgs<R> &a, const Integrator &in, long long step,
                                            const double *g1, const double *g2, double *ftot, double *x_out, int r,
                                            int k, double dtfm, double tsqrt, uint64_t nkey, double *ke)
{
  const int rep = a.res_sys[r];
  const SlotRun sr = a.slot_run[rep];
  const bool final_kick = step > sr.begin, next = step < sr.end && step < in.stop;
  const size_t e = (size_t) 9 * r + k;  // element of the [atom][3] arrays
  if (a.lst_x0 && a.lst_build[rep]) a.lst_x0[e] = x_out[e];  // the emulated lists were built at these positions
  const int at = 3 * r + k / 3, c = k % 3;
  // Every multiply and add below is rounded on its own (no contraction), as
  // the x86-64 CPU build computes fix langevin / fix nve, and identically in
  // every kernel that inlines this.
  const double m = a.mass[at];
  double f = (double) (long long) a.s.facc[e] * F_UNSCALE;
  double v = a.v[e];
  if (in.langevin)
    f = __dadd_rn(f, __dadd_rn(__dmul_rn(g1[at], v),
                               __dmul_rn(__dmul_rn(g2[at], tsqrt), __dsub_rn(uniform01_k(nkey, a.atom_tag[at], c), 0.5))));
  if (ftot) ftot[e] = f;
  if (final_kick) v = __dadd_rn(v, __dmul_rn(dtfm, f));
  *ke = __dmul_rn(__dmul_rn(m, v), v);
  if (next) {
    v = __dadd_rn(v, __dmul_rn(dtfm, f));
    x_out[e] = __dadd_rn(x_out[e], __dmul_rn(in.dt, v));
  }
  a.v[e] = v;
}

// kinetic energy of a residue from its nine terms, summed in component order
__device__ __forceinline__ double kinetic(const double t[9])
{
  double ke = 0.0;
#pragma unroll
  for (int k = 0; k < 9; k++) ke = __dadd_rn(ke, t[k]);
  return 0.5 * 48.88821291 * 48.88821291 * ke;
}

// all nine components of residue r by one thread (the persistent step form)
template <typename R>
__device__ __forceinline__ void finish_one(const StepArgs<R> &a, const Integrator &in, long long step, const double *g1,
                                           const double *g2, double *ftot, double *x_out, int r)
{
  double tsqrt, t[9];
  uint64_t nkey;
  if (!finish_residue(a, in, step, r, &tsqrt, &nkey)) return;
  for (int k = 0; k < 9; k++)
    finish_comp(a, in, step, g1, g2, ftot, x_out, r, k, in.dtf / a.mass[3 * r + k / 3], tsqrt, nkey, &t[k]);
  a.e_res[(size_t) E_KIN * a.s.n_res + r] = kinetic(t);
}

template <typename R>
__device__ __forceinline__ void finish_pass(const StepArgs<R> &a, const Integrator *inp, const double *g1,
                                            const double *g2, double *ftot, double *x_out, Span sp)
{
  const Integrator in = *inp;
  const long long step = *a.step;
  for (int r = sp.t; r < a.n_run; r += sp.nthr) finish_one(a, in, step, g1, g2, ftot, x_out, r);
}

// The standalone kernel: one thread per component (nine per residue, 32
// residues per block), so that every array is read and written with
// consecutive threads on consecutive elements.  The values shared by a
// residue (its window, the noise key) and by an atom (dtf / m) are formed
// once into shared memory, by the same operations as finish_one forms them;
// the residue's kinetic energy is summed from shared memory in the order
// finish_one sums it.  Compiled for 4 blocks (36 warps) per SM.
constexpr int kFinishRes = 32, kFinishThreads = 9 * kFinishRes;
template <typename R>
__global__ void __launch_bounds__(kFinishThreads, 4) k_finish(StepArgs<R> a, const Integrator *inp, const double *g1,
                                                             const double *g2, double *ftot, double *x_out)
{
  __shared__ double kt[kFinishThreads], s_dtfm[3 * kFinishRes], s_tsqrt[kFinishRes];
  __shared__ unsigned long long s_key[kFinishRes];
  __shared__ int on[kFinishRes];
  const Integrator in = *inp;
  const long long step = *a.step;
  const int lr = threadIdx.x / 9, k = threadIdx.x - 9 * lr;
  for (int r0 = blockIdx.x * kFinishRes; r0 < a.n_run; r0 += gridDim.x * kFinishRes) {
    if (threadIdx.x < kFinishRes) {
      const int r = r0 + threadIdx.x;
      double tsqrt = 0.0;
      uint64_t nkey = 0ull;
      on[threadIdx.x] = r < a.n_run && finish_residue(a, in, step, r, &tsqrt, &nkey);
      s_tsqrt[threadIdx.x] = tsqrt;
      s_key[threadIdx.x] = nkey;
    } else if (threadIdx.x < 4 * kFinishRes) {
      const int at = 3 * r0 + (int) threadIdx.x - kFinishRes;
      s_dtfm[threadIdx.x - kFinishRes] = at < 3 * a.n_run ? in.dtf / a.mass[at] : 0.0;
    }
    __syncthreads();
    const int r = r0 + lr;
    double t = 0.0;
    if (on[lr]) finish_comp(a, in, step, g1, g2, ftot, x_out, r, k, s_dtfm[3 * lr + k / 3], s_tsqrt[lr], s_key[lr], &t);
    kt[threadIdx.x] = t;
    __syncthreads();
    if (threadIdx.x < kFinishRes && on[threadIdx.x])
      a.e_res[(size_t) E_KIN * a.s.n_res + r0 + threadIdx.x] = kinetic(kt + 9 * threadIdx.x);
    __syncthreads();
  }
}

// Continuation of a run that stopped at step `*a.step` before its window's
// end: the initial integration (half kick and drift) finish_one would have
// done there, from the total force it stored in ftot -- the same operations
// in the same order, so a run split into calls equals the run in one call.
template <typename R>
__global__ void k_continue(StepArgs<R> a, const Integrator *inp, const double *ftot, double *x_out)
{
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= a.n_run) return;
  const int rep = a.res_sys[r];
  if (rep < 0) return;
  const Integrator in = *inp;
  const SlotRun sr = a.slot_run[rep];
  const long long step = *a.step;
  if (step < sr.begin || step >= sr.end) return;
  for (int b = 0; b < 3; b++) {
    const int at = 3 * r + b;
    const double dtfm = in.dtf / a.mass[at];
    for (int c = 0; c < 3; c++) {
      const double v = __dadd_rn(a.v[3 * at + c], __dmul_rn(dtfm, ftot[3 * at + c]));
      x_out[3 * at + c] = __dadd_rn(x_out[3 * at + c], __dmul_rn(in.dt, v));
      a.v[3 * at + c] = v;
    }
  }
}

// Caller-order staging <-> internal order: out[a] = in[perm[a]] / out[perm[a]] = in[a]
__global__ void k_gather3(const double *in, const int *perm, int n, double *out)
{
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const int p = perm[a];
  for (int c = 0; c < 3; c++) out[3 * a + c] = in[3 * p + c];
}

__global__ void k_scatter3(const double *in, const int *perm, int n, double *out)
{
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const int p = perm[a];
  for (int c = 0; c < 3; c++) out[3 * p + c] = in[3 * a + c];
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
__global__ void k_thermo(const double *e_res, const long long *e_fix, int efix_slots, int n_res, const long long *step,
                         const Integrator *inp, const int *sys_begin, const int *sys_end, long long nrows, double *rows)
{
  const long long begin = inp->begin;
  const int rep = blockIdx.x;
  __shared__ double sh[4][256];
  double acc[4] = {0, 0, 0, 0};
  for (int r = sys_begin[rep] + threadIdx.x; r < sys_end[rep]; r += blockDim.x) {
    double fx = 0.0;
    for (int t = 1; t < E_FIX_TERMS; t++) fx += e_res[(size_t) t * n_res + r];
    long long fq = e_fix[r] + e_fix[(size_t) n_res + r] + e_fix[(size_t) 2 * n_res + r] + e_fix[(size_t) 3 * n_res + r];
    for (int k = 5; k < efix_slots; k++) fq += e_fix[(size_t) k * n_res + r];
    fx += (double) fq * F_UNSCALE;
    acc[0] += fx;
    acc[1] += e_res[(size_t) E_PAIR * n_res + r] + (double) e_fix[(size_t) 4 * n_res + r] * F_UNSCALE;
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

// Q order parameters (compute qwolynes / qonuchic; QDefinition): block i
// sums row i of the pair terms over j > i, in a fixed tree order; k_q_sum
// adds the rows in a fixed order and normalises.  x: the replica's atoms
// from its first (CA, O, CB per residue).
__global__ void k_q_rows(const double *x, int n, int kind, int sep, double sigma_exp, const double *mat,
                         double *partial)
{
  const int i = blockIdx.x;
  __shared__ double sh[256];
  double acc = 0.0;
  const double xi0 = x[9 * i], xi1 = x[9 * i + 1], xi2 = x[9 * i + 2];
  for (int j = i + 1 + threadIdx.x; j < n; j += blockDim.x) {
    const int d = j - i;
    const double m = mat[(size_t) i * n + j];
    const double dx = xi0 - x[9 * j], dy = xi1 - x[9 * j + 1], dz = xi2 - x[9 * j + 2];
    const double rsq = dx * dx + dy * dy + dz * dz;
    if (kind == 0) {
      if (d <= sep) continue;
      const double sg = pow(1.0 + d, sigma_exp), dr = sqrt(rsq) - m;
      acc += exp(-(dr * dr) / (2.0 * (sg * sg)));
    } else {
      if (d <= 3 || m < 0.0) continue;
      if (kind == 1) {
        if (rsq < m) acc += 1.0;
      } else {
        const double s2 = pow(1.0 + d, 2.0 * sigma_exp), dr = sqrt(rsq) - sqrt(m);
        acc += exp(-(dr * dr) / (2.0 * s2));
      }
    }
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[i] = sh[0];
}

__global__ void k_q_sum(const double *partial, int n, double qnorm, double *out)
{
  __shared__ double sh[256];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partial[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0] * qnorm;
}

// Per-term sums of each replica's residues in a fixed tree order
// (block (t, r) sums energy slot t of replica rep0 + r)
__global__ void k_energy_reduce(const double *e_res, const long long *e_fix, int efix_slots, int n_res,
                                const int *sys_begin, const int *sys_end, double *out, int rep0)
{
  const int t = blockIdx.x, rep = rep0 + blockIdx.y;
  __shared__ double sh[256];
  double acc = 0.0;
  // pair-summed energies are kept in fixed point (e_fix slots)
  int k = t == E_DSSP ? 0 : t == E_PAP ? 1 : t == E_FRAGMEM ? 2 : t == E_WATER ? 3 : t == E_PAIR ? 4
              : t == E_SSB ? 5 : t == E_DH ? 6 : t == E_CONT_REST ? 7 : -1;
  if (k >= efix_slots) k = -1;
  const long long *fx = k >= 0 ? e_fix + (size_t) k * n_res : nullptr;
  for (int r = sys_begin[rep] + threadIdx.x; r < sys_end[rep]; r += blockDim.x)
    acc += e_res[(size_t) t * n_res + r] + (fx ? (double) fx[r] * F_UNSCALE : 0.0);
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
