// Single-system AWSEM engine: device buffers, the per-step launch sequence,
// CUDA-graph capture of MD steps, and the C ABI of include/awsem_gpu.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "awsem_gpu.h"
#include "awsem_step.cuh"
#include "awsem_model.h"

namespace awsem {

static thread_local std::string g_last_error;

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// invalid device state detected after a call (AWSEM_ESTATE)
struct StateError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

#define CK(call)                                                                                 \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      throw CudaError(std::string(#call) + ": " + cudaGetErrorString(e_) + " (" __FILE__ ":" + \
                      std::to_string(__LINE__) + ")");                                           \
  } while (0)

template <typename T> struct DBuf {
  T *p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
  ~DBuf() { release(); }
  void release()
  {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count)
  {
    release();
    n = count;
    if (count) CK(cudaMalloc(&p, count * sizeof(T)));
  }
  void upload(const std::vector<T> &h, cudaStream_t s)
  {
    alloc(std::max<size_t>(h.size(), 1));
    if (!h.empty()) CK(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void zero(cudaStream_t s)
  {
    if (n) CK(cudaMemsetAsync(p, 0, n * sizeof(T), s));
  }
};

constexpr double FTM2V = 1.0 / 48.88821291 / 48.88821291;
constexpr double MVV2E = 48.88821291 * 48.88821291;
constexpr double BOLTZ = 0.0019872067;

class EngineBase {
 public:
  virtual ~EngineBase() {}
  std::vector<std::unique_ptr<SystemInput>> reps;  // replicas as loaded (until commit)
  std::vector<unsigned long long> seeds;           // per-replica Langevin seed (0: the run's seed)
  Batch in;                                        // the committed batch
  bool committed = false;
  int device = 0;
  long long step = 0;
  int n_sys() const { return in.n_sys; }
  // atoms are 3 per residue in internal order: a replica's atoms follow its residues
  int rep_atom0(int r) const { return 3 * in.sys_res_begin[r]; }
  int rep_atoms(int r) const { return 3 * (in.sys_res_end[r] - in.sys_res_begin[r]); }
  int rep_res(int r) const { return in.sys_res_end[r] - in.sys_res_begin[r]; }
  void commit()
  {
    std::vector<const SystemInput *> v;
    for (auto &p : reps) v.push_back(p.get());
    assemble_batch(v, in);
    seeds.resize(in.n_sys, 0ull);
    setup();
    committed = true;
    reps.clear();  // host copies are no longer needed: state lives on the device
  }
  virtual void setup() = 0;
  virtual void compute(long long step, const double *x_ext, double *f_ext, double *energies, int groups) = 0;
  virtual void set_state(int rep, const double *x_ext, const double *v_ext) = 0;
  virtual void get_state(int rep, double *x_ext, double *v_ext) = 0;
  // every replica at once, replicas concatenated in replica order, each in its caller atom order
  virtual void set_state_all(const double *x_ext, const double *v_ext) = 0;
  virtual void get_state_all(double *x_ext, double *v_ext) = 0;
  virtual void run(long long nsteps, const awsem_run_params &rp, double *thermo) = 0;
  virtual void run_window(long long nsteps, const awsem_run_params &rp, long long wbegin, long long wend, bool cont,
                          double *thermo) = 0;
  virtual void energies(int rep, double *out) = 0;
  virtual void forces(int rep, double *f_ext) = 0;
  virtual void residue_arrays(int rep, double *out) = 0;
  virtual long long debug_selections(long long step, const double *x_ext, unsigned long long *keys, long long cap) = 0;
  virtual void nl_stats(int *nbuilds, double *radius, int *maxc, int *overflow) = 0;
  virtual void profile(int reps, double *ms) = 0;
  virtual void autotune(int reps, int *chosen) = 0;
  virtual void set_step_form(int form, int blocks, int stream_warps) = 0;
  virtual void set_launch_shapes(const int *shapes) = 0;
  virtual void set_neighbor(double skin, int delay, int every, int check) = 0;
  virtual void set_list_built(int built) = 0;
  virtual void set_wait_limits(long long fm_cycles, long long barrier_cycles, int hold) = 0;
  virtual int q_create(int rep, const std::string &words) = 0;
  virtual double q_value(int qid) = 0;
  virtual void get_step_form(int *out) = 0;
  virtual void model_info(long long *info) = 0;
  virtual double run_ms() const = 0;
  // device-resident fragment-memory table, for entry points outside the engine
  virtual FMView fm_view() const = 0;
  // serving handles (fixed capacity, requests admitted and released)
  bool server = false;
  virtual void server_setup(const SharedForceField &f, long long cap_res, int max_slots, long long cap_records,
                            double dt, double damp) = 0;
  virtual int admit(const ReplicaArrays &ra, unsigned long long seed, long long nsteps, double t_start,
                    double t_stop) = 0;  // slot, or -1 when the request does not fit now
  // admit in two parts: the host-side preparation (topology, memory table
  // slices; touches no device state and may run on another thread while
  // advance runs), then the placement and uploads
  virtual void *prepare_request(const ReplicaArrays &ra) = 0;
  virtual int admit_prepared(void *prep, unsigned long long seed, long long nsteps, double t_start,
                             double t_stop) = 0;
  using PreparedDeleter = void (*)(void *);
  virtual PreparedDeleter prepared_deleter() const = 0;
  virtual void progress(int slot, long long *done, long long *total) = 0;
  virtual void advance(long long nsteps) = 0;
  virtual void release(int slot) = 0;
  virtual void usage(long long *info) = 0;
};

void fragmem_noalloc(int device, const FMView &v, const double *d_x, double *d_f, double *d_energy,
                     cudaStream_t stream);  // awsem_noalloc.cu

static const char *kKernelNames[AWSEM_NKERNELS] = {"prepare", "nl_decide", "nl_build", "density",
                                                   "residue", "backbone",  "water_xi", "radial",
                                                   "pair",    "hbond",     "fragmem",  "finish"};
// the same kernels by index
enum KernelIndex {
  K_PREPARE, K_NL_DECIDE, K_NL_BUILD, K_DENSITY, K_RESIDUE, K_BACKBONE, K_WATER_XI, K_RADIAL, K_PAIR, K_HBOND,
  K_FRAGMEM, K_FINISH
};
static_assert(K_FINISH + 1 == AWSEM_NKERNELS, "kernel index table");

template <typename R> class Engine : public EngineBase {

 public:
  cudaStream_t s0 = nullptr, s1 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaStream_t s2 = nullptr;  // the detection pass and the hydrogen-bond terms
  cudaEvent_t ev_dens = nullptr, ev_join2 = nullptr;
  DBuf<int> res_type, res_flags, res_chain, chain_start, chain_end, atom_tag, atom_type;
  DBuf<double> aps, tables, x, v, mass, g1, g2, ftot, work, e_res, energy;
  DBuf<double4> pos, cpos, cb_build;
  DBuf<dev::RadRec> rrec;
  DBuf<unsigned long long> facc;
  DBuf<int2> pairs, cpairs;  // residue pair list; the near list of an evaluation
  DBuf<int> seg_n;           // near pairs per near-list segment
  DBuf<int> ncount, hbq;
  DBuf<long long> dacc;
  int pair_blocks = 1;
  DBuf<long long> e_fix;
  int hb_blocks = 1;
  DBuf<dev::NLState> nl;
  DBuf<long long> dstep;
  DBuf<double> ev_pref, ev_cs, ev_cl;
  DBuf<unsigned> excl_self, excl_next;
  DBuf<int> bond_i, bond_j;
  DBuf<double> bond_k, bond_r0;
  int bond_cap = 1;
  DBuf<int> fm_soff, fm_slen;
  DBuf<R> fm_rf, fm_coef;
  DBuf<double> tb_data;            // table fragment memory (energy, force pairs)
  DBuf<unsigned char> tb_present;
  DBuf<int> go_start, go_partner;  // AMH-Go native contacts
  DBuf<double> go_rnat, go_gamma, go_sig_sq, go_norm;
  DBuf<unsigned char> go_in;       // AMH-Go contacts in the emulated full list
  DBuf<double> lst_x0;             // emulated LAMMPS lists: positions at the last build
  DBuf<int> lst_ago, lst_over, lst_build;  // per replica: steps since the build, half-skin flag, built now
  DBuf<double> charge;             // Debye-Hueckel charges
  DBuf<int> cr_start, cr_j;        // contact restraints
  DBuf<double> cr_w, cr_r0;
  DBuf<int> zim;                   // membrane zones
  DBuf<int> vfm_start, vfm_j;      // vector fragment memory records
  DBuf<double> vfm_angle;
  int efix_slots = 5;
  int fm_groups = 0, fm_dsplit = 1;
  DBuf<double> thermo_rows;
  DBuf<int> res_sys, sys_begin, sys_end;
  DBuf<unsigned long long> sys_seed;
  int pcap = 0;  // residue pair list capacity (pairs)
  int sms_ = 148;  // multiprocessors of the device
  bool server_pending = false;  // setup() called for a serving handle (no replicas yet)
  // residues the per-residue kernels cover: all of them, or on a serving
  // handle the used prefix of its capacity (rounded up to 4,096)
  int launch_res = 0;
  int n_run() const { return launch_res > 0 ? launch_res : n(); }
  // pair-list room per residue: 48 covers a compact globule (about 66
  // partners within 16 A, half of them higher-numbered) with margin
  int pairs_per_res = 48;
  int prio_lo = 0, prio_hi = 0;  // stream priority range (prio_hi: highest)
  int groups_all = dev::G_FIX | dev::G_PAIR | dev::G_BOND;
  double skin = 2.0;
  int neigh_every = 0;
  std::vector<double> hx, hv;  // host staging (internal order)

  ~Engine() override
  {
    release_graphs();
    if (ev_run0) cudaEventDestroy(ev_run0);
    if (ev_run1) cudaEventDestroy(ev_run1);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (ev_dens) cudaEventDestroy(ev_dens);
    if (ev_join2) cudaEventDestroy(ev_join2);
    if (s0) cudaStreamDestroy(s0);
    if (s1) cudaStreamDestroy(s1);
    if (s2) cudaStreamDestroy(s2);
  }

  int n() const { return in.top.n_res; }
  int natoms() const { return in.top.n_atoms; }

  dev::StepArgs<R> args(int groups)
  {
    dev::StepArgs<R> a{};
    a.s.n_res = n();
    a.n_run = n_run();
    a.s.res_type = res_type.p;
    a.s.res_flags = res_flags.p;
    a.s.res_chain = res_chain.p;
    a.s.chain_start = chain_start.p;
    a.s.chain_end = chain_end.p;
    a.s.aps = aps.p;
    a.s.tables = tables.p;
    a.s.pos = pos.p;
    a.s.cpos = cpos.p;
    a.s.facc = facc.p;
    a.n_atoms = natoms();
    a.x = x.p;
    a.v = v.p;
    a.mass = mass.p;
    a.atom_tag = atom_tag.p;
    double *w = work.p;
    size_t nn = (size_t) n();
    a.rho_w = w;
    a.rho_h = w + nn;
    a.sig_w = w + 2 * nn;
    a.sigp_w = w + 3 * nn;
    a.sig_h = w + 4 * nn;
    a.sigp_h = w + 5 * nn;
    a.xi_w = w + 6 * nn;
    a.xi1 = w + 7 * nn;
    a.xi2 = w + 8 * nn;
    a.bur = w + 9 * nn;
    a.rrec = rrec.p;
    a.e_res = e_res.p;
    a.pairs = pairs.p;
    a.cpairs = cpairs.p;
    a.seg_n = seg_n.p;
    a.dacc = dacc.p;
    a.hbq = hbq.p;
    a.e_fix = e_fix.p;
    a.ncount = ncount.p;
    a.pcap = pcap;
    a.cb_build = cb_build.p;
    a.nl = nl.p;
    a.ntypes = in.top.ntypes;
    a.ev_p = in.top.ev_p;
    a.ev_pref = ev_pref.p;
    a.ev_cs = ev_cs.p;
    a.ev_cl = ev_cl.p;
    a.atom_type = atom_type.p;
    a.excl_self = excl_self.p;
    a.excl_next = excl_next.p;
    a.bond_cap = bond_cap;
    a.bond_i = bond_i.p;
    a.bond_j = bond_j.p;
    a.bond_k = bond_k.p;
    a.bond_r0 = bond_r0.p;
    a.fm.soff = fm_soff.p;
    a.fm.slen = fm_slen.p;
    a.fm.rf = fm_rf.p;
    a.fm.coef = in.fm.uniform ? nullptr : fm_coef.p;
    a.fm.uniform = in.fm.uniform_coef;
    a.fm.nd = in.ff.p.fm_nd;
    a.fm.min_sep = in.ff.p.fm_min_sep;
    // residue groups the fragment-memory kernel walks: those of the launch
    // extent (on a serving handle the used prefix, not the whole capacity)
    a.fm.groups = std::min(fm_groups, (n_run() + 31) / 32);
    a.fm.dsplit = fm_dsplit;
    a.fm.wait_limit = fm_wait_limit;
    a.fm.hold_tx = (hold_waits & 1) ? 16u : 0u;
    a.tb_data = reinterpret_cast<const double2 *>(tb_data.p);
    a.tb_present = tb_present.p;
    a.go_start = go_start.p;
    a.go_partner = go_partner.p;
    a.go_rnat = go_rnat.p;
    a.go_gamma = go_gamma.p;
    a.go_sig_sq = go_sig_sq.p;
    a.go_norm = go_norm.p;
    const bool lst_on = lists_emulated();
    a.go_in = go_in.p;
    a.lst_x0 = lst_on ? lst_x0.p : nullptr;
    a.lst_ago = lst_on ? lst_ago.p : nullptr;
    a.lst_over = lst_on ? lst_over.p : nullptr;
    a.lst_build = lst_on ? lst_build.p : nullptr;
    a.charge = charge.p;
    a.cr_start = cr_start.p;
    a.cr_j = cr_j.p;
    a.cr_w = cr_w.p;
    a.cr_r0 = cr_r0.p;
    a.efix_slots = efix_slots;
    a.zim = zim.p;
    a.vfm_start = vfm_start.p;
    a.vfm_j = vfm_j.p;
    a.vfm_angle = vfm_angle.p;
    a.groups = groups;
    a.step = dstep.p;
    a.res_sys = res_sys.p;
    a.sys_begin = sys_begin.p;
    a.sys_end = sys_end.p;
    a.sys_seed = sys_seed.p;
    a.slot_run = slot_run.p;
    a.sel = sel_cap > 0 ? sel_keys.p : nullptr;
    a.sel_n = sel_count.p;
    a.sel_cap = sel_cap;
    return a;
  }

  // selection records of one evaluation (awsem_debug_selections)
  DBuf<unsigned long long> sel_keys, sel_count;
  long long sel_cap = 0;

  long long debug_selections(long long st, const double *x_ext, unsigned long long *keys, long long cap) override
  {
    need_single("awsem_debug_selections");
    if (cap < 0) throw std::invalid_argument("negative selection capacity");
    sel_keys.alloc((size_t) std::max<long long>(cap, 1));
    sel_count.alloc(1);
    sel_count.zero(s0);
    std::vector<double> f((size_t) 3 * natoms(), 0.0);
    sel_cap = std::max<long long>(cap, 1);
    try {
      compute(st, x_ext, f.data(), nullptr, groups_all);
    } catch (...) {
      sel_cap = 0;
      throw;
    }
    sel_cap = 0;
    unsigned long long got = 0;
    CK(cudaMemcpy(&got, sel_count.p, sizeof got, cudaMemcpyDeviceToHost));
    const long long keep = std::min<long long>((long long) got, cap);
    if (keep > 0) CK(cudaMemcpy(keys, sel_keys.p, sizeof(unsigned long long) * keep, cudaMemcpyDeviceToHost));
    sel_keys.release();
    sel_count.release();
    return (long long) got;
  }

  void setup() override
  {
    CK(cudaSetDevice(device));
    // the pair-pass chain (s0) is the critical path: it gets the higher
    // priority, so the block scheduler serves it first and the bandwidth-bound
    // fragment-memory kernel (s1) fills the remaining room
    CK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    CK(cudaStreamCreateWithPriority(&s0, cudaStreamNonBlocking, prio_hi));
    CK(cudaStreamCreateWithPriority(&s1, cudaStreamNonBlocking, prio_lo));
    CK(cudaStreamCreateWithPriority(&s2, cudaStreamNonBlocking, prio_hi));
    CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ev_dens, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ev_join2, cudaEventDisableTiming));
    const Topology &t = in.top;
    int nn = n(), na = natoms();
    res_sys.upload(in.res_sys, s0);
    sys_begin.upload(in.sys_res_begin, s0);
    sys_end.upload(in.sys_res_end, s0);
    sys_seed.alloc(std::max(in.n_sys, 1));
    slot_run.alloc(std::max(in.n_sys, 1));
    slot_run.zero(s0);
    energy.alloc((size_t) E_SLOTS * std::max(in.n_sys, 1));
    res_type.upload(t.res_type, s0);
    res_flags.upload(t.res_flags, s0);
    res_chain.upload(t.res_chain, s0);
    chain_start.upload(t.chain_start, s0);
    chain_end.upload(t.chain_end, s0);
    atom_tag.upload(t.atom_tag, s0);
    atom_type.upload(t.atom_type, s0);
    aps.upload(t.aps, s0);
    tables.upload(in.ff.tables, s0);
    x.upload(in.x, s0);
    v.upload(in.v, s0);
    mass.upload(t.mass, s0);
    g1.alloc(na);
    g2.alloc(na);
    ftot.alloc((size_t) 3 * na);
    ftot.zero(s0);
    work.alloc((size_t) 10 * nn);
    work.zero(s0);
    e_res.alloc((size_t) E_SLOTS * nn);
    e_res.zero(s0);
    pos.alloc((size_t) dev::N_BEADS * nn);
    cpos.alloc((size_t) nn);
    rrec.alloc((size_t) nn);
    pos.zero(s0);  // residues of no replica keep finite (zero) working positions
    cb_build.alloc(nn);
    cb_build.zero(s0);
    facc.alloc((size_t) 3 * na);
    facc.zero(s0);
    ncount.alloc(nn);
    ncount.zero(s0);
    nl.alloc(1);
    dstep.alloc(1);
    ev_pref.upload(t.ev_pref, s0);
    ev_cs.upload(t.ev_cs, s0);
    ev_cl.upload(t.ev_cl, s0);
    excl_self.upload(t.excl_self, s0);
    excl_next.upload(t.excl_next, s0);
    // bonds in fixed slots per residue of their first atom, in input order
    std::vector<int> cnt(nn, 0);
    for (size_t b = 0; b < t.bond_i.size(); b++) cnt[t.bond_i[b] / 3]++;
    bond_cap = std::max(1, nn ? *std::max_element(cnt.begin(), cnt.end()) : 1);
    std::vector<int> bi((size_t) nn * bond_cap, -1), bj((size_t) nn * bond_cap, -1);
    std::vector<double> bk((size_t) nn * bond_cap, 0.0), br((size_t) nn * bond_cap, 0.0);
    std::fill(cnt.begin(), cnt.end(), 0);
    for (size_t b = 0; b < t.bond_i.size(); b++) {
      int r = t.bond_i[b] / 3;
      size_t at = (size_t) r * bond_cap + cnt[r]++;
      bi[at] = t.bond_i[b];
      bj[at] = t.bond_j[b];
      bk[at] = t.bond_k[b];
      br[at] = t.bond_r0[b];
    }
    bond_i.upload(bi, s0);
    bond_j.upload(bj, s0);
    bond_k.upload(bk, s0);
    bond_r0.upload(br, s0);
    if (!(in.ff.p.terms & T_FM)) in.ff.p.fm_nd = 0;
    upload_fm_slices();
    if (in.ff.p.terms & T_FM_TABLE) {
      tb_data.upload(in.tb.data, s0);
      std::vector<unsigned char> pr(in.tb.present.begin(), in.tb.present.end());
      tb_present.upload(pr, s0);
      CK(cudaStreamSynchronize(s0));
      std::vector<double>().swap(in.tb.data);  // the device holds the tables now
    }
    if (in.ff.p.terms & T_AMHGO) {
      go_start.upload(in.go.start, s0);
      go_partner.upload(in.go.partner.empty() ? std::vector<int>{0} : in.go.partner, s0);
      go_rnat.upload(in.go.rnat.empty() ? std::vector<double>{0.0} : in.go.rnat, s0);
      go_gamma.upload(in.go.gamma.empty() ? std::vector<double>{0.0} : in.go.gamma, s0);
      go_sig_sq.upload(in.go.sig_sq.empty() ? std::vector<double>{1.0} : in.go.sig_sq, s0);
      go_norm.upload(in.go.norm, s0);
      go_in.alloc(std::max<size_t>(in.go.partner.size(), 1));
      go_in.zero(s0);
    }
    if (lists_emulated()) {
      lst_x0.alloc((size_t) 9 * nn);
      lst_x0.zero(s0);
      for (DBuf<int> *b : {&lst_ago, &lst_over, &lst_build}) {
        b->alloc((size_t) std::max(n_sys(), 1));
        b->zero(s0);
      }
    }
    if (in.ff.p.terms & T_DH) {
      std::vector<double> q(in.charge);
      q.resize((size_t) nn, 0.0);
      charge.upload(q, s0);
    }
    if (in.ff.p.terms & T_CONTREST) {
      std::vector<int> st(in.cr.start);
      st.resize((size_t) nn + 1, st.empty() ? 0 : st.back());
      cr_start.upload(st, s0);
      cr_j.upload(in.cr.j.empty() ? std::vector<int>{0} : in.cr.j, s0);
      cr_w.upload(in.cr.w.empty() ? std::vector<double>{0.0} : in.cr.w, s0);
      cr_r0.upload(in.cr.r0.empty() ? std::vector<double>{0.0} : in.cr.r0, s0);
    }
    efix_slots = (in.ff.p.terms & (T_SSB | T_DH | T_CONTREST)) ? 8 : 5;
    if (in.ff.p.terms & T_VFM) {
      std::vector<int> st(in.vfm.start);
      st.resize((size_t) nn + 1, st.empty() ? 0 : st.back());
      vfm_start.upload(st, s0);
      vfm_j.upload(in.vfm.j.empty() ? std::vector<int>{0} : in.vfm.j, s0);
      vfm_angle.upload(in.vfm.angle.empty() ? std::vector<double>{0.0} : in.vfm.angle, s0);
    }
    if (in.ff.p.terms & T_MEMB) {
      std::vector<int> z(in.zim);
      z.resize((size_t) nn, 1);
      zim.upload(z, s0);
    }
    CK(cudaFuncSetAttribute(dev::k_fragmem<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            4 * dev::fm_warp_smem<R>(true)));
    // pair-list radii of the terms
    dev::NLState st{};
    const FFParams &p = in.ff.p;
    float rc = 0.f;
    for (int w = 0; w < p.n_wells; w++) rc = std::max(rc, (float) p.w_rmax_th[w]);
    if (p.terms & T_HELIX) rc = std::max(rc, (float) p.h_rmax_th);
    if (p.terms & T_CONTREST) rc = std::max(rc, (float) sqrt(p.cr_cut_sq) * 1.0001f);
    st.r_contact = rc;
    st.r_dssp = (p.terms & T_DSSP) ? (float) p.dssp_cut : 0.f;
    st.r_pap = (p.terms & T_PAP) ? (float) sqrt(p.pap_cutoff_sq) : 0.f;
    double evmax = 0.0;
    int N = t.ntypes + 1;
    for (int a = 1; a <= t.ntypes; a++)
      for (int b = 1; b <= t.ntypes; b++)
        if (t.ev_pref[a * N + b] != 0.0) evmax = std::max(evmax, std::max(t.ev_cl[a * N + b], t.ev_cs[a * N + b]));
    st.r_ev = (float) evmax;
    // excluded-volume cutoffs by bead kind (CA, CB, O): over the atom types
    // found at each position, or (serving handles, whose requests bring
    // their own types) over every type
    {
      std::vector<std::vector<char>> at_pos(3, std::vector<char>(N, server ? 1 : 0));
      if (!server)
        for (size_t k = 0; k < t.atom_type.size(); k++) {
          const int ty = t.atom_type[k];
          if (ty >= 0 && ty < N) at_pos[k % 3][ty] = 1;
        }
      for (int b0 = 0; b0 < 3; b0++)
        for (int b1 = 0; b1 < 3; b1++) {
          double cs = 0.0, cl = 0.0;
          for (int a = 1; a < N; a++)
            for (int b = 1; b < N; b++)
              if (at_pos[b0][a] && at_pos[b1][b] && t.ev_pref[a * N + b] != 0.0) {
                cs = std::max(cs, t.ev_cs[a * N + b]);
                cl = std::max(cl, t.ev_cl[a * N + b]);
              }
          // rounded up so that the float bound never falls below the cutoff
          st.ev_cutk[0][b0][b1] = cs > 0.0 ? std::nextafter((float) cs, 1e30f) : 0.f;
          st.ev_cutk[1][b0][b1] = cl > 0.0 ? std::nextafter((float) cl, 1e30f) : 0.f;
        }
    }
    st.skin = (float) skin;
    // LAMMPS defaults: neigh_modify delay 0 every 1 check yes
    st.lst_skin = skin;
    st.lst_delay = 0;
    st.lst_every = 1;
    st.lst_check = 1;
    st.lst_force = 1;
    st.lst_pair_cut = pair_cut_now();
    CK(cudaMemcpyAsync(nl.p, &st, sizeof st, cudaMemcpyHostToDevice, s0));
    long long s = step;
    CK(cudaMemcpyAsync(dstep.p, &s, sizeof s, cudaMemcpyHostToDevice, s0));
    e_fix.alloc((size_t) efix_slots * nn);
    e_fix.zero(s0);
    dacc.alloc((size_t) 3 * nn);
    dacc.zero(s0);
    int sms = 148;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    sms_ = sms;
    hb_blocks = std::max(1, std::min((nn * 8 + 127) / 128, 16 * sms));
    if (!server_pending) setup_grids();
    // size the pair list from a first build: room for 4x the initial pairs
    // (chains that collapse gain neighbours), at least pairs_per_res per residue
    resize_pairs(std::max<long long>(64, 16LL * nn));
    for (int attempt = 0; attempt < 8; attempt++) {
      launch_prepare_and_list(args(groups_all), s0, true, false);
      dev::NLState got;
      CK(cudaMemcpyAsync(&got, nl.p, sizeof got, cudaMemcpyDeviceToHost, s0));
      CK(cudaStreamSynchronize(s0));
      if (!got.overflow) {
        long long want = std::max(4LL * got.npairs, (long long) pairs_per_res * nn) + 1024;
        long long expect = std::max(3LL * got.npairs / 2, 12LL * nn);
        pair_blocks = (int) std::max(1LL, std::min<long long>((expect + 127) / 128, 16LL * sms));
        if (want > pcap) {
          resize_pairs(want);
          continue;
        }
        break;
      }
      resize_pairs(std::max<long long>(2LL * pcap, 2LL * got.overflow));
    }
  }

  int max_count()
  {
    std::vector<int> c(n());
    CK(cudaMemcpyAsync(c.data(), ncount.p, sizeof(int) * n(), cudaMemcpyDeviceToHost, s0));
    CK(cudaStreamSynchronize(s0));
    return c.empty() ? 0 : *std::max_element(c.begin(), c.end());
  }

  void resize_pairs(long long newcap)
  {
    // pair indices (and their complements in the DSSP queue) are ints
    if (newcap >= (1ll << 31)) throw std::invalid_argument("residue pair list exceeds 2^31 pairs");
    pcap = (int) newcap;
    pairs.alloc((size_t) pcap);
    cpairs.alloc((size_t) pcap);
    seg_n.alloc((size_t) pcap / 32 + 2);
    hbq.alloc((size_t) 3 * pcap);
    dev::NLState st;
    CK(cudaMemcpyAsync(&st, nl.p, sizeof st, cudaMemcpyDeviceToHost, s0));
    CK(cudaStreamSynchronize(s0));
    st.overflow = 0;
    st.r_list = 0.f;  // forces a rebuild
    CK(cudaMemcpyAsync(nl.p, &st, sizeof st, cudaMemcpyHostToDevice, s0));
  }

  // cell grids of the large replicas (see k_grid_setup)
  DBuf<int> big_rep, big_of, cell_count, cell_start, cell_fill, res_cell, sorted_res;
  DBuf<dev::GridDesc> grid_desc;
  int nbig = 0;

  void setup_grids()
  {
    std::vector<int> br, bo(std::max(n_sys(), 1), -1);
    std::vector<dev::GridDesc> gd;
    int cells = 0;
    for (int r = 0; r < n_sys(); r++) {
      const int nr = rep_res(r);
      if (nr <= dev::kGridMin) continue;
      bo[r] = (int) br.size();
      br.push_back(r);
      dev::GridDesc d{};
      d.cell0 = cells;
      d.cap = std::max(64, 2 * nr);
      cells += d.cap;
      gd.push_back(d);
    }
    nbig = (int) br.size();
    if (!nbig) return;
    big_rep.upload(br, s0);
    big_of.upload(bo, s0);
    grid_desc.upload(gd, s0);
    cell_count.alloc(cells);
    cell_start.alloc(cells);
    cell_fill.alloc(cells);
    res_cell.alloc(n());
    sorted_res.alloc(n());
    CK(cudaStreamSynchronize(s0));
  }

  dev::GridArgs grid_args() const
  {
    return dev::GridArgs{nbig, big_rep.p, big_of.p, grid_desc.p, cell_count.p, cell_start.p, cell_fill.p,
                         res_cell.p, sorted_res.p};
  }

  void launch_list_build(const dev::StepArgs<R> &a, cudaStream_t s)
  {
    const int nn = n_run(), tb = 128, nb = (nn + tb - 1) / tb;
    const int wb = std::min((nn * 32 + tb - 1) / tb, 8 * sms_);
    const dev::GridArgs g = grid_args();
    if (nbig) {
      dev::k_grid_setup<R><<<nbig, 256, 0, s>>>(a, g);
      dev::k_grid_count<R><<<nb, tb, 0, s>>>(a, g);
      dev::k_grid_scan<R><<<nbig, 1024, 0, s>>>(a, g);
      dev::k_grid_fill<R><<<nb, tb, 0, s>>>(a, g);
    }
    dev::k_nl_build<R><<<wb, tb, 0, s>>>(a, g, nn);
  }

  void launch_prepare_and_list(const dev::StepArgs<R> &a, cudaStream_t s, bool force, bool advance)
  {
    const FFParams &p = in.ff.p;
    const int nn = n_run(), tb = 128, nb = (nn + tb - 1) / tb;
    dev::k_prepare<R><<<nb, tb, 0, s>>>(a, p);
    dev::k_nl_decide<<<1, 1, 0, s>>>(nl.p, force ? 1 : 0, advance ? dstep.p : nullptr);
    launch_list_build(a, s);
  }

  // one force evaluation (everything up to the fixed-point force sums)
  void launch_eval(const dev::StepArgs<R> &a, bool advance)
  {
    const FFParams &p = in.ff.p;
    int nn = n_run();
    int tb = 128, nb = (nn + tb - 1) / tb;
    launch_prepare_and_list(a, s0, false, advance);
    bool fm = (a.groups & dev::G_FIX) && p.fm_nd > 0;
    const bool fmt = (a.groups & dev::G_FIX) && (p.terms & T_FM_TABLE);
    const bool go = (a.groups & dev::G_FIX) && (p.terms & T_AMHGO);
    const bool px = (a.groups & dev::G_FIX) && (p.terms & (T_SSB | T_DH | T_CONTREST));
    const bool rx = (a.groups & dev::G_FIX) && (p.terms & (T_SHAKE | T_MEMB | T_VFM));
    // the emulated lists' decision for this step, before anything reads it
    if (lists_emulated())
      dev::k_list_decide<<<(n_sys() + 127) / 128, 128, 0, s0>>>(nl.p, n_sys(), lst_ago.p, lst_over.p, lst_build.p);
    // the backbone terms (chain, chi, rama; one kernel of the residue pass)
    // need only the positions; the recording pass of awsem_debug_selections
    // runs the whole residue pass instead
    const bool bb = !a.sel;
    if (fm || fmt || go || px || rx) {
      // fragment memory and the optional terms are independent of the pair
      // passes: second stream
      CK(cudaEventRecord(ev_fork, s0));
      CK(cudaStreamWaitEvent(s1, ev_fork, 0));
      if (fm) dev::k_fragmem<R><<<fm_blocks(), tb, fm_smem(), s1>>>(a, p);
      if (fmt) dev::k_fm_table<R><<<fm_table_blocks(), tb, 0, s1>>>(a, p);
      if (go) dev::k_amh_go<R><<<nb, tb, 0, s1>>>(a, p);
      if (px) dev::k_pair_extra<R><<<pair_blocks, tb, 0, s1>>>(a, p);
      if (rx) dev::k_residue_extra<R><<<nb, tb, 0, s1>>>(a, p);
      CK(cudaEventRecord(ev_join, s1));
    }
    if (a.sel) {  // awsem_debug_selections: the same passes, recording their selections
      dev::k_density_sel<R><<<pair_blocks, tb, 0, s0>>>(a, p);
      dev::k_residue_sel<R><<<nb, tb, 0, s0>>>(a, p);
      dev::k_water_xi_sel<R><<<pair_blocks, tb, 0, s0>>>(a, p);
      dev::k_radial_sel<R><<<pair_blocks, tb, 0, s0>>>(a, p);
      dev::k_pair_sel<R><<<pair_blocks, tb, 0, s0>>>(a, p);
      dev::k_hbond_sel<R><<<hb_blocks, 128, 0, s0>>>(a, p);
    } else {
      // the backbone terms need only the positions, detection, excluded
      // volume and the hydrogen-bond terms the positions and the near list:
      // a third stream, beside fragment memory (second) and the
      // density-dependent passes (first)
      CK(cudaEventRecord(ev_fork, s0));
      CK(cudaStreamWaitEvent(s2, ev_fork, 0));
      if (bb) dev::k_backbone<R><<<nb, tb, 0, s2>>>(a, p);
      dev::k_density<R><<<pair_blocks, tb, 0, s0>>>(a, p);
      CK(cudaEventRecord(ev_dens, s0));
      CK(cudaStreamWaitEvent(s2, ev_dens, 0));
      dev::k_pair<R><<<pair_blocks, tb, 0, s2>>>(a, p);
      dev::k_hbond<R><<<hb_blocks, 128, 0, s2>>>(a, p);
      CK(cudaEventRecord(ev_join2, s2));
      dev::k_residue<R><<<nb, tb, 0, s0>>>(a, p);
      dev::k_water_xi<R><<<pair_blocks, tb, 0, s0>>>(a, p);
      dev::k_radial<R><<<pair_blocks, tb, 0, s0>>>(a, p);
      CK(cudaStreamWaitEvent(s0, ev_join2, 0));
    }
    if (fm || fmt || go || px || rx) CK(cudaStreamWaitEvent(s0, ev_join, 0));
  }

  int finish_blocks() const { return (n_run() + dev::kFinishRes - 1) / dev::kFinishRes; }

  int fm_table_blocks() const
  {
    const long long items = (long long) n_run() * std::max(in.ff.p.tb_nbrs, 1);
    return (int) std::min<long long>((items + 127) / 128, 64LL * sms_);
  }

  void zero_unwritten_energies(int groups)
  {
    // slots the selected groups do not write must read as zero
    int nn = n();
    if (!(groups & dev::G_FIX) || !(in.ff.p.terms & T_FM) || in.ff.p.fm_nd == 0)
      CK(cudaMemsetAsync(e_res.p + (size_t) E_FRAGMEM * nn, 0, sizeof(double) * nn, s0));
    if (!(groups & dev::G_BOND)) CK(cudaMemsetAsync(e_res.p + (size_t) E_BOND * nn, 0, sizeof(double) * nn, s0));
    if (!(groups & dev::G_FIX) || !(in.ff.p.terms & T_AMHGO))
      CK(cudaMemsetAsync(e_res.p + (size_t) E_AMHGO * nn, 0, sizeof(double) * nn, s0));
    if (!(groups & dev::G_FIX))
      for (int t : {E_SHAKE, E_MEMB, E_VFRAGMEM}) CK(cudaMemsetAsync(e_res.p + (size_t) t * nn, 0, sizeof(double) * nn, s0));
  }

  // energy sums of replicas [rep0, rep0 + count) (all of them by default)
  void reduce_energies(int rep0 = 0, int count = -1)
  {
    dim3 grid(E_SLOTS, count < 0 ? n_sys() : count);
    dev::k_energy_reduce<<<grid, 256, 0, s0>>>(e_res.p, e_fix.p, efix_slots, n(), sys_begin.p, sys_end.p, energy.p,
                                               rep0);
  }

  void need_single(const char *what)
  {
    if (n_sys() != 1) throw std::invalid_argument(std::string(what) + " needs a single-system handle");
  }

  void compute(long long st, const double *x_ext, double *f_ext, double *energies_out, int groups) override
  {
    need_single("awsem_compute");
    cont_step = -1;
    const std::vector<int> &ext = in.ext_of[0];
    int na = natoms();
    hx.resize((size_t) 3 * na);
    for (int a = 0; a < na; a++)
      for (int k = 0; k < 3; k++) hx[3 * a + k] = x_ext[3 * ext[a] + k];
    CK(cudaMemcpyAsync(x.p, hx.data(), sizeof(double) * 3 * na, cudaMemcpyHostToDevice, s0));
    CK(cudaMemcpyAsync(dstep.p, &st, sizeof st, cudaMemcpyHostToDevice, s0));
    step = st;
    zero_unwritten_energies(groups);
    if (lists_emulated()) {
      // the host's MD loop decides whether this evaluation's lists are new
      set_list_flags(next_compute_built, 1);
      next_compute_built = 1;
    }
    int tb = 256;
    for (int attempt = 0; attempt < 2; attempt++) {
      auto a = args(groups);
      launch_eval(a, false);
      if (lists_emulated()) dev::k_list_hold<R><<<(n_run() + 127) / 128, 128, 0, s0>>>(a);
      dev::k_total_force<R><<<(3 * na + tb - 1) / tb, tb, 0, s0>>>(a, ftot.p);
      reduce_energies();
      CK(cudaGetLastError());
      // an evaluation whose pair list overflowed runs again on a grown list
      // (it changes no state, unless LAMMPS's lists are emulated, whose
      // per-step bookkeeping it advances: then the overflow is reported)
      int ovf = 0;
      CK(cudaMemcpyAsync(&ovf, &nl.p->overflow, sizeof ovf, cudaMemcpyDeviceToHost, s0));
      CK(cudaStreamSynchronize(s0));
      if (!ovf || attempt == 1 || lists_emulated()) break;
      grow_pairs(ovf);
    }
    std::vector<double> f((size_t) 3 * na);
    CK(cudaMemcpyAsync(f.data(), ftot.p, sizeof(double) * 3 * na, cudaMemcpyDeviceToHost, s0));
    double e[E_SLOTS];
    CK(cudaMemcpyAsync(e, energy.p, sizeof e, cudaMemcpyDeviceToHost, s0));
    CK(cudaStreamSynchronize(s0));
    check_list();
    for (int at = 0; at < na; at++)
      for (int k = 0; k < 3; k++) f_ext[3 * ext[at] + k] += f[3 * at + k];
    if (energies_out) finish_energies(e, energies_out, false);
  }

  void finish_energies(const double *e, double *out, bool with_ke)
  {
    for (int k = 0; k < E_SLOTS; k++) out[k] = e[k];
    out[E_TOTAL] = 0.0;
    for (int k = 1; k < E_FIX_TERMS; k++) out[E_TOTAL] += e[k];
    if (!with_ke) out[E_KIN] = 0.0;
  }

  // Limits of the bounded device waits (SM clock cycles; 0: the defaults).
  // The graphs carry the old limits as kernel parameters: recaptured.
  long long fm_wait_limit = dev::kFmWaitLimit, bar_wait_limit = dev::kBarWaitLimit;
  int hold_waits = 0;  // tests: bit 0 copy waits, bit 1 grid barriers made unreachable, so they run out
  void set_wait_limits(long long fm_cycles, long long barrier_cycles, int hold) override
  {
    if (fm_cycles < 0 || barrier_cycles < 0) throw std::invalid_argument("wait limits must not be negative");
    fm_wait_limit = fm_cycles ? fm_cycles : dev::kFmWaitLimit;
    bar_wait_limit = barrier_cycles ? barrier_cycles : dev::kBarWaitLimit;
    if (hold < 0 || hold > 3) throw std::invalid_argument("hold must be 0..3");
    hold_waits = hold;
    release_graphs();
  }

  // After a pair-list overflow the list grows to twice what the evaluation
  // needed (the graphs hold the old buffers and are recaptured), so the next
  // call runs clean.
  void grow_pairs(long long needed)
  {
    release_graphs();
    resize_pairs(std::max<long long>(2LL * pcap, 2LL * needed));
  }

  void check_list()
  {
    dev::NLState st;
    CK(cudaMemcpy(&st, nl.p, sizeof st, cudaMemcpyDeviceToHost));
    if (st.bad_x) {
      // positions are inputs: the next call with finite ones is clean
      set_nl_field(&dev::NLState::bad_x, 0);
      throw StateError("non-finite atom coordinates; results of this call are invalid");
    }
    if (st.overflow) {
      const long long old = pcap;
      grow_pairs(st.overflow);
      throw StateError("residue pair list overflow (capacity " + std::to_string(old) + " pairs, needed " +
                       std::to_string(st.overflow) + "); results of this call are invalid; the capacity is now " +
                       std::to_string(pcap) + " pairs");
    }
    if (st.fm_timeout) {
      set_nl_field(&dev::NLState::fm_timeout, 0);
      throw StateError("fragment-memory stream: a shared-memory copy wait gave up; results of this call are invalid");
    }
    if (st.tb_error) {
      // the reference stops the run with these messages (fix_backbone.cpp:4400, :4423)
      const int code = st.tb_error;
      set_nl_field(&dev::NLState::tb_error, 0);
      throw StateError(code == 1 ? "Table Fragment Memory: r is out of computed range."
                                 : "Table Fragment Memory: ir is out of range.");
    }
    if (gbar.p) {
      dev::GridBar gb;
      CK(cudaMemcpy(&gb, gbar.p, sizeof gb, cudaMemcpyDeviceToHost));
      if (gb.timeout) {
        CK(cudaMemset(gbar.p, 0, sizeof gb));
        throw StateError("persistent step: a grid barrier wait gave up; results of this call are invalid");
      }
    }
  }

  void check_rep(int rep)
  {
    if (rep < 0 || rep >= n_sys()) throw std::invalid_argument("replica index out of range");
  }

  // Whole-batch state transfer: one copy each way through a device staging
  // buffer, and a gather/scatter kernel between caller order and internal order.
  DBuf<int> perm;              // internal atom -> position in the concatenated caller arrays
  DBuf<double> stage;          // [n_atoms][3]

  void ensure_perm()
  {
    if (perm.p) return;
    if (server) throw std::invalid_argument("whole-batch state transfer is not available on a serving handle");
    std::vector<int> pm(natoms());
    for (int r = 0; r < n_sys(); r++) {
      const int a0 = rep_atom0(r), na = rep_atoms(r);
      for (int a = 0; a < na; a++) pm[a0 + a] = a0 + in.ext_of[r][a];
    }
    perm.upload(pm, s0);
    stage.alloc((size_t) 3 * natoms());
  }

  void set_state_all(const double *x_ext, const double *v_ext) override
  {
    ensure_perm();
    cont_step = -1;
    const int na = natoms(), tb = 256;
    for (int k = 0; k < 2; k++) {
      const double *src = k ? v_ext : x_ext;
      if (!src) continue;
      CK(cudaMemcpyAsync(stage.p, src, sizeof(double) * 3 * na, cudaMemcpyHostToDevice, s0));
      dev::k_gather3<<<(na + tb - 1) / tb, tb, 0, s0>>>(stage.p, perm.p, na, k ? v.p : x.p);
    }
    CK(cudaStreamSynchronize(s0));
  }

  void get_state_all(double *x_ext, double *v_ext) override
  {
    ensure_perm();
    const int na = natoms(), tb = 256;
    for (int k = 0; k < 2; k++) {
      double *dst = k ? v_ext : x_ext;
      if (!dst) continue;
      dev::k_scatter3<<<(na + tb - 1) / tb, tb, 0, s0>>>(k ? v.p : x.p, perm.p, na, stage.p);
      CK(cudaMemcpyAsync(dst, stage.p, sizeof(double) * 3 * na, cudaMemcpyDeviceToHost, s0));
      CK(cudaStreamSynchronize(s0));
    }
  }

  void set_state(int rep, const double *x_ext, const double *v_ext) override
  {
    check_rep(rep);
    cont_step = -1;
    const std::vector<int> &ext = in.ext_of[rep];
    int a0 = rep_atom0(rep), na = rep_atoms(rep);
    std::vector<double> bx((size_t) 3 * na), bv((size_t) 3 * na);
    for (int a = 0; a < na; a++)
      for (int k = 0; k < 3; k++) {
        if (x_ext) bx[3 * a + k] = x_ext[3 * ext[a] + k];
        if (v_ext) bv[3 * a + k] = v_ext[3 * ext[a] + k];
      }
    if (x_ext) CK(cudaMemcpyAsync(x.p + 3 * (size_t) a0, bx.data(), sizeof(double) * 3 * na, cudaMemcpyHostToDevice, s0));
    if (v_ext) CK(cudaMemcpyAsync(v.p + 3 * (size_t) a0, bv.data(), sizeof(double) * 3 * na, cudaMemcpyHostToDevice, s0));
    CK(cudaStreamSynchronize(s0));
  }

  void get_state(int rep, double *x_ext, double *v_ext) override
  {
    check_rep(rep);
    const std::vector<int> &ext = in.ext_of[rep];
    int a0 = rep_atom0(rep), na = rep_atoms(rep);
    std::vector<double> hx2((size_t) 3 * na), hv2((size_t) 3 * na);
    CK(cudaMemcpyAsync(hx2.data(), x.p + 3 * (size_t) a0, sizeof(double) * 3 * na, cudaMemcpyDeviceToHost, s0));
    CK(cudaMemcpyAsync(hv2.data(), v.p + 3 * (size_t) a0, sizeof(double) * 3 * na, cudaMemcpyDeviceToHost, s0));
    CK(cudaStreamSynchronize(s0));
    for (int a = 0; a < na; a++)
      for (int k = 0; k < 3; k++) {
        if (x_ext) x_ext[3 * ext[a] + k] = hx2[3 * a + k];
        if (v_ext) v_ext[3 * ext[a] + k] = hv2[3 * a + k];
      }
  }

  // Graphs of `count` consecutive MD steps.  Every per-run value (integrator
  // parameters, step counter, thermo buffer) lives in device memory, so a
  // graph stays valid across runs and is instantiated once.
  cudaGraphExec_t graphs[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [thermo][chunk]
  static constexpr int kChunk = 25;
  DBuf<dev::Integrator> d_integ;
  DBuf<dev::SlotRun> slot_run;  // [n_sys] run window of each replica
  long long thermo_nrows = 1;
  cudaEvent_t ev_run0 = nullptr, ev_run1 = nullptr;
  double last_run_ms = 0.0;

  void capture_steps(cudaGraphExec_t &exec, int count, bool thermo)
  {
    auto a = args(groups_all);
    int nn = n(), tb = 128, nb = (n_run() + tb - 1) / tb;
    const bool persistent = step_form == 1;
    if (persistent) prepare_persistent(a);
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
    for (int c = 0; c < count; c++) {
      if (persistent) {
        launch_step_persistent(a);
      } else {
        launch_eval(a, true);
        dev::k_finish<R><<<finish_blocks(), dev::kFinishThreads, 0, s0>>>(a, d_integ.p, g1.p, g2.p, ftot.p, x.p);
      }
      if (thermo)
        dev::k_thermo<<<n_sys(), 256, 0, s0>>>(e_res.p, e_fix.p, efix_slots, nn, dstep.p, d_integ.p, sys_begin.p, sys_end.p,
                                               thermo_nrows, thermo_rows.p);
    }
    CK(cudaStreamEndCapture(s0, &graph));
    set_node_priorities(graph);
    CK(cudaGraphInstantiate(&exec, graph, 0));
    CK(cudaGraphDestroy(graph));
  }

  // Step form: 0 = the chain of per-pass kernels above (fragment memory on a
  // second stream), 1 = the persistent step kernel of awsem_step.cuh (one
  // cooperative launch per step; replicas without cell grids only).
  int step_form = 0;
  int ps_blocks = 0;  // persistent grid requested (0: every block that fits)
  int ps_stream = 2;  // fragment-memory stream warps per block
  int ps_grid_now = 0, ps_smem_now = 0;
  DBuf<dev::GridBar> gbar;

  bool fm_on(const dev::StepArgs<R> &a) const { return (a.groups & dev::G_FIX) && in.ff.p.fm_nd > 0; }
  // warps with a shared-memory copy ring: as many as fit in about half an SM's shared memory
  int ps_ring_warps() const
  {
    return std::min(dev::kStepThreads / 32, (112 * 1024) / dev::fm_warp_smem<R>(!in.fm.uniform));
  }

  // grid and shared memory of the persistent kernel (outside stream capture)
  void prepare_persistent(const dev::StepArgs<R> &a)
  {
    if (nbig) throw std::invalid_argument("the persistent step kernel does not build cell grids (replicas above 2,048 residues)");
    // fresh barrier state for the graphs about to be captured (nothing is in flight on s0)
    if (!gbar.p) gbar.alloc(1);
    CK(cudaMemsetAsync(gbar.p, 0, sizeof(dev::GridBar), s0));
    CK(cudaStreamSynchronize(s0));
    ps_smem_now = fm_on(a) ? ps_ring_warps() * dev::fm_warp_smem<R>(!in.fm.uniform) : 0;
    CK(cudaFuncSetAttribute(dev::k_step<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, ps_smem_now));
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::k_step<R>, dev::kStepThreads, ps_smem_now));
    if (per_sm < 1) throw CudaError("the persistent step kernel does not fit on a multiprocessor");
    const int most = per_sm * sms_;
    ps_grid_now = ps_blocks > 0 ? std::min(ps_blocks, most) : most;
  }

  // one MD step (evaluation, Langevin, velocity Verlet) as one cooperative launch
  void launch_step_persistent(const dev::StepArgs<R> &a)
  {
    const bool fm = fm_on(a);
    dev::PersistArgs q{d_integ.p, g1.p, g2.p, ftot.p, x.p, gbar.p, n_run(), ps_stream,
                       fm ? ps_ring_warps() : 0, fm ? std::min(fm_groups, (n_run() + 31) / 32) * fm_dsplit : 0,
                       (a.groups & dev::G_FIX) && (in.ff.p.terms & T_FM_TABLE) ? 1 : 0,
                       (a.groups & dev::G_FIX) && (in.ff.p.terms & T_AMHGO) ? 1 : 0,
                       (a.groups & dev::G_FIX) && (in.ff.p.terms & (T_SSB | T_DH | T_CONTREST)) ? 1 : 0,
                       lists_emulated() ? n_sys() : 0,
                       (a.groups & dev::G_FIX) && (in.ff.p.terms & (T_SHAKE | T_MEMB | T_VFM)) ? 1 : 0,
                       bar_wait_limit, (hold_waits & 2) ? 1u : 0u};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ps_grid_now);
    cfg.blockDim = dim3(dev::kStepThreads);
    cfg.dynamicSmemBytes = ps_smem_now;
    cfg.stream = s0;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, dev::k_step<R>, a, in.ff.p, q));
  }

  void set_step_form(int form, int blocks, int stream_warps) override
  {
    if (form != 0 && form != 1) throw std::invalid_argument("step form must be 0 (per-pass kernels) or 1 (persistent)");
    if (blocks < 0) throw std::invalid_argument("blocks must be >= 0 (0: every block that fits)");
    if (stream_warps < 1 || stream_warps > dev::kStepThreads / 32 - 1)
      throw std::invalid_argument("stream_warps must be in 1..7");
    if (form == 1 && nbig)
      throw std::invalid_argument("the persistent step kernel does not build cell grids (replicas above 2,048 residues)");
    step_form = form;
    ps_blocks = blocks;
    ps_stream = stream_warps;
    release_graphs();
  }

  // shapes as awsem_autotune reports them: [dsplit, pair blocks, hbond blocks, fragmem blocks]
  void set_neighbor(double skin_, int delay, int every, int check) override
  {
    if (delay < 0 || every < 1 || (check != 0 && check != 1))
      throw std::invalid_argument("neigh_modify: delay >= 0, every >= 1, check 0 or 1");
    if (skin_ > 0 && skin_ != skin) {
      skin = skin_;
      set_nl_field(&dev::NLState::skin, (float) skin);
      set_nl_field(&dev::NLState::lst_skin, skin);
      set_nl_field(&dev::NLState::lst_pair_cut, pair_cut_now());
      set_nl_field(&dev::NLState::r_list, 0.f);  // the next evaluation rebuilds the pair list
    }
    set_nl_field(&dev::NLState::lst_delay, delay);
    set_nl_field(&dev::NLState::lst_every, every);
    set_nl_field(&dev::NLState::lst_check, check);
    CK(cudaStreamSynchronize(s0));
  }

  void set_launch_shapes(const int *sh) override
  {
    const int nd = std::max(in.ff.p.fm_nd, 1);
    if (sh[0] < 1 || sh[0] > nd)
      throw std::invalid_argument("separations per fragment-memory warp must be in 1.." + std::to_string(nd));
    if (sh[1] < 1 || sh[2] < 1) throw std::invalid_argument("pair and hydrogen-bond grids must be >= 1 block");
    if (sh[3] < 0) throw std::invalid_argument("fragment-memory grid must be >= 0 (0: one warp per unit)");
    fm_dsplit = sh[0];
    pair_blocks = sh[1];
    hb_blocks = sh[2];
    fm_grid = sh[3];
    release_graphs();
  }

  void get_step_form(int *out) override
  {
    out[0] = step_form;
    out[1] = step_form == 1 ? (ps_grid_now ? ps_grid_now : ps_blocks) : 0;
    out[2] = ps_stream;
  }

  // Kernel nodes keep the priority of the stream they were captured from
  // (fragment memory low, everything else high), set explicitly per node.
  void set_node_priorities(cudaGraph_t graph)
  {
    size_t count = 0;
    CK(cudaGraphGetNodes(graph, nullptr, &count));
    std::vector<cudaGraphNode_t> nodes(count);
    CK(cudaGraphGetNodes(graph, nodes.data(), &count));
    for (cudaGraphNode_t node : nodes) {
      cudaGraphNodeType type;
      CK(cudaGraphNodeGetType(node, &type));
      if (type != cudaGraphNodeTypeKernel) continue;
      cudaKernelNodeParams kp;
      CK(cudaGraphKernelNodeGetParams(node, &kp));
      cudaLaunchAttributeValue v;
      v.priority = kp.func == (void *) dev::k_fragmem<R> ? prio_lo : prio_hi;
      CK(cudaGraphKernelNodeSetAttribute(node, cudaLaunchAttributePriority, &v));
    }
  }

  void release_graphs()
  {
    for (auto &row : graphs)
      for (auto &g : row)
        if (g) {
          cudaGraphExecDestroy(g);
          g = nullptr;
        }
  }

  awsem_run_params last_rp{2.0, 1, 300.0, 300.0, 500.0, 1ull, 2.0, 0};

  void upload_integrator(const dev::Integrator &integ)
  {
    if (!d_integ.p) d_integ.alloc(1);
    CK(cudaMemcpyAsync(d_integ.p, &integ, sizeof integ, cudaMemcpyHostToDevice, s0));
  }

  // One run window for every replica (a run of the whole batch): steps
  // begin..end, noise keyed by the absolute step.
  void upload_runs(const awsem_run_params &rp, long long begin, long long end)
  {
    upload_integrator(make_integrator(rp, begin));
    std::vector<dev::SlotRun> w(n_sys(), dev::SlotRun{begin, end, 0, rp.t_start, rp.t_stop});
    CK(cudaMemcpyAsync(slot_run.p, w.data(), sizeof(dev::SlotRun) * w.size(), cudaMemcpyHostToDevice, s0));
    CK(cudaStreamSynchronize(s0));
  }

  // Launch-shape autotuner: separations per fragment-memory warp (dsplit),
  // grid of the pair-parallel passes and of the hydrogen-bond pass.  Each
  // candidate runs `reps` profiled steps on this handle's own system; the
  // fastest per knob wins.  The state and step counter are restored after.
  void autotune(int reps, int *chosen) override
  {
    if (server) throw std::invalid_argument("autotune: not available on a serving handle");
    if (reps <= 0) throw std::invalid_argument("reps must be positive");
    const int na = natoms();
    DBuf<double> sx, sv;
    sx.alloc((size_t) 3 * na);
    sv.alloc((size_t) 3 * na);
    CK(cudaMemcpyAsync(sx.p, x.p, sizeof(double) * 3 * na, cudaMemcpyDeviceToDevice, s0));
    CK(cudaMemcpyAsync(sv.p, v.p, sizeof(double) * 3 * na, cudaMemcpyDeviceToDevice, s0));
    const long long step_saved = step;
    int sms = 148;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    std::vector<double> ms(AWSEM_NKERNELS);
    auto time_of = [&](std::initializer_list<int> kernels) {
      release_graphs();
      profile(1, ms.data());  // warm-up of this shape
      profile(reps, ms.data());
      double t = 0;
      for (int k : kernels) t += ms[k];
      return t;
    };
    // fragment memory: separations per warp
    const int nd = std::max(in.ff.p.fm_nd, 1);
    if (in.ff.p.fm_nd > 0) {
      int best = fm_dsplit;
      double tbest = 1e30;
      for (int d : {1, 2, 3, 6, nd}) {
        if (d > nd) continue;
        fm_dsplit = d;
        const double t = time_of({K_FRAGMEM});
        if (t < tbest) tbest = t, best = d;
      }
      fm_dsplit = best;
    }
    // pair-parallel passes (density, water_xi, pair) and the hydrogen-bond pass
    auto tune_blocks = [&](int &blocks, std::initializer_list<int> kernels) {
      int best = blocks;
      double tbest = 1e30;
      for (int f : {1, 2, 4, 8, 16, 32}) {
        blocks = f * sms;
        const double t = time_of(kernels);
        if (t < tbest) tbest = t, best = blocks;
      }
      blocks = best;
    };
    tune_blocks(pair_blocks, {K_DENSITY, K_WATER_XI, K_RADIAL, K_PAIR});
    tune_blocks(hb_blocks, {K_HBOND});
    // fragment-memory grid with the pair-pass grid, judged together on whole
    // steps: fragment memory (HBM-bound, second stream) can only overlap the
    // latency-bound pair passes when their grids leave it room on the SMs
    if (in.ff.p.fm_nd > 0) {
      int best = 0, best_pb = pair_blocks;
      double tbest = 1e30;
      const int tuned_pb = pair_blocks;
      std::vector<int> grids{tuned_pb};
      for (int k : {4, 8, 16, 32})
        if (k * sms != tuned_pb) grids.push_back(k * sms);
      for (int pb : grids) {
        for (int f : {0, 1, 2, 3, 4}) {
          pair_blocks = pb;
          fm_grid = f * sms;
          release_graphs();
          run(reps, last_rp, nullptr);  // warm-up of this shape (graph capture)
          run(4 * reps, last_rp, nullptr);
          if (last_run_ms < tbest) tbest = last_run_ms, best = fm_grid, best_pb = pb;
        }
      }
      fm_grid = best;
      pair_blocks = best_pb;
    }
    // step form: the chain of per-pass kernels against the persistent step
    // kernel over its grid size and stream-warp count, on whole steps
    if (!nbig) {
      auto whole_steps = [&]() {
        release_graphs();
        run(reps, last_rp, nullptr);  // warm-up of this shape (graph capture)
        run(4 * reps, last_rp, nullptr);
        return last_run_ms;
      };
      step_form = 0;
      double tbest = whole_steps();
      int bform = 0, bblocks = ps_blocks, bstream = ps_stream;
      for (int blocks : {0, sms, sms / 2, sms / 4, 8})
        for (int sw : {1, 2, 3, 4}) {
          step_form = 1;
          ps_blocks = blocks;
          ps_stream = sw;
          const double t = whole_steps();
          if (t < tbest) tbest = t, bform = 1, bblocks = blocks, bstream = sw;
        }
      step_form = bform;
      ps_blocks = bblocks;
      ps_stream = bstream;
    }
    release_graphs();
    CK(cudaMemcpyAsync(x.p, sx.p, sizeof(double) * 3 * na, cudaMemcpyDeviceToDevice, s0));
    CK(cudaMemcpyAsync(v.p, sv.p, sizeof(double) * 3 * na, cudaMemcpyDeviceToDevice, s0));
    CK(cudaStreamSynchronize(s0));
    step = step_saved;
    cont_step = -1;
    set_nl_field(&dev::NLState::r_list, 0.f);
    if (chosen) {
      chosen[0] = fm_dsplit;
      chosen[1] = pair_blocks;
      chosen[2] = hb_blocks;
      chosen[3] = fm_grid;
    }
  }

  void profile(int reps, double *ms) override
  {
    if (reps <= 0) throw std::invalid_argument("reps must be positive");
    cont_step = -1;
    set_thermostat(last_rp);
    upload_runs(last_rp, step, step + reps + 1);
    long long pre = step;  // profiled steps continue the trajectory
    CK(cudaMemcpyAsync(dstep.p, &pre, sizeof pre, cudaMemcpyHostToDevice, s0));
    const FFParams &p = in.ff.p;
    auto a = args(groups_all);
    int nn = n_run(), tb = 128, nb = (nn + tb - 1) / tb;
    std::vector<cudaEvent_t> ev(2 * AWSEM_NKERNELS);
    for (auto &e : ev) CK(cudaEventCreate(&e));
    std::vector<double> acc(AWSEM_NKERNELS, 0.0);
    bool fm = p.fm_nd > 0;
    for (int r = 0; r < reps; r++) {
      for (int k = 0; k < AWSEM_NKERNELS; k++) {
        CK(cudaEventRecord(ev[2 * k], s0));
        switch (k) {
          case K_PREPARE: dev::k_prepare<R><<<nb, tb, 0, s0>>>(a, p); break;
          case K_NL_DECIDE: dev::k_nl_decide<<<1, 1, 0, s0>>>(nl.p, 0, dstep.p); break;
          case K_NL_BUILD: launch_list_build(a, s0); break;
          case K_DENSITY: dev::k_density<R><<<pair_blocks, tb, 0, s0>>>(a, p); break;
          case K_RESIDUE: dev::k_residue<R><<<nb, tb, 0, s0>>>(a, p); break;
          case K_BACKBONE: dev::k_backbone<R><<<nb, tb, 0, s0>>>(a, p); break;
          case K_WATER_XI: dev::k_water_xi<R><<<pair_blocks, tb, 0, s0>>>(a, p); break;
          case K_RADIAL: dev::k_radial<R><<<pair_blocks, tb, 0, s0>>>(a, p); break;
          case K_PAIR: dev::k_pair<R><<<pair_blocks, tb, 0, s0>>>(a, p); break;
          case K_HBOND: dev::k_hbond<R><<<hb_blocks, 128, 0, s0>>>(a, p); break;
          case K_FRAGMEM:
            if (fm) dev::k_fragmem<R><<<fm_blocks(), tb, fm_smem(), s0>>>(a, p);
            if (p.terms & T_FM_TABLE) dev::k_fm_table<R><<<fm_table_blocks(), tb, 0, s0>>>(a, p);
            if (p.terms & T_AMHGO) dev::k_amh_go<R><<<nb, tb, 0, s0>>>(a, p);
            if (p.terms & (T_SSB | T_DH | T_CONTREST)) dev::k_pair_extra<R><<<pair_blocks, tb, 0, s0>>>(a, p);
            if (p.terms & (T_SHAKE | T_MEMB | T_VFM)) dev::k_residue_extra<R><<<nb, tb, 0, s0>>>(a, p);
            break;
          case K_FINISH: dev::k_finish<R><<<finish_blocks(), dev::kFinishThreads, 0, s0>>>(a, d_integ.p, g1.p, g2.p, ftot.p, x.p); break;
        }
        CK(cudaEventRecord(ev[2 * k + 1], s0));
      }
      CK(cudaStreamSynchronize(s0));
      for (int k = 0; k < AWSEM_NKERNELS; k++) {
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, ev[2 * k], ev[2 * k + 1]));
        acc[k] += t;
      }
    }
    for (auto &e : ev) cudaEventDestroy(e);
    for (int k = 0; k < AWSEM_NKERNELS; k++) ms[k] = acc[k] / reps;
    step += reps;
    check_list();
  }

  double run_ms() const override { return last_run_ms; }

  FMView fm_view() const override
  {
    FMView v;
    v.soff = fm_soff.p;
    v.slen = fm_slen.p;
    v.rf = fm_rf.p;
    v.coef = in.fm.uniform ? nullptr : fm_coef.p;
    v.uniform = in.fm.uniform_coef;
    v.nd = in.ff.p.fm_nd;
    v.min_sep = in.ff.p.fm_min_sep;
    v.groups = fm_groups;
    v.dsplit = fm_dsplit;
    v.n_res = n();
    v.is_double = sizeof(R) == sizeof(double);
    v.sigma_sq = in.ff.p.fm_sigma_sq;
    return v;
  }

  // Fragment-memory table in the sliced, lane-interleaved layout of
  // awsem_fragmem.cuh, in the engine's arithmetic type.
  void upload_fm_slices()
  {
    const FMTable &fm = in.fm;
    const int nn = n(), nd = in.ff.p.fm_nd;
    fm_groups = (nn + 31) / 32;
    std::vector<int> soff((size_t) fm_groups * std::max(nd, 1), 0), slen(soff.size(), 0);
    long long stripes = 0;
    for (int g = 0; g < fm_groups; g++)
      for (int d = 0; d < nd; d++) {
        int len = 0;
        for (int l = 0; l < 32 && 32 * g + l < nn; l++) {
          size_t row = (size_t) (32 * g + l) * fm.nd + d;
          len = std::max(len, fm.row_start[row + 1] - fm.row_start[row]);
        }
        len += len & 1;  // even: the kernels take a row's records in pairs
        soff[(size_t) g * nd + d] = (int) stripes;
        slen[(size_t) g * nd + d] = len;
        stripes += len;
      }
    if (stripes * 32 * 4 >= (1ll << 31)) throw std::invalid_argument("fragment memory table exceeds 2^31 distances");
    const bool coef = !fm.uniform;
    std::vector<R> rf((size_t) stripes * 32 * 4, R(FMTable::FM_SKIP)), cf(coef ? (size_t) stripes * 32 : 0, R(0));
    for (int g = 0; g < fm_groups; g++)
      for (int d = 0; d < nd; d++) {
        const size_t s0b = soff[(size_t) g * nd + d];
        for (int l = 0; l < 32 && 32 * g + l < nn; l++) {
          size_t row = (size_t) (32 * g + l) * fm.nd + d;
          for (int m = 0, rec = fm.row_start[row]; rec < fm.row_start[row + 1]; m++, rec++) {
            size_t at = (s0b + m) * 32 + l;
            for (int k = 0; k < 4; k++) rf[at * 4 + k] = (R) fm.rf[(size_t) rec * 4 + k];
            if (coef) cf[at] = (R) fm.coef[rec];
          }
        }
      }
    fm_soff.upload(soff, s0);
    fm_slen.upload(slen, s0);
    fm_rf.upload(rf, s0);
    fm_coef.upload(cf, s0);
    // enough warps to fill the GPU on small systems: split each group's
    // separations over several warps when there are few groups
    int sms = 148;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    fm_dsplit = std::max(1, std::min(std::max(nd, 1), (16 * sms + fm_groups - 1) / std::max(fm_groups, 1)));
    CK(cudaStreamSynchronize(s0));  // host vectors go out of scope
  }

  // one warp per fragment-memory work unit, or a smaller persistent grid
  // (fm_grid blocks) whose warps loop over the units
  int fm_grid = 0;
  int fm_blocks() const
  {
    const int all = (((n_run() + 31) / 32) * fm_dsplit * 32 + 127) / 128;
    return fm_grid > 0 ? std::min(all, fm_grid) : all;
  }
  // dynamic shared memory of a fragment-memory block (4 warps)
  int fm_smem() const { return 4 * dev::fm_warp_smem<R>(!in.fm.uniform); }

  void model_info(long long *info) override
  {
    info[0] = n();
    info[1] = natoms();
    info[2] = in.fm.records();
    info[3] = sizeof(R);
    info[4] = in.ff.p.fm_nd;
    info[5] = pcap;
    dev::NLState st;
    CK(cudaMemcpyAsync(&st, nl.p, sizeof st, cudaMemcpyDeviceToHost, s0));
    CK(cudaStreamSynchronize(s0));
    info[6] = st.npairs;
    info[7] = in.fm.uniform ? 0 : 1;
  }

  awsem_run_params thermostat_rp{0, 0, 0, 0, 0, 0, 0, 0};

  void set_thermostat(const awsem_run_params &rp)
  {
    if (rp.dt == thermostat_rp.dt && rp.damp == thermostat_rp.damp) return;
    const Topology &t = in.top;
    int na = natoms();
    std::vector<double> h1(na), h2(na);
    for (int a = 0; a < na; a++) {
      double m = t.mass[a];
      h1[a] = -m / rp.damp / FTM2V;
      h2[a] = sqrt(m) * sqrt(24.0 * BOLTZ / rp.damp / rp.dt / MVV2E) / FTM2V;
    }
    CK(cudaMemcpyAsync(g1.p, h1.data(), sizeof(double) * na, cudaMemcpyHostToDevice, s0));
    CK(cudaMemcpyAsync(g2.p, h2.data(), sizeof(double) * na, cudaMemcpyHostToDevice, s0));
    CK(cudaStreamSynchronize(s0));
    thermostat_rp = rp;
  }

  dev::Integrator make_integrator(const awsem_run_params &rp, long long begin)
  {
    dev::Integrator integ{};
    integ.dt = rp.dt;
    integ.dtf = 0.5 * rp.dt * FTM2V;
    integ.langevin = rp.langevin;
    integ.begin = begin;
    integ.stop = std::numeric_limits<long long>::max();
    integ.damp = rp.damp;
    return integ;
  }

  // A run that stopped before its window's end leaves the state at the full
  // step `cont_step`, with that step's total force in ftot; a later call may
  // continue the window from there.  Anything else that touches the state or
  // ftot clears it (-1).
  long long cont_step = -1, cont_wbegin = 0, cont_wend = 0;

  void run(long long nsteps, const awsem_run_params &rp, double *thermo) override
  {
    run_window(nsteps, rp, step, step + nsteps, false, thermo);
  }

  // Steps step+1 .. step+nsteps of the window [wbegin, wend], whose ends set
  // the thermostat ramp and the integration window (setup evaluation at
  // wbegin, no drift after wend).  cont = false: the call begins with the
  // setup evaluation at the current step, which must be wbegin; cont = true:
  // it continues a call that stopped at the current step inside the same
  // window.
  void run_window(long long nsteps, const awsem_run_params &rp, long long wbegin, long long wend, bool cont,
                  double *thermo) override
  {
    if (nsteps < 0) throw std::invalid_argument("nsteps must be >= 0");
    if (cont) {
      if (cont_step != step || wbegin != cont_wbegin || wend != cont_wend)
        throw std::invalid_argument("continue: the previous call on this handle did not stop at step " +
                                    std::to_string(step) + " inside this window");
      if (nsteps < 1) throw std::invalid_argument("continue: nsteps must be >= 1");
    } else if (wbegin != step) {
      throw std::invalid_argument("the window must begin at the current step " + std::to_string(step));
    }
    if (step + nsteps > wend) throw std::invalid_argument("the call runs past the window's end");
    cont_step = -1;
    last_rp = rp;
    // thermostat factors per atom (fix langevin, units real)
    set_thermostat(rp);
    if (rp.skin > 0 && rp.skin != skin) {
      skin = rp.skin;
      set_nl_field(&dev::NLState::skin, (float) skin);
      set_nl_field(&dev::NLState::lst_skin, skin);
      set_nl_field(&dev::NLState::lst_pair_cut, pair_cut_now());
    }
    // a run's first evaluation is its setup: LAMMPS builds every list there;
    // the engine decides the later builds
    if (!cont && lists_emulated()) set_list_flags(1, 0);
    if (rp.neigh_every != neigh_every) {
      neigh_every = rp.neigh_every;
      set_nl_field(&dev::NLState::every, neigh_every);
    }
    const long long rows = cont ? nsteps : nsteps + 1;  // evaluations of this call
    dev::Integrator integ = make_integrator(rp, cont ? step + 1 : step);
    integ.stop = step + nsteps;
    upload_integrator(integ);
    std::vector<dev::SlotRun> w(n_sys(), dev::SlotRun{wbegin, wend, 0, rp.t_start, rp.t_stop});
    CK(cudaMemcpyAsync(slot_run.p, w.data(), sizeof(dev::SlotRun) * w.size(), cudaMemcpyHostToDevice, s0));
    // Langevin seed of each replica: its own when set, else the run's
    std::vector<unsigned long long> sd(n_sys());
    for (int k = 0; k < n_sys(); k++) sd[k] = seeds[k] ? seeds[k] : rp.seed;
    CK(cudaMemcpyAsync(sys_seed.p, sd.data(), sizeof(unsigned long long) * sd.size(), cudaMemcpyHostToDevice, s0));
    // a setup evaluation advances the counter to `step`; a continuation starts from it
    long long pre = cont ? step : step - 1;
    CK(cudaMemcpyAsync(dstep.p, &pre, sizeof pre, cudaMemcpyHostToDevice, s0));
    CK(cudaStreamSynchronize(s0));
    bool want_thermo = thermo != nullptr;
    int tv = want_thermo ? 1 : 0;
    if (want_thermo) {
      // thermo graphs bake the row buffer's address and row count: rebuilt per run
      thermo_nrows = rows;
      thermo_rows.alloc((size_t) 4 * rows * n_sys());
      for (auto &g : graphs[1])
        if (g) {
          cudaGraphExecDestroy(g);
          g = nullptr;
        }
    }
    long long total = rows;
    if (!graphs[tv][0]) capture_steps(graphs[tv][0], 1, want_thermo);
    if (total >= kChunk && !graphs[tv][1]) capture_steps(graphs[tv][1], kChunk, want_thermo);
    if (!ev_run0) {
      CK(cudaEventCreate(&ev_run0));
      CK(cudaEventCreate(&ev_run1));
    }
    long long done = 0;
    CK(cudaEventRecord(ev_run0, s0));
    if (cont) {
      const int tb = 128;
      dev::k_continue<R><<<(n_run() + tb - 1) / tb, tb, 0, s0>>>(args(groups_all), d_integ.p, ftot.p, x.p);
      CK(cudaGetLastError());
    }
    while (total - done >= kChunk) {
      CK(cudaGraphLaunch(graphs[tv][1], s0));
      done += kChunk;
    }
    while (done < total) {
      CK(cudaGraphLaunch(graphs[tv][0], s0));
      done++;
    }
    CK(cudaEventRecord(ev_run1, s0));
    CK(cudaStreamSynchronize(s0));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ev_run0, ev_run1));
    last_run_ms = ms;
    step += nsteps;
    check_list();
    if (want_thermo)
      CK(cudaMemcpy(thermo, thermo_rows.p, sizeof(double) * 4 * rows * n_sys(), cudaMemcpyDeviceToHost));
    if (step < wend) {
      cont_step = step;
      cont_wbegin = wbegin;
      cont_wend = wend;
    }
  }

  int next_compute_built = 1;  // awsem_set_list_built: the next awsem_compute's list is new

  // terms that read list membership itself: LAMMPS's lists are emulated
  bool lists_emulated() const { return in.ff.p.terms & (T_AMHGO | T_SSB | T_DH | T_CONTREST); }
  // the CA-CA reach of the fix's half list the residue pair list must cover (0: no term needs it)
  float pair_cut_now() const
  {
    return (in.ff.p.terms & (T_SSB | T_DH)) ? (float) (in.ff.p.pair_list_cutoff + skin) * 1.0001f : 0.f;
  }

  void set_list_flags(int force, int host)
  {
    dev::NLState st;
    CK(cudaMemcpyAsync(&st, nl.p, sizeof st, cudaMemcpyDeviceToHost, s0));
    CK(cudaStreamSynchronize(s0));
    st.lst_force = force;
    st.lst_host = host;
    CK(cudaMemcpyAsync(nl.p, &st, sizeof st, cudaMemcpyHostToDevice, s0));
  }

  void set_list_built(int built) override { next_compute_built = built ? 1 : 0; }

  // Q order parameters (compute qwolynes / qonuchic) of single replicas
  struct QDev {
    int rep = 0;
    QDefinition def;
    DBuf<double> mat, partial, out;
  };
  std::vector<std::unique_ptr<QDev>> qdefs;

  int q_create(int rep, const std::string &words) override
  {
    check_rep(rep);
    std::unique_ptr<QDev> q(new QDev());
    q->rep = rep;
    q->def = parse_q_compute(words, rep_res(rep));
    q->mat.upload(q->def.mat, s0);
    q->partial.alloc((size_t) std::max(q->def.n, 1));
    q->out.alloc(1);
    std::vector<double>().swap(q->def.mat);
    CK(cudaStreamSynchronize(s0));
    qdefs.push_back(std::move(q));
    return (int) qdefs.size() - 1;
  }

  double q_value(int qid) override
  {
    if (qid < 0 || qid >= (int) qdefs.size()) throw std::invalid_argument("no such Q definition");
    QDev &q = *qdefs[qid];
    const QDefinition &d = q.def;
    const double *xr = x.p + (size_t) 3 * rep_atom0(q.rep);
    if (d.n > 0) {
      dev::k_q_rows<<<d.n, 256, 0, s0>>>(xr, d.n, d.kind, d.sep, d.sigma_exp, q.mat.p, q.partial.p);
      dev::k_q_sum<<<1, 256, 0, s0>>>(q.partial.p, d.n, d.qnorm, q.out.p);
    }
    CK(cudaGetLastError());
    double v = 0.0;
    if (d.n > 0) CK(cudaMemcpyAsync(&v, q.out.p, sizeof v, cudaMemcpyDeviceToHost, s0));
    CK(cudaStreamSynchronize(s0));
    return v;
  }

  template <typename F> void set_nl_field(F dev::NLState::*field, F value)
  {
    dev::NLState st;
    CK(cudaMemcpyAsync(&st, nl.p, sizeof st, cudaMemcpyDeviceToHost, s0));
    CK(cudaStreamSynchronize(s0));
    st.*field = value;
    CK(cudaMemcpyAsync(nl.p, &st, sizeof st, cudaMemcpyHostToDevice, s0));
  }

  void energies(int rep, double *out) override
  {
    check_rep(rep);
    reduce_energies(rep, 1);
    double e[E_SLOTS];
    CK(cudaMemcpyAsync(e, energy.p + (size_t) rep * E_SLOTS, sizeof e, cudaMemcpyDeviceToHost, s0));
    CK(cudaStreamSynchronize(s0));
    finish_energies(e, out, true);
  }

  void forces(int rep, double *f_ext) override
  {
    check_rep(rep);
    const std::vector<int> &ext = in.ext_of[rep];
    int a0 = rep_atom0(rep), na = rep_atoms(rep);
    std::vector<double> f((size_t) 3 * na);
    CK(cudaMemcpyAsync(f.data(), ftot.p + 3 * (size_t) a0, sizeof(double) * 3 * na, cudaMemcpyDeviceToHost, s0));
    CK(cudaStreamSynchronize(s0));
    for (int at = 0; at < na; at++)
      for (int k = 0; k < 3; k++) f_ext[3 * ext[at] + k] = f[3 * at + k];
  }

  void residue_arrays(int rep, double *out) override
  {
    check_rep(rep);
    int nn = n(), r0 = in.sys_res_begin[rep], nr = rep_res(rep);
    std::vector<double> w((size_t) 10 * nn);
    std::vector<long long> raw(nn);
    CK(cudaMemcpyAsync(w.data(), work.p, sizeof(double) * 10 * nn, cudaMemcpyDeviceToHost, s0));
    CK(cudaMemcpyAsync(raw.data(), dacc.p + (size_t) 2 * nn, sizeof(long long) * nn, cudaMemcpyDeviceToHost, s0));
    CK(cudaStreamSynchronize(s0));
    // xi_water = raw pair sum (2^-40 fixed point) * sigma_water', as k_pair forms it
    for (int r = 0; r < nn; r++) w[(size_t) 6 * nn + r] = (double) raw[r] * dev::D_UNSCALE * w[(size_t) 3 * nn + r];
    // device order: rho_w rho_h sig_w sigp_w sig_h sigp_h xi_w xi1 xi2 bur
    const int src[8] = {0, 1, 6, 7, 8, 9, 2, 4};
    for (int r = 0; r < nr; r++)
      for (int c = 0; c < 8; c++) out[8 * r + c] = w[(size_t) src[c] * nn + r0 + r];
  }

  void nl_stats(int *nbuilds, double *radius, int *maxc, int *overflow) override
  {
    dev::NLState st;
    CK(cudaMemcpyAsync(&st, nl.p, sizeof st, cudaMemcpyDeviceToHost, s0));
    CK(cudaStreamSynchronize(s0));
    if (nbuilds) *nbuilds = st.nbuilds;
    if (radius) *radius = st.r_list;
    if (overflow) *overflow = st.overflow;
    if (maxc) *maxc = max_count();
  }

  // ----------------------------------------------------------------------
  // Serving: a fixed-capacity handle whose replicas (requests) come and go.
  // Residues are handed out in 32-residue groups (one fragment-memory group
  // never mixes requests) and memory records in 32-record stripes, first
  // fit; all device arrays are allocated once at creation, so admission
  // and release only copy a request's data in or out.
  struct Slot {
    bool used = false;
    int base = 0, n_res = 0, groups = 0;
    long long stripe0 = 0, stripes = 0;
    long long begin = 0, end = 0;  // run window (device steps)
  };
  std::vector<Slot> slots;
  std::map<long long, long long> free_groups, free_stripes;  // start -> length
  const SharedForceField *sf = nullptr;
  awsem_run_params srv_rp{};
  long long stripe_cap = 0;
  bool fm_coef_mode = false, fm_uniform_known = false;

  static bool take_range(std::map<long long, long long> &fr, long long want, long long &at)
  {
    if (want == 0) {
      at = 0;
      return true;
    }
    for (auto it = fr.begin(); it != fr.end(); ++it)
      if (it->second >= want) {
        at = it->first;
        long long rest = it->second - want;
        fr.erase(it);
        if (rest) fr[at + want] = rest;
        return true;
      }
    return false;
  }

  static void give_range(std::map<long long, long long> &fr, long long at, long long len)
  {
    if (len == 0) return;
    auto it = fr.emplace(at, len).first;
    auto nx = std::next(it);
    if (nx != fr.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      fr.erase(nx);
    }
    if (it != fr.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        fr.erase(it);
      }
    }
  }

  template <typename T> void put(DBuf<T> &b, size_t at, const T *src, size_t count)
  {
    if (count) CK(cudaMemcpyAsync(b.p + at, src, count * sizeof(T), cudaMemcpyHostToDevice, s0));
  }
  template <typename T> void fill(DBuf<T> &b, size_t at, size_t count, T value)
  {
    std::vector<T> h(count, value);
    put(b, at, h.data(), count);
    CK(cudaStreamSynchronize(s0));
  }

  void server_setup(const SharedForceField &f, long long cap_res, int max_slots, long long cap_records, double dt,
                    double damp) override
  {
    if (cap_res <= 0 || max_slots <= 0 || cap_records < 0) throw std::invalid_argument("server capacities must be positive");
    if (dt <= 0 || damp <= 0) throw std::invalid_argument("dt and damp must be positive");
    if (f.ff.p.terms & T_FM_TABLE)
      throw std::invalid_argument("serving handles do not support [Fragment_Memory_Table] (use [Fragment_Memory])");
    if (f.ff.p.terms & T_AMHGO) throw std::invalid_argument("serving handles do not support [AMH-Go]");
    if (f.ff.p.terms & (T_SSB | T_DH | T_CONTREST | T_MEMB))
      throw std::invalid_argument(
          "serving handles do not support [Solvent_Barrier], [DebyeHuckel], [Contact_Restraints] or [Membrane]");
    const long long groups = (cap_res + 31) / 32;
    if (groups * 32 * pairs_per_res >= (1ll << 31)) throw std::invalid_argument("residue capacity too large");
    sf = &f;
    server = true;
    const int nn = (int) (groups * 32);
    pairs_per_res = 64;  // requests that anneal collapse: room for the densest packing
    in = Batch();
    in.ff = f.ff;
    FFParams &p = in.ff.p;
    int nd = 0;
    if (p.terms & T_FM) {
      const int ms = f.gamma.min_sep(), xs = f.gamma.max_sep();
      nd = xs == -1 ? 64 - ms : xs - ms + 1;
      p.fm_min_sep = ms;
    }
    p.fm_nd = nd;
    Topology &t = in.top;
    t.n_res = nn;
    t.n_atoms = 3 * nn;
    t.n_chains = nn;
    t.ntypes = 5;
    set_pair_coeffs(t, f.pair_style, f.pair_coeffs);
    // residues of no request: flagged chain ends of no chain, fully excluded
    t.res_type.assign(nn, 0);
    t.res_flags.assign(nn, R_FIRST | R_LAST);
    t.res_chain.assign(nn, -1);
    t.chain_start.assign(nn, 0);  // chain ids are the global index of a chain's first residue
    t.chain_end.assign(nn, 0);
    t.aps.assign((size_t) 12 * nn, 0.0);
    t.atom_type.assign(3 * nn, 1);
    t.atom_tag.assign(3 * nn, 0);
    t.mass.assign(3 * nn, 1.0);
    t.excl_self.assign(nn, 0x1ffu);
    t.excl_next.assign(nn, 0u);
    in.x.assign((size_t) 9 * nn, 0.0);
    in.v.assign((size_t) 9 * nn, 0.0);
    in.res_sys.assign(nn, -1);
    in.n_sys = max_slots;
    in.sys_res_begin.assign(max_slots, 0);
    in.sys_res_end.assign(max_slots, 0);
    in.ext_of.assign(max_slots, std::vector<int>());
    in.fm.nd = nd;
    in.fm.row_start.assign((size_t) nn * nd + 1, 0);
    in.fm.uniform = true;
    seeds.assign(max_slots, 0ull);
    server_pending = true;
    setup();
    server_pending = false;
    committed = true;
    // four bond slots per residue: CA-O, CA-CB/HB, CA-CA(+1), O-CA(+1)
    bond_cap = 4;
    bond_i.alloc((size_t) 4 * nn);
    bond_j.alloc((size_t) 4 * nn);
    bond_k.alloc((size_t) 4 * nn);
    bond_r0.alloc((size_t) 4 * nn);
    fill(bond_i, 0, (size_t) 4 * nn, -1);
    // memory-record pool (stripes of 32 records)
    stripe_cap = (cap_records + 31) / 32;
    fm_rf.alloc((size_t) std::max(stripe_cap, 1LL) * 32 * 4);
    if (stripe_cap) free_stripes[0] = stripe_cap;
    free_groups[0] = groups;
    slots.assign(max_slots, Slot());
    srv_rp = awsem_run_params{dt, 1, 300.0, 300.0, damp, 1ull, skin, 0};
    update_launch_extent();
    upload_integrator(make_integrator(srv_rp, step + 1));
    CK(cudaStreamSynchronize(s0));
    release_graphs();  // buffers were reallocated after setup
  }

  // Langevin factors (fix langevin, units real) of atoms [a0, a0 + na) with masses m
  void set_thermostat_factors(int a0, const double *m, int na)
  {
    std::vector<double> h1(na), h2(na);
    for (int a = 0; a < na; a++) {
      h1[a] = -m[a] / srv_rp.damp / FTM2V;
      h2[a] = sqrt(m[a]) * sqrt(24.0 * BOLTZ / srv_rp.damp / srv_rp.dt / MVV2E) / FTM2V;
    }
    put(g1, a0, h1.data(), na);
    put(g2, a0, h2.data(), na);
    CK(cudaStreamSynchronize(s0));
  }

  // A request prepared on the host: its system, the slices of its memory
  // table in the engine's arithmetic type, at local stripe offsets
  struct Prepared {
    SystemInput S;
    std::vector<int> slen, loff;  // [groups][nd] block lengths and first local stripes
    long long stripes = 0;
    int groups = 0;
    std::vector<R> rf, cf;  // [stripes][32][4] distances, [stripes][32] coefficients
  };

  void *prepare_request(const ReplicaArrays &ra) override
  {
    if (!server) throw std::invalid_argument("not a serving handle");
    auto P = std::make_unique<Prepared>();
    SystemInput &S = P->S;
    load_system_arrays(*sf, ra, S);
    const Topology &t = S.top;
    const FMTable &fm = S.fm;
    const int nd = in.ff.p.fm_nd, n = t.n_res, groups = (n + 31) / 32;
    if ((in.ff.p.terms & T_FM) && fm.nd > nd)
      throw std::invalid_argument("memory separations exceed the fragment-memory table of this handle");
    // slices of the request's rows (local groups)
    P->groups = groups;
    P->slen.assign((size_t) groups * std::max(nd, 1), 0);
    P->loff.assign(P->slen.size(), 0);
    long long stripes = 0;
    for (int g = 0; g < groups; g++)
      for (int d = 0; d < fm.nd; d++) {
        int len = 0;
        for (int l = 0; l < 32 && 32 * g + l < n; l++) {
          size_t row = (size_t) (32 * g + l) * fm.nd + d;
          len = std::max(len, fm.row_start[row + 1] - fm.row_start[row]);
        }
        len += len & 1;  // even: the kernels take a row's records in pairs
        P->slen[(size_t) g * nd + d] = len;
        stripes += len;
      }
    P->stripes = stripes;
    if (nd > 0) {
      P->rf.assign((size_t) stripes * 32 * 4, R(FMTable::FM_SKIP));
      P->cf.assign((size_t) stripes * 32, R(0));
      long long at_stripe = 0;
      for (int g = 0; g < groups; g++)
        for (int d = 0; d < nd; d++) {
          const size_t blk = (size_t) g * nd + d;
          P->loff[blk] = (int) at_stripe;
          for (int l = 0; l < 32 && 32 * g + l < n && d < fm.nd; l++) {
            size_t row = (size_t) (32 * g + l) * fm.nd + d;
            for (int m = 0, rec = fm.row_start[row]; rec < fm.row_start[row + 1]; m++, rec++) {
              size_t e = (size_t) (at_stripe + m) * 32 + l;
              for (int k = 0; k < 4; k++) P->rf[e * 4 + k] = (R) fm.rf[(size_t) rec * 4 + k];
              P->cf[e] = (R) (fm.uniform ? fm.uniform_coef : fm.coef[rec]);
            }
          }
          at_stripe += P->slen[blk];
        }
    }
    return P.release();
  }

  static void delete_prepared(void *prep) { delete static_cast<Prepared *>(prep); }
  PreparedDeleter prepared_deleter() const override { return &Engine::delete_prepared; }

  int admit(const ReplicaArrays &ra, unsigned long long seed, long long nsteps, double t_start, double t_stop) override
  {
    if (nsteps < 0) throw std::invalid_argument("nsteps must be >= 0");
    if (t_start < 0 || t_stop < 0) throw std::invalid_argument("temperatures must be >= 0");
    std::unique_ptr<Prepared> P(static_cast<Prepared *>(prepare_request(ra)));
    return admit_prepared(P.get(), seed, nsteps, t_start, t_stop);
  }

  int admit_prepared(void *prep, unsigned long long seed, long long nsteps, double t_start, double t_stop) override
  {
    if (!server) throw std::invalid_argument("not a serving handle");
    if (nsteps < 0) throw std::invalid_argument("nsteps must be >= 0");
    if (t_start < 0 || t_stop < 0) throw std::invalid_argument("temperatures must be >= 0");
    Prepared &P = *static_cast<Prepared *>(prep);
    SystemInput &S = P.S;
    const Topology &t = S.top;
    const FMTable &fm = S.fm;
    const int nd = in.ff.p.fm_nd, n = t.n_res, groups = P.groups;
    const long long stripes = P.stripes;
    const std::vector<int> &slen = P.slen;
    // coefficient mode: a uniform coefficient shared by every request so far,
    // else a per-record coefficient pool
    if ((in.ff.p.terms & T_FM) && fm.records() > 0 && !fm_coef_mode) {
      if (!fm_uniform_known && fm.uniform) {
        in.fm.uniform_coef = fm.uniform_coef;
        fm_uniform_known = true;
        release_graphs();
      } else if (!fm.uniform || fm.uniform_coef != in.fm.uniform_coef) {
        fm_coef_mode = true;
        in.fm.uniform = false;
        fm_coef.alloc((size_t) std::max(stripe_cap, 1LL) * 32);
        fill(fm_coef, 0, (size_t) std::max(stripe_cap, 1LL) * 32, (R) in.fm.uniform_coef);
        release_graphs();
      }
    }
    int slot_id = -1;
    for (int k = 0; k < (int) slots.size(); k++)
      if (!slots[k].used) {
        slot_id = k;
        break;
      }
    long long g0 = 0, st0 = 0;
    if (slot_id < 0 || !take_range(free_groups, groups, g0)) return -1;
    if (!take_range(free_stripes, stripes, st0)) {
      give_range(free_groups, g0, groups);
      return -1;
    }
    const int base = (int) (g0 * 32), N = n_res_cap();
    // topology at residue offset `base`; chain ids are global first residues
    std::vector<int> rc(n), cs(t.n_chains), ce(t.n_chains);
    for (int r = 0; r < n; r++) rc[r] = base + t.chain_start[t.res_chain[r]];
    put(res_type, base, t.res_type.data(), n);
    put(res_flags, base, t.res_flags.data(), n);
    put(res_chain, base, rc.data(), n);
    for (int c = 0; c < t.n_chains; c++) {
      int id = base + t.chain_start[c], a = base + t.chain_start[c], b = base + t.chain_end[c];
      put(chain_start, id, &a, 1);
      put(chain_end, id, &b, 1);
      CK(cudaStreamSynchronize(s0));  // a and b are reused
    }
    for (int k = 0; k < 12; k++) put(aps, (size_t) k * N + base, t.aps.data() + (size_t) k * n, n);
    put(atom_tag, 3 * base, t.atom_tag.data(), 3 * n);
    put(atom_type, 3 * base, t.atom_type.data(), 3 * n);
    put(mass, 3 * base, t.mass.data(), 3 * n);
    put(x, (size_t) 9 * base, S.x.data(), (size_t) 9 * n);
    put(v, (size_t) 9 * base, S.v.data(), (size_t) 9 * n);
    std::vector<unsigned> es(t.excl_self.begin(), t.excl_self.end()), en(t.excl_next.begin(), t.excl_next.end());
    put(excl_self, base, es.data(), n);
    put(excl_next, base, en.data(), n);
    // bonds: slots of the residue of their first atom
    std::vector<int> bi((size_t) 4 * n, -1), bj((size_t) 4 * n, -1), cnt(n, 0);
    std::vector<double> bk((size_t) 4 * n, 0.0), br((size_t) 4 * n, 0.0);
    for (size_t b = 0; b < t.bond_i.size(); b++) {
      int r = t.bond_i[b] / 3;
      if (cnt[r] >= 4) throw std::invalid_argument("more than four bonds start at one residue");
      size_t at = (size_t) 4 * r + cnt[r]++;
      bi[at] = t.bond_i[b] + 3 * base;
      bj[at] = t.bond_j[b] + 3 * base;
      bk[at] = t.bond_k[b];
      br[at] = t.bond_r0[b];
    }
    put(bond_i, (size_t) 4 * base, bi.data(), 4 * n);
    put(bond_j, (size_t) 4 * base, bj.data(), 4 * n);
    put(bond_k, (size_t) 4 * base, bk.data(), 4 * n);
    put(bond_r0, (size_t) 4 * base, br.data(), 4 * n);
    // fragment memory: the request's blocks at stripe st0
    if (nd > 0) {
      std::vector<int> soff((size_t) groups * nd, 0);
      for (size_t blk = 0; blk < soff.size(); blk++) soff[blk] = (int) (st0 + P.loff[blk]);
      put(fm_soff, (size_t) g0 * nd, soff.data(), soff.size());
      put(fm_slen, (size_t) g0 * nd, slen.data(), slen.size());
      put(fm_rf, (size_t) st0 * 32 * 4, P.rf.data(), P.rf.size());
      if (fm_coef_mode) put(fm_coef, (size_t) st0 * 32, P.cf.data(), P.cf.size());
      CK(cudaStreamSynchronize(s0));
    }
    // run window: the next evaluation is this request's setup evaluation
    Slot &sl = slots[slot_id];
    sl.used = true;
    sl.base = base;
    sl.n_res = n;
    sl.groups = groups;
    sl.stripe0 = st0;
    sl.stripes = stripes;
    sl.begin = step + 1;
    sl.end = step + 1 + nsteps;
    dev::SlotRun w{sl.begin, sl.end, sl.begin, t_start, t_stop};
    int b0 = base, b1 = base + n;
    put(slot_run, slot_id, &w, 1);
    put(sys_begin, slot_id, &b0, 1);
    put(sys_end, slot_id, &b1, 1);
    put(sys_seed, slot_id, &seed, 1);
    std::vector<int> rs(n, slot_id);
    put(res_sys, base, rs.data(), n);
    CK(cudaStreamSynchronize(s0));
    set_thermostat_factors(3 * base, t.mass.data(), 3 * n);
    in.sys_res_begin[slot_id] = base;
    in.sys_res_end[slot_id] = base + n;
    in.ext_of[slot_id] = t.ext_of;
    seeds[slot_id] = seed;
    set_nl_field(&dev::NLState::r_list, 0.f);  // the next evaluation rebuilds the pair list
    update_launch_extent();
    return slot_id;
  }

  // Kernels cover residues [0, high-water mark of the used groups), rounded
  // up to 4,096 so that admissions rarely change the launch shapes (which
  // are baked into the step graphs: a change re-captures them).
  void update_launch_extent()
  {
    int hwm = 0;
    for (const Slot &sl : slots)
      if (sl.used) hwm = std::max(hwm, sl.base + 32 * sl.groups);
    int want = std::min(n(), std::max(4096, (hwm + 4095) / 4096 * 4096));
    if (want != launch_res) {
      launch_res = want;
      release_graphs();
    }
  }

  int n_res_cap() const { return in.top.n_res; }

  void check_slot(int k) const
  {
    if (!server) throw std::invalid_argument("not a serving handle");
    if (k < 0 || k >= (int) slots.size() || !slots[k].used) throw std::invalid_argument("no request in this slot");
  }

  void progress(int k, long long *done, long long *total) override
  {
    check_slot(k);
    const Slot &sl = slots[k];
    if (total) *total = sl.end - sl.begin;
    if (done) *done = std::max(0LL, std::min(step, sl.end) - sl.begin);
  }

  void advance(long long nsteps) override
  {
    if (!server) throw std::invalid_argument("not a serving handle");
    if (nsteps <= 0) return;
    if (!graphs[0][0]) capture_steps(graphs[0][0], 1, false);
    if (nsteps >= kChunk && !graphs[0][1]) capture_steps(graphs[0][1], kChunk, false);
    if (!ev_run0) {
      CK(cudaEventCreate(&ev_run0));
      CK(cudaEventCreate(&ev_run1));
    }
    long long done = 0;
    CK(cudaEventRecord(ev_run0, s0));
    while (nsteps - done >= kChunk) {
      CK(cudaGraphLaunch(graphs[0][1], s0));
      done += kChunk;
    }
    while (done < nsteps) {
      CK(cudaGraphLaunch(graphs[0][0], s0));
      done++;
    }
    CK(cudaEventRecord(ev_run1, s0));
    CK(cudaStreamSynchronize(s0));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ev_run0, ev_run1));
    last_run_ms = ms;
    step += nsteps;
    check_list();
  }

  void release(int k) override
  {
    check_slot(k);
    Slot &sl = slots[k];
    const int base = sl.base, n = sl.n_res, N = n_res_cap();
    (void) N;
    fill(res_sys, base, n, -1);
    fill(res_flags, base, n, (int) (R_FIRST | R_LAST));
    fill(res_chain, base, n, -1);
    fill(excl_self, base, n, 0x1ffu);
    fill(excl_next, base, n, 0u);
    fill(bond_i, (size_t) 4 * base, (size_t) 4 * n, -1);
    fill(x, (size_t) 9 * base, (size_t) 9 * n, 0.0);
    fill(v, (size_t) 9 * base, (size_t) 9 * n, 0.0);
    const int nd = in.ff.p.fm_nd;
    if (nd > 0) {
      fill(fm_slen, (size_t) (base / 32) * nd, (size_t) sl.groups * nd, 0);
      fill(fm_soff, (size_t) (base / 32) * nd, (size_t) sl.groups * nd, 0);
    }
    int zero = 0;
    dev::SlotRun w{0, 0, 0, 0.0, 0.0};
    put(sys_begin, k, &zero, 1);
    put(sys_end, k, &zero, 1);
    put(slot_run, k, &w, 1);
    CK(cudaStreamSynchronize(s0));
    give_range(free_groups, base / 32, sl.groups);
    give_range(free_stripes, sl.stripe0, sl.stripes);
    in.sys_res_begin[k] = in.sys_res_end[k] = 0;
    in.ext_of[k].clear();
    sl = Slot();
    set_nl_field(&dev::NLState::r_list, 0.f);
    update_launch_extent();
  }

  void usage(long long *info) override
  {
    if (!server) throw std::invalid_argument("not a serving handle");
    long long active = 0, res = 0, free_st = 0;
    for (const Slot &sl : slots)
      if (sl.used) {
        active++;
        res += 32LL * sl.groups;
      }
    for (auto &kv : free_stripes) free_st += kv.second;
    info[0] = active;
    info[1] = res;
    info[2] = n_res_cap();
    info[3] = 32 * (stripe_cap - free_st);
    info[4] = 32 * stripe_cap;
    info[5] = device_bytes();
    info[6] = step;
    info[7] = (long long) slots.size();
  }

  long long device_bytes() const
  {
    long long b = 0;
    auto add = [&](const auto &buf) { b += (long long) (buf.n * sizeof(*buf.p)); };
    add(res_type), add(res_flags), add(res_chain), add(chain_start), add(chain_end), add(atom_tag), add(atom_type);
    add(aps), add(tables), add(x), add(v), add(mass), add(g1), add(g2), add(ftot), add(work), add(e_res), add(energy);
    add(pos), add(cpos), add(rrec), add(cb_build), add(facc), add(pairs), add(ncount), add(hbq), add(dacc), add(e_fix), add(nl), add(dstep);
    add(ev_pref), add(ev_cs), add(ev_cl), add(excl_self), add(excl_next), add(bond_i), add(bond_j), add(bond_k);
    add(bond_r0), add(fm_soff), add(fm_slen), add(fm_rf), add(fm_coef), add(tb_data), add(tb_present);
    add(go_start), add(go_partner), add(go_rnat), add(go_gamma), add(go_sig_sq), add(go_norm);
    add(go_in), add(lst_x0), add(lst_ago), add(lst_over), add(lst_build), add(charge), add(cr_start), add(cr_j),
        add(cr_w), add(cr_r0), add(zim), add(vfm_start), add(vfm_j), add(vfm_angle);
    add(thermo_rows), add(res_sys), add(sys_begin);
    add(sys_end), add(sys_seed), add(slot_run), add(d_integ);
    return b;
  }
};

}  // namespace awsem

using namespace awsem;

struct awsem_system {
  std::unique_ptr<EngineBase> eng;
  std::unique_ptr<SharedForceField> shared;  // force field of array-described replicas
};

// The caller's current device, put back when an entry point returns (the
// engine makes the handle's device current for its work).
struct DeviceRestore {
  int prev = -1;
  DeviceRestore()
  {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      prev = -1;
      cudaGetLastError();
    }
  }
  ~DeviceRestore()
  {
    int now = -1;
    if (prev >= 0 && cudaGetDevice(&now) == cudaSuccess && now != prev) cudaSetDevice(prev);
  }
};

template <typename Fn> static int guarded(Fn fn)
{
  DeviceRestore restore;
  try {
    fn();
    return AWSEM_OK;
  } catch (CudaError &e) {
    g_last_error = e.what();
    return AWSEM_ECUDA;
  } catch (StateError &e) {
    g_last_error = e.what();
    return AWSEM_ESTATE;
  } catch (std::invalid_argument &e) {
    g_last_error = e.what();
    return AWSEM_EINVAL;
  } catch (std::bad_alloc &) {
    g_last_error = "host allocation failed";
    return AWSEM_ENOMEM;
  } catch (std::runtime_error &e) {
    g_last_error = e.what();
    std::string m = e.what();
    return m.find("overflow") != std::string::npos ? AWSEM_ESTATE : AWSEM_EPARSE;
  } catch (std::exception &e) {
    g_last_error = e.what();
    return AWSEM_EINVAL;
  }
}

extern "C" {

const char *awsem_last_error(void) { return g_last_error.c_str(); }

int awsem_version(void) { return 1; }

int awsem_batch_create(int precision, int device, awsem_system **out)
{
  if (!out) {
    g_last_error = "awsem_batch_create: null argument";
    return AWSEM_EINVAL;
  }
  *out = nullptr;
  if (precision != AWSEM_FP64 && precision != AWSEM_MIXED) {
    g_last_error = "precision must be AWSEM_FP64 or AWSEM_MIXED";
    return AWSEM_EINVAL;
  }
  auto *sys = new awsem_system();
  if (precision == AWSEM_FP64) sys->eng.reset(new Engine<double>());
  else sys->eng.reset(new Engine<float>());
  sys->eng->device = device;
  *out = sys;
  return AWSEM_OK;
}

int awsem_batch_add_files(awsem_system *sys, const char *workdir, const char *data_file, const char *coeff_file,
                          const char *seq_file, const char *pair_style, const char *pair_coeffs,
                          unsigned long long seed, int *replica)
{
  if (!sys || !data_file || !coeff_file || !seq_file || !pair_style) {
    g_last_error = "awsem_batch_add_files: null argument";
    return AWSEM_EINVAL;
  }
  if (sys->eng->committed) {
    g_last_error = "awsem_batch_add_files: the batch is already committed";
    return AWSEM_ESTATE;
  }
  return guarded([&] {
    std::unique_ptr<SystemInput> S(new SystemInput());
    load_system_dir(workdir ? workdir : "", data_file, coeff_file, seq_file, pair_style,
                    pair_coeffs ? pair_coeffs : "", *S);
    sys->eng->reps.push_back(std::move(S));
    sys->eng->seeds.push_back(seed);
    if (replica) *replica = (int) sys->eng->reps.size() - 1;
  });
}

int awsem_batch_set_forcefield(awsem_system *sys, const char *workdir, const char *coeff_file,
                               const char *pair_style, const char *pair_coeffs)
{
  if (!sys || !coeff_file || !pair_style) {
    g_last_error = "awsem_batch_set_forcefield: null argument";
    return AWSEM_EINVAL;
  }
  return guarded([&] {
    sys->shared.reset(new SharedForceField());
    load_shared_forcefield(workdir ? workdir : "", coeff_file, pair_style, pair_coeffs ? pair_coeffs : "",
                           *sys->shared);
  });
}

int awsem_batch_add_replica(awsem_system *sys, const awsem_replica_desc *d, int *replica)
{
  if (!sys || !d) {
    g_last_error = "awsem_batch_add_replica: null argument";
    return AWSEM_EINVAL;
  }
  if (!sys->shared) {
    g_last_error = "awsem_batch_add_replica: call awsem_batch_set_forcefield first";
    return AWSEM_ESTATE;
  }
  if (sys->eng->committed) {
    g_last_error = "awsem_batch_add_replica: the batch is already committed";
    return AWSEM_ESTATE;
  }
  return guarded([&] {
    ReplicaArrays ra{d->n_res, d->n_chains, d->chain_len, d->seq, d->ssweight, d->x, d->v, d->n_mem,
                     d->mem_pos, d->mem_len, d->mem_weight, d->mem_seq, d->mem_ca, d->mem_cb};
    std::unique_ptr<SystemInput> S(new SystemInput());
    load_system_arrays(*sys->shared, ra, *S);
    sys->eng->reps.push_back(std::move(S));
    sys->eng->seeds.push_back(d->seed);
    if (replica) *replica = (int) sys->eng->reps.size() - 1;
  });
}

int awsem_batch_commit(awsem_system *sys)
{
  if (!sys) return AWSEM_EINVAL;
  if (sys->eng->committed) {
    g_last_error = "awsem_batch_commit: already committed";
    return AWSEM_ESTATE;
  }
  if (sys->eng->reps.empty()) {
    g_last_error = "awsem_batch_commit: no replicas";
    return AWSEM_EINVAL;
  }
  return guarded([&] {
    std::vector<unsigned long long> sd = sys->eng->seeds;
    sys->eng->commit();
    sys->eng->seeds = sd;
  });
}

int awsem_create_from_files(const char *workdir, const char *data_file, const char *coeff_file, const char *seq_file,
                            const char *pair_style, const char *pair_coeffs, int precision, int device,
                            awsem_system **out)
{
  int rc = awsem_batch_create(precision, device, out);
  if (rc != AWSEM_OK) return rc;
  rc = awsem_batch_add_files(*out, workdir, data_file, coeff_file, seq_file, pair_style, pair_coeffs, 0ull, nullptr);
  if (rc == AWSEM_OK) rc = awsem_batch_commit(*out);
  if (rc != AWSEM_OK) {
    std::string msg = g_last_error;
    delete *out;
    *out = nullptr;
    g_last_error = msg;
  }
  return rc;
}

int awsem_create_from_atoms(const char *workdir, const char *coeff_file, const char *seq_file, int natoms,
                            const int *role, const int *residue, const int *molecule, const int *type, const int *tag,
                            const double *mass_by_type, int ntypes, const double *x, int nbonds, const int *bond_a,
                            const int *bond_b, const double *bond_k, const double *bond_r0, const char *pair_style,
                            const char *pair_coeffs, int precision, int device, awsem_system **out)
{
  if (!out || (!coeff_file) != (!seq_file) || natoms <= 0 || !role || !residue || !molecule || !type || !tag ||
      !mass_by_type || (nbonds > 0 && (!bond_a || !bond_b || !bond_k || !bond_r0))) {
    g_last_error = "awsem_create_from_atoms: null or empty argument";
    return AWSEM_EINVAL;
  }
  int rc = awsem_batch_create(precision, device, out);
  if (rc != AWSEM_OK) return rc;
  rc = guarded([&] {
    std::unique_ptr<SystemInput> S(new SystemInput());
    load_system_atoms(workdir ? workdir : "", coeff_file ? coeff_file : "", seq_file ? seq_file : "", natoms, role,
                      residue, molecule, type, tag,
                      mass_by_type, ntypes, x, nullptr, std::max(nbonds, 0), bond_a, bond_b, bond_k, bond_r0,
                      pair_style ? pair_style : "2 3.5 3.5", pair_coeffs ? pair_coeffs : "", *S, true);
    (*out)->eng->reps.push_back(std::move(S));
    (*out)->eng->seeds.push_back(0ull);
  });
  if (rc == AWSEM_OK) rc = awsem_batch_commit(*out);
  if (rc != AWSEM_OK) {
    std::string msg = g_last_error;
    delete *out;
    *out = nullptr;
    g_last_error = msg;
  }
  return rc;
}

void awsem_destroy(awsem_system *sys) { delete sys; }

static bool ready(const awsem_system *sys)
{
  if (!sys || !sys->eng->committed) {
    g_last_error = "handle is null or not committed";
    return false;
  }
  return true;
}

int awsem_natoms(const awsem_system *sys) { return ready(sys) ? sys->eng->in.top.n_atoms : 0; }
int awsem_nres(const awsem_system *sys) { return ready(sys) ? sys->eng->in.top.n_res : 0; }
int awsem_nreplicas(const awsem_system *sys) { return ready(sys) ? sys->eng->in.n_sys : 0; }
int awsem_replica_natoms(const awsem_system *sys, int r)
{
  return ready(sys) && r >= 0 && r < sys->eng->in.n_sys ? sys->eng->rep_atoms(r) : 0;
}
int awsem_replica_nres(const awsem_system *sys, int r)
{
  return ready(sys) && r >= 0 && r < sys->eng->in.n_sys ? sys->eng->rep_res(r) : 0;
}
long long awsem_step(const awsem_system *sys) { return sys ? sys->eng->step : 0; }

int awsem_compute(awsem_system *sys, long long step, const double *x, double *f, double *energies, int terms)
{
  if (!ready(sys) || !x || !f) {
    g_last_error = "awsem_compute: null argument or uncommitted handle";
    return AWSEM_EINVAL;
  }
  if (terms <= 0 || terms > AWSEM_TERMS_ALL) {
    g_last_error = "awsem_compute: terms must be a non-empty set of AWSEM_TERMS_* bits";
    return AWSEM_EINVAL;
  }
  return guarded([&] { sys->eng->compute(step, x, f, energies, terms); });
}

int awsem_replica_set_state(awsem_system *sys, int r, const double *x, const double *v)
{
  if (!ready(sys)) return AWSEM_EINVAL;
  return guarded([&] { sys->eng->set_state(r, x, v); });
}

int awsem_replica_get_state(awsem_system *sys, int r, double *x, double *v)
{
  if (!ready(sys)) return AWSEM_EINVAL;
  return guarded([&] { sys->eng->get_state(r, x, v); });
}

int awsem_batch_set_state(awsem_system *sys, const double *x, const double *v)
{
  if (!ready(sys)) return AWSEM_EINVAL;
  return guarded([&] { sys->eng->set_state_all(x, v); });
}

int awsem_batch_get_state(awsem_system *sys, double *x, double *v)
{
  if (!ready(sys)) return AWSEM_EINVAL;
  return guarded([&] { sys->eng->get_state_all(x, v); });
}

int awsem_replica_energies(awsem_system *sys, int r, double *energies)
{
  if (!ready(sys) || !energies) return AWSEM_EINVAL;
  return guarded([&] { sys->eng->energies(r, energies); });
}

int awsem_replica_forces(awsem_system *sys, int r, double *f)
{
  if (!ready(sys) || !f) return AWSEM_EINVAL;
  return guarded([&] { sys->eng->forces(r, f); });
}

int awsem_set_state(awsem_system *sys, const double *x, const double *v) { return awsem_replica_set_state(sys, 0, x, v); }
int awsem_get_state(awsem_system *sys, double *x, double *v) { return awsem_replica_get_state(sys, 0, x, v); }
int awsem_energies(awsem_system *sys, double *energies) { return awsem_replica_energies(sys, 0, energies); }
int awsem_forces(awsem_system *sys, double *f) { return awsem_replica_forces(sys, 0, f); }

int awsem_run_window(awsem_system *sys, long long nsteps, const awsem_run_params *rp, long long window_begin,
                     long long window_end, int cont, double *thermo)
{
  if (!ready(sys) || !rp) {
    g_last_error = "awsem_run_window: null argument or uncommitted handle";
    return AWSEM_EINVAL;
  }
  if (rp->dt <= 0 || rp->damp <= 0 || (rp->langevin && (rp->t_start < 0 || rp->t_stop < 0))) {
    g_last_error = "awsem_run_window: dt and damp must be positive, temperatures non-negative";
    return AWSEM_EINVAL;
  }
  if (sys->eng->server) {
    g_last_error = "awsem_run_window: a serving handle advances with awsem_server_advance";
    return AWSEM_EINVAL;
  }
  return guarded([&] { sys->eng->run_window(nsteps, *rp, window_begin, window_end, cont != 0, thermo); });
}

int awsem_run(awsem_system *sys, long long nsteps, const awsem_run_params *rp, double *thermo)
{
  if (!ready(sys) || !rp) {
    g_last_error = "awsem_run: null argument or uncommitted handle";
    return AWSEM_EINVAL;
  }
  if (rp->dt <= 0 || rp->damp <= 0 || (rp->langevin && (rp->t_start < 0 || rp->t_stop < 0))) {
    g_last_error = "awsem_run: dt and damp must be positive, temperatures non-negative";
    return AWSEM_EINVAL;
  }
  if (sys->eng->server) {
    g_last_error = "awsem_run: a serving handle advances with awsem_server_advance";
    return AWSEM_EINVAL;
  }
  return guarded([&] { sys->eng->run(nsteps, *rp, thermo); });
}

// --------------------------------------------------------------------------
// Serving

int awsem_server_create(const char *workdir, const char *coeff_file, const char *pair_style, const char *pair_coeffs,
                        int precision, int device, long long max_residues, int max_requests,
                        long long max_memory_records, double dt, double damp, awsem_system **out)
{
  if (!out || !coeff_file || !pair_style) {
    g_last_error = "awsem_server_create: null argument";
    return AWSEM_EINVAL;
  }
  int rc = awsem_batch_create(precision, device, out);
  if (rc != AWSEM_OK) return rc;
  rc = awsem_batch_set_forcefield(*out, workdir, coeff_file, pair_style, pair_coeffs);
  if (rc == AWSEM_OK) {
    awsem_system *sys = *out;
    rc = guarded([&] {
      CK(cudaSetDevice(sys->eng->device));
      sys->eng->server_setup(*sys->shared, max_residues, max_requests, max_memory_records, dt, damp);
    });
  }
  if (rc != AWSEM_OK) {
    std::string keep = g_last_error;
    awsem_destroy(*out);
    *out = nullptr;
    g_last_error = keep;
  }
  return rc;
}

static bool serving(const awsem_system *sys, const char *what)
{
  if (!sys || !sys->eng->server) {
    g_last_error = std::string(what) + ": not a serving handle";
    return false;
  }
  return true;
}

int awsem_server_admit(awsem_system *sys, const awsem_replica_desc *d, long long nsteps, double t_start,
                       double t_stop, int *slot)
{
  if (!serving(sys, "awsem_server_admit")) return AWSEM_EINVAL;
  if (!d) {
    g_last_error = "awsem_server_admit: null request";
    return AWSEM_EINVAL;
  }
  int got = -1;
  int rc = guarded([&] {
    CK(cudaSetDevice(sys->eng->device));
    ReplicaArrays ra{d->n_res, d->n_chains, d->chain_len, d->seq, d->ssweight, d->x, d->v, d->n_mem,
                     d->mem_pos, d->mem_len, d->mem_weight, d->mem_seq, d->mem_ca, d->mem_cb};
    got = sys->eng->admit(ra, d->seed, nsteps, t_start, t_stop);
  });
  if (rc != AWSEM_OK) return rc;
  if (got < 0) {
    g_last_error = "awsem_server_admit: no free slot, residue range or memory-record room now";
    return AWSEM_EBUSY;
  }
  if (slot) *slot = got;
  return AWSEM_OK;
}

// A request prepared on the host for one serving handle
struct awsem_request {
  const EngineBase *eng;  // the handle it was prepared for
  void *prep;
  EngineBase::PreparedDeleter del;
  unsigned long long seed;
};

int awsem_server_prepare(awsem_system *sys, const awsem_replica_desc *d, awsem_request **out)
{
  if (!serving(sys, "awsem_server_prepare")) return AWSEM_EINVAL;
  if (!d || !out) {
    g_last_error = "awsem_server_prepare: null request or output";
    return AWSEM_EINVAL;
  }
  *out = nullptr;
  return guarded([&] {
    ReplicaArrays ra{d->n_res, d->n_chains, d->chain_len, d->seq, d->ssweight, d->x, d->v, d->n_mem,
                     d->mem_pos, d->mem_len, d->mem_weight, d->mem_seq, d->mem_ca, d->mem_cb};
    void *prep = sys->eng->prepare_request(ra);
    *out = new awsem_request{sys->eng.get(), prep, sys->eng->prepared_deleter(), d->seed};
  });
}

int awsem_server_admit_prepared(awsem_system *sys, awsem_request *req, long long nsteps, double t_start,
                                double t_stop, int *slot)
{
  if (!serving(sys, "awsem_server_admit_prepared")) return AWSEM_EINVAL;
  if (!req || req->eng != sys->eng.get()) {
    g_last_error = "awsem_server_admit_prepared: the request was not prepared for this handle";
    return AWSEM_EINVAL;
  }
  int got = -1;
  int rc = guarded([&] {
    CK(cudaSetDevice(sys->eng->device));
    got = sys->eng->admit_prepared(req->prep, req->seed, nsteps, t_start, t_stop);
  });
  if (rc != AWSEM_OK) return rc;
  if (got < 0) {
    g_last_error = "awsem_server_admit_prepared: no free slot, residue range or memory-record room now";
    return AWSEM_EBUSY;
  }
  if (slot) *slot = got;
  return AWSEM_OK;
}

void awsem_request_free(awsem_request *req)
{
  if (!req) return;
  req->del(req->prep);
  delete req;
}

int awsem_server_advance(awsem_system *sys, long long nsteps)
{
  if (!serving(sys, "awsem_server_advance")) return AWSEM_EINVAL;
  return guarded([&] {
    CK(cudaSetDevice(sys->eng->device));
    sys->eng->advance(nsteps);
  });
}

int awsem_server_progress(awsem_system *sys, int slot, long long *done, long long *total)
{
  if (!serving(sys, "awsem_server_progress")) return AWSEM_EINVAL;
  return guarded([&] { sys->eng->progress(slot, done, total); });
}

int awsem_server_collect(awsem_system *sys, int slot, double *x, double *v, double *energies)
{
  if (!serving(sys, "awsem_server_collect")) return AWSEM_EINVAL;
  return guarded([&] {
    CK(cudaSetDevice(sys->eng->device));
    long long done = 0, total = 0;
    sys->eng->progress(slot, &done, &total);
    if (done < total) throw std::invalid_argument("awsem_server_collect: the request has not finished");
    if (x || v) sys->eng->get_state(slot, x, v);
    if (energies) sys->eng->energies(slot, energies);
    sys->eng->release(slot);
  });
}

int awsem_server_usage(awsem_system *sys, long long *info)
{
  if (!serving(sys, "awsem_server_usage") || !info) return AWSEM_EINVAL;
  return guarded([&] { sys->eng->usage(info); });
}

int awsem_residue_arrays(awsem_system *sys, double *out)
{
  if (!ready(sys) || !out) return AWSEM_EINVAL;
  return guarded([&] { sys->eng->residue_arrays(0, out); });
}

int awsem_debug_selections(awsem_system *sys, long long step, const double *x, unsigned long long *keys,
                           long long cap, long long *count)
{
  if (!ready(sys) || !x || (cap > 0 && !keys) || !count) return AWSEM_EINVAL;
  long long got = 0;
  int rc = guarded([&] { got = sys->eng->debug_selections(step, x, keys, cap); });
  *count = got;
  if (rc == AWSEM_OK && got > cap) {
    g_last_error = "selection records exceed the capacity given (" + std::to_string(cap) + " < " +
                   std::to_string(got) + ")";
    return AWSEM_ESTATE;
  }
  return rc;
}

int awsem_neighbor_stats(awsem_system *sys, int *nbuilds, double *radius, int *max_count, int *overflow)
{
  if (!ready(sys)) return AWSEM_EINVAL;
  return guarded([&] { sys->eng->nl_stats(nbuilds, radius, max_count, overflow); });
}

double awsem_last_run_ms(const awsem_system *sys) { return sys ? sys->eng->run_ms() : 0.0; }

const char *awsem_kernel_name(int k) { return (k >= 0 && k < AWSEM_NKERNELS) ? kKernelNames[k] : ""; }

int awsem_profile_step(awsem_system *sys, int reps, double *ms)
{
  if (!ready(sys) || !ms) return AWSEM_EINVAL;
  return guarded([&] { sys->eng->profile(reps, ms); });
}

int awsem_autotune(awsem_system *sys, int reps, int *chosen)
{
  if (!ready(sys)) return AWSEM_EINVAL;
  return guarded([&] {
    CK(cudaSetDevice(sys->eng->device));
    sys->eng->autotune(reps, chosen);
  });
}

int awsem_set_step_form(awsem_system *sys, int form, int blocks, int stream_warps)
{
  if (!ready(sys)) return AWSEM_EINVAL;
  return guarded([&] {
    CK(cudaSetDevice(sys->eng->device));
    sys->eng->set_step_form(form, blocks, stream_warps);
  });
}

int awsem_set_neighbor(awsem_system *sys, double skin, int delay, int every, int check)
{
  if (!ready(sys)) return AWSEM_EINVAL;
  return guarded([&] { sys->eng->set_neighbor(skin, delay, every, check); });
}

int awsem_q_create(awsem_system *sys, int rep, const char *words, int *qid)
{
  if (!ready(sys) || !words || !qid) return AWSEM_EINVAL;
  return guarded([&] { *qid = sys->eng->q_create(rep, words); });
}

int awsem_q_value(awsem_system *sys, int qid, double *value)
{
  if (!ready(sys) || !value) return AWSEM_EINVAL;
  return guarded([&] { *value = sys->eng->q_value(qid); });
}

int awsem_set_wait_limits(awsem_system *sys, long long fm_copy_wait_cycles, long long grid_barrier_wait_cycles,
                          int hold)
{
  if (!ready(sys)) return AWSEM_EINVAL;
  return guarded([&] { sys->eng->set_wait_limits(fm_copy_wait_cycles, grid_barrier_wait_cycles, hold); });
}

int awsem_set_list_built(awsem_system *sys, int built)
{
  if (!ready(sys) || (built != 0 && built != 1)) return AWSEM_EINVAL;
  return guarded([&] { sys->eng->set_list_built(built); });
}

int awsem_set_launch_shapes(awsem_system *sys, const int *shapes)
{
  if (!ready(sys) || !shapes) return AWSEM_EINVAL;
  return guarded([&] { sys->eng->set_launch_shapes(shapes); });
}

int awsem_get_step_form(awsem_system *sys, int *form)
{
  if (!ready(sys) || !form) return AWSEM_EINVAL;
  return guarded([&] { sys->eng->get_step_form(form); });
}

int awsem_model_info(awsem_system *sys, long long *info)
{
  if (!ready(sys) || !info) return AWSEM_EINVAL;
  return guarded([&] { sys->eng->model_info(info); });
}

int awsem_fragmem_noalloc(awsem_system *sys, const double *d_x, double *d_f, double *d_energy, void *stream)
{
  if (!ready(sys) || !d_x || !d_f || !d_energy) {
    g_last_error = "awsem_fragmem_noalloc: null argument or uncommitted handle";
    return AWSEM_EINVAL;
  }
  return guarded([&] {
    CK(cudaSetDevice(sys->eng->device));
    fragmem_noalloc(sys->eng->device, sys->eng->fm_view(), d_x, d_f, d_energy, (cudaStream_t) stream);
  });
}

}  // extern "C"
