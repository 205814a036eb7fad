// Persistent step kernel: one cooperative launch per MD step.
//
// The passes of awsem_kernels.cuh run inside one kernel whose blocks are all
// resident (cooperative launch), separated by a grid barrier instead of a
// kernel boundary:
//
//   all warps      prepare | barrier (+ list decision) | ......... | barrier | finish
//   pass warps               [build | barrier] density | b | residue | b |
//                            water_xi | b | pair | b | hbond | fragment memory left over
//   stream warps             fragment-memory units from the first barrier on
//
// The last `stream_warps` warps of every block stream fragment-memory work
// units (HBM-bound) while the other warps run the pair passes (latency- and
// atomic-bound), so the two kinds of work share every SM at the same time.
// Units are taken from a global counter, by the stream warps from the start
// and by the pass warps once the hydrogen-bond pass is done, so neither side
// waits for the other.  All sums are fixed-point, so the result is the
// multi-kernel step's bit for bit, whoever evaluates a unit.
//
// Barrier waits are bounded: a wait that gives up (about a second) sets
// GridBar::timeout, and that block skips the rest of its work while still
// arriving at the later barriers without waiting.  Barrier sites have their
// own counters, so no barrier opens before every block has arrived at it and
// no pass ever overlaps the one before it.  The host reports the launch as
// invalid and clears the barrier state.
#pragma once

#include "awsem_kernels.cuh"

namespace awsem {
namespace dev {

// Barrier state of the persistent kernel.  Each barrier site j of the kernel
// has its own arrival counter and release word, so a block that gave up a
// wait and ran on can only arrive early at a LATER site: no barrier ever
// opens before every block has arrived at it.
constexpr int kBarSites = 8;
struct GridBar {
  unsigned arrive[kBarSites];  // blocks arrived at site j in the current launch (0 between launches)
  unsigned rel[kBarSites];     // site j released (incremented once per launch)
  int timeout;                 // a barrier wait gave up: results of the launch are invalid
  int fm_next;                 // next fragment-memory work unit of the step
};

constexpr long long kBarWaitLimit = 2000000000LL;  // about one second at 2 GHz
constexpr int kStepThreads = 256;                  // 8 warps per block

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int ld_volatile(const int *p) { return *(const volatile int *) p; }

// arrival: acquire the earlier arrivals' writes, release this block's
__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned *p, unsigned v)
{
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

__device__ __forceinline__ void red_add_release(unsigned *p, unsigned v)
{
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void st_relaxed(unsigned *p, unsigned v)
{
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// block-level barrier of the first `nthreads` threads (named barrier `id`)
__device__ __forceinline__ void named_sync(int id, int nthreads)
{
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Grid barrier at site j among the first `nthreads` threads of every block
// (named barrier `id` inside the block).  The block's threads meet at the
// named barrier; thread 0 then arrives with an acquire-release add (carrying
// the block's writes, ordered before it by the named barrier).  The last
// block to arrive runs `serial()`, with every block's earlier writes
// visible, clears the site's counter for the next launch and releases the
// others by a release add on the site's word, which they poll with acquire
// loads against `seen` (the word's value read at launch start: it cannot
// change before this block arrives).  A block with ok == false (an earlier
// wait gave up) still arrives but does not wait.  Returns the block's ok.
template <class Serial>
__device__ __forceinline__ bool grid_sync(GridBar *b, int j, unsigned seen, int id, int nthreads, bool ok,
                                          long long limit, unsigned hold, Serial serial)
{
  __shared__ int s_ok;
  named_sync(id, nthreads);
  if (threadIdx.x == 0) {
    const unsigned prev = atom_add_acq_rel(&b->arrive[j], 1u);
    if (prev == gridDim.x - 1 + hold) {  // hold 1 (tests): no block is the last, every wait runs out
      serial();
      st_relaxed(&b->arrive[j], 0u);  // ordered before the release below
      red_add_release(&b->rel[j], 1u);
    } else if (ok) {
      const long long t0 = clock64();
      for (unsigned it = 1; ld_acquire(&b->rel[j]) == seen; it++)
        if ((it & 63u) == 0 && clock64() - t0 > limit) {  // the clock is read every 64th poll
          atomicExch(&b->timeout, 1);
          ok = false;
          break;
        }
    }
    s_ok = ok;
  }
  named_sync(id, nthreads);
  return s_ok;
}

struct NoSerial {
  __device__ void operator()() const {}
};

struct PersistArgs {
  const Integrator *integ;
  const double *g1, *g2;
  double *ftot, *x_out;
  GridBar *bar;
  int n_launch;      // residues the list build covers
  int stream_warps;  // fragment-memory stream warps per block (the last ones); 1..7
  int ring_warps;    // warps with a shared-memory copy ring (the last ones); the others load into registers
  int fm_units;      // fragment-memory work units of the step (0: term off)
  int fm_table;      // table fragment memory on
  int amh_go;        // AMH-Go on
  int pair_extra;    // solvent barrier, Debye-Hueckel or contact restraints on
  int list_reps;     // replicas whose LAMMPS lists are emulated (0: none)
  int residue_extra; // Shake or the membrane potential on
  long long bar_wait_limit;  // SM clock cycles a block waits at a grid barrier before it gives up
  unsigned hold;             // 0, or 1 (tests of the give-up path): the barriers wait for one block too many
};

// Fragment-memory units taken from the step's counter until none is left
// (or a copy wait gave up, which the unit records).
template <typename R>
__device__ __forceinline__ void fragmem_take_units(const StepArgs<R> &a, const FFParams &p, const PersistArgs &q,
                                                   bool ring, unsigned char *wsm, unsigned &kbase)
{
  const BeadPos<R> pos{&a.s};
  unsigned long long *e_acc = (unsigned long long *) (a.e_fix + (size_t) 2 * a.s.n_res);
  const int lane = threadIdx.x & 31;
  while (true) {
    int u = 0;
    if (lane == 0) u = atomicAdd(&q.bar->fm_next, 1);
    u = __shfl_sync(0xffffffffu, u, 0);
    if (u >= q.fm_units) return;
    if (ring) {
      if (!fragmem_unit_bulk(u, a.fm, p.fm_sigma_sq, a.s.n_res, pos, a.s.facc, e_acc, 1, &a.nl->fm_timeout, wsm,
                             kbase))
        return;
    } else {
      fragmem_unit_reg(u, a.fm, p.fm_sigma_sq, a.s.n_res, pos, a.s.facc, e_acc, 1);
    }
  }
}

// Serial part of the first barrier: the list decision of the step (and the
// step counter), and the fragment-memory unit counter.
struct FirstSerial {
  NLState *nl;
  long long *step;
  GridBar *bar;
  __device__ void operator()() const
  {
    nl_decide(nl, 0, step);
    bar->fm_next = 0;
  }
};

// dynamic shared memory: ring_warps copy rings of fm_warp_smem<R>(coef) bytes
template <typename R> __global__ void __launch_bounds__(kStepThreads, 2) k_step(StepArgs<R> a, FFParams p, PersistArgs q)
{
  extern __shared__ __align__(128) unsigned char step_smem[];
  const int warp = threadIdx.x >> 5, nwarps = kStepThreads / 32;
  const int pass_threads = (nwarps - q.stream_warps) * 32;
  GridBar *const b = q.bar;
  unsigned seen[7] = {0, 0, 0, 0, 0, 0, 0};  // release words at launch start (thread 0)
  if (threadIdx.x == 0)
    for (int j = 0; j < 7; j++) seen[j] = ld_acquire(&b->rel[j]);
  const bool ring = q.fm_units > 0 && warp >= nwarps - q.ring_warps;
  unsigned char *wsm = ring ? step_smem + (size_t) (warp - (nwarps - q.ring_warps)) * fm_warp_smem<R>(a.fm.coef != nullptr)
                            : nullptr;
  if (ring) fragmem_ring_init(wsm);
  unsigned kbase = 0;

  const Span all{(int) (blockIdx.x * kStepThreads + threadIdx.x), (int) (gridDim.x * kStepThreads)};
  prepare_pass(a, p, all);
  bool ok = grid_sync(b, 0, seen[0], 0, kStepThreads, true, q.bar_wait_limit, q.hold, FirstSerial{a.nl, a.step, b});
  if ((int) threadIdx.x >= pass_threads) {
    if (ok) fragmem_take_units(a, p, q, ring, wsm, kbase);
  } else {
    const Span sp{(int) (blockIdx.x * pass_threads + threadIdx.x), (int) (gridDim.x * pass_threads)};
    // the emulated lists' decision (read after the next barrier)
    if (ok)
      for (int r = sp.t; r < q.list_reps; r += sp.nthr)
        list_decide_one(*a.nl, a.lst_ago, a.lst_over, const_cast<int *>(a.lst_build), r);
    if (a.nl->rebuild) {
      if (ok) nl_build_pass(a, GridArgs{}, q.n_launch, sp);
      ok = grid_sync(b, 1, seen[1], 1, pass_threads, ok, q.bar_wait_limit, q.hold, NoSerial{});
    }
    if (ok) density_pass(a, p, sp);
    ok = grid_sync(b, 2, seen[2], 1, pass_threads, ok, q.bar_wait_limit, q.hold, NoSerial{});
    if (ok) residue_pass(a, p, sp);
    ok = grid_sync(b, 3, seen[3], 1, pass_threads, ok, q.bar_wait_limit, q.hold, NoSerial{});
    if (ok) water_xi_pass(a, p, sp);
    ok = grid_sync(b, 4, seen[4], 1, pass_threads, ok, q.bar_wait_limit, q.hold, NoSerial{});
    if (ok) {
      radial_pass(a, p, sp);
      pair_pass(a, p, sp);
    }
    ok = grid_sync(b, 5, seen[5], 1, pass_threads, ok, q.bar_wait_limit, q.hold, NoSerial{});
    if (ok) {
      hbond_pass(a, p, sp);
      if (q.fm_table) fm_table_pass(a, p, sp);
      if (q.amh_go) amh_go_pass(a, p, sp);
      if (q.pair_extra) pair_extra_pass(a, p, sp);
      if (q.residue_extra) residue_extra_pass(a, p, sp);
      fragmem_take_units(a, p, q, ring, wsm, kbase);
    }
  }
  // thread 0 (a pass thread) carries the block's state into the last barrier
  ok = grid_sync(b, 6, seen[6], 0, kStepThreads, ok, q.bar_wait_limit, q.hold, NoSerial{});
  if (ok) finish_pass(a, q.integ, q.g1, q.g2, q.ftot, q.x_out, all);
}

}  // namespace dev
}  // namespace awsem
