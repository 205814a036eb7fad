/* Serial MD host for the reference AWSEM plugins (oracle; test infrastructure).

   Hosts the reference `FixBackbone` and `PairExcludedVolume` classes, compiled
   unmodified from the reference sources against the LAMMPS-API shim, inside a
   minimal LAMMPS-like step loop, and exposes them through a small C ABI that
   the tests and the CPU baseline load with ctypes.

   What LAMMPS would supply and the reference does not vendor is restated here
   from the LAMMPS documentation:
     - `read_data` for atom_style awsemmd (`id molecule residue type q x y z`,
       the Atoms line declared at atom_vec_awsemmd.cpp:56), Masses, Velocities,
       Bonds, Bond Coeffs;
     - half neighbour lists (one per request, cutoff = requested cutoff +
       skin) with `special_bonds fene` semantics: 1-2 bonded pairs are dropped,
       1-3 and 1-4 pairs kept with weight 1;
     - `bond_style harmonic`: E = K (r - r0)^2;
     - `fix nve` velocity Verlet and `fix langevin` (uniform noise variant),
       units real;
     - the Verlet::setup / Verlet::run call order around the fix hooks
       (post_neighbor, pre_force, pair, bond, post_force, final_integrate).
   The one deliberate change: the Langevin noise comes from a counter-based
   generator keyed by (seed, step, atom tag, component) instead of LAMMPS's
   sequential RanMars stream, so the GPU engine can draw the same numbers.

   Built with AWSEM_GPU_FIX, the host can also run the GPU adapter `fix
   backbone/gpu` (awsemmd_b200/lammps) in place of the reference fix, through
   the same LAMMPS fix hooks (ref_create_gpufix). */
#include "lmp_shim.h"
#include "fix_backbone.h"
#ifdef AWSEM_GPU_FIX
#include "fix_backbone_gpu.h"
#include "pair_excluded_volume_gpu.h"
#endif
#include "pair_excluded_volume.h"
#include "compute_q_onuchic.h"
#include "compute_q_wolynes.h"
#include "atom_vec_awsemmd.h"

#include <unistd.h>
#include <cmath>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>
#include <algorithm>
#include <cstdint>

using namespace LAMMPS_NS;

namespace {

/* units real (LAMMPS `units` documentation) */
const double BOLTZ_REAL = 0.0019872067;
const double MVV2E_REAL = 48.88821291 * 48.88821291;
const double FTM2V_REAL = 1.0 / 48.88821291 / 48.88821291;

/* Counter-based uniform in [0,1): SplitMix64 finaliser (Steele et al. 2014). */
inline uint64_t mix64(uint64_t z)
{
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
inline double uniform01(uint64_t seed, int64_t step, int64_t tag, int comp)
{
  uint64_t key = mix64(seed ^ mix64((uint64_t) step));
  uint64_t r = mix64(key ^ ((uint64_t) tag * 4ULL + (uint64_t) comp));
  return (double) (r >> 11) * (1.0 / 9007199254740992.0);
}

struct Cwd {
  char old[4096];
  bool ok;
  explicit Cwd(const std::string &dir)
  {
    ok = getcwd(old, sizeof old) != nullptr;
    if (!dir.empty() && chdir(dir.c_str()) != 0) throw std::runtime_error("cannot chdir to " + dir);
  }
  ~Cwd()
  {
    if (ok && chdir(old) != 0) { /* nothing sensible to do */
    }
  }
};

std::vector<std::string> split_ws(const std::string &s)
{
  std::istringstream is(s);
  std::vector<std::string> out;
  std::string t;
  while (is >> t) out.push_back(t);
  return out;
}

}  // namespace

/* Read access to private members of the reference's classes, for
   ref_touches: an explicit instantiation may name a private member
   ([temp.explicit]: access checking does not apply to the names in an
   explicit instantiation), so the reference sources stay unmodified. */
template <typename Tag, typename Tag::type M> struct Expose {
  friend typename Tag::type get(Tag) { return M; }
};
#define EXPOSE(NAME, CLASS, TYPE, MEMBER)         \
  struct NAME {                                    \
    typedef TYPE CLASS::*type;                     \
    friend type get(NAME);                         \
  };                                               \
  template struct Expose<NAME, &CLASS::MEMBER>;
typedef cWell<double, FixBackbone> WellT;
typedef cR<double, FixBackbone> RT;
typedef cP_AP<double, FixBackbone> PapT;
EXPOSE(FbWell, FixBackbone, WellT *, well)
EXPOSE(FbHWell, FixBackbone, WellT *, helix_well)
EXPOSE(FbR, FixBackbone, RT *, R)
EXPOSE(FbPap, FixBackbone, PapT *, p_ap)
EXPOSE(WellG, WellT, int ***, gTheta)
EXPOSE(WellN, WellT, int, n)
EXPOSE(WellM, WellT, int, m)
EXPOSE(WellNW, WellT, int, nw)
EXPOSE(RGNO, RT, int **, gNO)
EXPOSE(RGHO, RT, int **, gHO)
EXPOSE(RN, RT, int, n)
EXPOSE(RM, RT, int, m)
EXPOSE(PapG, PapT, int **, g)
EXPOSE(PapN, PapT, int, n)
EXPOSE(PapM, PapT, int, m)
#undef EXPOSE

struct RefHost {
  LAMMPS *lmp = nullptr;
  Fix *fix = nullptr;
  FixBackbone *fb = nullptr;  // the reference fix (null when the GPU adapter is hosted)
  Pair *pair = nullptr;
  std::string workdir;

  int natoms = 0, ntypes = 0, nbondtypes = 0;
  std::vector<double> mass;  // by type, 1-based
  std::vector<int> bond_t, bond_a, bond_b;
  std::vector<double> bond_k, bond_r0;
  std::vector<std::vector<int>> special;  // 1-2 partners (local indices)

  NeighList fixlist, pairlist, fixfull;
  double fix_cut = 0.0, pair_cut = 0.0;
  bool want_full = false;  // the fix asked for a full list too (AMH-Go)
  double skin = 2.0;
  int every = 1, delay = 0, check = 1;
  bigint last_build = 0;
  std::vector<double> xhold;
  long nbuilds = 0;

  double e_pair = 0.0, e_bond = 0.0;
  bool setup_done = false;

  // Langevin
  int langevin = 0;
  double t_start = 300.0, t_stop = 300.0, t_period = 100.0;
  uint64_t seed = 1;

  ~RefHost()
  {
    delete fix;  // writes timer.log into the workdir through its open handle
    delete pair;
    if (lmp) {
      Atom *a = lmp->atom;
      lmp->memory->destroy(a->x);
      lmp->memory->destroy(a->v);
      lmp->memory->destroy(a->f);
      if (a->nspecial) lmp->memory->destroy(a->nspecial);
      if (a->special) lmp->memory->destroy(a->special);
      free(a->tag);
      free(a->type);
      free(a->mask);
      free(a->image);
      free(a->molecule);
      free(a->residue);
      free(a->mass);
      delete (AtomVecAWSEM *) a->avec;
      free(lmp->update->integrate_style);
      delete lmp;
    }
  }

  // term k of the fix's energy vector (0: total)
  double fix_energy(int k) { return fb ? fb->energy[k] : (k ? fix->compute_vector(k - 1) : fix->compute_scalar()); }

  void read_data(const std::string &path);
  void build_lists();
  void build_one(NeighList &list, double cut, bool full);
  bool need_rebuild(bigint step);
  void force_clear();
  void compute_bonds();
  void langevin_force();
  double kinetic();
  void forces(bool setup);
};

void RefHost::read_data(const std::string &path)
{
  std::ifstream in(path);
  if (!in) throw std::runtime_error("cannot open data file " + path);
  std::string line;
  Atom *a = lmp->atom;
  Domain *d = lmp->domain;
  int nbonds = 0;
  std::getline(in, line);  // title
  // header
  std::streampos body;
  while (std::getline(in, line)) {
    auto hash = line.find('#');
    if (hash != std::string::npos) line = line.substr(0, hash);
    auto t = split_ws(line);
    if (t.empty()) continue;
    if (t.size() >= 2 && t[1] == "atoms") natoms = std::stoi(t[0]);
    else if (t.size() >= 2 && t[1] == "bonds") nbonds = std::stoi(t[0]);
    else if (t.size() >= 3 && t[1] == "atom" && t[2] == "types") ntypes = std::stoi(t[0]);
    else if (t.size() >= 3 && t[1] == "bond" && t[2] == "types") nbondtypes = std::stoi(t[0]);
    else if (t.size() >= 4 && t[2] == "xlo") { d->boxlo[0] = std::stod(t[0]); d->boxhi[0] = std::stod(t[1]); }
    else if (t.size() >= 4 && t[2] == "ylo") { d->boxlo[1] = std::stod(t[0]); d->boxhi[1] = std::stod(t[1]); }
    else if (t.size() >= 4 && t[2] == "zlo") { d->boxlo[2] = std::stod(t[0]); d->boxhi[2] = std::stod(t[1]); }
    else if (t.size() >= 2 && (t[1] == "angles" || t[1] == "dihedrals" || t[1] == "impropers")) {}
    else if (t.size() >= 3 && t[2] == "types") {}
    else break;  // first section keyword
  }
  a->natoms = a->nlocal = natoms;
  a->nghost = 0;
  a->nmax = natoms;
  a->ntypes = ntypes;
  a->molecular = 1;
  lmp->memory->create(a->x, natoms, 3, "x");
  lmp->memory->create(a->v, natoms, 3, "v");
  lmp->memory->create(a->f, natoms, 3, "f");
  for (int i = 0; i < natoms; i++)
    for (int k = 0; k < 3; k++) a->x[i][k] = a->v[i][k] = a->f[i][k] = 0.0;
  a->tag = (tagint *) calloc(natoms, sizeof(tagint));
  a->type = (int *) calloc(natoms, sizeof(int));
  a->mask = (int *) calloc(natoms, sizeof(int));
  a->image = (imageint *) calloc(natoms, sizeof(imageint));
  a->molecule = (tagint *) calloc(natoms, sizeof(tagint));
  a->residue = (tagint *) calloc(natoms, sizeof(tagint));
  a->mass = (double *) calloc(ntypes + 1, sizeof(double));
  mass.assign(ntypes + 1, 0.0);
  bond_k.assign(nbondtypes + 1, 0.0);
  bond_r0.assign(nbondtypes + 1, 0.0);
  for (int i = 0; i < natoms; i++) a->image[i] = (512 << 20) | (512 << 10) | 512;

  // sections; `line` holds the first keyword
  std::map<int, int> tag2idx;
  std::vector<std::string> atoms_lines, vel_lines, bond_lines;
  auto read_block = [&](int count, std::vector<std::string> *dst) {
    int got = 0;
    while (got < count && std::getline(in, line)) {
      auto hash = line.find('#');
      std::string l = hash == std::string::npos ? line : line.substr(0, hash);
      if (split_ws(l).empty()) continue;
      if (dst) dst->push_back(l);
      got++;
    }
  };
  std::string key = split_ws(line).empty() ? "" : line;
  while (true) {
    auto t = split_ws(key);
    std::string kw = t.empty() ? "" : t[0];
    if (kw == "Masses") {
      std::vector<std::string> l;
      read_block(ntypes, &l);
      for (auto &s : l) {
        auto v = split_ws(s);
        mass[std::stoi(v[0])] = std::stod(v[1]);
      }
    } else if (kw == "Atoms") {
      read_block(natoms, &atoms_lines);
    } else if (kw == "Velocities") {
      read_block(natoms, &vel_lines);
    } else if (kw == "Bonds") {
      read_block(nbonds, &bond_lines);
    } else if (kw == "Bond" && t.size() > 1 && t[1] == "Coeffs") {
      std::vector<std::string> l;
      read_block(nbondtypes, &l);
      for (auto &s : l) {
        auto v = split_ws(s);
        int bt = std::stoi(v[0]);
        bond_k[bt] = std::stod(v[1]);
        bond_r0[bt] = std::stod(v[2]);
      }
    } else if (!kw.empty()) {
      throw std::runtime_error("unsupported data file section: " + kw);
    }
    // next keyword
    key.clear();
    while (std::getline(in, line)) {
      auto hash = line.find('#');
      std::string l = hash == std::string::npos ? line : line.substr(0, hash);
      if (!split_ws(l).empty()) {
        key = l;
        break;
      }
    }
    if (key.empty()) break;
  }
  if ((int) atoms_lines.size() != natoms) throw std::runtime_error("Atoms section incomplete");
  // atoms sorted by tag (atom_modify sort 0: the order a serial read keeps)
  std::vector<std::pair<int, std::string>> rows;
  for (auto &s : atoms_lines) rows.push_back({std::stoi(split_ws(s)[0]), s});
  std::sort(rows.begin(), rows.end());
  for (int i = 0; i < natoms; i++) {
    auto v = split_ws(rows[i].second);
    if (v.size() < 8) throw std::runtime_error("Atoms line needs id molecule residue type q x y z");
    a->tag[i] = std::stoi(v[0]);
    a->molecule[i] = std::stoi(v[1]);
    a->residue[i] = std::stoi(v[2]);
    a->type[i] = std::stoi(v[3]);
    a->x[i][0] = std::stod(v[5]);
    a->x[i][1] = std::stod(v[6]);
    a->x[i][2] = std::stod(v[7]);
    tag2idx[a->tag[i]] = i;
  }
  for (auto &s : vel_lines) {
    auto v = split_ws(s);
    int i = tag2idx.at(std::stoi(v[0]));
    a->v[i][0] = std::stod(v[1]);
    a->v[i][1] = std::stod(v[2]);
    a->v[i][2] = std::stod(v[3]);
  }
  special.assign(natoms, {});
  for (auto &s : bond_lines) {
    auto v = split_ws(s);
    int bt = std::stoi(v[1]);
    int i = tag2idx.at(std::stoi(v[2])), j = tag2idx.at(std::stoi(v[3]));
    bond_t.push_back(bt);
    bond_a.push_back(i);
    bond_b.push_back(j);
    special[i].push_back(j);
    special[j].push_back(i);
  }
  // LAMMPS's special list of the 1-2 partners (what a pair style reads)
  size_t maxsp = 1;
  for (auto &v : special) maxsp = std::max(maxsp, v.size());
  lmp->memory->create(a->nspecial, natoms, 3, "nspecial");
  lmp->memory->create(a->special, natoms, (int) maxsp, "special");
  for (int i = 0; i < natoms; i++) {
    a->nspecial[i][0] = a->nspecial[i][1] = a->nspecial[i][2] = (int) special[i].size();
    for (size_t k = 0; k < special[i].size(); k++) a->special[i][k] = a->tag[special[i][k]];
  }
  for (int t = 1; t <= ntypes; t++) a->mass[t] = mass[t];
  for (int k = 0; k < 3; k++) d->periodicity[k] = 0;
  d->xperiodic = d->yperiodic = d->zperiodic = 0;
  d->xprd = d->boxhi[0] - d->boxlo[0];
  d->yprd = d->boxhi[1] - d->boxlo[1];
  d->zprd = d->boxhi[2] - d->boxlo[2];
  d->dimension = 3;
}

/* Half list, newton on, serial: each pair once (i < j in atom order), pairs
   within cut+skin, 1-2 bonded pairs removed (special_bonds fene); or, with
   `full`, every other atom within that range for each atom (LAMMPS's full
   list).  Binned so that the CPU baseline's list cost stays the O(N) it is in
   LAMMPS. */
void RefHost::build_one(NeighList &list, double cut, bool full)
{
  Atom *a = lmp->atom;
  int n = a->nlocal;
  double cutneigh = cut + skin, cutsq = cutneigh * cutneigh;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) {
      lo[k] = std::min(lo[k], a->x[i][k]);
      hi[k] = std::max(hi[k], a->x[i][k]);
    }
  int nb[3];
  for (int k = 0; k < 3; k++) nb[k] = std::max(1, std::min(512, (int) ((hi[k] - lo[k]) / cutneigh) + 1));
  std::vector<int> head((size_t) nb[0] * nb[1] * nb[2], -1), next(n, -1), bin(n);
  for (int i = n - 1; i >= 0; i--) {
    int c[3];
    for (int k = 0; k < 3; k++) c[k] = std::min(nb[k] - 1, (int) ((a->x[i][k] - lo[k]) / cutneigh));
    int b = (c[2] * nb[1] + c[1]) * nb[0] + c[0];
    bin[i] = b;
    next[i] = head[b];
    head[b] = i;
  }
  list.ilist_store.resize(n);
  list.numneigh_store.assign(n, 0);
  list.firstneigh_store.assign(n, nullptr);
  list.pages.clear();
  std::vector<std::vector<int>> nbr(n);
  for (int i = 0; i < n; i++) {
    int b = bin[i];
    int cx = b % nb[0], cy = (b / nb[0]) % nb[1], cz = b / (nb[0] * nb[1]);
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          int x = cx + dx, y = cy + dy, z = cz + dz;
          if (x < 0 || y < 0 || z < 0 || x >= nb[0] || y >= nb[1] || z >= nb[2]) continue;
          for (int j = head[(z * nb[1] + y) * nb[0] + x]; j != -1; j = next[j]) {
            if (full ? j == i : j <= i) continue;
            double ddx = a->x[i][0] - a->x[j][0];
            double ddy = a->x[i][1] - a->x[j][1];
            double ddz = a->x[i][2] - a->x[j][2];
            double rsq = ddx * ddx + ddy * ddy + ddz * ddz;
            if (rsq >= cutsq) continue;
            bool excluded = false;
            for (int s : special[i])
              if (s == j) excluded = true;
            if (!excluded) nbr[i].push_back(j);
          }
        }
    std::sort(nbr[i].begin(), nbr[i].end());
  }
  size_t total = 0;
  for (int i = 0; i < n; i++) total += nbr[i].size();
  list.pages.resize(std::max<size_t>(total, 1));
  size_t off = 0;
  for (int i = 0; i < n; i++) {
    list.ilist_store[i] = i;
    list.numneigh_store[i] = (int) nbr[i].size();
    std::copy(nbr[i].begin(), nbr[i].end(), list.pages.begin() + off);
    off += nbr[i].size();
  }
  off = 0;
  for (int i = 0; i < n; i++) {
    list.firstneigh_store[i] = list.pages.data() + off;
    off += nbr[i].size();
  }
  list.inum = n;
  list.ilist = list.ilist_store.data();
  list.numneigh = list.numneigh_store.data();
  list.firstneigh = list.firstneigh_store.data();
}

void RefHost::build_lists()
{
  build_one(fixlist, fix_cut, false);
  if (want_full) build_one(fixfull, fix_cut, true);
  build_one(pairlist, pair_cut, false);
  Atom *a = lmp->atom;
  xhold.resize((size_t) a->nlocal * 3);
  for (int i = 0; i < a->nlocal; i++)
    for (int k = 0; k < 3; k++) xhold[3 * i + k] = a->x[i][k];
  last_build = lmp->update->ntimestep;
  lmp->neighbor->ago = 0;
  nbuilds++;
}

/* Neighbor::decide(): delay/every/check with the half-skin trigger. */
bool RefHost::need_rebuild(bigint step)
{
  bigint ago = step - last_build;
  if (ago < delay) return false;
  if (every > 1 && ago % every != 0) return false;
  if (!check) return true;
  Atom *a = lmp->atom;
  double trigger = 0.25 * skin * skin;
  for (int i = 0; i < a->nlocal; i++) {
    double dx = a->x[i][0] - xhold[3 * i], dy = a->x[i][1] - xhold[3 * i + 1],
           dz = a->x[i][2] - xhold[3 * i + 2];
    if (dx * dx + dy * dy + dz * dz > trigger) return true;
  }
  return false;
}

void RefHost::force_clear()
{
  Atom *a = lmp->atom;
  for (int i = 0; i < a->nlocal; i++) a->f[i][0] = a->f[i][1] = a->f[i][2] = 0.0;
}

/* bond_style harmonic: E = K (r - r0)^2, newton_bond on. */
void RefHost::compute_bonds()
{
  Atom *a = lmp->atom;
  e_bond = 0.0;
  for (size_t b = 0; b < bond_t.size(); b++) {
    int i1 = bond_a[b], i2 = bond_b[b], t = bond_t[b];
    double delx = a->x[i1][0] - a->x[i2][0];
    double dely = a->x[i1][1] - a->x[i2][1];
    double delz = a->x[i1][2] - a->x[i2][2];
    double rsq = delx * delx + dely * dely + delz * delz;
    double r = sqrt(rsq);
    double dr = r - bond_r0[t];
    double rk = bond_k[t] * dr;
    double fbond = r > 0.0 ? -2.0 * rk / r : 0.0;
    e_bond += rk * dr;
    a->f[i1][0] += delx * fbond;
    a->f[i1][1] += dely * fbond;
    a->f[i1][2] += delz * fbond;
    a->f[i2][0] -= delx * fbond;
    a->f[i2][1] -= dely * fbond;
    a->f[i2][2] -= delz * fbond;
  }
}

/* fix langevin post_force (uniform noise, no tally, ratio 1), units real. */
void RefHost::langevin_force()
{
  if (!langevin) return;
  Atom *a = lmp->atom;
  Update *u = lmp->update;
  double delta = (double) (u->ntimestep - u->beginstep);
  if (u->endstep != u->beginstep) delta /= (double) (u->endstep - u->beginstep);
  else delta = 0.0;
  double t_target = t_start + delta * (t_stop - t_start);
  double tsqrt = sqrt(t_target);
  for (int i = 0; i < a->nlocal; i++) {
    double m = a->mass[a->type[i]];
    double gamma1 = -m / t_period / FTM2V_REAL;
    double gamma2 = sqrt(m) * sqrt(24.0 * BOLTZ_REAL / t_period / u->dt / MVV2E_REAL) / FTM2V_REAL;
    gamma2 *= tsqrt;
    for (int k = 0; k < 3; k++) {
      double fran = gamma2 * (uniform01(seed, u->ntimestep, a->tag[i], k) - 0.5);
      a->f[i][k] += gamma1 * a->v[i][k] + fran;
    }
  }
}

double RefHost::kinetic()
{
  Atom *a = lmp->atom;
  double ke = 0.0;
  for (int i = 0; i < a->nlocal; i++) {
    double m = a->mass[a->type[i]];
    ke += m * (a->v[i][0] * a->v[i][0] + a->v[i][1] * a->v[i][1] + a->v[i][2] * a->v[i][2]);
  }
  return 0.5 * MVV2E_REAL * ke;
}

/* One force evaluation in Verlet order: fix pre_force, pair, bond, langevin. */
void RefHost::forces(bool setup)
{
  force_clear();
  if (setup) {
    fix->setup_pre_force(1);
    pair->compute(1, 0);
    compute_bonds();
    fix->setup(1);  // pre_force
  } else {
    fix->pre_force(1);
    pair->compute(1, 0);
    compute_bonds();
  }
  e_pair = pair->eng_vdwl;
  langevin_force();
}

static thread_local std::string g_ref_err;

extern "C" {

const char *ref_last_error() { return g_ref_err.c_str(); }

/* Create the host, read the data file, construct the reference fix and pair.
   pair_style: "p cut_short cut_long"; pair_coeffs: ';'-separated
   "i j lambda [cs cl]" records; groups by atom type: CA, CB (and H-beta), O. */
static void *create_host(const char *workdir, const char *data_file, const char *coeff_file,
                         const char *seq_file, const char *pair_style, const char *pair_coeffs,
                         double skin, int every, int delay, int check, int gpu_fix, int gpu_pair = -1)
{
  RefHost *h = new RefHost();
  try {
    h->workdir = workdir ? workdir : "";
    Cwd cwd(h->workdir);
    h->lmp = new LAMMPS();
    LAMMPS *lmp = h->lmp;
    h->read_data(data_file);
    h->skin = skin;
    h->every = every;
    h->delay = delay;
    h->check = check;
    lmp->neighbor->skin = skin;
    Atom *a = lmp->atom;
    a->avec = new AtomVecAWSEM();
    lmp->update->integrate_style = strdup("verlet");
    lmp->update->integrate = nullptr;
    lmp->update->dt = 2.0;
    lmp->force->special_lj[0] = 1.0;
    lmp->force->special_lj[1] = 0.0;
    lmp->force->special_lj[2] = 1.0;
    lmp->force->special_lj[3] = 1.0;
    for (int k = 0; k < 4; k++) lmp->force->special_coul[k] = lmp->force->special_lj[k];
    lmp->force->newton_pair = lmp->force->newton_bond = lmp->force->newton = 1;
    lmp->force->boltz = BOLTZ_REAL;
    lmp->force->mvv2e = MVV2E_REAL;
    lmp->force->ftm2v = FTM2V_REAL;
    // groups: all, alpha_carbons (type 1), beta_atoms (types 4,5), oxygens (type 3)
    Group *g = lmp->group;
    const char *gnames[4] = {"all", "alpha_carbons", "beta_atoms", "oxygens"};
    for (int k = 0; k < 4; k++) {
      g->names[k] = gnames[k];
      g->bitmask[k] = 1 << k;
    }
    g->ngroup = 4;
    for (int i = 0; i < a->nlocal; i++) {
      int t = a->type[i];
      a->mask[i] = 1;
      if (t == 1) a->mask[i] |= 2;
      if (t == 4 || t == 5) a->mask[i] |= 4;
      if (t == 3) a->mask[i] |= 8;
    }
    // pair vexcluded
#ifdef AWSEM_GPU_FIX
    if (gpu_pair >= 0)
      h->pair = new PairExcludedVolumeGPU(lmp);
    else
#endif
      h->pair = new PairExcludedVolume(lmp);
    lmp->force->pair = h->pair;
    {
      auto v = split_ws(pair_style);
      if (gpu_pair >= 0) v.push_back(gpu_pair == 1 ? "mixed" : "fp64");
      std::vector<char *> args;
      for (auto &s : v) args.push_back(strdup(s.c_str()));
      h->pair->settings((int) args.size(), args.data());
      for (char *c : args) free(c);
    }
    {
      std::string all = pair_coeffs ? pair_coeffs : "";
      std::stringstream ss(all);
      std::string rec;
      while (std::getline(ss, rec, ';')) {
        auto v = split_ws(rec);
        if (v.empty()) continue;
        std::vector<char *> args;
        for (auto &s : v) args.push_back(strdup(s.c_str()));
        h->pair->coeff((int) args.size(), args.data());
        for (char *c : args) free(c);
      }
    }
    // fix backbone: fix 2 alpha_carbons backbone beta_atoms oxygens <coeff> <seq>
    {
      std::vector<std::string> v = {"2", "alpha_carbons", "backbone", "beta_atoms", "oxygens",
                                    coeff_file, seq_file};
      std::vector<char *> args;
      for (auto &s : v) args.push_back(strdup(s.c_str()));
#ifdef AWSEM_GPU_FIX
      if (gpu_fix >= 0) {
        free(args[2]);
        args[2] = strdup("backbone/gpu");
        args.push_back(strdup(gpu_fix == 1 ? "mixed" : "fp64"));
        h->fix = new FixBackboneGPU(lmp, (int) args.size(), args.data());
      } else
#endif
        h->fix = h->fb = new FixBackbone(lmp, 7, args.data());
      for (char *c : args) free(c);
    }
    // init: force (pair) first, then fixes, then neighbour lists to requestors
    h->pair->init();
    h->fix->init();
    for (NeighRequest *r : lmp->neighbor->requests) {
      if (r->requestor_is_fix) {
        h->fix_cut = r->cut ? r->cutoff : h->pair->cutforce;
        if (r->flags & NeighConst::REQ_FULL) {
          h->want_full = true;
          h->fix->init_list(r->id, &h->fixfull);
        } else {
          h->fix->init_list(r->id, &h->fixlist);
        }
      } else {
        h->pair_cut = h->pair->cutforce;
        h->pair->init_list(0, &h->pairlist);
      }
    }
  } catch (std::exception &e) {
    g_ref_err = e.what();
    delete h;
    return nullptr;
  }
  return h;
}

void *ref_create(const char *workdir, const char *data_file, const char *coeff_file,
                 const char *seq_file, const char *pair_style, const char *pair_coeffs,
                 double skin, int every, int delay, int check)
{
  return create_host(workdir, data_file, coeff_file, seq_file, pair_style, pair_coeffs, skin, every, delay,
                     check, -1);
}

#ifdef AWSEM_GPU_FIX
/* The same host with `fix backbone/gpu` (precision 0 FP64, 1 mixed) in place
   of the reference fix. */
void *ref_create_gpufix(const char *workdir, const char *data_file, const char *coeff_file,
                        const char *seq_file, const char *pair_style, const char *pair_coeffs,
                        double skin, int every, int delay, int check, int precision)
{
  return create_host(workdir, data_file, coeff_file, seq_file, pair_style, pair_coeffs, skin, every, delay,
                     check, precision);
}

/* The same host with the reference fix and `pair_style vexcluded/gpu`
   (precision 0 FP64, 1 mixed) in place of the reference pair style. */
void *ref_create_gpupair(const char *workdir, const char *data_file, const char *coeff_file,
                         const char *seq_file, const char *pair_style, const char *pair_coeffs,
                         double skin, int every, int delay, int check, int precision)
{
  return create_host(workdir, data_file, coeff_file, seq_file, pair_style, pair_coeffs, skin, every, delay,
                     check, -1, precision);
}
#endif

void ref_destroy(void *hp)
{
  RefHost *h = (RefHost *) hp;
  if (!h) return;
  try {
    Cwd cwd(h->workdir);
    delete h;
  } catch (std::exception &e) {
    g_ref_err = e.what();
  }
}

int ref_natoms(void *hp) { return ((RefHost *) hp)->natoms; }

double ref_fix_cutoff(void *hp) { return ((RefHost *) hp)->fix_cut; }

/* what: "x", "v", "f"; arrays are [natoms][3] in tag order. */
int ref_get(void *hp, const char *what, double *out)
{
  RefHost *h = (RefHost *) hp;
  Atom *a = h->lmp->atom;
  double **src = !strcmp(what, "x") ? a->x : !strcmp(what, "v") ? a->v : !strcmp(what, "f") ? a->f : nullptr;
  if (!src) return -1;
  for (int i = 0; i < a->nlocal; i++)
    for (int k = 0; k < 3; k++) out[3 * i + k] = src[i][k];
  return 0;
}

int ref_set(void *hp, const char *what, const double *in)
{
  RefHost *h = (RefHost *) hp;
  Atom *a = h->lmp->atom;
  double **dst = !strcmp(what, "x") ? a->x : !strcmp(what, "v") ? a->v : nullptr;
  if (!dst) return -1;
  for (int i = 0; i < a->nlocal; i++)
    for (int k = 0; k < 3; k++) dst[i][k] = in[3 * i + k];
  return 0;
}

/* Energies of the last force evaluation: out[0..17] = the fix's energy[]
   (ET_TOTAL first), out[18] = pair vexcluded, out[19] = bonds, out[20] = KE. */
int ref_energies(void *hp, double *out)
{
  RefHost *h = (RefHost *) hp;
  for (int k = 0; k < 18; k++) out[k] = h->fix_energy(k);
  out[18] = h->e_pair;
  out[19] = h->e_bond;
  out[20] = h->kinetic();
  return 0;
}

/* One force evaluation at the current positions, as LAMMPS's setup at
   timestep `step` does it (fresh lists, caches reset), without Langevin. */
int ref_compute(void *hp, long long step, double *f_out)
{
  RefHost *h = (RefHost *) hp;
  try {
    Cwd cwd(h->workdir);
    h->lmp->update->ntimestep = step;
    h->lmp->update->beginstep = h->lmp->update->endstep = step;
    int lg = h->langevin;
    h->langevin = 0;
    h->build_lists();
    h->fix->setup_post_neighbor();
    h->forces(true);
    h->langevin = lg;
    if (f_out) ref_get(hp, "f", f_out);
  } catch (std::exception &e) {
    g_ref_err = e.what();
    return -1;
  }
  return 0;
}

/* Per-residue pair-pass intermediates of the last evaluation, residue order:
   rho_water, rho_helix, water_xi, helix_xi_1, helix_xi_2, burial_force. */
int ref_residue_arrays(void *hp, double *out)
{
  RefHost *h = (RefHost *) hp;
  FixBackbone *fb = h->fb;
  if (!fb) return 0;
  int n = fb->n;
  for (int i = 0; i < n; i++) {
    out[6 * i + 0] = fb->water_ro[i];
    out[6 * i + 1] = fb->helix_ro[i];
    out[6 * i + 2] = fb->water_xi[i];
    out[6 * i + 3] = fb->helix_xi_1[i];
    out[6 * i + 4] = fb->helix_xi_2[i];
    out[6 * i + 5] = fb->burial_force[i];
  }
  return n;
}

/* The entries of the reference's n x n caches (cWell for the water and
   helix wells, cR for r_NO / r_HO, cP_AP for nu; smart_matrix_lib.h) that
   the last evaluation read or filled: those whose generation tag equals the
   fix's current ntimestep.  Keys kind << 56 | aux << 44 | i << 22 | j with
   kind 32 water well (aux = well, i < j), 33 helix well (i < j), 34 r_NO,
   35 r_HO, 36 nu (ordered pairs), sorted.  Returns the number of keys (up
   to cap stored), -1 when no reference fix is hosted. */
long long ref_touches(void *hp, unsigned long long *out, long long cap)
{
  RefHost *h = (RefHost *) hp;
  FixBackbone *fb = h->fb;
  if (!fb) return -1;
  const int t = fb->ntimestep;
  std::vector<unsigned long long> keys;
  auto key = [](int kind, int aux, int i, int j) {
    return (unsigned long long) kind << 56 | (unsigned long long) aux << 44 | (unsigned long long) i << 22 |
           (unsigned long long) j;
  };
  auto wells = [&](WellT *w, int kind) {
    if (!w) return;
    int ***g = w->*get(WellG());
    const int n = w->*get(WellN()), m = w->*get(WellM()), nw = w->*get(WellNW());
    for (int k = 0; k < nw; k++)
      for (int i = 0; i < n; i++)
        for (int j = i + 1; j < m; j++)
          if (g[k][i][j] == t) keys.push_back(key(kind, k, i, j));
  };
  wells(fb->*get(FbWell()), 32);
  wells(fb->*get(FbHWell()), 33);
  if (RT *r = fb->*get(FbR())) {
    int **gno = r->*get(RGNO()), **gho = r->*get(RGHO());
    const int n = r->*get(RN()), m = r->*get(RM());
    for (int i = 0; i < n; i++)
      for (int j = 0; j < m; j++) {
        if (gno[i][j] == t) keys.push_back(key(34, 0, i, j));
        if (gho[i][j] == t) keys.push_back(key(35, 0, i, j));
      }
  }
  if (PapT *q = fb->*get(FbPap())) {
    int **g = q->*get(PapG());
    const int n = q->*get(PapN()), m = q->*get(PapM());
    for (int i = 0; i < n; i++)
      for (int j = 0; j < m; j++)
        if (g[i][j] == t) keys.push_back(key(36, 0, i, j));
  }
  std::sort(keys.begin(), keys.end());
  for (long long k = 0; k < (long long) keys.size() && k < cap; k++) out[k] = keys[k];
  return (long long) keys.size();
}

/* `run nsteps` with fix nve (+ fix langevin when langevin != 0).
   thermo_out (optional): (nsteps+1) rows of [pe_fix, e_pair, e_bond, ke]. */
int ref_run(void *hp, long long nsteps, double dt, int langevin, double t_start, double t_stop,
            double damp, unsigned long long seed, double *thermo_out)
{
  RefHost *h = (RefHost *) hp;
  try {
    Cwd cwd(h->workdir);
    LAMMPS *lmp = h->lmp;
    Update *u = lmp->update;
    Atom *a = lmp->atom;
    u->dt = dt;
    h->langevin = langevin;
    h->t_start = t_start;
    h->t_stop = t_stop;
    h->t_period = damp;
    h->seed = seed;
    u->beginstep = u->firststep = u->ntimestep;
    u->endstep = u->laststep = u->ntimestep + nsteps;
    // Verlet::setup
    h->build_lists();
    h->fix->setup_post_neighbor();
    h->forces(true);
    auto thermo = [&](long long row) {
      if (!thermo_out) return;
      thermo_out[4 * row + 0] = h->fix_energy(0);
      thermo_out[4 * row + 1] = h->e_pair;
      thermo_out[4 * row + 2] = h->e_bond;
      thermo_out[4 * row + 3] = h->kinetic();
    };
    thermo(0);
    double dtf = 0.5 * dt * FTM2V_REAL;
    for (long long s = 1; s <= nsteps; s++) {
      u->ntimestep++;
      for (int i = 0; i < a->nlocal; i++) {
        double dtfm = dtf / a->mass[a->type[i]];
        for (int k = 0; k < 3; k++) {
          a->v[i][k] += dtfm * a->f[i][k];
          a->x[i][k] += dt * a->v[i][k];
        }
      }
      if (h->need_rebuild(u->ntimestep)) {
        h->build_lists();
        h->fix->post_neighbor();
      } else {
        h->lmp->neighbor->ago = (int) (u->ntimestep - h->last_build);
      }
      h->forces(false);
      for (int i = 0; i < a->nlocal; i++) {
        double dtfm = dtf / a->mass[a->type[i]];
        for (int k = 0; k < 3; k++) a->v[i][k] += dtfm * a->f[i][k];
      }
      thermo(s);
    }
  } catch (std::exception &e) {
    g_ref_err = e.what();
    return -1;
  }
  return 0;
}

long ref_nbuilds(void *hp) { return ((RefHost *) hp)->nbuilds; }

/* The reference's `compute ID group qwolynes ...` / `compute ID group
   qonuchic ...` (the whitespace-separated words after `compute`), created in
   the run directory and evaluated once at the current positions. */
int ref_compute_q(void *hp, const char *words, double *out)
{
  RefHost *h = (RefHost *) hp;
  try {
    Cwd cwd(h->workdir);
    std::vector<std::string> v = split_ws(words);
    if (v.size() < 3) throw std::runtime_error("compute: ID group style ...");
    std::vector<char *> args;
    for (auto &s : v) args.push_back(strdup(s.c_str()));
    Compute *c = nullptr;
    try {
      if (v[2] == "qwolynes") c = new ComputeQWolynes(h->lmp, (int) args.size(), args.data());
      else if (v[2] == "qonuchic") c = new ComputeQOnuchic(h->lmp, (int) args.size(), args.data());
      else throw std::runtime_error("compute style " + v[2] + " is not hosted");
      c->init();
      *out = c->compute_scalar();
    } catch (...) {
      delete c;
      for (char *a : args) free(a);
      throw;
    }
    delete c;
    for (char *a : args) free(a);
  } catch (std::exception &e) {
    g_ref_err = e.what();
    return -1;
  }
  return 0;
}

/* Uniform draw of the shared Langevin stream (exported for cross-checks). */
double ref_uniform(unsigned long long seed, long long step, long long tag, int comp)
{
  return uniform01(seed, step, tag, comp);
}

}  // extern "C"
