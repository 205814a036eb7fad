/* Behaviour behind the LAMMPS-API shim declarations (lmp_shim.h).
   Test infrastructure for the oracle: serial, one rank, no ghost atoms. */
#include "lmp_shim.h"
#include <cmath>
#include <regex>

namespace LAMMPS_NS {

Pointers::Pointers(LAMMPS *ptr)
    : lmp(ptr), memory(ptr->memory), error(ptr->error), atom(ptr->atom), update(ptr->update),
      neighbor(ptr->neighbor), comm(ptr->comm), domain(ptr->domain), force(ptr->force),
      modify(ptr->modify), group(ptr->group), output(ptr->output), timer(ptr->timer),
      world(ptr->world), screen(ptr->screen), logfile(ptr->logfile)
{
}

void *Memory::smalloc(bigint n, const char *)
{
  if (n == 0) return nullptr;
  void *p = malloc((size_t) n);
  if (!p) throw std::runtime_error("shim: out of memory");
  return p;
}

void *Memory::srealloc(void *ptr, bigint n, const char *)
{
  if (n == 0) {
    free(ptr);
    return nullptr;
  }
  void *p = realloc(ptr, (size_t) n);
  if (!p) throw std::runtime_error("shim: out of memory");
  return p;
}

void Memory::sfree(void *ptr) { free(ptr); }

void Error::all(const char *file, int line, const char *msg)
{
  char buf[1024];
  snprintf(buf, sizeof buf, "ERROR: %s (%s:%d)", msg, file, line);
  throw std::runtime_error(buf);
}

void Error::one(const char *file, int line, const char *msg) { all(file, line, msg); }

void Error::warning(const char *file, int line, const char *msg)
{
  fprintf(stderr, "WARNING: %s (%s:%d)\n", msg, file, line);
}

AtomVec *Atom::style_match(const char *name)
{
  if (avec && avec->style == name) return avec;
  return nullptr;
}

int Group::find(const char *name)
{
  for (int i = 0; i < ngroup; i++)
    if (names[i] == name) return i;
  return -1;
}

bigint Group::count(int igroup)
{
  bigint c = 0;
  Atom *a = lmp->atom;
  for (int i = 0; i < a->nlocal; i++)
    if (a->mask[i] & bitmask[igroup]) c++;
  return c;
}

NeighRequest *Neighbor::add_request(Fix *f, int flags)
{
  NeighRequest *r = new NeighRequest();
  r->requestor = f;
  r->requestor_is_fix = 1;
  r->id = 0;
  r->flags = flags;
  r->cut = 0;
  r->cutoff = 0.0;
  requests.push_back(r);
  return r;
}

NeighRequest *Neighbor::add_request(Pair *p, int flags)
{
  NeighRequest *r = new NeighRequest();
  r->requestor = p;
  r->requestor_is_fix = 0;
  r->id = 0;
  r->flags = flags;
  r->cut = 0;
  r->cutoff = 0.0;
  requests.push_back(r);
  return r;
}

Neighbor::~Neighbor()
{
  for (auto *r : requests) delete r;
}

namespace utils {
bool strmatch(const std::string &text, const std::string &pattern)
{
  return std::regex_search(text, std::regex(pattern));
}

/* "n", "*", "n*", "*n", "m*n" as in the LAMMPS type-range convention. */
void bounds(const char *file, int line, const std::string &str, bigint nmin, bigint nmax,
            int &nlo, int &nhi, Error *error)
{
  size_t found = str.find('*');
  if (found == std::string::npos) {
    nlo = nhi = std::stoi(str);
  } else if (str.size() == 1) {
    nlo = (int) nmin;
    nhi = (int) nmax;
  } else if (found == 0) {
    nlo = (int) nmin;
    nhi = std::stoi(str.substr(1));
  } else if (found == str.size() - 1) {
    nlo = std::stoi(str.substr(0, found));
    nhi = (int) nmax;
  } else {
    nlo = std::stoi(str.substr(0, found));
    nhi = std::stoi(str.substr(found + 1));
  }
  if (nlo < nmin || nhi > nmax || nlo > nhi) error->all(file, line, "Numeric index is out of bounds");
}
}  // namespace utils

Fix::Fix(LAMMPS *lmp, int, char **arg) : Pointers(lmp)
{
  id = strdup(arg[0]);
  style = strdup(arg[2]);
  igroup = lmp->group->find(arg[1]);
  if (igroup == -1) error->all(FLERR, "Could not find fix group ID");
  groupbit = lmp->group->bitmask[igroup];
  scalar_flag = vector_flag = array_flag = 0;
  size_vector = size_array_rows = size_array_cols = 0;
  global_freq = 1;
  extscalar = extvector = 0;
  thermo_energy = thermo_virial = 0;
  energy_global_flag = energy_peratom_flag = 0;
  virial_global_flag = virial_peratom_flag = 0;
  nevery = 1;
  respa_level_support = 0;
  respa_level = -1;
  dynamic_group_allow = 0;
  restart_global = restart_peratom = 0;
}

Fix::~Fix()
{
  free(id);
  free(style);
}

Compute::Compute(LAMMPS *lmp, int, char **arg) : Pointers(lmp)
{
  id = strdup(arg[0]);
  style = strdup(arg[2]);
  igroup = lmp->group->find(arg[1]);
  if (igroup == -1) error->all(FLERR, "Could not find compute group ID");
  groupbit = lmp->group->bitmask[igroup];
  scalar_flag = vector_flag = extscalar = 0;
  scalar = 0.0;
  invoked_scalar = -1;
}

Compute::~Compute()
{
  free(id);
  free(style);
}

Pair::Pair(LAMMPS *lmp) : Pointers(lmp)
{
  eng_vdwl = eng_coul = 0.0;
  for (double &v : virial) v = 0.0;
  cutforce = 0.0;
  cutsq = nullptr;
  setflag = nullptr;
  allocated = 0;
  mix_flag = GEOMETRIC;
  evflag = eflag_either = eflag_global = vflag_either = vflag_global = vflag_fdotr = 0;
  restartinfo = single_enable = 1;
  one_coeff = manybody_flag = 0;
  list = nullptr;
}

/* Pair::init as LAMMPS runs it: style init, then init_one for each type
   pair (i<=j), the maximum of which becomes the force cutoff. */
void Pair::init()
{
  init_style();
  cutforce = 0.0;
  int n = atom->ntypes;
  for (int i = 1; i <= n; i++)
    for (int j = i; j <= n; j++) {
      double cut = init_one(i, j);
      cutsq[i][j] = cutsq[j][i] = cut * cut;
      cutforce = MAX(cutforce, cut);
    }
}

void Pair::ev_init(int eflag, int vflag)
{
  evflag = eflag || vflag;
  eflag_either = eflag_global = eflag;
  vflag_either = vflag_global = vflag;
  vflag_fdotr = 0;
  if (eflag_global) eng_vdwl = eng_coul = 0.0;
  if (vflag_global)
    for (double &v : virial) v = 0.0;
}

void Pair::ev_tally(int i, int j, int nlocal, int newton_pair, double evdwl, double ecoul,
                    double fpair, double delx, double dely, double delz)
{
  if (eflag_global) {
    if (newton_pair) {
      eng_vdwl += evdwl;
      eng_coul += ecoul;
    } else {
      double evdwlhalf = 0.5 * evdwl, ecoulhalf = 0.5 * ecoul;
      if (i < nlocal) {
        eng_vdwl += evdwlhalf;
        eng_coul += ecoulhalf;
      }
      if (j < nlocal) {
        eng_vdwl += evdwlhalf;
        eng_coul += ecoulhalf;
      }
    }
  }
  if (vflag_global) {
    double v[6] = {delx * delx * fpair, dely * dely * fpair, delz * delz * fpair,
                   delx * dely * fpair, delx * delz * fpair, dely * delz * fpair};
    for (int k = 0; k < 6; k++) virial[k] += v[k];
  }
}

/* LAMMPS mixing rules for distances (geometric default). */
double Pair::mix_distance(double sig1, double sig2)
{
  if (mix_flag == GEOMETRIC) return sqrt(sig1 * sig2);
  if (mix_flag == ARITHMETIC) return 0.5 * (sig1 + sig2);
  return pow(0.5 * (pow(sig1, 6.0) + pow(sig2, 6.0)), 1.0 / 6.0);
}

double Pair::mix_energy(double eps1, double eps2, double, double) { return sqrt(eps1 * eps2); }

LAMMPS::LAMMPS()
{
  memory = new Memory();
  error = new Error();
  atom = new Atom();
  memset(atom, 0, sizeof(Atom));
  atom->tag_enable = 1;
  update = new Update();
  memset(update, 0, sizeof(Update));
  neighbor = new Neighbor();
  neighbor->skin = 2.0;
  comm = new Comm();
  comm->me = 0;
  comm->nprocs = 1;
  comm->cutghostuser = 0.0;
  domain = new Domain();
  memset(domain, 0, sizeof(Domain));
  force = new Force();
  memset(force, 0, sizeof(Force));
  modify = new Modify();
  group = new Group();
  group->ngroup = 0;
  group->lmp = this;
  output = new Output();
  output->thermo_every = 1000000000;
  timer = new Timer();
  world = MPI_COMM_WORLD;
  screen = nullptr;
  logfile = nullptr;
}

LAMMPS::~LAMMPS()
{
  delete memory;
  delete error;
  delete atom;
  delete update;
  delete neighbor;
  delete comm;
  delete domain;
  delete force;
  delete modify;
  delete group;
  delete output;
  delete timer;
}

}  // namespace LAMMPS_NS
