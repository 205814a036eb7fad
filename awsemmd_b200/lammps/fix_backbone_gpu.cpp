/* fix backbone/gpu: see fix_backbone_gpu.h. */
#include "fix_backbone_gpu.h"

#include <cstdlib>
#include <cstring>
#include <string>

#include "atom.h"
#include "domain.h"
#include "error.h"
#include "group.h"
#include "neighbor.h"
#include "update.h"

using namespace LAMMPS_NS;
using namespace FixConst;

FixBackboneGPU::FixBackboneGPU(LAMMPS *lmp, int narg, char **arg) : Fix(lmp, narg, arg)
{
  if (narg < 7) error->all(FLERR, "Illegal fix backbone/gpu command");
  scalar_flag = 1;
  vector_flag = 1;
  size_vector = 17;
  global_freq = 1;
  extscalar = 1;
  extvector = 1;
  thermo_energy = 1;
  energy_global_flag = 1;
  respa_level_support = 1;
  const int cb = group->find(arg[3]), o = group->find(arg[4]);
  if (cb == -1) error->all(FLERR, "Beta atoms group id does not exist");
  if (o == -1) error->all(FLERR, "Oxygens group id does not exist");
  cb_bit = group->bitmask[cb];
  o_bit = group->bitmask[o];
  coeff_file = arg[5];
  seq_file = arg[6];
  for (int k = 7; k < narg; k++) {
    if (!strcmp(arg[k], "fp64")) precision = AWSEM_FP64;
    else if (!strcmp(arg[k], "mixed")) precision = AWSEM_MIXED;
    else if (!strcmp(arg[k], "device") && k + 1 < narg) device = atoi(arg[++k]);
    else error->all(FLERR, "Illegal fix backbone/gpu keyword");
  }
}

FixBackboneGPU::~FixBackboneGPU() { awsem_destroy(handle); }

int FixBackboneGPU::setmask()
{
  return PRE_FORCE | PRE_FORCE_RESPA | MIN_PRE_FORCE;
}

void FixBackboneGPU::init()
{
  if (atom->natoms != atom->nlocal) error->all(FLERR, "fix backbone/gpu needs every atom on one MPI rank");
  if (!handle) create_handle();
}

// The handle from the atom data LAMMPS holds: roles from the three groups,
// molecule and residue ids, types, tags and masses, in tag order.
void FixBackboneGPU::create_handle()
{
  const int n = atom->nlocal;
  std::vector<int> role(n, -1), res(n), mol(n), typ(n), tag(n);
  std::vector<int> order(n);
  for (int i = 0; i < n; i++) {
    const int t = (int) atom->tag[i];
    if (t < 1 || t > n) error->all(FLERR, "fix backbone/gpu needs atom ids 1..natoms");
    order[t - 1] = i;
  }
  for (int k = 0; k < n; k++) {
    const int i = order[k];
    const int m = atom->mask[i];
    role[k] = (m & groupbit) ? 0 : (m & cb_bit) ? 1 : (m & o_bit) ? 2 : -1;
    res[k] = (int) atom->residue[i];
    mol[k] = (int) atom->molecule[i];
    typ[k] = atom->type[i];
    tag[k] = (int) atom->tag[i];
  }
  const int rc = awsem_create_from_atoms(".", coeff_file.c_str(), seq_file.c_str(), n, role.data(), res.data(),
                                         mol.data(), typ.data(), tag.data(), atom->mass, atom->ntypes, nullptr, 0,
                                         nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, precision, device,
                                         &handle);
  if (rc != AWSEM_OK) error->all(FLERR, awsem_last_error());
  // the reach of the fix's neighbour lists: pair-list cutoff + LAMMPS's skin
  if (awsem_set_neighbor(handle, neighbor->skin, 0, 1, 1) != AWSEM_OK) error->all(FLERR, awsem_last_error());
  xg.assign(3 * (size_t) n, 0.0);
  fg.assign(3 * (size_t) n, 0.0);
}

// Forces of the fix terms at the current (unwrapped) positions, added to atom->f.
void FixBackboneGPU::evaluate()
{
  if (!handle) create_handle();
  const int n = atom->nlocal;
  double **x = atom->x, **f = atom->f;
  const imageint *image = atom->image;
  const double prd[3] = {domain->xprd, domain->yprd, domain->zprd};
  const int per[3] = {domain->xperiodic, domain->yperiodic, domain->zperiodic};
  for (int i = 0; i < n; i++) {
    const size_t k = 3 * (size_t) (atom->tag[i] - 1);
    const int box[3] = {(int) (image[i] & IMGMASK) - IMGMAX, (int) (image[i] >> IMGBITS & IMGMASK) - IMGMAX,
                        (int) (image[i] >> IMG2BITS) - IMGMAX};
    for (int d = 0; d < 3; d++) xg[k + d] = x[i][d] + (per[d] ? box[d] * prd[d] : 0.0);
  }
  std::fill(fg.begin(), fg.end(), 0.0);
  // [AMH-Go] reads the fix's full neighbour list: new only on build steps
  if (awsem_set_list_built(handle, neighbor->ago == 0 ? 1 : 0) != AWSEM_OK) error->all(FLERR, awsem_last_error());
  const int rc = awsem_compute(handle, (long long) update->ntimestep, xg.data(), fg.data(), energy, AWSEM_TERMS_FIX);
  if (rc != AWSEM_OK) error->all(FLERR, awsem_last_error());
  for (int i = 0; i < n; i++) {
    const size_t k = 3 * (size_t) (atom->tag[i] - 1);
    for (int d = 0; d < 3; d++) f[i][d] += fg[k + d];
  }
  evaluated_step = update->ntimestep;
}

void FixBackboneGPU::setup(int) { evaluate(); }
void FixBackboneGPU::min_setup(int) { evaluate(); }
void FixBackboneGPU::setup_pre_force(int) {}
void FixBackboneGPU::pre_force(int) { evaluate(); }
void FixBackboneGPU::pre_force_respa(int, int ilevel, int)
{
  if (ilevel == respa_level) evaluate();
}
void FixBackboneGPU::min_pre_force(int) { evaluate(); }

double FixBackboneGPU::compute_scalar() { return energy[0]; }
double FixBackboneGPU::compute_vector(int i) { return energy[i + 1]; }
