/* pair_style vexcluded/gpu: see pair_excluded_volume_gpu.h. */
#include "pair_excluded_volume_gpu.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>

#include "atom.h"
#include "atom_vec_awsemmd.h"
#include "domain.h"
#include "error.h"
#include "force.h"
#include "group.h"
#include "memory.h"
#include "neigh_request.h"
#include "neighbor.h"
#include "update.h"

using namespace LAMMPS_NS;

PairExcludedVolumeGPU::PairExcludedVolumeGPU(LAMMPS *lmp) : Pair(lmp)
{
  single_enable = 0;
  restartinfo = 0;
}

PairExcludedVolumeGPU::~PairExcludedVolumeGPU()
{
  awsem_destroy(handle);
  if (allocated) {
    memory->destroy(setflag);
    memory->destroy(cutsq);
    memory->destroy(lambda);
    memory->destroy(cut_short);
    memory->destroy(cut_long);
  }
}

void PairExcludedVolumeGPU::allocate()
{
  allocated = 1;
  const int n = atom->ntypes;
  memory->create(setflag, n + 1, n + 1, "pair:setflag");
  memory->create(cutsq, n + 1, n + 1, "pair:cutsq");
  memory->create(lambda, n + 1, n + 1, "pair:lambda");
  memory->create(cut_short, n + 1, n + 1, "pair:cut_short");
  memory->create(cut_long, n + 1, n + 1, "pair:cut_long");
  for (int i = 1; i <= n; i++)
    for (int j = i; j <= n; j++) {
      setflag[i][j] = 0;
      lambda[i][j] = 0.0;
    }
}

// pair_style vexcluded/gpu p cut_short cut_long [fp64|mixed] [device N] [groups CA CB O]
// (the first three as PairExcludedVolume::settings, src/pair_excluded_volume.cpp:175-195)
void PairExcludedVolumeGPU::settings(int narg, char **arg)
{
  if (narg < 3) error->all(FLERR, "Illegal pair_style command");
  p = atoi(arg[0]);
  if (p < 1) error->all(FLERR, "Illegal pair_style command");
  cut_global[0] = atof(arg[1]);
  cut_global[1] = atof(arg[2]);
  for (int k = 3; k < narg; k++) {
    if (!strcmp(arg[k], "fp64")) precision = AWSEM_FP64;
    else if (!strcmp(arg[k], "mixed")) precision = AWSEM_MIXED;
    else if (!strcmp(arg[k], "device") && k + 1 < narg) device = atoi(arg[++k]);
    else if (!strcmp(arg[k], "groups") && k + 3 < narg) {
      for (int g = 0; g < 3; g++) groups[g] = arg[++k];
    } else {
      error->all(FLERR, "Illegal pair_style vexcluded/gpu keyword");
    }
  }
  // explicitly set coefficients take the new global cutoffs, as in the reference
  if (allocated)
    for (int i = 1; i <= atom->ntypes; i++)
      for (int j = i + 1; j <= atom->ntypes; j++)
        if (setflag[i][j]) {
          cut_short[i][j] = cut_global[0];
          cut_long[i][j] = cut_global[1];
        }
}

// pair_coeff i j lambda [cut_short cut_long] (PairExcludedVolume::coeff, :201-232)
void PairExcludedVolumeGPU::coeff(int narg, char **arg)
{
  if (narg != 3 && narg != 5) error->all(FLERR, "Incorrect args for pair coefficients");
  if (!allocated) allocate();
  int ilo, ihi, jlo, jhi;
  utils::bounds(FLERR, arg[0], 1, atom->ntypes, ilo, ihi, error);
  utils::bounds(FLERR, arg[1], 1, atom->ntypes, jlo, jhi, error);
  const double lambda_one = atof(arg[2]);
  double cut_one[2] = {cut_global[0], cut_global[1]};
  if (narg == 5) {
    cut_one[0] = atof(arg[3]);
    cut_one[1] = atof(arg[4]);
  }
  int count = 0;
  for (int i = ilo; i <= ihi; i++)
    for (int j = MAX(jlo, i); j <= jhi; j++) {
      lambda[i][j] = lambda_one;
      cut_short[i][j] = cut_one[0];
      cut_long[i][j] = cut_one[1];
      setflag[i][j] = 1;
      count++;
    }
  if (count == 0) error->all(FLERR, "Incorrect args for pair coefficients");
}

void PairExcludedVolumeGPU::init_style()
{
  if (!dynamic_cast<AtomVecAWSEM *>(atom->style_match("awsemmd")))
    error->all(FLERR, "Pair excluded_volume requires atom style awsemmd");
  if (atom->natoms != atom->nlocal) error->all(FLERR, "pair vexcluded/gpu needs every atom on one MPI rank");
  // the GPU leaves out the 1-2 bonded pairs (special_bonds fene: lj 0 1 1)
  // or keeps them (lj 1 1 1); it cannot weight pairs
  const double *w = force->special_lj;
  if ((w[1] != 0.0 && w[1] != 1.0) || w[2] != 1.0 || w[3] != 1.0)
    error->all(FLERR, "pair vexcluded/gpu needs special_bonds lj 0 1 1 (fene) or 1 1 1");
  // LAMMPS sizes ghost cutoffs from the pair's list; the GPU lists its own pairs
  neighbor->add_request(this, NeighConst::REQ_DEFAULT);
}

// geometric mixing of lambda and both cutoffs (PairExcludedVolume::init_one, :246-262)
double PairExcludedVolumeGPU::init_one(int i, int j)
{
  if (setflag[i][j] == 0) {
    lambda[i][j] = sqrt(lambda[i][i] * lambda[j][j]);
    cut_short[i][j] = mix_distance(cut_short[i][i], cut_short[j][j]);
    cut_long[i][j] = mix_distance(cut_long[i][i], cut_long[j][j]);
  }
  lambda[j][i] = lambda[i][j];
  cut_short[j][i] = cut_short[i][j];
  cut_long[j][i] = cut_long[i][j];
  return cut_long[i][j];
}

// every type pair's final (mixed) coefficients, as explicit pair_coeff records
std::string PairExcludedVolumeGPU::coeff_text() const
{
  std::ostringstream os;
  os.precision(17);
  for (int i = 1; i <= atom->ntypes; i++)
    for (int j = i; j <= atom->ntypes; j++)
      os << i << ' ' << j << ' ' << lambda[i][j] << ' ' << cut_short[i][j] << ' ' << cut_long[i][j] << ';';
  return os.str();
}

// The handle from LAMMPS's atoms: roles from the three groups, residue and
// molecule ids, types, tags and masses in tag order; the 1-2 partners of
// LAMMPS's special list as the excluded pairs (under special_bonds fene).
void PairExcludedVolumeGPU::create_handle()
{
  awsem_destroy(handle);
  handle = nullptr;
  const int n = atom->nlocal;
  int bits[3];
  for (int g = 0; g < 3; g++) {
    const int id = group->find(groups[g].c_str());
    if (id == -1) error->all(FLERR, ("pair vexcluded/gpu: group " + groups[g] + " does not exist").c_str());
    bits[g] = group->bitmask[id];
  }
  std::vector<int> order(n), role(n), res(n), mol(n), typ(n), tag(n);
  for (int i = 0; i < n; i++) {
    const int t = (int) atom->tag[i];
    if (t < 1 || t > n) error->all(FLERR, "pair vexcluded/gpu needs atom ids 1..natoms");
    order[t - 1] = i;
  }
  for (int k = 0; k < n; k++) {
    const int i = order[k], m = atom->mask[i];
    role[k] = (m & bits[0]) ? 0 : (m & bits[1]) ? 1 : (m & bits[2]) ? 2 : -1;
    res[k] = (int) atom->residue[i];
    mol[k] = (int) atom->molecule[i];
    typ[k] = atom->type[i];
    tag[k] = (int) atom->tag[i];
  }
  std::vector<int> ba, bb;
  if (force->special_lj[1] == 0.0) {
    if (!atom->nspecial || !atom->special) error->all(FLERR, "pair vexcluded/gpu needs the special list");
    for (int i = 0; i < n; i++)
      for (int s = 0; s < atom->nspecial[i][0]; s++) {
        const int t = (int) atom->special[i][s];
        if (t > atom->tag[i]) {
          ba.push_back((int) atom->tag[i] - 1);
          bb.push_back(t - 1);
        }
      }
  }
  const std::vector<double> zero(ba.size() + 1, 0.0);  // excluded pairs only: no bond terms evaluated
  std::ostringstream style;
  style.precision(17);
  style << p << ' ' << cut_global[0] << ' ' << cut_global[1];
  handle_coeffs = coeff_text();
  const int rc = awsem_create_from_atoms(".", nullptr, nullptr, n, role.data(), res.data(), mol.data(), typ.data(),
                                         tag.data(), atom->mass, atom->ntypes, nullptr, (int) ba.size(), ba.data(),
                                         bb.data(), zero.data(), zero.data(), style.str().c_str(),
                                         handle_coeffs.c_str(), precision, device, &handle);
  if (rc != AWSEM_OK) error->all(FLERR, awsem_last_error());
  xg.assign(3 * (size_t) n, 0.0);
  fg.assign(3 * (size_t) n, 0.0);
}

// PairExcludedVolume::compute (:50-138) for every pair on the GPU
void PairExcludedVolumeGPU::compute(int eflag, int vflag)
{
  ev_init(eflag, vflag);
  if (!handle || coeff_text() != handle_coeffs) create_handle();
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
  double e[21];
  const int rc = awsem_compute(handle, (long long) update->ntimestep, xg.data(), fg.data(), e, AWSEM_TERMS_PAIR);
  if (rc != AWSEM_OK) error->all(FLERR, awsem_last_error());
  for (int i = 0; i < n; i++) {
    const size_t k = 3 * (size_t) (atom->tag[i] - 1);
    for (int d = 0; d < 3; d++) f[i][d] += fg[k + d];
  }
  if (eflag_global) eng_vdwl += e[18];
  if (vflag_fdotr) virial_fdotr_compute();
}
