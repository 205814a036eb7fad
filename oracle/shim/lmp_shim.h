/* Minimal LAMMPS-API shim: test infrastructure for the oracle.

   The reference AWSEM plugins (fix backbone, pair vexcluded) are LAMMPS style
   classes.  LAMMPS itself is not vendored and cannot be built here, so this
   header declares just the slice of the LAMMPS class surface those plugins
   touch (Pointers, Fix, Pair, Atom, Neighbor/NeighList/NeighRequest, Domain,
   Comm, Group, Update/Respa, Output, Force, Memory, Error, utils) with the
   same names and member types, so that the reference sources compile
   unmodified against it.  The behaviour behind these declarations
   (lmp_shim.cpp, ref_host.cpp) is a serial, single-rank host: no ghost atoms,
   a half neighbour list with `special_bonds fene` 1-2 exclusion, and the MPI
   calls reduced to copies.

   Only tests/, the package smoke check and bench.py's CPU baseline use this. */
#ifndef AWSEM_ORACLE_LMP_SHIM_H
#define AWSEM_ORACLE_LMP_SHIM_H

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <stdexcept>
#include "mpi.h"

#ifndef MAX
#define MAX(A, B) ((A) > (B) ? (A) : (B))
#endif
#ifndef MIN
#define MIN(A, B) ((A) < (B) ? (A) : (B))
#endif
#define FLERR __FILE__, __LINE__

namespace LAMMPS_NS {

typedef int tagint;
typedef int imageint;
typedef long long bigint;

#define NEIGHMASK 0x1FFFFFFF
#define SBBITS 30
// image flags of LAMMPS's default (smallbig) build: three 10-bit fields
#define IMGMASK 1023
#define IMGMAX 512
#define IMGBITS 10
#define IMG2BITS 20
static inline int sbmask(int j) { return j >> SBBITS & 3; }

class LAMMPS;
class Memory;
class Error;
class Atom;
class Update;
class Neighbor;
class Comm;
class Domain;
class Force;
class Modify;
class Group;
class Output;
class Timer;
class Pair;
class Fix;
class NeighList;
class NeighRequest;
class AtomVec;
class Integrate;

class Pointers {
 public:
  Pointers(LAMMPS *ptr);
  virtual ~Pointers() {}

 protected:
  LAMMPS *lmp;
  Memory *&memory;
  Error *&error;
  Atom *&atom;
  Update *&update;
  Neighbor *&neighbor;
  Comm *&comm;
  Domain *&domain;
  Force *&force;
  Modify *&modify;
  Group *&group;
  Output *&output;
  Timer *&timer;
  MPI_Comm &world;
  FILE *&screen;
  FILE *&logfile;
};

class Memory {
 public:
  void *smalloc(bigint n, const char *);
  void *srealloc(void *ptr, bigint n, const char *);
  void sfree(void *ptr);

  template <typename T> T **create(T **&array, int n1, int n2, const char *name)
  {
    T *data = (T *) smalloc((bigint) n1 * n2 * sizeof(T), name);
    array = (T **) smalloc((bigint) n1 * sizeof(T *), name);
    for (int i = 0; i < n1; i++) array[i] = &data[(bigint) i * n2];
    return array;
  }
  template <typename T> void destroy(T **&array)
  {
    if (array == nullptr) return;
    sfree(array[0]);
    sfree(array);
    array = nullptr;
  }
  template <typename T> T *create(T *&array, int n, const char *name)
  {
    array = (T *) smalloc((bigint) n * sizeof(T), name);
    return array;
  }
  template <typename T> void destroy(T *&array)
  {
    sfree(array);
    array = nullptr;
  }
};

/* Error::all throws; the host catches it and reports the message. */
class Error {
 public:
  [[noreturn]] void all(const char *file, int line, const char *msg);
  [[noreturn]] void one(const char *file, int line, const char *msg);
  void warning(const char *file, int line, const char *msg);
};

class AtomVec {
 public:
  virtual ~AtomVec() {}
  std::string style;
};

class Atom {
 public:
  int natoms, nlocal, nghost, nmax, ntypes;
  tagint *tag;
  int *type, *mask;
  imageint *image;
  double **x, **v, **f;
  tagint *molecule;
  tagint *residue;
  double *mass;
  int molecular;
  int tag_enable = 1;
  // special neighbours: nspecial[i] = cumulative counts of 1-2, 1-3, 1-4
  // partners, special[i] their atom ids (this host fills the 1-2 ones)
  int **nspecial = nullptr;
  tagint **special = nullptr;
  AtomVec *avec;
  AtomVec *style_match(const char *name);
};

class Domain {
 public:
  int xperiodic, yperiodic, zperiodic;
  int periodicity[3];
  double xprd, yprd, zprd;
  double boxlo[3], boxhi[3];
  int dimension;
};

class Comm {
 public:
  int me, nprocs;
  double cutghostuser;
};

class Group {
 public:
  static const int MAX_GROUP = 32;
  int ngroup;
  std::string names[MAX_GROUP];
  int bitmask[MAX_GROUP];
  LAMMPS *lmp;
  int find(const char *name);
  bigint count(int igroup);
};

class Integrate {
 public:
  virtual ~Integrate() {}
};

class Respa : public Integrate {
 public:
  int nlevels;
  void copy_flevel_f(int) {}
  void copy_f_flevel(int) {}
};

class Update {
 public:
  bigint ntimestep, firststep, laststep, beginstep, endstep;
  double dt;
  char *integrate_style;
  Integrate *integrate;
};

class Output {
 public:
  int thermo_every;
};

class Timer {};
class Modify {};

class Force {
 public:
  Pair *pair;
  double special_lj[4], special_coul[4];
  int newton_pair, newton_bond, newton;
  double boltz, mvv2e, ftm2v;
};

namespace NeighConst {
  enum { REQ_DEFAULT = 0, REQ_FULL = 1 << 0, REQ_GHOST = 1 << 1, REQ_SIZE = 1 << 2 };
}

class NeighList {
 public:
  int inum;
  int *ilist;
  int *numneigh;
  int **firstneigh;
  std::vector<int> ilist_store, numneigh_store, pages;
  std::vector<int *> firstneigh_store;
};

class NeighRequest {
 public:
  void *requestor;
  int requestor_is_fix;
  int id;
  int flags;
  int cut;
  double cutoff;
  void set_id(int i) { id = i; }
  void set_cutoff(double c) { cut = 1; cutoff = c; }
};

class Neighbor {
 public:
  double skin;
  int ago = 0;  // steps since the lists were built
  std::vector<NeighRequest *> requests;
  NeighRequest *add_request(Fix *, int flags = 0);
  NeighRequest *add_request(Pair *, int flags = 0);
  ~Neighbor();
};

namespace utils {
  bool strmatch(const std::string &text, const std::string &pattern);
  void bounds(const char *file, int line, const std::string &str, bigint nmin, bigint nmax,
              int &nlo, int &nhi, Error *error);
}

namespace FixConst {
  enum {
    INITIAL_INTEGRATE = 1 << 0,
    POST_INTEGRATE = 1 << 1,
    PRE_EXCHANGE = 1 << 2,
    PRE_NEIGHBOR = 1 << 3,
    POST_NEIGHBOR = 1 << 4,
    PRE_FORCE = 1 << 5,
    PRE_REVERSE = 1 << 6,
    POST_FORCE = 1 << 7,
    FINAL_INTEGRATE = 1 << 8,
    END_OF_STEP = 1 << 9,
    POST_RUN = 1 << 10,
    INITIAL_INTEGRATE_RESPA = 1 << 11,
    POST_INTEGRATE_RESPA = 1 << 12,
    PRE_FORCE_RESPA = 1 << 13,
    POST_FORCE_RESPA = 1 << 14,
    FINAL_INTEGRATE_RESPA = 1 << 15,
    MIN_PRE_EXCHANGE = 1 << 16,
    MIN_PRE_NEIGHBOR = 1 << 17,
    MIN_POST_NEIGHBOR = 1 << 18,
    MIN_PRE_FORCE = 1 << 19,
    MIN_PRE_REVERSE = 1 << 20,
    MIN_POST_FORCE = 1 << 21,
    MIN_ENERGY = 1 << 22
  };
}

// LAMMPS's Compute base, as far as the reference computes use it
class Compute : protected Pointers {
 public:
  char *id, *style;
  int igroup, groupbit;
  int scalar_flag, vector_flag, extscalar;
  double scalar;
  bigint invoked_scalar;
  Compute(LAMMPS *, int, char **);
  virtual ~Compute();
  virtual void init() {}
  virtual double compute_scalar() { return 0.0; }
};

class Fix : protected Pointers {
 public:
  char *id, *style;
  int igroup, groupbit;
  int scalar_flag, vector_flag, array_flag, size_vector, size_array_rows, size_array_cols;
  int global_freq, extscalar, extvector, thermo_energy, thermo_virial, energy_global_flag,
      energy_peratom_flag, virial_global_flag, virial_peratom_flag;
  int nevery, respa_level_support, respa_level;
  int dynamic_group_allow, restart_global, restart_peratom;

  Fix(LAMMPS *, int, char **);
  virtual ~Fix();
  virtual int setmask() = 0;
  virtual void init() {}
  virtual void init_list(int, NeighList *) {}
  virtual void setup(int) {}
  virtual void min_setup(int) {}
  virtual void setup_pre_force(int) {}
  virtual void setup_pre_force_respa(int, int) {}
  virtual void setup_post_neighbor() {}
  virtual void post_neighbor() {}
  virtual void min_post_neighbor() {}
  virtual void pre_force(int) {}
  virtual void pre_force_respa(int, int, int) {}
  virtual void min_pre_force(int) {}
  virtual double compute_scalar() { return 0.0; }
  virtual double compute_vector(int) { return 0.0; }
};

class Pair : protected Pointers {
 public:
  double eng_vdwl, eng_coul;
  double virial[6];
  double cutforce;
  double **cutsq;
  int **setflag;
  int allocated;
  int mix_flag;
  int evflag, eflag_either, eflag_global, vflag_either, vflag_global, vflag_fdotr;
  int restartinfo, single_enable, one_coeff, manybody_flag;
  NeighList *list;
  enum { GEOMETRIC, ARITHMETIC, SIXTHPOWER };

  Pair(LAMMPS *);
  virtual ~Pair() {}
  virtual void compute(int, int) = 0;
  virtual void settings(int, char **) = 0;
  virtual void coeff(int, char **) = 0;
  virtual void init_style() {}
  virtual double init_one(int, int) { return 0.0; }
  virtual void init_list(int, NeighList *ptr) { list = ptr; }
  virtual void write_restart(FILE *) {}
  virtual void read_restart(FILE *) {}
  virtual void write_restart_settings(FILE *) {}
  virtual void read_restart_settings(FILE *) {}
  virtual double single(int, int, int, int, double, double, double, double &) { return 0.0; }
  void init();

 protected:
  void ev_init(int eflag, int vflag);
  void ev_tally(int i, int j, int nlocal, int newton_pair, double evdwl, double ecoul, double fpair,
                double delx, double dely, double delz);
  void virial_fdotr_compute() {}
  double mix_distance(double sig1, double sig2);
  double mix_energy(double eps1, double eps2, double sig1, double sig2);
};

class LAMMPS {
 public:
  Memory *memory;
  Error *error;
  Atom *atom;
  Update *update;
  Neighbor *neighbor;
  Comm *comm;
  Domain *domain;
  Force *force;
  Modify *modify;
  Group *group;
  Output *output;
  Timer *timer;
  MPI_Comm world;
  FILE *screen;
  FILE *logfile;
  LAMMPS();
  ~LAMMPS();
};

}  // namespace LAMMPS_NS

#endif
