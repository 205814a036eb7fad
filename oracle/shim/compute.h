/* LAMMPS-API shim header: forwards to lmp_shim.h (test infrastructure). */
#include "lmp_shim.h"
