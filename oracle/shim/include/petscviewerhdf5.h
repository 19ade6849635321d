/* forwards to the PETSc subset used by CIPHER (oracle shim) */
#include "petsc_shim.h"
