/* ORACLE build only: see petsc.h. */
#include "petsc.h"
