/* ORACLE build only: Apollo's solver header holds a pointer to its PETSc
 * time-stepping wrapper; the limiter harness never creates one. */
#include "petsc.h"
template <typename REAL, typename CLS> class WxPetscTimeSteppingSolver;
