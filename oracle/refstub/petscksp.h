/* single-rank stand-in: see petsc_stub.h */
#include "petsc_stub.h"
