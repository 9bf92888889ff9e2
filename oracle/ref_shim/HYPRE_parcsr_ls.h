/* hypre stand-in: everything is in HYPRE.h (test infrastructure). */
#include "HYPRE.h"
