/* matrix.h stand-in: everything lives in the mex.h stub of this directory. */
#include "mex.h"
