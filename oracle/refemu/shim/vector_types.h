/* host stand-in header for the reference CPU build; see refemu_cuda.h */
#include "refemu_cuda.h"
