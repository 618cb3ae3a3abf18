/* mkl_rci.h -- empty stand-in: the reference includes it but its FGMRES path
 * uses no RCI routine (see mkl.h for the scope). */
#pragma once
#include "mkl.h"
