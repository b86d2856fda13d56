/* Compile check (test infrastructure): the reference's unity build
 * (pardiso/i3mg.c:1-19, without its main) with vpiterate(), ronurecalc(),
 * movemark(), effbulkvisccalc() and titerate() taken from
 * pardiso2_b200/csrc/move3mg_cuda.c: the CPU functions are renamed by macros
 * around their files and the shim is included after them.
 * Built with -c only: it proves the shim compiles against the reference's
 * globals and the p2cuda.h declarations. */
#include <stdio.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>
#include <time.h>
#include <hdf5.h>

#include "head3mg.c"
#include "load3mg.c"
#define vpiterate vpiterate_cpu
#define ronurecalc ronurecalc_cpu
#define movemark movemark_cpu
#define effbulkvisccalc effbulkvisccalc_cpu
#include "move3mgNew.c"
#include "mark3mg.c"
#undef vpiterate
#undef ronurecalc
#undef movemark
#undef effbulkvisccalc
#include "gaus3mg_SerieMG.c"
#define titerate titerate_cpu
#include "heat3mg.c"
#undef titerate
#include "move3mg_cuda.c"
