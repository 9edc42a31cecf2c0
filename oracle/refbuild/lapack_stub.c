/* Stand-ins for the reference's LAPACK wrappers (src/num/lapack.c), whose
 * Fortran LAPACK dependency is absent here. None of them is reached on the
 * NUFFT / CG-SENSE path; a call aborts loudly. Test infrastructure only. */
#include <stdio.h>
#include <stdlib.h>

#define STUB(name) void name(void); void name(void) { fprintf(stderr, "refbuild: LAPACK routine %s is not available\n", #name); abort(); }

STUB(lapack_schur)
STUB(lapack_schur_double)
STUB(lapack_solve_real)
STUB(lapack_svd)
STUB(lapack_svd_econ)
STUB(lapack_qr_econ)
STUB(lapack_sylvester)
STUB(lapack_trimat_solve)
