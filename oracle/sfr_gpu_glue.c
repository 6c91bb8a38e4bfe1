/*
 * The solverC drop-in glue a maintainer adds to the reference's build,
 * compiled here so that the reference's own program runs end to end on the
 * B200 path (oracle/Makefile target `dropin`; test
 * tests/test_gpu_dropin_program.py).
 *
 * Linked with -Wl,--wrap=solverC, every solverC call the reference's program
 * makes (Simple.c:2983,3003,3023,3136; Diffusion.c:145; Solv.h:59-70 for the
 * signature) lands in __wrap_solverC.  PCG and PBICGSTAB on CSRD, CSRC or
 * ELLPACK in a one-process run go to sfr_solverC (include/sfr3d_b200.h),
 * which keeps the pattern resident on the GPU, uploads al/ad/au/b, solves,
 * writes x back and prints the reference's log line; any other call goes to
 * the reference's own solverC (__real_solverC).
 */
#include <Solv.h>
#include <ParallelMpi.h>

#include "sfr3d_b200.h"

void __real_solverC(Memoria *m, INT const nEq, INT const nEqNov, INT const nAd,
                    INT const nAdR, INT *ia, INT *ja, DOUBLE *al, DOUBLE *ad,
                    DOUBLE *au, DOUBLE *b, DOUBLE *x, Interface *iNeq,
                    BufferOmp *bOmp, DOUBLE const tol, unsigned int maxIt,
                    short const storage, short const solver, FILE *fSolvLog,
                    bool const fLog, bool const newX, bool const unSym,
                    const char *name);

void __wrap_solverC(Memoria *m, INT const nEq, INT const nEqNov, INT const nAd,
                    INT const nAdR, INT *ia, INT *ja, DOUBLE *al, DOUBLE *ad,
                    DOUBLE *au, DOUBLE *b, DOUBLE *x, Interface *iNeq,
                    BufferOmp *bOmp, DOUBLE const tol, unsigned int maxIt,
                    short const storage, short const solver, FILE *fSolvLog,
                    bool const fLog, bool const newX, bool const unSym,
                    const char *name)
{
  if ((solver == PCG || solver == PBICGSTAB) &&
      (storage == CSRD || storage == CSRC || storage == ELLPACK) &&
      mpiVar.nPrcs == 1 && nEq == nEqNov) {
    sfr_solverC(m, nEq, nEqNov, nAd, nAdR, ia, ja, al, ad, au, b, x, iNeq, bOmp,
                tol, maxIt, storage, solver, fSolvLog, fLog, newX, unSym, name);
    return;
  }
  __real_solverC(m, nEq, nEqNov, nAd, nAdR, ia, ja, al, ad, au, b, x, iNeq, bOmp,
                 tol, maxIt, storage, solver, fSolvLog, fLog, newX, unSym, name);
}
