// Test infrastructure only: the reference's spatial interpolation Interpolate()
// (src/Interpolation/Interpolate.cpp:90, with Interpolate_Iterate and the Int_*.cpp schemes, compiled
// unmodified from the reference tree by oracle/build_ref.sh into the hydro MHM variants) as the oracle
// of gb_interpolate_device.
//
// It defines the globals those files read from the rest of GAMER (src/Main/Main.cpp) and the routine
// the iterative path calls only to report a failure (Aux_Message), and exports one plain C function
// that runs Interpolate() on every region of a batch.  Interpolate.cpp is included here, unmodified and
// read where it lies (its path arrives as GREF_INTERPOLATE from oracle/build_ref.sh), so that its
// MPI_Exit() -- in a serial build the macro of include/Serial.h that ends the process -- ends the call
// with an exception instead.  Nothing in the product links this file.

#include "GAMER.h"
#include <cstdarg>
#include <cstring>
#include <stdexcept>
#include <vector>

#undef  MPI_Exit
#define MPI_Exit()   throw std::runtime_error( "Interpolate_Iterate failed" )
#include GREF_INTERPOLATE

// ---- globals normally defined by src/Main/Main.cpp ---------------------------------------------
double INT_MONO_COEFF           = 2.0;
int    MONO_MAX_ITER            = 10;
bool   OPT__INT_FRAC_PASSIVE_LR = false;
int    PassiveIntFrac_NVar      = 0;
int    PassiveIntFrac_VarIdx[ NCOMP_PASSIVE ];

extern double GAMMA, MIN_PRES;
void EoS_Init_Gamma();

void Aux_Message( FILE *Type, const char *Format, ... ) {}

extern "C" {

// Interpolate() on nbatch regions: cdata [nbatch][ncomp][CSize z][y][x] (copied first: the reference
// may overwrite its input), fdata [nbatch][ncomp][FSize z][y][x] (cells outside the fine range keep
// their values).  monotonic: int[ncomp].  iterate = 0: the plain path with INT_MONO_COEFF = mono_coeff;
// iterate = 1: AllCons with OPT__INT_PRIM = int_prim and MONO_MAX_ITER = mono_max_iter
// (ReduceMonoCoeff when > 0), which Interpolate() sends to Interpolate_Iterate when either is on;
// GAMMA = gamma, MIN_PRES = min_pres.  Returns 0, or 2 when an iteration ended in failure (the
// reference's abort).
__attribute__((visibility("default")))
int gref_interpolate( const void *cdata_in, void *fdata_out, const int csize[3], const int cstart[3],
                      const int crange[3], const int fsize[3], const int fstart[3], const int ncomp,
                      const int scheme, const int *monotonic, const int opp, const int iterate, const int int_prim,
                      const double mono_coeff, const int mono_max_iter, const double gamma, const double min_pres,
                      const int nbatch )
{
   GAMMA = gamma;
   EoS_Init_Gamma();
   MIN_PRES = min_pres;
   INT_MONO_COEFF = mono_coeff;
   MONO_MAX_ITER = mono_max_iter;
   const long c3 = (long)csize[0]*csize[1]*csize[2], f3 = (long)fsize[0]*fsize[1]*fsize[2];
   std::vector<real> cbuf( ncomp*c3 );
   bool mono[64];
   for (int v=0; v<ncomp && v<64; v++)   mono[v] = monotonic[v] != 0;
   int rc = 0;
   for (int b=0; b<nbatch; b++)
   {
      memcpy( cbuf.data(), (const real*)cdata_in + b*ncomp*c3, sizeof(real)*ncomp*c3 );
      real *f = (real*)fdata_out + b*ncomp*f3;
      try {
         Interpolate( cbuf.data(), csize, cstart, crange, f, fsize, fstart, ncomp, (IntScheme_t)scheme, false, mono,
                      opp != 0, iterate != 0, ( iterate && int_prim ) ? INT_PRIM_YES : INT_PRIM_NO,
                      ( iterate && mono_max_iter > 0 ) ? INT_REDUCE_MONO_COEFF : INT_FIX_MONO_COEFF, NULL, NULL );
      } catch ( const std::exception & ) { rc = 2; }
   }
   return rc;
}

} // extern "C"
