// Test infrastructure only: the reference's Flu_FixUp_Flux() (src/Fluid/Flu_FixUp_Flux.cpp:23) as
// an oracle for the device coarse-fine flux fix-up.
//
// Flu_FixUp_Flux walks the patches of one AMR level and, on every face that holds a flux
// difference (patch_t::flux[s], filled by StoreFlux / CorrectFlux of Flu_Close), corrects the layer
// of cells along that face.  This file builds that level from caller-owned arrays: one patch_t per
// patch of the batch (the reference's own class, include/Patch.h), its fluid, dual-energy status
// and flux arrays filled from the caller's, then calls Flu_FixUp_Flux (compiled unmodified from
// its source, oracle/build_ref.sh) and copies the fluid back.  The globals it reads (amr, MIN_*,
// PassiveFloorMask, ...) are the ones oracle/ref_close.cpp defines in the same library.
//
// Nothing in the product links this file.

#include "GAMER.h"

extern double GAMMA;
void EoS_Init_Gamma();
void Flu_FixUp_Flux( const int lv, const long TVar );

// patch_t::Activate derives a patch's padded-cell and load-balance indices from its corner
// (src/Miscellaneous/Mis_Idx3D2Idx1D.cpp, src/LoadBalance/LB_Corner2Index.cpp); the fix-up reads
// neither, so the batch's patches take index 0
ulong Mis_Idx3D2Idx1D( const int Size[], const int Idx3D[] )  { return 0; }
long  LB_Corner2Index( const int lv, const int Corner[], const Check_t Check )  { return 0; }

extern "C" {

// fluid   [NP][NCOMP_TOTAL][PS1^3]  corrected in place
// de      [NP][PS1^3] (DUAL_ENERGY builds; may be NULL otherwise)
// flux    [NP][6][NCOMP_TOTAL][PS1^2]  the flux differences of the six faces
// has_flux[NP][6]  1 where the face carries a flux array (patch_t::flux[s] != NULL)
// tvar: the bit mask of corrected variables (FixUpVar_Flux).  *seconds (if not NULL): the wall time
// of the Flu_FixUp_Flux call alone.  Returns 0.
__attribute__((visibility("default")))
int gref_fixup_flux( void *fluid, const char *de, const void *flux, const unsigned char *has_flux, const int NP,
                     const double dh, const long tvar, const double min_dens, const double min_pres,
                     const double min_eint, const double gamma, const int nthreads, double *seconds )
{
   GAMMA = gamma;
   EoS_Init_Gamma();
   if ( amr == NULL )  amr = new AMR_t;
   const int lv = 0;
   amr->dh[lv]    = dh;
   amr->FluSg[lv] = 0;
   amr->NPatchComma[lv][1] = NP;
   MIN_DENS = min_dens;  MIN_PRES = min_pres;  MIN_EINT = min_eint;
#  ifdef DUAL_ENERGY
   PassiveFloorMask = BIDX( DUAL );
#  else
   PassiveFloorMask = 0L;
#  endif
   if ( nthreads > 0 )  omp_set_num_threads( nthreads );
   omp_set_schedule( omp_sched_static, 0 );

   const int    BoxScale[3] = { PS1, PS1, PS1 };
   const double BoxEdgeL[3] = { 0.0, 0.0, 0.0 };
   real       (*F )[NCOMP_TOTAL][CUBE(PS1)]           = ( real (*)[NCOMP_TOTAL][CUBE(PS1)] )fluid;
   const real (*FX)[6][NFLUX_TOTAL][SQR(PS1)]          = ( const real (*)[6][NFLUX_TOTAL][SQR(PS1)] )flux;
   for (int p=0; p<NP; p++)
   {
      patch_t *pa = new patch_t( 0, 0, 0, -1, true, false, false, true, lv, BoxScale, BoxEdgeL, dh );
      amr->patch[0][lv][p] = pa;
      for (int v=0; v<NCOMP_TOTAL; v++)
         memcpy( pa->fluid[v], F[p][v], CUBE(PS1)*sizeof(real) );
#     ifdef DUAL_ENERGY
      if ( de != NULL )  memcpy( pa->de_status, de + (long)p*CUBE(PS1), CUBE(PS1) );
#     endif
      for (int s=0; s<6; s++)
      {
         if ( !has_flux[ 6*p + s ] )  continue;
         pa->fnew( s, false );
         memcpy( pa->flux[s], FX[p][s], NFLUX_TOTAL*SQR(PS1)*sizeof(real) );
      }
   }

   const double t0 = omp_get_wtime();
   Flu_FixUp_Flux( lv, tvar );
   if ( seconds != NULL )  *seconds = omp_get_wtime() - t0;

   for (int p=0; p<NP; p++)
   {
      patch_t *pa = amr->patch[0][lv][p];
      for (int v=0; v<NCOMP_TOTAL; v++)
         memcpy( F[p][v], pa->fluid[v], CUBE(PS1)*sizeof(real) );
      delete pa;
      amr->patch[0][lv][p] = NULL;
   }
   amr->NPatchComma[lv][1] = 0;
   return 0;
}

} // extern "C"
