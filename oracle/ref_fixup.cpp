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
// In the CTU+MHD variant the patches also carry the face-centred magnetic field (patch_t::magnetic,
// read by Flu_FixUp_Flux for the magnetic energy), and gref_fixup_electric runs the reference's
// MHD_FixUp_Electric() (src/Model_Hydro/MHD_FixUp_Electric.cpp:22) on patches built the same way.
//
// Nothing in the product links this file.

#include "GAMER.h"

extern double GAMMA;
void EoS_Init_Gamma();
void Flu_FixUp_Flux( const int lv, const long TVar );
#ifdef MHD
void MHD_FixUp_Electric( const int lv );
#endif

// patch_t::Activate derives a patch's padded-cell and load-balance indices from its corner
// (src/Miscellaneous/Mis_Idx3D2Idx1D.cpp, src/LoadBalance/LB_Corner2Index.cpp); the fix-up reads
// neither, so the batch's patches take index 0
ulong Mis_Idx3D2Idx1D( const int Size[], const int Idx3D[] )  { return 0; }
long  LB_Corner2Index( const int lv, const int Corner[], const Check_t Check )  { return 0; }

// the physical set-up shared by the entry points
static void set_level( const double dh, const double min_dens, const double min_pres, const double min_eint,
                       const double gamma, const int nthreads )
{
   GAMMA = gamma;
   EoS_Init_Gamma();
   if ( amr == NULL )  amr = new AMR_t;
   const int lv = 0;
   amr->dh[lv]    = dh;
   amr->FluSg[lv] = 0;
#  ifdef MHD
   amr->MagSg[lv] = 0;
#  endif
   MIN_DENS = min_dens;  MIN_PRES = min_pres;  MIN_EINT = min_eint;
#  ifdef DUAL_ENERGY
   PassiveFloorMask = BIDX( DUAL );
#  else
   PassiveFloorMask = 0L;
#  endif
   if ( nthreads > 0 )  omp_set_num_threads( nthreads );
   omp_set_schedule( omp_sched_static, 0 );
}

static patch_t *new_patch( const double dh, const bool mag )
{
   const int    BoxScale[3] = { PS1, PS1, PS1 };
   const double BoxEdgeL[3] = { 0.0, 0.0, 0.0 };
   return new patch_t( 0, 0, 0, -1, true, mag, false, true, 0, BoxScale, BoxEdgeL, dh );
}

#ifdef MHD
typedef real Mag_t[NCOMP_MAG][ PS1P1*SQR(PS1) ];
#endif

static int run_fixup_flux( void *fluid, const char *de, const void *flux, const unsigned char *has_flux,
                           const void *magnetic, const int NP, const double dh, const long tvar,
                           const double min_dens, const double min_pres, const double min_eint,
                           const double gamma, const int nthreads, double *seconds )
{
   set_level( dh, min_dens, min_pres, min_eint, gamma, nthreads );
   const int lv = 0;
   amr->NPatchComma[lv][1] = NP;

   real       (*F )[NCOMP_TOTAL][CUBE(PS1)]           = ( real (*)[NCOMP_TOTAL][CUBE(PS1)] )fluid;
   const real (*FX)[6][NFLUX_TOTAL][SQR(PS1)]          = ( const real (*)[6][NFLUX_TOTAL][SQR(PS1)] )flux;
   for (int p=0; p<NP; p++)
   {
      patch_t *pa = new_patch( dh, magnetic != NULL );
      amr->patch[0][lv][p] = pa;
      for (int v=0; v<NCOMP_TOTAL; v++)
         memcpy( pa->fluid[v], F[p][v], CUBE(PS1)*sizeof(real) );
#     ifdef MHD
      if ( magnetic != NULL )
         for (int v=0; v<NCOMP_MAG; v++)
            memcpy( pa->magnetic[v], ( (const Mag_t*)magnetic )[p][v], PS1P1*SQR(PS1)*sizeof(real) );
#     endif
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

extern "C" {

// fluid   [NP][NCOMP_TOTAL][PS1^3]  corrected in place
// de      [NP][PS1^3] (DUAL_ENERGY builds; may be NULL otherwise)
// flux    [NP][6][NCOMP_TOTAL][PS1^2]  the flux differences of the six faces
// has_flux[NP][6]  1 where the face carries a flux array (patch_t::flux[s] != NULL)
// tvar: the bit mask of corrected variables (FixUpVar_Flux).  *seconds (if not NULL): the wall time
// of the Flu_FixUp_Flux call alone.  Returns 0 (2 in an MHD build, which needs the magnetic field:
// gref_fixup_flux_mhd).
__attribute__((visibility("default")))
int gref_fixup_flux( void *fluid, const char *de, const void *flux, const unsigned char *has_flux, const int NP,
                     const double dh, const long tvar, const double min_dens, const double min_pres,
                     const double min_eint, const double gamma, const int nthreads, double *seconds )
{
#  ifdef MHD
   return 2;
#  else
   return run_fixup_flux( fluid, de, flux, has_flux, NULL, NP, dh, tvar, min_dens, min_pres, min_eint, gamma,
                          nthreads, seconds );
#  endif
}

#ifdef MHD
// The same with the patches' face-centred magnetic field, magnetic [NP][3][(PS1+1)*PS1^2].
__attribute__((visibility("default")))
int gref_fixup_flux_mhd( void *fluid, const void *magnetic, const void *flux, const unsigned char *has_flux,
                         const int NP, const double dh, const long tvar, const double min_dens,
                         const double min_pres, const double min_eint, const double gamma, const int nthreads,
                         double *seconds )
{
   return run_fixup_flux( fluid, NULL, flux, has_flux, magnetic, NP, dh, tvar, min_dens, min_pres, min_eint,
                          gamma, nthreads, seconds );
}

// MHD_FixUp_Electric() on NP patches of one level:
//    magnetic        [NP][3][(PS1+1)*PS1^2]   corrected in place
//    electric,
//    electric_bitrep [NP][GREF_ELE_PER_PATCH]  patch_t::electric[s] / electric_bitrep[s] of the 18
//                                             sides packed: face s < 6 at s*2*(PS1-1)*PS1
//                                             ([2][(PS1-1)*PS1]), edge s >= 6 at
//                                             6*2*(PS1-1)*PS1 + (s-6)*PS1 ([PS1]); zeroed on return
//                                             where present, as the reference leaves them
//    has_ele         [NP][18]  1 where the side carries electric arrays (patch_t::electric[s] != NULL)
//    sib_leaf        [NP][6]   1 where the sibling across face s is a leaf patch (son == -1), 0 where
//                              it has children
// Returns 0.
#define GREF_ELE_PER_PATCH ( 6*NCOMP_ELE*PS1M1*PS1 + 12*PS1 )
__attribute__((visibility("default")))
int gref_fixup_electric( void *magnetic, void *electric, void *electric_bitrep, const unsigned char *has_ele,
                         const unsigned char *sib_leaf, const int NP, const double dh, const int nthreads,
                         double *seconds )
{
   set_level( dh, 0.0, 0.0, 0.0, 5.0/3.0, nthreads );
   const int lv = 0;
   // two sibling stand-ins after the batch: a leaf patch (son -1) and a patch with children
   const int LEAF = NP, PARENT = NP + 1;
   for (int p=0; p<NP+2; p++)
   {
      patch_t *pa = new_patch( dh, p < NP );
      amr->patch[0][lv][p] = pa;
   }
   amr->patch[0][lv][LEAF  ]->son = -1;
   amr->patch[0][lv][PARENT]->son =  1;
   amr->NPatchComma[lv][1]  = NP;
   amr->NPatchComma[lv][27] = NP;
   amr->WithElectric = true;

   Mag_t *M  = (Mag_t*)magnetic;
   real  *E  = (real*)electric;
   real  *EB = (real*)electric_bitrep;
   for (int p=0; p<NP; p++)
   {
      patch_t *pa = amr->patch[0][lv][p];
      for (int v=0; v<NCOMP_MAG; v++)  memcpy( pa->magnetic[v], M[p][v], PS1P1*SQR(PS1)*sizeof(real) );
      for (int s=0; s<6; s++)  pa->sibling[s] = sib_leaf[ 6*p + s ] ? LEAF : PARENT;
      for (int s=0; s<18; s++)
      {
         if ( !has_ele[ 18*p + s ] )  continue;
         pa->enew( s, false );
         const int  size = ( s < 6 ) ? NCOMP_ELE*PS1M1*PS1 : PS1;
         const long off  = (long)p*GREF_ELE_PER_PATCH + ( ( s < 6 ) ? s*NCOMP_ELE*PS1M1*PS1
                                                                    : 6*NCOMP_ELE*PS1M1*PS1 + (s-6)*PS1 );
         memcpy( pa->electric       [s], E  + off, size*sizeof(real) );
         memcpy( pa->electric_bitrep[s], EB + off, size*sizeof(real) );
      }
   }

   const double t0 = omp_get_wtime();
   MHD_FixUp_Electric( lv );
   if ( seconds != NULL )  *seconds = omp_get_wtime() - t0;

   for (int p=0; p<NP+2; p++)
   {
      patch_t *pa = amr->patch[0][lv][p];
      if ( p < NP )
      {
         for (int v=0; v<NCOMP_MAG; v++)  memcpy( M[p][v], pa->magnetic[v], PS1P1*SQR(PS1)*sizeof(real) );
         for (int s=0; s<18; s++)
         {
            if ( pa->electric[s] == NULL )  continue;
            const int  size = ( s < 6 ) ? NCOMP_ELE*PS1M1*PS1 : PS1;
            const long off  = (long)p*GREF_ELE_PER_PATCH + ( ( s < 6 ) ? s*NCOMP_ELE*PS1M1*PS1
                                                                       : 6*NCOMP_ELE*PS1M1*PS1 + (s-6)*PS1 );
            memcpy( E  + off, pa->electric       [s], size*sizeof(real) );
            memcpy( EB + off, pa->electric_bitrep[s], size*sizeof(real) );
         }
      }
      delete pa;
      amr->patch[0][lv][p] = NULL;
   }
   amr->NPatchComma[lv][1]  = 0;
   amr->NPatchComma[lv][27] = 0;
   return 0;
}
#endif // #ifdef MHD

} // extern "C"
