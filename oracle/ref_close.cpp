// Test infrastructure only: the reference's CorrectUnphysical() as an oracle.
//
// CorrectUnphysical (src/Fluid/Flu_Close.cpp:542-1200) is a file-static function of the reference's
// Flu_Close.cpp, so this translation unit includes that file, unmodified and read where it lies
// (its path arrives as the macro GREF_FLU_CLOSE from oracle/build_ref.sh), and exports one plain C
// function that calls it on caller-owned arrays.  It also defines the globals that Flu_Close.cpp
// expects from the rest of GAMER (src/Main/Main.cpp, src/Fluid/Flu_AdvanceDt.cpp) and stubs the
// two routines it calls only to abort or to dump a failed patch (Aux_Error, Output_Patch).
//
// Linked into the same library as oracle/ref_stub.cpp (hydro MHM variants, and the CTU+MHD variant,
// where gref_correct_unphysical_mhd passes the face-centred magnetic field of the MHD branch).
// Nothing in the product links this file.

#include <stdexcept>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include GREF_FLU_CLOSE

// ---- globals normally defined by src/Main/Main.cpp and src/Fluid/Flu_AdvanceDt.cpp ------------
AMR_t  *amr = NULL;
double  Time[NLEVEL];
long    Step = 0, AdvanceCounter[NLEVEL], NCorrUnphy[NLEVEL];
int     MPI_Rank = 0;
char    OUTPUT_DIR[MAX_STRING] = ".";
char    FieldLabel[NCOMP_TOTAL][MAX_STRING];
double  MIN_DENS = 0.0, MIN_PRES = 0.0, MIN_EINT = 0.0, UNIT_V = 1.0;
double  DUAL_ENERGY_SWITCH = 2.0e-2;
long    PassiveFloorMask = 0L;
bool    AUTO_REDUCE_DT = false, OPT__FIXUP_FLUX = true, OPT__LAST_RESORT_FLOOR = true;
bool    OPT__NORMALIZE_PASSIVE = false;
int     PassiveNorm_NVar = 0, PassiveNorm_VarIdx[NCOMP_PASSIVE];
int     OPT__CHECK_PRES_AFTER_FLU = 0;
Opt1stFluxCorr_t OPT__1ST_FLUX_CORR        = FIRST_FLUX_CORR_3D;
OptRSolver1st_t  OPT__1ST_FLUX_CORR_SCHEME = RSOLVER_1ST_HLLE;
real   *h_EoS_Table[EOS_NTABLE_MAX];
#ifdef MHD
char    MagLabel[NCOMP_MAG][MAX_STRING];
bool    OPT__FIXUP_ELECTRIC = true;
#endif
int     FluStatus_ThisRank = GAMER_SUCCESS;
bool    AutoReduceDt_Continue = false;

extern double GAMMA;
void EoS_Init_Gamma();

// Aux_Error ends the program in the reference; here it ends the call with status 2
void Aux_Error( const char *File, const int Line, const char *Func, const char *Format, ... )
{
   char msg[512];
   va_list ap;
   va_start( ap, Format );
   vsnprintf( msg, sizeof(msg), Format, ap );
   va_end( ap );
   throw std::runtime_error( msg );
}

static int g_NOutputPatch = 0;
void Output_Patch( const int lv, const int PID, const int FluSg, const int MagSg, const int PotSg,
                   const char *comment )
{
   g_NOutputPatch ++;
}

// the set-up of the globals CorrectUnphysical() reads, then one call of it
static int run_correct( const void *flu_in, void *flu_out, char *de_out, void *flux, const void *mag_in,
                        const void *mag_out, const int NPG, const double dt, const double dh, const int corr,
                        const int scheme, const int fixup_flux, const int last_resort_floor,
                        const int auto_reduce_dt_continue, const int check_pres_after_flu,
                        const double min_dens, const double min_pres, const double min_eint,
                        const double de_switch, const double gamma, const char *outdir, const int nthreads,
                        long *ncorr )
{
   GAMMA = gamma;
   EoS_Init_Gamma();
   if ( amr == NULL )  amr = new AMR_t;
   amr->dh[0] = dh;
   MIN_DENS = min_dens;  MIN_PRES = min_pres;  MIN_EINT = min_eint;  DUAL_ENERGY_SWITCH = de_switch;
#  ifdef DUAL_ENERGY
   PassiveFloorMask = BIDX( DUAL );
#  else
   PassiveFloorMask = 0L;
#  endif
   OPT__1ST_FLUX_CORR        = corr;
   OPT__1ST_FLUX_CORR_SCHEME = scheme;
   OPT__FIXUP_FLUX           = fixup_flux != 0;
   OPT__LAST_RESORT_FLOOR    = last_resort_floor != 0;
   OPT__CHECK_PRES_AFTER_FLU = check_pres_after_flu;
   AUTO_REDUCE_DT            = auto_reduce_dt_continue != 0;
   AutoReduceDt_Continue     = auto_reduce_dt_continue != 0;
   FluStatus_ThisRank        = GAMER_SUCCESS;
   NCorrUnphy[0]             = 0;
   if ( outdir != NULL )  snprintf( OUTPUT_DIR, MAX_STRING, "%s", outdir );
   if ( nthreads > 0 )  omp_set_num_threads( nthreads );
   omp_set_schedule( omp_sched_static, 0 );

   int *PID0_List = new int [ ( NPG > 0 ) ? NPG : 1 ];
   for (int t=0; t<NPG; t++)  PID0_List[t] = 8*t;

   typedef real FluIn_t  [FLU_NIN ][ CUBE(FLU_NXT) ];
   typedef real FluOut_t [FLU_NOUT][ CUBE(PS2) ];
   typedef char DE_t     [ CUBE(PS2) ];
   typedef real Flux_t   [9][NFLUX_TOTAL][ SQR(PS2) ];
   typedef real MagIn_t  [NCOMP_MAG][ FLU_NXT_P1*SQR(FLU_NXT) ];
   typedef real MagOut_t [NCOMP_MAG][ PS2P1*SQR(PS2) ];
   int rc = 0;
   try
   {
      CorrectUnphysical( 0, NPG, PID0_List, (const FluIn_t*)flu_in, (FluOut_t*)flu_out, (DE_t*)de_out,
                         (Flux_t*)flux, (const MagIn_t*)mag_in, (const MagOut_t*)mag_out, (real)dt );
      if ( FluStatus_ThisRank == GAMER_FAILED )  rc = 1;
   }
   catch ( const std::exception & )
   {
      rc = 2;
   }
   delete [] PID0_List;
   if ( ncorr != NULL )  *ncorr = NCorrUnphy[0];
   return rc;
}

extern "C" {

// CorrectUnphysical() on NPG patch groups of level 0 with cell size dh:
//    flu_in [NPG][NCOMP_TOTAL][FLU_NXT^3]   flu_out[NPG][NCOMP_TOTAL][PS2^3]   (corrected in place)
//    de_out [NPG][PS2^3] (DUAL_ENERGY builds) flux [NPG][9][NCOMP_TOTAL][PS2^2]  (patched in place)
// corr: OPT__1ST_FLUX_CORR (0 none, 1 3D, 2 3D1D); scheme: OPT__1ST_FLUX_CORR_SCHEME (1 Roe,
// 2 HLLC, 3 HLLE, 4 HLLD).  Debug dumps of failed cells go to outdir.  Returns 0 if every cell is
// physical afterwards, 1 if some cell failed while auto_reduce_dt_continue is set
// (FluStatus_ThisRank = GAMER_FAILED), 2 if the reference would have aborted; *ncorr = cells
// corrected.
__attribute__((visibility("default")))
int gref_correct_unphysical( const void *flu_in, void *flu_out, char *de_out, void *flux, const int NPG,
                             const double dt, const double dh, const int corr, const int scheme,
                             const int fixup_flux, const int last_resort_floor,
                             const int auto_reduce_dt_continue, const int check_pres_after_flu,
                             const double min_dens, const double min_pres, const double min_eint,
                             const double de_switch, const double gamma, const char *outdir,
                             const int nthreads, long *ncorr )
{
#  ifdef MHD
   return 2;      // the MHD branch needs the magnetic field: gref_correct_unphysical_mhd
#  else
   return run_correct( flu_in, flu_out, de_out, flux, NULL, NULL, NPG, dt, dh, corr, scheme, fixup_flux,
                       last_resort_floor, auto_reduce_dt_continue, check_pres_after_flu, min_dens, min_pres,
                       min_eint, de_switch, gamma, outdir, nthreads, ncorr );
#  endif
}

#ifdef MHD
// The same with the face-centred magnetic field of the MHD branch:
//    mag_in [NPG][3][(FLU_NXT+1)*FLU_NXT^2]   mag_out [NPG][3][(PS2+1)*PS2^2]
__attribute__((visibility("default")))
int gref_correct_unphysical_mhd( const void *flu_in, const void *mag_in, void *flu_out, const void *mag_out,
                                 void *flux, const int NPG, const double dt, const double dh, const int corr,
                                 const int scheme, const int fixup_flux, const int last_resort_floor,
                                 const int auto_reduce_dt_continue, const int check_pres_after_flu,
                                 const double min_dens, const double min_pres, const double min_eint,
                                 const double gamma, const char *outdir, const int nthreads, long *ncorr )
{
   return run_correct( flu_in, flu_out, NULL, flux, mag_in, mag_out, NPG, dt, dh, corr, scheme, fixup_flux,
                       last_resort_floor, auto_reduce_dt_continue, check_pres_after_flu, min_dens, min_pres,
                       min_eint, 0.0, gamma, outdir, nthreads, ncorr );
}
#endif

} // extern "C"
