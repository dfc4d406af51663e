/* gamer_b200_fluid.h — C ABI of the B200 patch-group fluid solver.
 *
 * Drop-in for GAMER's patch-group fluid solver call:
 *    CPU_FluidSolver()         src/Fluid/CPU_FluidSolver.cpp:210-232
 *    CUAPI_Asyn_FluidSolver()  src/GPU_API/CUAPI_Asyn_FluidSolver.cu:266-288
 * Array layouts are GAMER's (x fastest, IDX321 of include/Macro.h:1197):
 *    Flu_Array_In  [NPG][NCOMP_TOTAL][FLU_NXT^3]          Flu_Array_Out [NPG][NCOMP_TOTAL][PS2^3]
 *    Flux_Array    [NPG][9][NCOMP_TOTAL][PS2^2]           DE_Array_Out  [NPG][PS2^3]  (char)
 *    Mag_Array_In  [NPG][3][(FLU_NXT+1)*FLU_NXT^2]        Mag_Array_Out [NPG][3][(PS2+1)*PS2^2]
 *    Ele_Array     [NPG][9][NCOMP_ELE][(PS2+1)*PS2]
 * with PS2 = 16 and NCOMP_TOTAL = 5 (+ npassive_user, +1 with dual energy).  The element type ("real") is float
 * for GB_PREC_FP32 / GB_PREC_MIXED and double for GB_PREC_FP64 (GAMER's FLOAT8 build).
 *
 * Every function returns GB_OK (0) or a negative GB_E* code and never aborts; kernel-side
 * conditions are reported through gb_fluid_get_status().  Streams are passed as void*
 * (a cudaStream_t; NULL = the legacy default stream).
 */
#ifndef GAMER_B200_FLUID_H
#define GAMER_B200_FLUID_H

#ifdef __cplusplus
extern "C" {
#endif

/* scheme / reconstruction / Riemann solver / dual-energy codes: same values as the reference's
 * compile-time macros (include/Macro.h:73-94) */
#define GB_SCHEME_MHM      3
#define GB_SCHEME_MHM_RP   4
#define GB_SCHEME_CTU      5
#define GB_LR_PLM          1
#define GB_LR_PPM          2
#define GB_RSOLVER_EXACT   1
#define GB_RSOLVER_ROE     2
#define GB_RSOLVER_HLLE    3
#define GB_RSOLVER_HLLC    4
#define GB_RSOLVER_HLLD    5
#define GB_DE_NONE         0
#define GB_DE_ENPY         1
/* slope limiters: include/Typedef.h:184-194 */
#define GB_LIM_VANLEER     1
#define GB_LIM_GMINMOD     2
#define GB_LIM_ALBADA      3
#define GB_LIM_VL_GMINMOD  4
#define GB_LIM_CENTRAL     6
/* arithmetic policies */
#define GB_PREC_FP32       0   /* float arrays, float arithmetic */
#define GB_PREC_MIXED      1   /* float arrays; E-1/2 m^2/rho recovery, dual-energy selection and
                                  flux-difference accumulation in double */
#define GB_PREC_FP64       2   /* double arrays and arithmetic */

/* return codes */
#define GB_OK               0
#define GB_E_INVALID       -1   /* bad argument (NULL pointer, size, unsupported combination) */
#define GB_E_ALIGN         -2   /* an array is not 16-byte aligned */
#define GB_E_CUDA          -3   /* a CUDA runtime call failed */
#define GB_E_NOMEM         -4   /* device or pinned-host allocation failed */
#define GB_E_UNSUPPORTED   -5   /* configuration not built into this library */

/* status bits accumulated on the device (gb_fluid_get_status) */
#define GB_STATUS_TMA_TIMEOUT  1   /* a bulk-copy wait gave up; outputs of that launch are invalid */
#define GB_STATUS_UNPHYSICAL   2   /* a patch group still had an unphysical cell after all MinMod
                                      retries (GAMER leaves these cells to Flu_Close) */

typedef struct gb_fluid_solver gb_fluid_solver;

/* Compile-time choices of the reference become creation-time choices here. */
typedef struct gb_fluid_config {
   int    scheme;       /* GB_SCHEME_MHM, GB_SCHEME_MHM_RP or GB_SCHEME_CTU, each hydro or MHD; the
                           multi-level entry points take hydro MHM only.  HLLD selects MHD (PLM or PPM in every scheme):
                           the calls then take the magnetic arrays */
   int    lr_scheme;    /* GB_LR_PLM / GB_LR_PPM */
   int    rsolver;      /* GB_RSOLVER_*: hydro HLLC / HLLE / ROE (and EXACT in MHM and CTU), or HLLD
                           for MHD in every scheme */
   int    precision;    /* GB_PREC_* */
   int    dual_energy;  /* GB_DE_NONE / GB_DE_ENPY */
   int    flu_nxt;      /* FLU_NXT of the input arrays: 16 + 2*FLU_GHOST_SIZE of the scheme (20 for
                           MHM+PLM and hydro CTU+PLM, 22 for MHM+PPM, hydro CTU+PPM, MHM_RP+PLM and
                           CTU+MHD+PLM, 24 for MHM_RP+PPM (hydro and MHD) and CTU+MHD+PPM); MHM also takes that
                           plus 2, in which case the central window is read */
   double gamma;        /* GAMMA of the ideal-gas EoS */
   int    char_reconstruction;  /* CHAR_RECONSTRUCTION: limit the slopes in characteristic
                                   variables (MHM with PLM or PPM, MHM_RP and CTU, hydro and MHD;
                                   0 = off, so initialisers that end at gamma keep the
                                   primitive-variable limiter) */
   int    npassive_user;        /* NCOMP_PASSIVE_USER: user passive scalars after the five fluid
                                   variables (0 or GB_NPASSIVE_USER; hydro MHM, MHM_RP, CTU).  With dual energy the
                                   dual-energy field is the last variable, as in the reference
                                   (DUAL = NCOMP_TOTAL-1, include/Macro.h:290-305) */
} gb_fluid_config;

/* user passive scalars built into the hydro MHM, MHM_RP and CTU kernels (NCOMP_PASSIVE_USER of the reference build) */
#define GB_NPASSIVE_USER   2
/* largest NCOMP_PASSIVE (user passive scalars + the dual-energy field) */
#define GB_MAX_PASSIVE     3

/* The run-time scalars of CPU_FluidSolver() (src/Fluid/CPU_FluidSolver.cpp:210-232).  Members after
 * dual_energy_switch may be left zero: that is the reference with JeansMinPres, NormPassive and
 * FracPassive off and no passive scalar floored (GAMER itself floors the dual-energy field:
 * passive_floor = 1 << DUAL, src/Init/Init_Field.cpp). */
typedef struct gb_fluid_params {
   double dt, dh;
   int    store_flux;          /* StoreFlux     */
   int    store_electric;      /* StoreElectric */
   int    lr_limiter;          /* LR_Limiter    */
   double minmod_coeff;        /* MinMod_Coeff  */
   int    minmod_maxiter;      /* MinMod_MaxIter */
   double min_dens, min_pres, min_eint;
   double dual_energy_switch;  /* DualEnergySwitch */
   long long passive_floor;    /* PassiveFloor: bit v set = variable v (v >= 5) floored at TINY_NUMBER */
   int    norm_passive;        /* NormPassive: rescale the NormIdx passive scalars to sum to the density */
   int    nnorm;               /* NNorm */
   int    norm_idx[GB_MAX_PASSIVE];   /* NormIdx: passive indices (0 = first passive scalar) */
   int    frac_passive;        /* FracPassive: reconstruct the FracIdx passive scalars as mass fractions */
   int    nfrac;               /* NFrac */
   int    frac_idx[GB_MAX_PASSIVE];   /* FracIdx */
   int    jeans_min_pres;      /* JeansMinPres: pressure floor JeansMinPres_Coeff*rho^2 in the cell-centred
                                  primitive variables (every scheme) */
   double jeans_min_pres_coeff;       /* JeansMinPres_Coeff */
} gb_fluid_params;

/* Create a solver; replaces the set-up done by CUAPI_SetDevice/CUAPI_SetCache/CUAPI_SetConstMemory/
 * CUAPI_MemAllocate_Fluid (src/Init/Init_GAMER.cpp:73-176).  Uses the current CUDA device. */
int gb_fluid_create( const gb_fluid_config *cfg, gb_fluid_solver **out );
int gb_fluid_destroy( gb_fluid_solver *s );

/* One batch of patch groups on DEVICE arrays, asynchronous on `stream`.  Replaces the kernel launch
 * inside CUAPI_Asyn_FluidSolver (src/GPU_API/CUAPI_Asyn_FluidSolver.cu:539-682).  Unused outputs may be
 * NULL (flux when store_flux == 0, DE without dual energy, magnetic/electric arrays without MHD,
 * ele when store_electric == 0).  CTU replaces CPU_FluidSolver_CTU
 * (src/Model_Hydro/CPU_Hydro/CPU_FluidSolver_CTU.cpp:157-342): hydro (PLM, characteristic tracing,
 * HLLC or HLLE) or MHD (PLM, HLLD with the HLLE rescue, constrained transport; needs mag_in and
 * mag_out).
 * pg_fail (optional, int[npg]) receives 1 for each patch group still unphysical after the retries. */
int gb_fluid_solve_device( gb_fluid_solver *s, const void *flu_in, void *flu_out,
                           const void *mag_in, void *mag_out, char *de_out,
                           void *flux, void *ele, int *pg_fail, int npg,
                           const gb_fluid_params *prm, void *stream );

/* Same on HOST arrays, asynchronous: the whole of CUAPI_Asyn_FluidSolver
 * (src/GPU_API/CUAPI_Asyn_FluidSolver.cu:266-749).  The batch is split into chunks that go
 * round-robin over the solver's own streams (the reference's GPU_NSTREAM split), each chunk as
 * H2D -> solve -> D2H, and the call returns as soon as everything is enqueued; gb_fluid_synchronize(s)
 * ends it.  Calls on one solver may be queued back to back: each chunk runs after the chunks of the
 * earlier calls on its stream, so the copies of one call overlap the kernels of the next, as the
 * reference's own streams do.  `stream` (a cudaStream_t) may be NULL: no ordering with any caller
 * stream, the reference's behaviour.  A non-NULL stream orders the call both ways: its work starts
 * after the work already enqueued on `stream`, and `stream` waits for its completion (so a
 * cudaStreamSynchronize(stream) also ends it).  The host arrays must stay valid and untouched until
 * the call has ended: GAMER prepares the next batch in its other pinned buffer set meanwhile
 * (src/Main/InvokeSolver.cpp:214-245).  Host arrays are best allocated with gb_fluid_host_alloc
 * (pinned); pageable arrays work but are copied synchronously by CUDA. */
int gb_fluid_solve_host_async( gb_fluid_solver *s, const void *flu_in, void *flu_out,
                               const void *mag_in, void *mag_out, char *de_out,
                               void *flux, void *ele, int npg, const gb_fluid_params *prm, void *stream );

/* Wait for every host-array call of this solver: CUAPI_Synchronize (src/GPU_API/CUAPI_Synchronize.cu).
 * Returns GB_E_CUDA if a copy or kernel of those calls failed. */
int gb_fluid_synchronize( gb_fluid_solver *s );

/* gb_fluid_solve_host_async on no external stream followed by gb_fluid_synchronize. */
int gb_fluid_solve_host( gb_fluid_solver *s, const void *flu_in, void *flu_out,
                         const void *mag_in, void *mag_out, char *de_out,
                         void *flux, void *ele, int npg, const gb_fluid_params *prm );

/* All patch groups of several AMR levels in one launch (no reference counterpart: GAMER calls the
 * solver once per level, src/Main/InvokeSolver.cpp:64).  Patch groups of level l occupy
 * [sum(level_npg[0..l-1]), +level_npg[l]) and advance by level_dt[l] with cell size level_dh[l];
 * prm->dt and prm->dh are ignored.  nlevel <= 16. */
int gb_fluid_solve_levels_device( gb_fluid_solver *s, const void *flu_in, void *flu_out, char *de_out,
                                  void *flux, int *pg_fail, int nlevel, const int *level_npg,
                                  const double *level_dt, const double *level_dh,
                                  const gb_fluid_params *prm, void *stream );

/* The same multi-level launch captured once into a CUDA graph (fixed arrays and sizes), replayed
 * with gb_fluid_graph_launch.  gb_fluid_graph_set_dt records the launch again with the new per-level
 * time steps and updates the instantiated graph in place (cudaGraphExecUpdate), so a new sub-step
 * needs no re-instantiation.  No reference counterpart (GAMER launches per level and per stream). */
typedef struct gb_fluid_graph gb_fluid_graph;
int gb_fluid_graph_create_levels( gb_fluid_solver *s, const void *flu_in, void *flu_out, char *de_out,
                                  void *flux, int *pg_fail, int nlevel, const int *level_npg,
                                  const double *level_dt, const double *level_dh,
                                  const gb_fluid_params *prm, gb_fluid_graph **out );
int gb_fluid_graph_set_dt( gb_fluid_graph *g, const double *level_dt );
int gb_fluid_graph_launch( gb_fluid_graph *g, void *stream );
int gb_fluid_graph_destroy( gb_fluid_graph *g );

/* Read (and clear) the accumulated GB_STATUS_* bits; synchronizes the solver's last stream. */
int gb_fluid_get_status( gb_fluid_solver *s, int *status );

/* Pinned host memory for the host-array entry point (the reference allocates its host arrays with
 * cudaMallocHost, src/GPU_API/CUAPI_MemAllocate_Fluid.cu:288-322). */
int gb_fluid_host_alloc( void **ptr, unsigned long long bytes );
int gb_fluid_host_free( void *ptr );

/* Launch shape (threads per CTA) used by the solver; 0 = the tuned default.  Valid: multiples of
 * 32 in [256, 512] (the MHM kernel gives each of a patch group's 16x16 columns its own thread). */
int gb_fluid_set_block_size( gb_fluid_solver *s, int threads );
int gb_fluid_get_block_size( gb_fluid_solver *s, int *threads );

/* The whole launch of the MHM kernel, as gamer_b200/autotune.py tunes it per batch size:
 *    threads        threads per CTA (0 = the tuned default; else as gb_fluid_set_block_size)
 *    ctas_per_sm    at most this many CTAs per SM in the persistent grid (0 = as many as fit; 1-8)
 *    max_registers  the register-capped instantiation of the kernel: 0 (default: 96 per thread in
 *                   float, 255 in FP64), 64, 72, 80 or 128; built for the float policies' MHM +
 *                   PLM + HLLC, 5 variables, FLU_NXT = 20, generalized MinMod (the headline
 *                   kernel); launches of other configurations use their default instantiation
 * Invalid values → GB_E_INVALID; a launch whose shape does not fit an SM fails with GB_E_CUDA. */
int gb_fluid_set_launch( gb_fluid_solver *s, int threads, int ctas_per_sm, int max_registers );
int gb_fluid_get_launch( gb_fluid_solver *s, int *threads, int *ctas_per_sm, int *max_registers );

/* CTU only: patch groups per chunk of its multi-kernel pipeline (0 = default: 2048 in FP32 and
 * mixed, 1024 in FP64; the host-array entry point uses at most 512, to pipeline its copies).
 * Each stream slot holds a device scratch of ~2.8 MB (MHD, FP32; hydro ~1.2 MB; twice that in
 * FP64) per patch group of the largest chunk used so far (a call of fewer patch groups than the
 * chunk needs only those), allocated on first use.  Concurrent calls on one solver share the
 * scratch of the device entry point and must not overlap. */
int gb_fluid_set_mhd_chunk( gb_fluid_solver *s, int npg );

/* CTU + MHD solve that allocates no memory (no counterpart in the reference).  It is for callers
 * that cannot call cudaMalloc: a host code whose device memory is all owned by its own pool
 * allocator (a cudaMalloc would fail or fragment the pool), or a time step that must not pay the
 * device-wide synchronisation cudaMalloc/cudaFree can imply.  gb_fluid_create and the CTU path of
 * gb_fluid_solve_device allocate (status word, streams, scratch); this entry point does not.  No
 * solver object: the configuration is passed per call (CTU, PLM, HLLD, no dual energy,
 * FLU_NXT = 22; any precision).  The pipeline's scratch is a fixed device array of
 * GB_CTU_STATIC_SCRATCH_BYTES (64 MiB) inside the library, which every device that runs this entry
 * point keeps until the process exits, so one call handles at most gb_ctu_mhd_static_capacity()
 * patch groups (23 in FP32/mixed and 11 in FP64 with the current pipeline); a larger npg returns
 * GB_E_INVALID (split the batch).  Nothing in the scratch needs to start at zero: every
 * element a call reads was written earlier in the same call.  The first call on each device looks
 * up the scratch address (cudaGetSymbolAddress, which loads the module); make that call before any
 * stream capture.  The address is that of the device's primary context and is kept for the rest of
 * the process: do not call this entry point on a device after cudaDeviceReset, nor from a context
 * of your own.  All calls on one device share the one scratch: calls that overlap in time (other
 * streams or host threads) race and give wrong results.  Array and parameter meanings and the other
 * error codes are those of gb_fluid_solve_device. */
#define GB_CTU_STATIC_SCRATCH_BYTES  67108864ull
int gb_ctu_mhd_solve_static( const gb_fluid_config *cfg, const void *flu_in, const void *mag_in,
                             void *flu_out, void *mag_out, void *flux, void *ele, int npg,
                             const gb_fluid_params *prm, void *stream );
/* Largest npg one gb_ctu_mhd_solve_static call takes for this precision (GB_PREC_*): the fixed
 * scratch over the pipeline's scratch per patch group.  No reference counterpart. */
int gb_ctu_mhd_static_capacity( int precision, int *npg );

/* CFL time step per patch: dt[p] = safety*dh / max over the 8^3 cells and 3 directions of
 * |v_d| + c_d (sound speed, or the fast magnetosonic speed along d with MHD).  Replaces
 * CUFLU_dtSolver_HydroCFL (src/Model_Hydro/CPU_Hydro/CPU_dtSolver_HydroCFL.cpp:57-233); the caller
 * takes the minimum as GAMER's dt_Close does.  Only cfg->scheme (CTU = MHD), precision, dual_energy
 * and gamma are used.  Asynchronous on `stream`.
 *   gb_dt_cfl_device: GAMER's dt arrays, flu [npatch][5][8^3], mag [npatch][3][9*8*8] (MHD), dt [npatch]
 *   gb_dt_cfl_from_output_device: the fluid solver's own outputs flu_out [npg][NCOMP][16^3] and
 *     mag_out [npg][3][17*16*16]; dt [8*npg] with the 8 patches of each group in GAMER's LocalID
 *     order (src/Tables/Table_02.cpp) -- no host-side dt_Prepare_Flu repacking (no reference
 *     counterpart). */
int gb_dt_cfl_device( const gb_fluid_config *cfg, const void *flu, const void *mag, void *dt, int npatch,
                      double dh, double safety, double min_pres, void *stream );
int gb_dt_cfl_from_output_device( const gb_fluid_config *cfg, const void *flu_out, const void *mag_out, void *dt,
                                  int npg, double dh, double safety, double min_pres, void *stream );

/* First-order-flux correction of unphysical cells: CorrectUnphysical() of Flu_Close
 * (src/Fluid/Flu_Close.cpp:542-1200), called from Flu_Close (:98) right after the solver.  The
 * options are the reference's run-time parameters of that step. */
#define GB_FIRST_FLUX_CORR_NONE  0   /* OPT__1ST_FLUX_CORR (include/Typedef.h:461-465) */
#define GB_FIRST_FLUX_CORR_3D    1
#define GB_FIRST_FLUX_CORR_3D1D  2
#define GB_RSOLVER_1ST_ROE       1   /* OPT__1ST_FLUX_CORR_SCHEME (include/Typedef.h:467-474) */
#define GB_RSOLVER_1ST_HLLC      2
#define GB_RSOLVER_1ST_HLLE      3

typedef struct gb_close_params {
   int first_flux_corr;          /* OPT__1ST_FLUX_CORR */
   int first_flux_scheme;        /* OPT__1ST_FLUX_CORR_SCHEME */
   int last_resort_floor;        /* OPT__LAST_RESORT_FLOOR */
   int auto_reduce_dt_continue;  /* AutoReduceDt_Continue (src/Fluid/Flu_AdvanceDt.cpp): floors off,
                                    and the final test checks Eint instead of Etot */
   int check_pres_after_flu;     /* OPT__CHECK_PRES_AFTER_FLU */
} gb_close_params;

/* In place on the device arrays of one gb_fluid_solve_device call (same flu_in, flu_out, de_out,
 * flux and npg, same prm: dt, dh, store_flux = OPT__FIXUP_FLUX, the floors and the dual-energy
 * switch).  Every output cell that fails the reference's Unphysical() test is re-advanced with
 * first-order fluxes and floored; a cell that passes replaces the output (and, with store_flux,
 * its first-order fluxes replace the coarse-fine fluxes it touches), a cell that still fails is
 * left as it was.  counts: DEVICE int[2], incremented by the cells corrected ([0]) and the cells
 * still unphysical ([1]); the reference aborts on [1] > 0 unless auto_reduce_dt_continue is set,
 * in which case it redoes the step with a smaller dt.  Asynchronous on stream.  Hydro (MHM and
 * CTU); a CTU+MHD solver → GB_E_INVALID (it has the call below).  The speed-of-light test of
 * OPT__UNIT is not applied. */
int gb_fluid_correct_unphysical_device( gb_fluid_solver *s, const void *flu_in, void *flu_out, char *de_out,
                                        void *flux, int npg, const gb_fluid_params *prm,
                                        const gb_close_params *cp, int *counts, void *stream );

/* The MHD branch of the same pass (CorrectUnphysical under MHD, src/Fluid/Flu_Close.cpp:542-1200)
 * for a CTU+MHD solver: the arrays of one gb_fluid_solve_device call with its magnetic field,
 *    mag_in  [npg][3][(FLU_NXT+1)*FLU_NXT^2]   mag_out [npg][3][17*16*16]   (read only).
 * Every test includes the cell's magnetic energy from mag_out; the first-order fluxes use the
 * cell-centred input field with the longitudinal component reset to the face value (ResetLongB).
 * first_flux_scheme: 1 Roe, 3 HLLE, 4 HLLD (RSOLVER_1ST_*; HLLC → GB_E_INVALID);
 * first_flux_corr = 2 (3D1D) → GB_E_UNSUPPORTED, as in the reference for MHD.  Any other solver →
 * GB_E_INVALID. */
int gb_fluid_correct_unphysical_mhd_device( gb_fluid_solver *s, const void *flu_in, const void *mag_in,
                                            void *flu_out, const void *mag_out, void *flux, int npg,
                                            const gb_fluid_params *prm, const gb_close_params *cp, int *counts,
                                            void *stream );

/* Coarse-fine flux fix-up: Flu_FixUp_Flux() (src/Fluid/Flu_FixUp_Flux.cpp:23), called per level
 * after the finer level has been advanced (src/Main/EvolveLevel.cpp).  In place on a batch of
 * npatch patches of one level in device memory:
 *    fluid     [npatch][NCOMP][8][8][8]   (the patches' fluid[], FluSg)
 *    de_status [npatch][8][8][8]          (dual energy only; NULL otherwise)
 *    flux      [npatch][6][NCOMP][8][8]   (patch_t::flux[s]: coarse minus fine flux of face s)
 *    has_flux  [npatch][6]                (1 where the face carries a flux difference)
 * prm supplies dh and the floors MIN_DENS / MIN_PRES / MIN_EINT; tvar is FixUpVar_Flux (bit v =
 * correct variable v).  Asynchronous on stream.  Hydro; a CTU+MHD configuration → GB_E_INVALID
 * (it has the call below). */
int gb_flux_fixup_device( const gb_fluid_config *cfg, void *fluid, const char *de_status, const void *flux,
                          const unsigned char *has_flux, int npatch, const gb_fluid_params *prm, long tvar,
                          void *stream );

/* Flu_FixUp_Flux() of an MHD build, for a CTU+MHD configuration: as gb_flux_fixup_device, with the
 * patches' face-centred field magnetic [npatch][3][9*8*8] (patch_t::magnetic, MagSg; read only),
 * whose cell-centred energy enters the internal energy and the rebuilt total energy. */
int gb_flux_fixup_mhd_device( const gb_fluid_config *cfg, void *fluid, const void *magnetic, const void *flux,
                              const unsigned char *has_flux, int npatch, const gb_fluid_params *prm, long tvar,
                              void *stream );

/* Coarse-fine electric-field fix-up: MHD_FixUp_Electric() (src/Model_Hydro/MHD_FixUp_Electric.cpp:22),
 * called per level after the finer level (src/Main/EvolveLevel.cpp:778).  In place on a batch of
 * npatch patches of one level in device memory, for a CTU+MHD configuration (precision from cfg):
 *    magnetic        [npatch][3][9*8*8]          patch_t::magnetic (MagSg), corrected
 *    electric,
 *    electric_bitrep [npatch][GB_ELE_PER_PATCH]  patch_t::electric[s] and electric_bitrep[s] of the
 *                    18 sides packed: face s (0..5) at s*2*56 as [2][7*8], edge s (6..17) at
 *                    672 + (s-6)*8 as [8]; zero on return on every side that has_ele lists
 *                    (the reference zeroes them), with the other slots of such a patch; a patch
 *                    without any listed side is not touched
 *    has_ele         [npatch][18]  1 where the side carries electric arrays (electric[s] != NULL)
 *    sib_leaf        [npatch][6]   1 where the sibling across face s is a leaf patch (son == -1) or
 *                    lies beyond a non-periodic domain boundary (sibling <= SIB_OFFSET_NONPERIODIC)
 * dh is amr->dh[lv].  The result equals the reference's bit for bit.  Asynchronous on stream. */
#define GB_ELE_PER_PATCH ( 6*2*7*8 + 12*8 )
int gb_mhd_fixup_electric_device( const gb_fluid_config *cfg, void *magnetic, void *electric, void *electric_bitrep,
                                  const unsigned char *has_ele, const unsigned char *sib_leaf, int npatch, double dh,
                                  void *stream );

/* Bytes per patch group of each array for this configuration (sizes helpers for callers). */
int gb_fluid_array_bytes( const gb_fluid_solver *s, unsigned long long *in_bytes, unsigned long long *out_bytes,
                          unsigned long long *flux_bytes );

/* The configuration a solver was created with. */
int gb_fluid_get_config( const gb_fluid_solver *s, gb_fluid_config *cfg );

/* ---- adjoint of one solver step (no reference counterpart) ---------------------------------
 * gout [npg][5][16^3] (double) is d loss / d flu_out; gin [npg][5][FLU_NXT^3] (double) receives
 * d loss / d flu_in for the same flu_in.  Supported: MHM + PLM, GMinMod with MinMod_Coeff < 2, no
 * retries, no dual energy, FLU_NXT = 20, GB_PREC_FP32 (double accumulation) or GB_PREC_FP64.
 * The caller provides the device workspace (gb_fluid_adjoint_workspace_bytes per batch; a smaller
 * workspace is used in chunks of patch groups, at least one patch group's worth is required). */
int gb_fluid_adjoint_workspace_bytes( const gb_fluid_solver *s, int npg, unsigned long long *bytes );
int gb_fluid_adjoint_step_device( gb_fluid_solver *s, const void *flu_in, const double *gout, double *gin, int npg,
                                  const gb_fluid_params *prm, void *workspace, unsigned long long ws_bytes,
                                  void *stream );

/* ---- periodic uniform box <-> patch-group windows (single-level ghost-zone fill) -------------
 * box [ncomp][16*npz][16*npy][16*npx] (x fastest); patch group p = (pz*npy + py)*npx + px;
 * windows [npg][ncomp][nxt^3] with ghost width (nxt-16)/2, wrapped periodically.  The adjoints take
 * and return double arrays. */
int gb_box_gather_device( const void *box, void *windows, int npx, int npy, int npz, int nxt, int ncomp,
                          int precision, void *stream );
int gb_box_scatter_device( const void *pg_out, void *box, int npx, int npy, int npz, int ncomp, int precision,
                           void *stream );
int gb_box_gather_adjoint_device( const double *wbar, double *boxbar, int npx, int npy, int npz, int nxt, int ncomp,
                                  void *stream );
int gb_box_scatter_adjoint_device( const double *boxbar, double *outbar, int npx, int npy, int npz, int ncomp,
                                   void *stream );

/* ---- coarse-to-fine interpolation of the AMR ghost-zone fill and refinement --------------------
 * Interpolate() (src/Interpolation/Interpolate.cpp:90-206) for a batch of nbatch independent regions
 * of one shape: cdata [nbatch][ncomp][csize_z][csize_y][csize_x] (x fastest), fdata
 * [nbatch][ncomp][fsize_z][fsize_y][fsize_x].  The coarse cells cstart .. cstart+crange-1 (x, y, z)
 * are interpolated into the fine cells fstart .. fstart+2*crange-1; other fine cells are untouched.
 * The region must keep the scheme's CGhost coarse cells (1; 2 for the quartic schemes) inside cdata
 * (Int_Table, src/Interpolation/Int_Table.cpp).  GB_INTERP_PLAIN interpolates with mono_coeff;
 * GB_INTERP_ITERATE is Interpolate_Iterate (:208-560, with the reference's INTERP_MASK), the path of
 * GAMER's hydro ghost-zone fill (src/Main/InterpolateGhostZone.cpp:1805): ncomp = 5 conserved hydro
 * variables, fstart = 0; a parent with an unphysical child is interpolated again in primitive
 * variables (int_prim) and then with the coefficient reduced mono_max_iter times; a parent that still
 * fails sets GB_INTERP_FAILED in *status (the reference aborts the run there).  As in the reference,
 * ITERATE with int_prim = 0 and mono_max_iter = 0 is the plain interpolation.  Asynchronous on stream. */
#define GB_INT_MINMOD3D    1   /* IntScheme_t (include/Typedef.h:171-180) */
#define GB_INT_MINMOD1D    2
#define GB_INT_VANLEER     3
#define GB_INT_CQUAD       4
#define GB_INT_QUAD        5
#define GB_INT_CQUAR       6
#define GB_INT_QUAR        7
#define GB_INTERP_PLAIN    0
#define GB_INTERP_ITERATE  1
#define GB_INTERP_FAILED   1   /* status bit */

typedef struct gb_interp_params {
   int      scheme;              /* GB_INT_* (INT_SPECTRAL is not built: GB_E_UNSUPPORTED) */
   int      precision;           /* GB_PREC_FP32 (float arrays) or GB_PREC_FP64 (double) */
   int      ncomp;               /* NComp */
   int      csize[3], cstart[3], crange[3];   /* CSize, CStart, CRange (x, y, z) */
   int      fsize[3], fstart[3];              /* FSize, FStart */
   unsigned monotonic;           /* bit v: Monotonic[v] */
   double   mono_coeff;          /* INT_MONO_COEFF */
   int      opp_sign_0th_order;  /* OppSign0thOrder (INT_OPP_SIGN_0TH_ORDER) */
   int      mode;                /* GB_INTERP_PLAIN or GB_INTERP_ITERATE */
   int      int_prim;            /* ITERATE: OPT__INT_PRIM */
   int      mono_max_iter;       /* ITERATE: MONO_MAX_ITER (0 = INT_FIX_MONO_COEFF) */
   double   gamma, min_pres;     /* ITERATE: GAMMA, MIN_PRES */
   int     *status;              /* ITERATE: device int, GB_INTERP_FAILED OR-ed in */
} gb_interp_params;
int gb_interpolate_device( const gb_interp_params *p, const void *cdata, void *fdata, int nbatch, void *stream );

/* Window assembly of the ghost-zone fill (Prepare_PatchData, src/Main/Prepare_PatchData.cpp, for one
 * level): windows [npg][ncomp][nxt^3] (ghost width (nxt-16)/2 <= 16) take their 16^3 interior from
 * fine [npg][ncomp][16^3] and each of the 26 ghost regions from the same-level patch group across that
 * side, nbr[p][s] (the adjacent cells of its interior), or, where nbr[p][s] < 0, from cint
 * [npg][ncomp][nxt^3]: the window interpolated from the coarse level (gb_interpolate_device with the
 * parents of the window as the coarse range; its values depend only on each parent's neighbourhood,
 * so they equal the reference's side-by-side InterpolateGhostZone calls).  Side s = (dz+1)*9 +
 * (dy+1)*3 + (dx+1) with d in {-1, 0, +1} (s = 13 is the interior and is not read); nbr is a device
 * int [npg][27].  cint may be NULL when no side is coarse; a coarse side without cint, or a neighbour
 * index >= npg, reads NaN.  Asynchronous on stream. */
int gb_assemble_windows_device( const void *fine, const int *nbr, const void *cint, void *windows, int npg, int ncomp,
                                int nxt, int precision, void *stream );

const char *gb_fluid_strerror( int code );
int gb_fluid_version( void );

#ifdef __cplusplus
}
#endif

#endif /* GAMER_B200_FLUID_H */
