/*
 * fc2d_b200.h -- C ABI of the B200 (sm_100a) clawpack 4.6 patch-update package.
 *
 * A drop-in for ForestClaw's per-patch wave-propagation update, the ghost fill
 * around it and the conservative fine/coarse correction.  All leaf patches of a
 * forest live in device memory in level-major slabs; the entry points below are
 * the batched equivalents of the reference's patch / clawpatch / clawpack46
 * vtable calls.  Every function returns 0 on success and a negative
 * FC2D_B200_E* code on failure; fc2d_b200_last_error() describes the failure.
 *
 * Host arrays of patch data use the reference's FArrayBox layout per patch
 * (fclaw2d_clawpatch.hpp:46-81; Fortran order q(1-mbc:mx+mbc, 1-mbc:my+mbc, meqn)),
 * patches concatenated in level-major order (level, then block, then Morton
 * order within the block).
 */
#ifndef FC2D_B200_H
#define FC2D_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FC2D_B200_OK          0
#define FC2D_B200_EINVAL     -1   /* bad argument or option combination */
#define FC2D_B200_ECUDA      -2   /* CUDA runtime error */
#define FC2D_B200_ESTATE     -3   /* call made in the wrong state */
#define FC2D_B200_EDEVICE    -4   /* device status word reported a kernel-side failure */
#define FC2D_B200_EFOREST    -5   /* forest is not 2:1 balanced / adapt failed */

/* Riemann solvers compiled into the package as __device__ functions.  They are
 * registered by id, the way cudaclaw apps register __device__ function pointers
 * (fc2d_cudaclaw.h:156-162, fc2d_cudaclaw_cuda.h:52-73); the ids select a
 * compile-time specialisation of the fused update so the solver inlines. */
#define FC2D_B200_RP_ADVECTION   0   /* clawpack46_rpn2adv.f / clawpack46_rpt2adv.f */
#define FC2D_B200_RP_SW_ROE      1   /* shallow/2d/rp/clawpack46_rpn2.f / clawpack46_rpt2.f (Roe + HH fix) */
#define FC2D_B200_RP_SW_FWAVE    2   /* shallow/2d/rp/rpn2_tsunami.f90 / rpt2_tsunami.f90 (f-waves, bathymetry) */
#define FC2D_B200_RP_EULER_EXACT 3   /* Euler, exact Riemann solver (Newton on p*) + clawpack46_rpt2_euler4.f transverse */
#define FC2D_B200_RP_ADVECTION_MANIFOLD 4   /* advection/2d/all/clawpack46_rpn2adv_manifold.f / _rpt2adv_manifold.f
                                               (aux = capacity, x-edge and y-edge normal velocities) */
#define FC2D_B200_RP_USER      100   /* application __device__ solvers installed by fc2d_b200_set_user_variants
                                        (include/fc2d_b200_user.cuh); FP64, no time sync */

/* Built-in application callbacks (qinit / setaux / b4step2 / tagging). */
#define FC2D_B200_APP_NONE       0   /* q and aux supplied by the caller */
#define FC2D_B200_APP_SWIRL      1   /* advection/2d/swirl */
#define FC2D_B200_APP_RADIALDAM  2   /* shallow/2d/radialdam (cell-centre disc) */
#define FC2D_B200_APP_TSUNAMI    3   /* bathymetry + Gaussian bumps */
#define FC2D_B200_APP_SHOCKBUBBLE 4  /* euler/2d/shockbubble: Mach-M shock, light bubble, inflow on the left */
#define FC2D_B200_APP_SPHERE     5   /* advection/2d/sphere: cubed sphere (6 blocks, manifold metric on the device),
                                        solid-body rotation, two Gaussians; pdata = axis[3], omega, centre 1[3],
                                        centre 2[3], width, background; minmax tagging */

/* Arithmetic of the update kernel. */
#define FC2D_B200_PREC_FP64      0   /* FP64 throughout, no FMA contraction (bitwise with the FP64 CPU path) */
#define FC2D_B200_PREC_FP32WAVE  1   /* FP32 waves/limiter/transverse, FP64 q accumulation */

typedef struct fc2d_b200_options {
    /* clawpatch options (fclaw2d_clawpatch_options.c) */
    int mx, my, mbc, meqn, maux;
    /* clawpack46 options (fc2d_clawpack46_options.c:37-99) */
    int mwaves;
    int order[2];          /* method(2), method(3) */
    int mthlim[8];
    int mthbc[4];
    int mcapa;
    int use_fwaves;
    int rp;                /* FC2D_B200_RP_* */
    /* forest / time stepping options (fclaw_options.c:93-220) */
    int minlevel, maxlevel;
    int subcycle;
    int time_sync, flux_correction, fluctuation_correction;
    double refine_threshold, coarsen_threshold;
    double ax, bx, ay, by;
    int mi, mj;            /* brick of mi x mj equally oriented blocks */
    /* application */
    int app;               /* FC2D_B200_APP_* */
    double grav, tperiod;
    double r0, hin, hout, x0, y0;
    double pdata[32];
    /* Euler: gas constant, shock Mach number, bubble density (bubble centre and
     * radius in x0, y0, r0), Newton tolerance on the relative change of p* */
    double gamma, mach, rhob, newton_tol;
    /* B200 specifics */
    int precision;         /* FC2D_B200_PREC_* */
    int device;            /* CUDA device ordinal */
    /* refinement strategy: smooth-refine / smooth-level (fclaw_options.c:203-209,
     * applied in fclaw2d_domain_adapt, src/fclaw2d_convenience.c:507-645),
     * refinement-criteria / threshold-variable (fclaw2d_clawpatch_options.c:107-114) */
    int smooth_refine, smooth_level;
    int refinement_criteria;   /* FC2D_B200_TAG_* */
    int threshold_variable;    /* field tested by the criterion, 1..meqn (0 = 1) */
    int qinit_cellave;         /* radial dam: 1 = cell averages of the disc (cellave2.f), 0 = cell-centre test */
    /* fclaw2d_run outstyle 1 (fclaw_options.c: regrid_interval, nout, use_fixed_dt,
     * tfinal, initial_dt, max_cfl, desired_cfl) */
    int regrid_interval, nout, use_fixed_dt;
    double tfinal, initial_dt, max_cfl, desired_cfl;
} fc2d_b200_options_t;

/* Tagging criteria: FCLAW_REFINE_CRITERIA_* (fclaw2d_clawpatch_options.h:48-56) + 1
 * (fort_user/fclaw2d_clawpatch_{value,difference,minmax,gradient}_exceeds_th.f90 in
 * fort_4.6/fclaw2d_clawpatch46_tag4refinement.f / _tag4coarsening.f).  TAG_APP keeps
 * the app's built-in criterion: minmax for the sphere, the gradient times dx
 * (refine where |grad q| dx exceeds the threshold) for the others. */
#define FC2D_B200_TAG_APP         0
#define FC2D_B200_TAG_VALUE       1
#define FC2D_B200_TAG_DIFFERENCE  2
#define FC2D_B200_TAG_MINMAX      3
#define FC2D_B200_TAG_GRADIENT    4
#define FC2D_B200_TAG_GRADIENT_DX 5

/* Counters of fc2d_b200_run (fclaw2d_global_t count_amr_advance, count_amr_regrid,
 * count_amr_new_domain; the reference's regression check, src/fclaw2d_finalize.c:119-165,
 * compares count_amr_advance, global_num_patches and count_amr_new_domain). */
typedef struct fc2d_b200_run_stats {
    int count_amr_advance;     /* advances taken, retaken ones included */
    int count_amr_regrid;      /* regrids called */
    int count_amr_new_domain;  /* regrids that changed the forest */
    int global_num_patches;    /* patches at the end */
    int rejected;              /* steps retaken because max_cfl was exceeded */
    int steps;                 /* accepted coarse steps */
    double t_final;
} fc2d_b200_run_stats_t;

typedef struct fc2d_b200_solver fc2d_b200_solver_t;

/* Last error message of the calling thread. */
const char* fc2d_b200_last_error(void);

/* Solver package lifetime.  Replaces fc2d_clawpack46_solver_initialize
 * (fc2d_clawpack46.cpp:483-538) + clawpatch allocation (fclaw2d_clawpatch.cpp:192-471). */
int fc2d_b200_create(const fc2d_b200_options_t* opt, fc2d_b200_solver_t** out);
int fc2d_b200_destroy(fc2d_b200_solver_t* s);

/* Select the registered __device__ Riemann pair (vt->fort_rpn2 / fort_rpt2,
 * fc2d_clawpack46.h:161-188; cudaclaw's cuda_rpn2 / cuda_rpt2). */
int fc2d_b200_set_riemann(fc2d_b200_solver_t* s, int rp_id);

/* Install update kernels an application compiled with its own __device__ rpn2 / rpt2
 * (and optional b4step2 / src2): the cudaclaw vtable fields cuda_rpn2, cuda_rpt2,
 * cuda_b4step2 (fc2d_cudaclaw.h:156-162) and clawpack46's src2 (fc2d_clawpack46.h:161-188).
 * table / n: the variant table the FC2D_B200_USER_SOLVER* macros of
 * include/fc2d_b200_user.cuh build in the application's module; abi: that header's
 * FC2D_B200_USER_ABI.  The solver must have rp = FC2D_B200_RP_USER, precision FP64,
 * time sync off, and the given meqn, mwaves, maux. */
int fc2d_b200_set_user_variants(fc2d_b200_solver_t* s, const void* table, int n, int abi, int meqn, int mwaves,
                                int maux);

/* fclaw2d_initialize (src/fclaw2d_initialize.c:75-250): uniform forest at minlevel,
 * setaux + qinit, then the initial-refinement loop.  Needs app != NONE. */
int fc2d_b200_initialize(fc2d_b200_solver_t* s);

/* Install an externally built forest (e.g. p4est leaves): level and
 * brick-global integer coordinates of each leaf, any order.  Patch data is zero
 * until fc2d_b200_set_q / fc2d_b200_set_aux. */
int fc2d_b200_set_forest(fc2d_b200_solver_t* s, int npatches, const int* level, const int* gx, const int* gy);

int fc2d_b200_num_patches(const fc2d_b200_solver_t* s, int* npatches);
/* level, block, brick-global gx, gy of each patch in level-major order. */
int fc2d_b200_patch_info(const fc2d_b200_solver_t* s, int* level, int* block, int* gx, int* gy);

/* Host <-> device copies of all patches (level-major FArrayBox layout). */
int fc2d_b200_get_q(fc2d_b200_solver_t* s, double* q);
int fc2d_b200_set_q(fc2d_b200_solver_t* s, const double* q);
int fc2d_b200_get_aux(fc2d_b200_solver_t* s, double* aux);
int fc2d_b200_set_aux(fc2d_b200_solver_t* s, const double* aux);
/* Conservation registers per patch: fp0 fp1 fm0 fm1 (my*meqn each), gp0 gp1
 * gm0 gm1 (mx*meqn each), edge fluxes 0..3 (2*{my,my,mx,mx}*meqn)
 * (fclaw2d_clawpatch_conservation.h:56-77). */
int fc2d_b200_registers_size(const fc2d_b200_solver_t* s, int* ndoubles_per_patch);
int fc2d_b200_get_registers(fc2d_b200_solver_t* s, double* regs);

/* Batched patch_vt->single_step_update for every patch of `level`
 * (fclaw2d_patch_single_step_update_t, src/fclaw2d_patch.h:937-943, called from
 * src/fclaw2d_update_single_step.c:44-70; clawpack46_update,
 * fc2d_clawpack46.cpp:402-444).  Includes b4step2, save_current_step,
 * time-sync flux/wave accumulation and the q update.  *cfl = level max CFL. */
int fc2d_b200_level_update(fc2d_b200_solver_t* s, int level, double t, double dt, double* cfl);

/* The cudaclaw buffering protocol (fc2d_cudaclaw.cpp:309-349) with plain types:
 * call once per patch of `level` with iter = 0..total_count-1; the launch
 * happens on the last call, which returns the level CFL in *cfl (0 before). */
int fc2d_b200_single_step_update(fc2d_b200_solver_t* s, int level, int iter, int total_count,
                                 double t, double dt, double* cfl);
/* The same protocol for callers whose patch data lives in host arrays, as
 * ForestClaw's FArrayBoxes do (fclaw2d_clawpatch.hpp:46-81) when its own ghost fill
 * (fclaw2d_ghost_update on host data) runs between the level updates: each call
 * hands over one patch of `level` -- its brick-global position gx, gy and its q (and
 * aux, or NULL to keep the device's) in the FArrayBox layout, ghost cells included.
 * The last call (iter + 1 == total_count, every patch of the level handed over once,
 * in any order) copies the arrays into their device slots, updates the level
 * (clawpack46_update on each patch), writes the new q back into every array and
 * returns the level CFL.  Time-sync registers stay on the device. */
int fc2d_b200_single_step_update_host(fc2d_b200_solver_t* s, int level, int gx, int gy, double* q,
                                      const double* aux, int iter, int total_count, double t, double dt,
                                      double* cfl);

/* fclaw2d_ghost_update (src/fclaw2d_ghost_fill.c:838-856). */
int fc2d_b200_ghost_update(fc2d_b200_solver_t* s, int minlevel, int maxlevel, double sync_time, int time_interp);
/* fclaw2d_timeinterp (src/fclaw2d_timeinterp.c:49-57). */
int fc2d_b200_timeinterp(fc2d_b200_solver_t* s, int level, double alpha);
/* fclaw2d_time_sync (src/fclaw2d_time_sync.c:157-202). */
int fc2d_b200_time_sync(fc2d_b200_solver_t* s, int minlevel, int maxlevel);
/* fclaw2d_advance_all_levels (src/fclaw2d_advance.c:247-357). */
int fc2d_b200_advance(fc2d_b200_solver_t* s, double t, double dt, double* maxcfl);
/* fclaw2d_regrid (src/fclaw2d_regrid.c:230-335): device tagging, host tree edit,
 * device repopulation, ghost update.  *changed = 1 if the forest changed. */
int fc2d_b200_regrid(fc2d_b200_solver_t* s, int* changed);
/* patch_vt->save_step / restore_step (fclaw2d_clawpatch.cpp:446-471, called by
 * save_time_step / restore_time_step of src/fclaw2d_run.c:42-82): a device copy of q
 * of every patch (ghosts included), and its return.  The forest must not change
 * in between. */
int fc2d_b200_save_step(fc2d_b200_solver_t* s);
int fc2d_b200_restore_step(fc2d_b200_solver_t* s);
/* fclaw2d_run with outstyle 1 (src/fclaw2d_run.c:113-265) from t = 0 after
 * fc2d_b200_initialize: nout output intervals up to tfinal, dt from the CFL of the
 * last step (desired_cfl), a step above max_cfl retaken from the saved copy with a
 * smaller dt, the last step of an interval stretched or shortened to end on it,
 * regrid every regrid_interval accepted steps.  *out (may be null) gets the counters. */
int fc2d_b200_run(fc2d_b200_solver_t* s, fc2d_b200_run_stats_t* out);

/* ---- output: clawpack 4.6 ASCII frames ----
 * fclaw2d_clawpatch_output_ascii (src/patches/clawpatch/fclaw2d_clawpatch_output_ascii.c:112-170,
 * fort_4.6/fclaw2d_clawpatch46_output_ascii.f): <dir>/fort.tNNNN (time, meqn, ngrids, num_aux,
 * num_dim) and <dir>/fort.qNNNN (per patch a header and the interior cells), patches in
 * the reference's order (block, then along the space-filling curve), Fortran E format.
 * fc2d_b200_write_ascii_frame writes caller-supplied patches (host memory, q in the
 * FArrayBox layout, ghosts included); it needs no device. */
int fc2d_b200_output_ascii(fc2d_b200_solver_t* s, const char* dir, int iframe, double time);
int fc2d_b200_write_ascii_frame(const char* dir, int iframe, double time, int meqn, int maux, int mx, int my,
                                int mbc, int npatch, const int* level, const int* block, const double* xlower,
                                const double* ylower, const double* dx, const double* dy, const double* q);
/* fclaw2d_clawpatch_output_vtk (src/patches/clawpatch/fclaw2d_clawpatch_output_vtk.c:593-900):
 * <prefix>_frame_NNNN.vtu, an XML UnstructuredGrid with raw appended data (UInt64 byte
 * count before each array): per patch (mx+1)(my+1) points (Float64 x 3; the
 * cubed-sphere mapping for the sphere app), mx*my quads with connectivity, offsets and
 * types, cell fields mpirank, blockno, patchno and the meqn values as Float32, patches
 * block by block along the curve.  Points and values are packed on the device.
 * fc2d_b200_write_vtk_file writes caller-supplied arrays (host memory, patches in file
 * order): points[np][(mx+1)(my+1)][3], values[np][mx*my][meqn], block[np]. */
int fc2d_b200_output_vtk(fc2d_b200_solver_t* s, const char* prefix, int iframe);
int fc2d_b200_write_vtk_file(const char* path, int mx, int my, int meqn, int npatch, const int* block,
                             const double* points, const float* values);

/* ---- one forest partitioned over ranks (one process per GPU) ----
 * The reference partitions the leaves along the space-filling curve
 * (src/fclaw2d_partition.c:113, p4est_partition with weights), exchanges ghost
 * patches once per ghost update (fclaw2d_exchange_ghost_patches_begin/end,
 * src/fclaw2d_exchange.c:308-413, called from src/fclaw2d_ghost_fill.c:700-720) with the
 * time-sync registers packed in the payload (fclaw2d_clawpatch_conservation.c:112-203),
 * and reduces the CFL number (src/fclaw2d_run.c:206) and the mass over ranks.  Here every
 * rank keeps the whole tree and the same slot numbering; it owns one range of the
 * curve (leaf weight 2^(level - minlevel present), its substeps per coarse step),
 * updates its own patches, fills the ghost cells of its own patches and of the first
 * ring of other ranks' patches around them, and before each ghost update receives
 * q, qlast and registers of the two rings of other ranks' patches around its own.
 * A regrid tags each rank's own patches, reduces the tags over ranks, gathers every
 * patch's q on every rank, adapts the (identical) tree and partitions it again.
 * The transport is the caller's, through these callbacks (return 0 on success):
 *   exchange:      for k < npeers, send send_bytes[k] bytes at send[k] to rank peers[k]
 *                  and receive recv_bytes[k] bytes from it into recv[k]; the buffers are
 *                  device memory of the solver's device, the solver's stream is idle on
 *                  entry, and the data must be in place on return (NCCL send/recv, or
 *                  host staging for gloo);
 *   allreduce_max / allreduce_sum: in place over ranks, n doubles in host memory.
 * Results are bitwise those of one rank holding the whole forest. */
typedef struct fc2d_b200_comm {
    int rank, size;
    void* user;
    int (*exchange)(void* user, int npeers, const int* peers, void* const* send, const size_t* send_bytes,
                    void* const* recv, const size_t* recv_bytes);
    int (*allreduce_max)(void* user, double* v, int n);
    int (*allreduce_sum)(void* user, double* v, int n);
} fc2d_b200_comm_t;
/* Partition this solver's forest among comm->size ranks (comm NULL: back to one rank,
 * every rank then holding the whole forest).  Every rank calls it with the same forest;
 * CUDA-graph replay is off while partitioned. */
int fc2d_b200_set_partition(fc2d_b200_solver_t* s, const fc2d_b200_comm_t* comm);
/* Owner rank of each patch (level-major order). */
int fc2d_b200_partition_owner(const fc2d_b200_solver_t* s, int* owner);
/* Gather every patch's current q, qlast and registers on every rank (before reading
 * the whole forest with fc2d_b200_get_q, writing output, or checkpointing). */
int fc2d_b200_sync_replicas(fc2d_b200_solver_t* s);
/* The partition plan of `rank` among `size` for a forest given by its leaves, computed
 * on the host without a device: owner[np], and per rank r the number of patches sent to
 * and received from r and a checksum of each list (sum over slots p of p * 2654435761 + 1). */
int fc2d_b200_partition_plan(const fc2d_b200_options_t* opt, int np, const int* level, const int* gx,
                             const int* gy, int rank, int size, int* owner, int* nsend, int* nrecv,
                             unsigned long long* send_sum, unsigned long long* recv_sum);

/* ---- patch-to-CTA variants of the fused update (no counterpart in the reference) ----
 * Each solver shape (precision, Riemann solver, patch size) is compiled with
 * several mappings of a patch onto its CTA: threads per CTA and an occupancy
 * target (CTAs per SM, which caps registers per thread); reg = 1 when every
 * interface of a sweep has its own thread; persistent = 1 for the persistent
 * form (a grid of resident CTAs looping over the level's patches, one launch
 * per level-step however many patches and instances).  Variant 0 is the default.  FP64
 * variants give identical results.  fc2d_b200_autotune times every variant on
 * the current forest (reps passes over all levels, dt = 0 so q is unchanged),
 * keeps the fastest and returns it; ms[v] (may be null, num_variants entries)
 * receives the time of one pass of variant v.  It then times every variant on
 * each level alone and keeps, per level, the fastest there (a level's patch
 * count decides how its CTAs fill the device's waves); fc2d_b200_level_variants
 * reports the variant each level 0..32 uses.  fc2d_b200_set_variant sets one
 * variant for every level; fc2d_b200_set_level_variants sets each level's (33
 * entries, e.g. another solver's fc2d_b200_level_variants) without timing. */
int fc2d_b200_num_variants(const fc2d_b200_solver_t* s, int* n, int* current);
int fc2d_b200_variant_info(const fc2d_b200_solver_t* s, int v, int* threads, int* min_blocks, int* reg,
                           int* smem_bytes, int* persistent);
int fc2d_b200_set_variant(fc2d_b200_solver_t* s, int v);
int fc2d_b200_autotune(fc2d_b200_solver_t* s, int reps, int* best, double* ms);
int fc2d_b200_level_variants(const fc2d_b200_solver_t* s, int* variant /* 33 entries */);
int fc2d_b200_set_level_variants(fc2d_b200_solver_t* s, const int* variant /* 33 entries */);

/* ---- batches of independent forests (instances; no counterpart in the reference) ----
 * One solver can hold up to FC2D_B200_MAX_INSTANCES independent forests with the
 * same patch size, meqn and solver: every level-step launch then covers the
 * patches of all instances.  Each instance has its own brick, levels, app
 * parameters (pdata) and time step; its patches are numbered by levels relative
 * to its own minlevel, so every instance takes the same subcycled steps as it
 * would alone.  Set before fc2d_b200_initialize; the app must not depend on t. */
#define FC2D_B200_MAX_INSTANCES 256
typedef struct fc2d_b200_instance {
    int minlevel, maxlevel;
    double ax, bx, ay, by;
    int mi, mj;
    double pdata[32];
} fc2d_b200_instance_t;
int fc2d_b200_set_instances(fc2d_b200_solver_t* s, int n, const fc2d_b200_instance_t* inst);
int fc2d_b200_num_instances(const fc2d_b200_solver_t* s, int* n);
/* Instance of each patch (level-major order; patch_info reports absolute levels). */
int fc2d_b200_patch_instance(const fc2d_b200_solver_t* s, int* inst);
/* One coarse step of every instance, instance i with its own dt[i]; cfl[i] = its CFL. */
int fc2d_b200_advance_instances(fc2d_b200_solver_t* s, const double* dt, double* cfl);
/* The same in two halves: _begin launches the step on the solver's stream and
 * returns at once, _end waits for it and returns the CFL numbers, so the steps of
 * several solvers (one per patch size, say) run concurrently. */
int fc2d_b200_advance_instances_begin(fc2d_b200_solver_t* s, const double* dt);
int fc2d_b200_advance_instances_end(fc2d_b200_solver_t* s, double* cfl);
/* Kahan-summed mass per instance and field: out[i * meqn + m]. */
int fc2d_b200_mass_instances(fc2d_b200_solver_t* s, double* out);

/* Kahan-summed mass per field over interior cells, FP64
 * (fclaw2d_clawpatch46_diagnostics.f:13-55). */
int fc2d_b200_mass(fc2d_b200_solver_t* s, double* out);
/* fc2d_b200_mass computed without allocating memory (no counterpart in the
 * reference).  It is for callers that must not allocate device memory between
 * steps: an application whose device memory is all handed out by its own pool,
 * or one that takes diagnostics while its other streams keep running, where the
 * device-wide synchronisation of cudaFree would stall them.  The patch partials
 * and the per-field sums go to one static device array of
 * FC2D_B200_MASS_SCRATCH_DOUBLES doubles (1 MiB, held by every GPU that loads
 * the library until the process exits), so npatches*meqn + meqn must not exceed
 * it (else FC2D_B200_EINVAL, nothing runs).
 * Same result as fc2d_b200_mass, bit for bit.  No part of the scratch has to
 * start at zero.  fc2d_b200_create loads the module that holds the array and
 * resolves its device address (cudaGetSymbolAddress, once per device per
 * process), so this call itself loads and looks up nothing.  The cached address
 * is invalid after the device's primary context is destroyed (cudaDeviceReset):
 * create no solver across such a reset.  Calls that overlap in time on one
 * device (several host threads) share the scratch and race. */
#define FC2D_B200_MASS_SCRATCH_DOUBLES 131072
int fc2d_b200_mass_noalloc(fc2d_b200_solver_t* s, double* out);
/* Newton iterations of the exact Euler solver: out[k] = interfaces solved in k
 * iterations since creation or the last reset (k = 31: 31 or more). */
int fc2d_b200_newton_histogram(fc2d_b200_solver_t* s, unsigned long long* out, int reset);
/* Interior cell updates performed so far (sum over levels of patches*mx*my per step). */
int fc2d_b200_cell_updates(const fc2d_b200_solver_t* s, double* out);
/* Wait for all device work of the solver's stream. */
int fc2d_b200_synchronize(fc2d_b200_solver_t* s);

/* Device kernel timing of the most recent fc2d_b200_advance: milliseconds spent
 * in the update kernels and the bytes they moved algorithmically (interior
 * cells, q read + write + aux read). */
int fc2d_b200_last_update_stats(const fc2d_b200_solver_t* s, double* update_ms, double* update_bytes,
                                int* update_launches, int* total_launches);
/* The most recent advance (fc2d_b200_advance or _advance_instances): host_ms, the
 * wall time the host spent building its launch schedule before any device work;
 * device_ms, the CUDA-event span of its work on the solver's stream, from the
 * first copy of its parameters to the end of its last launch (a graph rebuilt
 * after a regrid is captured inside that span). */
int fc2d_b200_last_step_timing(const fc2d_b200_solver_t* s, double* host_ms, double* device_ms);
/* Wall-clock breakdown of the most recent fc2d_b200_regrid, milliseconds
 * (ms[8]): 0 tagging on the device and the flags back on the host, 1 coarsen /
 * refine marks, smoothing and the 2:1-balanced leaves, 2 the new forest (neighbour
 * search), 3 repopulation (ops, aux, device copies), 4 gather-table build on the
 * host, 5 descriptor and table upload (partition plan included), 6 the ghost
 * update on the new forest, 7 the whole call. */
int fc2d_b200_last_regrid_stats(const fc2d_b200_solver_t* s, double* ms);
/* Replay each fclaw2d_advance_all_levels as a CUDA graph captured once per
 * forest (on by default; disabled while update timing is on). */
int fc2d_b200_set_graphs(fc2d_b200_solver_t* s, int enable);
/* The advance graphs so far: builds, instantiations of a captured graph (the first
 * advance, or a capture whose launches differ from the graph's); updates, captures
 * after a regrid applied to the existing graph in place (cudaGraphExecUpdate). */
int fc2d_b200_graph_stats(const fc2d_b200_solver_t* s, int* builds, int* updates);
/* Launch the kernels of an advance (level updates, ghost-fill stages, time
 * sync, time interpolation) with programmatic dependent launch: each grid is
 * scheduled while its predecessor's last CTAs run and waits in-kernel for the
 * predecessor's completion before touching memory, which hides the launch gap
 * between the many short dependent grids of a subcycled step.  Results are
 * identical either way.  On by default. */
int fc2d_b200_set_programmatic_launch(fc2d_b200_solver_t* s, int enable);
/* Enable/disable CUDA-event timing of the update kernels (off by default). */
int fc2d_b200_set_timing(fc2d_b200_solver_t* s, int enable);

/* CUDA events on the solver's stream, for callers that time device work:
 * record into one of 64 slots, then read the elapsed milliseconds between two
 * recorded slots (waits for the later event). */
int fc2d_b200_event_record(fc2d_b200_solver_t* s, int slot);
int fc2d_b200_event_elapsed(fc2d_b200_solver_t* s, int slot_a, int slot_b, double* ms);
/* The cudaStream_t the solver launches on (returned as void*). */
int fc2d_b200_get_stream(const fc2d_b200_solver_t* s, void** stream);

/* ---- learned p* start of the exact Euler solver (no counterpart in the reference) ----
 * A 6 -> 64 -> 64 -> 1 tanh network predicts the correction log(pstar/p_pvrs) of
 * the PVRS estimate from the normalised primitive interface states; where the
 * jump |dp|/pbar + |du|/cbar exceeds 0.2 Newton starts from p_pvrs exp(y)
 * instead of p_pvrs and still iterates to newton_tol, so converged fluxes are
 * unchanged to tolerance.  Parameters (FC2D_B200_MLP_NPARAM floats):
 * W1[64][6] b1[64] W2[64][64] b2[64] w3[64] b3.  Training runs on the GPU:
 * tensor-core forward (BF16 inputs, FP32 accumulation), FP32 backward, Adam. */
#define FC2D_B200_MLP_NPARAM 4673
typedef struct fc2d_b200_mlp fc2d_b200_mlp_t;
int fc2d_b200_mlp_create(int device, unsigned long long seed, fc2d_b200_mlp_t** out);
int fc2d_b200_mlp_destroy(fc2d_b200_mlp_t* m);
int fc2d_b200_mlp_set_params(fc2d_b200_mlp_t* m, const float* params);
int fc2d_b200_mlp_get_params(fc2d_b200_mlp_t* m, float* params);
/* Training set: n primitive states (rhoL, uL, pL, rhoR, uR, pR) in the normal
 * frame; targets are computed on the device by Newton (PVRS start) to `tol`. */
int fc2d_b200_mlp_set_data(fc2d_b200_mlp_t* m, const double* prim, int n, double gamma, double tol);
/* Features X[n][6] and targets Y[n] of the training set. */
int fc2d_b200_mlp_get_data(fc2d_b200_mlp_t* m, float* X, float* Y);
/* Minibatch Adam over shuffled epochs; *loss = mean squared error of the last epoch. */
int fc2d_b200_mlp_train(fc2d_b200_mlp_t* m, int epochs, int batch, float lr, unsigned long long seed, double* loss);
/* Gradient of the mean squared error over (X, Y) without an update. */
int fc2d_b200_mlp_gradient(fc2d_b200_mlp_t* m, const float* X, const float* Y, int n, float* grad, double* loss);
/* The deployed forward (approximate tanh, as inside the solver). */
int fc2d_b200_mlp_predict(fc2d_b200_mlp_t* m, const float* X, int n, float* Y);
/* Batched evaluation (fc2d_b200_mlp_predict, fc2d_b200_mlp_newton_histogram): tcgen05 = 1
 * (default) runs tiles of 128 states on the tcgen05 tensor cores (accumulators in tensor
 * memory), 0 the per-warp mma.sync form the solver's update uses for its 32 interfaces;
 * the two agree to FP32 rounding.  A tensor-core tile that does not complete returns
 * FC2D_B200_EDEVICE. */
int fc2d_b200_mlp_set_tensor_form(fc2d_b200_mlp_t* m, int tcgen05);
/* Newton-iteration histogram over the training set from the PVRS (0) or network (1) start. */
int fc2d_b200_mlp_newton_histogram(fc2d_b200_mlp_t* m, int use_mlp, long long* hist32);
/* Uniform sample of n normal-direction interfaces of the solver's forest (Euler). */
int fc2d_b200_sample_interfaces(fc2d_b200_solver_t* s, int n, unsigned long long seed, double* prim);
/* Seed the solver's Newton iterations with the network (m = NULL: back to PVRS). */
int fc2d_b200_set_pstar_seed(fc2d_b200_solver_t* s, const fc2d_b200_mlp_t* m);

#ifdef __cplusplus
}
#endif
#endif
