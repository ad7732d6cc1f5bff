/*
 * oracle.h -- CPU FP64 oracle for the ForestClaw clawpack 4.6 patch-update hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a plain-C restatement of the
 * reference's Fortran/C algorithms (clawpack46 step2/flux2/limiter, the
 * clawpatch 4.6 ghost-fill kernels, time-sync, the level/ghost-fill/time-sync
 * orchestration).  It is the checker the CUDA product is compared against and
 * the timed CPU baseline; the product never links, loads or calls it.
 *
 * Parity status: the reference's hot path is Fortran and cannot be compiled in
 * this environment (no Fortran compiler; p4est/libsc are empty submodules), and
 * the reference's own tests pin no field values.  Parity of this oracle against
 * the reference is therefore "parity unpinned": it rests on line-by-line review
 * against the cited Fortran plus mathematical known-answer tests (constant-state
 * preservation, exact translation at CFL 1, conservation, symmetry).
 *
 * Floating-point semantics: every expression is evaluated left to right in the
 * Fortran order of the cited line, without FMA contraction
 * (-ffp-contract=off), so that a no-contraction FP64 GPU kernel can match it
 * bit for bit.
 */
#ifndef FCB_ORACLE_H
#define FCB_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Riemann solver identifiers (mirrors the user solvers of the reference apps). */
enum {
    ORC_RP_ADVECTION = 0,     /* applications/clawpack/advection/2d/all/clawpack46_rpn2adv.f, rpt2adv.f */
    ORC_RP_SW_ROE = 1,        /* applications/clawpack/shallow/2d/rp/clawpack46_rpn2.f, clawpack46_rpt2.f */
    ORC_RP_SW_FWAVE = 2,      /* applications/clawpack/shallow/2d/rp/rpn2_tsunami.f90, rpt2_tsunami.f90 */
    ORC_RP_EULER_EXACT = 3,   /* build-originated exact Euler solver (no reference counterpart) */
    ORC_RP_ADVECTION_MANIFOLD = 4,  /* applications/clawpack/advection/2d/all/clawpack46_rpn2adv_manifold.f, _rpt2adv_manifold.f */
    ORC_RP_ACOUSTICS = 5      /* applications/cudaclaw/acoustics/2d/radial/user_cuda/rpn2acoustics.cu, rpt2acoustics.cu
                                 (an application's own device solver; rho, bulk in pdata[24], pdata[25]) */
};

/* Problem (app) identifiers: qinit/b4step2/setprob of the reference apps. */
enum {
    ORC_PROB_SWIRL = 0,       /* applications/clawpack/advection/2d/swirl */
    ORC_PROB_RADIALDAM = 1,   /* applications/clawpack/shallow/2d/radialdam */
    ORC_PROB_UNIFORM_SW = 2,  /* radial dam initial data on a uniform grid (same app) */
    ORC_PROB_TSUNAMI = 3,     /* batched bathymetry problem (rpn2_tsunami) */
    ORC_PROB_SHOCKBUBBLE = 4, /* applications/clawpack/euler/2d/shockbubble (Mach-M shock, light bubble) */
    ORC_PROB_SPHERE = 5,      /* applications/clawpack/advection/2d/sphere on the cubed sphere (6 blocks) */
    ORC_PROB_ROTATION = 6,    /* test app of the application-solver interface: b4step2 sets edge velocities
                                 from a quadratic stream function, q = disc (cell centre) */
    ORC_PROB_ACOUSTICS = 7    /* test app: pressure disc at rest (cell centre) for ORC_RP_ACOUSTICS */
};

typedef struct orc_config {
    /* clawpatch options (fclaw2d_clawpatch_options.c) */
    int mx, my, mbc, meqn, maux;
    /* clawpack46 options (fc2d_clawpack46_options.c:37-99) */
    int mwaves;
    int order[2];          /* method(2), method(3) */
    int mthlim[8];
    int mthbc[4];
    int mcapa;
    int use_fwaves;
    int rp;                /* ORC_RP_* */
    /* fclaw options (fclaw_options.c) */
    int minlevel, maxlevel;
    int subcycle;
    int time_sync, flux_correction, fluctuation_correction;
    int regrid_interval;
    double refine_threshold, coarsen_threshold;
    double ax, bx, ay, by;
    int mi, mj;            /* brick blocks; 1x1 = single block */
    /* problem */
    int problem;           /* ORC_PROB_* */
    double grav;
    double tperiod;        /* swirl time period T */
    double r0, hin, hout, x0, y0;   /* radial dam */
    int qinit_sharp;       /* 1: cell-centre test instead of cellave2 quadrature */
    double pdata[32];      /* extra problem parameters (tsunami bumps etc.) */
    /* Euler (shock-bubble): gas constant, shock Mach number, bubble density,
     * Newton tolerance on p* (relative change); bubble centre/radius in x0, y0, r0 */
    double gamma, mach, rhob, newton_tol;
    int nthreads;          /* OpenMP threads for the patch loops (0 = default) */
    /* refinement strategy: fclaw_options.c:203-213 (smooth-refine, smooth-level),
     * fclaw2d_clawpatch_options.c:107-114 (refinement-criteria, threshold-variable) */
    int smooth_refine, smooth_level;
    int tag_criteria;      /* ORC_TAG_* */
    int threshold_variable;   /* 1-based field tested by the criterion (0 = field 1) */
    /* fclaw2d_run outstyle 1 (fclaw_options.c: tfinal, nout, initial_dt, max_cfl,
     * desired_cfl, use_fixed_dt, regrid_interval above) */
    double tfinal, initial_dt, max_cfl, desired_cfl;
    int nout, use_fixed_dt;
    /* src2 after step2 (fc2d_clawpack46.cpp:436-441): 0 none, 1 q(:,:,1) -= dt*rate*q(:,:,1)
     * over the padded patch (the test source of the application-solver interface) */
    int src_kind;
    double src_rate;
} orc_config;

/* Tagging criteria: FCLAW_REFINE_CRITERIA_* (fclaw2d_clawpatch_options.h:48-56) + 1;
 * ORC_TAG_APP keeps each problem's built-in criterion (gradient times dx for the
 * shallow-water and Euler problems, minmax for the sphere). */
enum { ORC_TAG_APP = 0, ORC_TAG_VALUE = 1, ORC_TAG_DIFFERENCE = 2, ORC_TAG_MINMAX = 3,
       ORC_TAG_GRADIENT = 4, ORC_TAG_GRADIENT_DX = 5 };

/* Counters of one fclaw2d_run (fclaw2d_global.h: count_amr_advance, count_amr_regrid,
 * count_amr_new_domain; src/fclaw2d_finalize.c:119-165 checks three of them). */
typedef struct orc_run_stats {
    int count_amr_advance;     /* calls of fclaw2d_advance_all_levels, retaken steps included */
    int count_amr_regrid;      /* calls of fclaw2d_regrid */
    int count_amr_new_domain;  /* regrids that changed the forest */
    int global_num_patches;    /* leaves at the end */
    int rejected;              /* steps retaken because max_cfl was exceeded */
    int steps;                 /* accepted coarse steps */
    double t_final;
} orc_run_stats;

typedef struct orc_sim orc_sim;

orc_sim* orc_create(const orc_config* cfg);
void     orc_destroy(orc_sim* s);

/* Uniform forest at minlevel + qinit (+ init-regrid when maxlevel > minlevel). */
int    orc_initialize(orc_sim* s);
/* fclaw2d_advance_all_levels (src/fclaw2d_advance.c:247-357); returns max CFL. */
double orc_advance(orc_sim* s, double t, double dt);
/* fclaw2d_regrid (src/fclaw2d_regrid.c). Returns 1 if the forest changed. */
int    orc_regrid(orc_sim* s);
/* Ghost update over all levels at sync time t (time_interp = 0). */
void   orc_ghost_update_all(orc_sim* s, double t);
/* fclaw2d_run outstyle 1 (src/fclaw2d_run.c:113-265) from t = 0 after orc_initialize:
 * CFL-driven dt, small/big final steps, retake above max_cfl, regrid every
 * regrid_interval steps.  Returns 0. */
int    orc_run(orc_sim* s, orc_run_stats* out);
/* patch_vt->save_step / restore_step (fclaw2d_clawpatch.cpp:446-471): q of every patch. */
void   orc_save_step(orc_sim* s);
void   orc_restore_step(orc_sim* s);

int    orc_num_patches(const orc_sim* s);
/* Patches in level-major order: level, block, ix, iy (integer coordinates at the patch level). */
void   orc_patch_info(const orc_sim* s, int* level, int* block, int* ix, int* iy);
/* Copy q (Fortran layout, ghosts included) of all patches in level-major order. */
void   orc_get_q(const orc_sim* s, double* out);
void   orc_set_q(orc_sim* s, const double* in);
void   orc_get_aux(const orc_sim* s, double* out);
/* Kahan-summed mass per field (fclaw2d_clawpatch46_diagnostics.f:13-55). */
void   orc_mass(const orc_sim* s, double* out);
/* Number of interior cell updates performed so far. */
double orc_cell_updates(const orc_sim* s);
/* Registers of all patches (for tests): per patch 4*? doubles, see orc_registers_size. */
int    orc_registers_size(const orc_sim* s);
void   orc_get_registers(const orc_sim* s, double* out);

/* ---- single-patch numerics, exposed for unit tests ---------------------- */
/* clawpack46_step2_wrap on one patch: q updated in place, returns cfl.
 * fm/fp/gm/gp (size (mx+2mbc)(my+2mbc)meqn each) receive the flux arrays. */
double orc_patch_step2(const orc_config* cfg, double* q, const double* aux,
                       double dx, double dy, double dt,
                       double* fm, double* fp, double* gm, double* gp);
/* clawpack46_inlinelimiter phi(r) for one r (tests of the limiter table). */
double orc_limiter_phi(int mthlim, double r);

/* ---- exact Euler Riemann solver (orc_euler.c), exposed for unit tests ----- */
double orc_log(double x);
double orc_exp(double y);
double orc_pow(double x, double a);
/* primitive (rho, u, p) states; seed <= 0 selects the PVRS start.  out[6] =
 * p*, u*, rho*L, rho*R, a*L, a*R.  Returns the Newton iterations. */
int  orc_euler_star(double gam, const double* wl, const double* wr, double seed, double tol, double* out);
/* conserved (rho, m_n, m_t, E) states -> waves[3][4], speeds[3], amdq, apdq */
int  orc_euler_interface(double gam, double tol, const double* ql, const double* qr, double seed,
                         double wave[3][4], double s[3], double* amdq, double* apdq);
/* clawpack46_rpt2_euler4 of one interface with its Roe averages (tests). */
void orc_euler_rpt2_point(double gam, int ixy, const double* qlo, const double* qhi, const double* asdq, double* bm,
                          double* bp);
void orc_euler_postshock(double gam, double mach, double* out);
/* Newton-iteration histogram of all exact solves so far (32 bins; reset if asked). */
void orc_newton_hist(long* out, int reset);

#ifdef __cplusplus
}
#endif
#endif
