/*
 * orc_amr.h -- oracle data structures for the forest of patches (test infrastructure).
 */
#ifndef FCB_ORC_AMR_H
#define FCB_ORC_AMR_H

#include "orc_internal.h"

/* fclaw2d_patch_relation_t */
enum { NB_BOUNDARY = 0, NB_HALF = 1, NB_SAME = 2, NB_DOUBLE = 3 };

/* Register index helpers: (j,m) of a (n, meqn) array and (j,m,k) of (n, meqn, 0:1). */
#define RJ(j, m, n) ((size_t)((j) - 1) + (size_t)((m) - 1) * (size_t)(n))
#define RJK(j, m, k, n, meqn) ((size_t)((j) - 1) + (size_t)((m) - 1) * (size_t)(n) + (size_t)(k) * (size_t)(n) * (size_t)(meqn))

/* fclaw2d_clawpatch_registers_t (fclaw2d_clawpatch_conservation.h:56-77). */
typedef struct orc_regs {
    double* fp[2]; double* fm[2];     /* my*meqn: left (0) / right (1) */
    double* gp[2]; double* gm[2];     /* mx*meqn: bottom (0) / top (1) */
    double* ef[4];                    /* 2*{my,my,mx,mx}*meqn: edge fluxes, k=0 interior, k=1 ghost */
    double* el[4];                    /* edge lengths */
    double* area[4];                  /* areas of the edge cells */
    double* mem;
} orc_regs;

typedef struct orc_patch {
    int level, block, gx, gy;         /* gx, gy: brick-global integer coords at `level` */
    double xlower, ylower, dx, dy;
    double *q, *qlast, *qinterp, *aux;
    double* qsave;                    /* save_step copy (allocated on first use) */
    double* area;                     /* cubed sphere: cell areas, -mbc..mx+mbc+1 in both directions */
    orc_regs regs;
    int face_type[4];
    int face_nbr[4][2];               /* 1 (same/double) or 2 (half) neighbour indices */
    int corner_type[4];               /* valid when has_corner */
    int corner_nbr[4];
    int has_corner[4];
    int phys[4];                      /* face lies on the physical boundary */
    int has_fine_nbr, on_cf;
    int bcc[4];                       /* block_corner_count */
    unsigned long long morton;
} orc_patch;

struct orc_sim {
    orc_config cfg;
    int nx, ny;
    size_t nq, naux;
    int np;
    orc_patch* p;                     /* p4est order: block, then Morton */
    int* lev_list;                    /* patch indices ordered by (level, p4est order) */
    int lev_start[32];                /* lev_list range for level l: [lev_start[l], lev_start[l+1]) */
    int minlevel_present, maxlevel_present;
    /* hash (level, gx, gy) -> patch index */
    int hcap;
    long long* hkey;
    int* hval;
    double* dummy;                    /* time-sync scratch */
    double cell_updates;
    int nthreads;
    double t_curr;
    double inflow[8];                 /* shock-bubble inflow state (mthbc = 0 side) */
};

void orc_copy_face(const orc_sim* s, double* qthis, const double* qnbr, const orc_patch* P, const orc_patch* N, int iface);
void orc_copy_corner(const orc_sim* s, double* qthis, const double* qnbr, const orc_patch* P, const orc_patch* N, int icorner);
void orc_average_face(const orc_sim* s, double* qc, const double* qf, const orc_patch* C, const orc_patch* F, int iface_coarse);
void orc_average_corner(const orc_sim* s, double* qc, const double* qf, const orc_patch* C, const orc_patch* F, int icorner);
void orc_interpolate_face(const orc_sim* s, const double* qc, double* qf, const orc_patch* C, const orc_patch* F, int iface_coarse);
void orc_interpolate_corner(const orc_sim* s, const double* qc, double* qf, const orc_patch* C, const orc_patch* F, int icorner);
/* acoarse / afine: cell areas on a manifold (fixcapaq2 / area weights), else NULL */
void orc_interpolate2fine(const orc_sim* s, const double* qcoarse, double* qfine, int igrid,
                          const double* acoarse, const double* afine);
void orc_average2coarse(const orc_sim* s, double* qcoarse, const double* qfine, int igrid,
                        const double* acoarse, const double* afine);
void orc_timeinterp(const orc_sim* s, const double* qcurr, const double* qlast, double* qinterp, double alpha);
void orc_time_sync_f2c(const orc_sim* s, orc_patch* C, const orc_patch* F, int iface_coarse);
void orc_time_sync_samesize(const orc_sim* s, orc_patch* P, const orc_patch* N, int this_iface);
void orc_store_flux(const orc_sim* s, orc_patch* P, double dt);
void orc_accumulate_waves(const orc_sim* s, orc_patch* P, double dt, double dx, double dy,
                          const double* fp, const double* fm, const double* gp, const double* gm);
void orc_regs_reset_face(const orc_sim* s, orc_patch* P, int k);

/* cubed sphere (orc_sphere.c) */
double orc_tan(double x);
void orc_cs_map(int block, double xc, double yc, double* xp, double* yp, double* zp);
int  orc_cs_nb(int b, int f);
int  orc_step(const orc_sim* s, int l, int x, int y, int dx, int dy, int* ox, int* oy);
void orc_xf_same(const orc_sim* s, const orc_patch* P, const orc_patch* N, int i, int j, int* i2, int* j2);
void orc_xf_half(const orc_sim* s, const orc_patch* C, const orc_patch* F, int ic, int jc, int* i2, int* j2);
void orc_sphere_area(const orc_sim* s, orc_patch* P, int ghost_only);
void orc_sphere_area_from_fine(const orc_sim* s, orc_patch* C, const orc_patch* F, int igrid);
void orc_sphere_setaux(const orc_sim* s, orc_patch* P);
void orc_sphere_flow(const orc_config* c, double* axis, double* omega);
#define ORC_AIDX(i, j, mbc, ax) ((size_t)((j) + (mbc)) * (size_t)(ax) + (size_t)((i) + (mbc)))

/* problems (orc_problems.c) */
void orc_setaux(const orc_sim* s, orc_patch* P);
void orc_qinit(const orc_sim* s, orc_patch* P);
void orc_b4step2(const orc_sim* s, orc_patch* P, double t, double dt);
int  orc_tag_refine(const orc_sim* s, const orc_patch* P, int init_flag);
int  orc_tag_coarsen(const orc_sim* s, const orc_patch* const* fam, int init_flag);

#endif
