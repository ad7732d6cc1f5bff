/*
 * orc_internal.h -- shared declarations of the CPU oracle (test infrastructure).
 */
#ifndef FCB_ORC_INTERNAL_H
#define FCB_ORC_INTERNAL_H

#include <stddef.h>
#include "oracle.h"

/* 1D work-array index of Fortran index i in (1-mbc:maxm+mbc); needs `mbc` in scope. */
#define I1(i) ((i) + mbc - 1)
/* q(i,j,m) of a (1-mbc:mx+mbc, 1-mbc:my+mbc, meqn) array, 1-based i,j,m. */
#define QIDX(i, j, m, mbc_, nx_, ny_) \
    ((size_t)((i) + (mbc_) - 1) + (size_t)((j) + (mbc_) - 1) * (size_t)(nx_) + (size_t)((m) - 1) * (size_t)(nx_) * (size_t)(ny_))

typedef struct orc_rpctx {
    double grav;
    double dry_tolerance;
    double* u; double* v; double* a; double* h;   /* common /comroe/ */
    double* e;                                    /* Euler: gamma1/a^2 (g1a2 of comroe) */
    double gamma, newton_tol;
    const orc_config* cfg;
} orc_rpctx;

typedef void (*orc_rpn2_t)(orc_rpctx*, int ixy, int maxm, int meqn, int mwaves, int maux, int mbc, int mx,
                           const double* ql, const double* qr, const double* auxl, const double* auxr,
                           double* wave, double* s, double* amdq, double* apdq);
typedef void (*orc_rpt2_t)(orc_rpctx*, int ixy, int maxm, int meqn, int mwaves, int maux, int mbc, int mx,
                           const double* ql, const double* qr, const double* aux1, const double* aux2,
                           const double* aux3, int imp, const double* asdq, double* bmasdq, double* bpasdq);

void orc_rp_select(int rp, orc_rpn2_t* rpn2, orc_rpt2_t* rpt2);
void orc_rpn2_fwave(orc_rpctx*, int, int, int, int, int, int, int, const double*, const double*,
                    const double*, const double*, double*, double*, double*, double*);
void orc_rpt2_fwave(orc_rpctx*, int, int, int, int, int, int, int, const double*, const double*,
                    const double*, const double*, const double*, int, const double*, double*, double*);

void orc_rpn2_euler(orc_rpctx*, int, int, int, int, int, int, int, const double*, const double*,
                    const double*, const double*, double*, double*, double*, double*);
void orc_rpt2_euler(orc_rpctx*, int, int, int, int, int, int, int, const double*, const double*,
                    const double*, const double*, const double*, int, const double*, double*, double*);
void orc_euler_cons_flux(double gam, int idir, const double* q, double* flux);

size_t orc_ws_size(int mx, int my, int mbc, int meqn, int maux, int mwaves);
double orc_step2(const orc_config* cfg, orc_rpn2_t rpn2, orc_rpt2_t rpt2, double* work,
                 double* qold, const double* aux, double dx, double dy, double dt,
                 double* fm, double* fp, double* gm, double* gp, const int* block_corner_count);
/* inflow: state written by mthbc = 0 (user) sides, NULL for none */
void orc_bc2(int mx, int my, int mbc, int meqn, double* q, const int* mthbc, const double* inflow);

#endif
