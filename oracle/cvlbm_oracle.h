/*
 * CPU oracle for the curved-boundary VLBM time step -- TEST INFRASTRUCTURE.
 *
 * A plain-C restatement of the reference's Warp kernels
 * (src/curved_lbm/two_d/curved_boundary_warp.py and
 *  src/curved_lbm/three_d/curved_boundary_warp3d.py of curved_lbm 1.0.0),
 * executed serially in IEEE binary64 with floating-point contraction disabled.
 * Parity is pinned: the oracle reproduces the fixtures the reference itself
 * produced (tests/golden, see tests/test_oracle.py).  Only tests/, smoke() and
 * bench.py's CPU-baseline leg use it; the product never calls it.
 *
 * The problem/state descriptions reuse the layout of include/cvlbm.h, with
 * every pointer a HOST pointer.  Links are processed in ascending link order,
 * which is the order in which the reference's serial atomics accumulate the
 * cut-point anchors.
 */
#ifndef CVLBM_ORACLE_H
#define CVLBM_ORACLE_H

#include <stdint.h>

#include "../include/cvlbm.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Scratch the reference keeps between kernels (bc_diag/bc_rhs, u_next). */
typedef struct oracle2d_scratch {
  double *bc_diag; /* [N] */
  double *bc_rhs;  /* [2*N] */
} oracle2d_scratch;

typedef struct oracle3d_scratch {
  double *bc_diag; /* [3*N] */
  double *bc_rhs;  /* [3*N] */
} oracle3d_scratch;

/* One step each, exactly WarpCurvedBoundaryLBM2D.step / WarpSparseCurvedBoundaryLBM3D.step;
 * f->f0 and f->f1 are swapped on return.  `threads` > 1 runs the node loops
 * with OpenMP (results are identical: node loops are independent and the
 * anchor accumulation stays serial in link order). */
int oracle2d_step(const cvlbm2d_problem *p, cvlbm2d_fields *f, oracle2d_scratch *s, double time,
                  int64_t step, int threads);
int oracle2d_apply_boundary(const cvlbm2d_problem *p, cvlbm2d_fields *f, double t, int in_place);
int oracle2d_refresh(const cvlbm2d_problem *p, cvlbm2d_fields *f);
/* C2:3101-3124 kinetic ghost filter on fields->f0 (initialisation) */
int oracle2d_kinetic_filter(const cvlbm2d_problem *p, cvlbm2d_fields *f);

int oracle3d_step(const cvlbm3d_problem *p, cvlbm3d_fields *f, oracle3d_scratch *s, double time,
                  int64_t step, int threads);
int oracle3d_apply_boundary(const cvlbm3d_problem *p, cvlbm3d_fields *f, double t, int in_place);
int oracle3d_refresh(const cvlbm3d_problem *p, cvlbm3d_fields *f);

#ifdef __cplusplus
}
#endif

#endif
