/* CPU restatement of LBFlow's solver step loop -- TEST INFRASTRUCTURE ONLY.
 *
 * This is the checker the CUDA engine is compared against.  Only the tests,
 * the package's smoke check and the benchmark's CPU-baseline leg may load it;
 * the product path never does.  Every function restates the reference C++
 * (zhou1800/lbflow, solver/src/lbm/ sources) in plain C, in the same arithmetic
 * order, on dense arrays laid out exactly like the reference:
 * populations [phase][q][voxel], voxel = (z*ny + y)*nx + x, lattice vectors
 * in the reference's {z,y,x} component order. */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Label types: the bit values of FilePrm::IDXTYPE (solver/inc/file/fileprm.h:44-53). */
enum { LBO_VD = 0x1, LBO_GV = 0x2, LBO_PB = 0x4, LBO_VB = 0x8,
       LBO_AB = 0x10, LBO_BB = 0x20, LBO_HF = 0x40, LBO_SD = 0x80 };

/* One geometry label (a line `N "TYPE" "value" "dir" "phase"` of input.prm). */
typedef struct {
    int    type;   /* 0 = label not defined */
    double value;  /* GV force magnitude, PB density, VB speed or SD contact angle (degrees) */
    int    dir;    /* GV lattice direction; PB/VB boundary direction 1..2D */
    int    phase;  /* fluid phase (0 or 1) */
} lbo_label;

typedef struct {
    int    dims;        /* 2 (D2Q9) or 3 (D3Q19) */
    int    nx, ny, nz;  /* nz = 1 in 2D */
    int    color;       /* 0: single phase (SCSP); 1: color-gradient two-phase */
    int    mrt;         /* 0: SRT; 1: MRT */
    double tau[2];      /* relaxation times (tau[1] used by color only) */
    double rho[2];      /* reference densities */
    double alpha0;      /* color: rest weight of phase 0 */
    double sigma;       /* color: surface tension */
    double beta;        /* color: recoloring parameter */
} lbo_params;

typedef struct lbo_sim lbo_sim;

/* Error codes returned by the stepping calls (the reference throws). */
enum { LBO_OK = 0, LBO_ERR_ARG = -1, LBO_ERR_DENSITY = -2, LBO_ERR_COMPONENT = -3,
       LBO_ERR_TAU = -4, LBO_ERR_VELOCITY = -5, LBO_ERR_NONFINITE = -6 };

lbo_sim *lbo_create(const lbo_params *p, const lbo_label labels[256], const uint8_t *geometry);
void     lbo_destroy(lbo_sim *s);
/* t = 0: initialize + calcMacroVar + bodyForce (macros then match the t=0 VTI),
 * without the initial collision. */
int      lbo_initialize(lbo_sim *s);
/* The collision (post-macro), as called once at t = 0 and at the end of a step. */
int      lbo_collide(lbo_sim *s);
/* n full steps: streaming, bounce-back, macros, body force, collision. */
int      lbo_step(lbo_sim *s, int n);
/* Stream + bounce-back + macros + body force only (the state a report sees). */
int      lbo_stream_macros(lbo_sim *s);
size_t   lbo_voxels(const lbo_sim *s);
int      lbo_q(const lbo_sim *s);
void     lbo_get_populations(const lbo_sim *s, double *out);   /* [phase][q][N] */
void     lbo_set_populations(lbo_sim *s, const double *in);    /* [phase][q][N] */
/* rho0 (single phase: density), rho1 (color only, may be NULL), u as [3][N] in
 * x,y,z order (z = 0 in 2D). */
void     lbo_get_macros(const lbo_sim *s, double *rho0, double *rho1, double *u);
/* Color phase field (rho0-rho1)/rho on fluid voxels, 86 on solids. */
void     lbo_get_phi(const lbo_sim *s, double *phi);
/* Link classification: per voxel, bit (q-1) set when voxel is a fluid voxel
 * whose q-neighbour is a BB/SD solid; 0 elsewhere. */
void     lbo_link_mask(const lbo_sim *s, uint32_t *out);
/* Wall data per voxel (0 away from walls): mean contact angle cos/sin. */
void     lbo_wall_angles(const lbo_sim *s, double *cosca, double *sinca);
/* The MRT matrices the reference builds: M, M^-1 (QxQ row-major) and S at tau. */
void     lbo_mrt_tables(int q, double tau, double *m, double *minv, double *s);

#ifdef __cplusplus
}
#endif
#endif
