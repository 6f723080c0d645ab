/* CPU restatement of LBFlow's solver step loop -- TEST INFRASTRUCTURE ONLY.
 *
 * The CUDA engine is checked against this file (and this file against the
 * reference binary built by `make ref`).  It is never part of the product
 * path.  Each routine names the reference function it restates; citations are
 * file:line within the zhou1800/lbflow project.  Arithmetic is written in the
 * reference's order (left-to-right sums starting from 0.0, the same operand
 * grouping) so that, compiled without FMA contraction, it reproduces the
 * reference bit for bit. */
#include "lbm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define QMAX 19
#define SOLID_DENS_N 86.0   /* colorfluid.cpp:49 */

/* ---- lattice tables (solver/src/grid/gridspace.cpp:82-144) ------------------
 * Vectors are stored in the reference's component order: {y,x} in 2D and
 * {z,y,x} in 3D.  The q ordering fixes the checkpoint block order. */
static const int E9[9][3] = { {0,0,0},{0,1,0},{1,0,0},{0,-1,0},{-1,0,0},
                              {1,1,0},{1,-1,0},{-1,-1,0},{-1,1,0} };
static const int OP9[9] = {0,3,4,1,2,7,8,5,6};
static const int E19[19][3] = { {0,0,0},{0,0,1},{0,0,-1},
    {0,1,0},{0,-1,0},{1,0,0},{-1,0,0},
    {0,1,1},{0,1,-1},{0,-1,1},{0,-1,-1},
    {1,0,1},{1,0,-1},{-1,0,1},{-1,0,-1},
    {1,1,0},{1,-1,0},{-1,1,0},{-1,-1,0} };
static const int OP19[19] = {0,2,1,4,3,6,5,10,9,8,7,14,13,12,11,18,17,16,15};
/* QrelD: per axis, the directions entering the gradient (gridspace.cpp:93,132-134). */
static const int RELD9[2][6] = { {2,5,6,4,7,8}, {1,5,8,3,6,7} };
static const int RELD19[3][10] = { {5,11,12,15,16,6,13,14,17,18},
                                   {3,8,7,15,17,4,9,10,16,18},
                                   {1,7,9,11,13,2,8,10,12,14} };

/* Zou-He tables per boundary direction dir = 1..2D (gridspace.cpp:87-91 for
 * D2Q9, 122-141 for D3Q19): REL[dir] = the directions with the same sign as
 * dir along its axis, in the reference's order; PERP[dir] = the directions
 * with no component along it; AXIS[dir] = its component index ({y,x} or
 * {z,y,x}); SIGN[dir] = +1 or -1. */
static const int REL9[5][3] = { {0,0,0}, {1,5,8}, {2,5,6}, {3,6,7}, {4,7,8} };
static const int PERP9[5][3] = { {0,0,0}, {0,2,4}, {0,1,3}, {0,2,4}, {0,1,3} };
static const int AXIS9[5] = {0, 1, 0, 1, 0};
static const int SIGN9[5] = {0, 1, 1, -1, -1};
static const int REL19[7][5] = { {0,0,0,0,0},
    {1,7,9,11,13}, {2,8,10,12,14}, {3,8,7,15,17}, {4,9,10,16,18},
    {5,11,12,15,16}, {6,13,14,17,18} };
static const int PERP19[7][9] = { {0,0,0,0,0,0,0,0,0},
    {0,3,4,5,6,15,16,17,18}, {0,3,4,5,6,15,16,17,18},
    {0,1,2,5,6,11,12,13,14}, {0,1,2,5,6,11,12,13,14},
    {0,1,2,3,4,7,8,9,10}, {0,1,2,3,4,7,8,9,10} };
static const int AXIS19[7] = {0, 2, 2, 1, 1, 0, 0};
static const int SIGN19[7] = {0, 1, -1, 1, -1, 1, -1};

/* MRT transform matrices (solver/src/lbm/simulator.cpp:162-197). */
static const double M9[81] = {
     1, 1, 1, 1, 1, 1, 1, 1, 1,
    -4,-1,-1,-1,-1, 2, 2, 2, 2,
     4,-2,-2,-2,-2, 1, 1, 1, 1,
     0, 1, 0,-1, 0, 1,-1,-1, 1,
     0,-2, 0, 2, 0, 1,-1,-1, 1,
     0, 0, 1, 0,-1, 1, 1,-1,-1,
     0, 0,-2, 0, 2, 1, 1,-1,-1,
     0, 1,-1, 1,-1, 0, 0, 0, 0,
     0, 0, 0, 0, 0, 1,-1, 1,-1 };
static const double M19[361] = {
      1,  1,  1,  1,  1,  1,  1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1,
    -30,-11,-11,-11,-11,-11,-11, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8,
     12, -4, -4, -4, -4, -4, -4, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1,
      0,  1, -1,  0,  0,  0,  0, 1,-1, 1,-1, 1,-1, 1,-1, 0, 0, 0, 0,
      0, -4,  4,  0,  0,  0,  0, 1,-1, 1,-1, 1,-1, 1,-1, 0, 0, 0, 0,
      0,  0,  0,  1, -1,  0,  0, 1, 1,-1,-1, 0, 0, 0, 0, 1,-1, 1,-1,
      0,  0,  0, -4,  4,  0,  0, 1, 1,-1,-1, 0, 0, 0, 0, 1,-1, 1,-1,
      0,  0,  0,  0,  0,  1, -1, 0, 0, 0, 0, 1, 1,-1,-1, 1, 1,-1,-1,
      0,  0,  0,  0,  0, -4,  4, 0, 0, 0, 0, 1, 1,-1,-1, 1, 1,-1,-1,
      0,  2,  2, -1, -1, -1, -1, 1, 1, 1, 1, 1, 1, 1, 1,-2,-2,-2,-2,
      0, -4, -4,  2,  2,  2,  2, 1, 1, 1, 1, 1, 1, 1, 1,-2,-2,-2,-2,
      0,  0,  0,  1,  1, -1, -1, 1, 1, 1, 1,-1,-1,-1,-1, 0, 0, 0, 0,
      0,  0,  0, -2, -2,  2,  2, 1, 1, 1, 1,-1,-1,-1,-1, 0, 0, 0, 0,
      0,  0,  0,  0,  0,  0,  0, 1,-1,-1, 1, 0, 0, 0, 0, 0, 0, 0, 0,
      0,  0,  0,  0,  0,  0,  0, 0, 0, 0, 0, 0, 0, 0, 0, 1,-1,-1, 1,
      0,  0,  0,  0,  0,  0,  0, 0, 0, 0, 0, 1,-1,-1, 1, 0, 0, 0, 0,
      0,  0,  0,  0,  0,  0,  0, 1,-1, 1,-1,-1, 1,-1, 1, 0, 0, 0, 0,
      0,  0,  0,  0,  0,  0,  0,-1,-1, 1, 1, 0, 0, 0, 0, 1,-1, 1,-1,
      0,  0,  0,  0,  0,  0,  0, 0, 0, 0, 0, 1, 1,-1,-1,-1,-1, 1, 1 };

struct lbo_sim {
    lbo_params p;
    lbo_label lab[256];
    int D, Q;
    size_t N;
    size_t sz[3];       /* reference order: {y,x} or {z,y,x} */
    size_t stride[3];
    int e[QMAX][3];     /* D components used */
    int op[QMAX];
    int reld[3][10];
    int nreld;
    double w[QMAX], qnorm[QMAX], qp[QMAX][3];
    uint8_t *geom;
    int phases;
    double *f, *fold;   /* [phase][q][N] */
    double *dens[2], *densT, *densN, *tau, *v[3];
    /* MRT */
    double M[QMAX*QMAX], MInv[QMAX*QMAX];
    double MInvSMT[QMAX*QMAX], forceMatrix[QMAX*QMAX];
    double uniformCollision[QMAX*QMAX], uniformForce[QMAX*QMAX];
    /* color weights */
    double ai[2][QMAX], bi[QMAX];
    /* link classification */
    uint32_t *link;     /* bit (q-1): q-neighbour solid */
    uint32_t *film[2];  /* bit (q-1): q-neighbour a half film (HF) of phase 0 / 1 */
    size_t *ibI;        /* 0 = not a wall node, else 1-based wall id */
    size_t nwall;
    double *ibSin, *ibCos, *tib, *tibInv, *ibNorm;  /* per wall id */
};

/* ---- small dense helpers (solver/src/algorithm/fn.cpp) ---------------------- */
/* MatMulMat (fn.cpp:53-68): r[i][j] = sum_k a[i][k] * b[k][j], from 0.0. */
static void matmul(const double *a, const double *b, int m, int p, int n, double *r)
{
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < n; ++j) {
            double s = 0.0;
            for (int k = 0; k < p; ++k) s += a[i*p + k] * b[k*n + j];
            r[i*n + j] = s;
        }
}
/* MatMulVec (fn.cpp:29-39): r[i] = sum_k v[k] * m[i][k], from 0.0. */
static void matvec(const double *m, const double *v, int rows, int cols, double *r)
{
    for (int i = 0; i < rows; ++i) {
        double s = 0.0;
        for (int k = 0; k < cols; ++k) s += v[k] * m[i*cols + k];
        r[i] = s;
    }
}
/* InvOrthoRow (fn.cpp:204-218): inverse of a matrix with orthogonal rows. */
static void inv_ortho_row(const double *mat, int m, int n, double *r)
{
    for (int j = 0; j < m; ++j) {
        double s = 0.0;
        for (int k = 0; k < n; ++k) s += mat[j*n + k] * mat[j*n + k];
        s = 1 / s;
        for (int i = 0; i < n; ++i) r[m*i + j] = mat[j*n + i] * s;
    }
}
/* RotateT2D/RotateTx3D/RotateTz3D (fn.cpp:118-166). */
static void rot_cs(double o, double a, double *c, double *s)
{
    double h = sqrt(o * o + a * a);
    *c = 1; *s = 0;
    if (h != 0) { *c = a / h; *s = o / h; }
}
static void rot2d(double o, double a, double *r)
{ double c, s; rot_cs(o, a, &c, &s); r[0] = c; r[1] = -s; r[2] = s; r[3] = c; }
static void rotx3d(double o, double a, double *r)
{
    double c, s; rot_cs(o, a, &c, &s);
    r[0] = c; r[1] = -s; r[2] = 0; r[3] = s; r[4] = c; r[5] = 0; r[6] = 0; r[7] = 0; r[8] = 1;
}
static void rotz3d(double o, double a, double *r)
{
    double c, s; rot_cs(o, a, &c, &s);
    r[0] = 1; r[1] = 0; r[2] = 0; r[3] = 0; r[4] = c; r[5] = -s; r[6] = 0; r[7] = s; r[8] = c;
}

/* Simulator::getMRTS (simulator.cpp:199-216), legacy spectrum. */
static void mrt_rates(int Q, double rt, double *s)
{
    const double su = 1.0 / rt;
    const double sq = 8.0 * (2.0 - su) / (8.0 - su);
    if (Q == 9) {
        const double r[9] = {0, su, su, 0, sq, 0, sq, su, su};
        memcpy(s, r, sizeof r);
    } else {
        const double r[19] = {0, su, su, 0, sq, 0, sq, 0, sq, su, su, su, su,
                              su, su, su, sq, sq, sq};
        memcpy(s, r, sizeof r);
    }
}

void lbo_mrt_tables(int q, double tau, double *m, double *minv, double *s)
{
    const double *src = q == 9 ? M9 : M19;
    memcpy(m, src, sizeof(double) * (size_t)(q * q));
    inv_ortho_row(src, q, q, minv);
    mrt_rates(q, tau, s);
}

/* Voxels that carry populations (the fluid sets of initialize, collision and
 * buildIb: VD, GV, PB, VB and, for the color model, HF). */
static int is_fluid_type(int t) { return t == LBO_VD || t == LBO_GV || t == LBO_PB || t == LBO_VB || t == LBO_HF; }
/* Voxels whose moments come from the populations (calcMacroVar's VD, GV). */
static int is_bulk_type(int t) { return t == LBO_VD || t == LBO_GV; }
static int is_solid_type(int t) { return t == LBO_BB || t == LBO_SD; }

/* Grid::calcAdjI (solver/inc/grid/grid.h:179-189): periodic neighbour. */
static size_t adj(const lbo_sim *s, size_t i, int q)
{
    size_t a = i;
    for (int d = 0; d < s->D; ++d) {
        size_t block = s->stride[d] * s->sz[d];
        a += (i + (size_t)((long)s->e[q][d] * (long)s->stride[d]) + block) % block - i % block;
    }
    return a;
}

/* Simulator::forceForIndex (simulator.cpp:218-228). */
static void label_force(const lbo_sim *s, int label, double *force)
{
    for (int d = 0; d < 3; ++d) force[d] = 0.0;
    const lbo_label *l = &s->lab[label];
    if (l->type != LBO_GV) return;
    for (int d = 0; d < s->D; ++d) force[d] = s->qp[l->dir][d] * l->value;
}

/* Simulator::forceSource (simulator.cpp:230-246). */
static void force_source(const lbo_sim *s, size_t i, const double *force, double *src)
{
    double uf = 0.0;
    for (int d = 0; d < s->D; ++d) uf += s->v[d][i] * force[d];
    for (int q = 0; q < s->Q; ++q) {
        double eu = 0.0, ef = 0.0;
        for (int d = 0; d < s->D; ++d) {
            eu += s->e[q][d] * s->v[d][i];
            ef += s->e[q][d] * force[d];
        }
        src[q] = s->w[q] * (3.0 * (ef - uf) + 9.0 * eu * ef);
    }
}

/* Simulator::buildIb (simulator.cpp:386-436) and ColorFluid::calcTibNorm
 * (colorfluid.cpp:1111-1129). */
static void build_ib(lbo_sim *s)
{
    static const double pi = 3.1415926535897932384626433832795;
    s->link = calloc(s->N, sizeof(uint32_t));
    s->film[0] = calloc(s->N, sizeof(uint32_t));
    s->film[1] = calloc(s->N, sizeof(uint32_t));
    s->ibI = calloc(s->N, sizeof(size_t));
    size_t cap = 1024, c = 1;
    s->ibSin = malloc(cap * sizeof(double));
    s->ibCos = malloc(cap * sizeof(double));
    s->ibNorm = malloc(cap * 3 * sizeof(double));
    /* Labels in ascending order, voxels in ascending order (set/valarray order). */
    for (int label = 0; label < 256; ++label) {
        if (!is_fluid_type(s->lab[label].type)) continue;
        for (size_t i = 0; i < s->N; ++i) {
            if (s->geom[i] != label) continue;
            int isIB = 0, nCA = 0;
            double norm[3] = {0.0, 0.0, 0.0}, ca = 0;
            for (int q = 1; q < s->Q; ++q) {
                const lbo_label *nb = &s->lab[s->geom[adj(s, i, q)]];
                if (is_solid_type(nb->type)) {
                    s->link[i] |= 1u << (q - 1);
                    isIB = 1;
                    for (int d = 0; d < s->D; ++d) norm[d] -= s->e[q][d];
                    ca += nb->value;
                    nCA++;
                } else if (nb->type == LBO_HF) {   /* half permeable film (simulator.cpp:418-421) */
                    s->film[nb->phase][i] |= 1u << (q - 1);
                }
            }
            if (isIB) {
                if (c >= cap) {
                    cap *= 2;
                    s->ibSin = realloc(s->ibSin, cap * sizeof(double));
                    s->ibCos = realloc(s->ibCos, cap * sizeof(double));
                    s->ibNorm = realloc(s->ibNorm, cap * 3 * sizeof(double));
                }
                ca /= nCA;
                s->ibI[i] = c;
                memcpy(&s->ibNorm[3*c], norm, sizeof norm);
                s->ibSin[c] = sin(ca / 180.0 * pi);
                s->ibCos[c] = cos(ca / 180.0 * pi);
                c++;
            }
        }
    }
    s->nwall = c;
    s->tib = calloc(c * 9, sizeof(double));
    s->tibInv = calloc(c * 9, sizeof(double));
    for (size_t k = 1; k < c; ++k) {
        const double *n = &s->ibNorm[3*k];
        if (s->D == 3) {
            double tx[9], txInv[9], tz[9], tzInv[9];
            rotx3d(n[0], n[1], tx);
            rotx3d(-n[0], n[1], txInv);
            double val = sqrt(n[0] * n[0] + n[1] * n[1]);
            rotz3d(val, n[2], tz);
            rotz3d(-val, n[2], tzInv);
            matmul(tz, tx, 3, 3, 3, &s->tib[9*k]);
            matmul(txInv, tzInv, 3, 3, 3, &s->tibInv[9*k]);
        } else {
            rot2d(n[0], n[1], &s->tib[9*k]);
            rot2d(-n[0], n[1], &s->tibInv[9*k]);
        }
    }
}

lbo_sim *lbo_create(const lbo_params *p, const lbo_label labels[256], const uint8_t *geometry)
{
    if (!p || !labels || !geometry) return NULL;
    if (!((p->dims == 2) || (p->dims == 3))) return NULL;
    lbo_sim *s = calloc(1, sizeof *s);
    s->p = *p;
    memcpy(s->lab, labels, sizeof s->lab);
    s->D = p->dims;
    s->Q = p->dims == 2 ? 9 : 19;
    if (s->D == 2) { s->sz[0] = (size_t)p->ny; s->sz[1] = (size_t)p->nx; }
    else { s->sz[0] = (size_t)p->nz; s->sz[1] = (size_t)p->ny; s->sz[2] = (size_t)p->nx; }
    s->stride[s->D - 1] = 1;
    for (int d = s->D - 1; d > 0; --d) s->stride[d-1] = s->stride[d] * s->sz[d];
    s->N = s->stride[0] * s->sz[0];
    const double ns = sqrt(2), sq = ns / 2;
    for (int q = 0; q < s->Q; ++q) {
        int nz = 0;
        for (int d = 0; d < s->D; ++d) {
            s->e[q][d] = s->D == 2 ? E9[q][d] : E19[q][d];
            nz += s->e[q][d] != 0;
        }
        s->op[q] = s->D == 2 ? OP9[q] : OP19[q];
        s->qnorm[q] = nz == 0 ? 0 : (nz == 1 ? 1 : ns);
        for (int d = 0; d < s->D; ++d)
            s->qp[q][d] = nz == 2 ? s->e[q][d] * sq : (double)s->e[q][d];
    }
    s->nreld = s->D == 2 ? 6 : 10;
    for (int d = 0; d < s->D; ++d)
        for (int k = 0; k < s->nreld; ++k)
            s->reld[d][k] = s->D == 2 ? RELD9[d][k] : RELD19[d][k];
    /* Simulator::getWi (simulator.cpp:438-463). */
    if (s->Q == 9) {
        const double w[9] = {4.0/9, 1.0/9, 1.0/9, 1.0/9, 1.0/9, 1.0/36, 1.0/36, 1.0/36, 1.0/36};
        memcpy(s->w, w, sizeof w);
    } else {
        const double w[19] = {1.0/3, 1.0/18, 1.0/18, 1.0/18, 1.0/18, 1.0/18, 1.0/18,
                              1.0/36, 1.0/36, 1.0/36, 1.0/36, 1.0/36, 1.0/36,
                              1.0/36, 1.0/36, 1.0/36, 1.0/36, 1.0/36, 1.0/36};
        memcpy(s->w, w, sizeof w);
    }
    s->phases = p->color ? 2 : 1;
    for (size_t i = 0; i < s->N; ++i) {
        const lbo_label *l = &labels[geometry[i]];
        int t = l->type;
        if (!is_fluid_type(t) && !is_solid_type(t)) { free(s); return NULL; }
        /* Half films are a two-phase label (ColorFluid::clearHalfFilm). */
        if (t == LBO_HF && (!p->color || l->phase < 0 || l->phase > 1)) { free(s); return NULL; }
        /* FilePrm checks (fileprm.cpp:280-289). */
        if (t == LBO_PB || t == LBO_VB) {
            if (l->dir < 1 || l->dir > 2 * s->D || !isfinite(l->value) ||
                (t == LBO_PB && l->value <= 0.0) || l->phase < 0 || l->phase > (p->color ? 1 : 0)) {
                free(s); return NULL;
            }
        }
    }
    s->geom = malloc(s->N);
    memcpy(s->geom, geometry, s->N);
    const size_t fsz = (size_t)s->phases * (size_t)s->Q * s->N;
    s->f = calloc(fsz, sizeof(double));
    s->fold = calloc(fsz, sizeof(double));
    s->dens[0] = calloc(s->N, sizeof(double));
    s->dens[1] = calloc(s->N, sizeof(double));
    s->densT = calloc(s->N, sizeof(double));
    s->densN = malloc(s->N * sizeof(double));
    for (size_t i = 0; i < s->N; ++i) s->densN[i] = SOLID_DENS_N;
    s->tau = calloc(s->N, sizeof(double));
    for (int d = 0; d < 3; ++d) s->v[d] = calloc(s->N, sizeof(double));

    /* Static MRT operators (scsp.cpp:420-427; colorfluid.cpp:315-322). */
    const int Q = s->Q;
    double S[QMAX], tmp[QMAX*QMAX], MInvSM[QMAX*QMAX], half[QMAX];
    lbo_mrt_tables(Q, p->tau[0], s->M, s->MInv, S);
    for (int i = 0; i < Q; ++i) for (int j = 0; j < Q; ++j) tmp[i*Q + j] = s->MInv[i*Q + j] * S[j];
    matmul(tmp, s->M, Q, Q, Q, MInvSM);
    for (int i = 0; i < Q; ++i) for (int j = 0; j < Q; ++j) s->MInvSMT[i*Q + j] = MInvSM[j*Q + i];
    for (int j = 0; j < Q; ++j) half[j] = 1.0 - 0.5 * S[j];
    for (int i = 0; i < Q; ++i) for (int j = 0; j < Q; ++j) tmp[i*Q + j] = s->MInv[i*Q + j] * half[j];
    matmul(tmp, s->M, Q, Q, Q, s->forceMatrix);
    memcpy(s->uniformCollision, MInvSM, sizeof MInvSM);
    memcpy(s->uniformForce, s->forceMatrix, sizeof s->forceMatrix);

    /* ColorFluid::initPhi (colorfluid.cpp:1131-1150) and getBi (:1152-1168). */
    if (p->color) {
        double alpha[2];
        alpha[0] = p->alpha0;
        alpha[1] = 1 - p->rho[0] / p->rho[1] * (1 - alpha[0]);
        for (int ph = 0; ph < 2; ++ph) {
            if (Q == 9) {
                double a = (1 - alpha[ph]) / 5, b = (1 - alpha[ph]) / 20;
                const double r[9] = {alpha[ph], a, a, a, a, b, b, b, b};
                memcpy(s->ai[ph], r, sizeof r);
            } else {
                double a = (1 - alpha[ph]) / 12, b = (1 - alpha[ph]) / 24;
                for (int q = 0; q < 19; ++q) s->ai[ph][q] = q == 0 ? alpha[ph] : (q < 7 ? a : b);
            }
        }
        if (Q == 9) {
            const double b[9] = {-4.0/27, 2.0/27, 2.0/27, 2.0/27, 2.0/27,
                                 5.0/108, 5.0/108, 5.0/108, 5.0/108};
            memcpy(s->bi, b, sizeof b);
        } else {
            const double x = 2, c2 = 1.0;
            const double b0 = -(2.0 + 2.0*x) / (3.0*x + 12.0) * c2;
            const double b1 = x / (6.0*x + 24.0) * c2;
            const double b7 = 1.0 / (6.0*x + 24.0) * c2;
            for (int q = 0; q < 19; ++q) s->bi[q] = q == 0 ? b0 : (q < 7 ? b1 : b7);
        }
    }
    build_ib(s);
    return s;
}

void lbo_destroy(lbo_sim *s)
{
    if (!s) return;
    free(s->geom); free(s->f); free(s->fold);
    free(s->dens[0]); free(s->dens[1]); free(s->densT); free(s->densN); free(s->tau);
    for (int d = 0; d < 3; ++d) free(s->v[d]);
    free(s->link); free(s->film[0]); free(s->film[1]); free(s->ibI); free(s->ibSin); free(s->ibCos); free(s->ibNorm);
    free(s->tib); free(s->tibInv);
    free(s);
}

#define F(ph, q, i) s->f[((size_t)(ph) * (size_t)s->Q + (size_t)(q)) * s->N + (i)]
#define FO(ph, q, i) s->fold[((size_t)(ph) * (size_t)s->Q + (size_t)(q)) * s->N + (i)]

/* ---- single phase (SCSP) ---------------------------------------------------- */
/* SCSP::initialize (scsp.cpp:116-134). */
static void scsp_initialize(lbo_sim *s)
{
    const double rho = s->p.rho[0];
    for (size_t i = 0; i < s->N; ++i) {
        int label = s->geom[i];
        if (!is_fluid_type(s->lab[label].type)) continue;
        double force[3];
        label_force(s, label, force);
        for (int q = 0; q < s->Q; ++q) {
            F(0, q, i) = s->w[q] * rho;
            double ef = 0.0;
            for (int d = 0; d < s->D; ++d) ef += s->e[q][d] * force[d];
            F(0, q, i) -= 1.5 * s->w[q] * ef;
        }
        s->dens[0][i] = rho;
    }
}

/* SCSP::calcMacroVar (scsp.cpp:136-160) + SCSP::bodyForce (:162-175). */
static int scsp_macros(lbo_sim *s)
{
    const double dens0 = s->p.rho[0];
    int bad = 0;
    /* Voxels are independent: the OpenMP split changes no arithmetic. */
#pragma omp parallel for schedule(static) reduction(|:bad)
    for (size_t i = 0; i < s->N; ++i) {
        if (!is_bulk_type(s->lab[s->geom[i]].type)) continue;
        double r = F(0, 0, i);
        for (int q = 1; q < s->Q; ++q) r += F(0, q, i);
        s->dens[0][i] = r;
        if (!isfinite(r) || r <= 0.0) bad = 1;
        for (int d = 0; d < s->D; ++d) {
            double v = 0;
            for (int q = 1; q < s->Q; ++q) {
                if (s->e[q][d] == 1) v += F(0, q, i);
                else if (s->e[q][d] == -1) v -= F(0, q, i);
            }
            s->v[d][i] = v / dens0;
        }
    }
    if (bad) return LBO_ERR_DENSITY;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < s->N; ++i) {
        int label = s->geom[i];
        if (s->lab[label].type != LBO_GV) continue;
        double force[3];
        label_force(s, label, force);
        for (int d = 0; d < s->D; ++d) s->v[d][i] += force[d] * 0.5 / dens0;
    }
    return LBO_OK;
}

/* SCSP::equilSRT (scsp.cpp:374-409) / SCSP::equilMRT (scsp.cpp:411-464). */
static int scsp_collide(lbo_sim *s)
{
    const int Q = s->Q;
    const double c1 = 3.0, c2 = 4.5, c3 = 1.5;
    const double omega = 1.0 / s->p.tau[0];
    const double dens0 = s->p.rho[0];
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < s->N; ++i) {
        int label = s->geom[i];
        if (!is_fluid_type(s->lab[label].type)) continue;
        double force[3];
        label_force(s, label, force);
        double ff2 = 0.0;
        for (int d = 0; d < s->D; ++d) ff2 += force[d] * force[d];
        const int forced = ff2 != 0.0;
        double usq = 0;
        for (int d = 0; d < s->D; ++d) usq += s->v[d][i] * s->v[d][i];
        double source[QMAX] = {0};
        if (forced) force_source(s, i, force, source);
        if (!s->p.mrt) {
            for (int q = 0; q < Q; ++q) {
                double ui = 0;
                for (int d = 0; d < s->D; ++d) ui += s->v[d][i] * s->e[q][d];
                double feq = s->w[q] * (s->dens[0][i] + dens0 * (c1*ui + c2*ui*ui - c3*usq));
                F(0, q, i) += (feq - F(0, q, i)) * omega;
                if (forced) F(0, q, i) += (1.0 - 0.5 * omega) * source[q];
            }
        } else {
            double ff[QMAX] = {0};
            const double *im = s->MInvSMT;
            for (int q = 0; q < Q; ++q) {
                double ui = 0;
                for (int d = 0; d < s->D; ++d) ui += s->v[d][i] * s->e[q][d];
                double feq = s->w[q] * (s->dens[0][i] + dens0 * (c1*ui + c2*ui*ui - c3*usq));
                for (int qq = 0; qq < Q; ++qq) ff[qq] += *im++ * (feq - F(0, q, i));
            }
            for (int q = 0; q < Q; ++q) F(0, q, i) += ff[q];
            if (forced) {
                double corr[QMAX];
                matvec(s->forceMatrix, source, Q, Q, corr);
                for (int q = 0; q < Q; ++q) F(0, q, i) += corr[q];
            }
        }
    }
    /* Simulator::validatePopulations (simulator.cpp:327-333). */
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(|:bad)
    for (size_t k = 0; k < (size_t)Q * s->N; ++k)
        if (!isfinite(s->f[k])) bad = 1;
    return bad ? LBO_ERR_NONFINITE : LBO_OK;
}

/* SCSP::zouHeBoundary (scsp.cpp:188-275): velocity (VB) and pressure (PB)
 * boundary voxels get their density and velocity from the known populations,
 * then every unknown population (those along the boundary's direction) is
 * rebuilt from its opposite.  wiT = 6 w / latticeSpeed (simulator.cpp:28),
 * latticeSpeed = 1. */
static void scsp_zou_he(lbo_sim *s)
{
    const int D = s->D;
    for (size_t i = 0; i < s->N; ++i) {
        const lbo_label *l = &s->lab[s->geom[i]];
        if (l->type != LBO_PB && l->type != LBO_VB) continue;
        const int dir = l->dir;
        const int nrel = D == 2 ? 3 : 5, nperp = D == 2 ? 3 : 9;
        const int opdir = s->op[dir];
        const int *oprel = D == 2 ? REL9[opdir] : REL19[opdir];
        const int *perp = D == 2 ? PERP9[dir] : PERP19[dir];
        const int axis = D == 2 ? AXIS9[dir] : AXIS19[dir];
        const int sign = D == 2 ? SIGN9[dir] : SIGN19[dir];
        double sumF = 0;
        for (int k = 0; k < nrel; ++k) sumF += F(0, oprel[k], i) + F(0, oprel[k], i);
        for (int k = 0; k < nperp; ++k) sumF += F(0, perp[k], i);
        if (l->type == LBO_VB) {
            const double velocity = sign == 1 ? l->value : -l->value;
            const double vel_1 = 1.0 / (1.0 - velocity);
            for (int d = 0; d < D; ++d) s->v[d][i] = 0;
            s->v[axis][i] = velocity;
            s->dens[0][i] = sumF * vel_1;
        } else {
            const double density = l->value;
            s->dens[0][i] = density;
            for (int d = 0; d < D; ++d) s->v[d][i] = 0;
            sumF /= density;
            sumF--;
            s->v[axis][i] = sign == 1 ? -sumF : sumF;
        }
    }
    for (size_t i = 0; i < s->N; ++i) {
        const lbo_label *l = &s->lab[s->geom[i]];
        if (l->type != LBO_PB && l->type != LBO_VB) continue;
        const int dir = l->dir;
        const int nrel = D == 2 ? 3 : 5, nperp = D == 2 ? 3 : 9;
        const int *rel = D == 2 ? REL9[dir] : REL19[dir];
        const int *perp = D == 2 ? PERP9[dir] : PERP19[dir];
        const int axis = D == 2 ? AXIS9[dir] : AXIS19[dir];
        const int sign = D == 2 ? SIGN9[dir] : SIGN19[dir];
        for (int k = 0; k < nrel; ++k) {
            const int q = rel[k];
            F(0, q, i) = F(0, s->op[q], i);
            F(0, q, i) += sign * (6.0 * s->w[q]) * s->dens[0][i] * s->v[axis][i];
            double sumF = 0;
            for (int m = 0; m < nperp; ++m) {
                const int qn = perp[m];
                for (int d = 0; d < D; ++d) {
                    if (s->e[qn][d] == 0 || s->e[q][d] == 0) continue;
                    else if (s->e[qn][d] == s->e[q][d]) sumF += F(0, qn, i);
                    else sumF -= F(0, qn, i);
                }
            }
            F(0, q, i) -= sumF * 0.5;
        }
    }
}

/* ---- two-phase color gradient (ColorFluid) ----------------------------------- */
/* ColorFluid::zouHeBoundary (colorfluid.cpp:638-734): the single-phase rule
 * applied to the total distribution f0 + f1; the rebuilt unknowns go to the
 * label's phase and the other phase's unknowns are cleared.  The density and
 * velocity it sets are intermediates: calcMacroVar recomputes them from the
 * populations (PB/VB are in its node set). */
static void color_zou_he(lbo_sim *s)
{
    const int D = s->D;
    for (size_t i = 0; i < s->N; ++i) {
        const lbo_label *l = &s->lab[s->geom[i]];
        if (l->type != LBO_PB && l->type != LBO_VB) continue;
        const int dir = l->dir;
        const int nrel = D == 2 ? 3 : 5, nperp = D == 2 ? 3 : 9;
        const int *oprel = D == 2 ? REL9[s->op[dir]] : REL19[s->op[dir]];
        const int *perp = D == 2 ? PERP9[dir] : PERP19[dir];
        const int axis = D == 2 ? AXIS9[dir] : AXIS19[dir];
        const int sign = D == 2 ? SIGN9[dir] : SIGN19[dir];
        double sumF = 0;
        for (int k = 0; k < nrel; ++k)
            sumF += F(0, oprel[k], i) + F(0, oprel[k], i) + F(1, oprel[k], i) + F(1, oprel[k], i);
        for (int k = 0; k < nperp; ++k) sumF += F(0, perp[k], i) + F(1, perp[k], i);
        for (int d = 0; d < D; ++d) s->v[d][i] = 0;
        if (l->type == LBO_VB) {
            const double velocity = sign == 1 ? l->value : -l->value;
            const double vel_1 = 1.0 / (1.0 - velocity);
            s->v[axis][i] = velocity;
            s->densT[i] = sumF * vel_1;
        } else {
            const double density = l->value;
            s->densT[i] = density;
            sumF /= density;
            sumF--;
            s->v[axis][i] = sign == 1 ? -sumF : sumF;
        }
    }
    for (size_t i = 0; i < s->N; ++i) {
        const lbo_label *l = &s->lab[s->geom[i]];
        if (l->type != LBO_PB && l->type != LBO_VB) continue;
        const int dir = l->dir;
        const int nrel = D == 2 ? 3 : 5, nperp = D == 2 ? 3 : 9;
        const int *rel = D == 2 ? REL9[dir] : REL19[dir];
        const int *perp = D == 2 ? PERP9[dir] : PERP19[dir];
        const int axis = D == 2 ? AXIS9[dir] : AXIS19[dir];
        const int sign = D == 2 ? SIGN9[dir] : SIGN19[dir];
        const int phs = l->phase, phsOp = 1 - phs;
        for (int k = 0; k < nrel; ++k) {
            const int q = rel[k];
            double fT = F(0, s->op[q], i) + F(1, s->op[q], i);
            fT += sign * (6.0 * s->w[q]) * s->densT[i] * s->v[axis][i];
            double sumF = 0;
            for (int m = 0; m < nperp; ++m) {
                const int qn = perp[m];
                for (int d = 0; d < D; ++d) {
                    if (s->e[qn][d] == 0 || s->e[q][d] == 0) continue;
                    else if (s->e[qn][d] == s->e[q][d]) sumF += F(0, qn, i) + F(1, qn, i);
                    else sumF -= F(0, qn, i) + F(1, qn, i);
                }
            }
            fT -= sumF * 0.5;
            F(phs, q, i) = fT;
            F(phsOp, q, i) = 0;
        }
    }
}

/* ColorFluid::initialize (colorfluid.cpp:214-236). */
static void color_initialize(lbo_sim *s)
{
    for (size_t i = 0; i < s->N; ++i) {
        int label = s->geom[i];
        if (!is_fluid_type(s->lab[label].type)) continue;
        int phs = s->lab[label].phase;
        double force[3];
        label_force(s, label, force);
        for (int q = 0; q < s->Q; ++q) {
            F(phs, q, i) = s->ai[phs][q] * s->p.rho[phs];
            double ef = 0.0;
            for (int d = 0; d < s->D; ++d) ef += s->e[q][d] * force[d];
            F(phs, q, i) -= 1.5 * s->w[q] * ef;
        }
        s->densT[i] = s->dens[phs][i] = s->p.rho[phs];
        s->densN[i] = phs == 0 ? 1 : -1;
    }
}

/* ColorFluid::calcMacroVar (colorfluid.cpp:238-290) + bodyForce (:736-750). */
static int color_macros_voxel(lbo_sim *s, size_t i, double relax0, double relax1)
{
    double d0 = F(0, 0, i), d1 = F(1, 0, i);
    for (int q = 1; q < s->Q; ++q) { d0 += F(0, q, i); d1 += F(1, q, i); }
    s->dens[0][i] = d0; s->dens[1][i] = d1;
    double dt = d0 + d1;
    s->densT[i] = dt;
    if (!isfinite(d0) || !isfinite(d1) || !isfinite(dt) || dt <= 0.0) return LBO_ERR_DENSITY;
    if (d0 < -1e-10 * dt || d1 < -1e-10 * dt) return LBO_ERR_COMPONENT;
    s->densN[i] = (d0 - d1) / dt;
    s->tau[i] = (1 + s->densN[i]) * relax0 + (1 - s->densN[i]) * relax1;
    if (!isfinite(s->tau[i]) || s->tau[i] <= 0.5) return LBO_ERR_TAU;
    for (int d = 0; d < s->D; ++d) {
        double v = 0;
        for (int q = 1; q < s->Q; ++q) {
            if (s->e[q][d] == 1) v += F(0, q, i) + F(1, q, i);
            else if (s->e[q][d] == -1) v -= F(0, q, i) + F(1, q, i);
        }
        v /= dt;
        s->v[d][i] = v;
        if (!isfinite(v)) return LBO_ERR_VELOCITY;
    }
    return LBO_OK;
}

static int color_macros(lbo_sim *s)
{
    const double relax0 = s->p.tau[0] / 2.0, relax1 = s->p.tau[1] / 2.0;
    int bad = 0;
    /* Voxels are independent; the first failing voxel in voxel order names
     * the error, as in the reference's sequential loop. */
#pragma omp parallel for schedule(static) reduction(|:bad)
    for (size_t i = 0; i < s->N; ++i) {
        if (!is_fluid_type(s->lab[s->geom[i]].type)) continue;
        if (color_macros_voxel(s, i, relax0, relax1) != LBO_OK) bad = 1;
    }
    if (bad)
        for (size_t i = 0; i < s->N; ++i) {
            if (!is_fluid_type(s->lab[s->geom[i]].type)) continue;
            const int rc = color_macros_voxel(s, i, relax0, relax1);
            if (rc != LBO_OK) return rc;
        }
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < s->N; ++i) {
        int label = s->geom[i];
        if (s->lab[label].type != LBO_GV) continue;
        double force[3];
        label_force(s, label, force);
        for (int d = 0; d < s->D; ++d) s->v[d][i] += force[d] * 0.5 / s->densT[i];
    }
    return LBO_OK;
}

/* ColorFluid::colorGradient, legacy interior and geometric-wall branches
 * (colorfluid.cpp:435-486, 550-567). */
static void color_gradient(const lbo_sim *s, size_t i, double *g, double *norm)
{
    const int D = s->D;
    for (int d = 0; d < 3; ++d) g[d] = 0.0;
    if (!s->ibI[i]) {
        for (int d = 0; d < D; ++d)
            for (int k = 0; k < s->nreld; ++k) {
                int q = s->reld[d][k];
                double nb = s->densN[adj(s, i, q)];
                if (s->e[q][d] == 1) g[d] += s->w[q] * nb;
                else g[d] -= s->w[q] * nb;
            }
        double n2 = 0.0;
        for (int d = 0; d < D; ++d) g[d] *= 3.0;
        for (int d = 0; d < D; ++d) n2 += g[d] * g[d];
        *norm = sqrt(n2);
        return;
    }
    for (int d = 0; d < D; ++d)
        for (int k = 0; k < s->nreld; ++k) {
            int q = s->reld[d][k];
            double n0 = s->densN[i];
            double nq = s->densN[adj(s, i, q)];
            if (nq == SOLID_DENS_N) continue;
            if (s->e[q][d] == 1) g[d] += s->w[q] * (nq - n0);
            else g[d] -= s->w[q] * (nq - n0);
        }
    double n2 = 0.0;
    for (int d = 0; d < D; ++d) g[d] *= 3.0;
    for (int d = 0; d < D; ++d) n2 += g[d] * g[d];
    *norm = sqrt(n2);
    const size_t c = s->ibI[i];
    const double cA = s->ibCos[c], sA = s->ibSin[c];
    if (D == 3) {
        double gn[3], txInv[9], tInv[9], t[3];
        matmul(&s->tib[9*c], g, 3, 3, 1, gn);
        rotx3d(-gn[0], gn[1], txInv);
        matmul(&s->tibInv[9*c], txInv, 3, 3, 3, tInv);
        t[0] = 0; t[1] = *norm * sA; t[2] = *norm * cA;
        matmul(tInv, t, 3, 3, 1, g);
    } else {
        double gn[2], t[2];
        matmul(&s->tib[9*c], g, 2, 2, 1, gn);
        if (gn[0] >= 0) { t[0] = *norm * sA; t[1] = *norm * cA; }
        else { t[0] = -*norm * sA; t[1] = *norm * cA; }
        matmul(&s->tibInv[9*c], t, 2, 2, 1, g);
    }
}

/* ColorFluid::collision (colorfluid.cpp:292-433), perturbation capillary model
 * with cosine recoloring. */
static int color_collide(lbo_sim *s)
{
    const int Q = s->Q, D = s->D;
    const double c1 = 3.0, c2 = 4.5, c3 = 1.5;
    const double ak = 2.25 * s->p.sigma;
    const double beta = s->p.beta;
    const int uniformTau = s->p.tau[0] == s->p.tau[1];
    double *out0 = malloc(sizeof(double) * (size_t)Q * s->N);
    double *out1 = malloc(sizeof(double) * (size_t)Q * s->N);
    memcpy(out0, &F(0, 0, 0), sizeof(double) * (size_t)Q * s->N);
    memcpy(out1, &F(1, 0, 0), sizeof(double) * (size_t)Q * s->N);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < s->N; ++i) {
        int label = s->geom[i];
        if (!is_fluid_type(s->lab[label].type)) continue;
        double force[3];
        label_force(s, label, force);
        double ff2 = 0.0;
        for (int d = 0; d < D; ++d) ff2 += force[d] * force[d];
        const int forced = ff2 != 0.0;
        double usq = 0;
        for (int d = 0; d < D; ++d) usq += s->v[d][i] * s->v[d][i];
        double feq_u0[QMAX], fT[QMAX], source[QMAX] = {0};
        if (forced) force_source(s, i, force, source);
        const double d0 = s->dens[0][i], d1 = s->dens[1][i], dt = s->densT[i], tau = s->tau[i];
        if (!s->p.mrt) {
            for (int q = 0; q < Q; ++q) {
                fT[q] = F(0, q, i) + F(1, q, i);
                double ui = 0;
                for (int d = 0; d < D; ++d) ui += s->v[d][i] * s->e[q][d];
                feq_u0[q] = d0 * s->ai[0][q] + d1 * s->ai[1][q];
                double feq = feq_u0[q] + dt * s->w[q] * (c1*ui + c2*ui*ui - c3*usq);
                fT[q] += (feq - fT[q]) / tau;
                if (forced) fT[q] += (1.0 - 0.5 / tau) * source[q];
            }
        } else {
            double residual[QMAX], corr[QMAX];
            for (int q = 0; q < Q; ++q) {
                fT[q] = F(0, q, i) + F(1, q, i);
                double ui = 0;
                for (int d = 0; d < D; ++d) ui += s->v[d][i] * s->e[q][d];
                feq_u0[q] = d0 * s->ai[0][q] + d1 * s->ai[1][q];
                double feq = feq_u0[q] + dt * s->w[q] * (c1*ui + c2*ui*ui - c3*usq);
                residual[q] = feq - fT[q];
            }
            if (uniformTau) {
                matvec(s->uniformCollision, residual, Q, Q, corr);
                if (forced) {
                    double extra[QMAX];
                    matvec(s->uniformForce, source, Q, Q, extra);
                    for (int q = 0; q < Q; ++q) corr[q] += extra[q];
                }
            } else {
                double rates[QMAX], mr[QMAX];
                mrt_rates(Q, tau, rates);
                matvec(s->M, residual, Q, Q, mr);
                for (int q = 0; q < Q; ++q) mr[q] = mr[q] * rates[q];
                if (forced) {
                    double ms[QMAX];
                    matvec(s->M, source, Q, Q, ms);
                    for (int q = 0; q < Q; ++q) mr[q] += ms[q] * (1.0 - 0.5 * rates[q]);
                }
                matvec(s->MInv, mr, Q, Q, corr);
            }
            for (int q = 0; q < Q; ++q) fT[q] += corr[q];
        }
        double g[3], norm = 0.0;
        color_gradient(s, i, g, &norm);
        const double dens0T = d0 / dt;
        if (norm > 1e-9) {
            const double betaDens01TT = beta * dens0T * d1 / dt;
            const double AkNorm = ak * norm / tau;
            for (int q = 0; q < Q; ++q) {
                double angle = 0.0;
                for (int d = 0; d < D; ++d) {
                    if (s->e[q][d] == 1) angle += g[d];
                    else if (s->e[q][d] == -1) angle -= g[d];
                }
                angle /= norm;
                fT[q] += AkNorm * (s->w[q] * angle * angle - s->bi[q]);
                if (q != 0) angle /= s->qnorm[q];
                const double a = dens0T * fT[q] + betaDens01TT * angle * feq_u0[q];
                out0[(size_t)q * s->N + i] = a;
                out1[(size_t)q * s->N + i] = fT[q] - a;
            }
        } else {
            for (int q = 0; q < Q; ++q) {
                const double a = dens0T * fT[q];
                out0[(size_t)q * s->N + i] = a;
                out1[(size_t)q * s->N + i] = fT[q] - a;
            }
        }
    }
    memcpy(&F(0, 0, 0), out0, sizeof(double) * (size_t)Q * s->N);
    memcpy(&F(1, 0, 0), out1, sizeof(double) * (size_t)Q * s->N);
    free(out0); free(out1);
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(|:bad)
    for (size_t k = 0; k < 2 * (size_t)Q * s->N; ++k)
        if (!isfinite(s->f[k])) bad = 1;
    return bad ? LBO_ERR_NONFINITE : LBO_OK;
}

/* ---- common step pieces ----------------------------------------------------- */
/* Simulator::streaming (simulator.cpp:73-101): every voxel (fluid and solid)
 * pushes f_q one link along e_q with periodic wrap; fold keeps the pre-stream
 * (post-collision) values.  Simulator::bounceBack (simulator.cpp:103-111):
 * a fluid voxel whose q-neighbour is solid gets f_{op q} = fold_q. */
static void stream_bounce(lbo_sim *s)
{
    const size_t total = (size_t)s->phases * (size_t)s->Q * s->N;
    memcpy(s->fold, s->f, total * sizeof(double));
    for (int ph = 0; ph < s->phases; ++ph)
        for (int q = 1; q < s->Q; ++q) {
            /* adj(., q) is a bijection of the voxels: each target is written once. */
#pragma omp parallel for schedule(static)
            for (size_t i = 0; i < s->N; ++i) F(ph, q, adj(s, i, q)) = FO(ph, q, i);
        }
    for (int ph = 0; ph < s->phases; ++ph)
        for (int q = 1; q < s->Q; ++q) {
            const int opq = s->op[q];
#pragma omp parallel for schedule(static)
            for (size_t i = 0; i < s->N; ++i)
                if (s->link[i] & (1u << (q - 1))) F(ph, opq, i) = FO(ph, q, i);
        }
    if (s->phases == 2) {
        /* ColorFluid::Run (colorfluid.cpp:155-158): phase 0 bounces back from
         * films of phase 1 and phase 1 from films of phase 0; then
         * clearHalfFilm (colorfluid.cpp:752-765) empties the other phase at
         * every film voxel. */
        for (int ph = 0; ph < 2; ++ph)
            for (int q = 1; q < s->Q; ++q) {
                const int opq = s->op[q];
                for (size_t i = 0; i < s->N; ++i)
                    if (s->film[1 - ph][i] & (1u << (q - 1))) F(ph, opq, i) = FO(ph, q, i);
            }
        for (size_t i = 0; i < s->N; ++i) {
            const lbo_label *l = &s->lab[s->geom[i]];
            if (l->type != LBO_HF) continue;
            for (int q = 0; q < s->Q; ++q) F(1 - l->phase, q, i) = 0;
        }
    }
}

int lbo_initialize(lbo_sim *s)
{
    if (!s) return LBO_ERR_ARG;
    if (s->p.color) { color_initialize(s); return color_macros(s); }
    scsp_initialize(s);
    return scsp_macros(s);
}

int lbo_collide(lbo_sim *s)
{
    if (!s) return LBO_ERR_ARG;
    return s->p.color ? color_collide(s) : scsp_collide(s);
}

int lbo_stream_macros(lbo_sim *s)
{
    if (!s) return LBO_ERR_ARG;
    stream_bounce(s);
    if (s->p.color) {
        color_zou_he(s);
        return color_macros(s);
    }
    scsp_zou_he(s);
    return scsp_macros(s);
}

int lbo_step(lbo_sim *s, int n)
{
    for (int t = 0; t < n; ++t) {
        int rc = lbo_stream_macros(s);
        if (rc) return rc;
        rc = lbo_collide(s);
        if (rc) return rc;
    }
    return LBO_OK;
}

size_t lbo_voxels(const lbo_sim *s) { return s ? s->N : 0; }
int lbo_q(const lbo_sim *s) { return s ? s->Q : 0; }

void lbo_get_populations(const lbo_sim *s, double *out)
{ memcpy(out, s->f, sizeof(double) * (size_t)s->phases * (size_t)s->Q * s->N); }

void lbo_set_populations(lbo_sim *s, const double *in)
{ memcpy(s->f, in, sizeof(double) * (size_t)s->phases * (size_t)s->Q * s->N); }

void lbo_get_macros(const lbo_sim *s, double *rho0, double *rho1, double *u)
{
    if (rho0) memcpy(rho0, s->dens[0], sizeof(double) * s->N);
    if (rho1) memcpy(rho1, s->dens[1], sizeof(double) * s->N);
    if (u) {
        /* reference component d is z,y,x (3D) or y,x (2D); output x,y,z */
        for (int c = 0; c < 3; ++c) {
            int d = s->D - 1 - c;
            for (size_t i = 0; i < s->N; ++i) u[(size_t)c * s->N + i] = d >= 0 ? s->v[d][i] : 0.0;
        }
    }
}

void lbo_get_phi(const lbo_sim *s, double *phi)
{ memcpy(phi, s->densN, sizeof(double) * s->N); }

void lbo_link_mask(const lbo_sim *s, uint32_t *out)
{ memcpy(out, s->link, sizeof(uint32_t) * s->N); }

void lbo_wall_angles(const lbo_sim *s, double *cosca, double *sinca)
{
    for (size_t i = 0; i < s->N; ++i) {
        size_t c = s->ibI[i];
        cosca[i] = c ? s->ibCos[c] : 0.0;
        sinca[i] = c ? s->ibSin[c] : 0.0;
    }
}
