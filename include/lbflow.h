/* lbflow.h -- C ABI of the B200 lattice Boltzmann engine.
 *
 * The engine is the solver core of LBFlow (zhou1800/lbflow) rebuilt for one
 * NVIDIA B200: it replaces the per-step work of SCSP::Run and ColorFluid::Run
 * (solver/src/lbm/scsp.cpp:46-114, solver/src/lbm/colorfluid.cpp:109-212)
 * -- streaming, bounce-back, macroscopic variables, body force, collision, the
 * color-gradient operators and the reductions behind reports and convergence.
 * The C++11 host driver (the LBFlow command line) keeps the parameter file,
 * geometry, VTI and checkpoint formats and calls only the functions below.
 *
 * Conventions
 *  - Plain C types only; host arrays are copied in or out and never retained.
 *  - Dense host arrays use the reference's layout: voxel v = (z*ny + y)*nx + x,
 *    populations [phase][q][v] with the reference's q ordering
 *    (solver/src/grid/gridspace.cpp:82-144), vectors as [3][v] in x, y, z order.
 *  - Every function returns LBF_OK (0) or a negative LBF_E* code; the message
 *    is available from lbf_last_error().  Nothing traps on the device: numeric
 *    failures raise bits of a device error word, read by lbf_status().
 *  - One engine = one geometry on one GPU, driven by one host thread; all work
 *    is queued on the engine's CUDA stream.
 */
#ifndef LBFLOW_H
#define LBFLOW_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBF_ABI_VERSION 1

/* Return codes. */
enum {
    LBF_OK = 0,
    LBF_EINVAL = -1,    /* invalid argument or unsupported option */
    LBF_ECUDA = -2,     /* CUDA runtime failure (message from the runtime) */
    LBF_ESTATE = -3,    /* call out of order (e.g. step before initialize) */
    LBF_ENUMERIC = -4,  /* device error word is non-zero (see lbf_status) */
    LBF_ENOMEM = -5     /* device allocation failed */
};

/* Geometry label types: the bit values of FilePrm::IDXTYPE
 * (solver/inc/file/fileprm.h:44-53). */
enum {
    LBF_VD = 0x1, LBF_GV = 0x2, LBF_PB = 0x4, LBF_VB = 0x8,
    LBF_AB = 0x10, LBF_BB = 0x20, LBF_HF = 0x40, LBF_SD = 0x80
};

enum { LBF_MODEL_SCSP = 0, LBF_MODEL_COLOR = 1 };
enum { LBF_SRT = 0, LBF_MRT = 1 };
/* Population storage.  FP64 is the plain path (FP64 arithmetic).  The others
 * store shifted deviations f_q - w_q*rho0, scaled per direction, and collide
 * in FP32; reductions stay FP64.  BFP16 stores (f_q - w_q*rho0)/w_q as int16
 * mantissas with one power-of-two exponent byte per node (block floating
 * point); single phase only, like FP16 and BF16. */
enum { LBF_STORE_FP64 = 0, LBF_STORE_FP16 = 1, LBF_STORE_BF16 = 2, LBF_STORE_FP32 = 3,
       LBF_STORE_BFP16 = 4 };

/* Device error word bits (the reference's throw conditions). */
enum {
    LBF_ERR_DENSITY = 1u << 0,    /* non-finite or non-positive density */
    LBF_ERR_COMPONENT = 1u << 1,  /* negative component density (color) */
    LBF_ERR_TAU = 1u << 2,        /* local relaxation time <= 0.5 (color) */
    LBF_ERR_VELOCITY = 1u << 3,   /* non-finite velocity (color) */
    LBF_ERR_OUTPUT = 1u << 4      /* non-finite population met by
                                     lbf_populations_dense_async */
};

/* lbf_step flags: what the LAST step of the call also writes. */
enum {
    LBF_STEP_MACROS = 1u << 0,    /* density(ies) and velocity of that step */
    LBF_STEP_ADJACENT = 1u << 1   /* velocity (and phase indicator) kept as the
                                     "adjacent" history of the next report */
};

/* One geometry label: a line `N "TYPE" "value" "dir" "phase"` of input.prm
 * after FilePrm::IDXVAL parsing (solver/src/file/fileprm.cpp:633-670). */
typedef struct {
    int32_t type;     /* LBF_VD ... LBF_SD; 0 = label not defined */
    int32_t dir;      /* GV: lattice direction of the force; PB/VB: the axial
                         direction 1..2*dims pointing into the domain (the
                         direction of the populations the boundary rebuilds) */
    int32_t phase;    /* VD/GV/PB/VB: fluid phase; HF: the phase the film
                         lets through (color model only) */
    int32_t reserved;
    double value;     /* GV: force magnitude; PB: density; VB: speed along dir
                         (SCSP::zouHeBoundary, scsp.cpp:188-275;
                         ColorFluid::zouHeBoundary, colorfluid.cpp:638-734);
                         SD: contact angle in degrees */
} lbf_label;

typedef struct {
    uint32_t dims;        /* 2 (D2Q9) or 3 (D3Q19) */
    uint32_t nx, ny, nz;  /* nz = 1 in 2D; nx, ny <= 2048, nz <= 1024 */
    uint32_t model;       /* LBF_MODEL_SCSP or LBF_MODEL_COLOR */
    uint32_t collision;   /* LBF_SRT or LBF_MRT */
    uint32_t storage;     /* LBF_STORE_* */
    int32_t device;       /* CUDA device ordinal */
    double tau[2];        /* relaxation times (tau[1]: color phase 1) */
    double rho[2];        /* reference densities */
    double alpha0;        /* color: rest weight of phase 0 */
    double sigma;         /* color: surface tension */
    double beta;          /* color: recoloring parameter */
} lbf_config;

typedef struct lbf_engine lbf_engine;

/* Build an engine: classify links (Simulator::buildIb, simulator.cpp:386-436,
 * and Grid::calcAdjI periodic wrap, solver/inc/grid/grid.h:179-189), pack the
 * fluid nodes and allocate device state.  geometry holds nx*ny*nz labels.
 * Replaces the Simulator/SCSP/ColorFluid constructors
 * (simulator.cpp:17-38, scsp.cpp:22-44, colorfluid.cpp:20-107). */
int lbf_create(const lbf_config *cfg, const lbf_label labels[256],
               const uint8_t *geometry, lbf_engine **out);
void lbf_destroy(lbf_engine *e);

/* The t = 0 stage of Run: initialize, calcMacroVar, bodyForce and the initial
 * collision (scsp.cpp:60-71, 116-134; colorfluid.cpp:123-138, 214-236).  The
 * t = 0 macroscopic fields are kept for lbf_get_macros.  The device error
 * word is cleared first, so an engine can be restarted after an error. */
int lbf_initialize(lbf_engine *e);

/* Warm start (single-phase only): as lbf_initialize, but the t = 0
 * populations are the equilibrium of given fields instead of the fluid at
 * rest.  fields: DEVICE memory on the engine's device, one record of `ld`
 * floats (ld >= 4) per voxel in (z, y, x) order, x fastest: velocity x, y, z
 * (the macroscopic velocity, half force included) and density.  Solid voxels
 * are ignored.  The call first waits for all work queued on the device, so
 * fields written on any stream are complete; the read then happens on the
 * engine's stream and the caller keeps the array alive until lbf_synchronize
 * or any blocking call returns.
 * flags: reserved, 0. */
int lbf_initialize_equilibrium(lbf_engine *e, const float *fields, uint32_t ld, uint32_t flags);

/* Sums over block^3 cubes of the fields of the last step that wrote them
 * (LBF_STEP_MACROS or initialisation), single-phase only.  nx, ny and nz must
 * be multiples of block (nz = 1 in 2-D is taken as one layer); out: host,
 * n = (nx/block)(ny/block)(nz/block) * 5 doubles, cube (bz, by, bx) at
 * ((bz * NBy + by) * NBx + bx) * 5: { sum rho, sum u_x, sum u_y, sum u_z,
 * fluid voxels } over its fluid voxels, summed in voxel order.  out may be
 * host memory or device memory of the engine's device (filled without a
 * host round trip); the call returns when the sums are written. */
int lbf_block_sums(lbf_engine *e, uint32_t block, double *out, size_t n);

/* Adds w_q * drho(voxel) to every population of every fluid node of the
 * current state: a density change at unchanged momentum (single-phase
 * only).  drho: DEVICE memory of the engine's device, one float per voxel in
 * (z, y, x) order; solid voxels are ignored.  Waits for all queued device
 * work first, like lbf_initialize_equilibrium. */
int lbf_add_density(lbf_engine *e, const float *drho);

/* Block-scale Darcy pressure of a periodic porous medium (the solve of the
 * convergence accelerator; LBFlow has no counterpart): mob = DEVICE
 * double[nz][ny][nx], the Darcy mobility (flux per unit driving force) of
 * each block of edge h voxels; g: body force along +x.  Writes the
 * zero-mean pressure over rho0, phi (DEVICE double[nz][ny][nx]), whose block
 * fluxes M_f (g [x face] - grad phi) across block faces (M_f: geometric mean
 * of the two blocks) are conserved.  Multigrid-preconditioned conjugate
 * gradients stopped at relative residual rtol or max_iter iterations
 * (reported in *iterations).  The extents must halve down to a grid of at
 * most 1024 cells.  Runs on `stream`; returns after the result is written. */
int lbf_darcy_pressure(const double *mob, uint32_t nz, uint32_t ny, uint32_t nx, double h, double g,
                       double rtol, uint32_t max_iter, double *phi, uint32_t *iterations, void *stream);

/* nsteps steps of the Run loop body: streaming, bounce-back, calcMacroVar,
 * bodyForce, collision (scsp.cpp:75-104; colorfluid.cpp:142-198).  flags
 * (LBF_STEP_*) apply to the last step of the call. */
int lbf_step(lbf_engine *e, uint32_t nsteps, uint32_t flags);

/* Post-collision populations, dense FP64 [phase][q][voxel], the checkpoint
 * content of saveRst/loadRst (scsp.cpp:277-302; colorfluid.cpp:766-812).
 * Solid voxels are written as 0 and ignored on load.  n = element count. */
int lbf_get_populations(lbf_engine *e, double *host, size_t n);
int lbf_set_populations(lbf_engine *e, const double *host, size_t n);

/* Macroscopic fields of the last step that wrote them (LBF_STEP_MACROS or
 * lbf_initialize), dense: rho0 (density, or rho_0 for color), rho1 (color
 * only; may be NULL), u [3][voxel]; zero on solid voxels as in the VTI output
 * (filevti.cpp:113-172).  Any pointer may be NULL. */
int lbf_get_macros(lbf_engine *e, double *rho0, double *rho1, double *u);

/* Output without a host round trip per voxel: the dense arrays of
 * lbf_get_macros / lbf_get_populations written by the device, enqueued on the
 * engine's stream (the call returns at once; lbf_synchronize or lbf_status
 * waits).  `out` must be memory the device can write: device memory of the
 * engine's device, or page-locked host memory (lbf_host_alloc, or any
 * cudaHostAlloc/cudaHostRegister memory); pageable memory is refused.  Keep
 * it alive and unread until the wait returns.  Device memory is written in
 * place; page-locked host memory is filled by DMA copies from a 256 MiB
 * device staging buffer that the first such call allocates and the engine
 * keeps.
 *
 * lbf_fields_dense_async replaces the field gathering of FileVti::Save
 * (filevti.cpp:113-172): out holds, for N = nx*ny*nz voxels, rho0 [N], then
 * rho1 [N] for the color model, then the velocity [N][dims] with components
 * x, y(, z) interleaved -- the appended arrays of the VTI file in order.
 * n = (1 + color + dims) * N.  Zero on solid voxels.
 *
 * lbf_populations_dense_async replaces the gathering of saveRst
 * (scsp.cpp:277-302; colorfluid.cpp:766-812): out = [phase][q][voxel] FP64,
 * n = phases*Q*N, solid voxels 0, the bytes of the .rst file.  A non-finite
 * value sets LBF_ERR_OUTPUT in the error word (the reference refuses to
 * write such a checkpoint, simulator.cpp:327-333). */
int lbf_fields_dense_async(lbf_engine *e, double *out, size_t n);

/* Checkpoint compatibility: from now on also carry the populations of solid
 * voxels, streamed exactly as Simulator::streaming moves every voxel
 * (simulator.cpp:73-101; solid voxels are never collided, and bounce-back,
 * simulator.cpp:103-111, keeps their values out of the fluid), so that
 * lbf_get_populations / lbf_populations_dense_async reproduce saveRst
 * (scsp.cpp:277-302; colorfluid.cpp:766-812) at solid voxels too, and
 * lbf_set_populations loads them.  Call before lbf_initialize or
 * lbf_set_populations; FP64 storage only.  Costs one extra pass over all
 * voxels per step and 2 * phases * Q * 8 bytes per solid voxel.  Without it
 * solid entries are written as 0 (they never influence the flow). */
int lbf_keep_solid_populations(lbf_engine *e);
int lbf_populations_dense_async(lbf_engine *e, double *out, size_t n);

/* Page-locked host memory the device can write (cudaHostAlloc, portable and
 * mapped), for the two calls above. */
int lbf_host_alloc(size_t bytes, void **out);
void lbf_host_free(void *p);

/* Device reductions of Simulator::updateConvergence (simulator.cpp:248-325).
 * first != 0 only records the current velocity (and phase indicator) as the
 * previous report.  Otherwise out = { sum (u-u_prev)^2, sum u^2,
 * sum (u-u_adj)^2, max |ind-ind_prev|, max |ind-ind_adj|, 0 } over all voxels
 * and components, then the current fields become the previous report. */
int lbf_convergence(lbf_engine *e, int first, double out[6]);

/* Slice sums of SCSP::report / ColorFluid::report (scsp.cpp:325-341;
 * colorfluid.cpp:841-867) along axis (0 = x, 1 = y, 2 = z) between slices lo
 * and hi: out = { sum u_axis over lo..hi, sum rho0 over lo..hi,
 * sum rho1 over lo..hi, sum rho0 at lo, sum rho1 at lo, sum rho0 at hi,
 * sum rho1 at hi, fluid count at lo, fluid count at hi, fluid count lo..hi }.
 * Single phase: rho1 terms are 0. */
int lbf_report_sums(lbf_engine *e, uint32_t axis, uint32_t lo, uint32_t hi, double out[10]);

/* Pore measures of scripts/porous_media.py:20-44 on the last macros, summed
 * over fluid voxels: out = { sum u_x, sum u_y, sum u_z, sum phi0 u_x,
 * sum phi0 u_y, sum phi0 u_z, sum rho0, sum rho1, sum phi0 } with
 * phi0 = rho0/(rho0+rho1) (1 for single phase).  Divide by nx*ny*nz for the
 * Darcy velocity; permeability K = nu <u_x> / g_x. */
int lbf_flux_sums(lbf_engine *e, double out[9]);

/* Link classification as the kernels use it: per voxel, bit (q-1) set when
 * the voxel is fluid and its neighbour x + e_q is a BB/SD solid
 * (simulator.cpp:405-415).  n = nx*ny*nz. */
int lbf_link_mask(lbf_engine *e, uint32_t *host, size_t n);

/* Waits for queued work and returns the device error word (LBF_ERR_* bits). */
int lbf_status(lbf_engine *e, uint32_t *bits);

/* Number of fluid nodes (the reference's fluid_nodes, simulator.cpp:47-56). */
uint64_t lbf_fluid_nodes(const lbf_engine *e);
/* Device bytes held by the engine. */
uint64_t lbf_device_bytes(const lbf_engine *e);
/* Message of the last failed call on e (or of lbf_create when e is NULL). */
const char *lbf_last_error(const lbf_engine *e);
/* Wait for all queued work of the engine. */
int lbf_synchronize(lbf_engine *e);
/* The CUDA stream (a cudaStream_t) all of the engine's work is queued on,
 * for callers that time or order work against it. */
void *lbf_stream(const lbf_engine *e);

/* ---- Batched geometries ----------------------------------------------------
 * Many independent single-phase D3Q19 geometries of uneven size advanced
 * together: one launch per step walks a packed list of fluid-node tiles of all
 * active geometries (all-solid regions produce no tiles), each tile using its
 * geometry's size and relaxation time; plain steps are replayed from a CUDA
 * graph; per-geometry reductions let each geometry converge and retire on its
 * own.  No counterpart in the reference, which runs one geometry per process
 * (scripts/benchmarks.py:221-224 farms cases out to a thread pool). */
typedef struct {
    uint32_t nx, ny, nz;      /* voxels */
    const uint8_t *labels;    /* nx*ny*nz labels, x fastest (copied) */
    double tau;               /* relaxation time of this geometry */
} lbf_batch_geometry;

typedef struct lbf_batch lbf_batch;

/* labels: the shared label table; collision: LBF_SRT or LBF_MRT; storage:
 * LBF_STORE_FP64, _FP32 or _FP16; rho0: reference density. */
int lbf_batch_create(const lbf_batch_geometry *geoms, uint32_t count, const lbf_label labels[256],
                     uint32_t collision, uint32_t storage, int32_t device, double rho0, lbf_batch **out);
void lbf_batch_destroy(lbf_batch *b);
/* t = 0 stage for every geometry (as lbf_initialize). */
int lbf_batch_initialize(lbf_batch *b);
/* nsteps steps of every active geometry; flags as for lbf_step. */
int lbf_batch_step(lbf_batch *b, uint32_t nsteps, uint32_t flags);
/* Per geometry, the lbf_convergence sums: out[count][6]. */
int lbf_batch_convergence(lbf_batch *b, int first, double *out);
/* Per geometry, the lbf_flux_sums: out[count][9]. */
int lbf_batch_flux_sums(lbf_batch *b, double *out);
/* active[count]: 0 retires a geometry from the step schedule. */
int lbf_batch_set_active(lbf_batch *b, const uint8_t *active);
/* Times tile size and grid shape candidates over `steps` steps each and keeps
 * the fastest; the populations are restored afterwards.  out = { threads,
 * tile nodes, 128-thread blocks per SM, ms per step }. */
int lbf_batch_autotune(lbf_batch *b, uint32_t steps, double out[4]);
/* Dense fields of one geometry from the last step that wrote macros. */
int lbf_batch_get_macros(lbf_batch *b, uint32_t geometry, double *rho, double *u);
int lbf_batch_status(lbf_batch *b, uint32_t *bits);
int lbf_batch_synchronize(lbf_batch *b);
/* Fluid nodes of one geometry, or of all with geometry = UINT32_MAX. */
uint64_t lbf_batch_fluid_nodes(const lbf_batch *b, uint32_t geometry);
uint32_t lbf_batch_active_tiles(const lbf_batch *b);
void *lbf_batch_stream(const lbf_batch *b);
const char *lbf_batch_last_error(const lbf_batch *b);

/* Pore-measure sums of lbf_flux_sums over arrays the caller already holds on
 * the device, for callers that cannot allocate device memory (a frozen or
 * exhausted memory pool, an allocator that owns the whole device).  Nothing
 * is allocated: the per-tile partial sums live in a fixed scratch array
 * compiled into the library (1,179,648 bytes), which comes into a device's
 * memory with the library's module -- under CUDA's default lazy module
 * loading at the first call on that device -- and stays until exit.  No
 * counterpart in the reference.
 *   u:    [3][stride] x, y, z velocities;  rho0, rho1: [stride] densities
 *         (rho1 NULL for single phase);  n <= 16,777,216 nodes, else
 *         LBF_EINVAL;  out: 9 doubles in device memory, same order as
 *         lbf_flux_sums;  stream: a cudaStream_t (NULL = default stream).
 * The first call on a device looks up the scratch address (and loads the
 * module with its scratch): make it, n = 0 is enough, while device memory is
 * still free and before any stream capture.  Calls share the scratch: calls whose GPU work
 * overlaps race, so serialise them.  Errors: lbf_last_error(NULL). */
int lbf_flux_sums_noalloc(const double *u, const double *rho0, const double *rho1,
                          uint32_t n, uint32_t stride, double *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* LBFLOW_H */
