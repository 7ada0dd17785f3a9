/*
 * sphk.h -- C ABI of libsphk, the B200 (sm_100a) DEM step of sphere.
 *
 * The reference has no in-process interface for this path: its DEM class
 * (src/sphere.h:12-322) owns the state and drives the GPU from
 * DEM::startTime() (src/device.cu:576-1299), and Python reaches it through
 * binary files and a subprocess (python/sphere.py:1629-1655).  Each entry
 * point below replaces one step of that class, so the DEM class
 * (sphere_b200/csrc/host/sphere.cpp) and any FFI can sit on top:
 *
 *   sph_create       DEM::initializeGPU + transferToConstantDeviceMemory +
 *                    allocateGlobalDeviceMemory   (src/device.cu:34-84,201-324);
 *                    also captures the step's CUDA graphs
 *   sph_upload       DEM::transferToGlobalDeviceMemory (src/device.cu:394-488)
 *   sph_step         n iterations of the time loop body (src/device.cu:731-1109)
 *   sph_sync         the checkForCudaErrors after each kernel (src/utility.cu:9-28)
 *   sph_download     DEM::transferFromGlobalDeviceMemory (src/device.cu:490-572)
 *   sph_get_contacts the CONTACTINFO dump of slots (src/device.cu:1148-1176)
 *   sph_get_cells    the sorted arrays of the last step (src/device.cu:747-800)
 *   sph_destroy      DEM::freeGlobalDeviceMemory (src/device.cu:326-391)
 *   sph_darcy_init   DEM::initDarcy (src/darcy.cpp:760-798)
 *   sph_darcy_upload, sph_darcy_download
 *                    DEM::transferDarcy{To,From}GlobalDeviceMemory (src/darcy.cuh:60-121)
 *   sph_render       DEM::render (src/raytracer.cuh:303-553)
 *
 * Conventions: plain C types only; every entry point returns an int status,
 * SPH_OK (0) or a negative SPH_ERR_* code; the message of the last failure
 * is available from sph_last_error().  Host arrays use the reference's host
 * layout: "4 doubles per particle" rows (Float4, src/datatypes.h:17-33),
 * particle order = the caller's particle index.  A context is bound to one
 * device and is not thread safe; distinct contexts are independent.
 */
#ifndef SPHK_H_
#define SPHK_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPHK_VERSION 3
#define SPHK_NC 32        /* contact slots per particle (src/constants.h:24) */
#define SPHK_MAXWALLS 6   /* src/constants.h:11 */

#define SPH_OK 0
#define SPH_ERR_CUDA (-1)         /* a CUDA call failed (see sph_last_error) */
#define SPH_ERR_NC_OVERFLOW (-2)  /* a particle found more than SPHK_NC contacts */
#define SPH_ERR_OUT_OF_GRID (-3)  /* a particle left the cell grid */
#define SPH_ERR_TIMEOUT (-4)      /* a bounded device wait gave up */
#define SPH_ERR_BAD_INPUT (-5)    /* invalid argument or configuration */
#define SPH_ERR_BOND_ALIAS (-6)   /* a broken bond's marker (nb0 < np) aliases a particle */
#define SPH_ERR_NOMEM (-7)        /* device allocation failed */
#define SPH_ERR_TOO_LARGE (-8)    /* input exceeds the fixed scratch of sph_cell_list_noalloc */
#define SPH_ERR_UNSTABLE (-9)     /* sph_darcy_init: the explicit Darcy step would be unstable */

typedef struct sph_ctx sph_ctx;

/* Static configuration: the Grid, Params and Walls fields of the input file
 * (src/datatypes.h:43-101) plus the time step.  Mirrors readbin's fields. */
typedef struct sph_config {
    uint32_t np, nw, nb0, contactmodel;
    int32_t periodic;
    uint32_t num[3];
    double origo[3], L[3];
    double dt;
    double g[3], k_n, k_t, k_r, gamma_n, gamma_t, gamma_r, mu_s, mu_d, mu_r;
    double gamma_wn, gamma_wt, mu_ws, mu_wd, rho, kappa, db, V_b;
    double lambda_bar, sigma_b, tau_b, devs_A, devs_f;
    int32_t wmode[SPHK_MAXWALLS];
    int32_t device;              /* CUDA device ordinal */
} sph_config;

/* Host-side state, reference layout.  On upload, NULL pointers take the
 * reference's initial values: vel0 := vel and angvel0 := angvel
 * (src/device.cu:413-424), acc/angacc := 0, contacts := empty (np) with zero
 * history, walls_vel0 := walls_mvfd[].y (src/device.cu:461-464). */
typedef struct sph_host_state {
    double *x;        /* np*4: x, y, z, radius */
    double *xysum;    /* np*2 */
    double *vel;      /* np*4: vx, vy, vz, fixvel */
    double *vel0;     /* np*4 or NULL */
    double *acc;      /* np*4 or NULL (w lane not kept) */
    double *force;    /* np*4 */
    double *angpos;   /* np*4 */
    double *angvel;   /* np*4 */
    double *angvel0;  /* np*4 or NULL */
    double *angacc;   /* np*4 or NULL (w lane not kept) */
    double *torque;   /* np*4 */
    double *es_dot, *es, *ev_dot, *ev, *p;   /* np each */
    uint32_t *contacts;   /* np*SPHK_NC or NULL; value np marks an empty slot */
    double *distmod;      /* np*SPHK_NC*4 or NULL: periodic shift (0 or +-L) + radius */
    double *delta_t;      /* np*SPHK_NC*4 or NULL: tangential spring history */
    uint32_t *bonds;      /* nb0*2 */
    double *bonds_delta;  /* nb0*4: tangential xyz, normal w */
    double *bonds_omega;  /* nb0*4 */
    double *walls_nx;     /* nw*4: normal xyz, position w */
    double *walls_mvfd;   /* nw*4: mass, velocity, force, deviatoric stress */
    double *walls_vel0;   /* nw or NULL */
    double t_current;     /* simulation time */
} sph_host_state;

/* Counters of the current state. */
typedef struct sph_stats {
    uint64_t active_contacts;   /* occupied slots over all particles (directed) */
    uint64_t steps;             /* steps taken since upload */
    uint64_t relayouts;         /* storage re-orderings performed */
    uint64_t device_bytes;      /* device memory held by the context */
    uint64_t cell_rebuilds;     /* steps whose cell list was rebuilt (a particle changed cell) */
} sph_stats;

/* Options for sph_set_option. */
#define SPH_OPT_RELAYOUT_EVERY 1  /* re-sort storage every n steps (0: at upload only) */
#define SPH_OPT_GRAPH_STEPS 2     /* steps captured per CUDA graph (1..64, default 8) */
#define SPH_OPT_BLOCK_SHAPES 5    /* 0 (default) or 1: the block shapes of the contact
                                     search and the contact forces; results do not depend
                                     on it, only their cost does */
#define SPH_OPT_VERLET_SKIN 4     /* Verlet skin in thousandths of the largest radius
                                     (default 100; 0 sweeps the 27-cell stencil every
                                     step); set before sph_upload.  Results do not depend
                                     on it, only the cost of contact detection does. */
#define SPH_OPT_PROFILE 3         /* 1: launch kernels one by one with CUDA events around
                                     each phase (the reference's PROFILING switch,
                                     src/debug.h:7, src/device.cu:86-102); 0: graphs */
#define SPH_OPT_TOPO_SPAN 6       /* particles whose list decision each thread of the contact
                                     search makes at once: 0 (default) chooses from the
                                     particle count (4 at 1M on a B200, 1 below ~300k), or
                                     1, 2, 4; results do not depend on it, only its cost */

/* Phases timed in profile mode. */
#define SPH_PHASE_CELLS 0   /* cell list rebuild (hash histogram, scan, scatter, sort) */
#define SPH_PHASE_BONDS 1   /* per-bond forces */
#define SPH_PHASE_TOPO 2    /* contact detection into the slots */
#define SPH_PHASE_FORCE 3   /* slot sums, wall and bond forces + integration */
#define SPH_PHASE_WALLS 4   /* wall force reduction + wall integration */
#define SPH_PHASE_DARCY 5   /* Darcy flow (zero without sph_darcy_upload) */
#define SPH_PHASE_CONTACT 6 /* force laws of the contact slots (models 2 and 3) */
#define SPH_NPHASES 7

int sph_version(void);
int sph_create(const sph_config *cfg, sph_ctx **out);
/* Batched ensemble: ninst independent scenes stepped together by one
 * context, every kernel launched once over all of them (an addition for the
 * ensemble workload; the reference runs one scene per process).  Each scene
 * keeps its own grid, parameters and time step; results for each scene are
 * those of a context created for it alone, bit for bit.  Host arrays passed
 * to sph_upload / sph_download hold the scenes end to end: rows of scene 0,
 * then of scene 1, ...; contact partners are indices within the particle's
 * own scene (its np marks an empty slot).  Scenes must use contact model 2,
 * no dynamic walls (nw = 0) and no bonds (nb0 = 0), on one device.  A batched
 * context takes every other call of this header; sph_get_cells reports the
 * context-wide cell list (scene i's cells follow scene i-1's; perm holds
 * context-wide particle indices), and sph_download's t_current is scene 0's. */
int sph_batch_create(const sph_config *cfgs, uint32_t ninst, sph_ctx **out);
int sph_set_option(sph_ctx *ctx, int option, int64_t value);
int sph_upload(sph_ctx *ctx, const sph_host_state *st);
/* Enqueue nsteps time steps on `stream` (a cudaStream_t, NULL: the context's
 * own stream).  Asynchronous: device errors surface at sph_sync. */
int sph_step(sph_ctx *ctx, uint64_t nsteps, void *stream);
/* Wait for all work and report the first device-side error (sticky). */
int sph_sync(sph_ctx *ctx);
int sph_download(sph_ctx *ctx, sph_host_state *st);
/* Contact slots in the reference layout (np*SPHK_NC; distmod/delta_t
 * np*SPHK_NC*4).  Any pointer may be NULL.  distmod of empty slots is 0. */
int sph_get_contacts(sph_ctx *ctx, uint32_t *contacts, double *distmod, double *delta_t);
/* The cell list used by the most recent step: sorted cell ids and the
 * sorted->particle permutation (np each), cellStart/cellEnd (ncells each;
 * cellStart = 0xffffffff for empty cells, cellEnd defined for occupied ones). */
int sph_get_cells(sph_ctx *ctx, uint32_t *cell_sorted, uint32_t *perm, uint32_t *cell_start,
                  uint32_t *cell_end);
/* Wall-0 force of every particle in the most recent step (np doubles). */
int sph_get_wall_forces(sph_ctx *ctx, double *wall0_force);
int sph_get_stats(sph_ctx *ctx, sph_stats *out);
/* Accumulated milliseconds per phase (SPH_NPHASES doubles) and the number of
 * profiled steps since the last reset; reset != 0 clears the counters. */
int sph_get_profile(sph_ctx *ctx, double *ms, uint64_t *steps, int reset);
/* Re-sort particle storage into the current cell order (locality only;
 * results are unchanged). */
int sph_relayout(sph_ctx *ctx);
const char *sph_last_error(const sph_ctx *ctx);
int sph_destroy(sph_ctx *ctx);

/* ---- Darcy flow -------------------------------------------------------------
 * The reference's fluid coupling for darcy == 1 and nu > 0 (src/darcy.cuh,
 * src/darcy.cpp; DEM's darcyflow argument, src/sphere.h:254): each step,
 * between the contact forces and the integration, the porosity of every
 * cell from the step's start positions, the cell conductivities and an
 * explicit step of the pore pressure (src/device.cu:913-1021).  The flow
 * does not act on the particles.
 *
 * The fluid grid is the cell grid with one ghost node on every side:
 * (num[0]+2)(num[1]+2)(num[2]+2) nodes, x fastest; node (x, y, z), with
 * -1 <= x <= num[0] and so on, at (x+1) + (num[0]+2)(y+1) +
 * (num[0]+2)(num[1]+2)(z+1).  These are the reference's host arrays of
 * DEM::d (src/darcy.cpp:17-38): one double per node, three for V, dH, T. */
typedef struct sph_darcy_state {
    double *H, *H_new;   /* hydraulic pressure: current and spare buffer */
    double *V;           /* 3 per node: pore velocity */
    double *dH;          /* 3 per node: pressure gradient */
    double *K;           /* hydraulic conductivity */
    double *T;           /* 3 per node: transmissivity */
    double *Ss, *W;      /* specific storativity, recharge */
    double *phi, *dphi;  /* porosity and its change in the last step */
} sph_darcy_state;

/* DEM::initDarcy (src/darcy.cpp:760-798), on the host: Ss := 1 and W := 0
 * on every node; the porosity of every cell from the particles whose centres
 * it holds (x: np*4, the reference's host rows) into phi; K and T from it;
 * dphi := 0.  H, H_new, V and dH are left as they are (the input file gives
 * V and H; the reference leaves the rest unset, read here as zero by
 * convention of the caller).  *stability (may be NULL) receives the
 * criterion of checkDarcyTimestep (src/darcy.cpp:733-758); above 0.5 the
 * call returns SPH_ERR_UNSTABLE, where the reference exits. */
int sph_darcy_init(const sph_config *cfg, double nu, const double *x, sph_darcy_state *st,
                   double *stability);
/* transferDarcyToGlobalDeviceMemory (src/darcy.cuh:60-92) plus the
 * Kozeny-Carman factor of DEM::startTime (src/device.cu:673-678, from the
 * mean radius of the uploaded particles): after sph_upload, switches the
 * context to run the Darcy flow in every step, with dynamic viscosity nu.
 * The first step after this call leaves dphi zero (src/darcy.cuh:463-466).
 * Not for batched or differentiable contexts.  Every array is required. */
int sph_darcy_upload(sph_ctx *ctx, double nu, const sph_darcy_state *st);
/* transferDarcyFromGlobalDeviceMemory (src/darcy.cuh:95-121). */
int sph_darcy_download(sph_ctx *ctx, sph_darcy_state *st);

/* ---- Ray tracer -------------------------------------------------------------
 * DEM::render (src/raytracer.cuh:303-553, the kernels at :14-263): one image
 * of the context's current state, from the reference's camera (eye at
 * (2.3, -5, 1.3) x L, looking at half the largest coordinates, an image
 * plane 1.35 L[0] wide), white background, Lambertian shading, plain or
 * through the blue-white-red colour map.  The pixels are those of the
 * reference's brute-force search, bit for bit, with IEEE single-precision
 * arithmetic (the reference's GPU build used fast-math approximations). */
typedef struct sph_render_opts {
    int32_t method;        /* 0 plain; colour map of 1 pressure, 2 |velocity|,
                              3 |angular velocity|, 4 x displacement, 5 |rotation| */
    float maxval;          /* value at the top of the colour map */
    float lower_cutoff;    /* > 0 (methods 1-5): draw only spheres whose value exceeds
                              it and whose fixvel is zero */
    uint32_t width, height;   /* pixels, width * height < 2^24 (else SPH_ERR_TOO_LARGE) */
} sph_render_opts;
/* rgba: width * height * 4 bytes, rows top to bottom as the reference's
 * image buffer (pixel m = row * width + column); alpha is 0.  Not for
 * batched contexts. */
int sph_render(sph_ctx *ctx, const sph_render_opts *opts, uint8_t *rgba);

/* ---- Differentiable step ----------------------------------------------------
 * No counterpart in the reference: gradients of a run with respect to the
 * contact parameters, for calibration.  sph_diff_begin switches an uploaded
 * single-scene context (contact model 2, nw = 0, nb0 = 0) to the
 * differentiable step: contact model 2 with exact FP64 vector lengths (the
 * reference narrows them to float) and per-particle friction mu (np values,
 * caller order; NULL: every particle gets the configuration's mu_s), a
 * contact using the mean of its two particles' values for mu_s and mu_d.
 * Energy rates and pressure are not computed in this mode.  Every
 * sph_step after it keeps a checkpoint of the state every checkpoint_every
 * steps (about 1.4 KB per particle each) and the context holds a tape of
 * checkpoint_every steps (about 1.3 KB per particle per step); storage is
 * not re-ordered while the mode is on.
 * sph_diff_backward runs the adjoint of every step taken since
 * sph_diff_begin, seeded with x_bar and v_bar (np*3 each, caller order, the
 * derivatives of a loss with respect to the current positions and
 * velocities; NULL means zero): each checkpoint segment is stepped again
 * with the tape recorded, then reversed step by step.  It returns the
 * gradient with respect to k_n, k_t and gamma_n (grad_params[3]), per-
 * particle friction (grad_mu[np]) and the starting positions and velocities
 * (x0_bar, v0_bar, np*3); any output may be NULL.  The context's state after
 * the call is the state before it.  sph_diff_end returns to the plain step
 * and frees the checkpoints and tape. */
int sph_diff_begin(sph_ctx *ctx, const double *mu, uint32_t checkpoint_every);
int sph_diff_backward(sph_ctx *ctx, const double *x_bar, const double *v_bar, double *grad_params,
                      double *grad_mu, double *x0_bar, double *v0_bar);
int sph_diff_end(sph_ctx *ctx);

/* ---- Cell list without device allocation ----------------------------------
 * No counterpart in the reference: an addition for callers that cannot
 * allocate device memory -- a plugin whose host owns the device memory pool
 * through its own allocator and forbids cudaMalloc, or a latency-critical
 * loop that must not pay the device-wide synchronisation of cudaMalloc and
 * cudaFree.  Computes, for device-resident positions x_dev (np*4 doubles,
 * x, y, z, radius, the caller's particle order), the same cell list as
 * sph_get_cells reports for a context holding those positions: sorted cell
 * ids and the sorted -> particle permutation (np each), cellStart (0xffffffff
 * for empty cells) and cellEnd (0 for empty cells), ncells each.  Every
 * output is a device pointer supplied by the caller; the work is enqueued on
 * `stream` (a cudaStream_t; NULL is the default stream).  Only cfg->np,
 * num, origo, L and device are read.
 * A position outside the grid or not finite goes to one bucket after the
 * last cell (0xffffffff in cell_sorted), members of every bucket in particle
 * order; the work is linear in np however the particles spread over cells.
 * Limits: np <= SPHK_NOALLOC_MAX_PARTICLES and num[0]*num[1]*num[2] <=
 * SPHK_NOALLOC_MAX_CELLS, otherwise SPH_ERR_TOO_LARGE and nothing is
 * launched.  It calls no cudaMalloc, cudaFree or allocating library routine:
 * its scratch is one fixed array of about 9 MB inside the library, held by
 * every GPU that loads the library until the process exits, and the
 * caller's cell_sorted and perm serve as scratch until the call's last
 * kernel writes them.  The first call on a device looks up that array's
 * device address (cudaGetSymbolAddress); make that first call before any
 * stream capture.  All calls share the array, so calls that overlap on the
 * GPU race and give wrong results.  The caller's current device is the same
 * after the call; a launch error pending from the caller's own earlier work
 * is reported as SPH_ERR_CUDA (and left pending). */
#define SPHK_NOALLOC_MAX_PARTICLES 1048576u
#define SPHK_NOALLOC_MAX_CELLS 524288u
int sph_cell_list_noalloc(const sph_config *cfg, const double *x_dev, uint32_t *cell_sorted,
                          uint32_t *perm, uint32_t *cell_start, uint32_t *cell_end, void *stream);

#ifdef __cplusplus
}
#endif

#endif
