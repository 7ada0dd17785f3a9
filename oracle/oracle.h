/*
 * oracle/oracle.h -- C interface shared by the two CPU oracles of the sphere
 * DEM step.
 *
 * TEST INFRASTRUCTURE ONLY.  Two libraries export this interface:
 *   oracle/liborc.so      -- dem_oracle.c, a plain-C restatement of the
 *                            reference algorithm;
 *   oracle/_ref/libref.so -- the reference's own kernel bodies
 *                            (src/sorting.cuh, src/contactsearch.cuh,
 *                            src/contactmodels.cuh, src/cohesion.cuh,
 *                            src/integration.cuh) compiled as host C++ under a
 *                            shim, driven in the order of src/device.cu:731-1109.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * them, as checkers.  The product path never links or calls either.
 *
 * All arrays use the reference's host layout (array-of-structs, "Float4" =
 * four doubles): Kinematics/Energies/Walls in src/datatypes.h:17-105.
 */
#ifndef SPHERE_ORACLE_H_
#define SPHERE_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_NC 32       /* contact slots per particle, src/constants.h:24 */
#define ORC_MAXWALLS 6  /* src/constants.h:11 */

/* status codes (bit flags, OR-ed over the run) */
#define ORC_OK 0
#define ORC_ERR_NC_OVERFLOW 1   /* a contact would be written past slot NC-1 */
#define ORC_ERR_OUT_OF_GRID 2   /* a cell index fell outside [0, ncells) */
#define ORC_ERR_BAD_INPUT 4

typedef struct orc_scene {
    /* sizes and switches */
    uint32_t np, nw, nb0, contactmodel;
    int32_t periodic;
    uint32_t num[3];
    double origo[3], L[3];
    double dt, t_current;
    /* Params (src/datatypes.h:74-101) */
    double g[3], k_n, k_t, k_r, gamma_n, gamma_t, gamma_r, mu_s, mu_d, mu_r;
    double gamma_wn, gamma_wt, mu_ws, mu_wd, rho, kappa, db, V_b;
    double lambda_bar, sigma_b, tau_b, devs_A, devs_f;
    int32_t wmode[ORC_MAXWALLS];
    /* per particle: 4 doubles each (xysum: 2) */
    double *x, *vel, *vel0, *acc, *force, *angpos, *angvel, *angvel0,
        *angacc, *torque, *xysum;
    double *es_dot, *es, *ev_dot, *ev, *p;
    /* contact bookkeeping: np*NC slots (distmod/delta_t 4 doubles each) */
    uint32_t *contacts;
    double *distmod, *delta_t;
    /* bonds: nb0 pairs, 4 doubles of history each */
    uint32_t *bonds;
    double *bonds_delta, *bonds_omega;
    /* walls: nw entries */
    double *walls_nx, *walls_mvfd, *walls_vel0;
    /* cell list of the most recent step (outputs): sorted cell ids and the
     * sorted-to-original permutation (np each); cell start/end (ncells each) */
    uint32_t *cell_sorted, *perm, *cell_start, *cell_end;
    /* wall-0 force of every particle in the most recent step (np) */
    double *wall0_force;
    /* Darcy flow (src/darcy.cuh:169-779, launched at src/device.cu:913-1021
     * between bondsLinear and integrate), run when darcy == 1 and nu > 0.
     * The fluid grid is the cell grid with one ghost node on every side:
     * (num[0]+2)(num[1]+2)(num[2]+2) nodes, x fastest, node (x,y,z) at
     * (x+1) + (num[0]+2)(y+1) + (num[0]+2)(num[1]+2)(z+1).  The pressure
     * has two buffers, H = d_Hbuf[d_hsel] and H_new = d_Hbuf[1 - d_hsel];
     * each step swaps them (d_hsel ^= 1), as the reference swaps pointers. */
    double nu;
    int32_t darcy;
    uint32_t iteration;     /* steps since the run started: at 0 the porosity change is zero */
    double d_factor;        /* grain-size factor of the Kozeny-Carman relation */
    double *d_Hbuf[2];
    uint32_t d_hsel;
    double *d_V, *d_dH, *d_T;                 /* 3 doubles per node */
    double *d_K, *d_Ss, *d_W, *d_phi, *d_dphi;
} orc_scene;

/* ---- ray tracer (src/raytracer.cuh:14-553, DEM::render) ------------------ */
typedef struct orc_render {
    uint32_t np;
    const double *x;        /* np*4: positions and radii, particle order */
    const double *vel;      /* np*4: the fourth lane is fixvel */
    const double *values;   /* np colour-map values (methods 1-5), else NULL */
    double L[3];            /* grid.L */
    int32_t method;         /* 0 plain, 1 pressure, 2 |v|, 3 |omega|, 4 x displacement, 5 |rotation| */
    float maxval, lower_cutoff;
    uint32_t width, height;
} orc_render;

/* the camera that DEM::render and DEM::cameraInit set up
 * (src/raytracer.cuh:269-300, 351-367), the raytracer's __constant__ values */
typedef struct orc_camera {
    float u[3], v[3], w[3], eye[3], light[3];
    float imgplane[4];
    float d;
} orc_camera;

/* Fill *cam for the scene and image size of *r (plain-C restatement only). */
void orc_render_camera(const orc_render *r, orc_camera *cam);
/* DEM::render's colour-map array for `method` (plain-C restatement only). */
void orc_render_values(int method, uint32_t np, const double *vel, const double *angvel,
                       const double *angpos, const double *xysum, const double *p, double *out);
/* Render one image into rgba (width*height*4 bytes; alpha 0).  Both
 * oracles provide it: the restatement and the reference kernels. */
int orc_render_image(const orc_render *r, const orc_camera *cam, uint8_t *rgba, int nthreads);
/* The same for the pixel rows [row0, row0 + nrows) only (the rest of rgba
 * is left alone): a bounded sample for timing. */
int orc_render_rows(const orc_render *r, const orc_camera *cam, uint8_t *rgba, uint32_t row0,
                    uint32_t nrows, int nthreads);

/* Advance the scene by nsteps time steps.  nthreads <= 0 uses the OpenMP
 * default.  Returns the OR of the ORC_ERR_* flags raised (0 when clean). */
int orc_step(orc_scene *s, uint64_t nsteps, int nthreads);

/* Which oracle this is: 1 = plain-C restatement, 2 = reference kernels. */
int orc_kind(void);

/* Number of OpenMP threads a parallel region gets with nthreads as above. */
int orc_threads(int nthreads);
/* FP32 transcendentals of the force laws (expf, powf): 0 (default) evaluates
 * each as the float nearest to the double-precision result, as the CUDA path
 * does; 1 calls the C library's expf/powf, as the reference's host build
 * does.  Not provided by the reference harness (oracle/_ref), which always
 * calls the C library. */
void orc_set_libm_float_math(int on);

#ifdef __cplusplus
}
#endif

#endif
