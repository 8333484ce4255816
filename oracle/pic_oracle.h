/* CPU restatement of Mandor's PIC time step (TEST INFRASTRUCTURE ONLY).
 *
 * This is the oracle the CUDA path is checked against.  It restates, in
 * plain C on one global mesh with ghost layers, what the reference core.out
 * does per step (core/main.c:353-478): Yee H half-steps, E step, field
 * boundary conditions, the relativistic Boris push with CIC gather and the
 * charge-conserving current deposition, particle and current boundary
 * conditions, and the energy diagnostics.  It is pinned against the
 * reference binaries built from source (oracle/Makefile) by the tests.
 *
 * Only tests/, the package smoke check and the bench's CPU-baseline leg may
 * load it.  It is never part of the product path.
 */
#ifndef PIC_ORACLE_H
#define PIC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Marker record of the reference with the tracer id (type_marker.h:12-25). */
typedef struct {
   double x, y, z;
   double vx, vy, vz;
   float  rho;
   float  qDivM;
   int    id;
   int    pad_;
} po_marker_t;

/* Boundary condition codes (misc_parameters.h:38-42). */
enum { PO_BC_PERIODIC = 0, PO_BC_MIRROR = 1, PO_BC_OPEN = 2 };

/* Analytic laser: paraxial Gaussian beam, Ey-polarised, moving along +x,
 * with a sin^2 field envelope, injected as a one-sided soft source at the
 * x-planes i = plane (H) and i = plane - 1 (E). */
typedef struct {
   double a0;          /* normalised amplitude; E amplitude = 2*pi*a0      */
   double waist;       /* w0, in wavelengths                               */
   double x_focus;     /* focal plane position                             */
   double duration;    /* sin^2 envelope length (field), in periods        */
   double t_start;     /* time the envelope front crosses the source plane */
   double phase;       /* carrier phase offset                             */
   int    plane;       /* H plane index (E plane is plane - 1)             */
   int    margin;      /* transverse nodes kept free next to each wall     */
} po_laser_t;

typedef struct po_run po_run_t;

po_run_t *po_create (const int n[3], const double h[3], double tau,
                     const int bc_min[3], const int bc_max[3], double time);
void      po_destroy (po_run_t *r);

/* Fields over the checkpoint region [0,n] per axis, reference AoS layout
 * (vec3D_t, k fastest, i slowest). */
void po_set_fields (po_run_t *r, const double *E, const double *H);
void po_get_fields (const po_run_t *r, double *E, double *H);
void po_get_current (const po_run_t *r, double *J);   /* region [-2,n+2] */

void po_set_markers (po_run_t *r, const po_marker_t *m, long n);
long po_marker_count (const po_run_t *r);
void po_get_markers (const po_run_t *r, po_marker_t *m);

void po_set_laser (po_run_t *r, const po_laser_t *l);

/* Hard gauss-spot source: the fields of .gaussSpot.cfg in its order
 * (core/em_gaussSpot.c:46-56), frequency in omega_0. */
typedef struct {
   double ampl, frequency, x, y, z, width, duration, front_offset, t_plateau;
   int    ey, ez;
} po_gauss_spot_t;
void po_set_gauss_spot (po_run_t *r, const po_gauss_spot_t *s);

/* TF/SF interface (core/em_TFSF.c).  24 faces: E faces f = 0..11 in the
 * reference's order (Ey_xMin, Ez_xMin, Ey_xMax, Ez_xMax, Ez_yMin, Ex_yMin,
 * ..., Ey_zMax), then the H faces (Hz_xMin, Hy_xMin, ...).  A frame holds
 * the recorded values of the 12 E faces then of the 12 H faces, each over
 * its face region with the first tangential axis ep = (a+1)%3 slowest and
 * eq = (a+2)%3 fastest, as the recording files store them (values already
 * times the face's source factor). */
enum { PO_TFSF_PLAY = 0, PO_TFSF_REC = 1, PO_TFSF_BACK = 2 };
typedef struct {
   int lo[3], hi[3];       /* interface bounding box (TFSF.cfg)               */
   int mode;               /* PO_TFSF_*                                        */
   int open[2][3];         /* play: faces removed, [min/max][axis]            */
   int frames;             /* play: frames recorded (lastFrameTime.bin)       */
} po_tfsf_t;
/* Play: frames[frames x frame size]; record: frames NULL.  Returns 0, or -1
 * when a played face is closer than 5 cells to a wall. */
int  po_set_tfsf (po_run_t *r, const po_tfsf_t *t, const double *frames);
/* Face regions (24 x {min[3], max[3]}; volume <= 0: face unused) and the
 * doubles per frame. */
long po_tfsf_faces (const po_run_t *r, int *regions);
/* Frames recorded so far (record mode), copied to out when out != NULL. */
long po_tfsf_recorded (const po_run_t *r, double *out);

/* Focused-laser soft source of a parabolic mirror (scpic/em_mirror.c,
 * scpic/em_sources.c): v = the nine "@" doubles of a .EM_sources/laser
 * mirror file in its order (amplitude, f-number, focus x, y, z [micron],
 * duration [fs], arrival [fs], phase, radius ratio), direction = its last
 * value; r0, t0 = units(mc_r0), units(mc_t0) (binData/units.bin values 0
 * and 2); E, H = the file's two profiles, (n1-9)(n2-9) records {y_cos,
 * y_sin, z_cos, z_sin} each, j-major.  Up to 8 mirrors. */
void po_add_mirror (po_run_t *r, const double v[9], int direction, double r0, double t0,
                    const double *E, const double *H);

/* em_init / cap_init equivalent: ghost fill and Mur history from E. */
void po_init (po_run_t *r);

/* One full time step; out[5] = {W_E, W_M, W_Tx, W_Ty, W_Tz} at t = n*tau
 * (wDensity_addPoint arguments).  Returns 0. */
int  po_step (po_run_t *r, double out[5]);
/* po_step with the probe samples of core/diag_probe.c:409-429 taken after the
 * field energy: 7 doubles {t, Ex, Ey, Ez, Hx, Hy, Hz} per node of ijk. */
int  po_step_probes (po_run_t *r, const int *ijk, int n, double *samples, double out[5]);
/* E^n and H^n of the coming step over [0, n]^3, the run's state unchanged. */
void po_fields_n (po_run_t *r, double *E, double *H);
double po_time (const po_run_t *r);

/* Stage-level entry points (same order as core/main.c's loop). */
void po_em_h_half (po_run_t *r);
void po_em_energy (const po_run_t *r, double *we, double *wm);
void po_plasma_move (po_run_t *r, double wt[3]);
void po_em_h_step (po_run_t *r);
void po_em_e_step (po_run_t *r);
void po_jbc (po_run_t *r);
void po_em_e_finish (po_run_t *r);

/* Charge density (plasma.c:322-329, plasma_rho.c restated, walls folded)
 * into an internal mesh of po_mesh_size doubles. */
void po_rho (const po_run_t *r, double *rho);
long po_mesh_size (const po_run_t *r);
/* The region [-2, n+2]^3 of an internal mesh, k fastest. */
void po_region (const po_run_t *r, const double *mesh, double *out);
/* Gauss-law test (plasma_gaussTest.c:110-149): out = {max |(rho2-rho1)/tau
 * + div J|, max |div E - rho2|} over nodes [0, n]^3. */
void po_gauss (const po_run_t *r, const double *rho1, const double *rho2, double out[2]);

/* Marsaglia-Zaman "ranmar" generator (misc_ranmar.c:79-146 restated). */
typedef struct {
   double u[97], c, cd, cm;
   int    i97, j97;
} po_ranmar_t;

void po_ranmar_init (po_ranmar_t *g, int ij, int kl);
void po_ranmar (po_ranmar_t *g, double *out, long n);

/* Uniform random placer (new component, no reference counterpart).  Cells
 * [lo,hi) per axis in i-major, k-minor order; per marker seven draws:
 * three in-cell offsets, then two Box-Muller pairs of which the first three
 * normals scale u_th.  Stream = ranmar(ij,kl) after `skip` draws. */
typedef struct {
   int    lo[3], hi[3];
   int    ppc;
   double rho;          /* marker weight (charge density per marker)  */
   double qDivM;
   double drift[3];     /* mean u = gamma v / c                       */
   double uth[3];       /* per-axis normal spread of u                */
   int    seed_ij, seed_kl;
   long   skip;
   int    id0;          /* first id (ids are consecutive)             */
} po_place_t;

long po_place_count (const po_place_t *s);
long po_place (const po_place_t *s, const double h[3], po_marker_t *out);

/* Laser incident field used by the soft source (for tests). */
double po_laser_ey (const po_laser_t *l, double x, double y, double z,
                    double t, double ymid, double zmid);

#ifdef __cplusplus
}
#endif

#endif
