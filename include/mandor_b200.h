/* mandor_b200.h -- C ABI of the B200 particle-in-cell core.
 *
 * The reference Mandor (cvarin/mandor3) exposes no plugin or FFI layer: its
 * hot path is the in-process L2 C API that core/main.c calls once per time
 * step (core/em.h:32-39, core/plasma.h:82-87) over global meshes and the
 * global marker array.  This header replaces that API with an opaque,
 * device-resident run object:
 *
 *   reference call (file:line)                    replacement
 *   em_init            (core/em.c:40-49)          mg_run_init
 *   plasma_init        (core/plasma.c:343-418)    mg_run_init
 *   em_HHalfStep       (core/em.c:85-110)         mg_em_HHalfStep
 *   em_energy          (core/em.c:227-252)        mg_em_energy
 *   plasma_move        (core/plasma.c:269-305)    mg_plasma_move
 *   plasma_temperature (core/plasma.c:311-316)    mg_plasma_temperature
 *   em_HStep           (core/em.c:115-131)        mg_em_HStep
 *   em_EStep_start     (core/em.c:135-163)        mg_em_EStep_start
 *   jbc_finish         (core/plasma_currentWalls.c:172-209)  mg_jbc_finish
 *   em_EStep_finish    (core/em.c:189-222)        mg_em_EStep_finish
 *   plasma_rho         (core/plasma.c:321-329)    mg_plasma_rho
 *   sysIO_loadEM / plasma_load (IO_sys.c:130-142, core/plasma_IO.c:227-266)
 *                                                 mg_run_set_fields / mg_run_set_markers
 *   sysIO_save / plasma_save   (IO_sys.c:99-124, core/plasma_IO.c:273-287)
 *                                                 mg_run_get_fields / mg_run_get_markers
 *   the whole step loop (core/main.c:353-478)     mg_run_step
 *
 * Data crossing the boundary keeps the reference's layouts: fields are the
 * checkpoint region [0,n] per axis of vec3D_t nodes (k fastest), markers are
 * the 64-byte marker_t records with the tracer id.  Every call returns an
 * int status (MG_OK == 0, negative on error) instead of the reference's
 * ENSURE/DIE exit; mg_last_error() returns the message of the last failure
 * on the calling thread.  Calls on one run are not thread-safe; distinct
 * runs may be driven from distinct threads.
 */
#ifndef MANDOR_B200_H
#define MANDOR_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MG_OK             0
#define MG_ERR_CUDA      (-1)   /* CUDA runtime error                        */
#define MG_ERR_ARG       (-2)   /* bad argument                              */
#define MG_ERR_OOM       (-3)   /* device allocation failed                  */
#define MG_ERR_STATE     (-4)   /* stage called out of order                 */
#define MG_ERR_CAPACITY  (-5)   /* marker capacity exceeded                  */
#define MG_ERR_BOUNDS    (-6)   /* device bounds check tripped (marker left
                                   the J ghost layers: Courant violated)     */
#define MG_ERR_IO        (-7)   /* input file error: core_b200.out exits 7   */
#define MG_ERR_ADMISSION (-8)   /* serving admission refused (HBM budget)    */
#define MG_ERR_TIMEOUT   (-9)   /* a bounded device wait gave up             */

/* Boundary condition codes, same values as misc_parameters.h:38-42. */
enum { MG_BC_PERIODIC = 0, MG_BC_MIRROR = 1, MG_BC_OPEN = 2 };

/* Precision forms. */
enum {
   MG_FP64 = 0,         /* reference arithmetic: FP64 positions, momenta, fields */
   MG_FP32_OFFSET = 1   /* int cell + FP32 offset, FP32 u/E/H/J, FP64 reductions */
};

/* marker_t with ACTIVATE_TRACER=1 (type_marker.h:12-25): 64 bytes. */
typedef struct {
   double x, y, z;       /* absolute position, wavelengths            */
   double vx, vy, vz;    /* u = gamma v / c                           */
   float  rho;           /* charge density weight                     */
   float  qDivM;         /* charge to mass ratio                      */
   int    id;            /* tracer id                                 */
   int    pad_;
} mg_marker_t;

typedef struct {
   int       n[3];        /* cells per axis (dmn_max, dmn_min = 0)     */
   double    h[3];        /* mesh steps h1, h2, h3                     */
   double    tau;         /* time step                                 */
   int       bc_min[3];   /* MG_BC_* per axis, lower wall              */
   int       bc_max[3];   /* MG_BC_* per axis, upper wall              */
   double    time;        /* start time                                */
   int       precision;   /* MG_FP64 or MG_FP32_OFFSET                 */
   int       device;      /* CUDA device ordinal                       */
   long long capacity;    /* marker capacity (0: grows on upload)      */
   int       sort_every;  /* re-sort markers every k steps: by tile and cell
                             (precision form) or by cell (plain form);
                             0 = every 16 (precision form) or 24 (plain
                             form); < 0 = never (precision form: untiled
                             push)                                        */
   int       tile[3];     /* precision form: tile of the push in cells,
                             {8,8,4} (also {0,0,0}), {4,4,4} or {8,8,8} */
   int       tile_warps;  /* precision form: warps per block of the tiled
                             push (markers of a tile pushed at once / 32):
                             8 (also 0), 4 or 16                          */
} mg_params_t;

/* Analytic laser source: paraxial Gaussian beam, Ey polarised, moving along
 * +x, sin^2 field envelope, injected as a one-sided soft source on the
 * x-planes i = plane (H) and i = plane - 1 (E), with the injection pattern
 * of the reference's plane soft source (scpic/em_mirror.c:666-717). */
typedef struct {
   double a0;          /* normalised amplitude; E amplitude = 2*pi*a0      */
   double waist;       /* w0, wavelengths                                  */
   double x_focus;     /* focal plane x, wavelengths                       */
   double duration;    /* sin^2 envelope length, periods                   */
   double t_start;     /* time the envelope front leaves x = 0             */
   double phase;       /* carrier phase offset                             */
   int    plane;       /* H plane index (E plane is plane - 1)             */
   int    margin;      /* transverse nodes kept free next to each wall     */
} mg_laser_t;

/* Uniform random marker placement driven by the reference's ranmar
 * generator (misc_ranmar.c:79-146).  Cells [lo, hi) per axis, i-major and
 * k-minor; per marker seven consecutive draws: three in-cell offsets, then
 * two Box-Muller pairs (r = sqrt(-2 log(1 - u)), angle 2 pi u') whose first
 * three normals scale uth.  The logarithm, sine and cosine are the
 * library's own series in IEEE +, -, *, /, sqrt only, so positions and
 * momenta are the same bits as a C restatement on the host.  The stream is
 * ranmar(seed_ij, seed_kl) after `skip` draws; marker m of the box uses
 * draws [skip + 7m, skip + 7m + 7). */
typedef struct {
   int       lo[3], hi[3];
   int       ppc;
   double    rho;        /* weight per marker                               */
   double    qDivM;
   double    drift[3];
   double    uth[3];
   int       seed_ij, seed_kl;
   long long skip;
   int       id0;        /* id of the first marker; ids are consecutive     */
} mg_place_t;

typedef struct mg_run mg_run_t;

/* ---- run lifetime ----------------------------------------------------- */
int  mg_run_create (const mg_params_t *params, mg_run_t **out);
int  mg_run_destroy (mg_run_t *run);

/* ---- state in the reference layouts (host buffers) ----------------------
 * Fields: E and H over [0,n0]x[0,n1]x[0,n2], 3 doubles per node, k fastest
 * (the checkpoint region written by sysIO_save, type_mesh.c:285-313).     */
int  mg_run_set_fields (mg_run_t *run, const double *E, const double *H);
int  mg_run_get_fields (mg_run_t *run, double *E, double *H);
/* J over [-2,n0+2]x[-2,n1+2]x[-2,n2+2] after mg_jbc_finish.                */
int  mg_run_get_current (mg_run_t *run, double *J);
int  mg_run_set_markers (mg_run_t *run, const mg_marker_t *m, long long n);
/* Live markers, in device order (ids identify them, as in the reference). */
int  mg_run_get_markers (mg_run_t *run, mg_marker_t *m, long long cap, long long *n);
int  mg_run_marker_count (mg_run_t *run, long long *n);
int  mg_run_set_laser (mg_run_t *run, const mg_laser_t *laser);
int  mg_run_set_time (mg_run_t *run, double time);
int  mg_run_get_time (mg_run_t *run, double *time);
/* Appends markers placed on the device (bit-exact with the CPU placement). */
int  mg_run_place_uniform (mg_run_t *run, const mg_place_t *spec);

/* em_init + plasma_init: ghost refresh, Mur history, checks. */
int  mg_run_init (mg_run_t *run);

/* ---- stage API, one call per reference call of core/main.c:353-478 ---- */
int  mg_em_HHalfStep (mg_run_t *run);
int  mg_em_energy (mg_run_t *run, double *W_E, double *W_M);
int  mg_plasma_move (mg_run_t *run);
int  mg_plasma_temperature (mg_run_t *run, double *WTx, double *WTy, double *WTz);
int  mg_em_HStep (mg_run_t *run);
int  mg_em_EStep_start (mg_run_t *run);
int  mg_jbc_finish (mg_run_t *run);
int  mg_em_EStep_finish (mg_run_t *run);
/* CIC charge density over [-2,n+2]^3 (not folded), host buffer.           */
int  mg_plasma_rho (mg_run_t *run, double *rho);

/* ---- whole steps --------------------------------------------------------
 * Runs nsteps full time steps on the device.  If energies is not NULL it
 * receives nsteps rows {t, W_E, W_M, W_Tx, W_Ty, W_Tz} (the arguments of
 * wDensity_addPoint, core/diag_WDensity.c:136-147), copied back once at the
 * end.  Steps are replayed from a captured CUDA graph.                     */
int  mg_run_step (mg_run_t *run, int nsteps, double *energies);
/* Same, but the energy rows stay on the device (device pointer, nsteps*6
 * doubles); no host synchronisation.                                      */
int  mg_run_step_async (mg_run_t *run, int nsteps, double *energies_dev);
int  mg_run_synchronize (mg_run_t *run);
/* The CUDA stream (cudaStream_t) the run launches on.                     */
int  mg_run_stream (mg_run_t *run, void **stream);
/* Device kernels launched per step (for launch accounting).               */
int  mg_run_kernels_per_step (mg_run_t *run, int *count);
/* Device memory the run holds, bytes.                                     */
int  mg_run_device_bytes (mg_run_t *run, long long *bytes);
/* Estimated device bytes for a run with these parameters and markers
 * (without markers it includes the second E and H arrays of the one-pass
 * field step).                                                            */
long long mg_estimate_bytes (const mg_params_t *params, long long markers);

/* ---- tecplot dumps (IO_tecplot.c:108-266) --------------------------------
 * Node-centred fields over [0, n]^3, AoS (n+1)^3 x 3 doubles, as tecIO_saveVec
 * interpolates them: E and J as 0.5 (F[p] + F[p + d_c]) per component c, H as
 * the average of its 4 nodes in the two other axes.  core.out writes E and H
 * after plasma_move (E^n and H^n: call mg_tecplot_fields after
 * mg_plasma_move) and J after the E step (mg_tecplot_currents after
 * mg_em_EStep_finish); core_b200.out does both at the tecplot period of
 * run_mandor.cfg.                                                          */
int  mg_tecplot_fields (mg_run_t *run, double *E, double *H);
int  mg_tecplot_currents (mg_run_t *run, double *J);

/* ---- asynchronous checkpoints -----------------------------------------------
 * mg_run_snapshot: the state mg_run_get_fields and mg_run_get_markers would
 * return (E, H over the checkpoint region; the live markers, compacted;
 * *n their count) is copied into device buffers of the run at the current
 * step boundary and then to E, H, m (NULL: skipped) on a stream of its own;
 * the call returns once the device copy is taken, and the run may keep
 * stepping.  The host buffers must not be read before mg_run_snapshot_wait
 * (the next snapshot, and mg_run_destroy, wait too).  Pinned buffers from
 * mg_host_alloc let the copy overlap the steps.  Replaces the synchronous
 * sysIO_save / plasma_save reads of core/main.c:445-460 with no change to
 * the files written.  No counterpart in the reference.                      */
int   mg_run_snapshot (mg_run_t *run, double *E, double *H, mg_marker_t *m, long long cap, long long *n);
int   mg_run_snapshot_wait (mg_run_t *run);
void *mg_host_alloc (size_t bytes);
void  mg_host_free (void *p);

/* ---- TF/SF interface (core/em_TFSF.c) -------------------------------------
 * Replaces TFSF_init / TFSF_preHStep / TFSF_postHStep / TFSF_postEStep /
 * TFSF_completeFrame (core/em_TFSF.c:480-853, called from core/em.c:92,
 * 125, 200, 218).  24 faces: the E faces Ey_xMin, Ez_xMin, Ey_xMax, Ez_xMax,
 * Ez_yMin, Ex_yMin, Ez_yMax, Ex_yMax, Ex_zMin, Ey_zMin, Ex_zMax, Ey_zMax, then
 * the H faces Hz_xMin, Hy_xMin, ..., Hx_zMax (core/em_TFSF.c:86-119).  A
 * frame is the values of the 12 E faces then of the 12 H faces, each over
 * its region (mg_run_tfsf_faces) with the face's first tangential axis
 * (a+1)%3 slowest: the layout of the recorded streams after their reg_t
 * header.
 *   record: every step stores E^n and H^(n-1/2) times the face's source
 *           factor at its start; mg_run_tfsf_recorded copies the frames of
 *           the last mg_run_step call (<= 4096 steps) or staged step.
 *   play:   frames come from the merged streams (*_99999.bin); the step
 *           with frame counter n (int (t/tau + 0.1) at mg_run_set_tfsf, +1
 *           per step) reads frame n and n + 1 forward, T - 1 - n backward,
 *           and plays while n + 1 < T - 1 (T = frames).  They must be on
 *           the device, in a ring of `ring` slots, before the step runs
 *           (mg_run_tfsf_put_frames); a missing frame fails the step with
 *           MG_ERR_STATE.  Played faces must stay 5 cells inside the walls.
 * mg_run_set_tfsf (run, NULL) removes the interface.                        */
enum { MG_TFSF_PLAY_FORWARD = 0, MG_TFSF_RECORD = 1, MG_TFSF_PLAY_BACKWARD = 2 };
typedef struct {
   int lo[3], hi[3];       /* interface bounding box (TFSF.cfg)               */
   int mode;               /* MG_TFSF_*                                        */
   int open[2][3];         /* play: faces removed, [min/max][axis]            */
   int frames;             /* play: frames recorded (lastFrameTime.bin)       */
   int ring;               /* play: device frame slots (>= 2)                 */
} mg_tfsf_t;
int  mg_run_set_tfsf (mg_run_t *run, const mg_tfsf_t *cfg);
int  mg_run_tfsf_faces (mg_run_t *run, int regions[24*6], long long *frame_doubles);
int  mg_run_tfsf_put_frames (mg_run_t *run, int first, int count, const double *frames);
int  mg_run_tfsf_recorded (mg_run_t *run, int nsteps, double *frames);

/* ---- probes (core/diag_probe.c:409-446) ----------------------------------
 * mg_run_set_probes: probe nodes ijk[3*q..3*q+2] in [0, n) (n = 0 removes
 * them).  Every step then records, right after the H half step (where
 * core/main.c:373 calls probe_postData), one row {t, Ex, Ey, Ez, Hx, Hy, Hz}
 * per probe of E^n and H^n interpolated to the node like the tecplot
 * dumps.  mg_run_probe_samples copies the rows of the steps of the last
 * mg_run_step call (nsteps <= 4096, rows step-major, nsteps x nprobes x 7) or,
 * after a staged step, its one row.                                       */
int  mg_run_set_probes (mg_run_t *run, const int *ijk, int nprobes);
int  mg_run_probe_samples (mg_run_t *run, int nsteps, double *out);

/* ---- the reference's placers (setup.out tags) on the device --------------
 * Markers are appended in setup.out's order with ids id0, id0+1, ... (the
 * ids setup/plasma.c:93-123 writes); positions, momenta and weights are
 * bit-identical to setup.out's.  Call mg_run_init afterwards.
 *
 * mg_run_place_maxwell: [plasma] (setup/tag_plasma.c:45-152, no filters)
 * then [DF:Maxwell] (setup/tag_maxwell.c:36-168): in every cell (I-major) the
 * lattice points ((i + 1/2)/nx) h1 + I h1, ... of nx*ny*nz per cell, `layers`
 * markers on each (an even number); momenta from the quiet-start pattern
 * (Hammersley radix-2/3/5 quartets, setup/setup_denavit.c, mapped through the
 * inverse of the integral of exp(-x^2), setup/setup_distrMapper.c, or uniform
 * spacing with exp(-x^2) weights), mirrored pairs, weights normalised to
 * rho = omega_pe2 4 pi^2 / qDivM / markers-per-cell, optionally the thermal
 * energy tuned (tune_energy).                                              */
typedef struct {
   int    nx, ny, nz, layers;
   double omega_pe2;      /* (omega_pe/omega_0)^2                         */
   double qDivM;
   double ux, uy, uz;     /* thermal momenta per axis                      */
   int    tune_energy, uniform_weight;
   int    id0;
} mg_maxwell_t;
int  mg_run_place_maxwell (mg_run_t *run, const mg_maxwell_t *spec);

/* mg_run_place_foil: [DF:foil] (setup/tag_foil.c:60-230): lattice points of
 * nx*ny*nz per cell in the cells [5, n-5) of every axis whose lower wall is
 * not periodic ([0, n) otherwise) where alpha = (shift - (r - r0).l)/width
 * + 1/2 lies in [m, 1 - m], m = 1e-10 (h1+h2+h3)/(3 width); rho =
 * (n1 + (n2 - n1) alpha)/(nx ny nz) (profile 0) or n1 (n2/n1)^alpha/(nx ny nz)
 * (profile 1), with n1, n2 converted as the deck gives them (< 0: critical
 * densities, > 0: cm^-3) for charge q and wavelength lambda_cm
 * (misc_units.c:95-120); u = 0, qDivM = q/M.  Lengths in wavelengths.     */
typedef struct {
   double x0, y0, z0;     /* foil centre                                   */
   double lx, ly, lz;     /* normal (normalised here)                      */
   double width, shift;
   int    profile;        /* 0 linear, 1 exponential                       */
   double n1, n2;
   double q, M;           /* charge in |e|, mass in m_e                    */
   int    nx, ny, nz;
   double lambda_cm;      /* wavelength, cm ([units] tag x 1e-4)           */
   int    id0;
} mg_foil_t;
int  mg_run_place_foil (mg_run_t *run, const mg_foil_t *spec);

/* mg_run_place_two_stream: [DF:two-stream] (setup/tag_twoStream.c:23-103):
 * n[0] n[1] n[2] lattice nodes ((i + 1/2) L_x/n_x, ...) each with a marker
 * of u = +V and one of u = -V (in that order), V = gamma sqrt(3)/(2|k|)
 * along k = 2 pi (m_x/L_x, m_y/L_y, m_z/L_z), rho = gamma^2/qDivM
 * L_x L_y L_z/(h1 h2 h3 n_x n_y n_z); L: the domain lengths of
 * binData/domain.bin; ids id0, id0 + 1, ...                               */
typedef struct {
   double gamma, qDivM;   /* growth rate, q/M (|q/M| <= 1)                 */
   int    n[3], m[3];     /* markers per beam along each axis; mode numbers */
   double L[3];
   int    id0;
} mg_two_stream_t;
int  mg_run_place_two_stream (mg_run_t *run, const mg_two_stream_t *spec);

/* mg_run_df_uniform: [DF:uniform] (setup/tag_DF_uniform.c:36-70) on the
 * placed markers [first, first + count) (before mg_run_init): u = u0 +
 * (rand ()/RAND_MAX - 1/2) du per axis with the GNU C library's rand () from
 * its default seed, three draws per marker (x, y, z), after draws_before
 * draws taken by earlier tags; rho = rho_deck rho_crit/ppc (rho_crit = e
 * n_cr/rho0 for wavelength lambda_cm), q/M as given.
 * mg_run_shift_velocity: [velocity shift] 'last' (setup/tag_vShift.c:29-49):
 * u += dv on [first, first + count).                                       */
typedef struct {
   double rho, qDivM, ux, uy, uz, dux, duy, duz;   /* the tag's values, its order */
   int    ppc;            /* particles per cell of the markers' [plasma] tag */
   double lambda_cm;
   long long draws_before;
} mg_df_uniform_t;
int  mg_run_df_uniform (mg_run_t *run, long long first, long long count, const mg_df_uniform_t *df);
int  mg_run_shift_velocity (mg_run_t *run, long long first, long long count, const double dv[3]);

/* ---- focused-laser soft sources (scpic/em_mirror.c, scpic/em_sources.c) ----
 * Replaces init_sources / add_H_sources / add_E_sources (scpic/em_sources.c,
 * called from core/em.c:126, 208).  A mirror as setup.out's [focused laser]
 * tag leaves it in .EM_sources/laser/mirror_NN: its nine "@" doubles in the
 * file's order (amplitude: < 0 e E/(m w c), > 0 intensity [W/cm^2]; f-number;
 * focus x, y, z [micron]; duration [fs]; arrival at the focus [fs]; phase;
 * radius ratio), the direction (> 0: +x), and its E and H profiles over the
 * x-plane nodes j, k in [5, n - 5] ((n1-9)(n2-9) records of {y_cos, y_sin,
 * z_cos, z_sin}, j-major); r0 and t0 are units (mc_r0) and units (mc_t0)
 * (binData/units.bin doubles 0 and 2).  After the H step (after TF/SF) the
 * H plane i = 5 (backward n0 - 4) gets Hy += a (z_cos cos p + z_sin sin p),
 * Hz += a (y_cos cos p + y_sin sin p) of the E profile at t, after the E
 * step the E plane i = 4 (backward n0 - 4) the same of the H profile at
 * t + tau/2, with a = exp (-(2 t'/dt)^2) tau/h1, p = 2 pi t' + phi0 and
 * t' = t - T0 + delay, all converted as scpic/em_mirror.c:292-332 does.   */
typedef struct {
   double values[9];
   int    direction;
   double r0, t0;
   const double *E, *H;
} mg_mirror_t;
int  mg_run_add_mirror (mg_run_t *run, const mg_mirror_t *mirror);
int  mg_run_clear_mirrors (mg_run_t *run);

/* ---- hard gauss-spot source (core/em_gaussSpot.c:31-156) -----------------
 * The fields of .gaussSpot.cfg (written by setup/tag_gaussSpot.c:126-140),
 * in its order.  After every E step (em_EStep_finish, core/em.c:216, at time
 * t + tau) Ey and Ez on the x-plane i = (int) (x/h1 + 0.5) are set, for all
 * j, k in [-1, n+1], to
 *   Ey = sgn(ey) ampl sin(w t) f(t) exp(-dy_^2 - dz^2),
 *   Ez = sgn(ez) ampl cos(w t) f(t) exp(-dy^2 - dz_^2),
 * w = 2 pi frequency, dy = (j h2 - y)/width, dy_ = ((j - 1/2) h2 - y)/width
 * (z alike), f = exp(-l^2) before front_offset with l = (t - front_offset)/
 * duration, 1 on the plateau, exp(-l^2) after it with l = (t - front_offset
 * - t_plateau)/duration.  NULL switches the source off.                    */
typedef struct {
   double ampl;          /* amplitude, units of E0                        */
   double frequency;     /* omega / omega_0                               */
   double x, y, z;       /* focal spot                                    */
   double width;
   double duration;
   double front_offset;
   double t_plateau;
   int    ey, ez;        /* polarisation flags (their signs are used)     */
} mg_gauss_spot_t;
int  mg_run_set_gauss_spot (mg_run_t *run, const mg_gauss_spot_t *spot);

/* ---- Gauss-law test (core/plasma_gaussTest.c:89-149) ---------------------
 * FP64 arithmetic in both precision forms.  mg_gauss_before stores the
 * charge density of the markers as they are (core/main.c:376 calls
 * gauss_before after em_energy, before plasma_move); mg_gauss_after computes
 * it again and returns out = {max |(rho2 - rho1)/tau + div J|,
 * max |div E - rho2|} over nodes [0, n]^3 (after em_EStep_finish,
 * core/main.c:428).  mg_run_step_gauss runs nsteps whole steps with the test
 * around each and writes nsteps rows {t, deltaRho_J, deltaRho_E}, the
 * columns of output/gauss_test.dat (t: the time at the start of the step).
 * The density is plasma_rho's (core/plasma.c:322-329, walls folded by
 * core/plasma_rho.c:23-97; VSP filter off).                              */
int  mg_gauss_before (mg_run_t *run);
int  mg_gauss_after (mg_run_t *run, double out[2]);
int  mg_run_step_gauss (mg_run_t *run, int nsteps, double *rows);

/* ---- batches of independent runs -----------------------------------------
 * No counterpart in the reference (one simulation per core.out process).  A
 * batch steps many runs of one device with ONE CUDA graph launch per step:
 * each run's captured step graph is an independent branch of the batch
 * graph, so small runs fill the GPU together.  Runs keep their own state,
 * streams and energy rows; a run may belong to several batches but must not
 * be stepped through another path while a batch step is in progress.
 * mg_batch_step runs nsteps steps of every run; energies[i] (host, nsteps*6
 * doubles, may be NULL) receives run i's rows.  Precision-form runs are
 * re-sorted by tile between launches at their own sort_every.            */
typedef struct mg_batch mg_batch_t;
int  mg_batch_create (mg_run_t *const *runs, int nruns, mg_batch_t **out);
int  mg_batch_step (mg_batch_t *batch, int nsteps, double *const *energies);
int  mg_batch_destroy (mg_batch_t *batch);

/* Kernel-level timing of the last mg_run_step: average device time of the
 * push kernel and of the whole step, milliseconds (CUDA events on the run's
 * stream).  Enabled by mg_run_profile(run, 1).                            */
int  mg_run_profile (mg_run_t *run, int enable);
int  mg_run_last_timing (mg_run_t *run, double *push_ms, double *step_ms);

/* ---- placement into caller-owned device memory ---------------------------
 * No counterpart in the reference.  Device arrays of one marker population
 * in structure-of-arrays form, each with room for `capacity` markers. */
typedef struct {
   double *x, *y, *z, *vx, *vy, *vz;
   float  *rho, *qDivM;
   int    *id;
} mg_device_markers_t;

/* Writes the markers of `spec` (the placement rule of mg_place_t, cell box
 * measured with steps h) to out[0 .. count), allocating nothing on the
 * device or the host.  It serves callers that cannot call cudaMalloc: a
 * host application whose caching allocator has already reserved the
 * GPU's memory and hands this library slices of it (a cudaMalloc there
 * fails or evicts the host's pool), and code that must not take the
 * implicit device-wide synchronisation of cudaMalloc/cudaFree while other
 * streams of the process are running.  The generator start states go
 * through a file-scope device array of at most 4096 states (1.59 MB,
 * resident on every GPU that loads the library until the process exits);
 * `threads` (0 = 4096) sets how many states, i.e. parallel generator
 * streams, are used and is rejected above 4096 with MG_ERR_ARG; output
 * arrays shorter than the box's marker count are rejected with
 * MG_ERR_CAPACITY.  The first call on a device looks up that array's device
 * address with the device current and keeps it, so make that first call
 * before any stream capture, and do not call it again on a device after
 * cudaDeviceReset.  A call runs on `stream` (a cudaStream_t, NULL for the
 * legacy stream) of the current device: it copies the start states there
 * from pageable host memory, launches one kernel and waits for the stream
 * before returning.  The array is shared by every call in the process
 * (calls are serialised by a lock) and overwritten each time, so other
 * work that overlapped a call on the GPU and used the array would race on
 * it.  Output is bit-identical to mg_run_place_uniform. */
int  mg_place_uniform_static (const mg_place_t *spec, const double h[3],
                              const mg_device_markers_t *out, long long capacity,
                              int threads, void *stream);

const char *mg_last_error (void);
const char *mg_version (void);

#ifdef __cplusplus
}
#endif

#endif
