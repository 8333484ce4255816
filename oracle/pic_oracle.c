/* CPU restatement of Mandor's PIC time step -- TEST INFRASTRUCTURE ONLY.
 *
 * Every function below names the reference code it restates (paths are
 * relative to the reference project).  The mesh is one global array per
 * field component with two ghost layers on every side; the reference's
 * boundary "caps" (core/em_caps.c) compute the same Yee update on boundary
 * slabs with a single full-tau H step instead of two half steps, so fields
 * near walls agree with the reference to round-off, not bit-for-bit.
 *
 * Build: oracle/Makefile target `port` -> oracle/_build/libpic_oracle.so.
 */
#include "pic_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define G 2                         /* ghost layers on every side */

struct po_run {
   int    n[3];
   double h[3], tau, time;
   int    bc[2][3];                 /* [min/max][axis] */
   int    dim[3];                   /* n + 1 + 2G */
   long   s[3];                     /* strides: s[2] = 1 */
   double *e[3], *b[3], *j[3];      /* E, H, J components */
   double *mur[2][3];               /* Mur history: 4 doubles per wall node */
   double mur_alpha[3];
   po_marker_t *p;
   long   np;
   po_laser_t laser;
   int    has_laser;
   po_gauss_spot_t gspot;
   int    has_gspot;
   /* focused-laser mirrors */
   int    nmirror;
   struct { double A, dt, T0, delay, phi0; int forward; double *E, *H; } mirror[8];
   /* TF/SF interface */
   int    has_tfsf, tfsf_on, tfsf_frame;
   po_tfsf_t tfsf;
   struct { int min[3], max[3], comp, ep, eq, used; double sf; long vol, at; } face[24];
   long   frame_size;
   double *frames;                  /* play: recorded frames */
   long   nrec;                     /* record: frames written */
   double *rec;
};

static inline long IX (const po_run_t *r, int i, int j, int k)
{
   return (i + G)*r->s[0] + (j + G)*r->s[1] + (k + G);
}

/* Offset of node (a along axis ea, p along ep, q along eq). */
static inline long IXA (const po_run_t *r, int ea, int a, int ep, int p, int eq, int q)
{
   int c[3];
   c[ea] = a;
   c[ep] = p;
   c[eq] = q;
   return IX (r, c[0], c[1], c[2]);
}

po_run_t *po_create (const int n[3], const double h[3], double tau,
                     const int bc_min[3], const int bc_max[3], double time)
{
   po_run_t *r = (po_run_t *) calloc (1, sizeof (po_run_t));
   for (int a = 0 ; a < 3 ; ++a) {
      r->n[a] = n[a];
      r->h[a] = h[a];
      r->bc[0][a] = bc_min[a];
      r->bc[1][a] = bc_max[a];
      r->dim[a] = n[a] + 1 + 2*G;
      r->mur_alpha[a] = (tau - h[a])/(tau + h[a]);   /* core/em_caps.c:380 via emCap_Mur.c:102 */
   }
   r->tau = tau;
   r->time = time;
   r->s[2] = 1;
   r->s[1] = r->dim[2];
   r->s[0] = (long) r->dim[1]*r->dim[2];
   long total = (long) r->dim[0]*r->s[0];
   for (int c = 0 ; c < 3 ; ++c) {
      r->e[c] = (double *) calloc (total, sizeof (double));
      r->b[c] = (double *) calloc (total, sizeof (double));
      r->j[c] = (double *) calloc (total, sizeof (double));
   }
   for (int t = 0 ; t < 2 ; ++t)
      for (int a = 0 ; a < 3 ; ++a) {
         int ep = (a + 1) % 3, eq = (a + 2) % 3;
         r->mur[t][a] = (double *) calloc ((size_t) 4*r->dim[ep]*r->dim[eq], sizeof (double));
      }
   return r;
}

void po_destroy (po_run_t *r)
{
   if (!r)
      return;
   for (int c = 0 ; c < 3 ; ++c) {
      free (r->e[c]);
      free (r->b[c]);
      free (r->j[c]);
   }
   for (int t = 0 ; t < 2 ; ++t)
      for (int a = 0 ; a < 3 ; ++a)
         free (r->mur[t][a]);
   free (r->p);
   free (r->frames);
   free (r->rec);
   for (int q = 0 ; q < r->nmirror ; ++q) {
      free (r->mirror[q].E);
      free (r->mirror[q].H);
   }
   free (r);
}

double po_time (const po_run_t *r) { return r->time; }

/* Checkpoint region [0,n]^3 in reference order (type_mesh.c:285-313). */
void po_set_fields (po_run_t *r, const double *E, const double *H)
{
   long q = 0;
   for (int i = 0 ; i <= r->n[0] ; ++i)
   for (int j = 0 ; j <= r->n[1] ; ++j)
   for (int k = 0 ; k <= r->n[2] ; ++k, q += 3) {
      long o = IX (r, i, j, k);
      for (int c = 0 ; c < 3 ; ++c) {
         r->e[c][o] = E[q + c];
         r->b[c][o] = H[q + c];
      }
   }
}

void po_get_fields (const po_run_t *r, double *E, double *H)
{
   long q = 0;
   for (int i = 0 ; i <= r->n[0] ; ++i)
   for (int j = 0 ; j <= r->n[1] ; ++j)
   for (int k = 0 ; k <= r->n[2] ; ++k, q += 3) {
      long o = IX (r, i, j, k);
      for (int c = 0 ; c < 3 ; ++c) {
         if (E) E[q + c] = r->e[c][o];
         if (H) H[q + c] = r->b[c][o];
      }
   }
}

void po_get_current (const po_run_t *r, double *J)
{
   long q = 0;
   for (int i = -G ; i <= r->n[0] + G ; ++i)
   for (int j = -G ; j <= r->n[1] + G ; ++j)
   for (int k = -G ; k <= r->n[2] + G ; ++k, q += 3) {
      long o = IX (r, i, j, k);
      for (int c = 0 ; c < 3 ; ++c)
         J[q + c] = r->j[c][o];
   }
}

void po_set_markers (po_run_t *r, const po_marker_t *m, long n)
{
   free (r->p);
   r->p = (po_marker_t *) malloc ((n > 0 ? n : 1)*sizeof (po_marker_t));
   if (n > 0)
      memcpy (r->p, m, n*sizeof (po_marker_t));
   r->np = n;
}

long po_marker_count (const po_run_t *r) { return r->np; }

void po_get_markers (const po_run_t *r, po_marker_t *m)
{
   if (r->np > 0)
      memcpy (m, r->p, r->np*sizeof (po_marker_t));
}

void po_set_laser (po_run_t *r, const po_laser_t *l)
{
   r->laser = *l;
   r->has_laser = 1;
}

/* ------------------------------------------------------------------------
 * Yee update ranges.  The union of the reference's inner loop and its six
 * cap regions (core/em_caps.c:66-109 tables, core/em.c:55-163 loops) is a
 * product of per-axis node ranges:
 *   H: periodic [0,n], mirror [1,n], Mur [0,n]
 *   E: lower bound 0 if periodic else 1; upper bound n-1 if periodic else n
 * ---------------------------------------------------------------------- */
static void h_range (const po_run_t *r, int a, int *lo, int *hi)
{
   *lo = (r->bc[0][a] == PO_BC_MIRROR) ? 1 : 0;
   *hi = r->n[a];
}

static void e_range (const po_run_t *r, int a, int *lo, int *hi)
{
   *lo = (r->bc[0][a] == PO_BC_PERIODIC) ? 0 : 1;
   *hi = (r->bc[1][a] == PO_BC_PERIODIC) ? r->n[a] - 1 : r->n[a];
}

/* H += frac*tau*(-curl E): core/em.c:55-77 (expression order kept). */
static void h_advance (po_run_t *r, double frac)
{
   const double c1 = frac*r->tau/r->h[0], c2 = frac*r->tau/r->h[1], c3 = frac*r->tau/r->h[2];
   const long sx = r->s[0], sy = r->s[1];
   double *Ex = r->e[0], *Ey = r->e[1], *Ez = r->e[2];
   double *Hx = r->b[0], *Hy = r->b[1], *Hz = r->b[2];
   int lo[3], hi[3];
   for (int a = 0 ; a < 3 ; ++a)
      h_range (r, a, lo + a, hi + a);
   for (int i = lo[0] ; i <= hi[0] ; ++i)
   for (int j = lo[1] ; j <= hi[1] ; ++j)
   for (int k = lo[2] ; k <= hi[2] ; ++k) {
      long o = IX (r, i, j, k);
      Hx[o] += c3*(Ey[o] - Ey[o - 1]) - c2*(Ez[o] - Ez[o - sy]);
      Hy[o] += c1*(Ez[o] - Ez[o - sx]) - c3*(Ex[o] - Ex[o - 1]);
      Hz[o] += c2*(Ex[o] - Ex[o - sy]) - c1*(Ey[o] - Ey[o - sx]);
   }
}

/* E -= tau*(curl H) without the current: core/em.c:135-163. */
static void e_advance (po_run_t *r)
{
   const double c1 = r->tau/r->h[0], c2 = r->tau/r->h[1], c3 = r->tau/r->h[2];
   const long sx = r->s[0], sy = r->s[1];
   double *Ex = r->e[0], *Ey = r->e[1], *Ez = r->e[2];
   double *Hx = r->b[0], *Hy = r->b[1], *Hz = r->b[2];
   int lo[3], hi[3];
   for (int a = 0 ; a < 3 ; ++a)
      e_range (r, a, lo + a, hi + a);
   for (int i = lo[0] ; i <= hi[0] ; ++i)
   for (int j = lo[1] ; j <= hi[1] ; ++j)
   for (int k = lo[2] ; k <= hi[2] ; ++k) {
      long o = IX (r, i, j, k);
      Ex[o] -= c3*(Hy[o + 1] - Hy[o]) - c2*(Hz[o + sy] - Hz[o]);
      Ey[o] -= c1*(Hz[o + sx] - Hz[o]) - c3*(Hx[o + 1] - Hx[o]);
      Ez[o] -= c2*(Hx[o + sy] - Hx[o]) - c1*(Hy[o + sx] - Hy[o]);
   }
}

/* Transverse extent of a wall operation: nodes [0, n+1] of the two other
 * axes (the flush regions of the caps, core/em_caps.c:140-146). */
#define FOR_WALL(r, ea, ep, eq, p, q)                          \
   for (int p = 0 ; p <= (r)->n[ep] + 1 ; ++p)                 \
   for (int q = 0 ; q <= (r)->n[eq] + 1 ; ++q)

/* H boundary conditions, axis by axis, min side then max side:
 * core/emCap_periodic.c:15-37, emCap_mirror.c:17-40, emCap_Mur.c:56-80. */
static void h_bc (po_run_t *r)
{
   for (int ea = 0 ; ea < 3 ; ++ea) {
      const int ep = (ea + 1) % 3, eq = (ea + 2) % 3, N = r->n[ea];
      double *Ha = r->b[ea], *Hp = r->b[ep], *Hq = r->b[eq];
      switch (r->bc[0][ea]) {
      case PO_BC_PERIODIC:
         FOR_WALL (r, ea, ep, eq, p, q) {
            long b0 = IXA (r, ea, 0, ep, p, eq, q), t0 = IXA (r, ea, N, ep, p, eq, q);
            long b1 = IXA (r, ea, 1, ep, p, eq, q), t1 = IXA (r, ea, N + 1, ep, p, eq, q);
            for (int c = 0 ; c < 3 ; ++c) {
               r->b[c][b0] = r->b[c][t0];
               r->b[c][t1] = r->b[c][b1];
            }
         }
         break;
      case PO_BC_MIRROR:
         FOR_WALL (r, ea, ep, eq, p, q) {
            long w = IXA (r, ea, 0, ep, p, eq, q), in = IXA (r, ea, 1, ep, p, eq, q);
            Ha[w] = 0;
            Hp[w] = Hp[in];
            Hq[w] = Hq[in];
         }
         break;
      case PO_BC_OPEN:
         FOR_WALL (r, ea, ep, eq, p, q) {
            long w = IXA (r, ea, 0, ep, p, eq, q), in = IXA (r, ea, 1, ep, p, eq, q);
            Hp[w] = Hp[in];
            Hq[w] = Hq[in];
         }
         break;
      }
      switch (r->bc[1][ea]) {
      case PO_BC_MIRROR:
         FOR_WALL (r, ea, ep, eq, p, q) {
            long w = IXA (r, ea, N, ep, p, eq, q), out = IXA (r, ea, N + 1, ep, p, eq, q);
            Ha[w] = 0;
            Hp[out] = Hp[w];
            Hq[out] = Hq[w];
         }
         break;
      case PO_BC_OPEN:
         FOR_WALL (r, ea, ep, eq, p, q) {
            long w = IXA (r, ea, N, ep, p, eq, q), out = IXA (r, ea, N + 1, ep, p, eq, q);
            Hp[out] = Hp[w];
            Hq[out] = Hq[w];
         }
         break;
      }
   }
}

/* Mur history index for wall node (p, q). */
static inline long MUR (const po_run_t *r, int ea, int p, int q)
{
   const int eq = (ea + 2) % 3;
   return 4*((long) p*r->dim[eq] + q);
}

/* E boundary conditions: core/emCap_periodic.c:42-67, emCap_mirror.c:45-70,
 * emCap_Mur.c:117-166 (history holds wall and first inner node, pre-current). */
static void e_bc (po_run_t *r)
{
   for (int ea = 0 ; ea < 3 ; ++ea) {
      const int ep = (ea + 1) % 3, eq = (ea + 2) % 3, N = r->n[ea];
      double *Ea = r->e[ea], *Ep = r->e[ep], *Eq = r->e[eq];
      const double alpha = r->mur_alpha[ea];
      switch (r->bc[0][ea]) {
      case PO_BC_PERIODIC:
         FOR_WALL (r, ea, ep, eq, p, q) {
            long b0 = IXA (r, ea, 0, ep, p, eq, q), t0 = IXA (r, ea, N, ep, p, eq, q);
            long b1 = IXA (r, ea, 1, ep, p, eq, q), t1 = IXA (r, ea, N + 1, ep, p, eq, q);
            for (int c = 0 ; c < 3 ; ++c) {
               r->e[c][t0] = r->e[c][b0];
               r->e[c][t1] = r->e[c][b1];
            }
         }
         break;
      case PO_BC_MIRROR:
         FOR_WALL (r, ea, ep, eq, p, q) {
            long w = IXA (r, ea, 0, ep, p, eq, q), in = IXA (r, ea, 1, ep, p, eq, q);
            Ep[w] = 0;
            Eq[w] = 0;
            Ea[w] = Ea[in];
         }
         break;
      case PO_BC_OPEN: {
         double *buf = r->mur[0][ea];
         FOR_WALL (r, ea, ep, eq, p, q) {
            long w = IXA (r, ea, 0, ep, p, eq, q), in = IXA (r, ea, 1, ep, p, eq, q);
            double *o = buf + MUR (r, ea, p, q);
            Ea[w] = Ea[in];
            Ep[w] = o[2] + alpha*(Ep[in] - o[0]);
            Eq[w] = o[3] + alpha*(Eq[in] - o[1]);
            o[0] = Ep[w];
            o[1] = Eq[w];
            o[2] = Ep[in];
            o[3] = Eq[in];
         }
         break;
      }
      }
      switch (r->bc[1][ea]) {
      case PO_BC_MIRROR:
         FOR_WALL (r, ea, ep, eq, p, q) {
            long w = IXA (r, ea, N, ep, p, eq, q), out = IXA (r, ea, N + 1, ep, p, eq, q);
            Ep[w] = 0;
            Eq[w] = 0;
            Ea[out] = Ea[w];
         }
         break;
      case PO_BC_OPEN: {
         double *buf = r->mur[1][ea];
         FOR_WALL (r, ea, ep, eq, p, q) {
            long w = IXA (r, ea, N, ep, p, eq, q), out = IXA (r, ea, N + 1, ep, p, eq, q);
            long in = IXA (r, ea, N - 1, ep, p, eq, q);
            double *o = buf + MUR (r, ea, p, q);
            Ea[out] = Ea[w];
            Ep[w] = o[2] + alpha*(Ep[in] - o[0]);
            Eq[w] = o[3] + alpha*(Eq[in] - o[1]);
            o[0] = Ep[w];
            o[1] = Eq[w];
            o[2] = Ep[in];
            o[3] = Eq[in];
         }
         break;
      }
      }
   }
}

static int particle_bc (const po_run_t *r, po_marker_t *m);

/* cap_init (core/em_caps.c:343-392): ghost refresh for periodic and mirror
 * walls, Mur history from the loaded E and the normal-E ghost copy
 * (emCap_Mur.c:86-112).  plasma_init (core/plasma.c:399-404) applies the
 * particle walls once to the loaded markers, which all start in the shell
 * (core/plasma_IO.c:265): markers within one cell of an open wall go. */
void po_init (po_run_t *r)
{
   long keep = 0;
   for (long n = 0 ; n < r->np ; ++n)
      if (!particle_bc (r, r->p + n))
         r->p[keep++] = r->p[n];
   r->np = keep;

   for (int ea = 0 ; ea < 3 ; ++ea) {
      const int ep = (ea + 1) % 3, eq = (ea + 2) % 3, N = r->n[ea];
      if (r->bc[0][ea] == PO_BC_PERIODIC) {
         FOR_WALL (r, ea, ep, eq, p, q) {
            long b0 = IXA (r, ea, 0, ep, p, eq, q), t0 = IXA (r, ea, N, ep, p, eq, q);
            long b1 = IXA (r, ea, 1, ep, p, eq, q), t1 = IXA (r, ea, N + 1, ep, p, eq, q);
            for (int c = 0 ; c < 3 ; ++c) {
               r->b[c][b0] = r->b[c][t0];
               r->b[c][t1] = r->b[c][b1];
               r->e[c][t0] = r->e[c][b0];
               r->e[c][t1] = r->e[c][b1];
            }
         }
      }
      for (int top = 0 ; top < 2 ; ++top) {
         int w_at = top ? N : 0;
         int in_at = top ? N - 1 : 1;
         if (r->bc[top][ea] == PO_BC_MIRROR) {
            FOR_WALL (r, ea, ep, eq, p, q) {
               long w = IXA (r, ea, w_at, ep, p, eq, q);
               long hin = IXA (r, ea, top ? N : 1, ep, p, eq, q);
               long hout = IXA (r, ea, top ? N + 1 : 0, ep, p, eq, q);
               r->b[ea][w] = 0;
               r->b[ep][hout] = r->b[ep][hin];
               r->b[eq][hout] = r->b[eq][hin];
               r->e[ep][w] = 0;
               r->e[eq][w] = 0;
               r->e[ea][hout] = r->e[ea][hin];
            }
         } else if (r->bc[top][ea] == PO_BC_OPEN) {
            double *buf = r->mur[top][ea];
            FOR_WALL (r, ea, ep, eq, p, q) {
               long w = IXA (r, ea, w_at, ep, p, eq, q);
               long in = IXA (r, ea, in_at, ep, p, eq, q);
               long nin = IXA (r, ea, top ? N : 1, ep, p, eq, q);
               long nout = IXA (r, ea, top ? N + 1 : 0, ep, p, eq, q);
               double *o = buf + MUR (r, ea, p, q);
               o[0] = r->e[ep][w];
               o[1] = r->e[eq][w];
               o[2] = r->e[ep][in];
               o[3] = r->e[eq][in];
               r->e[ea][nout] = r->e[ea][nin];
            }
         }
      }
   }
}

/* ------------------------------------------------------------------------
 * Laser soft source (new analytic source on the reference's one-sided
 * injection pattern, scpic/em_mirror.h:62-101 and scpic/em_mirror.c:666-717).
 * ---------------------------------------------------------------------- */
double po_laser_ey (const po_laser_t *l, double x, double y, double z,
                    double t, double ymid, double zmid)
{
   const double k = 2*M_PI, xr = M_PI*l->waist*l->waist;
   const double xi = x - l->x_focus;
   const double w = l->waist*sqrt (1 + (xi/xr)*(xi/xr));
   const double r2 = (y - ymid)*(y - ymid) + (z - zmid)*(z - zmid);
   const double tr = t - l->t_start - x;
   if (tr <= 0 || tr >= l->duration)
      return 0;
   const double s = sin (M_PI*tr/l->duration);
   const double env = s*s;
   const double phase = k*tr + atan (xi/xr) - k*r2*xi/(2*(xi*xi + xr*xr)) + l->phase;
   return 2*M_PI*l->a0*(l->waist/w)*exp (-r2/(w*w))*env*sin (phase);
}

static void laser_h (po_run_t *r, double t)
{
   const po_laser_t *l = &r->laser;
   const int I = l->plane;
   const double c1 = r->tau/r->h[0];
   const double ymid = 0.5*r->n[1]*r->h[1], zmid = 0.5*r->n[2]*r->h[2];
   const double x = (I - 1)*r->h[0];
   for (int j = l->margin ; j <= r->n[1] - l->margin ; ++j)
   for (int k = l->margin ; k <= r->n[2] - l->margin ; ++k) {
      double ey = po_laser_ey (l, x, (j - 0.5)*r->h[1], k*r->h[2], t, ymid, zmid);
      r->b[2][IX (r, I, j, k)] += c1*ey;
   }
}

static void laser_e (po_run_t *r, double t)
{
   const po_laser_t *l = &r->laser;
   const int I = l->plane;
   const double c1 = r->tau/r->h[0];
   const double ymid = 0.5*r->n[1]*r->h[1], zmid = 0.5*r->n[2]*r->h[2];
   const double x = (I - 0.5)*r->h[0];
   for (int j = l->margin ; j <= r->n[1] - l->margin ; ++j)
   for (int k = l->margin ; k <= r->n[2] - l->margin ; ++k) {
      double hz = po_laser_ey (l, x, (j - 0.5)*r->h[1], k*r->h[2], t, ymid, zmid);
      r->e[1][IX (r, I - 1, j, k)] += c1*hz;
   }
}

/* ------------------------------------------------------------------------
 * Particles.
 * ---------------------------------------------------------------------- */

/* MF_DBL_TO_INT (misc_PIC.h:18). */
static inline int dbl_to_int (double x) { return (int) (x + 128.0) - 128; }

/* One straight in-cell segment: plasmaCurrents_kernel
 * (core/plasma_currentKernel.c:21-124), 3D branch. */
static void deposit_segment (po_run_t *r, int i, int j, int k,
                             double x1, double x2, double y1, double y2,
                             double z1, double z2, double rho)
{
   const double h1 = r->h[0], h2 = r->h[1], h3 = r->h[2], tau = r->tau;
   const double dX = x2 - x1, dY = y2 - y1, dZ = z2 - z1;
   const double tX = 0.5*(x1 + x2) - i*h1;
   const double tY = 0.5*(y1 + y2) - j*h2;
   const double tZ = 0.5*(z1 + z2) - k*h3;
   const long sx = r->s[0], sy = r->s[1];
   double *Jx = r->j[0], *Jy = r->j[1], *Jz = r->j[2];
   const long o = IX (r, i, j, k);

   const double ax = rho*dX/(tau*h2*h3), dyz = dY*dZ/12;
   Jx[o + sx]          += ax*((h2 - tY)*(h3 - tZ) + dyz);
   Jx[o + sx + sy]     += ax*(tY*(h3 - tZ) - dyz);
   Jx[o + sx + 1]      += ax*((h2 - tY)*tZ - dyz);
   Jx[o + sx + sy + 1] += ax*(tY*tZ + dyz);

   const double ay = rho*dY/(tau*h1*h3), dxz = dX*dZ/12;
   Jy[o + sy]          += ay*((h1 - tX)*(h3 - tZ) + dxz);
   Jy[o + sx + sy]     += ay*(tX*(h3 - tZ) - dxz);
   Jy[o + sy + 1]      += ay*((h1 - tX)*tZ - dxz);
   Jy[o + sx + sy + 1] += ay*(tX*tZ + dxz);

   const double az = rho*dZ/(tau*h1*h2), dxy = dX*dY/12;
   Jz[o + 1]           += az*((h1 - tX)*(h2 - tY) + dxy);
   Jz[o + sx + 1]      += az*(tX*(h2 - tY) - dxy);
   Jz[o + sy + 1]      += az*((h1 - tX)*tY - dxy);
   Jz[o + sx + sy + 1] += az*(tX*tY + dxy);
}

#define SWAPI(a, b) do { int t_ = a; a = b; b = t_; } while (0)
#define SWAPD(a, b) do { double t_ = a; a = b; b = t_; } while (0)

/* plasmaCurrents_multiCellStep (core/plasma_currentKernel.c:157-279). */
static void deposit_multicell (po_run_t *r, int i1, int j1, int k1,
                               int i2, int j2, int k2,
                               double x1, double y1, double z1,
                               double x2, double y2, double z2, double rho)
{
   const double h1 = r->h[0], h2 = r->h[1], h3 = r->h[2];
   const int di = abs (i2 - i1), dj = abs (j2 - j1), dk = abs (k2 - k1);

   if (di + dj + dk == 2) {
      int i = i1, j = j1, k = k1;
      const double sX = di*((i1 + i2 + 1)*0.5*h1 - x1)/(x2 - x1 + ((1 - di) << 16));
      const double sY = dj*((j1 + j2 + 1)*0.5*h2 - y1)/(y2 - y1 + ((1 - dj) << 16));
      const double sZ = dk*((k1 + k2 + 1)*0.5*h3 - z1)/(z2 - z1 + ((1 - dk) << 16));
      double kap1 = sX + (1 - di)*sY;
      double kap2 = sZ + (1 - dk)*sY;
      int dIdx[2][3] = {{0, 0, 0}, {0, 0, 0}};
      int first = 0;
      dIdx[0][0] = di*(i2 - i1);
      dIdx[0][1] = (1 - di)*(j2 - j1);
      dIdx[1][1] = (1 - dk)*(j2 - j1);
      dIdx[1][2] = dk*(k2 - k1);
      if (kap1 > kap2) {
         SWAPD (kap1, kap2);
         first = 1;
      }
      const double xA = x1 + kap1*(x2 - x1), yA = y1 + kap1*(y2 - y1), zA = z1 + kap1*(z2 - z1);
      const double xB = x1 + kap2*(x2 - x1), yB = y1 + kap2*(y2 - y1), zB = z1 + kap2*(z2 - z1);
      deposit_segment (r, i, j, k, x1, xA, y1, yA, z1, zA, rho);
      i += dIdx[first][0];
      j += dIdx[first][1];
      k += dIdx[first][2];
      deposit_segment (r, i, j, k, xA, xB, yA, yB, zA, zB, rho);
      i += dIdx[1 - first][0];
      j += dIdx[1 - first][1];
      k += dIdx[1 - first][2];
      deposit_segment (r, i, j, k, xB, x2, yB, y2, zB, z2, rho);
      return;
   }

   const double xC = (i1 + i2 + 1)*0.5*h1, yC = (j1 + j2 + 1)*0.5*h2, zC = (k1 + k2 + 1)*0.5*h3;
   double s1 = (xC - x1)/(x2 - x1), s2 = (yC - y1)/(y2 - y1), s3 = (zC - z1)/(z2 - z1);
   double rc[3][3];
   int dI[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
   int a = 0, b = 1, c = 2, i = i1, j = j1, k = k1;
   rc[0][0] = xC;
   rc[0][1] = y1 + s1*(y2 - y1);
   rc[0][2] = z1 + s1*(z2 - z1);
   dI[0][0] = i2 - i1;
   rc[1][0] = x1 + s2*(x2 - x1);
   rc[1][1] = yC;
   rc[1][2] = z1 + s2*(z2 - z1);
   dI[1][1] = j2 - j1;
   rc[2][0] = x1 + s3*(x2 - x1);
   rc[2][1] = y1 + s3*(y2 - y1);
   rc[2][2] = zC;
   dI[2][2] = k2 - k1;
   if (s1 > s2) { SWAPI (a, b); SWAPD (s1, s2); }
   if (s1 > s3) { SWAPI (a, c); SWAPD (s1, s3); }
   if (s2 > s3) { SWAPI (b, c); SWAPD (s2, s3); }
   deposit_segment (r, i, j, k, x1, rc[a][0], y1, rc[a][1], z1, rc[a][2], rho);
   i += dI[a][0]; j += dI[a][1]; k += dI[a][2];
   deposit_segment (r, i, j, k, rc[a][0], rc[b][0], rc[a][1], rc[b][1], rc[a][2], rc[b][2], rho);
   i += dI[b][0]; j += dI[b][1]; k += dI[b][2];
   deposit_segment (r, i, j, k, rc[b][0], rc[c][0], rc[b][1], rc[c][1], rc[b][2], rc[c][2], rho);
   deposit_segment (r, i2, j2, k2, rc[c][0], x2, rc[c][1], y2, rc[c][2], z2, rho);
}

/* CIC read of one component (misc_PIC.h:72-126, 3D).  The macro expands to
 * one flat left-to-right sum of eight terms; the same order is kept. */
static inline double cic (const double *F, const po_run_t *r, int i, double sx,
                          int j, double sy, int k, double sz)
{
   const long o = IX (r, i, j, k), Sx = r->s[0], Sy = r->s[1];
   return F[o]*(1 - sx)*((1 - sy)*(1 - sz)) + F[o + Sx]*sx*((1 - sy)*(1 - sz))
        + F[o + Sy]*(1 - sx)*(sy*(1 - sz)) + F[o + Sx + Sy]*sx*(sy*(1 - sz))
        + F[o + 1]*(1 - sx)*((1 - sy)*sz) + F[o + Sx + 1]*sx*((1 - sy)*sz)
        + F[o + Sy + 1]*(1 - sx)*(sy*sz) + F[o + Sx + Sy + 1]*sx*(sy*sz);
}

/* Particle boundary conditions, faces in the reference's order
 * xMin, yMin, zMin, xMax, yMax, zMax (core/plasma_walls.c:27-104).
 * Returns 1 if the marker is removed. */
static int particle_bc (const po_run_t *r, po_marker_t *m)
{
   double *pos[3] = {&m->x, &m->y, &m->z};
   double *vel[3] = {&m->vx, &m->vy, &m->vz};
   const double L[3] = {r->n[0]*r->h[0], r->n[1]*r->h[1], r->n[2]*r->h[2]};
   for (int f = 0 ; f < 6 ; ++f) {
      const int a = f % 3, top = f / 3;
      const int bc = r->bc[top][a];
      double *x = pos[a];
      if (bc == PO_BC_PERIODIC) {
         if (!top && *x <= 0) *x += L[a];
         if (top && *x >= L[a]) *x -= L[a];
      } else if (bc == PO_BC_MIRROR) {
         if (!top && *x <= 0) { *x = -*x; *vel[a] *= -1; }
         if (top && *x >= L[a]) { *x = 2*L[a] - *x; *vel[a] *= -1; }
      } else {
         if (!top && *x <= r->h[a]) return 1;
         if (top && *x >= L[a] - r->h[a]) return 1;
      }
   }
   return 0;
}

/* plasma_timestep (core/plasma.c:95-263) over all markers; the shell/core
 * split only orders the work and is dropped. */
void po_plasma_move (po_run_t *r, double wt[3])
{
   const double h1 = r->h[0], h2 = r->h[1], h3 = r->h[2], tau = r->tau;
   const long total = (long) r->dim[0]*r->s[0];
   for (int c = 0 ; c < 3 ; ++c)
      memset (r->j[c], 0, total*sizeof (double));
   double Wx = 0, Wy = 0, Wz = 0;
   long keep = 0;
   for (long n = 0 ; n < r->np ; ++n) {
      po_marker_t *p = r->p + n;
      const double x1 = p->x, y1 = p->y, z1 = p->z;
      double sX = x1/h1, sY = y1/h2, sZ = z1/h3;
      double sX_ = sX + 0.5, sY_ = sY + 0.5, sZ_ = sZ + 0.5;
      const int i = dbl_to_int (sX), j = dbl_to_int (sY), k = dbl_to_int (sZ);
      const int i_ = dbl_to_int (sX_), j_ = dbl_to_int (sY_), k_ = dbl_to_int (sZ_);
      sX -= i; sY -= j; sZ -= k;
      sX_ -= i_; sY_ -= j_; sZ_ -= k_;

      const double Ex = cic (r->e[0], r, i_, sX_, j, sY, k, sZ);
      const double Ey = cic (r->e[1], r, i, sX, j_, sY_, k, sZ);
      const double Ez = cic (r->e[2], r, i, sX, j, sY, k_, sZ_);
      const double Hx = cic (r->b[0], r, i, sX, j_, sY_, k_, sZ_);
      const double Hy = cic (r->b[1], r, i_, sX_, j, sY, k_, sZ_);
      const double Hz = cic (r->b[2], r, i_, sX_, j_, sY_, k, sZ);

      const double tm = 0.5*tau*p->qDivM;
      const double px = p->vx + tm*Ex, py = p->vy + tm*Ey, pz = p->vz + tm*Ez;
      const double gamma = sqrt (1 + px*px + py*py + pz*pz);
      const double W = (gamma - 1.0)*p->rho/(px*px + py*py + pz*pz + 1e-19)*h1*h2*h3/p->qDivM;
      Wx += W*px*px;
      Wy += W*py*py;
      Wz += W*pz*pz;

      const double tg = tm/gamma;
      const double ax = tg*Hx, ay = tg*Hy, az = tg*Hz;
      const double u = px + py*az - pz*ay, v = py + pz*ax - px*az, w = pz + px*ay - py*ax;
      const double bxx = ax*ax, byy = ay*ay, bzz = az*az;
      const double bxy = ax*ay, byz = ay*az, bxz = az*ax;
      const double delta = 1.0/(1 + bxx + byy + bzz);
      p->vx = tm*Ex + ((1 + bxx)*u + (bxy + az)*v + (bxz - ay)*w)*delta;
      p->vy = tm*Ey + ((bxy - az)*u + (1 + byy)*v + (byz + ax)*w)*delta;
      p->vz = tm*Ez + ((bxz + ay)*u + (byz - ax)*v + (1 + bzz)*w)*delta;

      const double tgi = tau/sqrt (1 + p->vx*p->vx + p->vy*p->vy + p->vz*p->vz);
      const double x2 = p->x + p->vx*tgi, y2 = p->y + p->vy*tgi, z2 = p->z + p->vz*tgi;

      int i2 = dbl_to_int (x2/h1), j2 = dbl_to_int (y2/h2), k2 = dbl_to_int (z2/h3);
      int di = abs (i2 - i), dj = abs (j2 - j), dk = abs (k2 - k);
      if (fabs (x2 - x1) < 1e-10*h1) { di = 0; i2 = i; }
      if (fabs (y2 - y1) < 1e-10*h2) { dj = 0; j2 = j; }
      if (fabs (z2 - z1) < 1e-10*h3) { dk = 0; k2 = k; }

      if (di + dj + dk == 0) {
         deposit_segment (r, i, j, k, x1, x2, y1, y2, z1, z2, p->rho);
      } else if (di + dj + dk == 1) {
         const double alpha = dk*((k + k2 + 1)*0.5*h3 - z1)/(z2 - z1 + ((1 - dk) << 16))
                            + dj*((j + j2 + 1)*0.5*h2 - y1)/(y2 - y1 + ((1 - dj) << 16))
                            + di*((i + i2 + 1)*0.5*h1 - x1)/(x2 - x1 + ((1 - di) << 16));
         const double xC = x1 + alpha*(x2 - x1), yC = y1 + alpha*(y2 - y1), zC = z1 + alpha*(z2 - z1);
         deposit_segment (r, i, j, k, x1, xC, y1, yC, z1, zC, p->rho);
         deposit_segment (r, i2, j2, k2, xC, x2, yC, y2, zC, z2, p->rho);
      } else {
         deposit_multicell (r, i, j, k, i2, j2, k2, x1, y1, z1, x2, y2, z2, p->rho);
      }
      p->x = x2;
      p->y = y2;
      p->z = z2;
      if (!particle_bc (r, p))
         r->p[keep++] = *p;
   }
   r->np = keep;
   wt[0] = Wx;
   wt[1] = Wy;
   wt[2] = Wz;
}

/* Current boundary conditions (core/plasma_currentWalls.c:27-121); faces in
 * the order x-min, x-max, y-min, y-max, z-min, z-max; transverse extent
 * [-2, n+2]. */
void po_jbc (po_run_t *r)
{
   for (int f = 0 ; f < 6 ; ++f) {
      const int ea = f >> 1, top = f & 1;
      const int ep = (ea == 0) ? 1 : 0, eq = (ea == 2) ? 1 : 2;
      const int N = r->n[ea];
      const int bc = r->bc[top][ea];
      double *J[3] = {r->j[0], r->j[1], r->j[2]};
      if (bc == PO_BC_PERIODIC) {
         if (top)
            continue;
         const long shift = (long) N*r->s[ea];
         for (int p = -2 ; p <= r->n[ep] + 2 ; ++p)
         for (int q = -2 ; q <= r->n[eq] + 2 ; ++q)
         for (int a = -2 ; a <= 2 ; ++a) {
            long o = IXA (r, ea, a, ep, p, eq, q);
            for (int c = 0 ; c < 3 ; ++c) {
               J[c][o + shift] += J[c][o];
               J[c][o] = J[c][o + shift];
            }
         }
         continue;
      }
      const long st = r->s[ea];
      const long internal = (1 - top)*st, external = top*st;
      const long out = st*(2*top - 1);
      for (int p = -2 ; p <= r->n[ep] + 2 ; ++p)
      for (int q = -2 ; q <= r->n[eq] + 2 ; ++q) {
         const long o = IXA (r, ea, top ? N : 0, ep, p, eq, q);
         double *Ja = J[ea], *Jp = J[ep], *Jq = J[eq];
         Ja[o + internal] -= Ja[o + external];
         Jp[o - out] += Jp[o + out];
         Jq[o - out] += Jq[o + out];
         Ja[o + internal - out] -= Ja[o + external + out];
         Jp[o - 2*out] += Jp[o + 2*out];
         Jq[o - 2*out] += Jq[o + 2*out];
         Jp[o] = Jq[o] = 0;
         Ja[o + external] = Ja[o + internal];
         Jp[o + out] = -Jp[o - out];
         Jq[o + out] = -Jq[o - out];
         Ja[o + external + out] = Ja[o + internal - out];
         Jp[o + 2*out] = -Jp[o - 2*out];
         Jq[o + 2*out] = -Jq[o - 2*out];
      }
   }
}

/* em_EStep_addCurrents (core/em.c:167-184): E -= tau*J over [-1, n+1]. */
static void e_sub_current (po_run_t *r)
{
   for (int i = -1 ; i <= r->n[0] + 1 ; ++i)
   for (int j = -1 ; j <= r->n[1] + 1 ; ++j)
   for (int k = -1 ; k <= r->n[2] + 1 ; ++k) {
      long o = IX (r, i, j, k);
      for (int c = 0 ; c < 3 ; ++c)
         r->e[c][o] -= r->tau*r->j[c][o];
   }
}

/* em_energy (core/em.c:227-252). */
void po_em_energy (const po_run_t *r, double *we_out, double *wm_out)
{
   double we = 0, wb = 0;
   const long sx = r->s[0], sy = r->s[1];
   for (int i = 0 ; i < r->n[0] ; ++i)
   for (int j = 0 ; j < r->n[1] ; ++j)
   for (int k = 0 ; k < r->n[2] ; ++k) {
      long o = IX (r, i, j, k);
      double ex = r->e[0][o + sx], ey = r->e[1][o + sy], ez = r->e[2][o + 1];
      double hx = r->b[0][o + sy + 1], hy = r->b[1][o + sx + 1], hz = r->b[2][o + sx + sy];
      we += ex*ex + ey*ey + ez*ez;
      wb += hx*hx + hy*hy + hz*hz;
   }
   const double v = r->h[0]*r->h[1]*r->h[2];
   *we_out = 0.5*we*v;
   *wm_out = 0.5*wb*v;
}

/* em_HHalfStep (core/em.c:85-110): H^(n-1/2) -> H^n. */
void po_em_h_half (po_run_t *r)
{
   h_advance (r, 0.5);
   h_bc (r);
}

static void tfsf_h (po_run_t *r);
static void tfsf_e (po_run_t *r);
static void mirrors (po_run_t *r, int is_e);

/* em_HStep (core/em.c:115-131): H^n -> H^(n+1/2) plus source at t = n*tau. */
void po_em_h_step (po_run_t *r)
{
   h_advance (r, 0.5);
   tfsf_h (r);
   mirrors (r, 0);
   if (r->has_laser)
      laser_h (r, r->time);
   h_bc (r);
}

/* em_EStep_start + cap E update and boundary conditions. */
void po_em_e_step (po_run_t *r)
{
   e_advance (r);
   e_bc (r);
}

void po_set_gauss_spot (po_run_t *r, const po_gauss_spot_t *s)
{
   r->gspot = *s;
   r->has_gspot = 1;
}

/* gaussSpot_forceE (core/em_gaussSpot.c:129-156) at time t, with the
 * conversions of gaussSpot_init (:48, 70-73, 121-122): Ey and Ez set on the
 * x-plane i = (int) (x/h1 + 0.5) over j, k in [-1, n+1]. */
static void gauss_spot_e (po_run_t *r, double t)
{
   const po_gauss_spot_t *g = &r->gspot;
   const double omega = 2*M_PI*g->frequency;
   const double Ey = ((g->ey > 0) - (g->ey < 0))*g->ampl, Ez = ((g->ez > 0) - (g->ez < 0))*g->ampl;
   const int i = g->x/r->h[0] + 0.5;
   if (i < -1 || i > r->n[0] + 1)
      return;
   double timeFactor = 1;
   if (t < g->front_offset) {
      double l = (t - g->front_offset)/g->duration;
      timeFactor = exp (- l*l);
   }
   if (t > g->front_offset + g->t_plateau) {
      double l = (t - g->front_offset - g->t_plateau)/g->duration;
      timeFactor = exp (- l*l);
   }
   for (int j = -1 ; j <= r->n[1] + 1 ; j++) {
      const double dy_ = ((j - 0.5)*r->h[1] - g->y)/g->width, dy = (j*r->h[1] - g->y)/g->width;
      for (int k = -1 ; k <= r->n[2] + 1 ; k++) {
         const double dz = (k*r->h[2] - g->z)/g->width, dz_ = ((k - 0.5)*r->h[2] - g->z)/g->width;
         r->e[1][IX (r, i, j, k)] = Ey*sin (omega*t)*timeFactor*exp (- dy_*dy_ - dz*dz);
         r->e[2][IX (r, i, j, k)] = Ez*cos (omega*t)*timeFactor*exp (- dy*dy - dz_*dz_);
      }
   }
}

/* em_EStep_finish (core/em.c:189-222): TF/SF, source at t + tau/2,
 * E -= tau*J, hard gauss spot at t + tau, frame count. */
void po_em_e_finish (po_run_t *r)
{
   tfsf_e (r);
   mirrors (r, 1);
   if (r->has_laser)
      laser_e (r, r->time + 0.5*r->tau);
   e_sub_current (r);
   if (r->has_gspot)
      gauss_spot_e (r, r->time + r->tau);
   r->tfsf_frame++;                                            /* :849-853 */
}

/* ------------------------------------------------------------------------
 * TF/SF interface (core/em_TFSF.c:480-851).
 * ---------------------------------------------------------------------- */

/* TFSF_init (:480-558) face geometry; record mode cuts the faces to the
 * domain (TFSF_turnRec :239-252: E faces to [0, n-1], H faces to [1, n]),
 * play mode drops the open faces (TFSF_openFaces :296-323) and requires the
 * rest 5 cells inside the walls (TFSF_turnPlay :341-357). */
int po_set_tfsf (po_run_t *r, const po_tfsf_t *t, const double *frames)
{
   r->tfsf = *t;
   r->frame_size = 0;
   const int *side[2] = {t->lo, t->hi};
   for (int a = 0 ; a < 3 ; ++a) {
      const int ep = (a + 1) % 3, eq = (a + 2) % 3;
      for (int top = 0 ; top < 2 ; ++top)
         for (int comp = 0 ; comp < 2 ; ++comp) {
            const int f = 4*a + 2*top + comp;
            for (int fh = 0 ; fh < 2 ; ++fh) {
               const int q = f + 12*fh;
               for (int b = 0 ; b < 3 ; ++b) {
                  r->face[q].min[b] = t->lo[b];
                  r->face[q].max[b] = t->hi[b];
               }
               r->face[q].min[a] = r->face[q].max[a] = side[top][a];
               const int ce = (a + 1 + comp) % 3;
               r->face[q].min[ce] += 1;
               if (fh) {
                  r->face[q].min[a] += top;
                  r->face[q].max[a] += top;
               }
               r->face[q].comp = fh ? 3 - ce - a : ce;
               r->face[q].ep = ep;
               r->face[q].eq = eq;
               r->face[q].sf = (1 - 2*top)*(1 - 2*comp)*(r->tau/r->h[a]);
               if (t->mode == PO_TFSF_REC)
                  for (int b = 0 ; b < 3 ; ++b) {
                     const int lo = fh ? 1 : 0, hi = fh ? r->n[b] : r->n[b] - 1;
                     if (r->face[q].min[b] < lo) r->face[q].min[b] = lo;
                     if (r->face[q].max[b] > hi) r->face[q].max[b] = hi;
                  }
               long v = 1;
               for (int b = 0 ; b < 3 ; ++b)
                  v *= (r->face[q].max[b] >= r->face[q].min[b]) ? r->face[q].max[b] - r->face[q].min[b] + 1 : 0;
               r->face[q].vol = v;
               /* An open face keeps its slot in the frame layout of the
                * recorded files; only its use is dropped. */
               r->face[q].used = v > 0 && !(t->mode != PO_TFSF_REC && t->open[top][a]);
               if (r->face[q].used && t->mode != PO_TFSF_REC)
                  for (int b = 0 ; b < 3 ; ++b)
                     if (r->face[q].min[b] < 5 || r->face[q].max[b] > r->n[b] - 5)
                        return -1;
            }
         }
   }
   for (int q = 0 ; q < 24 ; ++q) {
      r->face[q].at = r->frame_size;
      r->frame_size += r->face[q].vol;
   }
   free (r->frames);
   r->frames = NULL;
   if (t->mode != PO_TFSF_REC) {
      r->frames = (double *) malloc (sizeof (double)*(size_t) r->frame_size*(t->frames > 0 ? t->frames : 1));
      memcpy (r->frames, frames, sizeof (double)*(size_t) r->frame_size*t->frames);
   }
   r->tfsf_frame = (int) (r->time/r->tau + 0.1);              /* :455 */
   r->tfsf_on = 1;
   r->has_tfsf = 1;
   r->nrec = 0;
   return 0;
}

long po_tfsf_faces (const po_run_t *r, int *regions)
{
   for (int q = 0 ; q < 24 && regions ; ++q)
      for (int b = 0 ; b < 3 ; ++b) {
         regions[6*q + b] = r->face[q].min[b];
         regions[6*q + 3 + b] = r->face[q].max[b];
      }
   return r->frame_size;
}

long po_tfsf_recorded (const po_run_t *r, double *out)
{
   if (out && r->nrec)
      memcpy (out, r->rec, sizeof (double)*(size_t) r->nrec*r->frame_size);
   return r->nrec;
}

static int tfsf_playing (const po_run_t *r)
{
   return r->has_tfsf && r->tfsf_on && r->tfsf.mode != PO_TFSF_REC;
}

/* Start of a step (em_HHalfStep, core/em.c:85-105).  Record: TFSF_writeMesh
 * (:565-594) of E^n and H^(n-1/2).  Play: the cap caching of the half step
 * already calls TFSF_postEStep on the boundary slabs (core/em_caps.c:602-608),
 * which switches the interface off for good once frame n + 1 is the last
 * (:831-834) -- before this step's H and E faces are touched. */
static void tfsf_record (po_run_t *r)
{
   if (tfsf_playing (r) && r->tfsf_frame + 1 >= r->tfsf.frames - 1)
      r->tfsf_on = 0;
   if (!r->has_tfsf || r->tfsf.mode != PO_TFSF_REC)
      return;
   r->rec = (double *) realloc (r->rec, sizeof (double)*(size_t) (r->nrec + 1)*r->frame_size);
   double *o = r->rec + r->nrec*r->frame_size;
   for (int q = 0 ; q < 24 ; ++q) {
      if (!r->face[q].used)
         continue;
      const double *F = q < 12 ? r->e[r->face[q].comp] : r->b[r->face[q].comp];
      const int ep = r->face[q].ep, eq = r->face[q].eq;
      int c[3] = {r->face[q].min[0], r->face[q].min[1], r->face[q].min[2]};
      for (c[ep] = r->face[q].min[ep] ; c[ep] <= r->face[q].max[ep] ; ++c[ep])
         for (c[eq] = r->face[q].min[eq] ; c[eq] <= r->face[q].max[eq] ; ++c[eq])
            *o++ = F[IX (r, c[0], c[1], c[2])]*r->face[q].sf;
   }
   r->nrec++;
}

/* TFSF_addSource / TFSF_subSource (:669-781) of frame fr's recorded values
 * of the other field onto faces [q0, q0 + 12). */
static void tfsf_apply (po_run_t *r, int q0, int fr, double sign)
{
   for (int q = q0 ; q < q0 + 12 ; ++q) {
      if (!r->face[q].used)
         continue;
      double *F = q < 12 ? r->e[r->face[q].comp] : r->b[r->face[q].comp];
      const double *src = r->frames + (long) fr*r->frame_size + r->face[(q + 12) % 24].at;
      const int ep = r->face[q].ep, eq = r->face[q].eq;
      int c[3] = {r->face[q].min[0], r->face[q].min[1], r->face[q].min[2]};
      for (c[ep] = r->face[q].min[ep] ; c[ep] <= r->face[q].max[ep] ; ++c[ep])
         for (c[eq] = r->face[q].min[eq] ; c[eq] <= r->face[q].max[eq] ; ++c[eq], ++src) {
            if (sign > 0)
               F[IX (r, c[0], c[1], c[2])] += *src;
            else
               F[IX (r, c[0], c[1], c[2])] -= *src;
         }
   }
}

/* TFSF_postHStep (:805-819): H faces get the recorded E of frame n
 * (backward: T - n). */
static void tfsf_h (po_run_t *r)
{
   const int tf = r->tfsf_frame, last = r->tfsf.frames;
   if (!tfsf_playing (r) || tf >= last - 1)
      return;
   tfsf_apply (r, 12, r->tfsf.mode == PO_TFSF_PLAY ? tf : last - 1 - tf, 1.0);
}

/* TFSF_postEStep (:825-844): E faces get the recorded H of frame n + 1
 * (backward: T - n, subtracted). */
static void tfsf_e (po_run_t *r)
{
   const int tf = r->tfsf_frame, last = r->tfsf.frames;
   if (!tfsf_playing (r))
      return;
   if (tf + 1 >= last - 1) {
      r->tfsf_on = 0;
      return;
   }
   if (r->tfsf.mode == PO_TFSF_PLAY)
      tfsf_apply (r, 0, tf + 1, 1.0);
   else
      tfsf_apply (r, 0, last - 1 - tf, -1.0);
}

/* ------------------------------------------------------------------------
 * Focused-laser soft sources (scpic/em_mirror.c:292-332, 667-717).
 * ---------------------------------------------------------------------- */

/* read_mirror_parameters (:292-332) for the values the play needs.  The
 * backward delay subtracts the focus from the cell count n0, not from the
 * domain length, as the reference does (:330). */
void po_add_mirror (po_run_t *r, const double v[9], int direction, double r0, double t0,
                    const double *E, const double *H)
{
   if (r->nmirror >= 8)
      return;
   const double pi = 3.141592653589793238462643;
   const double e = 4.8032e-10, c = 2.9979e+10, m = 9.1094e-28, wpc = 1e7;   /* misc_units.h:34-38 */
   double A = v[0];
   if (A > 0)
      A = r0*e*sqrt (8*pi*A*wpc/c)/(m*c*c);
   else
      A *= (-2*pi);
   const double xf = v[2]*1e-4/r0;
   double dt = v[5]*1e-15/t0;
   const double T0 = v[6]*1e-15/t0;
   dt *= sqrt (2.0/log (2));
   const int q = r->nmirror++;
   r->mirror[q].A = A;
   r->mirror[q].dt = dt;
   r->mirror[q].T0 = T0;
   r->mirror[q].phi0 = v[7];
   r->mirror[q].forward = direction > 0;
   r->mirror[q].delay = r->mirror[q].forward ? xf - 5*r->h[0] : r->n[0] - 5*r->h[0] - xf;
   const long nodes = (long) (r->n[1] - 9)*(r->n[2] - 9)*4;
   r->mirror[q].E = (double *) malloc (sizeof (double)*nodes);
   r->mirror[q].H = (double *) malloc (sizeof (double)*nodes);
   memcpy (r->mirror[q].E, E, sizeof (double)*nodes);
   memcpy (r->mirror[q].H, H, sizeof (double)*nodes);
}

/* add_mirror_H / add_mirror_E with add_source: the H plane i = 5 (backward
 * n0 - 4) gets the E profile at t, the E plane i = 4 (backward n0 - 4) the
 * H profile at t + tau/2, over j, k in [5, n - 5]:
 *   Fy += a (z_cos cos p + z_sin sin p), Fz += a (y_cos cos p + y_sin sin p),
 *   a = exp (-(2 t'/dt)^2) tau/h1, p = 2 pi t' + phi0, t' = t - T0 + delay. */
static void mirrors (po_run_t *r, int is_e)
{
   const double pi = 3.141592653589793238462643;
   for (int q = 0 ; q < r->nmirror ; ++q) {
      const double t = r->time + (is_e ? 0.5*r->tau : 0.0) - r->mirror[q].T0 + r->mirror[q].delay;
      const double ampl = exp (-pow (2*t/r->mirror[q].dt, 2));
      const int I = r->mirror[q].forward ? (is_e ? 4 : 5) : r->n[0] - 5 + 1;
      const double cs = cos (2*pi*t + r->mirror[q].phi0), sn = sin (2*pi*t + r->mirror[q].phi0);
      const double A = ampl*r->tau/r->h[0];
      const double *src = is_e ? r->mirror[q].H : r->mirror[q].E;
      double *Fy = is_e ? r->e[1] : r->b[1], *Fz = is_e ? r->e[2] : r->b[2];
      const int nk = r->n[2] - 9;
      for (int j = 5 ; j <= r->n[1] - 5 ; ++j)
         for (int k = 5 ; k <= r->n[2] - 5 ; ++k) {
            const double *w = src + 4*((long) (j - 5)*nk + (k - 5));
            Fy[IX (r, I, j, k)] += A*(w[2]*cs + w[3]*sn);
            Fz[IX (r, I, j, k)] += A*(w[0]*cs + w[1]*sn);
         }
   }
}

/* One step in core/main.c:353-478 order. */
int po_step (po_run_t *r, double out[5])
{
   double we, wm, wt[3];
   tfsf_record (r);
   po_em_h_half (r);
   po_em_energy (r, &we, &wm);
   po_plasma_move (r, wt);
   po_em_h_step (r);
   po_em_e_step (r);
   po_jbc (r);
   po_em_e_finish (r);
   r->time += r->tau;
   if (out) {
      out[0] = we;
      out[1] = wm;
      out[2] = wt[0];
      out[3] = wt[1];
      out[4] = wt[2];
   }
   return 0;
}

/* probe_postData (core/diag_probe.c:409-429): E^n and H^n at the node, E
 * averaged over its two edges along the component, H over the four faces
 * around the node's edge; the time is the step's t = n tau. */
static void probes (const po_run_t *r, const int *ijk, int n, double *o)
{
   const long Sx = r->s[0], Sy = r->s[1];
   for (int q = 0 ; q < n ; ++q, o += 7) {
      const long p = IX (r, ijk[3*q], ijk[3*q + 1], ijk[3*q + 2]);
      const double *const *E = (const double *const *) r->e, *const *H = (const double *const *) r->b;
      o[0] = r->time;
      o[1] = 0.5*(E[0][p] + E[0][p + Sx]);
      o[2] = 0.5*(E[1][p] + E[1][p + Sy]);
      o[3] = 0.5*(E[2][p] + E[2][p + 1]);
      o[4] = 0.25*(H[0][p] + H[0][p + Sy] + H[0][p + 1] + H[0][p + Sy + 1]);
      o[5] = 0.25*(H[1][p] + H[1][p + Sx] + H[1][p + 1] + H[1][p + Sx + 1]);
      o[6] = 0.25*(H[2][p] + H[2][p + Sx] + H[2][p + Sy] + H[2][p + Sx + Sy]);
   }
}

/* E^n and H^n of the coming step over [0, n]^3 (what spectr_dump writes,
 * core/main.c:395-402): H^n from a half step on a copy of H^(n-1/2). */
void po_fields_n (po_run_t *r, double *E, double *H)
{
   const long size = po_mesh_size (r);
   double *keep[3];
   for (int c = 0 ; c < 3 ; ++c) {
      keep[c] = (double *) malloc (sizeof (double)*size);
      memcpy (keep[c], r->b[c], sizeof (double)*size);
   }
   po_em_h_half (r);
   po_get_fields (r, E, H);
   for (int c = 0 ; c < 3 ; ++c) {
      memcpy (r->b[c], keep[c], sizeof (double)*size);
      free (keep[c]);
   }
}

int po_step_probes (po_run_t *r, const int *ijk, int n, double *samples, double out[5])
{
   double we, wm, wt[3];
   tfsf_record (r);
   po_em_h_half (r);
   po_em_energy (r, &we, &wm);
   probes (r, ijk, n, samples);
   po_plasma_move (r, wt);
   po_em_h_step (r);
   po_em_e_step (r);
   po_jbc (r);
   po_em_e_finish (r);
   r->time += r->tau;
   if (out) {
      out[0] = we;
      out[1] = wm;
      out[2] = wt[0];
      out[3] = wt[1];
      out[4] = wt[2];
   }
   return 0;
}

/* CIC charge density: core/plasma_rho.c:23-60 restated (no folding). */
/* Charge density: CIC deposit (plasma.c:322-329 calling plasmaRho_add,
 * plasma_rho.c:159-173, with the nested weights of mf_PIC_distribute,
 * misc_PIC.h:164-195: node (i+a, j+b, k+c) gets wx_a*(wy_b*(wz_c*rho)), nodes in
 * the macro's order), then the walls of plasmaRho_applyBoundary
 * (plasma_rho.c:23-97) in the order x, y, z, lower then upper:
 *   periodic (at the lower wall only): for the 5 layers a = -2..2,
 *     rho[a + n] += rho[a]; rho[a] = rho[a + n];
 *   mirror / open: with the wall node w and the outward step o,
 *     rho[w - o] += rho[w + o]; rho[w - 2o] += rho[w + 2o]; rho[w] = 0;
 *     rho[w + o] = -rho[w - o]; rho[w + 2o] = -rho[w - 2o];
 * over the wall plane's nodes [-2, n+2] in the two other axes.  The VSP
 * filter (plasma_VSP.c:32) is off at its default alpha = 1. */
static void rho_add (double *rho, long o, long Sx, long Sy, double sx, double sy, double sz, double v)
{
   const double z0 = (1 - sz)*v, z1 = sz*v;
   const double y00 = (1 - sy)*z0, y10 = sy*z0, y01 = (1 - sy)*z1, y11 = sy*z1;
   rho[o]               += (1 - sx)*y00;
   rho[o + Sx]          += sx*y00;
   rho[o + Sy]          += (1 - sx)*y10;
   rho[o + Sx + Sy]     += sx*y10;
   rho[o + 1]           += (1 - sx)*y01;
   rho[o + Sx + 1]      += sx*y01;
   rho[o + Sy + 1]      += (1 - sx)*y11;
   rho[o + Sx + Sy + 1] += sx*y11;
}

void po_rho (const po_run_t *r, double *rho)
{
   memset (rho, 0, sizeof (double)*(long) r->dim[0]*r->dim[1]*r->dim[2]);
   for (long n = 0 ; n < r->np ; ++n) {
      const po_marker_t *p = r->p + n;
      double sx = p->x/r->h[0], sy = p->y/r->h[1], sz = p->z/r->h[2];
      int i = dbl_to_int (sx), j = dbl_to_int (sy), k = dbl_to_int (sz);
      sx -= i; sy -= j; sz -= k;
      rho_add (rho, IX (r, i, j, k), r->s[0], r->s[1], sx, sy, sz, p->rho);
   }
   static const int axes[3][3] = {{0, 1, 2}, {1, 0, 2}, {2, 0, 1}};
   for (int b = 0 ; b < 6 ; ++b) {
      const int ea = axes[b/2][0], ep = axes[b/2][1], eq = axes[b/2][2], top = b & 1;
      const int bc = r->bc[top][ea], n = r->n[ea];
      for (int p = -2 ; p <= r->n[ep] + 2 ; ++p)
         for (int q = -2 ; q <= r->n[eq] + 2 ; ++q) {
            if (bc == PO_BC_PERIODIC) {
               if (top)
                  continue;
               for (int a = -2 ; a <= 2 ; ++a) {
                  const long lo = IXA (r, ea, a, ep, p, eq, q), hi = IXA (r, ea, a + n, ep, p, eq, q);
                  rho[hi] += rho[lo];
                  rho[lo] = rho[hi];
               }
            } else {
               const int w = top ? n : 0, o = top ? 1 : -1;
               const long in1 = IXA (r, ea, w - o, ep, p, eq, q), out1 = IXA (r, ea, w + o, ep, p, eq, q);
               const long in2 = IXA (r, ea, w - 2*o, ep, p, eq, q), out2 = IXA (r, ea, w + 2*o, ep, p, eq, q);
               rho[in1] += rho[out1];
               rho[in2] += rho[out2];
               rho[IXA (r, ea, w, ep, p, eq, q)] = 0;
               rho[out1] = -rho[in1];
               rho[out2] = -rho[in2];
            }
         }
   }
}

/* Gauss-law test (plasma_gaussTest.c:110-149): over nodes [0, n]^3 the
 * largest |(rho2 - rho1)/tau + div J| and |div E - rho2|, with the run's J
 * (after the current walls) and E (after the E step). */
void po_gauss (const po_run_t *r, const double *rho1, const double *rho2, double out[2])
{
   double d0 = -1, d1 = -1;
   const long Sx = r->s[0], Sy = r->s[1];
   for (int i = 0 ; i <= r->n[0] ; ++i)
      for (int j = 0 ; j <= r->n[1] ; ++j)
         for (int k = 0 ; k <= r->n[2] ; ++k) {
            const long o = IX (r, i, j, k);
            const double t0 = (rho2[o] - rho1[o])/r->tau +
                              (r->j[0][o + Sx] - r->j[0][o])/r->h[0] +
                              (r->j[1][o + Sy] - r->j[1][o])/r->h[1] +
                              (r->j[2][o + 1] - r->j[2][o])/r->h[2];
            const double t1 = (r->e[0][o + Sx] - r->e[0][o])/r->h[0] +
                              (r->e[1][o + Sy] - r->e[1][o])/r->h[1] +
                              (r->e[2][o + 1] - r->e[2][o])/r->h[2] -
                              rho2[o];
            d0 = (fabs (t0) > d0) ? fabs (t0) : d0;
            d1 = (fabs (t1) > d1) ? fabs (t1) : d1;
         }
   out[0] = d0;
   out[1] = d1;
}

long po_mesh_size (const po_run_t *r)
{
   return (long) r->dim[0]*r->dim[1]*r->dim[2];
}

/* Copies the region [-2, n+2]^3 of an internal mesh to out (k fastest). */
void po_region (const po_run_t *r, const double *mesh, double *out)
{
   long q = 0;
   for (int i = -G ; i <= r->n[0] + G ; ++i)
      for (int j = -G ; j <= r->n[1] + G ; ++j)
         for (int k = -G ; k <= r->n[2] + G ; ++k)
            out[q++] = mesh[IX (r, i, j, k)];
}

/* ------------------------------------------------------------------------
 * ranmar: misc_ranmar.c:79-146 restated (Marsaglia & Zaman, FSU-SCRI-87-50,
 * as modified by F. James).
 * ---------------------------------------------------------------------- */
void po_ranmar_init (po_ranmar_t *g, int ij, int kl)
{
   int i = (ij/177)%177 + 2, j = ij%177 + 2, k = (kl/169)%178 + 1, l = kl%169;
   for (int ii = 0 ; ii < 97 ; ii++) {
      double s = 0, t = 0.5;
      for (int jj = 0 ; jj < 24 ; jj++) {
         int m = (((i*j)%179)*k)%179;
         i = j;
         j = k;
         k = m;
         l = (53*l + 1)%169;
         if ((l*m)%64 >= 32)
            s += t;
         t *= 0.5;
      }
      g->u[ii] = s;
   }
   g->c  = 362436.0/16777216.0;
   g->cd = 7654321.0/16777216.0;
   g->cm = 16777213.0/16777216.0;
   g->i97 = 96;
   g->j97 = 32;
}

void po_ranmar (po_ranmar_t *g, double *out, long n)
{
   for (long v = 0 ; v < n ; v++) {
      double uni = g->u[g->i97] - g->u[g->j97];
      if (uni < 0.0) uni += 1.0;
      g->u[g->i97] = uni;
      g->i97 = (g->i97 + 96)%97;
      g->j97 = (g->j97 + 96)%97;
      g->c -= g->cd;
      if (g->c < 0.0) g->c += g->cm;
      uni -= g->c;
      if (uni < 0.0) uni += 1.0;
      out[v] = uni;
   }
}

/* The placer's Box-Muller transform (the rule of mg_place_t): its own
 * logarithm and sine/cosine from IEEE +, -, *, /, sqrt only, restated here
 * in the same operation order as the device's, so the momenta agree to
 * the bit.  log v: v = m 2^e, m in [sqrt(1/2), sqrt(2)), log v =
 * e ln2 + 2 s (1 + s^2/3 + ... + s^24/25), s = (m-1)/(m+1); (cos, sin) of
 * 2 pi u: quadrant q = floor(4u), f = 4u - q, angle (pi/2) min(f, 1-f) in
 * [0, pi/4], Taylor series of sin (to t^17) and cos (to t^18), then the
 * complementary swap and the quadrant rotation. */
static double po_log (double v)
{
   int e = 0;
   double m = frexp (v, &e);
   if (m < 0x1.6a09e667f3bcdp-1) {
      m = m*2.0;
      e = e - 1;
   }
   const double s = (m - 1.0)/(m + 1.0);
   const double z = s*s;
   static const double c[12] = {
      0x1.642c8590b2164p-5, 0x1.8618618618618p-5, 0x1.af286bca1af28p-5, 0x1.e1e1e1e1e1e1ep-5,
      0x1.1111111111111p-4, 0x1.3b13b13b13b14p-4, 0x1.745d1745d1746p-4, 0x1.c71c71c71c71cp-4,
      0x1.2492492492492p-3, 0x1.999999999999ap-3, 0x1.5555555555555p-2, 1.0};
   double p = 0x1.47ae147ae147bp-5;
   for (int q = 0 ; q < 12 ; ++q)
      p = p*z + c[q];
   const double de = (double) e;
   return de*0x1.62e42fee00000p-1 + (de*0x1.a39ef35793c76p-33 + 2.0*s*p);
}

static void po_sincos_2pi (double u, double *sn, double *cs)
{
   const double x = 4.0*u;
   const double q = floor (x);
   double f = x - q;
   const int swap = f > 0.5;
   if (swap)
      f = 1.0 - f;
   const double t = f*0x1.921fb54442d18p+0;
   const double z = t*t;
   static const double cs_[8] = {
      -0x1.ae7f3e733b81fp-41, 0x1.6124613a86d09p-33, -0x1.ae64567f544e4p-26, 0x1.71de3a556c734p-19,
      -0x1.a01a01a01a01ap-13, 0x1.1111111111111p-7, -0x1.5555555555555p-3, 1.0};
   static const double cc_[9] = {
      0x1.ae7f3e733b81fp-45, -0x1.93974a8c07c9dp-37, 0x1.1eed8eff8d898p-29, -0x1.27e4fb7789f5cp-22,
      0x1.a01a01a01a01ap-16, -0x1.6c16c16c16c17p-10, 0x1.5555555555555p-5, -0.5, 1.0};
   double ps = 0x1.952c77030ad4ap-49, pc = -0x1.6827863b97d97p-53;
   for (int k = 0 ; k < 8 ; ++k)
      ps = ps*z + cs_[k];
   for (int k = 0 ; k < 9 ; ++k)
      pc = pc*z + cc_[k];
   const double st = t*ps;
   const double s0 = swap ? pc : st, c0 = swap ? st : pc;
   switch ((int) q) {
   case 0:  *sn = s0;  *cs = c0;  break;
   case 1:  *sn = c0;  *cs = -s0; break;
   case 2:  *sn = -s0; *cs = -c0; break;
   default: *sn = -c0; *cs = s0;  break;
   }
}

static void po_box_muller (double u_r, double u_t, double *a, double *b)
{
   const double r = sqrt (-2.0*po_log (1.0 - u_r));
   double sn, cs;
   po_sincos_2pi (u_t, &sn, &cs);
   *a = r*cs;
   *b = r*sn;
}

long po_place_count (const po_place_t *s)
{
   long cells = 1;
   for (int a = 0 ; a < 3 ; ++a)
      cells *= (s->hi[a] > s->lo[a]) ? (s->hi[a] - s->lo[a]) : 0;
   return cells*s->ppc;
}

long po_place (const po_place_t *s, const double h[3], po_marker_t *out)
{
   po_ranmar_t g;
   po_ranmar_init (&g, s->seed_ij, s->seed_kl);
   double d[7];
   for (long k = s->skip ; k > 0 ; ) {
      long c = (k > 7) ? 7 : k;
      po_ranmar (&g, d, c);
      k -= c;
   }
   long n = 0;
   for (int i = s->lo[0] ; i < s->hi[0] ; ++i)
   for (int j = s->lo[1] ; j < s->hi[1] ; ++j)
   for (int k = s->lo[2] ; k < s->hi[2] ; ++k)
   for (int q = 0 ; q < s->ppc ; ++q, ++n) {
      po_ranmar (&g, d, 7);
      po_marker_t *m = out + n;
      m->x = (i + d[0])*h[0];
      m->y = (j + d[1])*h[1];
      m->z = (k + d[2])*h[2];
      double gx, gy, gz, gw;
      po_box_muller (d[3], d[4], &gx, &gy);
      po_box_muller (d[5], d[6], &gz, &gw);
      m->vx = s->drift[0] + s->uth[0]*gx;
      m->vy = s->drift[1] + s->uth[1]*gy;
      m->vz = s->drift[2] + s->uth[2]*gz;
      m->rho = (float) s->rho;
      m->qDivM = (float) s->qDivM;
      m->id = s->id0 + (int) n;
      m->pad_ = 0;
   }
   return n;
}
