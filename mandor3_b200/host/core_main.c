/* core_b200.out -- drop-in replacement for the reference's core.out.
 *
 * Run it in a Mandor run directory prepared by the reference's setup.out:
 * it reads the same inputs (run_mandor.cfg, binData/domain.bin, the last or
 * the first checkpoint record, tmp/stop.flag) and writes the same outputs
 * (checkpoint records, binData/diag.dat), so the reference's tools read its
 * results unchanged.  The time stepping runs on one B200 through the C ABI
 * of include/mandor_b200.h.
 *
 * Files and their reference writers/readers:
 *   run_mandor.cfg             core/main.c:205-213 (six "@ int" lines)
 *   binData/domain.bin         misc_parameters.c:98-131
 *   binData/sys.N, sys_%06d.txt, sys_E/H_%06d(000).bin, sys_prtn_%06d.bin
 *                              IO_sys.c:99-142, type_mesh.c:285-313
 *   binData/fileMap*.txt/.N    IO_fileMap.c:129-157
 *   binData/plasma_%06d_000.bin  core/plasma_IO.c:273-287
 *   binData/diag.dat           core/diag_WDensity.c:30-157
 *   tmp/stop.flag              core/main.c:120-189
 *   binData/tec_*, tecplot.N   IO_tecplot.c:108-266
 *   run_probes.cfg, binData/probe_*.bin, output/probe_locations.dat
 *                              core/diag_probe.c:48-446, probe.h
 *   tmp/spectrDump_%d_0, binData/spectr.N
 *                              spectr_dump.c:15-109, type_CFile.c:112-370
 *   .EM_sources/TFSF/TFSF.cfg, openFaces.cfg, consistencyCheck.dat,
 *   lastFrameTime.bin, TFSF_defrag.map, <face>_000.bin / <face>_99999.bin
 *                              core/em_TFSF.c:143-460, 565-594, 855-891
 *
 *   core_b200.out [--fp32] [--device N]
 */
#include <dirent.h>
#include <errno.h>
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include "mandor_b200.h"

#define HEADER_BYTES 112            /* 6 ints of valid region + 88-byte mesh_t */

/* Errors end the run like the reference's DIE (log.h:44-62), with a
 * non-zero status that names the kind: -MG_ERR_IO (7) for a missing,
 * truncated or malformed input file, -rc for a failed library call. */
static void die (const char *fmt, const char *arg)
{
   fprintf (stderr, "core_b200.out: ");
   fprintf (stderr, fmt, arg);
   fprintf (stderr, "\n");
   exit (-MG_ERR_IO);
}

static void check (int rc, const char *what)
{
   if (rc != MG_OK) {
      fprintf (stderr, "core_b200.out: %s: %s\n", what, mg_last_error ());
      exit (rc < 0 && rc > -128 ? -rc : EXIT_FAILURE);
   }
}

static double now (void)
{
   struct timespec ts;
   clock_gettime (CLOCK_MONOTONIC, &ts);
   return ts.tv_sec + 1e-9*ts.tv_nsec;
}

static FILE *open_or_die (const char *path, const char *mode)
{
   FILE *fp = fopen (path, mode);
   if (!fp)
      die ("cannot open '%s'", path);
   return fp;
}

/* "@ value ..." lines, as cfg_readInt reads them (misc_cfgReader.c:71-81). */
static int read_at_int (FILE *fp, const char *path)
{
   int c, v;
   while ((c = fgetc (fp)) != EOF && c != '@')
      ;
   if (c == EOF || fscanf (fp, "%d", &v) != 1)
      die ("bad integer line in '%s'", path);
   while ((c = fgetc (fp)) != EOF && c != '\n')
      ;
   return v;
}

static double read_at_double (FILE *fp, const char *path)
{
   int c;
   double v;
   while ((c = fgetc (fp)) != EOF && c != '@')
      ;
   if (c == EOF || fscanf (fp, "%lf", &v) != 1)
      die ("bad number line in '%s'", path);
   while ((c = fgetc (fp)) != EOF && c != '\n')
      ;
   return v;
}

static void read_exact (void *p, size_t n, FILE *fp, const char *path)
{
   if (fread (p, 1, n, fp) != n)
      die ("'%s' is truncated", path);
}

static void write_exact (const void *p, size_t n, FILE *fp, const char *path)
{
   if (fwrite (p, 1, n, fp) != n)
      die ("cannot write '%s'", path);
}

typedef struct {
   int    total, full, tecplot, cont, stop, spectr;
} run_cfg_t;

typedef struct {
   double h[3], L[3], tau;
   int    dmin[3], dmax[3], bcmin[3], bcmax[3];
} domain_t;

static domain_t read_domain (void)
{
   domain_t d;
   const char *path = "binData/domain.bin";
   FILE *fp = open_or_die (path, "rb");
   double v[7];
   int iv[12];
   read_exact (v, sizeof (v), fp, path);
   read_exact (iv, sizeof (iv), fp, path);
   fclose (fp);
   for (int a = 0 ; a < 3 ; ++a) {
      d.h[a] = v[a];
      d.L[a] = v[3 + a];
      d.dmin[a] = iv[a];
      d.dmax[a] = iv[3 + a];
      d.bcmin[a] = iv[6 + a];
      d.bcmax[a] = iv[9 + a];
   }
   d.tau = v[6];
   return d;
}

static void write_domain (const domain_t *d)
{
   const char *path = "binData/domain.bin";
   FILE *fp = open_or_die (path, "wb");
   double v[7] = {d->h[0], d->h[1], d->h[2], d->L[0], d->L[1], d->L[2], d->tau};
   int iv[12];
   for (int a = 0 ; a < 3 ; ++a) {
      iv[a] = d->dmin[a];
      iv[3 + a] = d->dmax[a];
      iv[6 + a] = d->bcmin[a];
      iv[9 + a] = d->bcmax[a];
   }
   write_exact (v, sizeof (v), fp, path);
   write_exact (iv, sizeof (iv), fp, path);
   fclose (fp);
}

/* Mesh file: region, the mesh_t struct, nodes of the region (k fastest). */
static double *read_mesh (const char *path, unsigned char header[HEADER_BYTES], long nodes)
{
   FILE *fp = open_or_die (path, "rb");
   read_exact (header, HEADER_BYTES, fp, path);
   int reg[6];
   memcpy (reg, header, sizeof (reg));
   const long n = (long) (reg[3] - reg[0] + 1)*(reg[4] - reg[1] + 1)*(reg[5] - reg[2] + 1);
   if (n != nodes || reg[0] || reg[1] || reg[2])
      die ("'%s': region does not match the domain", path);
   double *data = (double *) malloc (sizeof (double)*3*n);
   read_exact (data, sizeof (double)*3*n, fp, path);
   fclose (fp);
   return data;
}

static void write_mesh (const char *path, const unsigned char header[HEADER_BYTES], const double *data,
                        long nodes)
{
   FILE *fp = open_or_die (path, "wb");
   write_exact (header, HEADER_BYTES, fp, path);
   write_exact (data, sizeof (double)*3*nodes, fp, path);
   fclose (fp);
}

static mg_marker_t *read_markers (const char *path, long long *n)
{
   FILE *fp = open_or_die (path, "rb");
   long count = 0;
   read_exact (&count, sizeof (long), fp, path);
   if (count < 0)
      die ("'%s': negative marker count", path);
   mg_marker_t *m = (mg_marker_t *) malloc (sizeof (mg_marker_t)*(count > 0 ? count : 1));
   if (count > 0)
      read_exact (m, sizeof (mg_marker_t)*count, fp, path);
   fclose (fp);
   *n = count;
   return m;
}

static void write_markers (const char *path, const mg_marker_t *m, long long n)
{
   FILE *fp = open_or_die (path, "wb");
   long count = (long) n;
   write_exact (&count, sizeof (long), fp, path);
   if (n > 0)
      write_exact (m, sizeof (mg_marker_t)*n, fp, path);
   fclose (fp);
}

static void copy_file (const char *from, const char *to)
{
   FILE *in = fopen (from, "rb");
   if (!in)
      return;
   FILE *out = open_or_die (to, "wb");
   char buf[1 << 16];
   size_t k;
   while ((k = fread (buf, 1, sizeof (buf), in)) > 0)
      write_exact (buf, k, out, to);
   fclose (in);
   fclose (out);
}

static int read_count (const char *path)
{
   FILE *fp = fopen (path, "rt");
   if (!fp)
      return 0;
   int v = read_at_int (fp, path);
   fclose (fp);
   return v;
}

/* Energy rows are kept until the next checkpoint, then appended to diag.dat
 * the way wDensity_finalize does (core/diag_WDensity.c:82-104). */
typedef struct {
   double *rows;
   long    n, cap;
} diag_t;

static void diag_add (diag_t *d, const double *r6)
{
   if (d->n == d->cap) {
      d->cap = d->cap ? 2*d->cap : 1024;
      d->rows = (double *) realloc (d->rows, sizeof (double)*6*d->cap);
   }
   memcpy (d->rows + 6*d->n, r6, sizeof (double)*6);
   d->n++;
}

static void diag_flush (diag_t *d, int *fresh, double tau)
{
   FILE *fp;
   if (*fresh) {
      fp = open_or_die ("binData/diag.dat", "wt");
      fprintf (fp, "variables = t, W_E, W_M, W_T_x, W_T_y, W_T_z, W_p_e_r_p, W_k_i_n, W_E_M, W_`S\n"
                   "zone f=point\n");
      *fresh = 0;
   } else {
      fp = open_or_die ("binData/diag.dat", "at");
   }
   for (long q = 0 ; q < d->n ; ++q) {
      const double *r = d->rows + 6*q;
      if (r[0] < 0.5*tau)
         continue;
      fprintf (fp, "%e %e %e %e %e %e %e %e %e %e\n", r[0], r[1], r[2], r[3], r[4], r[5],
               r[4] + r[5], r[3] + r[4] + r[5], r[1] + r[2], r[1] + r[2] + r[3] + r[4] + r[5]);
   }
   fclose (fp);
   d->n = 0;
}

typedef struct {
   int sys_num;           /* next checkpoint record */
   int map_num;           /* next file map id */
   int tec_num;           /* next tecplot record */
   int spectr_num;        /* next spectral dump */
   unsigned char head_E[HEADER_BYTES], head_H[HEADER_BYTES];
   char prtn_src[256];
} records_t;

/* fileMap_save (IO_fileMap.c:129-157) for one rank: the map record, then
 * fileMap.N; returns the record's id. */
static int save_filemap (records_t *rec, const domain_t *dom)
{
   char path[512];
   const int map_id = rec->map_num++;
   snprintf (path, sizeof (path), "binData/fileMap_%06d.txt", map_id);
   FILE *fp = open_or_die (path, "wt");
   fprintf (fp, "%d cpus total.\n", 1);
   fprintf (fp, "%d: (%d %d %d) - (%d %d %d)\n", 0, dom->dmin[0], dom->dmin[1], dom->dmin[2],
            dom->dmax[0], dom->dmax[1], dom->dmax[2]);
   fclose (fp);
   fp = open_or_die ("binData/fileMap.N", "wt");
   fprintf (fp, "@ %d filemaps total is written.\n", rec->map_num);
   fclose (fp);
   return map_id;
}

/* Region (0,0,0)-(n) and the mesh_t fields (type_mesh.h:67-84) of a mesh
 * allocated over [-ghost, n+ghost], pointers zeroed: the header mesh_save and
 * tecIO_saveVec write (type_mesh.c:285-313). */
static void mesh_head (const int n[3], const char *name, int ghost, int vector,
                       unsigned char out[HEADER_BYTES])
{
   int v[16] = {0, 0, 0, n[0], n[1], n[2]};
   int w[3];
   for (int a = 0 ; a < 3 ; ++a) {
      v[6 + 2*a] = -ghost;
      v[7 + 2*a] = n[a] + ghost;
      w[a] = n[a] + 2*ghost + 1;
   }
   v[12] = vector ? 1 : 0;
   v[13] = w[2];
   v[14] = w[1]*w[2];
   v[15] = (vector ? 24 : 8)*w[0]*w[1]*w[2];
   memset (out, 0, HEADER_BYTES);
   memcpy (out, v, sizeof (v));
   strncpy ((char *) out + sizeof (v) + 16, name, 29);
}

/* sysIO_save + plasma_save (IO_sys.c:99-124, core/plasma_IO.c:273-287),
 * asynchronously: the run's state is snapshot on the device at the step
 * boundary (mg_run_snapshot), then a writer thread waits for its copy into
 * pinned host buffers and writes the record while the main loop steps on.
 * The small shared files (domain.bin, the file map) are written here, in
 * order with the tecplot records; the record's own files follow in the
 * thread, sys_%06d.txt and sys.N last, so sys.N never names an incomplete
 * record.  One record is in flight at a time. */
typedef struct {
   pthread_t   th;
   int         active;
   mg_run_t   *run;
   double     *E, *H;
   mg_marker_t *m;
   long long   cap, n;
   long        nodes;
   int         sys_num, map_id;
   double      time;
   unsigned char head_E[HEADER_BYTES], head_H[HEADER_BYTES];
   char        prtn_src[256];
} ckpt_t;

static void *ckpt_write (void *arg)
{
   ckpt_t *c = (ckpt_t *) arg;
   char path[512];
   check (mg_run_snapshot_wait (c->run), "checkpoint copy");
   snprintf (path, sizeof (path), "binData/plasma_%06d_%03d.bin", c->sys_num, 0);
   write_markers (path, c->m, c->n);
   snprintf (path, sizeof (path), "binData/sys_E_%06d(%03d).bin", c->sys_num, 0);
   write_mesh (path, c->head_E, c->E, c->nodes);
   snprintf (path, sizeof (path), "binData/sys_H_%06d(%03d).bin", c->sys_num, 0);
   write_mesh (path, c->head_H, c->H, c->nodes);
   snprintf (path, sizeof (path), "binData/sys_prtn_%06d.bin", c->sys_num);
   copy_file (c->prtn_src, path);
   snprintf (path, sizeof (path), "binData/sys_%06d.txt", c->sys_num);
   FILE *fp = open_or_die (path, "wt");
   fprintf (fp, "@ %.14e    time.\n", c->time);
   fprintf (fp, "@ %d       cpus total.\n", 1);
   fprintf (fp, "@ %d       file map id.\n", c->map_id);
   fprintf (fp, "That is checkpoint (record of the full system state) #%d.\n", c->sys_num);
   fclose (fp);
   fp = open_or_die ("binData/sys.N", "wt");
   fprintf (fp, "@ %d\t  system check-point records written.\n", c->sys_num + 1);
   fclose (fp);
   return NULL;
}

static void ckpt_join (ckpt_t *c)
{
   if (c->active) {
      pthread_join (c->th, NULL);
      c->active = 0;
   }
}

static void checkpoint (ckpt_t *c, mg_run_t *run, records_t *rec, const domain_t *dom, long nodes,
                        double time)
{
   ckpt_join (c);
   long long live = 0;
   check (mg_run_marker_count (run, &live), "marker count");
   if (!c->E) {
      c->E = (double *) mg_host_alloc (sizeof (double)*3*nodes);
      c->H = (double *) mg_host_alloc (sizeof (double)*3*nodes);
      if (!c->E || !c->H)
         die ("%s", "no pinned host memory for the checkpoint buffers");
   }
   if (live > c->cap) {
      mg_host_free (c->m);
      c->cap = live + 1;
      c->m = (mg_marker_t *) mg_host_alloc (sizeof (mg_marker_t)*c->cap);
      if (!c->m)
         die ("%s", "no pinned host memory for the checkpoint markers");
   }
   check (mg_run_snapshot (run, c->E, c->H, c->m, c->cap, &c->n), "checkpoint snapshot");
   write_domain (dom);
   c->map_id = save_filemap (rec, dom);
   c->run = run;
   c->nodes = nodes;
   c->sys_num = rec->sys_num++;
   c->time = time;
   memcpy (c->head_E, rec->head_E, HEADER_BYTES);
   memcpy (c->head_H, rec->head_H, HEADER_BYTES);
   memcpy (c->prtn_src, rec->prtn_src, sizeof (c->prtn_src));
   if (pthread_create (&c->th, NULL, ckpt_write, c) != 0)
      die ("%s", "cannot start the checkpoint writer");
   c->active = 1;
}

static void ckpt_free (ckpt_t *c)
{
   ckpt_join (c);
   mg_host_free (c->E);
   mg_host_free (c->H);
   mg_host_free (c->m);
}

/* main_throwStopFlag / main_catchStopFlag (core/main.c:120-189): the first
 * number asks to stop now, the second is the wall-time budget in seconds;
 * the run stops when the elapsed time plus one more stretch of steps and a
 * save would exceed it. */
static int stop_requested (double t0, double per_step, int stretch, double save_time)
{
   FILE *fp = fopen ("tmp/stop.flag", "rt");
   if (!fp)
      return 0;
   int alarm = 0, limit = 0;
   if (fscanf (fp, "%d %d", &alarm, &limit) != 2)
      alarm = 0, limit = 0;
   fclose (fp);
   if (alarm)
      return 1;
   return limit > 0 && now () - t0 + per_step*stretch + save_time > limit;
}

/* ---- probes (core/diag_probe.c) ------------------------------------------ */

typedef struct {
   int     n;          /* probes after de-duplication, nodes in ijk */
   int    *ijk;
   int     nact;       /* probes with every index in [0, n): these are sampled */
   int    *act;
   FILE  **fp;
   double *rows;       /* samples of one step call: steps x nact x 7 */
} probes_t;

static int dbl_to_int (double x) { return (int) (x + 128.0) - 128; }     /* misc_PIC.h:18 */

/* probe_addDraft (core/diag_probe.c:150-163). */
static void probe_add (probes_t *p, double x, double y, double z, double micron, const domain_t *d)
{
   p->ijk = (int *) realloc (p->ijk, sizeof (int)*3*(p->n + 1));
   int *q = p->ijk + 3*p->n++;
   q[0] = dbl_to_int (x*micron/d->h[0]);
   q[1] = dbl_to_int (y*micron/d->h[1]);
   q[2] = dbl_to_int (z*micron/d->h[2]);
}

/* cfg_readWord (misc_cfgReader.c:141-162): a line that starts with '@', its
 * first word after the '@', '>' and blanks. */
static void cfg_word (FILE *fp, char *word, size_t cap)
{
   char line[1024];
   if (!fgets (line, sizeof (line), fp) || line[0] != '@')
      die ("%s", "run_probes.cfg: parameter is absent");
   const char *w = line;
   while (*w == ' ' || *w == '@' || *w == '>')
      ++w;
   size_t l = 0;
   while (w[l] > ' ' && l + 1 < cap)
      ++l;
   memcpy (word, w, l);
   word[l] = 0;
}

/* cfg_readOptDouble / cfg_readOptInt (misc_cfgReader.c:88-111): '>' then the
 * number, the rest of the line skipped. */
static double cfg_opt_double (FILE *fp)
{
   double v = 0;
   char rest[1024];
   if (fgetc (fp) != '>' || fscanf (fp, "%le", &v) != 1)
      die ("%s", "run_probes.cfg: missing optional double parameter");
   if (!fgets (rest, sizeof (rest), fp))
      rest[0] = 0;
   return v;
}

static int cfg_opt_int (FILE *fp)
{
   int v = 0;
   char rest[1024];
   if (fgetc (fp) != '>' || fscanf (fp, "%d", &v) != 1)
      die ("%s", "run_probes.cfg: missing optional int parameter");
   if (!fgets (rest, sizeof (rest), fp))
      rest[0] = 0;
   return v;
}

/* One micron in code units: the 12th of the 15 doubles of binData/units.bin
 * (units_save / units_load, misc_units.c:39-88). */
static double micron_units (void)
{
   FILE *fp = open_or_die ("binData/units.bin", "rb");
   double u[12];
   read_exact (u, sizeof (u), fp, "binData/units.bin");
   fclose (fp);
   return u[11];
}

/* init_sources (scpic/em_sources.c:37-52): each .EM_sources/laser/mirror_NN
 * from 00 up to the first missing one read as mirror_source_is_loaded does
 * (scpic/em_mirror.c:464-486 with read_mirror_parameters, :292-328): the
 * title and dashes lines, nine "@ double" lines, an "@ int" line, the
 * dashes line (whose trailing newline directive, as in the reference, also
 * skips whitespace bytes at the start of the binary part), then the E and H
 * profiles of the (n1-9)(n2-9) nodes of the source plane; r0 and t0 are the
 * 1st and 3rd doubles of binData/units.bin. */
static int load_mirrors (mg_run_t *run, const domain_t *d)
{
   double u[3];
   int count = 0;
   for (;; ++count) {
      char name[64];
      snprintf (name, sizeof (name), ".EM_sources/laser/mirror_%02d", count);
      FILE *fp = fopen (name, "rb");
      if (!fp)
         break;
      if (count == 0) {
         FILE *uf = open_or_die ("binData/units.bin", "rb");
         read_exact (u, sizeof (u), uf, "binData/units.bin");
         fclose (uf);
      }
      mg_mirror_t m;
      memset (&m, 0, sizeof (m));
      if (fscanf (fp, "Mirror focused laser beam #%*d\n") < 0)
         die ("'%s' is truncated", name);
      if (fscanf (fp, "---------------------------------------\n") < 0)
         die ("'%s' is truncated", name);
      for (int q = 0 ; q < 9 ; ++q)
         if (fscanf (fp, "@ %le %*[^\n] ", &m.values[q]) != 1)
            die ("%s: cannot get double number", name);
      char rest[1024];
      if (fgetc (fp) != '@' || fscanf (fp, "%d", &m.direction) != 1 || !fgets (rest, sizeof (rest), fp))
         die ("%s: missing required int parameter", name);
      if (fscanf (fp, "---------------------------------------\n") < 0)
         die ("'%s' is truncated", name);
      const long nodes = (long) (d->dmax[1] - 9)*(d->dmax[2] - 9);
      double *E = (double *) malloc (sizeof (double)*4*nodes);
      double *H = (double *) malloc (sizeof (double)*4*nodes);
      if (!E || !H)
         die ("%s", "no host memory for the mirror profiles");
      read_exact (E, sizeof (double)*4*nodes, fp, name);
      read_exact (H, sizeof (double)*4*nodes, fp, name);
      fclose (fp);
      m.r0 = u[0];
      m.t0 = u[2];
      m.E = E;
      m.H = H;
      check (mg_run_add_mirror (run, &m), "mirror source");
      free (E);
      free (H);
   }
   return count;
}

/* probe_allocate + probe_touch (core/diag_probe.c:48-100, 121-395) for one
 * rank: old probe files removed unless the run continues, run_probes.cfg
 * read (point / line / rectangle / volume groups up to 'end'), repeated
 * nodes removed, output/probe_locations.dat and binData/probe_globals.bin
 * written and the files of the probes inside the domain opened. */
static void probes_open (probes_t *p, const domain_t *d, int cont)
{
   memset (p, 0, sizeof (*p));
   if (!cont) {
      DIR *dir = opendir ("./binData");
      if (!dir)
         die ("%s", "cannot open 'binData' folder");
      struct dirent *e;
      while ((e = readdir (dir))) {
         const size_t l = strlen (e->d_name);
         if (strncmp (e->d_name, "probe_", 6) || l < 4 || strncmp (e->d_name + l - 4, ".bin", 4))
            continue;
         char name[600];
         snprintf (name, sizeof (name), "binData/%s", e->d_name);
         remove (name);
      }
      closedir (dir);
   }
   FILE *fp = fopen ("run_probes.cfg", "rt");
   const double micron = micron_units ();
   while (fp) {
      char word[200];
      cfg_word (fp, word, sizeof (word));
      if (!strcmp (word, "end")) {
         fclose (fp);
         fp = NULL;
      } else if (!strcmp (word, "point")) {
         const double x = cfg_opt_double (fp), y = cfg_opt_double (fp), z = cfg_opt_double (fp);
         probe_add (p, x, y, z, micron, d);
      } else if (!strcmp (word, "line")) {
         double x1 = cfg_opt_double (fp), y1 = cfg_opt_double (fp), z1 = cfg_opt_double (fp);
         double x2 = cfg_opt_double (fp), y2 = cfg_opt_double (fp), z2 = cfg_opt_double (fp);
         const int N = 2 + abs (cfg_opt_int (fp));
         const double dx = (x2 - x1)/(N - 1), dy = (y2 - y1)/(N - 1), dz = (z2 - z1)/(N - 1);
         for (int i = 0 ; i < N ; ++i, x1 += dx, y1 += dy, z1 += dz)
            probe_add (p, x1, y1, z1, micron, d);
      } else if (!strcmp (word, "rectangle") || !strcmp (word, "volume")) {
         const int sides = strcmp (word, "volume") ? 2 : 3;
         double o[3], e[3][3];
         int N[3] = {1, 1, 1};
         for (int a = 0 ; a < 3 ; ++a)
            o[a] = cfg_opt_double (fp);
         for (int s = 0 ; s < sides ; ++s)
            for (int a = 0 ; a < 3 ; ++a)
               e[s][a] = cfg_opt_double (fp);
         for (int s = 0 ; s < sides ; ++s) {
            N[s] = 2 + abs (cfg_opt_int (fp));
            for (int a = 0 ; a < 3 ; ++a)
               e[s][a] = (e[s][a] - o[a])/(N[s] - 1);
         }
         for (int a = 0 ; a < N[0] ; ++a)
            for (int b = 0 ; b < N[1] ; ++b)
               for (int c = 0 ; c < N[2] ; ++c) {
                  double v[3];
                  for (int q = 0 ; q < 3 ; ++q)
                     v[q] = sides == 2 ? o[q] + a*e[0][q] + b*e[1][q]
                                       : o[q] + a*e[0][q] + b*e[1][q] + c*e[2][q];
                  probe_add (p, v[0], v[1], v[2], micron, d);
               }
      } else {
         die ("bad probe group '%s' (use 'point', 'line', 'rectangle', or 'volume')", word);
      }
   }
   /* Repeated nodes: the last probe takes the place of the repeat, which is
    * then tested again (core/diag_probe.c:343-350). */
   for (int p1 = 0 ; p1 < p->n ; ++p1)
      for (int p2 = p1 + 1 ; p2 < p->n ; ++p2)
         if (!memcmp (p->ijk + 3*p1, p->ijk + 3*p2, 3*sizeof (int))) {
            --p->n;
            memmove (p->ijk + 3*p2, p->ijk + 3*p->n, 3*sizeof (int));
            --p2;
         }

   fp = open_or_die ("output/probe_locations.dat", "wt");
   fprintf (fp, "variables = \"x [<greek>m</greek>m]\", \"y [<greek>m</greek>m]\", "
                "\"z [<greek>m</greek>m]\"\nzone t=\"domain\", f= point\n");
   for (int i = 0 ; i < 2 ; ++i)
      for (int j = 0 ; j < 2 ; ++j)
         for (int k = 0 ; k < 2 ; ++k)
            fprintf (fp, "%e %e %e\n", (d->dmin[0]*i + d->dmax[0]*(1 - i))*d->h[0]/micron,
                     (d->dmin[1]*j + d->dmax[1]*(1 - j))*d->h[1]/micron,
                     (d->dmin[2]*k + d->dmax[2]*(1 - k))*d->h[2]/micron);
   fprintf (fp, "zone t=\"probes\", f= point\n");
   for (int q = 0 ; q < p->n ; ++q)
      fprintf (fp, "%e %e %e\n", p->ijk[3*q]*d->h[0]/micron, p->ijk[3*q + 1]*d->h[1]/micron,
               p->ijk[3*q + 2]*d->h[2]/micron);
   fclose (fp);

   /* probeGlobals_t {tau, h1, h2, h3, min[3], max[3]} (probe.h) */
   double globals[10] = {d->tau, d->h[0], d->h[1], d->h[2]};
   for (int a = 0 ; a < 3 ; ++a) {
      globals[4 + a] = d->dmin[a]*d->h[a];
      globals[7 + a] = d->dmax[a]*d->h[a];
   }
   fp = open_or_die ("binData/probe_globals.bin", "wb");
   write_exact (globals, sizeof (globals), fp, "binData/probe_globals.bin");
   fclose (fp);

   p->act = (int *) malloc (sizeof (int)*3*(p->n > 0 ? p->n : 1));
   p->fp = (FILE **) malloc (sizeof (FILE *)*(p->n > 0 ? p->n : 1));
   for (int q = 0 ; q < p->n ; ++q) {
      const int *c = p->ijk + 3*q;
      int inside = 1;
      for (int a = 0 ; a < 3 ; ++a)
         inside &= c[a] >= d->dmin[a] && c[a] < d->dmax[a];
      if (!inside)
         continue;
      char name[200];
      snprintf (name, sizeof (name), "binData/probe_%d_%d_%d.bin", c[0], c[1], c[2]);
      FILE *f = fopen (name, "rb");
      if (!f) {
         /* probeHeader_t {char magic[8] = "probes", int i, j, k} */
         unsigned char head[20] = "probes";
         memcpy (head + 8, c, 3*sizeof (int));
         f = open_or_die (name, "wb");
         write_exact (head, sizeof (head), f, name);
      } else {
         fclose (f);
         f = open_or_die (name, "ab");
      }
      memcpy (p->act + 3*p->nact, c, 3*sizeof (int));
      p->fp[p->nact++] = f;
   }
   p->rows = (double *) malloc (sizeof (double)*7*256*(p->nact > 0 ? p->nact : 1));
}

/* probe_postData (core/diag_probe.c:409-429): one probeSample_t {time, Ex,
 * Ey, Ez, Hx, Hy, Hz} per step and probe, from the device's sample ring. */
static void probes_write (mg_run_t *run, probes_t *p, int steps)
{
   if (p->nact == 0 || steps == 0)
      return;
   check (mg_run_probe_samples (run, steps, p->rows), "probe samples");
   for (int s = 0 ; s < steps ; ++s)
      for (int q = 0 ; q < p->nact ; ++q)
         write_exact (p->rows + 7*((long) s*p->nact + q), 7*sizeof (double), p->fp[q], "probe file");
}

static void probes_close (probes_t *p)
{
   for (int q = 0 ; q < p->nact ; ++q)
      fclose (p->fp[q]);
   free (p->ijk);
   free (p->act);
   free (p->fp);
   free (p->rows);
}

/* ---- TF/SF interface (core/em_TFSF.c) ------------------------------------- */

static const char *const TFSF_NAME[24] = {                 /* core/em_TFSF.c:86-119 */
   "Ey_xMin", "Ez_xMin", "Ey_xMax", "Ez_xMax", "Ez_yMin", "Ex_yMin",
   "Ez_yMax", "Ex_yMax", "Ex_zMin", "Ey_zMin", "Ex_zMax", "Ey_zMax",
   "Hz_xMin", "Hy_xMin", "Hz_xMax", "Hy_xMax", "Hx_yMin", "Hz_yMin",
   "Hx_yMax", "Hz_yMax", "Hy_zMin", "Hx_zMin", "Hy_zMax", "Hx_zMax"};

typedef struct {
   int       on;
   mg_tfsf_t cfg;
   int       region[24][6];     /* regions in the frame layout */
   long long size;              /* doubles per frame */
   int       frame;             /* frame counter of the next step */
   int       written;           /* record: frames written by this run */
   FILE     *fp[24];            /* record: the face streams */
   double   *buf;               /* 257 frames */
} tfsf_t;

static long long region_volume (const int r[6])
{
   long long v = 1;
   for (int a = 0 ; a < 3 ; ++a)
      v *= (r[3 + a] >= r[a]) ? r[3 + a] - r[a] + 1 : 0;
   return v;
}

static void tfsf_path (char *out, size_t cap, int f, int cpu)
{
   snprintf (out, cap, ".EM_sources/TFSF/%s_%03d.bin", TFSF_NAME[f], cpu);   /* :143-148 */
}

/* TFSF_init for one rank: reads TFSF.cfg (and in play openFaces.cfg,
 * consistencyCheck.dat, lastFrameTime.bin), configures the run; record mode
 * opens the face streams and writes consistencyCheck.dat and the merge map
 * (TFSF_turnRec :229-283, TFSF_defragInit :199-224). */
static void tfsf_open (tfsf_t *t, mg_run_t *run, const domain_t *d, double time)
{
   memset (t, 0, sizeof (*t));
   if (!access (".EM_sources/TFSF/TFSF_defrag.map", F_OK))
      die ("%s", "input data is not compiled (use 'TFSFdefrag')");
   FILE *fp = fopen (".EM_sources/TFSF/TFSF.cfg", "rt");
   if (!fp)
      return;
   const char *cfg = ".EM_sources/TFSF/TFSF.cfg";
   for (int a = 0 ; a < 3 ; ++a) {
      t->cfg.lo[a] = read_at_int (fp, cfg);
      t->cfg.hi[a] = read_at_int (fp, cfg);
   }
   t->cfg.mode = read_at_int (fp, cfg);
   fclose (fp);
   if (t->cfg.mode != MG_TFSF_PLAY_FORWARD && t->cfg.mode != MG_TFSF_RECORD &&
       t->cfg.mode != MG_TFSF_PLAY_BACKWARD)
      return;                                   /* inactive */
   t->on = 1;
   if (t->cfg.mode == MG_TFSF_RECORD) {
      check (mg_run_set_tfsf (run, &t->cfg), "TF/SF interface");
      check (mg_run_tfsf_faces (run, (int *) t->region, &t->size), "TF/SF faces");
      for (int f = 0 ; f < 24 ; ++f) {
         if (region_volume (t->region[f]) <= 0)
            continue;
         char name[200];
         tfsf_path (name, sizeof (name), f, 0);
         t->fp[f] = open_or_die (name, "wb");
         /* reg_t {min[3], max[3], cpu, barcode = mode, wrap[3]} */
         const int head[11] = {t->region[f][0], t->region[f][1], t->region[f][2], t->region[f][3],
                               t->region[f][4], t->region[f][5], 0, t->cfg.mode, 0, 0, 0};
         write_exact (head, sizeof (head), t->fp[f], name);
      }
      fp = open_or_die (".EM_sources/TFSF/consistencyCheck.dat", "wt");
      fprintf (fp, "@ %d\tInterface size in X direction (nodes)\n", t->cfg.hi[0] - t->cfg.lo[0]);
      fprintf (fp, "@ %d\tInterface size in Y direction (nodes)\n", t->cfg.hi[1] - t->cfg.lo[1]);
      fprintf (fp, "@ %d\tInterface size in Z direction (nodes)\n", t->cfg.hi[2] - t->cfg.lo[2]);
      fprintf (fp, "@ %.12e\tTime step\n", d->tau);
      fprintf (fp, "@ %.12e\tSpatial step along X\n", d->h[0]);
      fprintf (fp, "@ %.12e\tSpatial step along Y\n", d->h[1]);
      fprintf (fp, "@ %.12e\tSpatial step along Z\n", d->h[2]);
      fclose (fp);
      /* The merge map: each face's full region (TFSF_init :505-553), its
       * unrolling axes, the merged stream and this rank's stream. */
      fp = open_or_die (".EM_sources/TFSF/TFSF_defrag.map", "at");
      const int *side[2] = {t->cfg.lo, t->cfg.hi};
      for (int f = 0 ; f < 24 ; ++f) {
         const int fe = f % 12, a = fe/4, top = (fe/2) % 2, comp = fe % 2, ce = (a + 1 + comp) % 3;
         int lo[3], hi[3];
         for (int b = 0 ; b < 3 ; ++b) {
            lo[b] = t->cfg.lo[b];
            hi[b] = t->cfg.hi[b];
         }
         lo[a] = hi[a] = side[top][a];
         lo[ce] += 1;
         if (f >= 12) {
            lo[a] += top;
            hi[a] += top;
         }
         char name[200];
         fprintf (fp, "[%d %d] [%d %d] [%d %d]\n", lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]);
         fprintf (fp, "ep = %d, eq = %d\n", (a + 1) % 3, (a + 2) % 3);
         tfsf_path (name, sizeof (name), f, 99999);
         fprintf (fp, "%s\n", name);
         if (t->fp[f]) {
            tfsf_path (name, sizeof (name), f, 0);
            fprintf (fp, "%s\n", name);
         }
         fprintf (fp, "---\n");
      }
      fclose (fp);
   } else {
      fp = fopen (".EM_sources/TFSF/openFaces.cfg", "rt");
      if (fp) {
         for (int a = 0 ; a < 3 ; ++a)
            for (int top = 0 ; top < 2 ; ++top)
               t->cfg.open[top][a] = read_at_int (fp, ".EM_sources/TFSF/openFaces.cfg");
         fclose (fp);
      }
      const char *cc = ".EM_sources/TFSF/consistencyCheck.dat";
      fp = fopen (cc, "rt");
      if (!fp)
         die ("%s", "there are no recorded data");
      for (int a = 0 ; a < 3 ; ++a)
         if (read_at_int (fp, cc) != t->cfg.hi[a] - t->cfg.lo[a])
            die ("inconsistent size along axis '%s'", a == 0 ? "X" : a == 1 ? "Y" : "Z");
      const double old_tau = read_at_double (fp, cc);
      if (!(fabs (1 - old_tau/d->tau) < 1e-11))
         die ("%s", "inconsistent time step");
      for (int a = 0 ; a < 3 ; ++a)
         if (!(fabs (1 - read_at_double (fp, cc)/d->h[a]) < 1e-11))
            die ("inconsistent spatial step along %s", a == 0 ? "X" : a == 1 ? "Y" : "Z");
      fclose (fp);
      fp = open_or_die (".EM_sources/TFSF/lastFrameTime.bin", "rb");
      read_exact (&t->cfg.frames, sizeof (int), fp, ".EM_sources/TFSF/lastFrameTime.bin");
      fclose (fp);
      t->cfg.ring = 512;
      check (mg_run_set_tfsf (run, &t->cfg), "TF/SF interface");
      check (mg_run_tfsf_faces (run, (int *) t->region, &t->size), "TF/SF faces");
      /* the merged streams stay open for the frames of each step call */
      for (int f = 0 ; f < 24 ; ++f) {
         char name[200];
         tfsf_path (name, sizeof (name), f, 99999);
         t->fp[f] = fopen (name, "rb");
         const int fe = f % 12, a = fe/4, top = (fe/2) % 2;
         if (!t->fp[f] && !t->cfg.open[top][a])
            die ("cannot open '%s'", name);
      }
   }
   t->frame = (int) (time/d->tau + 0.1);
   t->buf = (double *) malloc (sizeof (double)*(size_t) (t->size > 0 ? t->size : 1)*257);
}

/* Play: the frames steps frame .. frame + k - 1 read (TFSF_cacheFrame,
 * :785-806), from the merged streams to the device ring. */
static void tfsf_before (tfsf_t *t, mg_run_t *run, int k)
{
   if (!t->on || t->cfg.mode == MG_TFSF_RECORD || t->size == 0)
      return;
   const int last = t->cfg.frames;
   int lo, hi;
   if (t->cfg.mode == MG_TFSF_PLAY_FORWARD) {
      lo = t->frame;
      hi = t->frame + k;
   } else {
      lo = last - 1 - (t->frame + k - 1);
      hi = last - 1 - t->frame;
   }
   if (lo < 0) lo = 0;
   if (hi > last - 1) hi = last - 1;
   if (hi < lo)
      return;
   for (int fr = lo ; fr <= hi ; ++fr) {
      double *o = t->buf + (size_t) (fr - lo)*t->size;
      for (int f = 0 ; f < 24 ; ++f) {
         const long long v = region_volume (t->region[f]);
         if (!t->fp[f]) {
            memset (o, 0, sizeof (double)*v);
         } else {
            fseek (t->fp[f], 44 + (long) fr*v*(long) sizeof (double), SEEK_SET);
            if (fread (o, sizeof (double), v, t->fp[f]) != (size_t) v)
               die ("TF/SF stream '%s' ends before the frames the run plays", TFSF_NAME[f]);
         }
         o += v;
      }
   }
   check (mg_run_tfsf_put_frames (run, lo, hi - lo + 1, t->buf), "TF/SF frames");
}

/* Record: the frames of the last k steps to the face streams. */
static void tfsf_after (tfsf_t *t, mg_run_t *run, int k)
{
   if (!t->on)
      return;
   t->frame += k;
   if (t->cfg.mode != MG_TFSF_RECORD || t->size == 0)
      return;
   check (mg_run_tfsf_recorded (run, k, t->buf), "TF/SF record");
   for (int s = 0 ; s < k ; ++s) {
      const double *o = t->buf + (size_t) s*t->size;
      for (int f = 0 ; f < 24 ; ++f) {
         const long long v = region_volume (t->region[f]);
         if (t->fp[f])
            write_exact (o, sizeof (double)*v, t->fp[f], TFSF_NAME[f]);
         o += v;
      }
   }
   t->written += k;
}

/* TFSF_shutDown (:862-891): streams closed, record mode writes the frame
 * count. */
static void tfsf_close (tfsf_t *t)
{
   for (int f = 0 ; f < 24 ; ++f)
      if (t->fp[f])
         fclose (t->fp[f]);
   if (t->on && t->cfg.mode == MG_TFSF_RECORD) {
      FILE *fp = open_or_die (".EM_sources/TFSF/lastFrameTime.bin", "wb");
      write_exact (&t->written, sizeof (int), fp, ".EM_sources/TFSF/lastFrameTime.bin");
      fclose (fp);
   }
   free (t->buf);
}

/* ---- spectral dumps (spectr_dump.c:66-109) -------------------------------- */

static long chunk_open (FILE *fp, const char *name)
{
   const long pos = ftell (fp);
   const long long size = -1;
   const int deleted = 0, l = (int) strlen (name);
   write_exact (&size, sizeof (size), fp, "spectral dump");
   write_exact (&deleted, sizeof (int), fp, "spectral dump");
   write_exact (&l, sizeof (int), fp, "spectral dump");
   fputc ('\n', fp);
   write_exact (name, l, fp, "spectral dump");
   fputc ('\n', fp);
   return pos;
}

/* The chunk's size, header included, into its first 8 bytes
 * (CF_closeChunk, type_CFile.c:357-370). */
static void chunk_close (FILE *fp, long pos)
{
   const long long size = ftell (fp) - pos;
   fseek (fp, pos, SEEK_SET);
   write_exact (&size, sizeof (size), fp, "spectral dump");
   fseek (fp, 0, SEEK_END);
}

/* tmp/spectrDump_<num>_0: chunk file with the global parameters, the dumped
 * region [0, n-1]^3 and the raw E^n and H^n components over it; then
 * binData/spectr.N.  E, H: nodes [0, n]^3, 3 doubles a node. */
static void spectr_dump (records_t *rec, const domain_t *d, double time, const double *E, const double *H)
{
   char path[512];
   snprintf (path, sizeof (path), "tmp/spectrDump_%d_%d", rec->spectr_num, 0);
   FILE *fp = open_or_die (path, "wb");
   fputs ("============\n Chunk file\n============\n", fp);
   long c = chunk_open (fp, "global parameters");
   fprintf (fp, "%d\t  cpus total.\n", 1);
   fprintf (fp, "%d\t  i-min.\n", d->dmin[0]);
   fprintf (fp, "%d\t  j-min.\n", d->dmin[1]);
   fprintf (fp, "%d\t  k-min.\n", d->dmin[2]);
   fprintf (fp, "%d\t  i-max.\n", d->dmax[0]);
   fprintf (fp, "%d\t  j-max.\n", d->dmax[1]);
   fprintf (fp, "%d\t  k-max.\n", d->dmax[2]);
   fprintf (fp, "%.14e\t  time.\n", time);
   fprintf (fp, "%e\t  h1.\n", d->h[0]);
   fprintf (fp, "%e\t  h2.\n", d->h[1]);
   fprintf (fp, "%e\t  h3.\n", d->h[2]);
   chunk_close (fp, c);
   /* reg_t {min[3], max[3], cpu, barcode, wrap[3]} after mf_mesh_initUnroll
    * (type_mesh2.h:29-37): region [0, n-1]^3, strides of its own array. */
   const int n[3] = {d->dmax[0], d->dmax[1], d->dmax[2]};
   const int reg[11] = {0, 0, 0, n[0] - 1, n[1] - 1, n[2] - 1, 0, 0, n[1]*n[2], n[2], 1};
   c = chunk_open (fp, "cpu region");
   write_exact (reg, sizeof (reg), fp, path);
   chunk_close (fp, c);
   const long nk = n[2] + 1, nj = n[1] + 1;
   double *line = (double *) malloc (sizeof (double)*n[2]);
   for (int f = 0 ; f < 6 ; ++f) {
      const char names[6][4] = {"E.x", "E.y", "E.z", "H.x", "H.y", "H.z"};
      const double *src = f < 3 ? E : H;
      c = chunk_open (fp, names[f]);
      for (int i = 0 ; i < n[0] ; ++i)
         for (int j = 0 ; j < n[1] ; ++j) {
            for (int k = 0 ; k < n[2] ; ++k)
               line[k] = src[3*(((long) i*nj + j)*nk + k) + f % 3];
            write_exact (line, sizeof (double)*n[2], fp, path);
         }
      chunk_close (fp, c);
   }
   free (line);
   fclose (fp);
   rec->spectr_num++;
   fp = open_or_die ("binData/spectr.N", "wt");
   fprintf (fp, "@ %d  spectr dumps written.\n", rec->spectr_num);
   fclose (fp);
}

/* One step with a tecplot dump, a spectral dump or both (core/main.c:384-402,
 * 430-434): the staged step, with the probe samples after the field energy;
 * E^n, H^n and the density of the moved markers written after plasma_move
 * (tecIO_saveFields, IO_tecplot.c:220-245), then the spectral dump of E^n and
 * H^n, and J after the E step (tecIO_saveCurrents, IO_tecplot.c:250-266).
 * row: the step's energy row. */
static void staged_step (mg_run_t *run, records_t *rec, const domain_t *dom, long nodes, double time,
                         double row[6], int tec, int spectr, probes_t *probes, tfsf_t *tfsf)
{
   tfsf_before (tfsf, run, 1);
   char path[512];
   const int n[3] = {dom->dmax[0], dom->dmax[1], dom->dmax[2]};
   unsigned char head[HEADER_BYTES];
   double *a = (double *) malloc (sizeof (double)*3*nodes), *b = (double *) malloc (sizeof (double)*3*nodes);
   const long full = (long) (n[0] + 5)*(n[1] + 5)*(n[2] + 5);
   double *rho = (double *) malloc (sizeof (double)*full);

   check (mg_em_HHalfStep (run), "H half step");
   check (mg_em_energy (run, &row[1], &row[2]), "field energy");
   probes_write (run, probes, 1);
   check (mg_plasma_move (run), "plasma move");
   check (mg_plasma_temperature (run, &row[3], &row[4], &row[5]), "temperature");
   row[0] = time;
   if (spectr && !tec) {
      check (mg_run_get_fields (run, a, b), "download fields");
      spectr_dump (rec, dom, time, a, b);
   }
   if (!tec) {
      check (mg_em_HStep (run), "H step");
      check (mg_em_EStep_start (run), "E step");
      check (mg_jbc_finish (run), "current walls");
      check (mg_em_EStep_finish (run), "E step finish");
      tfsf_after (tfsf, run, 1);
      free (a);
      free (b);
      free (rho);
      return;
   }
   check (mg_plasma_rho (run, rho), "charge density");
   check (mg_tecplot_fields (run, a, b), "tecplot fields");
   write_domain (dom);                                        /* parameter_save */
   const int map_id = save_filemap (rec, dom);
   snprintf (path, sizeof (path), "binData/tec_E_%06d(%03d).bin", rec->tec_num, 0);
   write_mesh (path, rec->head_E, a, nodes);
   snprintf (path, sizeof (path), "binData/tec_H_%06d(%03d).bin", rec->tec_num, 0);
   write_mesh (path, rec->head_H, b, nodes);
   snprintf (path, sizeof (path), "binData/tec_%06d.txt", rec->tec_num);
   FILE *fp = open_or_die (path, "wb");
   const int cpus = 1;
   write_exact (&time, sizeof (double), fp, path);
   write_exact (&cpus, sizeof (int), fp, path);
   write_exact (&map_id, sizeof (int), fp, path);
   fclose (fp);
   snprintf (path, sizeof (path), "binData/tec_prtn_%06d.bin", rec->tec_num);
   copy_file (rec->prtn_src, path);
   if (spectr) {
      check (mg_run_get_fields (run, a, b), "download fields");
      spectr_dump (rec, dom, time, a, b);
   }

   check (mg_em_HStep (run), "H step");
   check (mg_em_EStep_start (run), "E step");
   check (mg_jbc_finish (run), "current walls");
   check (mg_em_EStep_finish (run), "E step finish");
   tfsf_after (tfsf, run, 1);
   check (mg_tecplot_currents (run, a), "tecplot currents");
   mesh_head (n, "vec_J", 2, 1, head);
   snprintf (path, sizeof (path), "binData/tec_J_%06d(%03d).bin", rec->tec_num, 0);
   write_mesh (path, head, a, nodes);
   /* rho over [0, n]^3 out of [-2, n+2]^3 */
   long q = 0;
   for (int i = 0 ; i <= n[0] ; ++i)
      for (int j = 0 ; j <= n[1] ; ++j)
         for (int k = 0 ; k <= n[2] ; ++k)
            b[q++] = rho[((long) (i + 2)*(n[1] + 5) + (j + 2))*(n[2] + 5) + (k + 2)];
   mesh_head (n, "rho", 2, 0, head);
   snprintf (path, sizeof (path), "binData/tec_rho_%06d(%03d).bin", rec->tec_num, 0);
   fp = open_or_die (path, "wb");
   write_exact (head, HEADER_BYTES, fp, path);
   write_exact (b, sizeof (double)*nodes, fp, path);
   fclose (fp);
   rec->tec_num++;
   fp = open_or_die ("binData/tecplot.N", "wt");
   fprintf (fp, "@ %d  tecplots' records written.\n", rec->tec_num);
   fclose (fp);
   free (a);
   free (b);
   free (rho);
}

int main (int argc, char **argv)
{
   int precision = MG_FP64, device = 0;
   for (int a = 1 ; a < argc ; ++a) {
      if (!strcmp (argv[a], "--fp32"))
         precision = MG_FP32_OFFSET;
      else if (!strcmp (argv[a], "--device") && a + 1 < argc)
         device = atoi (argv[++a]);
      else
         die ("unknown option '%s' (usage: core_b200.out [--fp32] [--device N])", argv[a]);
   }
   const double t_start = now ();

   FILE *fp = open_or_die ("run_mandor.cfg", "rt");
   run_cfg_t cfg;
   cfg.total = read_at_int (fp, "run_mandor.cfg");
   cfg.full = read_at_int (fp, "run_mandor.cfg");
   cfg.tecplot = read_at_int (fp, "run_mandor.cfg");
   cfg.cont = (read_at_int (fp, "run_mandor.cfg") == 1);
   cfg.stop = read_at_int (fp, "run_mandor.cfg");
   cfg.spectr = read_at_int (fp, "run_mandor.cfg");
   fclose (fp);
   if (!cfg.total || !cfg.full || !cfg.tecplot || !cfg.stop || !cfg.spectr)
      die ("'%s' contains zero step(s)", "run_mandor.cfg");

   if (!(fp = fopen ("tmp/stop.flag", "rt"))) {
      fp = open_or_die ("tmp/stop.flag", "wt");
      fprintf (fp, "0\n%d\n", 23*60*60 + 30*60);
   }
   fclose (fp);

   domain_t dom = read_domain ();
   const int records = read_count ("binData/sys.N");
   if (records < 1)
      die ("%s", "initial checkpoint is not prepared");
   int point = records - 1;
   records_t rec;
   if (cfg.cont && point != 0) {
      rec.sys_num = records;
      rec.map_num = read_count ("binData/fileMap.N");
      FILE *tn = fopen ("binData/tecplot.N", "rt");       /* tecIO_setRecordNum (-1) */
      rec.tec_num = tn ? read_at_int (tn, "binData/tecplot.N") : 0;
      if (tn)
         fclose (tn);
      rec.spectr_num = read_count ("binData/spectr.N");   /* spectr_continueDump */
   } else {
      point = 0;
      rec.sys_num = 1;
      rec.map_num = read_count ("binData/fileMap_start.txt");
      rec.tec_num = 1;                                  /* after setup's record 0 */
      rec.spectr_num = 0;
   }

   char path[512];
   snprintf (path, sizeof (path), "binData/sys_%06d.txt", point);
   fp = open_or_die (path, "rt");
   double time = read_at_double (fp, path);
   fclose (fp);

   mg_params_t p;
   memset (&p, 0, sizeof (p));
   for (int a = 0 ; a < 3 ; ++a) {
      if (dom.dmin[a] != 0)
         die ("%s", "domains not starting at node 0 are not supported");
      p.n[a] = dom.dmax[a];
      p.h[a] = dom.h[a];
      p.bc_min[a] = dom.bcmin[a];
      p.bc_max[a] = dom.bcmax[a];
   }
   p.tau = dom.tau;
   p.time = time;
   p.precision = precision;
   p.device = device;
   const long nodes = (long) (p.n[0] + 1)*(p.n[1] + 1)*(p.n[2] + 1);

   snprintf (path, sizeof (path), "binData/sys_E_%06d(%03d).bin", point, 0);
   double *E = read_mesh (path, rec.head_E, nodes);
   snprintf (path, sizeof (path), "binData/sys_H_%06d(%03d).bin", point, 0);
   double *H = read_mesh (path, rec.head_H, nodes);
   snprintf (rec.prtn_src, sizeof (rec.prtn_src), "binData/sys_prtn_%06d.bin", point);
   long long nm = 0;
   snprintf (path, sizeof (path), "binData/plasma_%06d_%03d.bin", point, 0);
   mg_marker_t *m = read_markers (path, &nm);
   p.capacity = nm;

   mg_run_t *run = NULL;
   check (mg_run_create (&p, &run), "create run");
   check (mg_run_set_fields (run, E, H), "upload fields");
   check (mg_run_set_markers (run, m, nm), "upload markers");
   /* Hard gauss-spot source when .gaussSpot.cfg exists (em_gaussSpot.c:42-62). */
   FILE *gs = fopen (".gaussSpot.cfg", "rt");
   if (gs) {
      mg_gauss_spot_t s;
      double *v[9] = {&s.ampl, &s.frequency, &s.x, &s.y, &s.z, &s.width, &s.duration,
                      &s.front_offset, &s.t_plateau};
      for (int q = 0 ; q < 9 ; ++q)
         *v[q] = read_at_double (gs, ".gaussSpot.cfg");
      s.ey = read_at_int (gs, ".gaussSpot.cfg");
      s.ez = read_at_int (gs, ".gaussSpot.cfg");
      fclose (gs);
      check (mg_run_set_gauss_spot (run, &s), "gauss spot");
   }
   const int mirrors = load_mirrors (run, &dom);
   tfsf_t tfsf;
   tfsf_open (&tfsf, run, &dom, time);
   probes_t probes;
   probes_open (&probes, &dom, cfg.cont && point > 0);
   if (probes.nact > 0)
      check (mg_run_set_probes (run, probes.act, probes.nact), "probes");
   check (mg_run_init (run), "init");
   free (E);
   free (H);
   free (m);
   const double save_time = now () - t_start;     /* loading time estimates saving time */

   printf ("core_b200.out: %lld markers, %d x %d x %d cells, %s, record %d, t = %.6e\n", nm,
           p.n[0], p.n[1], p.n[2], precision == MG_FP64 ? "FP64" : "FP32-offset", point, time);
   if (mirrors > 0)
      printf ("core_b200.out: %d focused-laser source(s)\n", mirrors);
   int fresh_diag = !(cfg.cont && point != 0);
   diag_t diag = {NULL, 0, 0};
   double rows[6*256];
   const double t_loop = now ();
   double last_saved = -1;
   ckpt_t ckpt;
   memset (&ckpt, 0, sizeof (ckpt));
   int stop = 0, t = 0;
   while (t < cfg.total && !stop) {
      /* Advance to the next checkpoint, stop-flag check or the end. */
      int next = cfg.total;
      const int nfull = (t/cfg.full + 1)*cfg.full;
      const int nstop = (t/cfg.stop + 1)*cfg.stop;
      if (nfull < next) next = nfull;
      if (nstop < next) next = nstop;
      if (next - t > 256) next = t + 256;
      /* core/main.c:384: a tecplot dump on every step t (counted from 1) with
       * t % chPoint_tecplot == 0. */
      /* The same for the spectral dumps (core/main.c:395). */
      const int every[2] = {cfg.tecplot, cfg.spectr};
      for (int q = 0 ; q < 2 ; ++q)
         if (every[q] > 0) {
            const int nd = (t/every[q] + 1)*every[q];
            if (nd - 1 > t && nd - 1 < next) next = nd - 1;
         }
      int k = next - t;
      const int tec = cfg.tecplot > 0 && (t + 1) % cfg.tecplot == 0;
      const int spectr = cfg.spectr > 0 && (t + 1) % cfg.spectr == 0;
      if (tec || spectr) {
         staged_step (run, &rec, &dom, nodes, time, rows, tec, spectr, &probes, &tfsf);
         k = 1;
         next = t + 1;
      } else {
         tfsf_before (&tfsf, run, k);
         check (mg_run_step (run, k, rows), "step");
         probes_write (run, &probes, k);
         tfsf_after (&tfsf, run, k);
      }
      for (int q = 0 ; q < k ; ++q)
         diag_add (&diag, rows + 6*q);
      t = next;
      time += k*dom.tau;
      for (int q = 0 ; q < k ; ++q) {
         const double *r = rows + 6*q;
         if (isnan (r[1] + r[2] + r[3] + r[4] + r[5]))
            die ("%s", "nan detected in the energies");
      }
      if (t % cfg.full == 0) {
         checkpoint (&ckpt, run, &rec, &dom, nodes, time);
         diag_flush (&diag, &fresh_diag, dom.tau);
         last_saved = time;
      }
      if (t % cfg.stop == 0) {
         const double per_step = (now () - t_loop)/t;
         stop = stop_requested (t_start, per_step, cfg.stop, save_time);
      }
   }
   const double loop = now () - t_loop;
   printf ("main: main loop have taken %f sec.\n", loop);
   if (last_saved != time) {
      printf ("Additional check-point to save the final state.\n");
      checkpoint (&ckpt, run, &rec, &dom, nodes, time);
   }
   ckpt_free (&ckpt);
   diag_flush (&diag, &fresh_diag, dom.tau);
   free (diag.rows);
   check (mg_run_destroy (run), "destroy run");
   probes_close (&probes);
   tfsf_close (&tfsf);
   remove ("tmp/stop.flag");
   return EXIT_SUCCESS;
}
