// The reference's own marker placers (setup.out tags), on the device:
//
//   [plasma] + [DF:Maxwell]  setup/tag_plasma.c:88-152, setup/tag_maxwell.c:36-168
//   [DF:foil]                 setup/tag_foil.c:60-230
//
// Marker positions, and the pattern lookup of the Maxwell tag, run on the
// GPU; the per-cell velocity pattern (a few hundred entries) and the unit
// conversions are host code.  Both follow the reference's expressions in the
// same operation order, so positions, momenta and weights come out
// bit-identical to setup.out's.  Markers are produced in the reference's
// order (cells I-major, then the in-cell lattice x-major) with consecutive
// ids, as setup/plasma.c writes them.
#include <cuda_runtime.h>

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "mg_internal.cuh"

#define TRY_T(x)                                                             \
   do {                                                                      \
      int rc_ = (x);                                                         \
      if (rc_ != MG_OK)                                                      \
         return rc_;                                                         \
   } while (0)

namespace {

// ---- host: units (misc_units.c:95-120), quiet start, mapper ---------------
const double PI = 3.141592653589793238462643;        // misc_units.h:39
const double CGS_C = 2.9979e+10, CGS_E = 4.8032e-10, CGS_M = 9.1094e-28;   // misc_units.h:34-36

struct Units {
   double rho0, ncr;
};

Units units_for (double lambda)
{
   const double v = CGS_C, t = lambda/v;
   const double omega = 2*PI/t;
   const double n = CGS_M*omega*omega/(16*PI*PI*PI*CGS_E*CGS_E);
   Units u;
   u.rho0 = CGS_E*n;
   u.ncr = omega*omega*CGS_M/(4*PI*CGS_E*CGS_E);
   return u;
}

// Radix-`radix` digit reversal of num (setup_denavit.c:24-36).
double bit_reverse (int num, int radix)
{
   double res = 0, inv = 1.0/(double) radix, w = inv;
   while (num > 0) {
      const int digit = num % radix;
      num /= radix;
      res += digit*w;
      w *= inv;
   }
   return res;
}

// Integral mapper of f over [x0, x1] with N intervals (setup_distrMapper.c:
// quadratic splines through three points, blended integrals, normalised).
struct Mapper {
   int N;
   double *f, *x;
};

double fmaxw (double x) { return exp (- x*x); }

inline double int_all (double h, double a, double b, double c) { return a*h*h*h/3.0 + 0.5*b*h*h + c*h; }
inline double int_right (double h, double a, double b, double c) { return a*h*h*h/4.0 + b*h*h/3.0 + 0.5*c*h; }
inline double int_left (double h, double a, double b, double c) { return int_all (h, a, b, c) - int_right (h, a, b, c); }
inline void quad (double h, double y0, double y1, double y2, double &a, double &b, double &c)
{
   a = (y2 - 2*y1 + y0)/(2*h*h);
   b = (y2 - y0)/(2*h);
   c = y1;
}

Mapper mapper_make (double xmin, double xmax, int N)
{
   Mapper m;
   m.N = N;
   m.f = (double *) malloc (sizeof (double)*(N + 1));
   m.x = (double *) malloc (sizeof (double)*(N + 1));
   const double dx = (xmax - xmin)/(double) N;
   double x = xmin + dx;
   double y0 = fmaxw (x - dx), y1 = fmaxw (x), y2 = fmaxw (x + dx), sum;
   double a, b, c;
   m.x[0] = xmin;
   m.f[0] = 0;
   quad (dx, y0, y1, y2, a, b, c);
   m.x[1] = x;
   sum = m.f[1] = int_all (dx, a, -b, c);
   x += dx;
   for (int i = 2 ; i < N ; ++i) {
      const double y3 = fmaxw (x + dx);
      double A, B, Cc;
      quad (dx, y1, y2, y3, A, B, Cc);
      sum += int_left (dx, a, b, c) + int_left (dx, A, -B, Cc);
      m.f[i] = sum;
      m.x[i] = x;
      x += dx;
      y0 = y1;
      y1 = y2;
      y2 = y3;
      a = A;
      b = B;
      c = Cc;
   }
   sum += int_all (dx, a, b, c);
   m.f[N] = sum;
   m.x[N] = x;
   sum = 1.0/m.f[N];
   for (int i = 1 ; i <= N ; i++)
      m.f[i] *= sum;
   (void) y0;
   return m;
}

// x with F(x) = y (setup_distrMapper.c: bisection, then two quadratic
// guesses blended linearly; linear at the ends).
double mapper_invoke (double y, const Mapper &m)
{
   int iL = 0, iR = m.N;
   while (iR - iL > 1) {
      const int i = (iL + iR) >> 1;
      if (y < m.f[i])
         iR = i;
      else
         iL = i;
   }
   if (iL == 0 || iL == m.N - 1) {
      const double delta = (y - m.f[iL])/(m.f[iL + 1] - m.f[iL]);
      return m.x[iL] + delta*(m.x[iL + 1] - m.x[iL]);
   }
   double x0 = m.f[iL - 1], x1 = m.f[iL], x2 = m.f[iL + 1];
   double y0 = m.x[iL - 1], y1 = m.x[iL], y2 = m.x[iL + 1];
   double a = ((y2 - y1)/(x2 - x1) - (y0 - y1)/(x0 - x1))/(x2 - x0);
   double b = (y2 - y1)/(x2 - x1) - a*(x2 - x1);
   double dy = y - m.f[iL], left = a*dy*dy + b*dy + m.x[iL];
   x0 = m.f[iL];
   x1 = m.f[iL + 1];
   x2 = m.f[iL + 2];
   y0 = m.x[iL];
   y1 = m.x[iL + 1];
   y2 = m.x[iL + 2];
   a = ((y2 - y1)/(x2 - x1) - (y0 - y1)/(x0 - x1))/(x2 - x0);
   b = (y2 - y1)/(x2 - x1) - a*(x2 - x1);
   dy = y - m.f[iL + 1];
   const double right = a*dy*dy + b*dy + m.x[iL + 1];
   return - dy/(m.f[iL + 1] - m.f[iL])*left + (1.0 + dy/(m.f[iL + 1] - m.f[iL]))*right;
}

struct Pattern {
   double vx, vy, vz, rho;
};

// The per-cell velocity pattern of tag_maxwell (setup/tag_maxwell.c:84-158).
int maxwell_pattern (const mg_maxwell_t *s, Pattern *pat, int ppc)
{
   const double VMAX = 6.0, WING = 1.6;                  // tag_maxwell.c:20-21
   const int SAMPLES = 5000;
   const double rho = s->omega_pe2*4*PI*PI/s->qDivM/(double) ppc;
   Mapper all = mapper_make (- VMAX, + VMAX, SAMPLES), pos = mapper_make (0, + VMAX, SAMPLES);
   for (int i = 0, p = 0 ; i < s->nx ; ++i)
      for (int j = 0 ; j < s->ny ; ++j)
         for (int k = 0 ; k < s->nz ; ++k)
            for (int l = 0 ; l < s->layers/2 ; ++l) {
               double vx = bit_reverse (p/2 + 1, 2), vy = bit_reverse (p/2 + 1, 3),
                      vz = bit_reverse (p/2 + 1, 5);
               if (s->uniform_weight) {
                  vx = mapper_invoke (vx, pos);
                  vy = mapper_invoke (vy, all);
                  vz = mapper_invoke (vz, all);
                  pat[p].rho = 1.0;
               } else {
                  vx *= WING;
                  vy = WING*2*(vy - 0.5);
                  vz = WING*2*(vz - 0.5);
                  pat[p].rho = fmaxw (vx)*fmaxw (vy)*fmaxw (vz);
               }
               pat[p].vx = vx*s->ux;
               pat[p].vy = vy*s->uy;
               pat[p].vz = vz*s->uz;
               ++p;
               pat[p].vx = - vx*s->ux;
               pat[p].vy = - vy*s->uy;
               pat[p].vz = - vz*s->uz;
               pat[p].rho = pat[p - 1].rho;
               ++p;
            }
   for (Mapper *m : {&all, &pos}) {
      free (m->f);
      free (m->x);
   }
   double norm = 0;
   for (int p = 0 ; p < ppc ; ++p)
      norm += pat[p].rho;
   norm = ppc*rho/norm;
   for (int p = 0 ; p < ppc ; ++p)
      pat[p].rho *= norm;
   if (s->tune_energy) {
      double Wx = 0, Wy = 0, Wz = 0;
      for (int p = 0 ; p < ppc ; ++p) {
         Wx += pat[p].vx*pat[p].vx*pat[p].rho;
         Wy += pat[p].vy*pat[p].vy*pat[p].rho;
         Wz += pat[p].vz*pat[p].vz*pat[p].rho;
      }
      if (Wx == 0 || Wy == 0 || Wz == 0) {
         mg_set_error ("mg_run_place_maxwell: zero temperature on an axis with tune_energy");
         return MG_ERR_ARG;
      }
      Wx = s->ux*sqrt (rho*ppc*0.5/Wx);
      Wy = s->uy*sqrt (rho*ppc*0.5/Wy);
      Wz = s->uz*sqrt (rho*ppc*0.5/Wz);
      for (int p = 0 ; p < ppc ; ++p) {
         pat[p].vx *= Wx;
         pat[p].vy *= Wy;
         pat[p].vz *= Wz;
      }
   }
   return MG_OK;
}

// ---- device -----------------------------------------------------------------
struct Lattice {
   int n[3], nx, ny, nz, layers, ppc;
   double h[3], dx, dy, dz;
   float qm;
   int id0;
};

// One thread per marker of [plasma]: cell (I, J, K) I-major, in-cell index
// p = ((i ny + j) nz + k) layers + l; x = (i + 1/2) dx + I h1 (the in-cell
// position, then the cell's corner added, tag_plasma.c:99-122).
__global__ void k_lattice (Lattice L, const Pattern *pat, Markers64 m, long long at, long long first,
                           long long count)
{
   for (long long qq = blockIdx.x*(long long) blockDim.x + threadIdx.x ; qq < count ;
        qq += (long long) gridDim.x*blockDim.x) {
      const long long q = first + qq;
      const long long cell = q/L.ppc;
      const int p = (int) (q - cell*L.ppc);
      const int K = (int) (cell % L.n[2]), J = (int) ((cell/L.n[2]) % L.n[1]), I = (int) (cell/((long long) L.n[2]*L.n[1]));
      const int l = p % L.layers, s = p/L.layers;
      const int k = s % L.nz, j = (s/L.nz) % L.ny, i = s/(L.nz*L.ny);
      double x = (i + 0.5)*L.dx, y = (j + 0.5)*L.dy, z = (k + 0.5)*L.dz;
      x += I*L.h[0];
      y += J*L.h[1];
      z += K*L.h[2];
      (void) l;
      const long long o = at + qq;
      m.x[o] = x;
      m.y[o] = y;
      m.z[o] = z;
      m.ux[o] = pat[p].vx;
      m.uy[o] = pat[p].vy;
      m.uz[o] = pat[p].vz;
      m.rho[o] = (float) pat[p].rho;
      m.qm[o] = L.qm;
      m.id[o] = L.id0 + (int) q;
   }
}

struct Foil {
   int lo[3], hi[3];             // cells [lo, hi]
   int nx, ny, nz;
   double h[3], dx, dy, dz;
   double x0, y0, z0, lx, ly, lz, width, shift, margin;
   double n1, n2, weight;
   int profile;
   float qm;
   int id0;
};

__device__ __forceinline__ bool foil_alpha (const Foil &F, int I, int J, int K, int i, int j, int k,
                                            double &x, double &y, double &z, double &alpha)
{
   x = I*F.h[0] + (i + 0.5)*F.dx;
   y = J*F.h[1] + (j + 0.5)*F.dy;
   z = K*F.h[2] + (k + 0.5)*F.dz;
   alpha = F.shift - ((x - F.x0)*F.lx + (y - F.y0)*F.ly + (z - F.z0)*F.lz);
   alpha = alpha/F.width + 0.5;
   return !(alpha < F.margin || alpha > 1.0 - F.margin);
}

__device__ __forceinline__ void foil_cell (const Foil &F, long long c, int &I, int &J, int &K)
{
   const int nk = F.hi[2] - F.lo[2] + 1, nj = F.hi[1] - F.lo[1] + 1;
   K = F.lo[2] + (int) (c % nk);
   J = F.lo[1] + (int) ((c/nk) % nj);
   I = F.lo[0] + (int) (c/((long long) nk*nj));
}

// Markers of each cell inside the slab.
__global__ void k_foil_count (Foil F, long long cells, int *count)
{
   for (long long c = blockIdx.x*(long long) blockDim.x + threadIdx.x ; c < cells ;
        c += (long long) gridDim.x*blockDim.x) {
      int I, J, K, n = 0;
      foil_cell (F, c, I, J, K);
      for (int i = 0 ; i < F.nx ; ++i)
         for (int j = 0 ; j < F.ny ; ++j)
            for (int k = 0 ; k < F.nz ; ++k) {
               double x, y, z, a;
               n += foil_alpha (F, I, J, K, i, j, k, x, y, z, a);
            }
      count[c] = n;
   }
}

// Writes each cell's markers from its first slot (exclusive prefix of the
// counts), in the in-cell order of tag_foil.c:187-212.
__global__ void k_foil_write (Foil F, long long cells, const long long *first, Markers64 m, long long at)
{
   for (long long c = blockIdx.x*(long long) blockDim.x + threadIdx.x ; c < cells ;
        c += (long long) gridDim.x*blockDim.x) {
      int I, J, K;
      foil_cell (F, c, I, J, K);
      long long o = first[c];
      for (int i = 0 ; i < F.nx ; ++i)
         for (int j = 0 ; j < F.ny ; ++j)
            for (int k = 0 ; k < F.nz ; ++k) {
               double x, y, z, a;
               if (!foil_alpha (F, I, J, K, i, j, k, x, y, z, a))
                  continue;
               // alpha passes through the marker's float rho field first
               // (tag_foil.c:208-210, 217-227).
               const double af = (double) (float) a;
               const double rho = F.profile == 0 ? F.weight*(F.n1 + (F.n2 - F.n1)*af)
                                                 : F.weight*F.n1*pow (F.n2/F.n1, af);
               m.x[at + o] = x;
               m.y[at + o] = y;
               m.z[at + o] = z;
               m.ux[at + o] = 0;
               m.uy[at + o] = 0;
               m.uz[at + o] = 0;
               m.rho[at + o] = (float) rho;
               m.qm[at + o] = F.qm;
               m.id[at + o] = F.id0 + (int) o;
               ++o;
            }
   }
}

// Exclusive prefix sum of n counts into first[0..n] (first[n] = total), one
// block of 1024 threads, each over a contiguous segment.
__global__ void k_prefix (const int *count, long long n, long long *first)
{
   __shared__ long long part[1024];
   const long long per = (n + blockDim.x - 1)/blockDim.x;
   const long long b = threadIdx.x*per, e = (b + per < n) ? b + per : n;
   long long acc = 0;
   for (long long q = b ; q < e ; ++q)
      acc += count[q];
   part[threadIdx.x] = acc;
   __syncthreads ();
   for (int d = 1 ; d < (int) blockDim.x ; d <<= 1) {
      const long long v = threadIdx.x >= (unsigned) d ? part[threadIdx.x - d] : 0;
      __syncthreads ();
      part[threadIdx.x] += v;
      __syncthreads ();
   }
   long long run = part[threadIdx.x] - acc;
   for (long long q = b ; q < e ; ++q) {
      first[q] = run;
      run += count[q];
   }
   if (threadIdx.x == blockDim.x - 1)
      first[n] = part[threadIdx.x];
}

} // namespace

int mg_ensure_capacity64 (mg_run_t *r, long long need);
int mg_ensure_capacity32 (mg_run_t *r, long long need);
void mg_convert64to32 (mg_run_t *r, const Markers64 &v, long long c, long long at);

// FP64 target arrays for `count` markers: the run's arrays at r->np, or (the
// precision form) a Markers64 view of the staging buffer.
static int target (mg_run_t *r, long long count, Markers64 &v, long long &at)
{
   if (r->prm.precision == MG_FP64) {
      TRY_T (mg_ensure_capacity64 (r, r->np + count));
      v = r->m64;
      at = r->np;
      return MG_OK;
   }
   TRY_T (mg_ensure_capacity32 (r, r->np + count));
   TRY_T (mg_ensure_stage (r, (size_t) (count > 0 ? count : 1)*sizeof (mg_marker_t)));
   char *base = (char *) r->stage;
   v.x = (double *) base;
   v.y = v.x + count; v.z = v.y + count; v.ux = v.z + count; v.uy = v.ux + count; v.uz = v.uy + count;
   v.rho = (float *) (v.uz + count);
   v.qm = v.rho + count;
   v.id = (int *) (v.qm + count);
   at = 0;
   return MG_OK;
}

static int commit (mg_run_t *r, const Markers64 &v, long long count)
{
   if (r->prm.precision != MG_FP64)
      mg_convert64to32 (r, v, count, r->np);
   MG_LAUNCH_CHECK ();
   MG_CUDA (cudaStreamSynchronize (r->stream));
   r->np += count;
   r->inited = 0;
   r->tiles_ok = 0;
   return MG_OK;
}

// Markers per pass through the staging buffer of the precision form.
static const long long STAGE_MARKERS = 1LL << 26;

extern "C" int mg_run_place_maxwell (mg_run_t *r, const mg_maxwell_t *s)
{
   if (!r || !s) {
      mg_set_error ("mg_run_place_maxwell: null argument");
      return MG_ERR_ARG;
   }
   MG_CUDA (cudaSetDevice (r->device));
   // tag_maxwell.c:45-46: rho = omega_pe2 4 pi^2/qDivM/PPC must share the sign of qDivM.
   if (s->nx <= 0 || s->ny <= 0 || s->nz <= 0 || s->layers <= 0 || s->layers % 2 || s->qDivM == 0 ||
       !(s->omega_pe2 > 0)) {
      mg_set_error ("mg_run_place_maxwell: lattice %dx%dx%d, %d layers (even), q/M %g (non-zero) and "
                    "omega_pe^2 %g (> 0) expected", s->nx, s->ny, s->nz, s->layers, s->qDivM, s->omega_pe2);
      return MG_ERR_ARG;
   }
   Lattice L;
   L.nx = s->nx; L.ny = s->ny; L.nz = s->nz; L.layers = s->layers;
   L.ppc = s->nx*s->ny*s->nz*s->layers;
   for (int a = 0 ; a < 3 ; ++a) {
      L.n[a] = r->g.n[a];
      L.h[a] = r->g.h[a];
   }
   L.dx = r->g.h[0]*1/(double) s->nx;
   L.dy = r->g.h[1]*1/(double) s->ny;
   L.dz = r->g.h[2]*1/(double) s->nz;
   L.qm = (float) s->qDivM;
   L.id0 = s->id0;
   Pattern *hp = (Pattern *) malloc (sizeof (Pattern)*L.ppc);
   int rc = maxwell_pattern (s, hp, L.ppc);
   if (rc != MG_OK) {
      free (hp);
      return rc;
   }
   const long long count = (long long) L.ppc*L.n[0]*L.n[1]*L.n[2];
   Pattern *dp = nullptr;
   if (cudaMalloc (&dp, sizeof (Pattern)*L.ppc) != cudaSuccess) {
      mg_set_error ("mg_run_place_maxwell: device allocation failed");
      rc = MG_ERR_OOM;
   }
   if (rc == MG_OK) {
      cudaMemcpyAsync (dp, hp, sizeof (Pattern)*L.ppc, cudaMemcpyHostToDevice, r->stream);
      if (r->prm.precision == MG_FP64)
         rc = mg_ensure_capacity64 (r, r->np + count);
      else
         rc = mg_ensure_capacity32 (r, r->np + count);
   }
   const long long chunk = r->prm.precision == MG_FP64 ? (count > 0 ? count : 1) : STAGE_MARKERS;
   for (long long done = 0 ; rc == MG_OK && done < count ; done += chunk) {
      const long long c = (count - done < chunk) ? count - done : chunk;
      Markers64 v;
      long long at = 0;
      rc = target (r, c, v, at);
      if (rc == MG_OK) {
         k_lattice<<<mg_blocks_for (c, 256, 8), 256, 0, r->stream>>> (L, dp, v, at, done, c);
         rc = commit (r, v, c);
      }
   }
   if (dp) cudaFree (dp);
   free (hp);
   return rc;
}

extern "C" int mg_run_place_foil (mg_run_t *r, const mg_foil_t *s)
{
   if (!r || !s) {
      mg_set_error ("mg_run_place_foil: null argument");
      return MG_ERR_ARG;
   }
   MG_CUDA (cudaSetDevice (r->device));
   Foil F;
   double lx = s->lx, ly = s->ly, lz = s->lz;
   const double l = sqrt (lx*lx + ly*ly + lz*lz);
   const double hsum = r->g.h[0] + r->g.h[1] + r->g.h[2];
   if (!(l > 1.0e-2) || !(s->width >= hsum/3) || s->nx <= 0 || s->ny <= 0 || s->nz <= 0 || s->M == 0 ||
       (s->profile != 0 && s->profile != 1) || !(s->lambda_cm > 0)) {
      mg_set_error ("mg_run_place_foil: bad normal, width (>= mean h), lattice, mass, profile or wavelength");
      return MG_ERR_ARG;
   }
   F.lx = lx/l; F.ly = ly/l; F.lz = lz/l;
   F.x0 = s->x0; F.y0 = s->y0; F.z0 = s->z0;
   F.width = s->width;
   F.shift = s->shift;
   F.profile = s->profile;
   // Densities as tag_foil.c:98-118 converts them.
   const Units u = units_for (s->lambda_cm);
   double n1 = s->n1, n2 = s->n2;
   n1 *= (n1 < 0) ? (- u.ncr) : 1;
   n2 *= (n2 < 0) ? (- u.ncr) : 1;
   n1 *= s->q*CGS_E/u.rho0;
   n2 *= s->q*CGS_E/u.rho0;
   F.n1 = n1;
   F.n2 = n2;
   F.nx = s->nx; F.ny = s->ny; F.nz = s->nz;
   for (int a = 0 ; a < 3 ; ++a)
      F.h[a] = r->g.h[a];
   F.dx = r->g.h[0]*1/(double) s->nx;
   F.dy = r->g.h[1]*1/(double) s->ny;
   F.dz = r->g.h[2]*1/(double) s->nz;
   F.margin = 1e-10*hsum/(3*s->width);
   F.weight = 1.0/((double) s->nx*s->ny*s->nz);
   F.qm = (float) (s->q/s->M);
   F.id0 = s->id0;
   for (int a = 0 ; a < 3 ; ++a) {
      const int m = 5*(r->g.bc[0][a] != MG_BC_PERIODIC);       // tag_foil.c:167-169
      F.lo[a] = m;
      F.hi[a] = r->g.n[a] - m - 1;
      if (F.hi[a] < F.lo[a])
         return MG_OK;
   }
   const long long cells = (long long) (F.hi[0] - F.lo[0] + 1)*(F.hi[1] - F.lo[1] + 1)*(F.hi[2] - F.lo[2] + 1);
   int *count = nullptr;
   long long *first = nullptr;
   if (cudaMalloc (&count, sizeof (int)*cells) != cudaSuccess ||
       cudaMalloc (&first, sizeof (long long)*(cells + 1)) != cudaSuccess) {
      if (count) cudaFree (count);
      mg_set_error ("mg_run_place_foil: device allocation failed");
      return MG_ERR_OOM;
   }
   k_foil_count<<<mg_blocks_for (cells, 256, 8), 256, 0, r->stream>>> (F, cells, count);
   k_prefix<<<1, 1024, 0, r->stream>>> (count, cells, first);
   long long total = 0;
   cudaMemcpyAsync (&total, first + cells, sizeof (total), cudaMemcpyDeviceToHost, r->stream);
   cudaError_t e = cudaStreamSynchronize (r->stream);
   int rc = MG_OK;
   if (e != cudaSuccess) {
      mg_set_error ("mg_run_place_foil: %s", cudaGetErrorString (e));
      rc = MG_ERR_CUDA;
   }
   Markers64 v;
   long long at = 0;
   if (rc == MG_OK && total > 0)
      rc = target (r, total, v, at);
   if (rc == MG_OK && total > 0) {
      k_foil_write<<<mg_blocks_for (cells, 256, 8), 256, 0, r->stream>>> (F, cells, first, v, at);
      rc = commit (r, v, total);
   }
   cudaFree (count);
   cudaFree (first);
   return rc;
}

// ---------------------------------------------------------------------------
// [DF:uniform] (setup/tag_DF_uniform.c:36-70): velocities of markers already
// placed, u = u0 + (rand ()/RAND_MAX - 1/2) du per axis, drawn from the C
// library's rand () (three draws per marker, x then y then z).
//
// rand () of the GNU C library with the default seed is the additive
// feedback generator published in its random(3) sources: r_0 = 1,
// r_i = 16807 r_(i-1) mod (2^31 - 1) for i < 31, r_i = r_(i-31) for
// i = 31..33, r_i = r_(i-3) + r_(i-31) mod 2^32 after that, and draw k is
// r_(k+344) >> 1.  The recurrence is linear over the integers mod 2^32, so
// the 31-value window at any draw is a power of its 31 x 31 step matrix
// applied to the window at draw 0; each thread starts from its own window
// and steps its draws in order.
// ---------------------------------------------------------------------------
namespace {

typedef unsigned int u32;
const int LAG = 31;

struct Mat31 { u32 a[LAG][LAG]; };

Mat31 mat_mul (const Mat31 &x, const Mat31 &y)
{
   Mat31 z;
   for (int i = 0 ; i < LAG ; ++i)
      for (int j = 0 ; j < LAG ; ++j) {
         u32 s = 0;
         for (int k = 0 ; k < LAG ; ++k)
            s += x.a[i][k]*y.a[k][j];
         z.a[i][j] = s;
      }
   return z;
}

void mat_vec (const Mat31 &m, const u32 *v, u32 *out)
{
   u32 t[LAG];
   for (int i = 0 ; i < LAG ; ++i) {
      u32 s = 0;
      for (int k = 0 ; k < LAG ; ++k)
         s += m.a[i][k]*v[k];
      t[i] = s;
   }
   memcpy (out, t, sizeof (t));
}

// One draw on a window (r_(i-31), ..., r_(i-1)) -> (r_(i-30), ..., r_i).
Mat31 step_matrix ()
{
   Mat31 m;
   memset (&m, 0, sizeof (m));
   for (int k = 0 ; k < LAG - 1 ; ++k)
      m.a[k][k + 1] = 1;
   m.a[LAG - 1][LAG - 3] = 1;
   m.a[LAG - 1][0] = 1;
   return m;
}

Mat31 mat_pow (long long e)
{
   Mat31 r, b = step_matrix ();
   memset (&r, 0, sizeof (r));
   for (int i = 0 ; i < LAG ; ++i)
      r.a[i][i] = 1;
   for ( ; e > 0 ; e >>= 1) {
      if (e & 1)
         r = mat_mul (r, b);
      b = mat_mul (b, b);
   }
   return r;
}

// The window before draw 0: r_313 .. r_343.
void rand_window0 (u32 *w)
{
   u32 r[344];
   long long s = 1;
   r[0] = 1;
   for (int i = 1 ; i < 31 ; ++i) {
      s = (16807*s) % 2147483647;
      r[i] = (u32) s;
   }
   for (int i = 31 ; i < 34 ; ++i)
      r[i] = r[i - 31];
   for (int i = 34 ; i < 344 ; ++i)
      r[i] = r[i - 3] + r[i - 31];
   memcpy (w, r + 344 - LAG, sizeof (u32)*LAG);
}

struct DfUniform {
   double u[3], du[3];
   float rho, qm;
};

template <typename U>
__global__ void k_df_uniform (U *ux, U *uy, U *uz, float *rho, float *qm, long long first, long long count,
                              long long per, int threads, const u32 *windows, DfUniform d)
{
   const int t = blockIdx.x*blockDim.x + threadIdx.x;
   if (t >= threads)
      return;
   u32 w[LAG];
   for (int k = 0 ; k < LAG ; ++k)
      w[k] = windows[(long long) t*LAG + k];
   int j = 0;
   const long long b = (long long) t*per, e = (b + per < count) ? b + per : count;
   for (long long q = b ; q < e ; ++q) {
      double v[3];
      for (int a = 0 ; a < 3 ; ++a) {
         const u32 x = w[(j + LAG - 3) % LAG] + w[j];
         w[j] = x;
         j = (j + 1) % LAG;
         const double f = (double) (int) (x >> 1)/(double) 2147483647;
         v[a] = d.u[a] + (f - 0.5)*d.du[a];
      }
      const long long o = first + q;
      ux[o] = (U) v[0];
      uy[o] = (U) v[1];
      uz[o] = (U) v[2];
      rho[o] = d.rho;
      qm[o] = d.qm;
   }
}

template <typename U>
__global__ void k_shift (U *ux, U *uy, U *uz, long long first, long long count, double dx, double dy, double dz)
{
   for (long long q = blockIdx.x*(long long) blockDim.x + threadIdx.x ; q < count ;
        q += (long long) gridDim.x*blockDim.x) {
      const long long o = first + q;
      ux[o] = (U) ((double) ux[o] + dx);
      uy[o] = (U) ((double) uy[o] + dy);
      uz[o] = (U) ((double) uz[o] + dz);
   }
}

struct TwoStream {
   int n[3];
   double d[3], v[3];
   float rho, qm;
   int id0;
};

__global__ void k_two_stream (TwoStream s, Markers64 m, long long at, long long first, long long count)
{
   for (long long qq = blockIdx.x*(long long) blockDim.x + threadIdx.x ; qq < count ;
        qq += (long long) gridDim.x*blockDim.x) {
      const long long q = first + qq, node = q/2;
      const int k = (int) (node % s.n[2]), j = (int) ((node/s.n[2]) % s.n[1]);
      const int i = (int) (node/((long long) s.n[2]*s.n[1]));
      const long long o = at + qq;
      m.x[o] = (i + 0.5)*s.d[0];
      m.y[o] = (j + 0.5)*s.d[1];
      m.z[o] = (k + 0.5)*s.d[2];
      m.ux[o] = (q & 1) ? - s.v[0] : s.v[0];
      m.uy[o] = (q & 1) ? - s.v[1] : s.v[1];
      m.uz[o] = (q & 1) ? - s.v[2] : s.v[2];
      m.rho[o] = s.rho;
      m.qm[o] = s.qm;
      m.id[o] = s.id0 + (int) q;
   }
}

int check_range (const mg_run_t *r, long long first, long long count, const char *fn)
{
   if (first < 0 || count < 0 || first + count > r->np) {
      mg_set_error ("%s: markers [%lld, %lld) outside the %lld placed", fn, first, first + count, r->np);
      return MG_ERR_ARG;
   }
   if (r->inited) {
      mg_set_error ("%s: markers are reordered by mg_run_init; apply tags before it", fn);
      return MG_ERR_STATE;
   }
   return MG_OK;
}

} // namespace

extern "C" int mg_run_df_uniform (mg_run_t *r, long long first, long long count, const mg_df_uniform_t *s)
{
   if (!r || !s) {
      mg_set_error ("mg_run_df_uniform: null argument");
      return MG_ERR_ARG;
   }
   TRY_T (check_range (r, first, count, "mg_run_df_uniform"));
   if (!(s->rho*s->qDivM > 0) || s->ppc <= 0 || !(s->lambda_cm > 0) || s->draws_before < 0) {
      mg_set_error ("mg_run_df_uniform: sign of rho differs from sign of q/M, or bad ppc, wavelength or draws");
      return MG_ERR_ARG;
   }
   if (count == 0)
      return MG_OK;
   MG_CUDA (cudaSetDevice (r->device));
   const Units u = units_for (s->lambda_cm);
   const double rho_crit = CGS_E*u.ncr/u.rho0;                     // tag_DF_uniform.c:38
   double rho = s->rho;
   rho *= rho_crit/s->ppc;                                           // :54
   DfUniform d;
   d.u[0] = s->ux; d.u[1] = s->uy; d.u[2] = s->uz;
   d.du[0] = s->dux; d.du[1] = s->duy; d.du[2] = s->duz;
   d.rho = (float) rho;
   d.qm = (float) s->qDivM;
   // Threads, each with a run of consecutive markers and its start window.
   const long long per = (count + 148*128 - 1)/(148*128) > 64 ? (count + 148*128 - 1)/(148*128) : 64;
   const int threads = (int) ((count + per - 1)/per);
   std::vector<u32> win ((size_t) threads*LAG);
   u32 w[LAG];
   rand_window0 (w);
   mat_vec (mat_pow (s->draws_before), w, w);
   const Mat31 jump = mat_pow (3*per);
   for (int t = 0 ; t < threads ; ++t) {
      memcpy (&win[(size_t) t*LAG], w, sizeof (w));
      if (t + 1 < threads)
         mat_vec (jump, w, w);
   }
   u32 *dw = nullptr;
   if (cudaMalloc (&dw, sizeof (u32)*win.size ()) != cudaSuccess) {
      mg_set_error ("mg_run_df_uniform: device allocation failed");
      return MG_ERR_OOM;
   }
   int rc = MG_OK;
   if (cudaMemcpy (dw, win.data (), sizeof (u32)*win.size (), cudaMemcpyHostToDevice) != cudaSuccess)
      rc = MG_ERR_CUDA;
   if (rc == MG_OK) {
      const int B = (threads + 127)/128;
      if (r->prm.precision == MG_FP64)
         k_df_uniform<double><<<B, 128, 0, r->stream>>> (r->m64.ux, r->m64.uy, r->m64.uz, r->m64.rho, r->m64.qm,
                                                        first, count, per, threads, dw, d);
      else
         k_df_uniform<float><<<B, 128, 0, r->stream>>> (r->m32.ux, r->m32.uy, r->m32.uz, r->m32.rho, r->m32.qm,
                                                       first, count, per, threads, dw, d);
      if (cudaGetLastError () != cudaSuccess || cudaStreamSynchronize (r->stream) != cudaSuccess) {
         mg_set_error ("mg_run_df_uniform: kernel failed");
         rc = MG_ERR_CUDA;
      }
   }
   cudaFree (dw);
   return rc;
}

extern "C" int mg_run_shift_velocity (mg_run_t *r, long long first, long long count, const double dv[3])
{
   if (!r || !dv) {
      mg_set_error ("mg_run_shift_velocity: null argument");
      return MG_ERR_ARG;
   }
   TRY_T (check_range (r, first, count, "mg_run_shift_velocity"));
   if (count == 0)
      return MG_OK;
   MG_CUDA (cudaSetDevice (r->device));
   const int B = mg_blocks_for (count, 256, 8);
   if (r->prm.precision == MG_FP64)
      k_shift<double><<<B, 256, 0, r->stream>>> (r->m64.ux, r->m64.uy, r->m64.uz, first, count, dv[0], dv[1], dv[2]);
   else
      k_shift<float><<<B, 256, 0, r->stream>>> (r->m32.ux, r->m32.uy, r->m32.uz, first, count, dv[0], dv[1], dv[2]);
   MG_LAUNCH_CHECK ();
   MG_CUDA (cudaStreamSynchronize (r->stream));
   return MG_OK;
}

extern "C" int mg_run_place_two_stream (mg_run_t *r, const mg_two_stream_t *s)
{
   if (!r || !s) {
      mg_set_error ("mg_run_place_two_stream: null argument");
      return MG_ERR_ARG;
   }
   if (s->n[0] <= 0 || s->n[1] <= 0 || s->n[2] <= 0 || !(s->gamma > 0) || !(fabs (s->qDivM) <= 1) ||
       s->qDivM == 0 || (s->m[0] == 0 && s->m[1] == 0 && s->m[2] == 0) ||
       !(s->L[0] > 0 && s->L[1] > 0 && s->L[2] > 0)) {
      mg_set_error ("mg_run_place_two_stream: bad input parameters");
      return MG_ERR_ARG;
   }
   MG_CUDA (cudaSetDevice (r->device));
   // setup/tag_twoStream.c:23-103 in its order.
   const int Nbeam = s->n[0]*s->n[1]*s->n[2];
   double rho = s->gamma*s->gamma/s->qDivM;
   const double kx = 2*PI*s->m[0]/s->L[0], ky = 2*PI*s->m[1]/s->L[1], kz = 2*PI*s->m[2]/s->L[2];
   const double kAbs = sqrt (kx*kx + ky*ky + kz*kz);
   const double V = s->gamma*sqrt (3.0)/(2*kAbs);
   TwoStream t;
   t.v[0] = V*kx/kAbs;
   t.v[1] = V*ky/kAbs;
   t.v[2] = V*kz/kAbs;
   rho *= s->L[0]*s->L[1]*s->L[2]/(r->g.h[0]*r->g.h[1]*r->g.h[2]*Nbeam);
   for (int a = 0 ; a < 3 ; ++a) {
      t.n[a] = s->n[a];
      t.d[a] = s->L[a]/(double) s->n[a];
   }
   t.rho = (float) rho;
   t.qm = (float) s->qDivM;
   t.id0 = s->id0;
   const long long total = 2LL*Nbeam;
   for (long long done = 0 ; done < total ; ) {
      const long long c = (total - done < STAGE_MARKERS) ? total - done : STAGE_MARKERS;
      Markers64 v;
      long long at = 0;
      TRY_T (target (r, c, v, at));
      k_two_stream<<<mg_blocks_for (c, 256, 8), 256, 0, r->stream>>> (t, v, at, done, c);
      TRY_T (commit (r, v, c));
      done += c;
   }
   return MG_OK;
}
