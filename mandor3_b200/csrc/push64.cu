// FP64 particle push: CIC gather of the staggered E and H, relativistic
// Boris rotation, position update, charge-conserving current deposition
// and particle boundary conditions, fused in one kernel.
//
// Reference semantics (paths relative to the reference project):
//   gather + Boris + move      core/plasma.c:106-171, misc_PIC.h:18-126
//   crossing classification    core/plasma.c:176-225
//   in-cell segment deposit    core/plasma_currentKernel.c:21-124
//   2- and 3-face crossings    core/plasma_currentKernel.c:157-279
//   thermal energy tally       core/plasma.c:140-143
//   particle walls             core/plasma_walls.c:27-104
//
// Compiled with --fmad=false: every product and sum rounds as the
// reference's C expressions do, so cell indices and per-marker updates are
// bit-identical given identical fields.
//
// Deposition: markers are stored in cell order (placement order, kept by
// the periodic sort), so consecutive lanes of a warp usually start in the
// same cell.  The twelve contributions of each marker's first segment (which
// always lies in its start cell) are summed across lanes that share the
// cell with a segmented warp scan (only as many rounds as the warp's longest
// run needs), and one lane per run of equal cells issues the twelve
// atomics.  (Letting every lane add its own weights when a warp spans many
// cells measured slower late in the laser-foil run: neighbouring cells
// share current nodes, so those atomics collide.)  Further segments of
// cell-crossing markers add their contributions directly.
#include <cuda_runtime.h>
#include <stdlib.h>

#include "mg_internal.cuh"

namespace {

// MF_DBL_TO_INT (misc_PIC.h:18) without conversion instructions: for
// y = s + 128 in [0, 2^31), t = y + 1.5*2^52 holds round(y) in the low bits
// of its significand, t - 1.5*2^52 is that integer as a double (exact), and
// one comparison turns rounding into truncation.  Returns the index as an
// int and, in fs, the same index as a double -- the values the reference's
// (int) cast and its int-to-double promotions produce.  Out-of-range input
// gives some integer, which the caller's range check rejects.
__device__ __forceinline__ int cell_of (double s, double &fs)
{
   const double M = 6755399441055744.0;
   const double y = s + 128.0;
   const double t = y + M;
   double r = t - M;
   int n = __double2loint (t);
   if (r > y) {
      r -= 1.0;
      n -= 1;
   }
   fs = r - 128.0;
   return n - 128;
}

struct Ctx {
   Grid   g;
   const double *E0, *E1, *E2, *H0, *H1, *H2;
   double *J0, *J1, *J2;
   // Correctly rounded reciprocals of the run's constant divisors: 1/h,
   // 1/((tau h2) h3), 1/((tau h1) h3), 1/((tau h1) h2) and 1/12.
   double rh[3], rjx, rjy, rjz, jdx, jdy, jdz;
};

// a/b for a divisor b known in advance, with y = RN(1/b): q0 = RN(a y),
// r = a - q0 b (exact with one fused multiply-add), q = RN(q0 + r y).  By
// Markstein's theorem (P. Markstein, IBM J. Res. Dev. 34(1), 1990; see also
// Muller et al., Handbook of Floating-Point Arithmetic, ch. 4) q is the
// correctly rounded quotient, i.e. bit-identical to the IEEE division the
// reference performs, for normal a and b.
__device__ __forceinline__ double div_by (double a, double b, double y)
{
   const double q0 = a*y;
   const double r = __fma_rn (-q0, b, a);
   return __fma_rn (r, y, q0);
}

#define R12 (1.0/12.0)

// 1/b for the thermal tally: the hardware's approximate reciprocal refined
// by two Newton-Raphson steps y <- y + y (1 - b y), each roughly doubling
// the correct bits (about 2^-23 after the first, below 2^-50 after the
// second), for |b| in the normal range.
__device__ __forceinline__ double recip (double b)
{
   double y;
   asm ("rcp.approx.ftz.f64 %0, %1;" : "=d" (y) : "d" (b));
   double e = __fma_rn (-b, y, 1.0);
   y = __fma_rn (y, e, y);
   e = __fma_rn (-b, y, 1.0);
   return __fma_rn (y, e, y);
}

__device__ __forceinline__ double cic (const double *F, const Grid &g, int i, double sx,
                                       int j, double sy, int k, double sz)
{
   const long o = g.at (i, j, k), Sx = g.sx, Sy = g.sy;
   // Fields are read-only during the push: the eight corners go through
   // the non-coherent read-only path, all issued before the sum.
   const double f0 = __ldg (F + o), f1 = __ldg (F + o + Sx);
   const double f2 = __ldg (F + o + Sy), f3 = __ldg (F + o + Sx + Sy);
   const double f4 = __ldg (F + o + 1), f5 = __ldg (F + o + Sx + 1);
   const double f6 = __ldg (F + o + Sy + 1), f7 = __ldg (F + o + Sx + Sy + 1);
   return f0*(1 - sx)*((1 - sy)*(1 - sz)) + f1*sx*((1 - sy)*(1 - sz))
        + f2*(1 - sx)*(sy*(1 - sz)) + f3*sx*(sy*(1 - sz))
        + f4*(1 - sx)*((1 - sy)*sz) + f5*sx*((1 - sy)*sz)
        + f6*(1 - sx)*(sy*sz) + f7*sx*(sy*sz);
}

// The twelve weights of one in-cell segment, in the reference's order:
// Jx at (i+1, j|j+1, k|k+1), Jy at (i|i+1, j+1, k|k+1), Jz at (i|i+1, j|j+1, k+1).
__device__ __forceinline__ void segment_weights (const Ctx &c, double fi, double fj, double fk,
                                                 double x1, double x2, double y1, double y2,
                                                 double z1, double z2, double rho, double w[12])
{
   const Grid &g = c.g;
   const double h1 = g.h[0], h2 = g.h[1], h3 = g.h[2];
   const double dX = x2 - x1, dY = y2 - y1, dZ = z2 - z1;
   const double tX = 0.5*(x1 + x2) - fi*h1;
   const double tY = 0.5*(y1 + y2) - fj*h2;
   const double tZ = 0.5*(z1 + z2) - fk*h3;
   const double ax = div_by (rho*dX, c.jdx, c.rjx), dyz = div_by (dY*dZ, 12.0, R12);
   w[0] = ax*((h2 - tY)*(h3 - tZ) + dyz);
   w[1] = ax*(tY*(h3 - tZ) - dyz);
   w[2] = ax*((h2 - tY)*tZ - dyz);
   w[3] = ax*(tY*tZ + dyz);
   const double ay = div_by (rho*dY, c.jdy, c.rjy), dxz = div_by (dX*dZ, 12.0, R12);
   w[4] = ay*((h1 - tX)*(h3 - tZ) + dxz);
   w[5] = ay*(tX*(h3 - tZ) - dxz);
   w[6] = ay*((h1 - tX)*tZ - dxz);
   w[7] = ay*(tX*tZ + dxz);
   const double az = div_by (rho*dZ, c.jdz, c.rjz), dxy = div_by (dX*dY, 12.0, R12);
   w[8] = az*((h1 - tX)*(h2 - tY) + dxy);
   w[9] = az*(tX*(h2 - tY) - dxy);
   w[10] = az*((h1 - tX)*tY - dxy);
   w[11] = az*(tX*tY + dxy);
}

__device__ __forceinline__ void scatter12 (const Ctx &c, int i, int j, int k, const double w[12])
{
   const long o = c.g.at (i, j, k), sx = c.g.sx, sy = c.g.sy;
   atomicAdd (c.J0 + o + sx, w[0]);
   atomicAdd (c.J0 + o + sx + sy, w[1]);
   atomicAdd (c.J0 + o + sx + 1, w[2]);
   atomicAdd (c.J0 + o + sx + sy + 1, w[3]);
   atomicAdd (c.J1 + o + sy, w[4]);
   atomicAdd (c.J1 + o + sx + sy, w[5]);
   atomicAdd (c.J1 + o + sy + 1, w[6]);
   atomicAdd (c.J1 + o + sx + sy + 1, w[7]);
   atomicAdd (c.J2 + o + 1, w[8]);
   atomicAdd (c.J2 + o + sx + 1, w[9]);
   atomicAdd (c.J2 + o + sy + 1, w[10]);
   atomicAdd (c.J2 + o + sx + sy + 1, w[11]);
}

__device__ __forceinline__ void deposit_direct (const Ctx &c, int i, int j, int k,
                                                double x1, double x2, double y1, double y2,
                                                double z1, double z2, double rho)
{
   double w[12];
   segment_weights (c, (double) i, (double) j, (double) k, x1, x2, y1, y2, z1, z2, rho, w);
   scatter12 (c, i, j, k, w);
}

// plasmaCurrents_multiCellStep (core/plasma_currentKernel.c:157-279) for
// everything after the first segment, which the caller has deposited.
// Returns the end point of the first segment in (xa, ya, za).
__device__ void multicell_first (const Grid &g, int i1, int j1, int k1, int i2, int j2, int k2,
                                 double x1, double y1, double z1, double x2, double y2, double z2,
                                 double &xa, double &ya, double &za)
{
   const double h1 = g.h[0], h2 = g.h[1], h3 = g.h[2];
   const int di = abs (i2 - i1), dj = abs (j2 - j1), dk = abs (k2 - k1);
   if (di + dj + dk == 2) {
      const double sX = di*((i1 + i2 + 1)*0.5*h1 - x1)/(x2 - x1 + ((1 - di) << 16));
      const double sY = dj*((j1 + j2 + 1)*0.5*h2 - y1)/(y2 - y1 + ((1 - dj) << 16));
      const double sZ = dk*((k1 + k2 + 1)*0.5*h3 - z1)/(z2 - z1 + ((1 - dk) << 16));
      double kap1 = sX + (1 - di)*sY;
      double kap2 = sZ + (1 - dk)*sY;
      if (kap1 > kap2) {
         const double t = kap1;
         kap1 = kap2;
         kap2 = t;
      }
      xa = x1 + kap1*(x2 - x1);
      ya = y1 + kap1*(y2 - y1);
      za = z1 + kap1*(z2 - z1);
      return;
   }
   const double xC = (i1 + i2 + 1)*0.5*h1, yC = (j1 + j2 + 1)*0.5*h2, zC = (k1 + k2 + 1)*0.5*h3;
   double s1 = (xC - x1)/(x2 - x1), s2 = (yC - y1)/(y2 - y1), s3 = (zC - z1)/(z2 - z1);
   double rc[3][3];
   rc[0][0] = xC;
   rc[0][1] = y1 + s1*(y2 - y1);
   rc[0][2] = z1 + s1*(z2 - z1);
   rc[1][0] = x1 + s2*(x2 - x1);
   rc[1][1] = yC;
   rc[1][2] = z1 + s2*(z2 - z1);
   rc[2][0] = x1 + s3*(x2 - x1);
   rc[2][1] = y1 + s3*(y2 - y1);
   rc[2][2] = zC;
   int a = 0, b = 1, cc = 2;
   if (s1 > s2) { int t = a; a = b; b = t; double u = s1; s1 = s2; s2 = u; }
   if (s1 > s3) { int t = a; a = cc; cc = t; double u = s1; s1 = s3; s3 = u; }
   (void) b;
   xa = rc[a][0];
   ya = rc[a][1];
   za = rc[a][2];
}

__device__ void multicell_rest (const Ctx &c, int i1, int j1, int k1, int i2, int j2, int k2,
                                double x1, double y1, double z1, double x2, double y2, double z2,
                                double rho)
{
   const Grid &g = c.g;
   const double h1 = g.h[0], h2 = g.h[1], h3 = g.h[2];
   const int di = abs (i2 - i1), dj = abs (j2 - j1), dk = abs (k2 - k1);
   if (di + dj + dk == 2) {
      int i = i1, j = j1, k = k1;
      const double sX = di*((i1 + i2 + 1)*0.5*h1 - x1)/(x2 - x1 + ((1 - di) << 16));
      const double sY = dj*((j1 + j2 + 1)*0.5*h2 - y1)/(y2 - y1 + ((1 - dj) << 16));
      const double sZ = dk*((k1 + k2 + 1)*0.5*h3 - z1)/(z2 - z1 + ((1 - dk) << 16));
      double kap1 = sX + (1 - di)*sY;
      double kap2 = sZ + (1 - dk)*sY;
      int d[2][3] = {{0, 0, 0}, {0, 0, 0}};
      int first = 0;
      d[0][0] = di*(i2 - i1);
      d[0][1] = (1 - di)*(j2 - j1);
      d[1][1] = (1 - dk)*(j2 - j1);
      d[1][2] = dk*(k2 - k1);
      if (kap1 > kap2) {
         const double t = kap1;
         kap1 = kap2;
         kap2 = t;
         first = 1;
      }
      const double xA = x1 + kap1*(x2 - x1), yA = y1 + kap1*(y2 - y1), zA = z1 + kap1*(z2 - z1);
      const double xB = x1 + kap2*(x2 - x1), yB = y1 + kap2*(y2 - y1), zB = z1 + kap2*(z2 - z1);
      i += d[first][0];
      j += d[first][1];
      k += d[first][2];
      deposit_direct (c, i, j, k, xA, xB, yA, yB, zA, zB, rho);
      i += d[1 - first][0];
      j += d[1 - first][1];
      k += d[1 - first][2];
      deposit_direct (c, i, j, k, xB, x2, yB, y2, zB, z2, rho);
      return;
   }
   const double xC = (i1 + i2 + 1)*0.5*h1, yC = (j1 + j2 + 1)*0.5*h2, zC = (k1 + k2 + 1)*0.5*h3;
   double s1 = (xC - x1)/(x2 - x1), s2 = (yC - y1)/(y2 - y1), s3 = (zC - z1)/(z2 - z1);
   double rc[3][3];
   int dI[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
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
   int a = 0, b = 1, cc = 2;
   if (s1 > s2) { int t = a; a = b; b = t; double u = s1; s1 = s2; s2 = u; }
   if (s1 > s3) { int t = a; a = cc; cc = t; double u = s1; s1 = s3; s3 = u; }
   if (s2 > s3) { int t = b; b = cc; cc = t; double u = s2; s2 = s3; s3 = u; }
   int i = i1 + dI[a][0], j = j1 + dI[a][1], k = k1 + dI[a][2];
   deposit_direct (c, i, j, k, rc[a][0], rc[b][0], rc[a][1], rc[b][1], rc[a][2], rc[b][2], rho);
   i += dI[b][0];
   j += dI[b][1];
   k += dI[b][2];
   deposit_direct (c, i, j, k, rc[b][0], rc[cc][0], rc[b][1], rc[cc][1], rc[b][2], rc[cc][2], rho);
   deposit_direct (c, i2, j2, k2, rc[cc][0], x2, rc[cc][1], y2, rc[cc][2], z2, rho);
}

__device__ __forceinline__ double warp_sum (double v)
{
   for (int d = 16 ; d > 0 ; d >>= 1)
      v += __shfl_xor_sync (0xffffffffu, v, d);
   return v;
}


// One wall of core/plasma_walls.c:27-104; returns true if the marker goes.
// Once removed, later walls leave it alone (it is dropped by the caller).
__device__ __forceinline__ bool wall (int bc, bool top, double &x, double &v, double L, double h)
{
   if (bc == MG_BC_PERIODIC) {
      if (!top && x <= 0) x += L;
      if (top && x >= L) x -= L;
      return false;
   }
   if (bc == MG_BC_MIRROR) {
      if (!top && x <= 0) { x = -x; v = -v; }
      if (top && x >= L) { x = 2*L - x; v = -v; }
      return false;
   }
   return (!top && x <= h) || (top && x >= L - h);
}

template <int MINB>
__global__ void __launch_bounds__ (256, MINB)
k_push64 (Ctx c, Markers64 m, long long np, DevScalars *dsc)
{
   const Grid &g = c.g;
   const double h1 = g.h[0], h2 = g.h[1], h3 = g.h[2], tau = g.tau;
   const double L0 = g.n[0]*h1, L1 = g.n[1]*h2, L2 = g.n[2]*h3;
   const int lane = threadIdx.x & 31;
   double Wx = 0, Wy = 0, Wz = 0;
   long long dead = 0;

   const long long warps_total = ((long long) gridDim.x*blockDim.x) >> 5;
   const long long warp0 = ((long long) blockIdx.x*blockDim.x + threadIdx.x) >> 5;
   for (long long base = warp0*32 ; base < np ; base += warps_total*32) {
      const long long n = base + lane;
      bool valid = n < np;
      double qm = 0, x1 = 0, y1 = 0, z1 = 0;
      // Markers stream through once per step: their loads and stores are
      // marked evict-first, leaving L1 and L2 to the field gather.  The
      // position loads go out with qDivM's, not after it, so that the
      // gather waits for one round trip to memory, not two.
      if (valid) {
         qm = __ldcs (m.qm + n);
         x1 = __ldcs (m.x + n);
         y1 = __ldcs (m.y + n);
         z1 = __ldcs (m.z + n);
         valid = (qm != 0.0);             // removed markers carry qDivM = 0
      }
      int i = 0, j = 0, k = 0, i2 = 0, j2 = 0, k2 = 0, nseg = 0;
      double fi = 0, fj = 0, fk = 0, fi2 = 0, fj2 = 0, fk2 = 0;   // the same as doubles
      double x2 = 0, y2 = 0, z2 = 0, rho = 0;
      double xa = 0, ya = 0, za = 0;         // end of the first segment
      if (valid) {
         double sX = div_by (x1, h1, c.rh[0]), sY = div_by (y1, h2, c.rh[1]), sZ = div_by (z1, h3, c.rh[2]);
         double sX_ = sX + 0.5, sY_ = sY + 0.5, sZ_ = sZ + 0.5;
         i = cell_of (sX, fi);
         j = cell_of (sY, fj);
         k = cell_of (sZ, fk);
         // The half-shifted cell floor(s + 1/2) is the cell plus one when
         // the offset s - floor(s) reaches 1/2: for s >= 0 the offset is
         // exact and s + 1/2 rounds to no other integer part; for s in
         // [-1, 0) both sides are exact near the threshold.
         const int hx = (sX - fi >= 0.5), hy = (sY - fj >= 0.5), hz = (sZ - fk >= 0.5);
         const int i_ = i + hx, j_ = j + hy, k_ = k + hz;
         const double fi_ = fi + hx, fj_ = fj + hy, fk_ = fk + hz;
         // Start cells outside [-1, n] would read or write past the two
         // ghost layers: flag and skip the marker.
         if (i < -1 || i > g.n[0] || j < -1 || j > g.n[1] || k < -1 || k > g.n[2]) {
            if (atomicOr (&dsc->err, 1) == 0) {
               dsc->err_info[0] = (int) n;
               dsc->err_info[1] = i;
               dsc->err_info[2] = j;
               dsc->err_info[3] = k;
            }
            valid = false;
         } else {
            sX -= fi; sY -= fj; sZ -= fk;
            sX_ -= fi_; sY_ -= fj_; sZ_ -= fk_;
            const double Ex = cic (c.E0, g, i_, sX_, j, sY, k, sZ);
            const double Ey = cic (c.E1, g, i, sX, j_, sY_, k, sZ);
            const double Ez = cic (c.E2, g, i, sX, j, sY, k_, sZ_);
            const double Hx = cic (c.H0, g, i, sX, j_, sY_, k_, sZ_);
            const double Hy = cic (c.H1, g, i_, sX_, j, sY, k_, sZ_);
            const double Hz = cic (c.H2, g, i_, sX_, j_, sY_, k, sZ);

            rho = (double) __ldcs (m.rho + n);
            const double tm = 0.5*tau*qm;
            const double px = __ldcs (m.ux + n) + tm*Ex, py = __ldcs (m.uy + n) + tm*Ey, pz = __ldcs (m.uz + n) + tm*Ez;
            const double gamma = sqrt (1.0 + px*px + py*py + pz*pz);
            // The tally's two divisions (core/plasma.c:140) by one
            // reciprocal: W is summed over markers and blocks in an order of
            // its own anyway, so a last-place difference per marker is
            // below the sums' own rounding.
            const double W = (gamma - 1.0)*rho*h1*h2*h3*recip ((px*px + py*py + pz*pz + 1e-19)*qm);
            Wx += W*px*px;
            Wy += W*py*py;
            Wz += W*pz*pz;

            const double tg = tm/gamma;
            const double ax = tg*Hx, ay = tg*Hy, az = tg*Hz;
            const double u = px + py*az - pz*ay, v = py + pz*ax - px*az, w = pz + px*ay - py*ax;
            const double bxx = ax*ax, byy = ay*ay, bzz = az*az;
            const double bxy = ax*ay, byz = ay*az, bxz = az*ax;
            const double delta = 1.0/(1.0 + bxx + byy + bzz);
            const double vx = tm*Ex + ((1.0 + bxx)*u + (bxy + az)*v + (bxz - ay)*w)*delta;
            const double vy = tm*Ey + ((bxy - az)*u + (1.0 + byy)*v + (byz + ax)*w)*delta;
            const double vz = tm*Ez + ((bxz + ay)*u + (byz - ax)*v + (1.0 + bzz)*w)*delta;

            const double tgi = tau/sqrt (1.0 + vx*vx + vy*vy + vz*vz);
            x2 = x1 + vx*tgi;
            y2 = y1 + vy*tgi;
            z2 = z1 + vz*tgi;

            i2 = cell_of (div_by (x2, h1, c.rh[0]), fi2);
            j2 = cell_of (div_by (y2, h2, c.rh[1]), fj2);
            k2 = cell_of (div_by (z2, h3, c.rh[2]), fk2);
            int di = abs (i2 - i), dj = abs (j2 - j), dk = abs (k2 - k);
            if (fabs (x2 - x1) < 1e-10*h1) { di = 0; i2 = i; fi2 = fi; }
            if (fabs (y2 - y1) < 1e-10*h2) { dj = 0; j2 = j; fj2 = fj; }
            if (fabs (z2 - z1) < 1e-10*h3) { dk = 0; k2 = k; fk2 = fk; }
            if (di > 1 || dj > 1 || dk > 1) {
               // More than one cell per step (Courant violated): flag, no deposit.
               if (atomicOr (&dsc->err, 2) == 0) {
                  dsc->err_info[0] = (int) n;
                  dsc->err_info[1] = i2;
                  dsc->err_info[2] = j2;
                  dsc->err_info[3] = k2;
               }
               valid = false;
            }
            nseg = di + dj + dk;
            if (nseg == 0) {
               xa = x2; ya = y2; za = z2;
            } else if (nseg == 1) {
               // core/plasma.c:214-216: d*(...)/(... + ((1 - d) << 16)) with d in
               // {0, 1}; a zero term adds a signed zero, which leaves the
               // crossing point unchanged, so it is skipped.
               double alpha = 0.0;
               if (dk) alpha = ((fk + fk2 + 1.0)*0.5*h3 - z1)/(z2 - z1);
               if (dj) alpha = ((fj + fj2 + 1.0)*0.5*h2 - y1)/(y2 - y1);
               if (di) alpha = ((fi + fi2 + 1.0)*0.5*h1 - x1)/(x2 - x1);
               xa = x1 + alpha*(x2 - x1);
               ya = y1 + alpha*(y2 - y1);
               za = z1 + alpha*(z2 - z1);
            } else {
               multicell_first (g, i, j, k, i2, j2, k2, x1, y1, z1, x2, y2, z2, xa, ya, za);
            }

            // Store the advanced marker, then apply the walls in the
            // reference's order xMin, yMin, zMin, xMax, yMax, zMax.
            double px_ = x2, py_ = y2, pz_ = z2, vx_ = vx, vy_ = vy, vz_ = vz;
            bool gone = false;
            gone |= wall (g.bc[0][0], false, px_, vx_, L0, h1);
            gone |= wall (g.bc[0][1], false, py_, vy_, L1, h2);
            gone |= wall (g.bc[0][2], false, pz_, vz_, L2, h3);
            gone |= wall (g.bc[1][0], true, px_, vx_, L0, h1);
            gone |= wall (g.bc[1][1], true, py_, vy_, L1, h2);
            gone |= wall (g.bc[1][2], true, pz_, vz_, L2, h3);
            __stcs (m.x + n, px_);
            __stcs (m.y + n, py_);
            __stcs (m.z + n, pz_);
            __stcs (m.ux + n, vx_);
            __stcs (m.uy + n, vy_);
            __stcs (m.uz + n, vz_);
            if (gone) {
               m.qm[n] = 0.0f;
               ++dead;
            }
         }
      }

      // Segments after the first, for markers that crossed cell faces.
      if (valid && nseg == 1) {
         double w2[12];
         segment_weights (c, fi2, fj2, fk2, xa, x2, ya, y2, za, z2, rho, w2);
         scatter12 (c, i2, j2, k2, w2);
      }
      else if (valid && nseg >= 2)
         multicell_rest (c, i, j, k, i2, j2, k2, x1, y1, z1, x2, y2, z2, rho);

      // First segment: warp-aggregated by start cell.
      double wgt[12];
      if (valid)
         segment_weights (c, fi, fj, fk, x1, xa, y1, ya, z1, za, rho, wgt);
      else
         for (int q = 0 ; q < 12 ; ++q) wgt[q] = 0;
      const long long key = valid ? g.at (i, j, k) : -1 - lane;
      const long long prev = __shfl_up_sync (0xffffffffu, key, 1);
      const long long next = __shfl_down_sync (0xffffffffu, key, 1);
      const bool head = (lane == 0) || (prev != key);
      const bool tail = (lane == 31) || (next != key);
      const unsigned heads = __ballot_sync (0xffffffffu, head);
      const unsigned le = (lane == 31) ? 0xffffffffu : ((1u << (lane + 1)) - 1);
      const int seg_start = 31 - __clz (heads & le);
      // Scan rounds up to the longest run of the warp (a cold, sorted foil
      // has runs of 16 lanes: four rounds instead of five).
      const unsigned longest = __reduce_max_sync (0xffffffffu, (unsigned) (lane - seg_start + 1));
      for (int d = 1 ; d < (int) longest ; d <<= 1) {
#pragma unroll
         for (int q = 0 ; q < 12 ; ++q) {
            const double t = __shfl_up_sync (0xffffffffu, wgt[q], d);
            if (lane - d >= seg_start)
               wgt[q] += t;
         }
      }
      if (valid && tail)
         scatter12 (c, i, j, k, wgt);
   }

   // Thermal energy tally: block reduction, one atomic per block.
   __shared__ double sw[3][8];
   Wx = warp_sum (Wx);
   Wy = warp_sum (Wy);
   Wz = warp_sum (Wz);
   const int wid = threadIdx.x >> 5;
   if (lane == 0) {
      sw[0][wid] = Wx;
      sw[1][wid] = Wy;
      sw[2][wid] = Wz;
   }
   for (int d = 16 ; d > 0 ; d >>= 1)
      dead += __shfl_xor_sync (0xffffffffu, dead, d);
   if (lane == 0 && dead)
      atomicAdd ((unsigned long long *) &dsc->dead, (unsigned long long) dead);
   __syncthreads ();
   if (wid == 0) {
      const int nw = blockDim.x >> 5;
      Wx = lane < nw ? sw[0][lane] : 0;
      Wy = lane < nw ? sw[1][lane] : 0;
      Wz = lane < nw ? sw[2][lane] : 0;
      Wx = warp_sum (Wx);
      Wy = warp_sum (Wy);
      Wz = warp_sum (Wz);
      if (lane == 0) {
         atomicAdd (&dsc->acc[2], Wx);
         atomicAdd (&dsc->acc[3], Wy);
         atomicAdd (&dsc->acc[4], Wz);
      }
   }
}

// Particle walls applied once to freshly loaded markers (plasma_init,
// core/plasma.c:399-404, on markers that all start in the shell).
__global__ void k_walls64 (Grid g, Markers64 m, long long np, DevScalars *dsc)
{
   long long dead = 0;
   const double L[3] = {g.n[0]*g.h[0], g.n[1]*g.h[1], g.n[2]*g.h[2]};
   for (long long n = blockIdx.x*(long long) blockDim.x + threadIdx.x ; n < np ;
        n += (long long) gridDim.x*blockDim.x) {
      if (m.qm[n] == 0.0f)
         continue;
      double pos[3] = {m.x[n], m.y[n], m.z[n]};
      double vel[3] = {m.ux[n], m.uy[n], m.uz[n]};
      bool gone = false;
      for (int f = 0 ; f < 6 && !gone ; ++f) {
         const int a = (f < 3) ? f : f - 3, top = (f >= 3);
         const int bc = g.bc[top][a];
         if (bc == MG_BC_PERIODIC) {
            if (!top && pos[a] <= 0) pos[a] += L[a];
            if (top && pos[a] >= L[a]) pos[a] -= L[a];
         } else if (bc == MG_BC_MIRROR) {
            if (!top && pos[a] <= 0) { pos[a] = -pos[a]; vel[a] *= -1; }
            if (top && pos[a] >= L[a]) { pos[a] = 2*L[a] - pos[a]; vel[a] *= -1; }
         } else if ((!top && pos[a] <= g.h[a]) || (top && pos[a] >= L[a] - g.h[a])) {
            gone = true;
         }
      }
      m.x[n] = pos[0];
      m.y[n] = pos[1];
      m.z[n] = pos[2];
      m.ux[n] = vel[0];
      m.uy[n] = vel[1];
      m.uz[n] = vel[2];
      if (gone) {
         m.qm[n] = 0.0f;
         ++dead;
      }
   }
   if (dead)
      atomicAdd ((unsigned long long *) &dsc->dead, (unsigned long long) dead);
}

} // namespace

int mg_walls64 (mg_run_t *r)
{
   if (r->np == 0)
      return MG_OK;
   k_walls64<<<mg_blocks_for (r->np, 256, 8), 256, 0, r->stream>>> (r->g, r->m64, r->np, r->dsc);
   MG_LAUNCH_CHECK ();
   return MG_OK;
}

int mg_push64 (mg_run_t *r)
{
   if (r->np == 0)
      return MG_OK;
   Ctx c;
   c.g = r->g;
   c.E0 = r->E[0]; c.E1 = r->E[1]; c.E2 = r->E[2];
   c.H0 = r->Hn[0]; c.H1 = r->Hn[1]; c.H2 = r->Hn[2];   // H at t = n tau
   c.J0 = r->J[0]; c.J1 = r->J[1]; c.J2 = r->J[2];
   const double *h = r->g.h, tau = r->g.tau;
   for (int a = 0 ; a < 3 ; ++a)
      c.rh[a] = 1.0/h[a];
   c.jdx = tau*h[1]*h[2];
   c.jdy = tau*h[0]*h[2];
   c.jdz = tau*h[0]*h[1];
   c.rjx = 1.0/c.jdx;
   c.rjy = 1.0/c.jdy;
   c.rjz = 1.0/c.jdz;
   const int T = 256;
   // Two blocks of 256 per SM (no register cap that spills): over the whole
   // 2000-step laser-foil run 0.376 ms per push against 0.387 with three
   // blocks (80 registers) and 0.403 with four (64 registers); early in the
   // run, with a cold sorted foil, four blocks lead (0.335 against 0.351).
   k_push64<2><<<mg_blocks_for (r->np, T, 8), T, 0, r->stream>>> (c, r->m64, r->np, r->dsc);
   MG_LAUNCH_CHECK ();
   return MG_OK;
}


// ---- cell sort of the FP64 markers -------------------------------------------
// Every sort_every steps (default 16) the markers are put in cell order
// (i, then j, then k), so that the markers of a warp share the 48 field
// values of their gather in L1 and their current atomics aggregate.  A
// counting sort: keys (the push's own cell index, removed markers last),
// counts, scan, scatter into scratch arrays, copy back -- the step graph
// keeps its marker pointers.  The push's arithmetic per marker is unchanged;
// only the order of the current sums on J changes.
namespace {

struct Key64 {
   int n[3];
   double h[3], rh[3];
   int cells;              // (n0+2)(n1+2)(n2+2): cells [-1, n]; then outside, removed
};

__device__ __forceinline__ int key64 (const Key64 &t, double x, double y, double z, float qm)
{
   if (qm == 0.0f)
      return t.cells + 1;
   double f;
   const int i = cell_of (div_by (x, t.h[0], t.rh[0]), f);
   const int j = cell_of (div_by (y, t.h[1], t.rh[1]), f);
   const int k = cell_of (div_by (z, t.h[2], t.rh[2]), f);
   if (i < -1 || i > t.n[0] || j < -1 || j > t.n[1] || k < -1 || k > t.n[2])
      return t.cells;
   return ((i + 1)*(t.n[1] + 2) + (j + 1))*(t.n[2] + 2) + (k + 1);
}

#define SORT64_ROWS 8
__global__ void k_hist64 (Key64 t, Markers64 m, long long np, int *count, long long kp)
{
   const int lane = threadIdx.x & 31;
   const long long stride = (long long) gridDim.x*blockDim.x*SORT64_ROWS;
   for (long long base = (blockIdx.x*(long long) blockDim.x + (threadIdx.x & ~31))*SORT64_ROWS ; base < np ;
        base += stride) {
      double x[SORT64_ROWS], y[SORT64_ROWS], z[SORT64_ROWS];
      float qm[SORT64_ROWS];
#pragma unroll
      for (int q = 0 ; q < SORT64_ROWS ; ++q) {
         const long long n = min (base + 32*q + lane, np - 1);
         x[q] = m.x[n];
         y[q] = m.y[n];
         z[q] = m.z[n];
         qm[q] = m.qm[n];
      }
#pragma unroll
      for (int q = 0 ; q < SORT64_ROWS ; ++q) {
         const int key = base + 32*q + lane < np ? key64 (t, x[q], y[q], z[q], qm[q]) : -1;
         int start, len;
         key_runs (key, lane, start, len);
         if (key >= 0 && start == lane)
            atomicAdd (count + spread (key, kp), len);
      }
   }
}

__global__ void k_scatter64 (Key64 t, Markers64 m, Markers64 o, long long np, const long long *offset,
                             int *fill, long long kp)
{
   const int lane = threadIdx.x & 31;
   const long long stride = (long long) gridDim.x*blockDim.x*SORT64_ROWS;
   for (long long base = (blockIdx.x*(long long) blockDim.x + (threadIdx.x & ~31))*SORT64_ROWS ; base < np ;
        base += stride) {
      double x[SORT64_ROWS], y[SORT64_ROWS], z[SORT64_ROWS], ux[SORT64_ROWS], uy[SORT64_ROWS], uz[SORT64_ROWS];
      float rho[SORT64_ROWS], qm[SORT64_ROWS];
      int id[SORT64_ROWS], key[SORT64_ROWS];
      long long at[SORT64_ROWS];
#pragma unroll
      for (int q = 0 ; q < SORT64_ROWS ; ++q) {
         const long long n = min (base + 32*q + lane, np - 1);
         x[q] = m.x[n]; y[q] = m.y[n]; z[q] = m.z[n];
         ux[q] = m.ux[n]; uy[q] = m.uy[n]; uz[q] = m.uz[n];
         rho[q] = m.rho[n]; qm[q] = m.qm[n]; id[q] = m.id[n];
      }
#pragma unroll
      for (int q = 0 ; q < SORT64_ROWS ; ++q) {
         key[q] = base + 32*q + lane < np ? key64 (t, x[q], y[q], z[q], qm[q]) : -1;
         int start, len;
         key_runs (key[q], lane, start, len);
         at[q] = 0;
         if (key[q] >= 0 && start == lane)
            at[q] = offset[key[q]] + atomicAdd (fill + spread (key[q], kp), len);
         at[q] = __shfl_sync (0xffffffffu, at[q], start) + (lane - start);
      }
#pragma unroll
      for (int q = 0 ; q < SORT64_ROWS ; ++q)
         if (key[q] >= 0) {
            const long long a = at[q];
            o.x[a] = x[q]; o.y[a] = y[q]; o.z[a] = z[q];
            o.ux[a] = ux[q]; o.uy[a] = uy[q]; o.uz[a] = uz[q];
            o.rho[a] = rho[q]; o.qm[a] = qm[q]; o.id[a] = id[q];
         }
   }
}

} // namespace

int mg_sort64 (mg_run_t *r)
{
   r->steps_since_sort = 0;
   if (r->np == 0)
      return MG_OK;
   Key64 t;
   for (int a = 0 ; a < 3 ; ++a) {
      t.n[a] = r->g.n[a];
      t.h[a] = r->g.h[a];
      t.rh[a] = 1.0/r->g.h[a];
   }
   const long long cells = (long long) (t.n[0] + 2)*(t.n[1] + 2)*(t.n[2] + 2);
   if (cells + 2 >= (1LL << 31)) {
      mg_set_error ("mg_sort64: %lld cells exceed the sort's key range", cells);
      return MG_ERR_ARG;
   }
   t.cells = (int) cells;
   const long long len = cells + 2, kp = (len + 7)/8;
   const long long nb = (len + SCAN_CHUNK - 1)/SCAN_CHUNK;
   const size_t a_count = ((size_t) kp*8*4 + 255) & ~(size_t) 255;
   const size_t a_off = ((size_t) len*8 + 255) & ~(size_t) 255;
   const size_t a_bsum = ((size_t) nb*8 + 255) & ~(size_t) 255;
   const size_t a_mark = (size_t) r->np*(6*8 + 3*4) + 9*256;
   const size_t need = a_count + a_off + a_bsum + a_mark;
   if (r->sort_tmp_bytes < need) {
      if (r->sort_tmp) {
         mg_dev_free (r, r->sort_tmp);
         r->dev_bytes -= r->sort_tmp_bytes;
         r->sort_tmp = nullptr;
         r->sort_tmp_bytes = 0;
      }
      const int rc = mg_dev_alloc (r, &r->sort_tmp, need);
      if (rc != MG_OK)
         return rc;
      r->sort_tmp_bytes = need;
   }
   char *p = (char *) r->sort_tmp;
   int *count = (int *) p;                 p += a_count;
   long long *offset = (long long *) p;    p += a_off;
   long long *bsum = (long long *) p;      p += a_bsum;
   Markers64 o;
   auto take = [&] (size_t bytes) { char *q = p; p += (bytes + 255) & ~(size_t) 255; return q; };
   o.x = (double *) take (r->np*8); o.y = (double *) take (r->np*8); o.z = (double *) take (r->np*8);
   o.ux = (double *) take (r->np*8); o.uy = (double *) take (r->np*8); o.uz = (double *) take (r->np*8);
   o.rho = (float *) take (r->np*4); o.qm = (float *) take (r->np*4); o.id = (int *) take (r->np*4);
   const int T = 256;
   MG_CUDA (cudaMemsetAsync (count, 0, (size_t) kp*8*4, r->stream));
   k_hist64<<<mg_blocks_for (r->np, T, 8), T, 0, r->stream>>> (t, r->m64, r->np, count, kp);
   MG_LAUNCH_CHECK ();
   const int rc = mg_scan_counts (r, count, kp, len, offset, bsum);
   if (rc != MG_OK)
      return rc;
   MG_CUDA (cudaMemsetAsync (count, 0, (size_t) kp*8*4, r->stream));
   k_scatter64<<<mg_blocks_for (r->np, T, 8), T, 0, r->stream>>> (t, r->m64, o, r->np, offset, count, kp);
   MG_LAUNCH_CHECK ();
   const Markers64 &m = r->m64;
   void *dst[9] = {m.x, m.y, m.z, m.ux, m.uy, m.uz, m.rho, m.qm, m.id};
   const void *src[9] = {o.x, o.y, o.z, o.ux, o.uy, o.uz, o.rho, o.qm, o.id};
   for (int q = 0 ; q < 9 ; ++q)
      MG_CUDA (cudaMemcpyAsync (dst[q], src[q], (size_t) r->np*(q < 6 ? 8 : 4), cudaMemcpyDeviceToDevice,
                                r->stream));
   return MG_OK;
}
