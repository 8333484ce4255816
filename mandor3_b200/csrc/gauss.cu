// Charge density and the Gauss-law test on the device, FP64 arithmetic in
// both precision forms.
//
// Density: CIC deposit of every live marker (core/plasma.c:322-329,
// core/plasma_rho.c:159-173) with the nested weights of mf_PIC_distribute
// (misc_PIC.h:164-195): node (i+a, j+b, k+c) receives wx_a*(wy_b*(wz_c*rho)),
// then the wall folding of plasmaRho_applyBoundary (core/plasma_rho.c:23-97),
// walls in the order x, y, z, lower then upper:
//   periodic (at the lower wall only): for the 5 layers a = -2..2,
//     rho[a + n] += rho[a]; rho[a] = rho[a + n];
//   mirror / open: with the wall node w and the outward step o,
//     rho[w - o] += rho[w + o]; rho[w - 2o] += rho[w + 2o]; rho[w] = 0;
//     rho[w + o] = -rho[w - o]; rho[w + 2o] = -rho[w - 2o];
// over the wall plane's nodes [-2, n+2] in the two other axes.  The VSP
// filter (core/plasma_VSP.c:32) is off at its default alpha = 1.
//
// Residuals (core/plasma_gaussTest.c:110-149): over nodes [0, n]^3 the
// largest |(rho2 - rho1)/tau + div J| and |div E - rho2|.
#include <cuda_runtime.h>

#include "mg_internal.cuh"

namespace {

__device__ __forceinline__ int dbl_to_int (double x) { return (int) (x + 128.0) - 128; }
__device__ __forceinline__ int unpack (int c, int s) { return ((c >> s) & 1023) - 1; }

__device__ __forceinline__ void rho_add (double *rho, const Grid &g, int i, int j, int k,
                                         double sx, double sy, double sz, double v)
{
   if (i < -2 || i > g.n[0] + 1 || j < -2 || j > g.n[1] + 1 || k < -2 || k > g.n[2] + 1)
      return;
   const long o = g.at (i, j, k), Sx = g.sx, Sy = g.sy;
   const double z0 = (1 - sz)*v, z1 = sz*v;
   const double y00 = (1 - sy)*z0, y10 = sy*z0, y01 = (1 - sy)*z1, y11 = sy*z1;
   atomicAdd (rho + o, (1 - sx)*y00);
   atomicAdd (rho + o + Sx, sx*y00);
   atomicAdd (rho + o + Sy, (1 - sx)*y10);
   atomicAdd (rho + o + Sx + Sy, sx*y10);
   atomicAdd (rho + o + 1, (1 - sx)*y01);
   atomicAdd (rho + o + Sx + 1, sx*y01);
   atomicAdd (rho + o + Sy + 1, (1 - sx)*y11);
   atomicAdd (rho + o + Sx + Sy + 1, sx*y11);
}

__global__ void k_rho_cic64 (Grid g, Markers64 m, long long np, double *rho)
{
   for (long long n = blockIdx.x*(long long) blockDim.x + threadIdx.x ; n < np ;
        n += (long long) gridDim.x*blockDim.x) {
      if (m.qm[n] == 0.0f)
         continue;
      double sx = m.x[n]/g.h[0], sy = m.y[n]/g.h[1], sz = m.z[n]/g.h[2];
      const int i = dbl_to_int (sx), j = dbl_to_int (sy), k = dbl_to_int (sz);
      sx -= i;
      sy -= j;
      sz -= k;
      rho_add (rho, g, i, j, k, sx, sy, sz, m.rho[n]);
   }
}

// Precision form: the cell and the offsets are the CIC index and weights.
__global__ void k_rho_cic32 (Grid g, Markers32 m, long long np, double *rho)
{
   for (long long n = blockIdx.x*(long long) blockDim.x + threadIdx.x ; n < np ;
        n += (long long) gridDim.x*blockDim.x) {
      if (m.qm[n] == 0.0f)
         continue;
      const int c = m.cell[n];
      rho_add (rho, g, unpack (c, 20), unpack (c, 10), unpack (c, 0), m.ox[n], m.oy[n], m.oz[n], m.rho[n]);
   }
}

// One wall of the folding; threads over the wall plane's (p, q) nodes.
__global__ void k_rho_wall (Grid g, double *rho, int ea, int ep, int eq, int top, int bc)
{
   const int np_ = g.n[ep] + 5, nq = g.n[eq] + 5;
   for (int t = blockIdx.x*blockDim.x + threadIdx.x ; t < np_*nq ; t += gridDim.x*blockDim.x) {
      int c[3];
      c[ep] = t/nq - 2;
      c[eq] = t % nq - 2;
      const int n = g.n[ea];
      auto at = [&] (int a) { c[ea] = a; return g.at (c[0], c[1], c[2]); };
      if (bc == MG_BC_PERIODIC) {
         if (top)
            continue;
         for (int a = -2 ; a <= 2 ; ++a) {
            const long lo = at (a), hi = at (a + n);
            rho[hi] += rho[lo];
            rho[lo] = rho[hi];
         }
      } else {
         const int w = top ? n : 0, o = top ? 1 : -1;
         const long in1 = at (w - o), out1 = at (w + o), in2 = at (w - 2*o), out2 = at (w + 2*o), wall = at (w);
         rho[in1] += rho[out1];
         rho[in2] += rho[out2];
         rho[wall] = 0;
         rho[out1] = -rho[in1];
         rho[out2] = -rho[in2];
      }
   }
}

// Non-negative doubles order like their bit patterns.
__device__ __forceinline__ void max_to (double *dst, double v)
{
   atomicMax ((unsigned long long *) dst, (unsigned long long) __double_as_longlong (v));
}

template <typename T>
__global__ void k_gauss (Grid g, const double *rho1, const double *rho2, const T *E0, const T *E1,
                         const T *E2, const T *J0, const T *J1, const T *J2, double *out)
{
   const long nk = g.n[2] + 1, nj = g.n[1] + 1, ni = g.n[0] + 1;
   double d0 = 0, d1 = 0;
   for (long t = blockIdx.x*(long) blockDim.x + threadIdx.x ; t < ni*nj*nk ; t += (long) gridDim.x*blockDim.x) {
      const int k = (int) (t % nk), j = (int) ((t/nk) % nj), i = (int) (t/(nk*nj));
      const long o = g.at (i, j, k), Sx = g.sx, Sy = g.sy;
      const double t0 = (rho2[o] - rho1[o])/g.tau +
                        ((double) J0[o + Sx] - (double) J0[o])/g.h[0] +
                        ((double) J1[o + Sy] - (double) J1[o])/g.h[1] +
                        ((double) J2[o + 1] - (double) J2[o])/g.h[2];
      const double t1 = ((double) E0[o + Sx] - (double) E0[o])/g.h[0] +
                        ((double) E1[o + Sy] - (double) E1[o])/g.h[1] +
                        ((double) E2[o + 1] - (double) E2[o])/g.h[2] -
                        rho2[o];
      d0 = fmax (d0, fabs (t0));
      d1 = fmax (d1, fabs (t1));
   }
   for (int d = 16 ; d > 0 ; d >>= 1) {
      d0 = fmax (d0, __shfl_xor_sync (0xffffffffu, d0, d));
      d1 = fmax (d1, __shfl_xor_sync (0xffffffffu, d1, d));
   }
   if ((threadIdx.x & 31) == 0) {
      max_to (out, d0);
      max_to (out + 1, d1);
   }
}

} // namespace

// Charge density of the current markers into rho (g.total doubles).
int mg_gauss_rho (mg_run_t *r, double *rho)
{
   MG_CUDA (cudaMemsetAsync (rho, 0, sizeof (double)*r->g.total, r->stream));
   const int T = 256;
   if (r->np > 0) {
      if (r->prm.precision == MG_FP32_OFFSET)
         k_rho_cic32<<<mg_blocks_for (r->np, T, 8), T, 0, r->stream>>> (r->g, r->m32, r->np, rho);
      else
         k_rho_cic64<<<mg_blocks_for (r->np, T, 8), T, 0, r->stream>>> (r->g, r->m64, r->np, rho);
      MG_LAUNCH_CHECK ();
   }
   static const int axes[3][3] = {{0, 1, 2}, {1, 0, 2}, {2, 0, 1}};
   for (int b = 0 ; b < 6 ; ++b) {
      const int ea = axes[b/2][0], ep = axes[b/2][1], eq = axes[b/2][2], top = b & 1;
      const long plane = (long) (r->g.n[ep] + 5)*(r->g.n[eq] + 5);
      k_rho_wall<<<mg_blocks_for (plane, T, 4), T, 0, r->stream>>> (r->g, rho, ea, ep, eq, top, r->g.bc[top][ea]);
      MG_LAUNCH_CHECK ();
   }
   return MG_OK;
}

// Residuals into out_dev[2] (device), from rho1, rho2 and the run's E and J.
int mg_gauss_residual (mg_run_t *r, const double *rho1, const double *rho2, double *out_dev)
{
   MG_CUDA (cudaMemsetAsync (out_dev, 0, 2*sizeof (double), r->stream));
   const long vol = (long) (r->g.n[0] + 1)*(r->g.n[1] + 1)*(r->g.n[2] + 1);
   const int T = 256;
   if (r->prm.precision == MG_FP32_OFFSET)
      k_gauss<float><<<mg_blocks_for (vol, T, 8), T, 0, r->stream>>> (
         r->g, rho1, rho2, r->E32[0], r->E32[1], r->E32[2], r->J32[0], r->J32[1], r->J32[2], out_dev);
   else
      k_gauss<double><<<mg_blocks_for (vol, T, 8), T, 0, r->stream>>> (
         r->g, rho1, rho2, r->E[0], r->E[1], r->E[2], r->J[0], r->J[1], r->J[2], out_dev);
   MG_LAUNCH_CHECK ();
   return MG_OK;
}
