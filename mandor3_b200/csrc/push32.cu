// Precision form of the particle push: integer cell + FP32 offset positions,
// FP32 momenta, fields and currents, FP64 energy sums.
//
// The algorithm is the reference's (core/plasma.c:95-263, misc_PIC.h:18-126,
// core/plasma_currentKernel.c:21-279, core/plasma_walls.c:27-104) restated in
// cell units: a marker sits at (i + ox) h1, ..., its offsets ox, oy, oz lie
// in [0, 1), and the charge-conserving weights of a segment use cell-local
// coordinates, where the reference's (h2 - tY)(h3 - tZ) + dY dZ/12 becomes
// h2 h3 [(1 - ty)(1 - tz) + dy dz/12] and the prefactor rho dX/(tau h2 h3)
// becomes rho h1 dx/tau.  Cell changes are exact integer arithmetic, so the
// periodic wrap adds no rounding at all.
//
// Marker cells are packed as ((i+1) << 20) | ((j+1) << 10) | (k+1) with
// i in [-1, 1022]: one 32-bit word, unpacked with shifts.
#include <cuda_runtime.h>

#include "mg_internal.cuh"

namespace {

struct Ctx32 {
   Grid   g;
   const float *E0, *E1, *E2, *H0, *H1, *H2;
   float  *J0, *J1, *J2;
   float  tau, rh[3];            // tau, 1/h
   float  kj[3];                 // h_a / tau: current prefactor per unit rho and cell-unit displacement
   double vol;                   // h1 h2 h3 for the thermal tally
};

__device__ __forceinline__ int unpack (int c, int s) { return ((c >> s) & 1023) - 1; }
__device__ __forceinline__ int pack (int i, int j, int k) { return ((i + 1) << 20) | ((j + 1) << 10) | (k + 1); }

__device__ __forceinline__ float cic (const float *F, const Grid &g, int i, float sx, int j, float sy,
                                      int k, float sz)
{
   const long o = g.at (i, j, k), Sx = g.sx, Sy = g.sy;
   const float f0 = __ldg (F + o), f1 = __ldg (F + o + Sx);
   const float f2 = __ldg (F + o + Sy), f3 = __ldg (F + o + Sx + Sy);
   const float f4 = __ldg (F + o + 1), f5 = __ldg (F + o + Sx + 1);
   const float f6 = __ldg (F + o + Sy + 1), f7 = __ldg (F + o + Sx + Sy + 1);
   const float a00 = f0 + sx*(f1 - f0), a10 = f2 + sx*(f3 - f2);
   const float a01 = f4 + sx*(f5 - f4), a11 = f6 + sx*(f7 - f6);
   const float b0 = a00 + sy*(a10 - a00), b1 = a01 + sy*(a11 - a01);
   return b0 + sz*(b1 - b0);
}

// Weights of one in-cell segment in cell-local coordinates, reference
// order (see segment_weights in push64.cu).
__device__ __forceinline__ void weights32 (const Ctx32 &c, float rho, float a1, float a2, float b1,
                                           float b2, float c1, float c2, float w[12])
{
   const float dx = a2 - a1, dy = b2 - b1, dz = c2 - c1;
   const float tx = 0.5f*(a1 + a2), ty = 0.5f*(b1 + b2), tz = 0.5f*(c1 + c2);
   const float qx = rho*c.kj[0]*dx, qy = rho*c.kj[1]*dy, qz = rho*c.kj[2]*dz;
   const float dyz = dy*dz*(1.0f/12), dxz = dx*dz*(1.0f/12), dxy = dx*dy*(1.0f/12);
   w[0] = qx*((1 - ty)*(1 - tz) + dyz);
   w[1] = qx*(ty*(1 - tz) - dyz);
   w[2] = qx*((1 - ty)*tz - dyz);
   w[3] = qx*(ty*tz + dyz);
   w[4] = qy*((1 - tx)*(1 - tz) + dxz);
   w[5] = qy*(tx*(1 - tz) - dxz);
   w[6] = qy*((1 - tx)*tz - dxz);
   w[7] = qy*(tx*tz + dxz);
   w[8] = qz*((1 - tx)*(1 - ty) + dxy);
   w[9] = qz*(tx*(1 - ty) - dxy);
   w[10] = qz*((1 - tx)*ty - dxy);
   w[11] = qz*(tx*ty + dxy);
}

__device__ __forceinline__ void scatter32 (const Ctx32 &c, int i, int j, int k, const float w[12])
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

__device__ __forceinline__ float seg_scan (float v, int lane, int seg_start)
{
#pragma unroll
   for (int d = 1 ; d < 32 ; d <<= 1) {
      const float t = __shfl_up_sync (0xffffffffu, v, d);
      if (lane - d >= seg_start)
         v += t;
   }
   return v;
}

// One wall in cell units (core/plasma_walls.c:27-104); returns true if the
// marker is removed.  c: cell index along the axis, o: offset, u: momentum.
__device__ __forceinline__ bool wall32 (int bc, bool top, int n, int &c, float &o, float &u)
{
   if (bc == MG_BC_PERIODIC) {
      if (!top && (c < 0 || (c == 0 && o == 0.0f))) c += n;    // x <= 0: x += L
      if (top && c >= n) c -= n;                                // x >= L: x -= L
      return false;
   }
   if (bc == MG_BC_MIRROR) {
      if (!top && (c < 0 || (c == 0 && o == 0.0f))) {         // x <= 0: x = -x
         if (c < 0) {
            c = 0;
            o = 1.0f - o;
            if (o >= 1.0f) o = 0.99999994f;
         }
         u = -u;
      }
      if (top && c >= n) {                                      // x >= L: x = 2L - x
         if (!(c == n && o == 0.0f)) {
            c = n - 1;
            o = 1.0f - o;
            if (o >= 1.0f) o = 0.99999994f;
         }
         u = -u;
      }
      return false;
   }
   return (!top && (c < 1 || (c == 1 && o == 0.0f))) || (top && c >= n - 1);
}

// Segment of the path between times ta and tb (start-cell coordinates),
// in the cell shifted by (si, sj, sk) from the start cell.
__device__ __forceinline__ void deposit_piece (const Ctx32 &c, float rho, int i, int j, int k,
                                               int si, int sj, int sk, float ox, float oy, float oz,
                                               float dx, float dy, float dz, float ta, float tb)
{
   float w[12];
   weights32 (c, rho, ox + ta*dx - si, ox + tb*dx - si, oy + ta*dy - sj, oy + tb*dy - sj,
              oz + ta*dz - sk, oz + tb*dz - sk, w);
   scatter32 (c, i + si, j + sj, k + sk, w);
}

#define CSWAP(ta, aa, tb, ab)                                                 \
   do {                                                                      \
      if (tb < ta) {                                                         \
         const float t_ = ta; ta = tb; tb = t_;                              \
         const int a_ = aa; aa = ab; ab = a_;                                \
      }                                                                      \
   } while (0)

__global__ void __launch_bounds__ (256, 3)
k_push32 (Ctx32 c, Markers32 m, long long np, DevScalars *dsc)
{
   const Grid &g = c.g;
   const int lane = threadIdx.x & 31;
   double Wx = 0, Wy = 0, Wz = 0;
   long long dead = 0;
   const long long warps_total = ((long long) gridDim.x*blockDim.x) >> 5;
   const long long warp0 = ((long long) blockIdx.x*blockDim.x + threadIdx.x) >> 5;
   for (long long base = warp0*32 ; base < np ; base += warps_total*32) {
      const long long n = base + lane;
      bool valid = n < np;
      float qm = 0.0f;
      if (valid) {
         qm = m.qm[n];
         valid = (qm != 0.0f);
      }
      int i = 0, j = 0, k = 0, di = 0, dj = 0, dk = 0;
      float ox = 0, oy = 0, oz = 0, dx = 0, dy = 0, dz = 0, rho = 0;
      if (valid) {
         const int cell = m.cell[n];
         i = unpack (cell, 20);
         j = unpack (cell, 10);
         k = unpack (cell, 0);
         if (i < -1 || i > g.n[0] || j < -1 || j > g.n[1] || k < -1 || k > g.n[2]) {
            if (atomicOr (&dsc->err, 1) == 0) {
               dsc->err_info[0] = (int) n;
               dsc->err_info[1] = i;
               dsc->err_info[2] = j;
               dsc->err_info[3] = k;
            }
            valid = false;
         } else {
            ox = m.ox[n];
            oy = m.oy[n];
            oz = m.oz[n];
            // Half-shifted meshes: node i_ and weight s_ of x/h + 1/2.
            const int i_ = i + (ox >= 0.5f), j_ = j + (oy >= 0.5f), k_ = k + (oz >= 0.5f);
            const float sx_ = ox >= 0.5f ? ox - 0.5f : ox + 0.5f;
            const float sy_ = oy >= 0.5f ? oy - 0.5f : oy + 0.5f;
            const float sz_ = oz >= 0.5f ? oz - 0.5f : oz + 0.5f;
            const float Ex = cic (c.E0, g, i_, sx_, j, oy, k, oz);
            const float Ey = cic (c.E1, g, i, ox, j_, sy_, k, oz);
            const float Ez = cic (c.E2, g, i, ox, j, oy, k_, sz_);
            const float Hx = cic (c.H0, g, i, ox, j_, sy_, k_, sz_);
            const float Hy = cic (c.H1, g, i_, sx_, j, oy, k_, sz_);
            const float Hz = cic (c.H2, g, i_, sx_, j_, sy_, k, oz);

            rho = m.rho[n];
            const float tm = 0.5f*c.tau*qm;
            const float px = m.ux[n] + tm*Ex, py = m.uy[n] + tm*Ey, pz = m.uz[n] + tm*Ez;
            const float p2 = px*px + py*py + pz*pz;
            const float rg = rsqrtf (1.0f + p2);             // 1/gamma
            const float gamma = (1.0f + p2)*rg;
            // (gamma - 1)/(p^2 + 1e-19) of core/plasma.c:140 written as
            // 1/(gamma + 1) up to the 1e-19 guard: no cancellation in FP32.
            const float W = __fdividef (p2, (gamma + 1.0f)*(p2 + 1e-19f))*rho*(float) c.vol/qm;
            Wx += (double) (W*px*px);
            Wy += (double) (W*py*py);
            Wz += (double) (W*pz*pz);
            const float tg = tm*rg;
            const float ax = tg*Hx, ay = tg*Hy, az = tg*Hz;
            const float u = px + py*az - pz*ay, v = py + pz*ax - px*az, w = pz + px*ay - py*ax;
            const float bxx = ax*ax, byy = ay*ay, bzz = az*az;
            const float bxy = ax*ay, byz = ay*az, bxz = az*ax;
            const float delta = __frcp_rn (1.0f + bxx + byy + bzz);
            float vx = tm*Ex + ((1.0f + bxx)*u + (bxy + az)*v + (bxz - ay)*w)*delta;
            float vy = tm*Ey + ((bxy - az)*u + (1.0f + byy)*v + (byz + ax)*w)*delta;
            float vz = tm*Ez + ((bxz + ay)*u + (byz - ax)*v + (1.0f + bzz)*w)*delta;
            const float tgi = c.tau*rsqrtf (1.0f + vx*vx + vy*vy + vz*vz);
            dx = vx*tgi*c.rh[0];
            dy = vy*tgi*c.rh[1];
            dz = vz*tgi*c.rh[2];
            float nx = ox + dx, ny = oy + dy, nz = oz + dz;
            di = (nx >= 1.0f) - (nx < 0.0f);
            dj = (ny >= 1.0f) - (ny < 0.0f);
            dk = (nz >= 1.0f) - (nz < 0.0f);
            if (fabsf (dx) >= 1.0f || fabsf (dy) >= 1.0f || fabsf (dz) >= 1.0f) {
               if (atomicOr (&dsc->err, 2) == 0)
                  dsc->err_info[0] = (int) n;
               valid = false;
            }
            int i2 = i + di, j2 = j + dj, k2 = k + dk;
            nx -= di;
            ny -= dj;
            nz -= dk;
            if (nx >= 1.0f) nx = 0.99999994f;
            if (ny >= 1.0f) ny = 0.99999994f;
            if (nz >= 1.0f) nz = 0.99999994f;
            bool gone = false;
            gone |= wall32 (g.bc[0][0], false, g.n[0], i2, nx, vx);
            gone |= wall32 (g.bc[0][1], false, g.n[1], j2, ny, vy);
            gone |= wall32 (g.bc[0][2], false, g.n[2], k2, nz, vz);
            gone |= wall32 (g.bc[1][0], true, g.n[0], i2, nx, vx);
            gone |= wall32 (g.bc[1][1], true, g.n[1], j2, ny, vy);
            gone |= wall32 (g.bc[1][2], true, g.n[2], k2, nz, vz);
            m.cell[n] = pack (i2, j2, k2);
            m.ox[n] = nx;
            m.oy[n] = ny;
            m.oz[n] = nz;
            m.ux[n] = vx;
            m.uy[n] = vy;
            m.uz[n] = vz;
            if (gone) {
               m.qm[n] = 0.0f;
               ++dead;
            }
         }
      }

      // Crossing times of the faces the path crosses (2 = none), sorted with
      // a three-element network; the path splits at each of them.
      float t0 = 2.0f, t1 = 2.0f, t2 = 2.0f;
      int a0 = 0, a1 = 1, a2 = 2;
      if (valid) {
         if (di) t0 = __fdividef ((di > 0 ? 1.0f : 0.0f) - ox, dx);
         if (dj) t1 = __fdividef ((dj > 0 ? 1.0f : 0.0f) - oy, dy);
         if (dk) t2 = __fdividef ((dk > 0 ? 1.0f : 0.0f) - oz, dz);
         CSWAP (t0, a0, t1, a1);
         CSWAP (t1, a1, t2, a2);
         CSWAP (t0, a0, t1, a1);
      }
      const float ta = fminf (t0, 1.0f);

      // Segments after the first: direct atomics in the cells entered.
      if (valid && t0 <= 1.0f) {
         int si = 0, sj = 0, sk = 0;
         const int d3[3] = {di, dj, dk};
         si += (a0 == 0) ? d3[0] : 0; sj += (a0 == 1) ? d3[1] : 0; sk += (a0 == 2) ? d3[2] : 0;
         deposit_piece (c, rho, i, j, k, si, sj, sk, ox, oy, oz, dx, dy, dz, t0, fminf (t1, 1.0f));
         if (t1 <= 1.0f) {
            si += (a1 == 0) ? d3[0] : 0; sj += (a1 == 1) ? d3[1] : 0; sk += (a1 == 2) ? d3[2] : 0;
            deposit_piece (c, rho, i, j, k, si, sj, sk, ox, oy, oz, dx, dy, dz, t1, fminf (t2, 1.0f));
            if (t2 <= 1.0f) {
               si += (a2 == 0) ? d3[0] : 0; sj += (a2 == 1) ? d3[1] : 0; sk += (a2 == 2) ? d3[2] : 0;
               deposit_piece (c, rho, i, j, k, si, sj, sk, ox, oy, oz, dx, dy, dz, t2, 1.0f);
            }
         }
      }

      // First segment (in the start cell): summed across lanes that share
      // the cell, one lane per run of equal cells issues the atomics.
      float wgt[12];
      if (valid)
         weights32 (c, rho, ox, ox + ta*dx, oy, oy + ta*dy, oz, oz + ta*dz, wgt);
      else
         for (int q = 0 ; q < 12 ; ++q) wgt[q] = 0.0f;
      const int key = valid ? (int) g.at (i, j, k) : -1 - lane;
      const int key0 = __shfl_sync (0xffffffffu, key, 0);
      if (__all_sync (0xffffffffu, key == key0 || !valid)) {
         // One cell for the whole warp: butterfly sums, lane 0 scatters.
#pragma unroll
         for (int q = 0 ; q < 12 ; ++q)
#pragma unroll
            for (int d = 16 ; d > 0 ; d >>= 1)
               wgt[q] += __shfl_xor_sync (0xffffffffu, wgt[q], d);
         const unsigned any = __ballot_sync (0xffffffffu, valid);
         if (any && lane == __ffs (any) - 1)
            scatter32 (c, i, j, k, wgt);
      } else {
         const int prev = __shfl_up_sync (0xffffffffu, key, 1);
         const int next = __shfl_down_sync (0xffffffffu, key, 1);
         const bool head = (lane == 0) || (prev != key);
         const bool tail = (lane == 31) || (next != key);
         const unsigned heads = __ballot_sync (0xffffffffu, head);
         const unsigned le = (lane == 31) ? 0xffffffffu : ((1u << (lane + 1)) - 1);
         const int seg_start = 31 - __clz (heads & le);
#pragma unroll
         for (int q = 0 ; q < 12 ; ++q)
            wgt[q] = seg_scan (wgt[q], lane, seg_start);
         if (valid && tail)
            scatter32 (c, i, j, k, wgt);
      }
   }

   __shared__ double sw[3][8];
   for (int d = 16 ; d > 0 ; d >>= 1) {
      Wx += __shfl_xor_sync (0xffffffffu, Wx, d);
      Wy += __shfl_xor_sync (0xffffffffu, Wy, d);
      Wz += __shfl_xor_sync (0xffffffffu, Wz, d);
      dead += __shfl_xor_sync (0xffffffffu, dead, d);
   }
   const int wid = threadIdx.x >> 5;
   if (lane == 0) {
      sw[0][wid] = Wx;
      sw[1][wid] = Wy;
      sw[2][wid] = Wz;
      if (dead)
         atomicAdd ((unsigned long long *) &dsc->dead, (unsigned long long) dead);
   }
   __syncthreads ();
   if (wid == 0) {
      const int nw = blockDim.x >> 5;
      Wx = lane < nw ? sw[0][lane] : 0;
      Wy = lane < nw ? sw[1][lane] : 0;
      Wz = lane < nw ? sw[2][lane] : 0;
      for (int d = 16 ; d > 0 ; d >>= 1) {
         Wx += __shfl_xor_sync (0xffffffffu, Wx, d);
         Wy += __shfl_xor_sync (0xffffffffu, Wy, d);
         Wz += __shfl_xor_sync (0xffffffffu, Wz, d);
      }
      if (lane == 0) {
         atomicAdd (&dsc->acc[2], Wx);
         atomicAdd (&dsc->acc[3], Wy);
         atomicAdd (&dsc->acc[4], Wz);
      }
   }
}

// Particle walls once at load time (plasma_init, core/plasma.c:399-404).
__global__ void k_walls32 (Grid g, Markers32 m, long long np, DevScalars *dsc)
{
   long long dead = 0;
   for (long long n = blockIdx.x*(long long) blockDim.x + threadIdx.x ; n < np ;
        n += (long long) gridDim.x*blockDim.x) {
      if (m.qm[n] == 0.0f)
         continue;
      const int cell = m.cell[n];
      int i = unpack (cell, 20), j = unpack (cell, 10), k = unpack (cell, 0);
      float ox = m.ox[n], oy = m.oy[n], oz = m.oz[n];
      float ux = m.ux[n], uy = m.uy[n], uz = m.uz[n];
      bool gone = false;
      gone |= wall32 (g.bc[0][0], false, g.n[0], i, ox, ux);
      gone |= wall32 (g.bc[0][1], false, g.n[1], j, oy, uy);
      gone |= wall32 (g.bc[0][2], false, g.n[2], k, oz, uz);
      gone |= wall32 (g.bc[1][0], true, g.n[0], i, ox, ux);
      gone |= wall32 (g.bc[1][1], true, g.n[1], j, oy, uy);
      gone |= wall32 (g.bc[1][2], true, g.n[2], k, oz, uz);
      m.cell[n] = pack (i, j, k);
      m.ox[n] = ox; m.oy[n] = oy; m.oz[n] = oz;
      m.ux[n] = ux; m.uy[n] = uy; m.uz[n] = uz;
      if (gone) {
         m.qm[n] = 0.0f;
         ++dead;
      }
   }
   if (dead)
      atomicAdd ((unsigned long long *) &dsc->dead, (unsigned long long) dead);
}

} // namespace

int mg_push32 (mg_run_t *r)
{
   if (r->np == 0)
      return MG_OK;
   Ctx32 c;
   c.g = r->g;
   c.E0 = r->E32[0]; c.E1 = r->E32[1]; c.E2 = r->E32[2];
   c.H0 = r->Hn32[0]; c.H1 = r->Hn32[1]; c.H2 = r->Hn32[2];
   c.J0 = r->J32[0]; c.J1 = r->J32[1]; c.J2 = r->J32[2];
   c.tau = (float) r->g.tau;
   for (int a = 0 ; a < 3 ; ++a) {
      c.rh[a] = (float) (1.0/r->g.h[a]);
      c.kj[a] = (float) (r->g.h[a]/r->g.tau);
   }
   c.vol = r->g.h[0]*r->g.h[1]*r->g.h[2];
   const int T = 256;
   k_push32<<<mg_blocks_for (r->np, T, 8), T, 0, r->stream>>> (c, r->m32, r->np, r->dsc);
   MG_LAUNCH_CHECK ();
   return MG_OK;
}

int mg_walls32 (mg_run_t *r)
{
   if (r->np == 0)
      return MG_OK;
   k_walls32<<<mg_blocks_for (r->np, 256, 8), 256, 0, r->stream>>> (r->g, r->m32, r->np, r->dsc);
   MG_LAUNCH_CHECK ();
   return MG_OK;
}
