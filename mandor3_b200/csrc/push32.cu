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
#include <cuda.h>                // CUtensorMap and the tensor-map encoder's types
#include <cuda_runtime.h>
#include <stdint.h>

#include "mg_internal.cuh"

namespace {

struct Ctx32 {
   Grid   g;
   const float *E0, *E1, *E2, *H0, *H1, *H2;
   float  *J0, *J1, *J2;
   float  tau, rh[3];            // tau, 1/h
   float  kj[3];                 // h_a / tau: current prefactor per unit rho and cell-unit displacement
   double vol;                   // h1 h2 h3 for the thermal tally
   int    kfront;                // nodes in front of k = 0 in a row (MG_GZ_FRONT32)
};

// Tensor maps of the six FP32 field arrays (Ex Ey Ez, Hx Hy Hz at t = n tau)
// of this GPU's run, for the tiled push's TMA copies of a tile's nodes.
struct TileMaps {
   CUtensorMap m[6];
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

// Block sums of the thermal tally and of the removed-marker count, added
// to the run's accumulators.
__device__ __forceinline__ void block_tally (double Wx, double Wy, double Wz, long long dead,
                                             DevScalars *dsc)
{
   __shared__ double sw[3][32];
   const int lane = threadIdx.x & 31;
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

// Markers [0, np), or [range[0], range[1]) when range is given (the markers
// that the tiled push leaves to global memory).
__global__ void __launch_bounds__ (256, 3)
k_push32 (Ctx32 c, long long np, const int *range, DevScalars *dsc)
{
   const Grid &g = c.g;
   const Markers32 m = dsc->m32;
   const int lane = threadIdx.x & 31;
   double Wx = 0, Wy = 0, Wz = 0;
   long long dead = 0;
   const long long warps_total = ((long long) gridDim.x*blockDim.x) >> 5;
   const long long warp0 = ((long long) blockIdx.x*blockDim.x + threadIdx.x) >> 5;
   const long long lo = range ? range[0] : 0, hi = range ? range[1] : np;
   for (long long base = lo + warp0*32 ; base < hi ; base += warps_total*32) {
      const long long n = base + lane;
      bool valid = n < hi;
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

   block_tally (Wx, Wy, Wz, dead, dsc);
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

// ---- tiled push --------------------------------------------------------------
// Markers are ordered by tile and cell (mg_sort32).  One CTA takes a tile at
// a time: it copies the E and H nodes around the tile into shared memory,
// pushes the tile's markers with gathers from there, accumulates their
// currents in a shared-memory copy of the tile's J nodes and adds that copy
// to J once per chunk of markers.  A marker may have drifted up to one cell
// outside its tile since the sort; further than that, it takes the
// global-memory path.
//
// The shared copy of J is fixed point in 32-bit integers, because integer
// shared-memory atomics are single instructions on this GPU while FP32 ones
// are compare-and-swap loops.  One marker adds at most (13/12) |rho| to any
// node over its whole path (|qx| = |rho v_x| <= |rho| and each weight factor
// lies in [-1/12, 13/12]), so with a quantum of 1.125 rho_max / Q for a
// chunk of L markers and Q = min(2^21, 2^30 / L), no node sum can leave the
// int32 range.  Contributions round to the nearest quantum: at most
// 2^-22 of the largest single contribution for chunks of up to 512 markers,
// 2^-17 at the 16384-marker limit.
#define MG_TILE_CHUNK 16384

// Fewest markers in a tile for the shared-memory staging of its fields and
// currents (about 13 staged values per marker at 256 markers of an 8x8x4
// tile); sparser tiles take the global-memory gather and current sums.
#ifndef MG_TILE_DENSE
#define MG_TILE_DENSE 256
#endif

// Asynchronous 4-byte copies global -> shared (completion per thread).
__device__ __forceinline__ void cp_async4 (void *sm, const void *gm)
{
   asm volatile ("cp.async.ca.shared.global [%0], [%1], 4;"
                 :: "r" ((unsigned) __cvta_generic_to_shared (sm)), "l" (gm) : "memory");
}

__device__ __forceinline__ void cp_async_commit ()
{
   asm volatile ("cp.async.commit_group;" ::: "memory");
}

__device__ __forceinline__ void cp_async_wait1 ()
{
   asm volatile ("cp.async.wait_group 1;" ::: "memory");
}


// ---- TMA tile copies and their mbarrier ----------------------------------------
__device__ __forceinline__ unsigned smem_u32 (const void *p)
{
   return (unsigned) __cvta_generic_to_shared (p);
}

__device__ __forceinline__ void mbar_init (uint64_t *bar, unsigned count)
{
   asm volatile ("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r" (smem_u32 (bar)), "r" (count) : "memory");
   asm volatile ("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One arrival that also announces `bytes` of copies completing on the barrier.
__device__ __forceinline__ void mbar_expect_tx (uint64_t *bar, unsigned bytes)
{
   asm volatile ("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r" (smem_u32 (bar)), "r" (bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait (uint64_t *bar, unsigned parity)
{
   unsigned ok;
   asm volatile ("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r" (ok) : "r" (smem_u32 (bar)), "r" (parity) : "memory");
   return ok != 0;
}

// Waits for the barrier's phase `parity` to complete, for at most
// MG_TMA_WAIT_CYCLES clock cycles (about 20 ms); false if it gave up.
#define MG_TMA_WAIT_CYCLES 40000000LL
__device__ __forceinline__ bool mbar_wait_bounded (uint64_t *bar, unsigned parity)
{
   const long long t0 = clock64 ();
   while (!mbar_try_wait (bar, parity))
      if (clock64 () - t0 > MG_TMA_WAIT_CYCLES)
         return false;
   return true;
}

// A 3D tile of a tensor map into shared memory (no multicast: the map
// covers this GPU's own field array), completing on `bar`.  c0 is the
// innermost (k) coordinate and must be a multiple of 4 floats.
__device__ __forceinline__ void tma_load3 (void *dst, const CUtensorMap *map, int c0, int c1, int c2,
                                           uint64_t *bar)
{
   asm volatile ("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4}], [%5];"
                 :: "r" (smem_u32 (dst)), "l" (map), "r" (c0), "r" (c1), "r" (c2), "r" (smem_u32 (bar))
                 : "memory");
}

// Starts the copy of marker n's nine pushed arrays into buffer b (the lane's
// column of the warp's staging area); n < 0: nothing to copy.
__device__ __forceinline__ void stage_marker (float *b, int lane, const Markers32 &m, int n)
{
   if (n >= 0) {
      cp_async4 (b + 0*32 + lane, m.cell + n);
      cp_async4 (b + 1*32 + lane, m.qm + n);
      cp_async4 (b + 2*32 + lane, m.ox + n);
      cp_async4 (b + 3*32 + lane, m.oy + n);
      cp_async4 (b + 4*32 + lane, m.oz + n);
      cp_async4 (b + 5*32 + lane, m.ux + n);
      cp_async4 (b + 6*32 + lane, m.uy + n);
      cp_async4 (b + 7*32 + lane, m.uz + n);
      cp_async4 (b + 8*32 + lane, m.rho + n);
   }
   cp_async_commit ();
}

template <int TX, int TY, int TZ, int NW = 8>
struct TileDims {
   // E, H nodes [x0-1, x0+TX+3): cells x0-1 .. x0+TX and the CIC stencil of
   // the half-shifted components.
   static constexpr int FX = TX + 4, FY = TY + 4, FZ = TZ + 4;
   static constexpr int FYZ = FY*FZ, FN = FX*FYZ;
   // J nodes [x0-2, x0+TX+3): a marker of cell x0-1 or x0+TX that moves one
   // more cell.
   static constexpr int JX = TX + 5, JY = TY + 5, JZ = TZ + 5;
   static constexpr int JYZ = JY*JZ, JN = JX*JYZ;
   // Per warp: two buffers of the nine marker arrays a push reads, 32 lanes each.
   static constexpr int STAGE = 2*9*32;
   // Per warp: a queue of QCAP markers that crossed cell faces, eight words
   // each (offsets, displacement, weight, packed cell and crossings).
   static constexpr int QCAP = 40, QUEUE = 8*QCAP;
   static constexpr size_t BYTES = (6*FN + 3*JN + NW*STAGE + NW*QUEUE)*sizeof (float);
   // Registers: at most 85 a thread for 4 and 8 warps a block, 64 for 16
   // (two blocks of 512 threads on an SM).
   static constexpr int MINB = NW == 4 ? 6 : NW == 8 ? 3 : 2;
};

template <int SX, int SY>
__device__ __forceinline__ float cic_s (const float *F, int q, float sx, float sy, float sz)
{
   const float f0 = F[q], f1 = F[q + SX], f2 = F[q + SY], f3 = F[q + SX + SY];
   const float f4 = F[q + 1], f5 = F[q + SX + 1], f6 = F[q + SY + 1], f7 = F[q + SX + SY + 1];
   const float a00 = f0 + sx*(f1 - f0), a10 = f2 + sx*(f3 - f2);
   const float a01 = f4 + sx*(f5 - f4), a11 = f6 + sx*(f7 - f6);
   const float b0 = a00 + sy*(a10 - a00), b1 = a01 + sy*(a11 - a01);
   return b0 + sz*(b1 - b0);
}

// Round w*S to the nearest integer (|w S| < 2^22): the sum with 1.5 * 2^23
// has unit spacing, so its bit pattern minus that of 1.5 * 2^23 is the result.
__device__ __forceinline__ int fixed (float w, float S)
{
   return __float_as_int (fmaf (w, S, 12582912.0f)) - 0x4B400000;
}

// Offset of weight `slot` (0..11) from the cell's node in the shared copy:
// the same nodes and order as scatter32 (Jx at (i+1, j+a, k+b), Jy at
// (i+a, j+1, k+b), Jz at (i+a, j+b, k+1)).
template <class D>
__device__ __forceinline__ int slot_offset (int slot)
{
   const int comp = slot >> 2, e = slot & 3, a = e & 1, b = e >> 1;
   const int off = comp == 0 ? D::JYZ + a*D::JZ + b
                 : comp == 1 ? D::JZ + a*D::JYZ + b
                 :             1 + a*D::JYZ + b*D::JZ;
   return comp*D::JN + off;
}

template <class D>
__device__ __forceinline__ void scatter_s (int *Jt, int q, const float w[12], float S)
{
#pragma unroll
   for (int s = 0 ; s < 12 ; ++s) {
      const int comp = s >> 2, e = s & 3, a = e & 1, b = e >> 1;
      const int off = comp*D::JN + (comp == 0 ? D::JYZ + a*D::JZ + b
                                  : comp == 1 ? D::JZ + a*D::JYZ + b
                                  :             1 + a*D::JYZ + b*D::JZ);
      atomicAdd (Jt + q + off, fixed (w[s], S));
   }
}

// Segments after the first of a marker that crossed cell faces: the
// crossing times in increasing order (ties keep the x, y, z order), then one
// in-cell segment per crossing, into the shared tile (FAST, node jq of the
// start cell) or into J (cell i, j, k).
template <class D, bool FAST>
__device__ __forceinline__ void later_segments (const Ctx32 &c, int *Jt, int jq, float S, int i, int j,
                                                int k, float ox, float oy, float oz, float dx, float dy,
                                                float dz, int di, int dj, int dk, float rho)
{
   float t0 = 2.0f, t1 = 2.0f, t2 = 2.0f;
   int a0 = 0, a1 = 1, a2 = 2;
   if (di) t0 = __fdividef ((di > 0 ? 1.0f : 0.0f) - ox, dx);
   if (dj) t1 = __fdividef ((dj > 0 ? 1.0f : 0.0f) - oy, dy);
   if (dk) t2 = __fdividef ((dk > 0 ? 1.0f : 0.0f) - oz, dz);
   CSWAP (t0, a0, t1, a1);
   CSWAP (t1, a1, t2, a2);
   CSWAP (t0, a0, t1, a1);
   int si = 0, sj = 0, sk = 0;
   float tb = t0;
   const int d3[3] = {di, dj, dk};
   const int ax3[3] = {a0, a1, a2};
   const float ts[4] = {t0, t1, t2, 2.0f};
#pragma unroll
   for (int p = 0 ; p < 3 ; ++p) {
      if (ts[p] <= 1.0f) {
         const int a = ax3[p];
         si += (a == 0) ? d3[0] : 0;
         sj += (a == 1) ? d3[1] : 0;
         sk += (a == 2) ? d3[2] : 0;
         const float te = fminf (ts[p + 1], 1.0f);
         float w[12];
         weights32 (c, rho, ox + tb*dx - si, ox + te*dx - si, oy + tb*dy - sj,
                    oy + te*dy - sj, oz + tb*dz - sk, oz + te*dz - sk, w);
         if (FAST)
            scatter_s<D> (Jt, jq + si*D::JYZ + sj*D::JZ + sk, w, S);
         else
            scatter32 (c, i + si, j + sj, k + sk, w);
         tb = te;
      }
   }
}

// The later segments of queue entry e of a warp's queue q.
template <class D>
__device__ __forceinline__ void queued_segments (const Ctx32 &c, int *Jt, const float *q, int e, float S)
{
   const int kb = __float_as_int (q[7*D::QCAP + e]);
   later_segments<D, true> (c, Jt, kb & 4095, S, 0, 0, 0, q[e], q[D::QCAP + e], q[2*D::QCAP + e],
                            q[3*D::QCAP + e], q[4*D::QCAP + e], q[5*D::QCAP + e], ((kb >> 12) & 3) - 1,
                            ((kb >> 14) & 3) - 1, ((kb >> 16) & 3) - 1, q[6*D::QCAP + e]);
}

// The tiled push: persistent blocks take tiles holding markers from the
// list built at the sort; per tile, the E and H nodes around it go to shared
// memory, each warp pushes its 32-marker rows from a cp.async double buffer,
// first-segment currents are summed per cell group into a fixed-point copy
// of the tile's J nodes, crossing markers queue their later segments, and
// the copy is added to J at the end of each chunk.  Tiles with fewer than
// MG_TILE_DENSE markers, and markers more than a cell outside their tile,
// gather from and add to global memory.
template <int TX, int TY, int TZ, int GROUP, bool PER, int NW>
__global__ void __launch_bounds__ (NW*32, (TileDims<TX, TY, TZ, NW>::MINB))
k_push32_tiles (Ctx32 c, const __grid_constant__ TileMaps maps, const int *tile_start, const int *tile_list,
                int nty, int ntz, int ntiles, DevScalars *dsc)
{
   const Markers32 m = dsc->m32;
   using D = TileDims<TX, TY, TZ, NW>;
   extern __shared__ __align__ (128) float smem[];
   __shared__ __align__ (8) uint64_t s_bar;   // completion of a tile's six TMA copies
   float *F = smem;                           // Ex Ey Ez Hx Hy Hz, D::FN each
   int *Jt = (int *) (smem + 6*D::FN);        // Jx Jy Jz, D::JN each
   float *stg = smem + 6*D::FN + 3*D::JN + (threadIdx.x >> 5)*D::STAGE;
   float *que = smem + 6*D::FN + 3*D::JN + NW*D::STAGE + (threadIdx.x >> 5)*D::QUEUE;
   __shared__ int s_tile;
   const Grid &g = c.g;
   const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
   const int soff = lane < 12 ? slot_offset<D> (lane) : 0;
   const float rmax = 1.125f*dsc->rho_max;
   const float vol = (float) c.vol;
   double Wx = 0, Wy = 0, Wz = 0;
   long long dead = 0;
   unsigned phase = 0;
   if (threadIdx.x == 0)
      mbar_init (&s_bar, 1);
   __syncthreads ();

   for (;;) {
      if (threadIdx.x == 0) {
         const int q = atomicAdd (&dsc->tile_next, 1);
         s_tile = q < tile_list[ntiles] ? tile_list[q] : -1;
      }
      __syncthreads ();
      const int t = s_tile;
      if (t < 0)
         break;
      const int mb = tile_start[t], me = tile_start[t + 1];
      if (mb < me) {
         const int x0 = (t/(nty*ntz))*TX, y0 = ((t/ntz) % nty)*TY, z0 = (t % ntz)*TZ;

         // A tile with few markers skips the staging: its markers gather
         // from and add to global memory.
         const bool dense = me - mb >= MG_TILE_DENSE;

         // Stage E and H nodes [x0-1, x0+TX+3) x ... : six TMA tile copies
         // (one per component, box FZ x FY x FX in allocation coordinates,
         // nodes past the arrays' ends read as zero) issued by one thread,
         // all threads waiting on the tile's mbarrier.  The barrier at the
         // end of the previous tile ordered every read of the old tile
         // before this proxy fence and the copies.
         if (dense) {
            if (threadIdx.x == 0) {
               asm volatile ("fence.proxy.async.shared::cta;" ::: "memory");
               mbar_expect_tx (&s_bar, 6*D::FN*(unsigned) sizeof (float));
#pragma unroll
               for (int comp = 0 ; comp < 6 ; ++comp)
                  tma_load3 (F + comp*D::FN, &maps.m[comp], z0 - 1 + c.kfront, y0 - 1 + MG_GX,
                             x0 - 1 + MG_GX, &s_bar);
            }
            const bool late = !mbar_wait_bounded (&s_bar, phase);
            phase ^= 1;
            if (__syncthreads_or (late)) {
               // The copies did not complete in time: report it and stop
               // this block (the step is flagged invalid on the host).
               if (threadIdx.x == 0)
                  atomicOr (&dsc->err, 8);
               break;
            }
         }

         for (int cb = mb ; cb < me ; cb += MG_TILE_CHUNK) {
            const int ce = min (cb + MG_TILE_CHUNK, me);
            const float Q = fminf (2097152.0f, 1073741824.0f/(float) (ce - cb));
            const float S = rmax > 0.0f ? Q/rmax : 0.0f;
            for (int q = threadIdx.x ; dense && q < 3*D::JN ; q += blockDim.x)
               Jt[q] = 0;
            __syncthreads ();

            // Each warp copies its next 32 markers into shared memory while
            // it pushes the current ones.
            stage_marker (stg, lane, m, cb + wid*32 + lane < ce ? cb + wid*32 + lane : -1);
            int it = 0, qn = 0;
            for (int base = cb + wid*32 ; base < ce ; base += nw*32, ++it) {
               const int n = base + lane;
               const int nn = n + nw*32;
               stage_marker (stg + ((it + 1) & 1)*(D::STAGE/2), lane, m, nn < ce ? nn : -1);
               cp_async_wait1 ();
               const float *cur = stg + (it & 1)*(D::STAGE/2) + lane;
               bool valid = n < ce;
               float qm = 0.0f;
               if (valid) {
                  qm = cur[1*32];
                  valid = (qm != 0.0f);
               }
               int i = 0, j = 0, k = 0, di = 0, dj = 0, dk = 0;
               float ox = 0, oy = 0, oz = 0, dx = 0, dy = 0, dz = 0, rho = 0;
               bool fast = false;
               if (valid) {
                  const int cell = __float_as_int (cur[0]);
                  i = unpack (cell, 20);
                  j = unpack (cell, 10);
                  k = unpack (cell, 0);
                  fast = dense && (unsigned) (i - x0 + 1) <= (unsigned) (TX + 1) &&
                         (unsigned) (j - y0 + 1) <= (unsigned) (TY + 1) &&
                         (unsigned) (k - z0 + 1) <= (unsigned) (TZ + 1);
                  if (!fast && (i < -1 || i > g.n[0] || j < -1 || j > g.n[1] || k < -1 || k > g.n[2])) {
                     if (atomicOr (&dsc->err, 1) == 0) {
                        dsc->err_info[0] = n;
                        dsc->err_info[1] = i;
                        dsc->err_info[2] = j;
                        dsc->err_info[3] = k;
                     }
                     valid = false;
                  }
               }
               if (valid) {
                  ox = cur[2*32];
                  oy = cur[3*32];
                  oz = cur[4*32];
                  const int hx = ox >= 0.5f, hy = oy >= 0.5f, hz = oz >= 0.5f;
                  const float sx_ = hx ? ox - 0.5f : ox + 0.5f;
                  const float sy_ = hy ? oy - 0.5f : oy + 0.5f;
                  const float sz_ = hz ? oz - 0.5f : oz + 0.5f;
                  float Ex, Ey, Ez, Hx, Hy, Hz;
                  if (fast) {
                     const int q = ((i - x0 + 1)*D::FY + (j - y0 + 1))*D::FZ + (k - z0 + 1);
                     const int qx = hx*D::FYZ, qy = hy*D::FZ, qz = hz;
                     Ex = cic_s<D::FYZ, D::FZ> (F, q + qx, sx_, oy, oz);
                     Ey = cic_s<D::FYZ, D::FZ> (F + D::FN, q + qy, ox, sy_, oz);
                     Ez = cic_s<D::FYZ, D::FZ> (F + 2*D::FN, q + qz, ox, oy, sz_);
                     Hx = cic_s<D::FYZ, D::FZ> (F + 3*D::FN, q + qy + qz, ox, sy_, sz_);
                     Hy = cic_s<D::FYZ, D::FZ> (F + 4*D::FN, q + qx + qz, sx_, oy, sz_);
                     Hz = cic_s<D::FYZ, D::FZ> (F + 5*D::FN, q + qx + qy, sx_, sy_, oz);
                  } else {
                     const int i_ = i + hx, j_ = j + hy, k_ = k + hz;
                     Ex = cic (c.E0, g, i_, sx_, j, oy, k, oz);
                     Ey = cic (c.E1, g, i, ox, j_, sy_, k, oz);
                     Ez = cic (c.E2, g, i, ox, j, oy, k_, sz_);
                     Hx = cic (c.H0, g, i, ox, j_, sy_, k_, sz_);
                     Hy = cic (c.H1, g, i_, sx_, j, oy, k_, sz_);
                     Hz = cic (c.H2, g, i_, sx_, j_, sy_, k, oz);
                  }

                  rho = cur[8*32];
                  const float tm = 0.5f*c.tau*qm;
                  const float px = cur[5*32] + tm*Ex, py = cur[6*32] + tm*Ey, pz = cur[7*32] + tm*Ez;
                  const float p2 = px*px + py*py + pz*pz;
                  const float rg = rsqrtf (1.0f + p2);
                  const float gamma = (1.0f + p2)*rg;
                  const float W = __fdividef (p2, (gamma + 1.0f)*(p2 + 1e-19f))*rho*vol/qm;
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
                        dsc->err_info[0] = n;
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
                  // PER: every wall periodic (the walls' branches fold away).
                  gone |= wall32 (PER ? MG_BC_PERIODIC : g.bc[0][0], false, g.n[0], i2, nx, vx);
                  gone |= wall32 (PER ? MG_BC_PERIODIC : g.bc[0][1], false, g.n[1], j2, ny, vy);
                  gone |= wall32 (PER ? MG_BC_PERIODIC : g.bc[0][2], false, g.n[2], k2, nz, vz);
                  gone |= wall32 (PER ? MG_BC_PERIODIC : g.bc[1][0], true, g.n[0], i2, nx, vx);
                  gone |= wall32 (PER ? MG_BC_PERIODIC : g.bc[1][1], true, g.n[1], j2, ny, vy);
                  gone |= wall32 (PER ? MG_BC_PERIODIC : g.bc[1][2], true, g.n[2], k2, nz, vz);
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

               // The first crossing time (see k_push32); markers of the tile
               // that crossed a face queue their later segments, the others
               // add theirs now.
               float tmin = 2.0f;
               if (valid) {
                  if (di) tmin = __fdividef ((di > 0 ? 1.0f : 0.0f) - ox, dx);
                  if (dj) tmin = fminf (tmin, __fdividef ((dj > 0 ? 1.0f : 0.0f) - oy, dy));
                  if (dk) tmin = fminf (tmin, __fdividef ((dk > 0 ? 1.0f : 0.0f) - oz, dz));
               }
               const float ta = fminf (tmin, 1.0f);
               const int jq = ((i - x0 + 2)*D::JY + (j - y0 + 2))*D::JZ + (k - z0 + 2);
               if (valid && !fast && tmin <= 1.0f)
                  later_segments<D, false> (c, Jt, 0, S, i, j, k, ox, oy, oz, dx, dy, dz, di, dj, dk, rho);

               // First segment: lanes are grouped by cell (match.any); a group
               // of at least GROUP lanes sums its weights across the warp
               // (redux.sync, one per weight) and lane q adds weight q; lanes
               // of smaller groups (markers that left the cell they were
               // sorted into) add their own.
               float wgt[12];
               if (valid)
                  weights32 (c, rho, ox, ox + ta*dx, oy, oy + ta*dy, oz, oz + ta*dz, wgt);
               else
                  for (int q = 0 ; q < 12 ; ++q) wgt[q] = 0.0f;
               if (valid && !fast)
                  scatter32 (c, i, j, k, wgt);
               // Lanes with key -1 (invalid, or pushed through global memory)
               // take part in no group sum, so their fx are never read.
               const int key = (valid && fast) ? jq : -1;
               int fx[12];
#pragma unroll
               for (int q = 0 ; q < 12 ; ++q)
                  fx[q] = fixed (wgt[q], S);
               const unsigned grp = __match_any_sync (0xffffffffu, key);
               const bool alone = key >= 0 && __popc (grp) < GROUP;
               unsigned heads = __ballot_sync (0xffffffffu, key >= 0 && !alone && (grp & ((1u << lane) - 1)) == 0);
#pragma unroll 1
               while (heads) {
                  const int k0 = __shfl_sync (0xffffffffu, key, __ffs (heads) - 1);
                  const bool mine = (key == k0);
                  int sum = 0;
#pragma unroll
                  for (int q = 0 ; q < 12 ; ++q) {
                     const int t = __reduce_add_sync (0xffffffffu, mine ? fx[q] : 0);
                     sum = lane == q ? t : sum;
                  }
                  if (lane < 12 && sum)
                     atomicAdd (Jt + k0 + soff, sum);
                  heads &= heads - 1;
               }
               if (alone) {
#pragma unroll
                  for (int q = 0 ; q < 12 ; ++q)
                     atomicAdd (Jt + key + slot_offset<D> (q), fx[q]);
               }

               // Queue the crossing markers; a full warp of them adds its
               // later segments at once.
               const bool cross = valid && fast && tmin <= 1.0f;
               const unsigned cm = __ballot_sync (0xffffffffu, cross);
               if (cm) {
                  const int nq = __popc (cm);
                  if (qn + nq > D::QCAP) {
                     if (lane < qn)
                        queued_segments<D> (c, Jt, que, lane, S);
                     qn = 0;
                     __syncwarp ();
                  }
                  if (cross) {
                     const int e = qn + __popc (cm & ((1u << lane) - 1));
                     que[e] = ox;
                     que[D::QCAP + e] = oy;
                     que[2*D::QCAP + e] = oz;
                     que[3*D::QCAP + e] = dx;
                     que[4*D::QCAP + e] = dy;
                     que[5*D::QCAP + e] = dz;
                     que[6*D::QCAP + e] = rho;
                     que[7*D::QCAP + e] = __int_as_float (jq | ((di + 1) << 12) | ((dj + 1) << 14) |
                                                          ((dk + 1) << 16));
                  }
                  qn += nq;
                  __syncwarp ();
                  if (qn >= 32) {
                     qn -= 32;
                     queued_segments<D> (c, Jt, que, qn + lane, S);
                     __syncwarp ();
                  }
               }
            }
            if (qn > 0 && lane < qn)
               queued_segments<D> (c, Jt, que, lane, S);
            __syncthreads ();

            // Add the chunk's currents to J.
            const float unit = S > 0.0f ? 1.0f/S : 0.0f;
            for (int q = threadIdx.x ; dense && q < 3*D::JN ; q += blockDim.x) {
               const int v = Jt[q];
               if (v == 0)
                  continue;
               const int comp = q/D::JN, rem = q - comp*D::JN;
               const int a = rem/D::JYZ, r2 = rem - a*D::JYZ, b = r2/D::JZ, cc = r2 - b*D::JZ;
               const int gi = x0 - 2 + a, gj = y0 - 2 + b, gk = z0 - 2 + cc;
               if (gi <= g.n[0] + MG_GX && gj <= g.n[1] + MG_GX && gk <= g.n[2] + MG_GX) {
                  float *dst = comp == 0 ? c.J0 : comp == 1 ? c.J1 : c.J2;
                  atomicAdd (dst + g.at (gi, gj, gk), (float) v*unit);
               }
            }
            __syncthreads ();
         }
      }
      __syncthreads ();
   }
   block_tally (Wx, Wy, Wz, dead, dsc);
}

} // namespace

// Smallest group of lanes in one cell whose first-segment weights are summed
// across the warp (measured on the 128^3 two-stream plasma, 64 markers per
// cell: 8 beats 3, 5, 12 and 16 lanes, and three rounds by first lane).
#ifndef MG_TILE_GROUP
#define MG_TILE_GROUP 8
#endif

#define TRY32(x)                                                             \
   do {                                                                      \
      int rc_ = (x);                                                         \
      if (rc_ != MG_OK)                                                      \
         return rc_;                                                         \
   } while (0)

// cuTensorMapEncodeTiled through the runtime's driver entry point (no
// link against the driver library).
typedef CUresult (*EncodeTiled) (CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                 CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                 CUtensorMapFloatOOBfill);

static EncodeTiled tensor_map_encoder ()
{
   static EncodeTiled fn = nullptr;
   if (!fn) {
      void *p = nullptr;
      cudaDriverEntryPointQueryResult q;
      if (cudaGetDriverEntryPoint ("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
          q == cudaDriverEntryPointSuccess)
         fn = (EncodeTiled) p;
   }
   return fn;
}

// The six field arrays as 3D tensors (k, j, i in allocation coordinates;
// k extent up to the last ghost node, so the row padding reads as zero)
// with a box of the tile's staged nodes.
template <int TX, int TY, int TZ>
static int make_tile_maps (const Ctx32 &c, TileMaps &tm)
{
   static_assert (TZ % 4 == 0, "TMA tile copies start at k = z0 - 1: z0 must be a multiple of 4");
   static_assert (MG_GZ_FRONT32 % 4 == 1, "k = z0 - 1 must fall on a multiple of 4 floats");
   const EncodeTiled enc = tensor_map_encoder ();
   if (!enc) {
      mg_set_error ("cuTensorMapEncodeTiled is not available from the CUDA driver");
      return MG_ERR_CUDA;
   }
   const Grid &g = c.g;
   const cuuint64_t dims[3] = {(cuuint64_t) (c.kfront + g.n[2] + 1 + MG_GX),
                               (cuuint64_t) (g.n[1] + 1 + 2*MG_GX), (cuuint64_t) (g.n[0] + 1 + 2*MG_GX)};
   const cuuint64_t strides[2] = {(cuuint64_t) g.sy*sizeof (float), (cuuint64_t) g.sx*sizeof (float)};
   const cuuint32_t box[3] = {TZ + 4, TY + 4, TX + 4};
   const cuuint32_t estr[3] = {1, 1, 1};
   const float *arr[6] = {c.E0, c.E1, c.E2, c.H0, c.H1, c.H2};
   if (strides[0] % 16 || strides[1] % 16) {
      mg_set_error ("field rows of %lld bytes cannot be copied by TMA", (long long) strides[0]);
      return MG_ERR_ARG;
   }
   for (int q = 0 ; q < 6 ; ++q) {
      if (((uintptr_t) arr[q]) % 16) {
         mg_set_error ("field array %d is not 16-byte aligned", q);
         return MG_ERR_ARG;
      }
      const CUresult e = enc (&tm.m[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *) arr[q], dims, strides, box,
                              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (e != CUDA_SUCCESS) {
         mg_set_error ("cuTensorMapEncodeTiled failed (%d) for field array %d", (int) e, q);
         return MG_ERR_CUDA;
      }
   }
   return MG_OK;
}

// Launches the tiled push of one tile size and block size (NW warps):
// persistent CTAs, as many as fit on the GPU (at most one per tile).
template <int TX, int TY, int TZ, int NW>
static int launch_tiles (mg_run_t *r, const Ctx32 &c, bool per)
{
   using D = TileDims<TX, TY, TZ, NW>;
   TileMaps tm;
   TRY32 ((make_tile_maps<TX, TY, TZ> (c, tm)));
   auto kp = k_push32_tiles<TX, TY, TZ, MG_TILE_GROUP, true, NW>;
   auto kn = k_push32_tiles<TX, TY, TZ, MG_TILE_GROUP, false, NW>;
   static int attr_dev = -1;
   static int per_sm = 1, sms = 148;
   if (attr_dev != r->device) {
      MG_CUDA (cudaFuncSetAttribute (kp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) D::BYTES));
      MG_CUDA (cudaFuncSetAttribute (kn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) D::BYTES));
      MG_CUDA (cudaOccupancyMaxActiveBlocksPerMultiprocessor (&per_sm, kn, NW*32, D::BYTES));
      MG_CUDA (cudaDeviceGetAttribute (&sms, cudaDevAttrMultiProcessorCount, r->device));
      if (per_sm < 1)
         per_sm = 1;
      attr_dev = r->device;
   }
   int blocks = sms*per_sm;
   if (blocks > r->ntiles)
      blocks = r->ntiles;
   MG_CUDA (cudaMemsetAsync (&r->dsc->tile_next, 0, sizeof (int), r->stream));
   (per ? kp : kn)<<<blocks, NW*32, D::BYTES, r->stream>>> (c, tm, r->tile_start, r->tile_list, r->tiles[1],
                                                              r->tiles[2], r->ntiles, r->dsc);
   MG_LAUNCH_CHECK ();
   return MG_OK;
}

template <int TX, int TY, int TZ>
static int launch_tiles_nw (mg_run_t *r, const Ctx32 &c, bool per)
{
   switch (r->prm.tile_warps) {
   case 4:  return launch_tiles<TX, TY, TZ, 4> (r, c, per);
   case 16: return launch_tiles<TX, TY, TZ, 16> (r, c, per);
   default: return launch_tiles<TX, TY, TZ, 8> (r, c, per);
   }
}

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
   c.kfront = (int) (r->g.origin - MG_GX*r->g.sx - MG_GX*r->g.sy);
   const int T = 256;
   if (!r->tiles_ok) {
      k_push32<<<mg_blocks_for (r->np, T, 8), T, 0, r->stream>>> (c, r->np, nullptr, r->dsc);
      MG_LAUNCH_CHECK ();
      return MG_OK;
   }
   bool per = true;
   for (int a = 0 ; a < 3 ; ++a)
      per = per && r->g.bc[0][a] == MG_BC_PERIODIC && r->g.bc[1][a] == MG_BC_PERIODIC;
   const int *td = r->tdim;
   if (td[0] == 4 && td[1] == 4 && td[2] == 4)
      TRY32 ((launch_tiles_nw<4, 4, 4> (r, c, per)));
   else if (td[0] == 8 && td[1] == 8 && td[2] == 8)
      TRY32 ((launch_tiles_nw<8, 8, 8> (r, c, per)));
   else
      TRY32 ((launch_tiles_nw<8, 8, 4> (r, c, per)));
   int sms = 148;
   MG_CUDA (cudaDeviceGetAttribute (&sms, cudaDevAttrMultiProcessorCount, r->device));
   // Markers outside the mesh at the last sort: global-memory path.
   k_push32<<<sms, T, 0, r->stream>>> (c, r->np, r->tile_start + r->ntiles, r->dsc);
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
