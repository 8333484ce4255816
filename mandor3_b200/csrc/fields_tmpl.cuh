// Yee solver, field boundary conditions, current folding and energy
// reductions of the B200 PIC core, templated on the field type: double for
// the FP64 form (fields64.cu), float for the FP32-offset form (fields32.cu).
// Energy sums, time and the laser phase are FP64 in both forms.
//
// Reference semantics (paths relative to the reference project):
//   H half step   core/em.c:55-77, caps core/em_caps.c:406-729
//   E step        core/em.c:135-163, E -= tau*J core/em.c:167-184
//   periodic BC   core/emCap_periodic.c:15-67
//   mirror BC     core/emCap_mirror.c:17-70
//   Mur BC        core/emCap_Mur.c:56-166
//   J folding     core/plasma_currentWalls.c:27-121
//   field energy  core/em.c:227-252
//
// The reference splits every update into an inner box and six boundary
// "caps" so that MPI exchange overlaps compute.  With the whole domain on
// one GPU the union of those regions is one box per field (per axis:
// H over [0,n] or [1,n] at a mirror wall; E over [0 or 1, n-1 or n]), so
// each update is a single launch over that box followed by thin wall
// kernels.  The caps advance H by one tau instead of two tau/2 halves, so
// near-wall values agree with the reference to round-off.
//
// The FP64 instantiation is compiled with --fmad=false so that every
// expression rounds exactly as the reference's C does.
#pragma once

#include <cuda_runtime.h>

#include <limits.h>

#include "mg_internal.cuh"

#define TRY_MG(x)                                                            \
   do {                                                                      \
      int rc_ = (x);                                                         \
      if (rc_ != MG_OK)                                                      \
         return rc_;                                                         \
   } while (0)

namespace {


template <typename T>
struct F3T {
   T *c[3];
};

__device__ __forceinline__ void box_index (long t, const int lo[3], const int ext[3],
                                           int &i, int &j, int &k)
{
   k = lo[2] + (int) (t % ext[2]);
   t /= ext[2];
   j = lo[1] + (int) (t % ext[1]);
   i = lo[0] + (int) (t / ext[1]);
}

struct Box {
   int lo[3], ext[3];
   long vol;
};

// Node indices of a grid-stride walk over a box without a division per
// node: the stride's own decomposition is added with one carry per axis
// (each digit of the stride is below its extent).
struct BoxWalk {
   int i, j, k;              // box coordinates of the current node
   int si, sj, sk;           // the stride in box coordinates
};

__device__ __forceinline__ void walk_init (BoxWalk &w, long t, long stride, const Box &b)
{
   w.k = (int) (t % b.ext[2]);
   t /= b.ext[2];
   w.j = (int) (t % b.ext[1]);
   w.i = (int) (t / b.ext[1]);
   w.sk = (int) (stride % b.ext[2]);
   stride /= b.ext[2];
   w.sj = (int) (stride % b.ext[1]);
   w.si = (int) (stride / b.ext[1]);
}

__device__ __forceinline__ void walk_step (BoxWalk &w, const Box &b)
{
   w.k += w.sk;
   int c = w.k >= b.ext[2];
   if (c) w.k -= b.ext[2];
   w.j += w.sj + c;
   c = w.j >= b.ext[1];
   if (c) w.j -= b.ext[1];
   w.i += w.si + c;
}


static Box make_box (const int lo[3], const int hi[3])
{
   Box b;
   b.vol = 1;
   for (int a = 0 ; a < 3 ; ++a) {
      b.lo[a] = lo[a];
      b.ext[a] = hi[a] - lo[a] + 1;
      if (b.ext[a] < 0) b.ext[a] = 0;
      b.vol *= b.ext[a];
   }
   return b;
}

// Both H half steps in one pass (core/em.c:55-77, called twice per step
// with the same E^n): Hn = H + c curl E is H at t = n tau (gathered by the
// push, summed by the energy), H = Hn + c curl E is H at t = (n+1/2) tau.
// Each result rounds exactly as the reference's two successive updates do.
// The field energy of core/em.c:227-252 is summed on the way: E^n at the
// staggered picks and Hn at its picks, where a node whose value the walls
// will replace is represented by the node the walls copy it from.
struct EnergyPick {
   int lo[3][3], hi[3][3];    // [component][axis] index ranges of E picks
   int hlo[3][3], hhi[3][3];  // same for H picks (after the periodic remap)
};

// HN: keep H^n in Hn (the push, the probes and the stage path read it); a
// run without markers or probes skips those stores.
// MG_BULK_NODES nodes per thread and iteration, all loads issued before
// the first store (a node writes only itself, so no load aliases an earlier
// store): twice the bytes in flight per thread.  The energy sums keep the
// node order of one node per iteration.
#ifndef MG_BULK_NODES
#define MG_BULK_NODES 2
#endif

template <typename T, bool HN = true>
__global__ void __launch_bounds__ (256)
k_h_fused (Grid g, F3T<T> E, F3T<T> H, F3T<T> Hn, Box b, T c1, T c2, T c3,
           EnergyPick ep, DevScalars *dsc)
{
   constexpr int NU = MG_BULK_NODES;
   __shared__ double sw[2][8];
   const T *Ex = E.c[0], *Ey = E.c[1], *Ez = E.c[2];
   const long sx = g.sx, sy = g.sy;
   const long stride = (long) gridDim.x*blockDim.x;
   double we = 0, wb = 0;   // FP64 reductions in both forms
   BoxWalk wk;
   walk_init (wk, blockIdx.x*(long) blockDim.x + threadIdx.x, stride, b);
   for (long t0 = blockIdx.x*(long) blockDim.x + threadIdx.x ; t0 < b.vol ; t0 += NU*stride) {
      long o[NU];
      int I[NU][3];
      T ex[NU], ey[NU], ez[NU], dy[NU], dzy[NU], dzx[NU], dx[NU], dxy[NU], dyx[NU], h0[NU], h1[NU], h2[NU];
#pragma unroll
      for (int u = 0 ; u < NU ; ++u) {
         const long t = t0 + u*stride;
         o[u] = -1;
         I[u][0] = b.lo[0] + wk.i;
         I[u][1] = b.lo[1] + wk.j;
         I[u][2] = b.lo[2] + wk.k;
         walk_step (wk, b);
         if (t < b.vol) {
            const long x = g.at (I[u][0], I[u][1], I[u][2]);
            o[u] = x;
            ex[u] = Ex[x];
            ey[u] = Ey[x];
            ez[u] = Ez[x];
            dy[u] = Ey[x - 1];
            dzy[u] = Ez[x - sy];
            dzx[u] = Ez[x - sx];
            dx[u] = Ex[x - 1];
            dxy[u] = Ex[x - sy];
            dyx[u] = Ey[x - sx];
            h0[u] = H.c[0][x];
            h1[u] = H.c[1][x];
            h2[u] = H.c[2][x];
         }
      }
      // The precision form sums an iteration's squares in FP32 and adds
      // them to the FP64 totals once; the FP64 form adds every square.
      float se = 0.0f, sb = 0.0f;
#pragma unroll
      for (int u = 0 ; u < NU ; ++u) {
         if (o[u] < 0)
            continue;
         const long x = o[u];
         const T cx = c3*(ey[u] - dy[u]) - c2*(ez[u] - dzy[u]);
         const T cy = c1*(ez[u] - dzx[u]) - c3*(ex[u] - dx[u]);
         const T cz = c2*(ex[u] - dxy[u]) - c1*(ey[u] - dyx[u]);
         const T hx = h0[u] + cx, hy = h1[u] + cy, hz = h2[u] + cz;
         if (HN) {
            Hn.c[0][x] = hx;
            Hn.c[1][x] = hy;
            Hn.c[2][x] = hz;
         }
         H.c[0][x] = hx + cx;
         H.c[1][x] = hy + cy;
         H.c[2][x] = hz + cz;
         const T ev[3] = {ex[u], ey[u], ez[u]}, hv[3] = {hx, hy, hz};
#pragma unroll
         for (int c = 0 ; c < 3 ; ++c) {
            bool in_e = true, in_h = true;
#pragma unroll
            for (int a = 0 ; a < 3 ; ++a) {
               in_e &= (I[u][a] >= ep.lo[c][a]) & (I[u][a] <= ep.hi[c][a]);
               in_h &= (I[u][a] >= ep.hlo[c][a]) & (I[u][a] <= ep.hhi[c][a]);
            }
            if (sizeof (T) == sizeof (float)) {
               if (in_e) se += (float) ev[c]*(float) ev[c];
               if (in_h) sb += (float) hv[c]*(float) hv[c];
            } else {
               if (in_e) we += (double) ev[c]*(double) ev[c];
               if (in_h) wb += (double) hv[c]*(double) hv[c];
            }
         }
      }
      if (sizeof (T) == sizeof (float)) {
         we += (double) se;
         wb += (double) sb;
      }
   }
   for (int d = 16 ; d > 0 ; d >>= 1) {
      we += __shfl_xor_sync (0xffffffffu, we, d);
      wb += __shfl_xor_sync (0xffffffffu, wb, d);
   }
   const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
   if (lane == 0) {
      sw[0][wid] = we;
      sw[1][wid] = wb;
   }
   __syncthreads ();
   if (wid == 0) {
      we = lane < (int) (blockDim.x >> 5) ? sw[0][lane] : 0;
      wb = lane < (int) (blockDim.x >> 5) ? sw[1][lane] : 0;
      for (int d = 16 ; d > 0 ; d >>= 1) {
         we += __shfl_xor_sync (0xffffffffu, we, d);
         wb += __shfl_xor_sync (0xffffffffu, wb, d);
      }
      if (lane == 0) {
         atomicAdd (&dsc->acc[0], we);
         atomicAdd (&dsc->acc[1], wb);
      }
   }
}

// E -= tau*(curl H) over the E box (core/em.c:155-162 expression order).
template <typename T>
__global__ void k_e_advance (Grid g, F3T<T> E, F3T<T> H, Box b, T c1, T c2, T c3)
{
   T *Ex = E.c[0], *Ey = E.c[1], *Ez = E.c[2];
   const T *Hx = H.c[0], *Hy = H.c[1], *Hz = H.c[2];
   const long sx = g.sx, sy = g.sy;
   for (long t = blockIdx.x*(long) blockDim.x + threadIdx.x ; t < b.vol ; t += (long) gridDim.x*blockDim.x) {
      int i, j, k;
      box_index (t, b.lo, b.ext, i, j, k);
      const long o = g.at (i, j, k);
      const T hx = Hx[o], hy = Hy[o], hz = Hz[o];
      Ex[o] -= c3*(Hy[o + 1] - hy) - c2*(Hz[o + sy] - hz);
      Ey[o] -= c1*(Hz[o + sx] - hz) - c3*(Hx[o + 1] - hx);
      Ez[o] -= c2*(Hx[o + sy] - hx) - c1*(Hy[o + sx] - hy);
   }
}

// E step with the current term (core/em.c:155-162 then 167-184) for nodes
// that no wall operation or source touches between the two: rim nodes
// (indices -1, 0, 1, n-1, n, n+1 on any axis, and the laser E plane) get
// only the curl here and their -tau J after the walls (k_e_rim).
struct Rim {
   int lo[3], hi[3];       // a node is inner on axis a if lo[a] <= idx <= hi[a]
   int laser_i;            // x index of the laser E plane, or INT_MIN
   int laser_lo[2], laser_hi[2];   // its j and k ranges
};

__device__ __forceinline__ bool rim_node (const Rim &rm, int i, int j, int k)
{
   return i < rm.lo[0] || i > rm.hi[0] || j < rm.lo[1] || j > rm.hi[1] ||
          k < rm.lo[2] || k > rm.hi[2] ||
          (i == rm.laser_i && j >= rm.laser_lo[0] && j <= rm.laser_hi[0] &&
           k >= rm.laser_lo[1] && k <= rm.laser_hi[1]);
}

// WJ: subtract tau J (a run without markers has J = 0 and skips its reads).
template <typename T, bool WJ = true>
__global__ void __launch_bounds__ (256)
k_e_fused (Grid g, F3T<T> E, F3T<T> H, F3T<T> J, Box b, T c1, T c2, T c3, Rim rm)
{
   constexpr int NU = MG_BULK_NODES;
   T *Ex = E.c[0], *Ey = E.c[1], *Ez = E.c[2];
   const T *Hx = H.c[0], *Hy = H.c[1], *Hz = H.c[2];
   const long sx = g.sx, sy = g.sy;
   const T tau = (T) g.tau;
   const long stride = (long) gridDim.x*blockDim.x;
   BoxWalk wk;
   walk_init (wk, blockIdx.x*(long) blockDim.x + threadIdx.x, stride, b);
   for (long t0 = blockIdx.x*(long) blockDim.x + threadIdx.x ; t0 < b.vol ; t0 += NU*stride) {
      long o[NU];
      bool sub[NU];
      T e0[NU], e1[NU], e2[NU], hx[NU], hy[NU], hz[NU], hy1[NU], hzy[NU], hzx[NU], hx1[NU], hxy[NU], hyx[NU];
      T j0[NU], j1[NU], j2[NU];
#pragma unroll
      for (int u = 0 ; u < NU ; ++u) {
         const long t = t0 + u*stride;
         o[u] = -1;
         const int i = b.lo[0] + wk.i, j = b.lo[1] + wk.j, k = b.lo[2] + wk.k;
         walk_step (wk, b);
         if (t < b.vol) {
            const long x = g.at (i, j, k);
            o[u] = x;
            hx[u] = Hx[x];
            hy[u] = Hy[x];
            hz[u] = Hz[x];
            hy1[u] = Hy[x + 1];
            hzy[u] = Hz[x + sy];
            hzx[u] = Hz[x + sx];
            hx1[u] = Hx[x + 1];
            hxy[u] = Hx[x + sy];
            hyx[u] = Hy[x + sx];
            e0[u] = Ex[x];
            e1[u] = Ey[x];
            e2[u] = Ez[x];
            sub[u] = WJ && !rim_node (rm, i, j, k);
            if (sub[u]) {
               j0[u] = J.c[0][x];
               j1[u] = J.c[1][x];
               j2[u] = J.c[2][x];
            }
         }
      }
#pragma unroll
      for (int u = 0 ; u < NU ; ++u) {
         if (o[u] < 0)
            continue;
         const long x = o[u];
         T ex = e0[u] - (c3*(hy1[u] - hy[u]) - c2*(hzy[u] - hz[u]));
         T ey = e1[u] - (c1*(hzx[u] - hz[u]) - c3*(hx1[u] - hx[u]));
         T ez = e2[u] - (c2*(hxy[u] - hx[u]) - c1*(hyx[u] - hy[u]));
         if (sub[u]) {
            ex -= tau*j0[u];
            ey -= tau*j1[u];
            ez -= tau*j2[u];
         }
         Ex[x] = ex;
         Ey[x] = ey;
         Ez[x] = ez;
      }
   }
}


// ---------------------------------------------------------------------------
// Field-only step in one pass (plain form: runs without markers, sources or
// probes).  E^(n+1) at a node needs H^(n+1/2) at the node and at its +1
// neighbours, computed from E^n and H^(n-1/2) with the H pass's expressions
// (the same bits, no contraction in the FP64 build).  E and H are
// double-buffered: the pass reads the old arrays and writes the new ones, so
// each node is one read of E and H and one write of each (96 B instead of
// the two passes' 144 B).
//
// Which nodes can skip the walls: the H walls write H at index 0 and n + 1
// of an axis, and the axis' own component at n (mirror); the new H at any
// node needs only E^n and H^(n-1/2), so one pass computes it over the whole
// H box.  The new E at index m of an axis reads the new H at m and, for the
// components across the axis, at m + 1; for m in [1, n - 1] none of those is
// a wall's, so the pass computes E over [1, n - 1]^3 as well.  What is left
// is the single layer of the E box at index 0 (periodic axes) or n (the
// others), updated from the walled H after the H walls.
// ---------------------------------------------------------------------------
struct Slabs {
   Box  b[6];
   long start[7];
};

// Box b minus the box [in_lo, in_hi]^3 (axis-wise), as six slabs.
static Slabs shell_slabs (const Box &b, const int in_lo[3], const int in_hi[3])
{
   int lo[3], hi[3];
   for (int a = 0 ; a < 3 ; ++a) {
      lo[a] = b.lo[a];
      hi[a] = b.lo[a] + b.ext[a] - 1;
   }
   Slabs s;
   int n = 0;
   auto add = [&] (int l0, int h0, int l1, int h1, int l2, int h2) {
      const int l[3] = {l0, l1, l2}, h[3] = {h0, h1, h2};
      s.b[n++] = make_box (l, h);
   };
   add (lo[0], in_lo[0] - 1, lo[1], hi[1], lo[2], hi[2]);
   add (in_hi[0] + 1, hi[0], lo[1], hi[1], lo[2], hi[2]);
   add (in_lo[0], in_hi[0], lo[1], in_lo[1] - 1, lo[2], hi[2]);
   add (in_lo[0], in_hi[0], in_hi[1] + 1, hi[1], lo[2], hi[2]);
   add (in_lo[0], in_hi[0], in_lo[1], in_hi[1], lo[2], in_lo[2] - 1);
   add (in_lo[0], in_hi[0], in_lo[1], in_hi[1], in_hi[2] + 1, hi[2]);
   s.start[0] = 0;
   for (int q = 0 ; q < 6 ; ++q) {
      if (s.b[q].vol < 0)
         s.b[q].vol = 0;
      s.start[q + 1] = s.start[q] + s.b[q].vol;
   }
   return s;
}

__device__ __forceinline__ bool slab_node (const Slabs &S, long t, int &i, int &j, int &k)
{
   if (t >= S.start[6])
      return false;
   int q = 0;
   while (t >= S.start[q + 1])
      ++q;
   box_index (t - S.start[q], S.b[q].lo, S.b[q].ext, i, j, k);
   return true;
}

// Energy sums of one node at its picks (core/em.c:241-247).
template <typename T>
__device__ __forceinline__ void energy_add (const EnergyPick &ep, int i, int j, int k, const T ev[3],
                                            const T hv[3], double &we, double &wb)
{
   const int I[3] = {i, j, k};
#pragma unroll
   for (int c = 0 ; c < 3 ; ++c) {
      bool in_e = true, in_h = true;
#pragma unroll
      for (int a = 0 ; a < 3 ; ++a) {
         in_e &= (I[a] >= ep.lo[c][a]) & (I[a] <= ep.hi[c][a]);
         in_h &= (I[a] >= ep.hlo[c][a]) & (I[a] <= ep.hhi[c][a]);
      }
      if (in_e) we += (double) ev[c]*(double) ev[c];
      if (in_h) wb += (double) hv[c]*(double) hv[c];
   }
}

__device__ __forceinline__ void energy_flush (double we, double wb, DevScalars *dsc)
{
   __shared__ double sw[2][8];
   for (int d = 16 ; d > 0 ; d >>= 1) {
      we += __shfl_xor_sync (0xffffffffu, we, d);
      wb += __shfl_xor_sync (0xffffffffu, wb, d);
   }
   const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
   if (lane == 0) {
      sw[0][wid] = we;
      sw[1][wid] = wb;
   }
   __syncthreads ();
   if (wid == 0) {
      we = lane < (int) (blockDim.x >> 5) ? sw[0][lane] : 0;
      wb = lane < (int) (blockDim.x >> 5) ? sw[1][lane] : 0;
      for (int d = 16 ; d > 0 ; d >>= 1) {
         we += __shfl_xor_sync (0xffffffffu, we, d);
         wb += __shfl_xor_sync (0xffffffffu, wb, d);
      }
      if (lane == 0) {
         atomicAdd (&dsc->acc[0], we);
         atomicAdd (&dsc->acc[1], wb);
      }
   }
}

// The H box as (y, z) tiles of YT x ZT nodes, each block marching along x
// over a chunk of planes [i0, i1).  Per plane p the block holds in shared
// memory E^n of planes p - 1, p (tile plus the -1 and +1 halos), p + 1 and
// p + 2 (arriving by cp.async while p is computed), and H^(n+1/2) of planes
// p - 1 and p on the tile plus the +1 halo: it computes the new H of plane p
// from E^n (planes p - 1, p) and H^(n-1/2), then the new E of plane p - 1
// from E^n and the new H of planes p - 1, p.  Tiles partition [lo, n - 1] on
// each axis; the last tile of an axis also owns node n, its +1 halo there.
// Halo values of the new H are computed again by each tile that needs them,
// from the same inputs, so they are the same bits.
// E rows move as 16-byte chunks: rows start at multiples of 4 elements and
// node k = 0 sits at offset 4 (FP64) or 5 (FP32) of its row, so node kb - A
// starts a chunk for kb a multiple of 4 (A = 2 for FP64, 1 for FP32); a row
// of the tile holds k in [kb - A, kb - A + EW).
template <typename T, int YT, int ZT>
struct YeeTile {
   static constexpr int NT = YT*ZT;               // threads, one per tile node
   static constexpr int V = 16/(int) sizeof (T);  // elements per chunk
   static constexpr int A = sizeof (T) == 8 ? 2 : 1;
   static constexpr int EW = (ZT + 1 + A + V - 1)/V*V;   // E row pitch: k in [kb - A, kb + ZT]
   static constexpr int NCH = EW/V;               // chunks per E row
   static constexpr int EP = (YT + 2)*EW;         // E plane: j in [jb - 1, jb + YT]
   static constexpr int HW = ZT + 1;              // new-H row pitch: k in [kb, kb + ZT]
   static constexpr int HP = (YT + 1)*HW;         // new-H plane: j in [jb, jb + YT]
   static constexpr int XH = YT + ZT + 1;         // +1 halo nodes of the new H
};

__device__ __forceinline__ void cp_async16 (void *sm, const void *gm)
{
   asm volatile ("cp.async.cg.shared.global [%0], [%1], 16;"
                 :: "r" ((unsigned) __cvta_generic_to_shared (sm)), "l" (gm) : "memory");
}

struct YeeTiles {
   int lo[3];              // first node of the H box on each axis (0, or 1 at a mirror)
   int n[3];               // cells: the H box ends at n, the E interior is [1, n - 1]
   int tj0, ntj, tk0, ntk; // first tile index and tile count along y and z
   int cx;                 // planes per chunk
};

template <typename T, int YT, int ZT>
__global__ void __launch_bounds__ (YT*ZT, 4)
k_yee_tile (Grid g, F3T<T> E, F3T<T> H, F3T<T> En, F3T<T> Hnw, YeeTiles tl, T c1, T c2, T c3,
            T d1, T d2, T d3, EnergyPick ep, DevScalars *dsc)
{
   using L = YeeTile<T, YT, ZT>;
   __shared__ __align__ (16) T sE[4][3][L::EP];
   __shared__ T sH[2][3][L::HP];
   const int tid = threadIdx.x;
   int b = blockIdx.x;
   const int tk = tl.tk0 + b % tl.ntk;
   b /= tl.ntk;
   const int tj = tl.tj0 + b % tl.ntj;
   b /= tl.ntj;
   const int nx = tl.n[0], ny = tl.n[1], nz = tl.n[2];
   const int i0 = tl.lo[0] + b*tl.cx, i1 = min (i0 + tl.cx, nx);
   const bool lasti = i1 == nx;                       // the chunk owns plane n too
   const int jb = tj*YT, kb = tk*ZT;                  // tile base
   const int ja = max (jb, tl.lo[1]), je = min (jb + YT - 1, ny - 1);   // rows
   const int ka = max (kb, tl.lo[2]), ke = min (kb + ZT - 1, nz - 1);   // columns
   const bool lastj = je == ny - 1, lastk = ke == nz - 1;
   const long sx = g.sx, sy = g.sy;

   // E^n of plane p into slot s: the chunks of rows [ja - 1, je + 1] that
   // meet columns [ka - 1, ke + 1].  A chunk may run up to three elements
   // past the row into the next one (rows up to n, never the last of the
   // allocation); those elements are not read.
   auto load_e = [&] (int p, int s) {
      for (int q = tid ; q < (YT + 2)*L::NCH ; q += L::NT) {
         const int r = q/L::NCH, m = q - r*L::NCH;
         const int j = jb - 1 + r, k = kb - L::A + m*L::V;
         if (j >= ja - 1 && j <= je + 1 && k + L::V - 1 >= ka - 1 && k <= ke + 1) {
            const long o = g.at (p, j, k);
#pragma unroll
            for (int e = 0 ; e < 3 ; ++e)
               cp_async16 (&sE[s][e][r*L::EW + m*L::V], E.c[e] + o);
         }
      }
   };
   // This thread's new-H nodes: the tile node (tid / ZT, tid % ZT), and for
   // the first XH threads one node of the +1 halo (row YT, then column ZT).
   // Computed where the tile's new E needs them; written where the tile owns
   // them.
   const int r0 = tid/ZT, q0 = tid - r0*ZT;
   const int r1 = tid <= ZT ? YT : tid - ZT - 1, q1 = tid <= ZT ? tid : ZT;
   const int j0 = jb + r0, k0 = kb + q0, j1 = jb + r1, k1 = kb + q1;
   const bool need0 = j0 >= ja && j0 <= je + 1 && k0 >= ka && k0 <= ke + 1;
   const bool need1 = tid < L::XH && j1 >= ja && j1 <= je + 1 && k1 >= ka && k1 <= ke + 1;
   const bool own0 = need0 && (j0 <= je || lastj) && (k0 <= ke || lastk);
   const bool own1 = need1 && (j1 <= je || lastj) && (k1 <= ke || lastk);
   const bool ownE = j0 >= max (ja, 1) && j0 <= je && k0 >= max (ka, 1) && k0 <= ke;
   T h0[3] = {0, 0, 0}, h1[3] = {0, 0, 0};             // H^(n-1/2) of the next plane
   auto load_h = [&] (int p) {
      if (need0) {
         const long o = g.at (p, j0, k0);
#pragma unroll
         for (int e = 0 ; e < 3 ; ++e) h0[e] = H.c[e][o];
      }
      if (need1) {
         const long o = g.at (p, j1, k1);
#pragma unroll
         for (int e = 0 ; e < 3 ; ++e) h1[e] = H.c[e][o];
      }
   };
   double we = 0, wb = 0;
   // The new H at tile-relative node (r, q) of plane p (E slot se, previous
   // plane's slot sp) into new-H slot sh, k_h_fused's expressions; written
   // to Hnw with its energy terms where owned.
   auto h_node = [&] (int p, int r, int q, int se, int sp, int sh, const T ho[3], bool own) {
      const int e0 = (r + 1)*L::EW + q + L::A;     // node in the E slot
      const T ex = sE[se][0][e0], ey = sE[se][1][e0], ez = sE[se][2][e0];
      const T cx = c3*(ey - sE[se][1][e0 - 1]) - c2*(ez - sE[se][2][e0 - L::EW]);
      const T cy = c1*(ez - sE[sp][2][e0]) - c3*(ex - sE[se][0][e0 - 1]);
      const T cz = c2*(ex - sE[se][0][e0 - L::EW]) - c1*(ey - sE[sp][1][e0]);
      const T hv[3] = {ho[0] + cx, ho[1] + cy, ho[2] + cz};
      const T hx = hv[0] + cx, hy = hv[1] + cy, hz = hv[2] + cz;
      const int hi = r*L::HW + q;
      sH[sh][0][hi] = hx;
      sH[sh][1][hi] = hy;
      sH[sh][2][hi] = hz;
      if (own) {
         const int j = jb + r, k = kb + q;
         const long o = g.at (p, j, k);
         Hnw.c[0][o] = hx;
         Hnw.c[1][o] = hy;
         Hnw.c[2][o] = hz;
         const T ev[3] = {ex, ey, ez};
         if (p >= 1 && p < nx && j >= 1 && j < ny && k >= 1 && k < nz) {
            // Inside every energy pick range.  The precision form sums a
            // node's three squares in FP32 (as its field passes do), one
            // conversion per sum.
            if (sizeof (T) == sizeof (float)) {
               float se = (float) ex*(float) ex, sb = (float) hv[0]*(float) hv[0];
               se += (float) ey*(float) ey;
               se += (float) ez*(float) ez;
               sb += (float) hv[1]*(float) hv[1];
               sb += (float) hv[2]*(float) hv[2];
               we += (double) se;
               wb += (double) sb;
            } else {
               we += (double) ex*(double) ex;
               we += (double) ey*(double) ey;
               we += (double) ez*(double) ez;
               wb += (double) hv[0]*(double) hv[0];
               wb += (double) hv[1]*(double) hv[1];
               wb += (double) hv[2]*(double) hv[2];
            }
         } else {
            energy_add (ep, p, j, k, ev, hv, we, wb);
         }
      }
   };

   // E slot of plane p: (p - i0 + 1) mod 4.  Groups of copies: planes
   // i0 - 1 and i0, then one group per plane; at the top of the step for
   // plane p the latest group is plane p + 1's.
   load_e (i0 - 1, 0);
   load_e (i0, 1);
   asm volatile ("cp.async.commit_group;" ::: "memory");
   if (i0 + 1 <= i1)
      load_e (i0 + 1, 2);
   asm volatile ("cp.async.commit_group;" ::: "memory");
   load_h (i0);
   for (int p = i0 ; p <= i1 ; ++p) {
      const int hs = (p - i0) & 1;                    // new-H slot of plane p
      const int u = p - i0 + 1, sp = (u - 1) & 3, se = u & 3;
      asm volatile ("cp.async.wait_group 1;" ::: "memory");
      __syncthreads ();
      if (p + 2 <= i1)
         load_e (p + 2, (u + 2) & 3);
      asm volatile ("cp.async.commit_group;" ::: "memory");
      const T ho0[3] = {h0[0], h0[1], h0[2]}, ho1[3] = {h1[0], h1[1], h1[2]};
      if (p < i1)
         load_h (p + 1);
      const bool ownp = p < i1 || lasti;
      if (need0)
         h_node (p, r0, q0, se, sp, hs, ho0, own0 && ownp);
      if (need1)
         h_node (p, r1, q1, se, sp, hs, ho1, own1 && ownp);
      __syncthreads ();
      if (p > i0 && p >= 2 && ownE) {
         // E^(n+1) of plane p - 1 (in [1, n - 1]) at the tile node.
         const int pe = (r0 + 1)*L::EW + q0 + L::A, ph = r0*L::HW + q0;
         const int hp = hs ^ 1;
         const T ex = sE[sp][0][pe], ey = sE[sp][1][pe], ez = sE[sp][2][pe];
         const T Hx = sH[hp][0][ph], Hy = sH[hp][1][ph], Hz = sH[hp][2][ph];
         const T Hy_z = sH[hp][1][ph + 1], Hx_z = sH[hp][0][ph + 1];
         const T Hz_y = sH[hp][2][ph + L::HW], Hx_y = sH[hp][0][ph + L::HW];
         const T Hz_x = sH[hs][2][ph], Hy_x = sH[hs][1][ph];
         const long o = g.at (p - 1, j0, k0);
         En.c[0][o] = ex - (d3*(Hy_z - Hy) - d2*(Hz_y - Hz));
         En.c[1][o] = ey - (d1*(Hz_x - Hz) - d3*(Hx_z - Hx));
         En.c[2][o] = ez - (d2*(Hx_y - Hx) - d1*(Hy_x - Hy));
      }
   }
   energy_flush (we, wb, dsc);
}

// The E update of the shell slabs: old E and the new (walled) H to the new E.
template <typename T>
__global__ void __launch_bounds__ (256)
k_shell_e (Grid g, F3T<T> E, F3T<T> En, F3T<T> Hnw, Slabs S, T d1, T d2, T d3)
{
   const long sx = g.sx, sy = g.sy;
   const T *Hx = Hnw.c[0], *Hy = Hnw.c[1], *Hz = Hnw.c[2];
   for (long t = blockIdx.x*(long) blockDim.x + threadIdx.x ; t < S.start[6] ; t += (long) gridDim.x*blockDim.x) {
      int i, j, k;
      slab_node (S, t, i, j, k);
      const long o = g.at (i, j, k);
      const T hx = Hx[o], hy = Hy[o], hz = Hz[o];
      En.c[0][o] = E.c[0][o] - (d3*(Hy[o + 1] - hy) - d2*(Hz[o + sy] - hz));
      En.c[1][o] = E.c[1][o] - (d1*(Hz[o + sx] - hz) - d3*(Hx[o + 1] - hx));
      En.c[2][o] = E.c[2][o] - (d2*(Hx[o + sy] - hx) - d1*(Hy[o + sx] - hy));
   }
}

// ---------------------------------------------------------------------------
// Precision form: the two bulk passes on float4 slots.  A row's node k sits
// at offset origin + i sx + j sy + k with origin = 1 (mod 4) and sx, sy
// multiples of 4, so the slots m = [4m - 1, 4m + 2] are 16-byte aligned;
// each thread takes one slot (four nodes) of a row, loads every stream of
// the stencil with one vector load (the k -/+ 1 neighbours of the slot's
// end nodes with one scalar load each), and stores whole slots inside the
// box (nodes outside it are computed from in-allocation ghosts and padding
// and not stored).  The arithmetic per node is that of the scalar kernels.
// ---------------------------------------------------------------------------
struct Slots {
   Box walk;                // (i, j, slot) over the box's rows
   int m0;                  // first slot of a row
   int klo, khi;            // the box's k range
};

static Slots make_slots (const Box &b)
{
   Slots s;
   s.klo = b.lo[2];
   s.khi = b.lo[2] + b.ext[2] - 1;
   s.m0 = (s.klo + 1) >> 2;
   const int m1 = (s.khi + 1) >> 2;
   s.walk = b;
   s.walk.lo[2] = 0;
   s.walk.ext[2] = m1 - s.m0 + 1;
   s.walk.vol = (long) b.ext[0]*b.ext[1]*s.walk.ext[2];
   return s;
}

__device__ __forceinline__ float4 ld4 (const float *p) { return *reinterpret_cast<const float4 *> (p); }
__device__ __forceinline__ void st4 (float *p, float4 v) { *reinterpret_cast<float4 *> (p) = v; }
__device__ __forceinline__ float el (const float4 &v, int e) { return e == 0 ? v.x : e == 1 ? v.y : e == 2 ? v.z : v.w; }

__device__ __forceinline__ void st_slot (float *p, const float r[4], int k0, int klo, int khi)
{
   if (k0 >= klo && k0 + 3 <= khi) {
      st4 (p, make_float4 (r[0], r[1], r[2], r[3]));
      return;
   }
#pragma unroll
   for (int e = 0 ; e < 4 ; ++e)
      if (k0 + e >= klo && k0 + e <= khi)
         p[e] = r[e];
}

template <bool HN>
__global__ void __launch_bounds__ (256)
k_h_fused4 (Grid g, F3T<float> E, F3T<float> H, F3T<float> Hn, Slots S, float c1, float c2, float c3,
            EnergyPick ep, DevScalars *dsc)
{
   __shared__ double sw[2][8];
   const float *Ex = E.c[0], *Ey = E.c[1], *Ez = E.c[2];
   const long sx = g.sx, sy = g.sy;
   const long stride = (long) gridDim.x*blockDim.x;
   double we = 0, wb = 0;
   BoxWalk wk;
   walk_init (wk, blockIdx.x*(long) blockDim.x + threadIdx.x, stride, S.walk);
   for (long t = blockIdx.x*(long) blockDim.x + threadIdx.x ; t < S.walk.vol ; t += stride) {
      const int i = S.walk.lo[0] + wk.i, j = S.walk.lo[1] + wk.j, k0 = 4*(S.m0 + wk.k) - 1;
      walk_step (wk, S.walk);
      const long o = g.at (i, j, k0);
      const float4 ex = ld4 (Ex + o), ey = ld4 (Ey + o), ez = ld4 (Ez + o);
      const float4 ezy = ld4 (Ez + o - sy), ezx = ld4 (Ez + o - sx);
      const float4 exy = ld4 (Ex + o - sy), eyx = ld4 (Ey + o - sx);
      const float4 h0 = ld4 (H.c[0] + o), h1 = ld4 (H.c[1] + o), h2 = ld4 (H.c[2] + o);
      const float eym = Ey[o - 1], exm = Ex[o - 1];
      float rx[4], ry[4], rz[4], nx[4], ny[4], nz[4];
      float se = 0.0f, sb = 0.0f;
#pragma unroll
      for (int e = 0 ; e < 4 ; ++e) {
         const float vex = el (ex, e), vey = el (ey, e), vez = el (ez, e);
         const float pey = e == 0 ? eym : el (ey, e - 1), pex = e == 0 ? exm : el (ex, e - 1);
         const float cx = c3*(vey - pey) - c2*(vez - el (ezy, e));
         const float cy = c1*(vez - el (ezx, e)) - c3*(vex - pex);
         const float cz = c2*(vex - el (exy, e)) - c1*(vey - el (eyx, e));
         const float hx = el (h0, e) + cx, hy = el (h1, e) + cy, hz = el (h2, e) + cz;
         nx[e] = hx;
         ny[e] = hy;
         nz[e] = hz;
         rx[e] = hx + cx;
         ry[e] = hy + cy;
         rz[e] = hz + cz;
         const int k = k0 + e;
         if (k < S.klo || k > S.khi)
            continue;
         const int I[3] = {i, j, k};
         const float ev[3] = {vex, vey, vez}, hv[3] = {hx, hy, hz};
#pragma unroll
         for (int c = 0 ; c < 3 ; ++c) {
            bool in_e = true, in_h = true;
#pragma unroll
            for (int a = 0 ; a < 3 ; ++a) {
               in_e &= (I[a] >= ep.lo[c][a]) & (I[a] <= ep.hi[c][a]);
               in_h &= (I[a] >= ep.hlo[c][a]) & (I[a] <= ep.hhi[c][a]);
            }
            if (in_e) se += ev[c]*ev[c];
            if (in_h) sb += hv[c]*hv[c];
         }
      }
      we += (double) se;
      wb += (double) sb;
      if (HN) {
         st_slot (Hn.c[0] + o, nx, k0, S.klo, S.khi);
         st_slot (Hn.c[1] + o, ny, k0, S.klo, S.khi);
         st_slot (Hn.c[2] + o, nz, k0, S.klo, S.khi);
      }
      st_slot (H.c[0] + o, rx, k0, S.klo, S.khi);
      st_slot (H.c[1] + o, ry, k0, S.klo, S.khi);
      st_slot (H.c[2] + o, rz, k0, S.klo, S.khi);
   }
   for (int d = 16 ; d > 0 ; d >>= 1) {
      we += __shfl_xor_sync (0xffffffffu, we, d);
      wb += __shfl_xor_sync (0xffffffffu, wb, d);
   }
   const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
   if (lane == 0) {
      sw[0][wid] = we;
      sw[1][wid] = wb;
   }
   __syncthreads ();
   if (wid == 0) {
      we = lane < (int) (blockDim.x >> 5) ? sw[0][lane] : 0;
      wb = lane < (int) (blockDim.x >> 5) ? sw[1][lane] : 0;
      for (int d = 16 ; d > 0 ; d >>= 1) {
         we += __shfl_xor_sync (0xffffffffu, we, d);
         wb += __shfl_xor_sync (0xffffffffu, wb, d);
      }
      if (lane == 0) {
         atomicAdd (&dsc->acc[0], we);
         atomicAdd (&dsc->acc[1], wb);
      }
   }
}

template <bool WJ>
__global__ void __launch_bounds__ (256)
k_e_fused4 (Grid g, F3T<float> E, F3T<float> H, F3T<float> J, Slots S, float c1, float c2, float c3, Rim rm)
{
   const float *Hx = H.c[0], *Hy = H.c[1], *Hz = H.c[2];
   const long sx = g.sx, sy = g.sy;
   const float tau = (float) g.tau;
   const long stride = (long) gridDim.x*blockDim.x;
   BoxWalk wk;
   walk_init (wk, blockIdx.x*(long) blockDim.x + threadIdx.x, stride, S.walk);
   for (long t = blockIdx.x*(long) blockDim.x + threadIdx.x ; t < S.walk.vol ; t += stride) {
      const int i = S.walk.lo[0] + wk.i, j = S.walk.lo[1] + wk.j, k0 = 4*(S.m0 + wk.k) - 1;
      walk_step (wk, S.walk);
      const long o = g.at (i, j, k0);
      const float4 hx = ld4 (Hx + o), hy = ld4 (Hy + o), hz = ld4 (Hz + o);
      const float4 hzy = ld4 (Hz + o + sy), hzx = ld4 (Hz + o + sx);
      const float4 hxy = ld4 (Hx + o + sy), hyx = ld4 (Hy + o + sx);
      const float hyp = Hy[o + 4], hxp = Hx[o + 4];
      const float4 e0 = ld4 (E.c[0] + o), e1 = ld4 (E.c[1] + o), e2 = ld4 (E.c[2] + o);
      float4 j0 = make_float4 (0, 0, 0, 0), j1 = j0, j2 = j0;
      if (WJ) {
         j0 = ld4 (J.c[0] + o);
         j1 = ld4 (J.c[1] + o);
         j2 = ld4 (J.c[2] + o);
      }
      float rx[4], ry[4], rz[4];
#pragma unroll
      for (int e = 0 ; e < 4 ; ++e) {
         const float vhx = el (hx, e), vhy = el (hy, e), vhz = el (hz, e);
         const float nhy = e == 3 ? hyp : el (hy, e + 1), nhx = e == 3 ? hxp : el (hx, e + 1);
         float ex = el (e0, e) - (c3*(nhy - vhy) - c2*(el (hzy, e) - vhz));
         float ey = el (e1, e) - (c1*(el (hzx, e) - vhz) - c3*(nhx - vhx));
         float ez = el (e2, e) - (c2*(el (hxy, e) - vhx) - c1*(el (hyx, e) - vhy));
         if (WJ && !rim_node (rm, i, j, k0 + e)) {
            ex -= tau*el (j0, e);
            ey -= tau*el (j1, e);
            ez -= tau*el (j2, e);
         }
         rx[e] = ex;
         ry[e] = ey;
         rz[e] = ez;
      }
      st_slot (E.c[0] + o, rx, k0, S.klo, S.khi);
      st_slot (E.c[1] + o, ry, k0, S.klo, S.khi);
      st_slot (E.c[2] + o, rz, k0, S.klo, S.khi);
   }
}

// ---------------------------------------------------------------------------
// Plain FP64 form: the H pass on double2 slots.  With four nodes in front
// of k = 0 the FP64 origin is a multiple of 4 elements, so the slots
// [2m, 2m + 1] are 16-byte aligned; the per-node arithmetic (compiled
// without contraction) is the scalar kernel's, so H and H^n are
// bit-identical to it.  The energy sums add the same squares, in slot order.
// ---------------------------------------------------------------------------
static Slots make_slots2 (const Box &b)
{
   Slots s;
   s.klo = b.lo[2];
   s.khi = b.lo[2] + b.ext[2] - 1;
   s.m0 = s.klo >> 1;
   const int m1 = s.khi >> 1;
   s.walk = b;
   s.walk.lo[2] = 0;
   s.walk.ext[2] = m1 - s.m0 + 1;
   s.walk.vol = (long) b.ext[0]*b.ext[1]*s.walk.ext[2];
   return s;
}

__device__ __forceinline__ double2 ld2 (const double *p) { return *reinterpret_cast<const double2 *> (p); }

__device__ __forceinline__ void st_slot2 (double *p, double a, double b, int k0, int klo, int khi)
{
   if (k0 >= klo && k0 + 1 <= khi) {
      *reinterpret_cast<double2 *> (p) = make_double2 (a, b);
      return;
   }
   if (k0 >= klo && k0 <= khi) p[0] = a;
   if (k0 + 1 >= klo && k0 + 1 <= khi) p[1] = b;
}

template <bool HN>
__global__ void __launch_bounds__ (256)
k_h_fused2 (Grid g, F3T<double> E, F3T<double> H, F3T<double> Hn, Slots S, double c1, double c2, double c3,
            EnergyPick ep, DevScalars *dsc)
{
   __shared__ double sw[2][8];
   const double *Ex = E.c[0], *Ey = E.c[1], *Ez = E.c[2];
   const long sx = g.sx, sy = g.sy;
   const long stride = (long) gridDim.x*blockDim.x;
   double we = 0, wb = 0;
   BoxWalk wk;
   walk_init (wk, blockIdx.x*(long) blockDim.x + threadIdx.x, stride, S.walk);
   for (long t = blockIdx.x*(long) blockDim.x + threadIdx.x ; t < S.walk.vol ; t += stride) {
      const int i = S.walk.lo[0] + wk.i, j = S.walk.lo[1] + wk.j, k0 = 2*(S.m0 + wk.k);
      walk_step (wk, S.walk);
      const long o = g.at (i, j, k0);
      const double2 ex = ld2 (Ex + o), ey = ld2 (Ey + o), ez = ld2 (Ez + o);
      const double2 ezy = ld2 (Ez + o - sy), ezx = ld2 (Ez + o - sx);
      const double2 exy = ld2 (Ex + o - sy), eyx = ld2 (Ey + o - sx);
      const double2 h0 = ld2 (H.c[0] + o), h1 = ld2 (H.c[1] + o), h2 = ld2 (H.c[2] + o);
      const double eym = Ey[o - 1], exm = Ex[o - 1];
      double rx[2], ry[2], rz[2], nx[2], ny[2], nz[2];
#pragma unroll
      for (int e = 0 ; e < 2 ; ++e) {
         const double vex = e ? ex.y : ex.x, vey = e ? ey.y : ey.x, vez = e ? ez.y : ez.x;
         const double pey = e ? ey.x : eym, pex = e ? ex.x : exm;
         const double cx = c3*(vey - pey) - c2*(vez - (e ? ezy.y : ezy.x));
         const double cy = c1*(vez - (e ? ezx.y : ezx.x)) - c3*(vex - pex);
         const double cz = c2*(vex - (e ? exy.y : exy.x)) - c1*(vey - (e ? eyx.y : eyx.x));
         const double hx = (e ? h0.y : h0.x) + cx, hy = (e ? h1.y : h1.x) + cy, hz = (e ? h2.y : h2.x) + cz;
         nx[e] = hx;
         ny[e] = hy;
         nz[e] = hz;
         rx[e] = hx + cx;
         ry[e] = hy + cy;
         rz[e] = hz + cz;
         const int k = k0 + e;
         if (k < S.klo || k > S.khi)
            continue;
         const int I[3] = {i, j, k};
         const double ev[3] = {vex, vey, vez}, hv[3] = {hx, hy, hz};
#pragma unroll
         for (int c = 0 ; c < 3 ; ++c) {
            bool in_e = true, in_h = true;
#pragma unroll
            for (int a = 0 ; a < 3 ; ++a) {
               in_e &= (I[a] >= ep.lo[c][a]) & (I[a] <= ep.hi[c][a]);
               in_h &= (I[a] >= ep.hlo[c][a]) & (I[a] <= ep.hhi[c][a]);
            }
            if (in_e) we += ev[c]*ev[c];
            if (in_h) wb += hv[c]*hv[c];
         }
      }
      if (HN) {
         st_slot2 (Hn.c[0] + o, nx[0], nx[1], k0, S.klo, S.khi);
         st_slot2 (Hn.c[1] + o, ny[0], ny[1], k0, S.klo, S.khi);
         st_slot2 (Hn.c[2] + o, nz[0], nz[1], k0, S.klo, S.khi);
      }
      st_slot2 (H.c[0] + o, rx[0], rx[1], k0, S.klo, S.khi);
      st_slot2 (H.c[1] + o, ry[0], ry[1], k0, S.klo, S.khi);
      st_slot2 (H.c[2] + o, rz[0], rz[1], k0, S.klo, S.khi);
   }
   for (int d = 16 ; d > 0 ; d >>= 1) {
      we += __shfl_xor_sync (0xffffffffu, we, d);
      wb += __shfl_xor_sync (0xffffffffu, wb, d);
   }
   const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
   if (lane == 0) {
      sw[0][wid] = we;
      sw[1][wid] = wb;
   }
   __syncthreads ();
   if (wid == 0) {
      we = lane < (int) (blockDim.x >> 5) ? sw[0][lane] : 0;
      wb = lane < (int) (blockDim.x >> 5) ? sw[1][lane] : 0;
      for (int d = 16 ; d > 0 ; d >>= 1) {
         we += __shfl_xor_sync (0xffffffffu, we, d);
         wb += __shfl_xor_sync (0xffffffffu, wb, d);
      }
      if (lane == 0) {
         atomicAdd (&dsc->acc[0], we);
         atomicAdd (&dsc->acc[1], wb);
      }
   }
}

// Wall kernels run over the two transverse axes, nodes [0, n+1] each (the
// flush extent of the reference's caps, core/em_caps.c:140-146).
struct Wall {
   int ea, ep, eq;
   int np_, nq_;           // extents n[ep]+2, n[eq]+2
   long s_a, s_p, s_q;     // strides along the three axes
};

// Transverse axes of a wall with the one of smallest stride as eq, the
// fastest thread index (z for the x and y walls, y for the z walls), so
// that a warp's nodes are contiguous in memory where they can be.  The
// wall operations treat the two tangential components alike.
static Wall make_wall (const Grid &g, int ea)
{
   Wall w;
   w.ea = ea;
   w.ep = ea == 0 ? 1 : 0;
   w.eq = ea == 2 ? 1 : 2;
   w.np_ = g.n[w.ep] + 2;
   w.nq_ = g.n[w.eq] + 2;
   const long s[3] = {g.sx, g.sy, 1};
   w.s_a = s[ea];
   w.s_p = s[w.ep];
   w.s_q = s[w.eq];
   return w;
}

__device__ __forceinline__ bool wall_node (const Grid &g, const Wall &w, int a,
                                           long &o, int &p, int &q)
{
   const long t = blockIdx.x*(long) blockDim.x + threadIdx.x;
   if (t >= (long) w.np_*w.nq_)
      return false;
   p = (int) (t / w.nq_);
   q = (int) (t % w.nq_);
   o = g.origin + a*w.s_a + p*w.s_p + q*w.s_q;
   return true;
}

enum { OP_PERIODIC = 0, OP_MIRROR_MIN, OP_MIRROR_MAX, OP_OPEN_MIN, OP_OPEN_MAX };

// Wall operations take their axis as a template argument: transverse axes,
// strides and extents are then compile-time picks among the kernel's
// parameters.  (Indexing a parameter array with a run-time axis makes the
// compiler copy the parameters to local memory, on the critical path of
// these latency-bound kernels.)
template <int AX> struct Axes {
   static constexpr int EP = AX == 0 ? 1 : 0, EQ = AX == 2 ? 1 : 2;
};

template <int AX>
__device__ __forceinline__ long axis_stride (const Grid &g) { return AX == 0 ? g.sx : AX == 1 ? g.sy : 1; }

// Host side: run the statement with the compile-time axis AX = ea.
#define MG_AXIS_SWITCH(ea, ...)                                               \
   switch (ea) {                                                              \
   case 0: { constexpr int AX = 0; __VA_ARGS__; } break;                      \
   case 1: { constexpr int AX = 1; __VA_ARGS__; } break;                      \
   default: { constexpr int AX = 2; __VA_ARGS__; } break;                     \
   }

// H wall operations (core/emCap_periodic.c:15-37, emCap_mirror.c:17-40,
// emCap_Mur.c:56-80).
template <typename T>
__global__ void k_h_wall (Grid g, F3T<T> H, Wall w, int op)
{
   long o;
   int p, q;
   const int N = g.n[w.ea];
   if (!wall_node (g, w, 0, o, p, q))
      return;
   T *Ha = H.c[w.ea], *Hp = H.c[w.ep], *Hq = H.c[w.eq];
   switch (op) {
   case OP_PERIODIC:
      for (int c = 0 ; c < 3 ; ++c) {
         H.c[c][o] = H.c[c][o + N*w.s_a];
         H.c[c][o + (N + 1)*w.s_a] = H.c[c][o + w.s_a];
      }
      break;
   case OP_MIRROR_MIN:
      Ha[o] = 0;
      Hp[o] = Hp[o + w.s_a];
      Hq[o] = Hq[o + w.s_a];
      break;
   case OP_MIRROR_MAX:
      o += N*w.s_a;
      Ha[o] = 0;
      Hp[o + w.s_a] = Hp[o];
      Hq[o + w.s_a] = Hq[o];
      break;
   case OP_OPEN_MIN:
      Hp[o] = Hp[o + w.s_a];
      Hq[o] = Hq[o + w.s_a];
      break;
   case OP_OPEN_MAX:
      o += N*w.s_a;
      Hp[o + w.s_a] = Hp[o];
      Hq[o + w.s_a] = Hq[o];
      break;
   }
}

// E wall operations (core/emCap_periodic.c:42-67, emCap_mirror.c:45-70,
// emCap_Mur.c:117-166).  The Mur history holds, per wall node, the wall and
// first inner tangential values of the previous step before E -= tau*J.
template <typename T>
__global__ void k_e_wall (Grid g, F3T<T> E, Wall w, int op, T *mur, T alpha)
{
   long o;
   int p, q;
   const int N = g.n[w.ea];
   if (!wall_node (g, w, 0, o, p, q))
      return;
   T *Ea = E.c[w.ea], *Ep = E.c[w.ep], *Eq = E.c[w.eq];
   switch (op) {
   case OP_PERIODIC:
      for (int c = 0 ; c < 3 ; ++c) {
         E.c[c][o + N*w.s_a] = E.c[c][o];
         E.c[c][o + (N + 1)*w.s_a] = E.c[c][o + w.s_a];
      }
      break;
   case OP_MIRROR_MIN:
      Ep[o] = 0;
      Eq[o] = 0;
      Ea[o] = Ea[o + w.s_a];
      break;
   case OP_MIRROR_MAX:
      o += N*w.s_a;
      Ep[o] = 0;
      Eq[o] = 0;
      Ea[o + w.s_a] = Ea[o];
      break;
   case OP_OPEN_MIN:
   case OP_OPEN_MAX: {
      const bool top = (op == OP_OPEN_MAX);
      if (top)
         o += N*w.s_a;
      const long in = top ? o - w.s_a : o + w.s_a;
      T *h = mur + 4*((long) p*w.nq_ + q);
      if (top)
         Ea[o + w.s_a] = Ea[o];
      else
         Ea[o] = Ea[o + w.s_a];
      const T ep = h[2] + alpha*(Ep[in] - h[0]);
      const T eq = h[3] + alpha*(Eq[in] - h[1]);
      Ep[o] = ep;
      Eq[o] = eq;
      h[0] = ep;
      h[1] = eq;
      h[2] = Ep[in];
      h[3] = Eq[in];
      break;
   }
   }
}

// Mur history from the loaded E and normal-E ghost copy (emCap_Mur.c:86-112).
template <typename T>
__global__ void k_mur_init (Grid g, F3T<T> E, Wall w, int top, T *mur)
{
   long o;
   int p, q;
   const int N = g.n[w.ea];
   if (!wall_node (g, w, 0, o, p, q))
      return;
   if (top)
      o += N*w.s_a;
   const long in = top ? o - w.s_a : o + w.s_a;
   T *h = mur + 4*((long) p*w.nq_ + q);
   h[0] = E.c[w.ep][o];
   h[1] = E.c[w.eq][o];
   h[2] = E.c[w.ep][in];
   h[3] = E.c[w.eq][in];
   if (top)
      E.c[w.ea][o + w.s_a] = E.c[w.ea][o];
   else
      E.c[w.ea][o] = E.c[w.ea][o + w.s_a];
}

// All wall operations of one axis in one launch: the lower wall, then the
// upper wall (they touch disjoint nodes for n >= 3).  H walls act on both
// H arrays (H at n and at n+1/2).
template <typename T, int AX>
__device__ __forceinline__ void h_line (const Grid &g, const F3T<T> &H, const F3T<T> &Hn, int op_min,
                                        int op_max, int both, long o)
{
   constexpr int EP = Axes<AX>::EP, EQ = Axes<AX>::EQ;
   const int N = g.n[AX];
   const long s = axis_stride<AX> (g);
   const long t = o + N*s;
   const int na = both ? 2 : 1;
   // Every load of both arrays first, then the stores: the wall nodes never
   // alias the sources, so this is the order of the operations on each node.
   if (op_min == OP_PERIODIC) {
      T top[2][3], one[2][3];
#pragma unroll
      for (int arr = 0 ; arr < 2 ; ++arr)
#pragma unroll
         for (int c = 0 ; c < 3 ; ++c)
            if (arr < na) {
               const T *F = arr ? Hn.c[c] : H.c[c];
               top[arr][c] = F[t];
               one[arr][c] = F[o + s];
            }
#pragma unroll
      for (int arr = 0 ; arr < 2 ; ++arr)
#pragma unroll
         for (int c = 0 ; c < 3 ; ++c)
            if (arr < na) {
               T *F = arr ? Hn.c[c] : H.c[c];
               F[o] = top[arr][c];
               F[o + (N + 1)*s] = one[arr][c];
            }
      return;
   }
   T p1[2], q1[2], pN[2], qN[2];
#pragma unroll
   for (int arr = 0 ; arr < 2 ; ++arr)
      if (arr < na) {
         const T *Hp = arr ? Hn.c[EP] : H.c[EP], *Hq = arr ? Hn.c[EQ] : H.c[EQ];
         p1[arr] = Hp[o + s];
         q1[arr] = Hq[o + s];
         pN[arr] = Hp[t];
         qN[arr] = Hq[t];
      }
#pragma unroll
   for (int arr = 0 ; arr < 2 ; ++arr)
      if (arr < na) {
         T *Ha = arr ? Hn.c[AX] : H.c[AX], *Hp = arr ? Hn.c[EP] : H.c[EP], *Hq = arr ? Hn.c[EQ] : H.c[EQ];
         Hp[o] = p1[arr];
         Hq[o] = q1[arr];
         if (op_min == OP_MIRROR_MIN)
            Ha[o] = 0;
         Hp[t + s] = pN[arr];
         Hq[t + s] = qN[arr];
         if (op_max == OP_MIRROR_MAX)
            Ha[t] = 0;
      }
}

template <typename T, int AX>
__global__ void k_h_walls (Grid g, F3T<T> H, F3T<T> Hn, Wall w, int op_min, int op_max, int both)
{
   long o;
   int p, q;
   if (!wall_node (g, w, 0, o, p, q))
      return;
   h_line<T, AX> (g, H, Hn, op_min, op_max, both, o);
}

template <typename T, int AX>
__device__ __forceinline__ void e_wall_op (const Grid &g, const F3T<T> &E, int op, long o, int p, int q,
                                           T *mur, T alpha)
{
   constexpr int EP = Axes<AX>::EP, EQ = Axes<AX>::EQ;
   const int N = g.n[AX];
   const long sa = axis_stride<AX> (g);
   const int nq_ = g.n[EQ] + 2;
   T *Ea = E.c[AX], *Ep = E.c[EP], *Eq = E.c[EQ];
   switch (op) {
   case OP_PERIODIC:
#pragma unroll
      for (int c = 0 ; c < 3 ; ++c) {
         E.c[c][o + N*sa] = E.c[c][o];
         E.c[c][o + (N + 1)*sa] = E.c[c][o + sa];
      }
      break;
   case OP_MIRROR_MIN:
      Ep[o] = 0;
      Eq[o] = 0;
      Ea[o] = Ea[o + sa];
      break;
   case OP_MIRROR_MAX:
      o += N*sa;
      Ep[o] = 0;
      Eq[o] = 0;
      Ea[o + sa] = Ea[o];
      break;
   case OP_OPEN_MIN:
   case OP_OPEN_MAX: {
      const bool top = (op == OP_OPEN_MAX);
      if (top)
         o += N*sa;
      const long in = top ? o - sa : o + sa;
      T *h = mur + 4*((long) p*nq_ + q);
      if (top)
         Ea[o + sa] = Ea[o];
      else
         Ea[o] = Ea[o + sa];
      const T ep = h[2] + alpha*(Ep[in] - h[0]);
      const T eq = h[3] + alpha*(Eq[in] - h[1]);
      Ep[o] = ep;
      Eq[o] = eq;
      h[0] = ep;
      h[1] = eq;
      h[2] = Ep[in];
      h[3] = Eq[in];
      break;
   }
   default:
      break;
   }
}

// E walls of one axis, then -tau J on the rim nodes of the wall lines this
// thread owns.  Rim nodes are those of [-1, n+1]^3 outside [2, n-2]^3; the
// z walls own every node with a rim z index, the y walls those with a rim y
// index and an inner z index, the x walls the rest.  After its own axis no
// later wall reads or writes such a node, so its -tau J comes after every
// wall operation on it, as in core/em.c:189-222.  Threads cover transverse
// indices [-1, n+1]; the wall operations act on [0, n+1].
template <typename T, int AX>
__global__ void k_e_walls (Grid g, F3T<T> E, F3T<T> J, Wall w, int op_min, int op_max, T *mur_min,
                           T *mur_max, T alpha, int sub_j)
{
   constexpr int EP = Axes<AX>::EP, EQ = Axes<AX>::EQ;
   const long t = blockIdx.x*(long) blockDim.x + threadIdx.x;
   const int np1 = w.np_ + 1, nq1 = w.nq_ + 1;          // [-1, n+1]
   if (t >= (long) np1*nq1)
      return;
   const int p = (int) (t / nq1) - 1, q = (int) (t % nq1) - 1;
   const long o = g.origin + p*w.s_p + q*w.s_q;
   if (p >= 0 && q >= 0) {
      e_wall_op<T, AX> (g, E, op_min, o, p, q, mur_min, alpha);
      e_wall_op<T, AX> (g, E, op_max, o, p, q, mur_max, alpha);
   }
   if (!sub_j)
      return;
   const int N = g.n[AX];
   const int Np = g.n[EP], Nq = g.n[EQ];
   const bool p_rim = p < 2 || p > Np - 2, q_rim = q < 2 || q > Nq - 2;
   bool own;
   if (AX == 2)
      own = true;
   else if (AX == 1)
      own = !q_rim;                 // eq = z
   else
      own = !p_rim && !q_rim;       // ep = y, eq = z
   if (!own)
      return;
   const T tau = (T) g.tau;
   const int vs[6] = {-1, 0, 1, N - 1, N, N + 1};
   T e[6][3], jv[6][3];
#pragma unroll
   for (int u = 0 ; u < 6 ; ++u) {
      const long x = o + vs[u]*axis_stride<AX> (g);
#pragma unroll
      for (int c = 0 ; c < 3 ; ++c) {
         e[u][c] = E.c[c][x];
         jv[u][c] = __ldg (J.c[c] + x);
      }
   }
#pragma unroll
   for (int u = 0 ; u < 6 ; ++u) {
      const long x = o + vs[u]*axis_stride<AX> (g);
#pragma unroll
      for (int c = 0 ; c < 3 ; ++c)
         E.c[c][x] = e[u][c] - tau*jv[u][c];
   }
}

// Current folding of one axis, lower wall then upper wall
// (plasma_currentWalls.c:27-121); transverse extent [-2, n+2].  The five
// nodes around a wall are loaded, folded in registers in the reference's
// order and stored back.
template <typename T>
__device__ __forceinline__ void j_fold_wall (T a[5], T pp[5], T qq[5], int top)
{
   // Index u = 2 + offset along the axis from the wall node (u = 0..4 for
   // offsets -2..2).  out = +1 at the upper wall, -1 at the lower wall;
   // internal/external pick the normal component's staggered neighbours.
   const int out = top ? 1 : -1;
   const int in_ = top ? 2 : 3, ex_ = top ? 3 : 2;          // wall + internal / external
   a[in_] -= a[ex_];
   pp[2 - out] += pp[2 + out];
   qq[2 - out] += qq[2 + out];
   a[in_ - out] -= a[ex_ + out];
   pp[2 - 2*out] += pp[2 + 2*out];
   qq[2 - 2*out] += qq[2 + 2*out];
   pp[2] = 0;
   qq[2] = 0;
   a[ex_] = a[in_];
   pp[2 + out] = -pp[2 - out];
   qq[2 + out] = -qq[2 - out];
   a[ex_ + out] = a[in_ - out];
   pp[2 + 2*out] = -pp[2 - 2*out];
   qq[2 + 2*out] = -qq[2 - 2*out];
}

template <typename T, int AX>
__device__ __forceinline__ void j_fold (const Grid &g, const F3T<T> &J, int top, int bc, long base)
{
   constexpr int EP = Axes<AX>::EP, EQ = Axes<AX>::EQ;
   const long st = axis_stride<AX> (g);
   if (bc == MG_BC_PERIODIC) {
      if (top)
         return;
      const long shift = (long) g.n[AX]*st;
      T lo[3][5], hi[3][5];
#pragma unroll
      for (int c = 0 ; c < 3 ; ++c)
#pragma unroll
         for (int u = 0 ; u < 5 ; ++u) {
            lo[c][u] = J.c[c][base + (u - 2)*st];
            hi[c][u] = J.c[c][base + (u - 2)*st + shift];
         }
#pragma unroll
      for (int c = 0 ; c < 3 ; ++c)
#pragma unroll
         for (int u = 0 ; u < 5 ; ++u) {
            const T v = hi[c][u] + lo[c][u];
            J.c[c][base + (u - 2)*st + shift] = v;
            J.c[c][base + (u - 2)*st] = v;
         }
      return;
   }
   const long o = base + (top ? g.n[AX] : 0)*st;
   T a[5], pp[5], qq[5];
#pragma unroll
   for (int u = 0 ; u < 5 ; ++u) {
      a[u] = J.c[AX][o + (u - 2)*st];
      pp[u] = J.c[EP][o + (u - 2)*st];
      qq[u] = J.c[EQ][o + (u - 2)*st];
   }
   if (top)
      j_fold_wall (a, pp, qq, 1);
   else
      j_fold_wall (a, pp, qq, 0);
#pragma unroll
   for (int u = 0 ; u < 5 ; ++u) {
      J.c[AX][o + (u - 2)*st] = a[u];
      J.c[EP][o + (u - 2)*st] = pp[u];
      J.c[EQ][o + (u - 2)*st] = qq[u];
   }
}

template <typename T, int AX>
__global__ void k_j_walls (Grid g, F3T<T> J)
{
   constexpr int EP = Axes<AX>::EP, EQ = Axes<AX>::EQ;
   const int np_ = g.n[EP] + 5, nq_ = g.n[EQ] + 5;
   const long t = blockIdx.x*(long) blockDim.x + threadIdx.x;
   if (t >= (long) np_*nq_)
      return;
   const int p = (int) (t / nq_) - 2, q = (int) (t % nq_) - 2;
   const long base = g.origin + p*axis_stride<EP> (g) + q*axis_stride<EQ> (g);
   j_fold<T, AX> (g, J, 0, g.bc[0][AX], base);
   j_fold<T, AX> (g, J, 1, g.bc[1][AX], base);
}



// E -= tau*J over [-1, n+1]^3 (core/em.c:167-184).
template <typename T>
__global__ void k_e_sub_j (Grid g, F3T<T> E, F3T<T> J, Box b)
{
   const T tau = (T) g.tau;
   for (long t = blockIdx.x*(long) blockDim.x + threadIdx.x ; t < b.vol ; t += (long) gridDim.x*blockDim.x) {
      int i, j, k;
      box_index (t, b.lo, b.ext, i, j, k);
      const long o = g.at (i, j, k);
      E.c[0][o] -= tau*J.c[0][o];
      E.c[1][o] -= tau*J.c[1][o];
      E.c[2][o] -= tau*J.c[2][o];
   }
}



// Laser soft source (one-sided injection of scpic/em_mirror.h:62-101 with an
// analytic paraxial Gaussian beam and sin^2 envelope).  The incident field
// is evaluated in FP64 from the device time.
__device__ double laser_ey (const mg_laser_t &l, double x, double y, double z,
                            double t, double ymid, double zmid)
{
   const double k = 2*M_PI, xr = M_PI*l.waist*l.waist;
   const double xi = x - l.x_focus;
   const double w = l.waist*sqrt (1 + (xi/xr)*(xi/xr));
   const double r2 = (y - ymid)*(y - ymid) + (z - zmid)*(z - zmid);
   const double tr = t - l.t_start - x;
   if (tr <= 0 || tr >= l.duration)
      return 0;
   const double s = sin (M_PI*tr/l.duration);
   const double env = s*s;
   const double phase = k*tr + atan (xi/xr) - k*r2*xi/(2*(xi*xi + xr*xr)) + l.phase;
   return 2*M_PI*l.a0*(l.waist/w)*exp (-r2/(w*w))*env*sin (phase);
}

// Hz[I] += (tau/h1) * Ey_inc(x = (I-1) h1, t = n tau)   (after the H step)
// Ey[I-1] += (tau/h1) * Hz_inc(x = (I-1/2) h1, t = (n+1/2) tau)
template <typename T>
__device__ __forceinline__ void laser_node (const Grid &g, T *F, const mg_laser_t &l, const DevScalars *dsc,
                                            int is_e, F3T<T> &E, const F3T<T> &J, int sub_j, long t)
{
   const int nj = g.n[1] - 2*l.margin + 1, nk = g.n[2] - 2*l.margin + 1;
   if (nj <= 0 || nk <= 0 || t >= (long) nj*nk)
      return;
   const int j = l.margin + (int) (t / nk), k = l.margin + (int) (t % nk);
   const double ymid = 0.5*g.n[1]*g.h[1], zmid = 0.5*g.n[2]*g.h[2];
   const double c1 = g.tau/g.h[0];
   const double time = dsc->time + (is_e ? 0.5*g.tau : 0.0);   // FP64 time and phase
   const double x = is_e ? (l.plane - 0.5)*g.h[0] : (l.plane - 1)*g.h[0];
   const int i = is_e ? l.plane - 1 : l.plane;
   const double v = laser_ey (l, x, (j - 0.5)*g.h[1], k*g.h[2], time, ymid, zmid);
   const long o = g.at (i, j, k);
   F[o] += (T) (c1*v);
   if (sub_j) {
      // These nodes skip -tau J in the fused E pass: it comes after the
      // source here (core/em.c:210-215 order).
      for (int c = 0 ; c < 3 ; ++c)
         E.c[c][o] -= (T) g.tau*J.c[c][o];
   }
}

template <typename T>
__global__ void k_laser (Grid g, T *F, mg_laser_t l, const DevScalars *dsc,
                         int is_e, F3T<T> E, F3T<T> J, int sub_j)
{
   laser_node (g, F, l, dsc, is_e, E, J, sub_j, blockIdx.x*(long) blockDim.x + threadIdx.x);
}

// Hard gauss-spot source (core/em_gaussSpot.c:129-156) at time t + tau:
// threads over (j, k) in [-1, n+1]^2 of the plane; FP64 profile.
template <typename T>
__global__ void k_gauss_spot (Grid g, T *Ey, T *Ez, GaussSpot s, const DevScalars *dsc)
{
   const int nj = g.n[1] + 3, nk = g.n[2] + 3;
   const long q = blockIdx.x*(long) blockDim.x + threadIdx.x;
   if (q >= (long) nj*nk)
      return;
   const int j = (int) (q/nk) - 1, k = (int) (q % nk) - 1;
   const double t = dsc->time + g.tau;
   double f = 1;
   if (t < s.front) {
      const double l = (t - s.front)/s.duration;
      f = exp (-l*l);
   }
   if (t > s.front + s.plateau) {
      const double l = (t - s.front - s.plateau)/s.duration;
      f = exp (-l*l);
   }
   const double dy_ = ((j - 0.5)*g.h[1] - s.y)/s.width, dy = (j*g.h[1] - s.y)/s.width;
   const double dz = (k*g.h[2] - s.z)/s.width, dz_ = ((k - 0.5)*g.h[2] - s.z)/s.width;
   const long o = g.at (s.i, j, k);
   Ey[o] = (T) (s.ey*sin (s.omega*t)*f*exp (-dy_*dy_ - dz*dz));
   Ez[o] = (T) (s.ez*cos (s.omega*t)*f*exp (-dy*dy - dz_*dz_));
}

// Focused-laser soft source of one mirror (add_source with add_mirror_H /
// add_mirror_E, scpic/em_mirror.c:667-717): the H plane i = 5 (backward
// n0 - 4) takes the E profile at t, the E plane i = 4 (backward n0 - 4) the
// H profile at t + tau/2, over j, k in [5, n - 5]:
//   Fy += a (z_cos cos p + z_sin sin p), Fz += a (y_cos cos p + y_sin sin p),
//   a = exp (-(2 t'/dt)^2) tau/h1, p = 2 pi t' + phi0, t' = t - T0 + delay,
// in FP64 whatever the field type.
template <typename T>
__global__ void k_mirror (Grid g, T *Fy, T *Fz, MirrorDev m, int is_e, const DevScalars *dsc)
{
   const int nk = g.n[2] - 9, nj = g.n[1] - 9;
   const int q = blockIdx.x*blockDim.x + threadIdx.x;
   if (q >= nj*nk)
      return;
   const int j = 5 + q/nk, k = 5 + q % nk;
   const double t = dsc->time + (is_e ? 0.5*g.tau : 0.0) - m.T0 + m.delay;
   const double x = 2*t/m.dt, ampl = exp (-(x*x));   // pow (x, 2) of the reference, exactly
   const double ph = 2*3.141592653589793238462643*t + m.phi0;
   const double cs = cos (ph), sn = sin (ph), A = ampl*g.tau/g.h[0];
   const int I = m.forward ? (is_e ? 4 : 5) : g.n[0] - 5 + 1;
   const double *w = (is_e ? m.H : m.E) + 4*(long) q;
   const long o = g.at (I, j, k);
   Fy[o] = (T) ((double) Fy[o] + A*(w[2]*cs + w[3]*sn));
   Fz[o] = (T) ((double) Fz[o] + A*(w[0]*cs + w[1]*sn));
}

// The field arrays of one precision form.
// ---------------------------------------------------------------------------
// All wall work of one field in one launch (the step graph's path).  A wall
// phase of axis a (the per-axis kernels above, run in the order x, y, z)
// reads and writes only nodes whose index along a lies in that axis' band
// {-2..2, N-2..N+2}.  The wall nodes split into regions that no two phases
// share work in:
//   face lines of axis a: both transverse indices outside their bands, so
//     phase a alone touches them (one thread per line);
//   edge slices of axes a < b at one index of the third axis outside its
//     band: the band_a x band_b nodes there, touched by phase a and then
//     phase b (one warp per slice, __syncwarp between the phases);
//   the corner band^3: phases x, y, z (one block, __syncthreads between).
// Each wall operation runs once, after the same operations on its inputs as
// with the per-axis kernels, so the results are bit-identical.  The E walls
// subtract tau J on the rim nodes of each region after its last phase (each
// rim node lies in exactly one region), and the analytic laser plane, which
// lies outside every band, is added by blocks of its own.
// ---------------------------------------------------------------------------
enum { WK_H = 0, WK_E = 1, WK_J = 2 };

struct WallPlan {
   Wall w[3];
   int  op0[3], op1[3];
   int  nface[3], bface[4];     // face lines per axis; first block per axis (bface[3]: first edge block)
   int  nslice[3], bslice[4];   // edge slices per third axis; first block (bslice[3]: the corner block)
   int  blaser, nlaser;         // laser blocks and nodes (0: none)
   int  lo, hi;                 // transverse extent of a line: [lo, n + hi]
};

template <typename T>
struct WallArgs {
   F3T<T> F, F2, J;             // H: H and Hn; E: E (and J); J: J
   T     *mur[2][3];
   T      alpha[3];
   int    flag;                 // H: also Hn; E: subtract tau J on the rim
   mg_laser_t l;
   const DevScalars *dsc;
};

__device__ __forceinline__ int band_at (int u, int N) { return u < 5 ? u - 2 : N - 7 + u; }

// The wall line of axis AX whose transverse indices (along Axes<AX>::EP
// and ::EQ) are p and q.
// Both E walls of a line and, with sub, -tau J on its six rim nodes
// (indices -1, 0, 1, N-1, N, N+1) as one chain: every value is loaded, the
// wall operations of the per-axis kernels act on registers in their order
// (lower wall, then upper wall: disjoint nodes), -tau J follows on the
// post-wall values, then every changed value is stored.
template <typename T, int AX>
__device__ __forceinline__ void e_line (const Grid &g, WallArgs<T> &A, const WallPlan &P, int p, int q,
                                        bool sub)
{
   constexpr int EP = Axes<AX>::EP, EQ = Axes<AX>::EQ;
   const int N = g.n[AX];
   const long sa = axis_stride<AX> (g);
   const long o = g.origin + p*axis_stride<EP> (g) + q*axis_stride<EQ> (g);
   const int op0 = P.op0[AX], op1 = P.op1[AX];
   const int vs[6] = {-1, 0, 1, N - 1, N, N + 1};
   T e[6][3], jv[6][3];
   bool chg[6][3];
#pragma unroll
   for (int u = 0 ; u < 6 ; ++u)
#pragma unroll
      for (int c = 0 ; c < 3 ; ++c) {
         e[u][c] = A.F.c[c][o + vs[u]*sa];
         chg[u][c] = sub;
         if (sub)
            jv[u][c] = __ldg (A.J.c[c] + o + vs[u]*sa);
      }
   const long hq = 4*((long) p*(g.n[EQ] + 2) + q);
   T *h0 = op0 == OP_OPEN_MIN ? A.mur[0][AX] + hq : nullptr;
   T *h1 = op1 == OP_OPEN_MAX ? A.mur[1][AX] + hq : nullptr;
   T hm[4], hM[4];
   if (op0 == OP_OPEN_MIN)
#pragma unroll
      for (int x = 0 ; x < 4 ; ++x) hm[x] = h0[x];
   if (op1 == OP_OPEN_MAX)
#pragma unroll
      for (int x = 0 ; x < 4 ; ++x) hM[x] = h1[x];
   const T alpha = A.alpha[AX];
   // Lower wall: index 0 is row 1, index 1 row 2.
   if (op0 == OP_PERIODIC) {
#pragma unroll
      for (int c = 0 ; c < 3 ; ++c) {
         e[4][c] = e[1][c];
         e[5][c] = e[2][c];
         chg[4][c] = chg[5][c] = true;
      }
   } else if (op0 == OP_MIRROR_MIN) {
      e[1][EP] = 0;
      e[1][EQ] = 0;
      e[1][AX] = e[2][AX];
      chg[1][EP] = chg[1][EQ] = chg[1][AX] = true;
   } else if (op0 == OP_OPEN_MIN) {
      e[1][AX] = e[2][AX];
      const T ep = hm[2] + alpha*(e[2][EP] - hm[0]);
      const T eq = hm[3] + alpha*(e[2][EQ] - hm[1]);
      e[1][EP] = ep;
      e[1][EQ] = eq;
      hm[0] = ep;
      hm[1] = eq;
      hm[2] = e[2][EP];
      hm[3] = e[2][EQ];
      chg[1][EP] = chg[1][EQ] = chg[1][AX] = true;
   }
   // Upper wall: index N-1 is row 3, N row 4, N+1 row 5.
   if (op1 == OP_MIRROR_MAX) {
      e[4][EP] = 0;
      e[4][EQ] = 0;
      e[5][AX] = e[4][AX];
      chg[4][EP] = chg[4][EQ] = chg[5][AX] = true;
   } else if (op1 == OP_OPEN_MAX) {
      e[5][AX] = e[4][AX];
      const T ep = hM[2] + alpha*(e[3][EP] - hM[0]);
      const T eq = hM[3] + alpha*(e[3][EQ] - hM[1]);
      e[4][EP] = ep;
      e[4][EQ] = eq;
      hM[0] = ep;
      hM[1] = eq;
      hM[2] = e[3][EP];
      hM[3] = e[3][EQ];
      chg[4][EP] = chg[4][EQ] = chg[5][AX] = true;
   }
   if (sub) {
      const T tau = (T) g.tau;
#pragma unroll
      for (int u = 0 ; u < 6 ; ++u)
#pragma unroll
         for (int c = 0 ; c < 3 ; ++c)
            e[u][c] = e[u][c] - tau*jv[u][c];
   }
#pragma unroll
   for (int u = 0 ; u < 6 ; ++u)
#pragma unroll
      for (int c = 0 ; c < 3 ; ++c)
         if (chg[u][c])
            A.F.c[c][o + vs[u]*sa] = e[u][c];
   if (op0 == OP_OPEN_MIN)
#pragma unroll
      for (int x = 0 ; x < 4 ; ++x) h0[x] = hm[x];
   if (op1 == OP_OPEN_MAX)
#pragma unroll
      for (int x = 0 ; x < 4 ; ++x) h1[x] = hM[x];
}

// Both current walls of a line (plasma_currentWalls.c:27-121) as one chain:
// the five nodes around each wall are loaded, folded in registers, stored.
template <typename T, int AX>
__device__ __forceinline__ void j_line (const Grid &g, const F3T<T> &J, long base)
{
   constexpr int EP = Axes<AX>::EP, EQ = Axes<AX>::EQ;
   if (g.bc[0][AX] == MG_BC_PERIODIC) {
      j_fold<T, AX> (g, J, 0, MG_BC_PERIODIC, base);
      return;
   }
   const long st = axis_stride<AX> (g);
   const long o0 = base, o1 = base + g.n[AX]*st;
   T a0[5], p0[5], q0[5], a1[5], p1[5], q1[5];
#pragma unroll
   for (int u = 0 ; u < 5 ; ++u) {
      a0[u] = J.c[AX][o0 + (u - 2)*st];
      p0[u] = J.c[EP][o0 + (u - 2)*st];
      q0[u] = J.c[EQ][o0 + (u - 2)*st];
      a1[u] = J.c[AX][o1 + (u - 2)*st];
      p1[u] = J.c[EP][o1 + (u - 2)*st];
      q1[u] = J.c[EQ][o1 + (u - 2)*st];
   }
   j_fold_wall (a0, p0, q0, 0);
   j_fold_wall (a1, p1, q1, 1);
#pragma unroll
   for (int u = 0 ; u < 5 ; ++u) {
      J.c[AX][o0 + (u - 2)*st] = a0[u];
      J.c[EP][o0 + (u - 2)*st] = p0[u];
      J.c[EQ][o0 + (u - 2)*st] = q0[u];
      J.c[AX][o1 + (u - 2)*st] = a1[u];
      J.c[EP][o1 + (u - 2)*st] = p1[u];
      J.c[EQ][o1 + (u - 2)*st] = q1[u];
   }
}

// The wall line of axis AX whose transverse indices (along Axes<AX>::EP
// and ::EQ) are p and q; the E lines' rim nodes are left to the caller.
template <typename T, int KIND, int AX>
__device__ __forceinline__ void wall_line (const Grid &g, WallArgs<T> &A, const WallPlan &P, int p, int q)
{
   constexpr int EP = Axes<AX>::EP, EQ = Axes<AX>::EQ;
   if (p < P.lo || p > g.n[EP] + P.hi || q < P.lo || q > g.n[EQ] + P.hi)
      return;
   const long o = g.origin + p*axis_stride<EP> (g) + q*axis_stride<EQ> (g);
   if (KIND == WK_H)
      h_line<T, AX> (g, A.F, A.F2, P.op0[AX], P.op1[AX], A.flag, o);
   else if (KIND == WK_E) {
      if (p >= 0 && q >= 0)
         e_line<T, AX> (g, A, P, p, q, false);
   } else
      j_line<T, AX> (g, A.J, o);
}

__device__ __forceinline__ bool rim_index (int v, int N) { return v < 2 || v > N - 2; }

// E -= tau J at up to four rim nodes of a thread (offsets x[u], -1 for
// none), all loads before the stores (the order of core/em.c:189-222:
// after every wall operation on the node).
template <typename T>
__device__ __forceinline__ void rim_sub_j4 (const Grid &g, WallArgs<T> &A, const long x[4])
{
   const T tau = (T) g.tau;
   T e[4][3], jv[4][3];
#pragma unroll
   for (int u = 0 ; u < 4 ; ++u)
      if (x[u] >= 0)
#pragma unroll
         for (int c = 0 ; c < 3 ; ++c) {
            e[u][c] = A.F.c[c][x[u]];
            jv[u][c] = __ldg (A.J.c[c] + x[u]);
         }
#pragma unroll
   for (int u = 0 ; u < 4 ; ++u)
      if (x[u] >= 0)
#pragma unroll
         for (int c = 0 ; c < 3 ; ++c)
            A.F.c[c][x[u]] = e[u][c] - tau*jv[u][c];
}

template <typename T, int KIND, int AX>
__device__ __forceinline__ void face_line (const Grid &g, WallArgs<T> &A, const WallPlan &P, long t)
{
   constexpr int EQ = Axes<AX>::EQ;
   if (t >= P.nface[AX])
      return;
   const int nq = g.n[EQ] - 5;
   const int p = 3 + (int) (t / nq), q = 3 + (int) (t % nq);
   if (KIND == WK_E)
      e_line<T, AX> (g, A, P, p, q, A.flag != 0);    // face lines own their six rim nodes
   else
      wall_line<T, KIND, AX> (g, A, P, p, q);
}

// Edge slice at index tc of axis C: phases of the two other axes, lower
// index first, on their lines through band x band.
template <typename T, int KIND, int C>
__device__ __forceinline__ void edge_slice (const Grid &g, WallArgs<T> &A, const WallPlan &P, int s, int lane)
{
   constexpr int AA = C == 0 ? 1 : 0, BB = C == 2 ? 1 : 2;     // AA < BB, both != C
   if (s >= P.nslice[C])
      return;                                   // whole warps leave together
   const int tc = 3 + s;
   if (lane < 10) {
      const int tb = band_at (lane, g.n[BB]);
      // Axis AA's lines: transverse axes {BB, C} in its (EP, EQ) order.
      if (Axes<AA>::EP == BB)
         wall_line<T, KIND, AA> (g, A, P, tb, tc);
      else
         wall_line<T, KIND, AA> (g, A, P, tc, tb);
   }
   __syncwarp ();
   if (lane < 10) {
      const int ta = band_at (lane, g.n[AA]);
      if (Axes<BB>::EP == AA)
         wall_line<T, KIND, BB> (g, A, P, ta, tc);
      else
         wall_line<T, KIND, BB> (g, A, P, tc, ta);
   }
   __syncwarp ();
   if (KIND == WK_E && A.flag) {
      long x[4];
#pragma unroll
      for (int r = 0 ; r < 4 ; ++r) {
         const int u = lane + 32*r;
         x[r] = -1;
         if (u >= 100)
            continue;
         const int va = band_at (u / 10, g.n[AA]), vb = band_at (u % 10, g.n[BB]);
         if (va < -1 || va > g.n[AA] + 1 || vb < -1 || vb > g.n[BB] + 1)
            continue;
         if (!rim_index (va, g.n[AA]) && !rim_index (vb, g.n[BB]))
            continue;
         const int i = AA == 0 ? va : C == 0 ? tc : vb;
         const int j = AA == 1 ? va : BB == 1 ? vb : tc;
         const int k = BB == 2 ? vb : tc;
         x[r] = g.at (i, j, k);
      }
      rim_sub_j4 (g, A, x);
   }
}

template <typename T, int KIND, int AX>
__device__ __forceinline__ void corner_phase (const Grid &g, WallArgs<T> &A, const WallPlan &P)
{
   constexpr int EP = Axes<AX>::EP, EQ = Axes<AX>::EQ;
   for (int u = threadIdx.x ; u < 100 ; u += blockDim.x)
      wall_line<T, KIND, AX> (g, A, P, band_at (u / 10, g.n[EP]), band_at (u % 10, g.n[EQ]));
   __syncthreads ();
}

template <typename T, int KIND>
__global__ void __launch_bounds__ (256)
k_walls_all (Grid g, WallArgs<T> A, WallPlan P)
{
   const int b = blockIdx.x;
   if (b < P.bface[3]) {
      if (b >= P.bface[2])
         face_line<T, KIND, 2> (g, A, P, (long) (b - P.bface[2])*blockDim.x + threadIdx.x);
      else if (b >= P.bface[1])
         face_line<T, KIND, 1> (g, A, P, (long) (b - P.bface[1])*blockDim.x + threadIdx.x);
      else
         face_line<T, KIND, 0> (g, A, P, (long) (b - P.bface[0])*blockDim.x + threadIdx.x);
      return;
   }
   if (b < P.bslice[3]) {
      const int w = (int) (threadIdx.x >> 5), lane = threadIdx.x & 31, nw = (int) (blockDim.x >> 5);
      if (b >= P.bslice[2])
         edge_slice<T, KIND, 2> (g, A, P, (b - P.bslice[2])*nw + w, lane);
      else if (b >= P.bslice[1])
         edge_slice<T, KIND, 1> (g, A, P, (b - P.bslice[1])*nw + w, lane);
      else
         edge_slice<T, KIND, 0> (g, A, P, (b - P.bslice[0])*nw + w, lane);
      return;
   }
   if (b == P.bslice[3]) {
      corner_phase<T, KIND, 0> (g, A, P);
      corner_phase<T, KIND, 1> (g, A, P);
      corner_phase<T, KIND, 2> (g, A, P);
      if (KIND == WK_E && A.flag)
         for (int u0 = threadIdx.x ; u0 < 1000 ; u0 += 4*blockDim.x) {
            long x[4];
#pragma unroll
            for (int r = 0 ; r < 4 ; ++r) {
               const int u = u0 + r*blockDim.x;
               x[r] = -1;
               if (u >= 1000)
                  continue;
               const int v0 = band_at (u / 100, g.n[0]), v1 = band_at ((u / 10) % 10, g.n[1]);
               const int v2 = band_at (u % 10, g.n[2]);
               if (v0 < -1 || v0 > g.n[0] + 1 || v1 < -1 || v1 > g.n[1] + 1 || v2 < -1 || v2 > g.n[2] + 1)
                  continue;
               if (!rim_index (v0, g.n[0]) && !rim_index (v1, g.n[1]) && !rim_index (v2, g.n[2]))
                  continue;
               x[r] = g.at (v0, v1, v2);
            }
            rim_sub_j4 (g, A, x);
         }
      return;
   }
   if (KIND != WK_J && P.nlaser > 0) {
      const long t = (long) (b - P.blaser)*blockDim.x + threadIdx.x;
      if (KIND == WK_H)
         laser_node (g, A.F.c[2], A.l, A.dsc, 0, A.F, A.J, 0, t);
      else
         laser_node (g, A.F.c[1], A.l, A.dsc, 1, A.F, A.J, A.flag, t);
   }
}

template <typename T>
struct FS {
   T *E[3], *H[3], *Hn[3], *J[3];
   T *mur[2][3];
};

template <typename T>
static F3T<T> f3 (T *const c[3])
{
   F3T<T> f;
   for (int a = 0 ; a < 3 ; ++a)
      f.c[a] = c[a];
   return f;
}

static int wall_ops (const Grid &g, int ea, int &op_min, int &op_max)
{
   const int b0 = g.bc[0][ea], b1 = g.bc[1][ea];
   if (b0 == MG_BC_PERIODIC) {
      op_min = OP_PERIODIC;
      op_max = -1;
      return 0;
   }
   op_min = (b0 == MG_BC_MIRROR) ? OP_MIRROR_MIN : OP_OPEN_MIN;
   op_max = (b1 == MG_BC_MIRROR) ? OP_MIRROR_MAX : OP_OPEN_MAX;
   return 0;
}

template <typename T>
static int launch_h_walls (mg_run_t *r, const FS<T> &fs, int both)
{
   const Grid &g = r->g;
   for (int ea = 0 ; ea < 3 ; ++ea) {
      Wall w = make_wall (g, ea);
      const long nodes = (long) w.np_*w.nq_;
      const int NT = 256, B = (int) ((nodes + NT - 1)/NT);
      int op0, op1;
      wall_ops (g, ea, op0, op1);
      MG_AXIS_SWITCH (ea, k_h_walls<T, AX><<<B, NT, 0, r->stream>>> (g, f3 (fs.H), f3 (fs.Hn), w, op0, op1, both));
      MG_LAUNCH_CHECK ();
   }
   return MG_OK;
}

template <typename T>
static int launch_hn_walls (mg_run_t *r, const FS<T> &fs)
{
   const Grid &g = r->g;
   for (int ea = 0 ; ea < 3 ; ++ea) {
      Wall w = make_wall (g, ea);
      const long nodes = (long) w.np_*w.nq_;
      const int NT = 256, B = (int) ((nodes + NT - 1)/NT);
      int op0, op1;
      wall_ops (g, ea, op0, op1);
      MG_AXIS_SWITCH (ea, k_h_walls<T, AX><<<B, NT, 0, r->stream>>> (g, f3 (fs.Hn), f3 (fs.Hn), w, op0, op1, 0));
      MG_LAUNCH_CHECK ();
   }
   return MG_OK;
}

// E walls of all axes; with sub_j the rim nodes also get their -tau J.
template <typename T>
static int launch_e_walls (mg_run_t *r, const FS<T> &fs, int sub_j)
{
   const Grid &g = r->g;
   for (int ea = 0 ; ea < 3 ; ++ea) {
      Wall w = make_wall (g, ea);
      const long nodes = (long) (w.np_ + 1)*(w.nq_ + 1);
      const int NT = 128, B = (int) ((nodes + NT - 1)/NT);
      const T alpha = (T) ((g.tau - g.h[ea])/(g.tau + g.h[ea]));
      int op0, op1;
      wall_ops (g, ea, op0, op1);
      MG_AXIS_SWITCH (ea, k_e_walls<T, AX><<<B, NT, 0, r->stream>>> (g, f3 (fs.E), f3 (fs.J), w, op0, op1, fs.mur[0][ea],
                                         fs.mur[1][ea], alpha, sub_j));
      MG_LAUNCH_CHECK ();
   }
   return MG_OK;
}

template <typename T>
static int launch_mirrors (mg_run_t *r, const FS<T> &fs, int is_e)
{
   const long nodes = (long) (r->g.n[1] - 9)*(r->g.n[2] - 9);
   const int NT = 256, B = (int) ((nodes + NT - 1)/NT);
   for (int q = 0 ; q < r->nmirrors ; ++q) {
      k_mirror<T><<<B, NT, 0, r->stream>>> (r->g, is_e ? fs.E[1] : fs.H[1], is_e ? fs.E[2] : fs.H[2],
                                            r->mirrors[q], is_e, r->dsc);
      MG_LAUNCH_CHECK ();
   }
   return MG_OK;
}

template <typename T>
static int launch_laser (mg_run_t *r, const FS<T> &fs, int is_e, int sub_j = 0)
{
   if (!r->has_laser)
      return MG_OK;
   const mg_laser_t &l = r->laser;
   const long nj = r->g.n[1] - 2*l.margin + 1, nk = r->g.n[2] - 2*l.margin + 1;
   if (nj <= 0 || nk <= 0)
      return MG_OK;
   const int NT = 256, B = (int) ((nj*nk + NT - 1)/NT);
   k_laser<<<B, NT, 0, r->stream>>> (r->g, is_e ? fs.E[1] : fs.H[2], l, r->dsc, is_e,
                                    f3 (fs.E), f3 (fs.J), sub_j);
   MG_LAUNCH_CHECK ();
   return MG_OK;
}

// The merged wall launch needs the two bands of every axis apart (n >= 6;
// a run has at least 8 cells per axis, so this holds for every run).
// A run stepped as one branch of a batch graph keeps the per-axis kernels:
// there the other runs' kernels fill the launch gaps, and the merged
// kernel's serial corner block (three phases, then the rim) lengthens each
// run's chain (served scan of 24 solves on one box: 7.6 s per-axis against
// 8.1-8.9 s merged; one run stepped alone: merged 2 % faster on the
// laser-foil step, 8 % on the served solves run one at a time).
static bool walls_merge (const mg_run_t *r)
{
   return !r->in_batch && r->g.n[0] >= 6 && r->g.n[1] >= 6 && r->g.n[2] >= 6;
}

// The analytic laser's planes (H at x index `plane`, E at `plane` - 1, over
// j, k in [margin, n - margin]) outside every wall band: they commute with
// the walls and join the merged launch.
static bool laser_merge (const mg_run_t *r)
{
   if (!r->has_laser)
      return false;
   const mg_laser_t &l = r->laser;
   return l.margin >= 3 && l.plane >= 4 && l.plane <= r->g.n[0] - 3 &&
          r->g.n[1] - 2*l.margin + 1 > 0 && r->g.n[2] - 2*l.margin + 1 > 0;
}

// One launch of k_walls_all for the field of KIND; flag: H also walls Hn,
// E subtracts tau J on the rim; laser: the H (KIND = WK_H) or E source too.
template <typename T, int KIND>
static int launch_walls_all (mg_run_t *r, const FS<T> &fs, int flag, bool laser)
{
   const Grid &g = r->g;
   const int NT = 256;
   WallPlan P;
   int blocks = 0;
   for (int a = 0 ; a < 3 ; ++a) {
      P.w[a] = make_wall (g, a);
      wall_ops (g, a, P.op0[a], P.op1[a]);
      P.nface[a] = (g.n[P.w[a].ep] - 5)*(g.n[P.w[a].eq] - 5);
      P.bface[a] = blocks;
      blocks += (P.nface[a] + NT - 1)/NT;
   }
   P.bface[3] = blocks;
   for (int c = 0 ; c < 3 ; ++c) {
      P.nslice[c] = g.n[c] - 5;
      P.bslice[c] = blocks;
      blocks += (P.nslice[c] + NT/32 - 1)/(NT/32);
   }
   P.bslice[3] = blocks++;
   P.blaser = blocks;
   P.nlaser = 0;
   if (laser && KIND != WK_J) {
      const mg_laser_t &l = r->laser;
      P.nlaser = (g.n[1] - 2*l.margin + 1)*(g.n[2] - 2*l.margin + 1);
      blocks += (P.nlaser + NT - 1)/NT;
   }
   P.lo = KIND == WK_H ? 0 : KIND == WK_E ? -1 : -2;
   P.hi = KIND == WK_J ? 2 : 1;
   WallArgs<T> A;
   memset (&A, 0, sizeof (A));
   if (KIND == WK_H) {
      A.F = f3 (fs.H);
      A.F2 = f3 (fs.Hn);
   } else {
      A.F = f3 (fs.E);
      A.F2 = f3 (fs.E);
   }
   A.J = f3 (fs.J);
   for (int a = 0 ; a < 3 ; ++a) {
      A.mur[0][a] = fs.mur[0][a];
      A.mur[1][a] = fs.mur[1][a];
      A.alpha[a] = (T) ((g.tau - g.h[a])/(g.tau + g.h[a]));
   }
   A.flag = flag;
   if (r->has_laser)
      A.l = r->laser;
   A.dsc = r->dsc;
   k_walls_all<T, KIND><<<blocks, NT, 0, r->stream>>> (g, A, P);
   MG_LAUNCH_CHECK ();
   return MG_OK;
}

static Box h_box (const Grid &g)
{
   int lo[3], hi[3];
   for (int a = 0 ; a < 3 ; ++a) {
      lo[a] = (g.bc[0][a] == MG_BC_MIRROR) ? 1 : 0;
      hi[a] = g.n[a];
   }
   return make_box (lo, hi);
}

static Box e_box (const Grid &g)
{
   int lo[3], hi[3];
   for (int a = 0 ; a < 3 ; ++a) {
      lo[a] = (g.bc[0][a] == MG_BC_PERIODIC) ? 0 : 1;
      hi[a] = (g.bc[1][a] == MG_BC_PERIODIC) ? g.n[a] - 1 : g.n[a];
   }
   return make_box (lo, hi);
}

// Pick ranges of em_energy (core/em.c:241-247): component c sums nodes with
// index in [1, n] on its own axis and [0, n-1] on the others (E), and
// [0, n-1] on its own axis and [1, n] on the others (H).  On a periodic axis
// the H value at node 0 is the copy of node n, so node n stands in for it.
static EnergyPick energy_pick (const Grid &g)
{
   EnergyPick ep;
   for (int c = 0 ; c < 3 ; ++c)
      for (int a = 0 ; a < 3 ; ++a) {
         const int N = g.n[a];
         if (a == c) {
            ep.lo[c][a] = 1; ep.hi[c][a] = N;
            const bool per = (g.bc[0][a] == MG_BC_PERIODIC);
            ep.hlo[c][a] = per ? 1 : 0;
            ep.hhi[c][a] = per ? N : N - 1;
         } else {
            ep.lo[c][a] = 0; ep.hi[c][a] = N - 1;
            ep.hlo[c][a] = 1; ep.hhi[c][a] = N;
         }
      }
   return ep;
}

static Rim rim (const mg_run_t *r)
{
   Rim rm;
   for (int a = 0 ; a < 3 ; ++a) {
      rm.lo[a] = 2;
      rm.hi[a] = r->g.n[a] - 2;
   }
   rm.laser_i = r->has_laser ? r->laser.plane - 1 : INT_MIN;
   const int margin = r->has_laser ? r->laser.margin : 0;
   rm.laser_lo[0] = margin;
   rm.laser_hi[0] = r->g.n[1] - margin;
   rm.laser_lo[1] = margin;
   rm.laser_hi[1] = r->g.n[2] - margin;
   return rm;
}



// H^(n-1/2) -> H^n (kept in Hn) and on to H^(n+1/2) (kept in H), with the
// field energy at t = n tau summed on the way; walls on Hn.
template <typename T>
int fields_h_half (mg_run_t *r, const FS<T> &fs)
{
   const Grid &g = r->g;
   Box b = h_box (g);
   const int NT = 256;
   MG_CUDA (cudaMemsetAsync (r->dsc->acc, 0, 2*sizeof (double), r->stream));
   k_h_fused<<<mg_blocks_for (b.vol, NT, 8), NT, 0, r->stream>>> (
      g, f3 (fs.E), f3 (fs.H), f3 (fs.Hn), b, (T) (0.5*g.tau/g.h[0]), (T) (0.5*g.tau/g.h[1]), (T) (0.5*g.tau/g.h[2]),
      energy_pick (g), r->dsc);
   MG_LAUNCH_CHECK ();
   return launch_hn_walls<T> (r, fs);
}

template <typename T>
int fields_energy (mg_run_t *r, const FS<T> &fs)
{
   (void) r;                      // summed by mg_fields64_h_half
   return MG_OK;
}

// Source at t = n tau on H^(n+1/2), then its walls (core/em.c:115-131).
template <typename T>
int fields_h_step (mg_run_t *r, const FS<T> &fs)
{
   TRY_MG (mg_tfsf_h (r));
   TRY_MG (launch_mirrors<T> (r, fs, 0));
   TRY_MG (launch_laser<T> (r, fs, 0));
   const Grid &g = r->g;
   for (int ea = 0 ; ea < 3 ; ++ea) {
      Wall w = make_wall (g, ea);
      const long nodes = (long) w.np_*w.nq_;
      const int NT = 256, B = (int) ((nodes + NT - 1)/NT);
      int op0, op1;
      wall_ops (g, ea, op0, op1);
      MG_AXIS_SWITCH (ea, k_h_walls<T, AX><<<B, NT, 0, r->stream>>> (g, f3 (fs.H), f3 (fs.H), w, op0, op1, 0));
      MG_LAUNCH_CHECK ();
   }
   return MG_OK;
}

// Graph path: both half steps, the source on H^(n+1/2), walls on both.
// H^n is kept only where something reads it: the push (markers) or the
// probes; a field-only run moves E and H once each per half-update.
template <typename T>
int fields_h_both (mg_run_t *r, const FS<T> &fs)
{
   const Grid &g = r->g;
   Box b = h_box (g);
   const int NT = 256;
   const bool hn = r->np > 0 || r->probe_ring;
   MG_CUDA (cudaMemsetAsync (r->dsc->acc, 0, 2*sizeof (double), r->stream));
   const T c1 = (T) (0.5*g.tau/g.h[0]), c2 = (T) (0.5*g.tau/g.h[1]), c3 = (T) (0.5*g.tau/g.h[2]);
   if constexpr (sizeof (T) == sizeof (float)) {
      const Slots sl = make_slots (b);
      const int B = mg_blocks_for (sl.walk.vol, NT, 8);
      if (hn)
         k_h_fused4<true><<<B, NT, 0, r->stream>>> (g, f3 (fs.E), f3 (fs.H), f3 (fs.Hn), sl, c1, c2, c3,
                                                    energy_pick (g), r->dsc);
      else
         k_h_fused4<false><<<B, NT, 0, r->stream>>> (g, f3 (fs.E), f3 (fs.H), f3 (fs.Hn), sl, c1, c2, c3,
                                                     energy_pick (g), r->dsc);
   } else {
      const Slots sl = make_slots2 (b);
      const int B = mg_blocks_for (sl.walk.vol, NT, 8);
      if (hn)
         k_h_fused2<true><<<B, NT, 0, r->stream>>> (g, f3 (fs.E), f3 (fs.H), f3 (fs.Hn), sl, c1, c2, c3,
                                                    energy_pick (g), r->dsc);
      else
         k_h_fused2<false><<<B, NT, 0, r->stream>>> (g, f3 (fs.E), f3 (fs.H), f3 (fs.Hn), sl, c1, c2, c3,
                                                     energy_pick (g), r->dsc);
   }
   MG_LAUNCH_CHECK ();
   TRY_MG (mg_tfsf_h (r));
   TRY_MG (launch_mirrors<T> (r, fs, 0));
   if (walls_merge (r)) {
      const bool lm = laser_merge (r);
      if (!lm)
         TRY_MG (launch_laser<T> (r, fs, 0));
      return launch_walls_all<T, WK_H> (r, fs, hn ? 1 : 0, lm);
   }
   TRY_MG (launch_laser<T> (r, fs, 0));
   return launch_h_walls<T> (r, fs, hn ? 1 : 0);
}

// The one-pass field-only step (plain form): reads fs.E, fs.H, writes the
// new arrays En, Hw (E^(n+1), H^(n+1/2)); the caller swaps the pointers.
// Used for runs without markers, sources, probes or TF/SF, stepped alone.
template <typename T>
int fields_one_pass (mg_run_t *r, const FS<T> &fs, T *const En[3], T *const Hw[3])
{
   const Grid &g = r->g;
   const int NT = 256;
   const T c1 = (T) (0.5*g.tau/g.h[0]), c2 = (T) (0.5*g.tau/g.h[1]), c3 = (T) (0.5*g.tau/g.h[2]);
   const T d1 = (T) (g.tau/g.h[0]), d2 = (T) (g.tau/g.h[1]), d3 = (T) (g.tau/g.h[2]);
   const Box hb = h_box (g);
   const int in_lo[3] = {1, 1, 1};
   const int in_hi[3] = {g.n[0] - 1, g.n[1] - 1, g.n[2] - 1};
   const Slabs se = shell_slabs (e_box (g), in_lo, in_hi);
   MG_CUDA (cudaMemsetAsync (r->dsc->acc, 0, 2*sizeof (double), r->stream));
   constexpr int YT = 8, ZT = 32;
   using L = YeeTile<T, YT, ZT>;
   if ((g.origin - L::A) % L::V != 0 || g.sy % L::V != 0 || g.sx % L::V != 0)
      return MG_ERR_STATE;               // the grid layout lost its chunk alignment
   YeeTiles tl;
   for (int a = 0 ; a < 3 ; ++a) {
      tl.lo[a] = hb.lo[a];
      tl.n[a] = g.n[a];
   }
   tl.tj0 = tl.lo[1]/YT;
   tl.ntj = (g.n[1] - 1)/YT - tl.tj0 + 1;
   tl.tk0 = tl.lo[2]/ZT;
   tl.ntk = (g.n[2] - 1)/ZT - tl.tk0 + 1;
   tl.cx = 16;
   const int chunks = (g.n[0] - tl.lo[0] + tl.cx - 1)/tl.cx;
   k_yee_tile<T, YT, ZT><<<tl.ntj*tl.ntk*chunks, YT*ZT, 0, r->stream>>> (
      g, f3 (fs.E), f3 (fs.H), f3 (En), f3 (Hw), tl, c1, c2, c3, d1, d2, d3, energy_pick (g), r->dsc);
   MG_LAUNCH_CHECK ();
   FS<T> fh = fs;
   for (int c = 0 ; c < 3 ; ++c)
      fh.H[c] = Hw[c];
   TRY_MG ((launch_walls_all<T, WK_H> (r, fh, 0, false)));
   if (se.start[6] > 0) {
      k_shell_e<T><<<mg_blocks_for (se.start[6], NT, 8), NT, 0, r->stream>>> (
         g, f3 (fs.E), f3 (En), f3 (Hw), se, d1, d2, d3);
      MG_LAUNCH_CHECK ();
   }
   FS<T> fe = fs;
   for (int c = 0 ; c < 3 ; ++c)
      fe.E[c] = En[c];
   return launch_walls_all<T, WK_E> (r, fe, 0, false);
}

// Stage path: E += curl H only, then the E walls (Mur history before -tau J).
template <typename T>
int fields_e_step (mg_run_t *r, const FS<T> &fs)
{
   const Grid &g = r->g;
   Box b = e_box (g);
   const int NT = 256;
   k_e_advance<<<mg_blocks_for (b.vol, NT, 16), NT, 0, r->stream>>> (
      g, f3 (fs.E), f3 (fs.H), b, (T) (g.tau/g.h[0]), (T) (g.tau/g.h[1]), (T) (g.tau/g.h[2]));
   MG_LAUNCH_CHECK ();
   return launch_e_walls<T> (r, fs, 0);
}

template <typename T>
int fields_jbc (mg_run_t *r, const FS<T> &fs)
{
   const Grid &g = r->g;
   for (int ea = 0 ; ea < 3 ; ++ea) {
      const int ep = (ea == 0) ? 1 : 0, eq = (ea == 2) ? 1 : 2;
      const long nodes = (long) (g.n[ep] + 5)*(g.n[eq] + 5);
      const int NT = 256, B = (int) ((nodes + NT - 1)/NT);
      MG_AXIS_SWITCH (ea, k_j_walls<T, AX><<<B, NT, 0, r->stream>>> (g, f3 (fs.J)));
      MG_LAUNCH_CHECK ();
   }
   return MG_OK;
}

// Step graph: the three axes' current folding in one launch where it can.
template <typename T>
int fields_jbc_graph (mg_run_t *r, const FS<T> &fs)
{
   if (walls_merge (r))
      return launch_walls_all<T, WK_J> (r, fs, 0, false);
   return fields_jbc<T> (r, fs);
}


template <typename T>
static int launch_gauss_spot (mg_run_t *r, const FS<T> &fs)
{
   if (!r->has_gspot || r->gspot.i < -1 || r->gspot.i > r->g.n[0] + 1)
      return MG_OK;
   const long nodes = (long) (r->g.n[1] + 3)*(r->g.n[2] + 3);
   const int NT = 256, B = (int) ((nodes + NT - 1)/NT);
   k_gauss_spot<<<B, NT, 0, r->stream>>> (r->g, fs.E[1], fs.E[2], r->gspot, r->dsc);
   MG_LAUNCH_CHECK ();
   return MG_OK;
}

// Stage path: TF/SF faces, source at t + tau/2, then E -= tau J over
// [-1, n+1]^3, then the hard gauss-spot source (core/em.c:189-222).
template <typename T>
int fields_e_finish (mg_run_t *r, const FS<T> &fs)
{
   TRY_MG (mg_tfsf_e (r));
   TRY_MG (launch_mirrors<T> (r, fs, 1));
   TRY_MG (launch_laser<T> (r, fs, 1));
   const int lo[3] = {-1, -1, -1};
   const int hi[3] = {r->g.n[0] + 1, r->g.n[1] + 1, r->g.n[2] + 1};
   Box b = make_box (lo, hi);
   const int NT = 256;
   k_e_sub_j<<<mg_blocks_for (b.vol, NT, 16), NT, 0, r->stream>>> (r->g, f3 (fs.E), f3 (fs.J), b);
   MG_LAUNCH_CHECK ();
   return launch_gauss_spot<T> (r, fs);
}

// Graph path: E += curl H - tau J in one pass away from the rim, E walls,
// source, then -tau J on the rim.  Bit-identical to the stage path: every
// node sees the same operations in the same order.  Needs the J walls done.
// A playing TF/SF interface or a focused-laser mirror adds to E between the
// curl and -tau J, so with one the graph takes the stage path's two passes.
template <typename T>
int fields_e_fused (mg_run_t *r, const FS<T> &fs)
{
   if (mg_tfsf_playing (r) || r->nmirrors > 0) {
      TRY_MG (fields_e_step<T> (r, fs));
      return fields_e_finish<T> (r, fs);
   }
   const Grid &g = r->g;
   Box b = e_box (g);
   Rim rm = rim (r);
   const int NT = 256;
   // Without markers J stays zero (cleared when the step graph is built)
   // and -tau J is left out.
   const bool wj = r->np > 0;
   const T c1 = (T) (g.tau/g.h[0]), c2 = (T) (g.tau/g.h[1]), c3 = (T) (g.tau/g.h[2]);
   if constexpr (sizeof (T) == sizeof (float)) {
      const Slots sl = make_slots (b);
      const int B = mg_blocks_for (sl.walk.vol, NT, 8);
      if (wj)
         k_e_fused4<true><<<B, NT, 0, r->stream>>> (g, f3 (fs.E), f3 (fs.H), f3 (fs.J), sl, c1, c2, c3, rm);
      else
         k_e_fused4<false><<<B, NT, 0, r->stream>>> (g, f3 (fs.E), f3 (fs.H), f3 (fs.J), sl, c1, c2, c3, rm);
   } else if (wj) {
      k_e_fused<T, true><<<mg_blocks_for (b.vol, NT, 8), NT, 0, r->stream>>> (
         g, f3 (fs.E), f3 (fs.H), f3 (fs.J), b, c1, c2, c3, rm);
   } else {
      k_e_fused<T, false><<<mg_blocks_for (b.vol, NT, 8), NT, 0, r->stream>>> (
         g, f3 (fs.E), f3 (fs.H), f3 (fs.J), b, c1, c2, c3, rm);
   }
   MG_LAUNCH_CHECK ();
   if (walls_merge (r)) {
      const bool lm = laser_merge (r);
      TRY_MG ((launch_walls_all<T, WK_E> (r, fs, wj ? 1 : 0, lm)));
      if (!lm)
         TRY_MG (launch_laser<T> (r, fs, 1, wj ? 1 : 0));
   } else {
      TRY_MG (launch_e_walls<T> (r, fs, wj ? 1 : 0));
      TRY_MG (launch_laser<T> (r, fs, 1, wj ? 1 : 0));
   }
   return launch_gauss_spot<T> (r, fs);
}

template <typename T>
int fields_zero_j (mg_run_t *r, const FS<T> &fs)
{
   for (int c = 0 ; c < 3 ; ++c)
      MG_CUDA (cudaMemsetAsync (fs.J[c], 0, r->g.total*sizeof (T), r->stream));
   return MG_OK;
}

// cap_init equivalent (core/em_caps.c:343-392), axis by axis.
template <typename T>
int fields_init (mg_run_t *r, const FS<T> &fs)
{
   const Grid &g = r->g;
   for (int ea = 0 ; ea < 3 ; ++ea) {
      Wall w = make_wall (g, ea);
      const long nodes = (long) w.np_*w.nq_;
      const int NT = 256, B = (int) ((nodes + NT - 1)/NT);
      if (g.bc[0][ea] == MG_BC_PERIODIC) {
         k_h_wall<<<B, NT, 0, r->stream>>> (g, f3 (fs.H), w, OP_PERIODIC);
         k_e_wall<<<B, NT, 0, r->stream>>> (g, f3 (fs.E), w, OP_PERIODIC, (T *) nullptr, (T) 0);
         MG_LAUNCH_CHECK ();
         continue;
      }
      for (int top = 0 ; top < 2 ; ++top) {
         if (g.bc[top][ea] == MG_BC_MIRROR) {
            const int op = top ? OP_MIRROR_MAX : OP_MIRROR_MIN;
            k_h_wall<<<B, NT, 0, r->stream>>> (g, f3 (fs.H), w, op);
            k_e_wall<<<B, NT, 0, r->stream>>> (g, f3 (fs.E), w, op, (T *) nullptr, (T) 0);
         } else if (g.bc[top][ea] == MG_BC_OPEN) {
            k_mur_init<<<B, NT, 0, r->stream>>> (g, f3 (fs.E), w, top, fs.mur[top][ea]);
         }
         MG_LAUNCH_CHECK ();
      }
   }
   return MG_OK;
}

} // namespace
