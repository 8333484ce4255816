// Precision form (int cell + FP32 offset markers, FP32 fields): transfers in
// the reference's layouts, marker storage, device placement, the step graph
// and the periodic counting sort of markers by cell.
#include <cuda_runtime.h>

#include <stdlib.h>
#include <string.h>

#include "mg_internal.cuh"

#define TRY32(x)                                                             \
   do {                                                                      \
      int rc_ = (x);                                                         \
      if (rc_ != MG_OK)                                                      \
         return rc_;                                                         \
   } while (0)

namespace {

__device__ __forceinline__ int pack (int i, int j, int k) { return ((i + 1) << 20) | ((j + 1) << 10) | (k + 1); }
__device__ __forceinline__ int unpack (int c, int s) { return ((c >> s) & 1023) - 1; }

// Absolute FP64 position -> cell index and FP32 offset in [0, 1).
__device__ __forceinline__ void split (double x, double rh, int &c, float &o)
{
   const double s = x*rh;
   const double f = floor (s);
   c = (int) f;
   o = (float) (s - f);
   if (o >= 1.0f)
      o = 0.99999994f;
}

__global__ void k_fields_in32 (Grid g, const double *aos, float *c0, float *c1, float *c2)
{
   const long nk = g.n[2] + 1, nj = g.n[1] + 1, ni = g.n[0] + 1;
   const long vol = ni*nj*nk;
   for (long t = blockIdx.x*(long) blockDim.x + threadIdx.x ; t < vol ; t += (long) gridDim.x*blockDim.x) {
      const int k = (int) (t % nk), j = (int) ((t / nk) % nj), i = (int) (t / (nk*nj));
      const long o = g.at (i, j, k);
      c0[o] = (float) aos[3*t];
      c1[o] = (float) aos[3*t + 1];
      c2[o] = (float) aos[3*t + 2];
   }
}

__global__ void k_fields_out32 (Grid g, double *aos, const float *c0, const float *c1, const float *c2,
                                int ghost)
{
   const int lo = -ghost;
   const long nk = g.n[2] + 1 + 2*ghost, nj = g.n[1] + 1 + 2*ghost, ni = g.n[0] + 1 + 2*ghost;
   const long vol = ni*nj*nk;
   for (long t = blockIdx.x*(long) blockDim.x + threadIdx.x ; t < vol ; t += (long) gridDim.x*blockDim.x) {
      const int k = lo + (int) (t % nk), j = lo + (int) ((t / nk) % nj), i = lo + (int) (t / (nk*nj));
      const long o = g.at (i, j, k);
      aos[3*t] = c0[o];
      aos[3*t + 1] = c1[o];
      aos[3*t + 2] = c2[o];
   }
}

__global__ void k_markers_in32 (Grid g, const mg_marker_t *src, long long n, Markers32 m, long long at)
{
   const double rh0 = 1.0/g.h[0], rh1 = 1.0/g.h[1], rh2 = 1.0/g.h[2];
   for (long long t = blockIdx.x*(long long) blockDim.x + threadIdx.x ; t < n ; t += (long long) gridDim.x*blockDim.x) {
      const mg_marker_t p = src[t];
      const long long o = at + t;
      int i, j, k;
      float ox, oy, oz;
      split (p.x, rh0, i, ox);
      split (p.y, rh1, j, oy);
      split (p.z, rh2, k, oz);
      // Keep out-of-range markers representable; the push flags them.
      i = max (-1, min (i, 1022));
      j = max (-1, min (j, 1022));
      k = max (-1, min (k, 1022));
      m.cell[o] = pack (i, j, k);
      m.ox[o] = ox; m.oy[o] = oy; m.oz[o] = oz;
      m.ux[o] = (float) p.vx; m.uy[o] = (float) p.vy; m.uz[o] = (float) p.vz;
      m.rho[o] = p.rho;
      m.qm[o] = p.qDivM;
      m.id[o] = p.id;
   }
}

__global__ void k_markers_out32 (Grid g, Markers32 m, long long from, long long n, mg_marker_t *dst,
                                 const long long *slot)
{
   for (long long t = blockIdx.x*(long long) blockDim.x + threadIdx.x ; t < n ; t += (long long) gridDim.x*blockDim.x) {
      const long long o = from + t;
      const float qm = m.qm[o];
      if (qm == 0.0f)
         continue;
      const int c = m.cell[o];
      mg_marker_t p;
      p.x = (unpack (c, 20) + (double) m.ox[o])*g.h[0];
      p.y = (unpack (c, 10) + (double) m.oy[o])*g.h[1];
      p.z = (unpack (c, 0) + (double) m.oz[o])*g.h[2];
      p.vx = m.ux[o];
      p.vy = m.uy[o];
      p.vz = m.uz[o];
      p.rho = m.rho[o];
      p.qDivM = qm;
      p.id = m.id[o];
      p.pad_ = 0;
      dst[slot[t]] = p;
   }
}

__global__ void k_live_scan32 (const float *qm, long long from, long long n, long long *slot, long long *total)
{
   __shared__ long long part[1024];
   const int T = blockDim.x;
   const long long per = (n + T - 1)/T;
   const long long b = threadIdx.x*per, e = (b + per < n) ? b + per : n;
   long long cnt = 0;
   for (long long t = b ; t < e ; ++t)
      cnt += (qm[from + t] != 0.0f);
   part[threadIdx.x] = cnt;
   __syncthreads ();
   if (threadIdx.x == 0) {
      long long s = 0;
      for (int q = 0 ; q < T ; ++q) {
         const long long v = part[q];
         part[q] = s;
         s += v;
      }
      *total = s;
   }
   __syncthreads ();
   long long s = part[threadIdx.x];
   for (long long t = b ; t < e ; ++t) {
      slot[t] = s;
      s += (qm[from + t] != 0.0f);
   }
}

// ---- counting sort by tile and cell ----------------------------------------
// Key: tile index (tiles of the run's tile size, power-of-two sides, x-major)
// times the cells per tile plus the cell within the tile, so that a tile's
// markers are contiguous and, inside it, grouped by cell.  Markers in cells
// outside [0, n) go to one bucket after the last tile (the push handles them
// through global memory), removed markers to one more bucket at the end.
struct TileKey {
   int n[3], nty, ntz, ntiles;
   int lx, ly, lz;         // log2 of the tile size per axis
   int lc;                 // log2 of the cells per tile
};

__device__ __forceinline__ int sort_key (const TileKey &t, int c, float qm)
{
   if (qm == 0.0f)
      return (t.ntiles << t.lc) + 1;
   const int i = unpack (c, 20), j = unpack (c, 10), k = unpack (c, 0);
   if ((unsigned) i >= (unsigned) t.n[0] || (unsigned) j >= (unsigned) t.n[1] ||
       (unsigned) k >= (unsigned) t.n[2])
      return t.ntiles << t.lc;
   const int tile = ((i >> t.lx)*t.nty + (j >> t.ly))*t.ntz + (k >> t.lz);
   const int cell = ((((i & ((1 << t.lx) - 1)) << t.ly) + (j & ((1 << t.ly) - 1))) << t.lz) + (k & ((1 << t.lz) - 1));
   return (tile << t.lc) + cell;
}

// Marker count per key, and the largest |rho| (non-negative floats order
// like their bit patterns).  One atomic per run of equal keys in a warp;
// sixteen warp-rows of markers per iteration keep loads in flight (the
// kernels are latency-bound: 16 rows measured 19 % less sort time than 4).
#define SORT_ROWS 16
__global__ void k_hist (TileKey t, Markers32 m, long long np, int *count, long long kp, DevScalars *dsc)
{
   const int lane = threadIdx.x & 31;
   int rmax = 0;
   const long long stride = (long long) gridDim.x*blockDim.x*SORT_ROWS;
   for (long long base = (blockIdx.x*(long long) blockDim.x + (threadIdx.x & ~31))*SORT_ROWS ; base < np ;
        base += stride) {
      int key[SORT_ROWS];
      // Loads first, all rows at once (indices clamped into the array).
      float qm[SORT_ROWS], rho[SORT_ROWS];
      int cell[SORT_ROWS];
#pragma unroll
      for (int q = 0 ; q < SORT_ROWS ; ++q) {
         const long long n = min (base + 32*q + lane, np - 1);
         qm[q] = m.qm[n];
         cell[q] = m.cell[n];
         rho[q] = m.rho[n];
      }
#pragma unroll
      for (int q = 0 ; q < SORT_ROWS ; ++q) {
         const bool in = base + 32*q + lane < np;
         key[q] = in ? sort_key (t, cell[q], qm[q]) : -1;
         if (in && qm[q] != 0.0f)
            rmax = max (rmax, __float_as_int (fabsf (rho[q])));
      }
#pragma unroll
      for (int q = 0 ; q < SORT_ROWS ; ++q) {
         int start, len;
         key_runs (key[q], lane, start, len);
         if (key[q] >= 0 && start == lane)
            atomicAdd (count + spread (key[q], kp), len);
      }
   }
   for (int d = 16 ; d > 0 ; d >>= 1)
      rmax = max (rmax, __shfl_xor_sync (0xffffffffu, rmax, d));
   if (lane == 0 && rmax > 0)
      atomicMax ((int *) &dsc->rho_max, rmax);
}

// Three-pass exclusive scan of `count` (length len) in place.
__global__ void k_scan_blocks (const int *count, long long kp, long long len, long long *block_sum)
{
   __shared__ long long s[256];
   const long long b0 = (long long) blockIdx.x*SCAN_CHUNK;
   long long acc = 0;
   for (int q = threadIdx.x ; q < SCAN_CHUNK ; q += blockDim.x)
      if (b0 + q < len) acc += count[spread (b0 + q, kp)];
   s[threadIdx.x] = acc;
   __syncthreads ();
   for (int d = blockDim.x/2 ; d > 0 ; d >>= 1) {
      if ((int) threadIdx.x < d) s[threadIdx.x] += s[threadIdx.x + d];
      __syncthreads ();
   }
   if (threadIdx.x == 0) block_sum[blockIdx.x] = s[0];
}

// Exclusive scan of the nb block sums in place, one block of 1024 threads
// (thread t owns a contiguous segment).
__global__ void k_scan_sums (long long *block_sum, int nb)
{
   __shared__ long long part[1024];
   const int per = (nb + blockDim.x - 1)/blockDim.x;
   const int b = threadIdx.x*per, e = min (b + per, nb);
   long long acc = 0;
   for (int q = b ; q < e ; ++q)
      acc += block_sum[q];
   part[threadIdx.x] = acc;
   __syncthreads ();
   for (int d = 1 ; d < (int) blockDim.x ; d <<= 1) {
      const long long v = threadIdx.x >= (unsigned) d ? part[threadIdx.x - d] : 0;
      __syncthreads ();
      part[threadIdx.x] += v;
      __syncthreads ();
   }
   long long run = part[threadIdx.x] - acc;
   for (int q = b ; q < e ; ++q) {
      const long long v = block_sum[q];
      block_sum[q] = run;
      run += v;
   }
}

__global__ void k_scan_apply (const int *count, long long kp, long long len, const long long *block_sum,
                              long long *offset)
{
   // One block per chunk; thread t owns SCAN_CHUNK/blockDim consecutive entries.
   __shared__ long long part[256];
   const long long b0 = (long long) blockIdx.x*SCAN_CHUNK;
   const int per = SCAN_CHUNK/blockDim.x;
   const long long my0 = b0 + (long long) threadIdx.x*per;
   long long acc = 0;
   for (int q = 0 ; q < per ; ++q)
      if (my0 + q < len) acc += count[spread (my0 + q, kp)];
   part[threadIdx.x] = acc;
   __syncthreads ();
   if (threadIdx.x == 0) {
      long long s = block_sum[blockIdx.x];
      for (int q = 0 ; q < (int) blockDim.x ; ++q) {
         const long long v = part[q];
         part[q] = s;
         s += v;
      }
   }
   __syncthreads ();
   long long s = part[threadIdx.x];
   for (int q = 0 ; q < per ; ++q)
      if (my0 + q < len) {
         const long long v = count[spread (my0 + q, kp)];
         offset[my0 + q] = s;
         s += v;
      }
}

// First marker of every tile, of the outside bucket and of the removed bucket
// (before k_rank advances the offsets).
__global__ void k_tile_start (const long long *offset, int ntiles, int lc, int *tile_start)
{
   for (int t = blockIdx.x*blockDim.x + threadIdx.x ; t <= ntiles + 1 ; t += gridDim.x*blockDim.x)
      tile_start[t] = (int) offset[t <= ntiles ? (long long) t << lc : ((long long) ntiles << lc) + 1];
}

// The tiles that hold markers, appended to list (count in list[ntiles],
// zero on entry); the pushes hand out only these.
__global__ void k_tile_list (const long long *offset, int ntiles, int lc, int *list)
{
   for (int t = blockIdx.x*blockDim.x + threadIdx.x ; t < ntiles ; t += gridDim.x*blockDim.x)
      if (offset[(long long) (t + 1) << lc] > offset[(long long) t << lc])
         list[atomicAdd (list + ntiles, 1)] = t;
}

// Moves every marker to its place in the other buffer set: the first free
// slot of its key (a run of equal keys in a warp takes consecutive slots);
// fill counts the slots taken per key.
__global__ void k_scatter (TileKey t, Markers32 m, Markers32 o, long long np, const long long *offset,
                           int *fill, long long kp)
{
   const int lane = threadIdx.x & 31;
   const long long stride = (long long) gridDim.x*blockDim.x*SORT_ROWS;
   for (long long base = (blockIdx.x*(long long) blockDim.x + (threadIdx.x & ~31))*SORT_ROWS ; base < np ;
        base += stride) {
      // All loads first (indices clamped into the array), then the slots.
      int key[SORT_ROWS], cell[SORT_ROWS], id[SORT_ROWS];
      float qm[SORT_ROWS], ox[SORT_ROWS], oy[SORT_ROWS], oz[SORT_ROWS];
      float ux[SORT_ROWS], uy[SORT_ROWS], uz[SORT_ROWS], rho[SORT_ROWS];
      long long at[SORT_ROWS];
#pragma unroll
      for (int q = 0 ; q < SORT_ROWS ; ++q) {
         const long long n = min (base + 32*q + lane, np - 1);
         cell[q] = m.cell[n];
         qm[q] = m.qm[n];
         ox[q] = m.ox[n];
         oy[q] = m.oy[n];
         oz[q] = m.oz[n];
         ux[q] = m.ux[n];
         uy[q] = m.uy[n];
         uz[q] = m.uz[n];
         rho[q] = m.rho[n];
         id[q] = m.id[n];
      }
#pragma unroll
      for (int q = 0 ; q < SORT_ROWS ; ++q)
         key[q] = base + 32*q + lane < np ? sort_key (t, cell[q], qm[q]) : -1;
#pragma unroll
      for (int q = 0 ; q < SORT_ROWS ; ++q) {
         int start, len;
         key_runs (key[q], lane, start, len);
         at[q] = 0;
         if (key[q] >= 0 && start == lane)
            at[q] = offset[key[q]] + atomicAdd (fill + spread (key[q], kp), len);
         at[q] = __shfl_sync (0xffffffffu, at[q], start) + (lane - start);
      }
#pragma unroll
      for (int q = 0 ; q < SORT_ROWS ; ++q) {
         if (key[q] >= 0) {
            const long long a = at[q];
            o.cell[a] = cell[q];
            o.qm[a] = qm[q];
            o.ox[a] = ox[q];
            o.oy[a] = oy[q];
            o.oz[a] = oz[q];
            o.ux[a] = ux[q];
            o.uy[a] = uy[q];
            o.uz[a] = uz[q];
            o.rho[a] = rho[q];
            o.id[a] = id[q];
         }
      }
   }
}

} // namespace

static void free_set (mg_run_t *r, Markers32 &m)
{
   void *ptrs[] = {m.cell, m.ox, m.oy, m.oz, m.ux, m.uy, m.uz, m.rho, m.qm, m.id};
   for (void *p : ptrs)
      if (p)
         mg_dev_free (r, p);
   memset (&m, 0, sizeof (m));
}

static int alloc_set (mg_run_t *r, Markers32 &m, long long cap)
{
   memset (&m, 0, sizeof (m));
   void **d[] = {(void **) &m.cell, (void **) &m.ox, (void **) &m.oy, (void **) &m.oz,
                 (void **) &m.ux, (void **) &m.uy, (void **) &m.uz, (void **) &m.rho,
                 (void **) &m.qm, (void **) &m.id};
   for (void **p : d)
      TRY32 (mg_dev_alloc (r, p, (size_t) cap*4));
   return MG_OK;
}

void mg_free_markers32 (mg_run_t *r)
{
   free_set (r, r->m32);
   free_set (r, r->m32b);
}

namespace {
__global__ void k_publish (DevScalars *dsc, Markers32 m)
{
   dsc->m32 = m;
}
} // namespace

// Makes the current buffer set the one the step graph's kernels read (in
// stream order, without waiting for the host).
int mg_publish_markers32 (mg_run_t *r)
{
   k_publish<<<1, 1, 0, r->stream>>> (r->dsc, r->m32);
   MG_LAUNCH_CHECK ();
   return MG_OK;
}

int mg_ensure_capacity32 (mg_run_t *r, long long need)
{
   if (need <= r->cap)
      return MG_OK;
   if (need >= (1LL << 31) - 1) {
      mg_set_error ("precision form: %lld markers exceed the 2^31 per-run limit", need);
      return MG_ERR_CAPACITY;
   }
   long long cap = need + need/8 + 1024;
   if (cap >= (1LL << 31) - 1)
      cap = (1LL << 31) - 2;
   Markers32 nm, nb;
   int rc = alloc_set (r, nm, cap);
   if (rc == MG_OK)
      rc = alloc_set (r, nb, cap);
   if (rc != MG_OK) {
      free_set (r, nm);
      free_set (r, nb);
      return rc;
   }
   if (r->m32.cell && r->np > 0) {
      void *src[] = {r->m32.cell, r->m32.ox, r->m32.oy, r->m32.oz, r->m32.ux, r->m32.uy, r->m32.uz,
                     r->m32.rho, r->m32.qm, r->m32.id};
      void *dst[] = {nm.cell, nm.ox, nm.oy, nm.oz, nm.ux, nm.uy, nm.uz, nm.rho, nm.qm, nm.id};
      for (int q = 0 ; q < 10 ; ++q)
         MG_CUDA (cudaMemcpyAsync (dst[q], src[q], r->np*4, cudaMemcpyDeviceToDevice, r->stream));
      MG_CUDA (cudaStreamSynchronize (r->stream));
   }
   if (r->m32.cell) {
      r->dev_bytes -= (long long) r->cap*80;
      mg_free_markers32 (r);
   }
   r->m32 = nm;
   r->m32b = nb;
   r->cap = cap;
   mg_drop_graphs (r);
   return mg_publish_markers32 (r);
}

int mg_run_set_fields32 (mg_run_t *r, const double *E, const double *H)
{
   const long vol = (long) (r->g.n[0] + 1)*(r->g.n[1] + 1)*(r->g.n[2] + 1);
   const size_t bytes = (size_t) vol*3*sizeof (double);
   TRY32 (mg_ensure_stage (r, bytes));
   const double *src[2] = {E, H};
   float **dst[2] = {r->E32, r->H32};
   for (int f = 0 ; f < 2 ; ++f) {
      if (!src[f])
         continue;
      MG_CUDA (cudaMemcpyAsync (r->stage, src[f], bytes, cudaMemcpyHostToDevice, r->stream));
      k_fields_in32<<<mg_blocks_for (vol, 256, 8), 256, 0, r->stream>>> (
         r->g, (const double *) r->stage, dst[f][0], dst[f][1], dst[f][2]);
      MG_LAUNCH_CHECK ();
   }
   MG_CUDA (cudaStreamSynchronize (r->stream));
   r->inited = 0;
   return MG_OK;
}

int mg_fields_out32 (mg_run_t *r, double *E, double *H, bool dev)
{
   const long vol = (long) (r->g.n[0] + 1)*(r->g.n[1] + 1)*(r->g.n[2] + 1);
   const size_t bytes = (size_t) vol*3*sizeof (double);
   if (!dev)
      TRY32 (mg_ensure_stage (r, bytes));
   double *dst[2] = {E, H};
   float **src[2] = {r->E32, (r->stage_no >= 1 && r->stage_no <= 3) ? r->Hn32 : r->H32};
   for (int f = 0 ; f < 2 ; ++f) {
      if (!dst[f])
         continue;
      k_fields_out32<<<mg_blocks_for (vol, 256, 8), 256, 0, r->stream>>> (
         r->g, dev ? dst[f] : (double *) r->stage, src[f][0], src[f][1], src[f][2], 0);
      MG_LAUNCH_CHECK ();
      if (!dev) {
         MG_CUDA (cudaMemcpyAsync (dst[f], r->stage, bytes, cudaMemcpyDeviceToHost, r->stream));
         MG_CUDA (cudaStreamSynchronize (r->stream));
      }
   }
   return MG_OK;
}

int mg_run_get_current32 (mg_run_t *r, double *J)
{
   const long vol = (long) (r->g.n[0] + 5)*(r->g.n[1] + 5)*(r->g.n[2] + 5);
   const size_t bytes = (size_t) vol*3*sizeof (double);
   TRY32 (mg_ensure_stage (r, bytes));
   k_fields_out32<<<mg_blocks_for (vol, 256, 8), 256, 0, r->stream>>> (
      r->g, (double *) r->stage, r->J32[0], r->J32[1], r->J32[2], 2);
   MG_LAUNCH_CHECK ();
   MG_CUDA (cudaMemcpyAsync (J, r->stage, bytes, cudaMemcpyDeviceToHost, r->stream));
   MG_CUDA (cudaStreamSynchronize (r->stream));
   return MG_OK;
}

static const long long CHUNK32 = 1LL << 22;

int mg_run_set_markers32 (mg_run_t *r, const mg_marker_t *m, long long n)
{
   TRY32 (mg_ensure_capacity32 (r, n));
   const long long chunk = n < CHUNK32 ? n : CHUNK32;
   TRY32 (mg_ensure_stage (r, (size_t) (chunk > 0 ? chunk : 1)*sizeof (mg_marker_t)));
   for (long long at = 0 ; at < n ; at += CHUNK32) {
      const long long c = (n - at < CHUNK32) ? n - at : CHUNK32;
      MG_CUDA (cudaMemcpyAsync (r->stage, m + at, c*sizeof (mg_marker_t), cudaMemcpyHostToDevice, r->stream));
      k_markers_in32<<<mg_blocks_for (c, 256, 8), 256, 0, r->stream>>> (
         r->g, (const mg_marker_t *) r->stage, c, r->m32, at);
      MG_LAUNCH_CHECK ();
   }
   r->np = n;
   r->tiles_ok = 0;
   MG_CUDA (cudaMemsetAsync (&r->dsc->dead, 0, sizeof (long long), r->stream));
   MG_CUDA (cudaStreamSynchronize (r->stream));
   return MG_OK;
}

int mg_markers_out32 (mg_run_t *r, mg_marker_t *out, long long cap, long long *n, bool dev)
{
   long long live = 0;
   TRY32 (mg_run_marker_count (r, &live));
   if (n)
      *n = live;
   if (!out)
      return MG_OK;
   if (cap < live) {
      mg_set_error ("mg_run_get_markers: buffer holds %lld markers, %lld live", cap, live);
      return MG_ERR_CAPACITY;
   }
   const long long chunk = r->np < CHUNK32 ? r->np : CHUNK32;
   const long long c1 = chunk > 0 ? chunk : 1;
   TRY32 (mg_ensure_stage (r, (size_t) c1*(sizeof (mg_marker_t) + sizeof (long long)) + 64));
   mg_marker_t *dst = (mg_marker_t *) r->stage;
   long long *slot = (long long *) ((char *) r->stage + (size_t) c1*sizeof (mg_marker_t));
   long long *total_d = slot + c1;
   long long written = 0;
   for (long long at = 0 ; at < r->np ; at += CHUNK32) {
      const long long c = (r->np - at < CHUNK32) ? r->np - at : CHUNK32;
      k_live_scan32<<<1, 1024, 0, r->stream>>> (r->m32.qm, at, c, slot, total_d);
      k_markers_out32<<<mg_blocks_for (c, 256, 8), 256, 0, r->stream>>> (r->g, r->m32, at, c, dst, slot);
      MG_LAUNCH_CHECK ();
      long long got = 0;
      MG_CUDA (cudaMemcpyAsync (&got, total_d, sizeof (got), cudaMemcpyDeviceToHost, r->stream));
      MG_CUDA (cudaStreamSynchronize (r->stream));
      if (written + got > cap) {
         mg_set_error ("mg_run_get_markers: live count changed during download");
         return MG_ERR_STATE;
      }
      MG_CUDA (cudaMemcpyAsync (out + written, dst, got*sizeof (mg_marker_t),
                                dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, r->stream));
      MG_CUDA (cudaStreamSynchronize (r->stream));
      written += got;
   }
   if (n)
      *n = written;
   return MG_OK;
}

// Placement: FP64 positions from the shared generator, then split into cell
// and FP32 offset (placer.cu writes into a Markers64 view of staging).
int mg_place64 (mg_run_t *r, const mg_place_t *spec, long long at, long long count);

int mg_place32 (mg_run_t *r, const mg_place_t *spec, long long at, long long count)
{
   r->tiles_ok = 0;
   // Place in FP64 into staging in chunks of up to 2^26 markers (4.3 GB of
   // staging; larger chunks keep the host jump-ahead per chunk cheap), then
   // convert.
   const long long CH = 1LL << 26;
   for (long long done = 0 ; done < count ; ) {
      // The placer works on whole cells; split the box along i.
      mg_place_t s = *spec;
      const long long cells_jk = (long long) (spec->hi[1] - spec->lo[1])*(spec->hi[2] - spec->lo[2]);
      const long long per_i = cells_jk*spec->ppc;
      long long planes = CH/per_i;
      if (planes < 1) planes = 1;
      const long long i0 = spec->lo[0] + done/per_i;
      long long i1 = i0 + planes;
      if (i1 > spec->hi[0]) i1 = spec->hi[0];
      s.lo[0] = (int) i0;
      s.hi[0] = (int) i1;
      s.skip = spec->skip + 7*done;
      s.id0 = spec->id0 + (int) done;
      const long long c = (i1 - i0)*per_i;
      TRY32 (mg_ensure_stage (r, (size_t) c*sizeof (mg_marker_t)));
      // A Markers64 view of the staging buffer: 6 double arrays + rho, qm, id.
      char *base = (char *) r->stage;
      Markers64 save = r->m64;
      Markers64 v;
      v.x = (double *) base;
      v.y = v.x + c; v.z = v.y + c; v.ux = v.z + c; v.uy = v.ux + c; v.uz = v.uy + c;
      v.rho = (float *) (v.uz + c);
      v.qm = v.rho + c;
      v.id = (int *) (v.qm + c);
      r->m64 = v;
      int rc = mg_place64 (r, &s, 0, c);
      r->m64 = save;
      TRY32 (rc);
      // Convert: reuse the AoS path by packing into marker records would
      // need a second buffer; convert directly from the SoA view instead.
      extern void mg_convert64to32 (mg_run_t *r, const Markers64 &v, long long c, long long at);
      mg_convert64to32 (r, v, c, at + done);
      done += c;
   }
   MG_CUDA (cudaStreamSynchronize (r->stream));
   return MG_OK;
}

namespace {
__global__ void k_convert (Grid g, Markers64 v, long long c, Markers32 m, long long at)
{
   const double rh0 = 1.0/g.h[0], rh1 = 1.0/g.h[1], rh2 = 1.0/g.h[2];
   for (long long t = blockIdx.x*(long long) blockDim.x + threadIdx.x ; t < c ; t += (long long) gridDim.x*blockDim.x) {
      int i, j, k;
      float ox, oy, oz;
      split (v.x[t], rh0, i, ox);
      split (v.y[t], rh1, j, oy);
      split (v.z[t], rh2, k, oz);
      const long long o = at + t;
      m.cell[o] = pack (i, j, k);
      m.ox[o] = ox; m.oy[o] = oy; m.oz[o] = oz;
      m.ux[o] = (float) v.ux[t]; m.uy[o] = (float) v.uy[t]; m.uz[o] = (float) v.uz[t];
      m.rho[o] = v.rho[t];
      m.qm[o] = v.qm[t];
      m.id[o] = v.id[t];
   }
}
} // namespace

void mg_convert64to32 (mg_run_t *r, const Markers64 &v, long long c, long long at)
{
   k_convert<<<mg_blocks_for (c, 256, 8), 256, 0, r->stream>>> (r->g, v, c, r->m32, at);
}

// tile_start and tile_list of a run from the exclusive scan of its sort
// keys (lc: log2 of the cells per tile).
int mg_tile_list (mg_run_t *r, const long long *offset, int lc)
{
   const int T = 256;
   k_tile_start<<<mg_blocks_for (r->ntiles + 2, T, 8), T, 0, r->stream>>> (offset, r->ntiles, lc, r->tile_start);
   MG_CUDA (cudaMemsetAsync (r->tile_list + r->ntiles, 0, sizeof (int), r->stream));
   k_tile_list<<<mg_blocks_for (r->ntiles, T, 8), T, 0, r->stream>>> (offset, r->ntiles, lc, r->tile_list);
   MG_LAUNCH_CHECK ();
   return MG_OK;
}

// Sorts the markers by tile and cell into the other buffer set and makes
// that set current; removed markers go to the end.
// Exclusive scan of the len counters (spread layout, kp keys per region)
// into offset; bsum: (len + SCAN_CHUNK - 1)/SCAN_CHUNK scratch entries.
int mg_scan_counts (mg_run_t *r, const int *count, long long kp, long long len, long long *offset,
                    long long *bsum)
{
   const int nb = (int) ((len + SCAN_CHUNK - 1)/SCAN_CHUNK);
   k_scan_blocks<<<nb, 256, 0, r->stream>>> (count, kp, len, bsum);
   k_scan_sums<<<1, 1024, 0, r->stream>>> (bsum, nb);
   k_scan_apply<<<nb, 256, 0, r->stream>>> (count, kp, len, bsum, offset);
   MG_LAUNCH_CHECK ();
   return MG_OK;
}

int mg_sort32 (mg_run_t *r)
{
   if (r->np == 0) {
      MG_CUDA (cudaMemsetAsync (r->tile_start, 0, sizeof (int)*(2*(size_t) r->ntiles + 4), r->stream));
      r->tiles_ok = 1;
      r->steps_since_sort = 0;
      return MG_OK;
   }
   TileKey tk;
   for (int a = 0 ; a < 3 ; ++a)
      tk.n[a] = r->g.n[a];
   tk.nty = r->tiles[1];
   tk.ntz = r->tiles[2];
   tk.ntiles = r->ntiles;
   tk.lx = __builtin_ctz (r->tdim[0]);
   tk.ly = __builtin_ctz (r->tdim[1]);
   tk.lz = __builtin_ctz (r->tdim[2]);
   tk.lc = tk.lx + tk.ly + tk.lz;
   const long long cells = ((long long) r->ntiles << tk.lc) + 2;
   const int nb = (int) ((cells + SCAN_CHUNK - 1)/SCAN_CHUNK);
   const long long kp = (cells + 7)/8;
   const size_t need = (size_t) kp*8*4 + (size_t) cells*8 + (size_t) nb*8 + 1024;
   if (r->sort_tmp_bytes < need) {
      if (r->sort_tmp) {
         mg_dev_free (r, r->sort_tmp);
         r->dev_bytes -= r->sort_tmp_bytes;
         r->sort_tmp = nullptr;
      }
      TRY32 (mg_dev_alloc (r, &r->sort_tmp, need));
      r->sort_tmp_bytes = need;
   }
   char *p = (char *) r->sort_tmp;
   int *count = (int *) p;                        p += ((size_t) kp*8*4 + 255) & ~(size_t) 255;
   long long *offset = (long long *) p;           p += ((size_t) cells*8 + 255) & ~(size_t) 255;
   long long *bsum = (long long *) p;
   MG_CUDA (cudaMemsetAsync (count, 0, (size_t) kp*8*4, r->stream));
   MG_CUDA (cudaMemsetAsync (&r->dsc->rho_max, 0, sizeof (float), r->stream));
   const int T = 256;
   k_hist<<<mg_blocks_for (r->np, T, 8), T, 0, r->stream>>> (tk, r->m32, r->np, count, kp, r->dsc);
   k_scan_blocks<<<nb, 256, 0, r->stream>>> (count, kp, cells, bsum);
   k_scan_sums<<<1, 1024, 0, r->stream>>> (bsum, nb);
   k_scan_apply<<<nb, 256, 0, r->stream>>> (count, kp, cells, bsum, offset);
   TRY32 (mg_tile_list (r, offset, tk.lc));
   // The counters become the per-key fill counts of the scatter.
   MG_CUDA (cudaMemsetAsync (count, 0, (size_t) kp*8*4, r->stream));
   k_scatter<<<mg_blocks_for (r->np, T, 8), T, 0, r->stream>>> (tk, r->m32, r->m32b, r->np, offset, count, kp);
   MG_LAUNCH_CHECK ();
   const Markers32 t = r->m32;
   r->m32 = r->m32b;
   r->m32b = t;
   // Removed markers now sit at the end; they stay there (the step graph
   // holds the marker count) and are dropped on download.
   r->steps_since_sort = 0;
   r->tiles_ok = 1;
   return mg_publish_markers32 (r);
}

int mg_enqueue_step32 (mg_run_t *r, int part)
{
   if (part < 0 && r->fo_graph) {        // field-only: one pass into Ealt32, Halt32
      TRY32 (mg_fields32_one_pass (r));
      return mg_end_step (r);
   }
   if (part < 0 || part == 0) {
      TRY32 (mg_tfsf_record (r));
      TRY32 (mg_fields32_h_both (r));
      TRY32 (mg_probes_enqueue (r));
      if (r->np > 0)                       // without markers J stays zero
         TRY32 (mg_fields32_zero_j (r));
   }
   if (part < 0 || part == 1)
      TRY32 (mg_push32 (r));
   if (part < 0 || part == 2) {
      if (r->np > 0)
         TRY32 (mg_fields32_jbc_graph (r));
      TRY32 (mg_fields32_e_fused (r));
      TRY32 (mg_end_step (r));
   }
   return MG_OK;
}
