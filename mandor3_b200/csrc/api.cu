// C ABI of the B200 PIC core (declared in include/mandor_b200.h): run
// lifetime, host<->device transfers in the reference's layouts, the stage
// API that mirrors core/main.c's step, and the graph-replayed step loop.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mg_internal.cuh"

// ---------------------------------------------------------------------------
// Errors.
// ---------------------------------------------------------------------------
static thread_local char g_err[1024];

void mg_set_error (const char *fmt, ...)
{
   va_list ap;
   va_start (ap, fmt);
   vsnprintf (g_err, sizeof (g_err), fmt, ap);
   va_end (ap);
}

extern "C" const char *mg_last_error (void) { return g_err; }
extern "C" const char *mg_version (void) { return "mandor_b200 1.0 (sm_100a)"; }

int mg_sm_count (void)
{
   static int count = 0;
   if (!count) {
      int dev = 0;
      cudaGetDevice (&dev);
      if (cudaDeviceGetAttribute (&count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || count <= 0)
         count = 148;
   }
   return count;
}

#define CHECK_RUN(r)                                                         \
   do {                                                                      \
      if (!(r)) {                                                            \
         mg_set_error ("%s: null run", __func__);                            \
         return MG_ERR_ARG;                                                  \
      }                                                                      \
      cudaSetDevice ((r)->device);                                           \
   } while (0)

#define TRY(x)                                                               \
   do {                                                                      \
      int rc_ = (x);                                                         \
      if (rc_ != MG_OK)                                                      \
         return rc_;                                                         \
   } while (0)

void mg_drop_graphs (mg_run_t *r);
#define MG_PROFILE_CHUNK 512

// ---------------------------------------------------------------------------
// Layout conversion kernels.
// ---------------------------------------------------------------------------
namespace {

// Reference AoS region [0,n]^3 (k fastest) <-> device SoA.
__global__ void k_fields_in (Grid g, const double *aos, double *c0, double *c1, double *c2)
{
   const long nk = g.n[2] + 1, nj = g.n[1] + 1, ni = g.n[0] + 1;
   const long vol = ni*nj*nk;
   for (long t = blockIdx.x*(long) blockDim.x + threadIdx.x ; t < vol ; t += (long) gridDim.x*blockDim.x) {
      const int k = (int) (t % nk), j = (int) ((t / nk) % nj), i = (int) (t / (nk*nj));
      const long o = g.at (i, j, k);
      c0[o] = aos[3*t];
      c1[o] = aos[3*t + 1];
      c2[o] = aos[3*t + 2];
   }
}

__global__ void k_fields_out (Grid g, double *aos, const double *c0, const double *c1, const double *c2,
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

__global__ void k_markers_in (const mg_marker_t *src, long long n, Markers64 m, long long at)
{
   for (long long t = blockIdx.x*(long long) blockDim.x + threadIdx.x ; t < n ; t += (long long) gridDim.x*blockDim.x) {
      const mg_marker_t p = src[t];
      const long long o = at + t;
      m.x[o] = p.x;
      m.y[o] = p.y;
      m.z[o] = p.z;
      m.ux[o] = p.vx;
      m.uy[o] = p.vy;
      m.uz[o] = p.vz;
      m.rho[o] = p.rho;
      m.qm[o] = p.qDivM;
      m.id[o] = p.id;
   }
}

// Live-marker flags and packing (removed markers carry qDivM = 0).
__global__ void k_markers_out (Markers64 m, long long from, long long n, mg_marker_t *dst,
                               const long long *slot)
{
   for (long long t = blockIdx.x*(long long) blockDim.x + threadIdx.x ; t < n ; t += (long long) gridDim.x*blockDim.x) {
      const long long o = from + t;
      const float qm = m.qm[o];
      if (qm == 0.0f)
         continue;
      mg_marker_t p;
      p.x = m.x[o];
      p.y = m.y[o];
      p.z = m.z[o];
      p.vx = m.ux[o];
      p.vy = m.uy[o];
      p.vz = m.uz[o];
      p.rho = m.rho[o];
      p.qDivM = qm;
      p.id = m.id[o];
      p.pad_ = 0;
      dst[slot ? slot[t] : t] = p;
   }
}

// Exclusive scan of live flags within one chunk, single block (chunks are
// at most a few million markers; this runs only on download).
__global__ void k_live_scan (const float *qm, long long from, long long n, long long *slot,
                             long long *total)
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

// End of a step: energy row {t, W_E, W_M, W_Tx, W_Ty, W_Tz} into the ring,
// accumulators cleared, time advanced (parameter_setTime, core/main.c:435).
__global__ void k_end_step (DevScalars *dsc, double *ring, double volume, double tau)
{
   const int s = dsc->step % MG_RING;
   double *row = ring + 6*s;
   row[0] = dsc->time;
   row[1] = 0.5*dsc->acc[0]*volume;
   row[2] = 0.5*dsc->acc[1]*volume;
   row[3] = dsc->acc[2];
   row[4] = dsc->acc[3];
   row[5] = dsc->acc[4];
   for (int q = 0 ; q < 8 ; ++q)
      dsc->acc[q] = 0;
   dsc->time += tau;
   dsc->step += 1;
   dsc->tfsf_frame += 1;          // TFSF_completeFrame (core/em_TFSF.c:849-853)
}

} // namespace

// ---------------------------------------------------------------------------
// Allocation.
// ---------------------------------------------------------------------------
// Run state comes from one stream-ordered memory pool per device.  A run
// that finishes returns its buffers to the pool, and the next run created
// on that device reuses them: no page mapping or unmapping and no
// device-wide synchronisation per buffer, which cudaMalloc and cudaFree
// would cost every solve a server admits and retires.  The pool keeps up to
// MG_POOL_KEEP bytes of freed memory for reuse and returns the rest to the
// device at the next synchronisation.
#define MG_POOL_KEEP (16ull << 30)

static std::mutex    g_pool_mutex;
static cudaMemPool_t g_pool[64];

static int device_pool (int dev, cudaMemPool_t *out)
{
   if (dev < 0 || dev >= 64) {
      mg_set_error ("device %d: no memory pool slot", dev);
      return MG_ERR_ARG;
   }
   std::lock_guard<std::mutex> lock (g_pool_mutex);
   if (!g_pool[dev]) {
      cudaMemPoolProps props;
      memset (&props, 0, sizeof (props));
      props.allocType = cudaMemAllocationTypePinned;
      props.handleTypes = cudaMemHandleTypeNone;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      cudaMemPool_t pool;
      cudaError_t e = cudaMemPoolCreate (&pool, &props);
      if (e != cudaSuccess) {
         cudaGetLastError ();
         mg_set_error ("cannot create the memory pool of device %d: %s", dev, cudaGetErrorString (e));
         return MG_ERR_CUDA;
      }
      uint64_t keep = MG_POOL_KEEP;
      cudaMemPoolSetAttribute (pool, cudaMemPoolAttrReleaseThreshold, &keep);
      g_pool[dev] = pool;
   }
   *out = g_pool[dev];
   return MG_OK;
}

// Allocates on the run's stream and waits for the allocation, so that the
// buffer is usable from any stream when this returns.
int mg_dev_alloc (mg_run_t *r, void **p, size_t bytes)
{
   *p = nullptr;
   cudaMemPool_t pool;
   TRY (device_pool (r->device, &pool));
   cudaError_t e = cudaMallocFromPoolAsync (p, bytes ? bytes : 16, pool, r->stream);
   if (e == cudaSuccess)
      e = cudaStreamSynchronize (r->stream);
   if (e != cudaSuccess) {
      cudaGetLastError ();
      mg_set_error ("device allocation of %.3f GB failed: %s", bytes/1e9, cudaGetErrorString (e));
      *p = nullptr;
      return MG_ERR_OOM;
   }
   if ((uintptr_t) *p & 255) {            // TMA and the padded rows rely on this
      cudaFreeAsync (*p, r->stream);
      *p = nullptr;
      mg_set_error ("device allocation not 256-byte aligned");
      return MG_ERR_CUDA;
   }
   r->dev_bytes += bytes;
   return MG_OK;
}

// Returns a buffer of the run to the pool.  Kernels and copies on the run's
// stream that use it are ordered before the free; the transfer and
// snapshot streams are waited for here.
void mg_dev_free (mg_run_t *r, void *p)
{
   if (!p)
      return;
   if (r->xfer)
      cudaStreamSynchronize (r->xfer);
   if (r->snap_stream)
      cudaStreamSynchronize (r->snap_stream);
   if (cudaFreeAsync (p, r->stream) != cudaSuccess)
      cudaGetLastError ();
}

int mg_ensure_stage (mg_run_t *r, size_t bytes)
{
   if (r->stage_bytes >= bytes)
      return MG_OK;
   if (r->stage) {
      mg_dev_free (r, r->stage);
      r->dev_bytes -= r->stage_bytes;
      r->stage = nullptr;
      r->stage_bytes = 0;
   }
   TRY (mg_dev_alloc (r, &r->stage, bytes));
   r->stage_bytes = bytes;
   return MG_OK;
}

// The copy stream and its events (created on first use).
static int ensure_xfer (mg_run_t *r)
{
   if (r->xfer)
      return MG_OK;
   MG_CUDA (cudaStreamCreateWithFlags (&r->xfer, cudaStreamNonBlocking));
   for (int b = 0 ; b < 2 ; ++b)
      for (int e = 0 ; e < 2 ; ++e)
         MG_CUDA (cudaEventCreateWithFlags (&r->xev[b][e], cudaEventDisableTiming));
   return MG_OK;
}

// Device -> host through the two halves of the staging buffer: chunk q is
// converted on the run's stream into half q % 2 (`convert` launches the
// kernel for chunk q, of `bytes[q]` bytes), then copied to host[q] on the
// copy stream while the run's stream converts chunk q + 1.
template <class Convert>
static int pipelined_d2h (mg_run_t *r, int chunks, size_t half, Convert convert, void *const *host,
                          const size_t *bytes)
{
   TRY (ensure_xfer (r));
   TRY (mg_ensure_stage (r, 2*half));
   for (int q = 0 ; q < chunks ; ++q) {
      const int b = q & 1;
      char *buf = (char *) r->stage + b*half;
      if (q >= 2)
         MG_CUDA (cudaStreamWaitEvent (r->stream, r->xev[b][1], 0));    // copy q-2 done with buf
      convert (q, buf);
      MG_LAUNCH_CHECK ();
      MG_CUDA (cudaEventRecord (r->xev[b][0], r->stream));
      MG_CUDA (cudaStreamWaitEvent (r->xfer, r->xev[b][0], 0));
      MG_CUDA (cudaMemcpyAsync (host[q], buf, bytes[q], cudaMemcpyDeviceToHost, r->xfer));
      MG_CUDA (cudaEventRecord (r->xev[b][1], r->xfer));
   }
   MG_CUDA (cudaStreamSynchronize (r->xfer));
   return MG_OK;
}

// Host -> device, the same two halves the other way: chunk q is copied on
// the copy stream into half q % 2, then converted on the run's stream while
// chunk q + 1 is copied.
template <class Convert>
static int pipelined_h2d (mg_run_t *r, int chunks, size_t half, Convert convert, const void *const *host,
                          const size_t *bytes)
{
   TRY (ensure_xfer (r));
   TRY (mg_ensure_stage (r, 2*half));
   MG_CUDA (cudaEventRecord (r->xev[0][1], r->stream));     // earlier work on the stage is ordered first
   MG_CUDA (cudaStreamWaitEvent (r->xfer, r->xev[0][1], 0));
   for (int q = 0 ; q < chunks ; ++q) {
      const int b = q & 1;
      char *buf = (char *) r->stage + b*half;
      if (q >= 2)
         MG_CUDA (cudaStreamWaitEvent (r->xfer, r->xev[b][1], 0));      // conversion q-2 done with buf
      MG_CUDA (cudaMemcpyAsync (buf, host[q], bytes[q], cudaMemcpyHostToDevice, r->xfer));
      MG_CUDA (cudaEventRecord (r->xev[b][0], r->xfer));
      MG_CUDA (cudaStreamWaitEvent (r->stream, r->xev[b][0], 0));
      convert (q, buf);
      MG_LAUNCH_CHECK ();
      MG_CUDA (cudaEventRecord (r->xev[b][1], r->stream));
   }
   return MG_OK;
}

static void free_markers (mg_run_t *r)
{
   void *ptrs[] = {r->m64.x, r->m64.y, r->m64.z, r->m64.ux, r->m64.uy, r->m64.uz,
                   r->m64.rho, r->m64.qm, r->m64.id};
   for (void *p : ptrs)
      if (p)
         mg_dev_free (r, p);
   memset (&r->m64, 0, sizeof (r->m64));
}

static size_t marker_bytes64 (long long cap) { return (size_t) cap*(6*8 + 4 + 4 + 4); }

static int ensure_capacity (mg_run_t *r, long long need)
{
   if (need <= r->cap)
      return MG_OK;
   long long cap = need + need/8 + 1024;
   Markers64 old = r->m64;
   long long old_np = r->np;
   Markers64 nm;
   memset (&nm, 0, sizeof (nm));
   void **d[] = {(void **) &nm.x, (void **) &nm.y, (void **) &nm.z, (void **) &nm.ux,
                 (void **) &nm.uy, (void **) &nm.uz};
   for (void **p : d)
      TRY (mg_dev_alloc (r, p, (size_t) cap*8));
   TRY (mg_dev_alloc (r, (void **) &nm.rho, (size_t) cap*4));
   TRY (mg_dev_alloc (r, (void **) &nm.qm, (size_t) cap*4));
   TRY (mg_dev_alloc (r, (void **) &nm.id, (size_t) cap*4));
   if (old.x && old_np > 0) {
      MG_CUDA (cudaMemcpyAsync (nm.x, old.x, old_np*8, cudaMemcpyDeviceToDevice, r->stream));
      MG_CUDA (cudaMemcpyAsync (nm.y, old.y, old_np*8, cudaMemcpyDeviceToDevice, r->stream));
      MG_CUDA (cudaMemcpyAsync (nm.z, old.z, old_np*8, cudaMemcpyDeviceToDevice, r->stream));
      MG_CUDA (cudaMemcpyAsync (nm.ux, old.ux, old_np*8, cudaMemcpyDeviceToDevice, r->stream));
      MG_CUDA (cudaMemcpyAsync (nm.uy, old.uy, old_np*8, cudaMemcpyDeviceToDevice, r->stream));
      MG_CUDA (cudaMemcpyAsync (nm.uz, old.uz, old_np*8, cudaMemcpyDeviceToDevice, r->stream));
      MG_CUDA (cudaMemcpyAsync (nm.rho, old.rho, old_np*4, cudaMemcpyDeviceToDevice, r->stream));
      MG_CUDA (cudaMemcpyAsync (nm.qm, old.qm, old_np*4, cudaMemcpyDeviceToDevice, r->stream));
      MG_CUDA (cudaMemcpyAsync (nm.id, old.id, old_np*4, cudaMemcpyDeviceToDevice, r->stream));
      MG_CUDA (cudaStreamSynchronize (r->stream));
   }
   if (old.x) {
      r->dev_bytes -= marker_bytes64 (r->cap);
      free_markers (r);
   }
   r->m64 = nm;
   r->cap = cap;
   // The captured graphs hold the old pointers.
   mg_drop_graphs (r);
   return MG_OK;
}

static int check_params (const mg_params_t *p)
{
   for (int a = 0 ; a < 3 ; ++a) {
      if (p->n[a] < 8) {
         mg_set_error ("axis %d: %d cells; at least 8 are needed (core/plasma.c:392-396)", a, p->n[a]);
         return MG_ERR_ARG;
      }
      if (!(p->h[a] > 0)) {
         mg_set_error ("axis %d: mesh step %g", a, p->h[a]);
         return MG_ERR_ARG;
      }
      for (int t = 0 ; t < 2 ; ++t) {
         const int bc = t ? p->bc_max[a] : p->bc_min[a];
         if (bc < MG_BC_PERIODIC || bc > MG_BC_OPEN) {
            mg_set_error ("axis %d: unknown boundary condition %d", a, bc);
            return MG_ERR_ARG;
         }
      }
      if ((p->bc_min[a] == MG_BC_PERIODIC) != (p->bc_max[a] == MG_BC_PERIODIC)) {
         mg_set_error ("axis %d: periodic must be set on both walls", a);
         return MG_ERR_ARG;
      }
   }
   const double c = 1.0/(p->tau*p->tau), s = 1.0/(p->h[0]*p->h[0]) + 1.0/(p->h[1]*p->h[1]) + 1.0/(p->h[2]*p->h[2]);
   if (!(p->tau > 0) || !(c > s)) {
      mg_set_error ("Yee-solver is unstable: tau = %g (core/em.c:43-44)", p->tau);
      return MG_ERR_ARG;
   }
   if (p->precision != MG_FP64 && p->precision != MG_FP32_OFFSET) {
      mg_set_error ("unknown precision form %d", p->precision);
      return MG_ERR_ARG;
   }
   {
      const int *t = p->tile;
      const bool ok = (t[0] == 0 && t[1] == 0 && t[2] == 0) || (t[0] == 8 && t[1] == 8 && t[2] == 4) ||
                      (t[0] == 4 && t[1] == 4 && t[2] == 4) || (t[0] == 8 && t[1] == 8 && t[2] == 8);
      if (!ok) {
         mg_set_error ("tile %dx%dx%d: the push is built for 8x8x4, 4x4x4 and 8x8x8", t[0], t[1], t[2]);
         return MG_ERR_ARG;
      }
      const int w = p->tile_warps;
      if (w != 0 && w != 4 && w != 8 && w != 16) {
         mg_set_error ("tile_warps %d: the tiled push is built for 4, 8 and 16 warps a block", w);
         return MG_ERR_ARG;
      }
   }
   return MG_OK;
}

extern "C" long long mg_estimate_bytes (const mg_params_t *p, long long markers)
{
   if (!p)
      return -1;
   Grid g = make_grid (p->n, p->h, p->tau, p->bc_min, p->bc_max,
                       p->precision == MG_FP64 ? MG_GZ_FRONT : MG_GZ_FRONT32);
   const long long elt = (p->precision == MG_FP64) ? 8 : 4;
   long long b = 12LL*g.total*elt;
   if (markers == 0)                  // one-pass field step: a second E and H set
      b += 6LL*g.total*elt;
   for (int a = 0 ; a < 3 ; ++a)
      b += 2LL*4*elt*(p->n[(a + 1) % 3] + 2)*(p->n[(a + 2) % 3] + 2);
   // FP64: SoA records; precision form: two buffer sets (the sort scatters
   // from one into the other) and 12 bytes of sort counters per cell.
   const long long per_marker = (p->precision == MG_FP64) ? 60 : 80;
   b += (markers + markers/8 + 1024)*per_marker;
   if (p->precision != MG_FP64)
      b += 12LL*(p->n[0] + 8)*(p->n[1] + 8)*(p->n[2] + 8);
   b += (long long) MG_RING*6*8 + (1 << 20);
   return b;
}

extern "C" int mg_run_create (const mg_params_t *params, mg_run_t **out)
{
   if (!params || !out) {
      mg_set_error ("mg_run_create: null argument");
      return MG_ERR_ARG;
   }
   *out = nullptr;
   TRY (check_params (params));
   int ndev = 0;
   if (cudaGetDeviceCount (&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError ();
      mg_set_error ("no CUDA device available: the B200 core has no CPU path");
      return MG_ERR_CUDA;
   }
   if (params->device < 0 || params->device >= ndev) {
      mg_set_error ("device %d out of range (%d devices)", params->device, ndev);
      return MG_ERR_ARG;
   }
   MG_CUDA (cudaSetDevice (params->device));
   mg_run_t *r = (mg_run_t *) calloc (1, sizeof (mg_run_t));
   r->prm = *params;
   r->device = params->device;
   r->g = make_grid (params->n, params->h, params->tau, params->bc_min, params->bc_max,
                     params->precision == MG_FP64 ? MG_GZ_FRONT : MG_GZ_FRONT32);
   r->time = params->time;
   if (cudaStreamCreateWithFlags (&r->stream, cudaStreamNonBlocking) != cudaSuccess) {
      free (r);
      mg_set_error ("cannot create a stream");
      return MG_ERR_CUDA;
   }
   int rc = MG_OK;
   const bool f32 = (params->precision == MG_FP32_OFFSET);
   const size_t elt = f32 ? sizeof (float) : sizeof (double);
   const size_t fb = (size_t) r->g.total*elt;
   for (int c = 0 ; c < 3 && rc == MG_OK ; ++c) {
      void **arrs[4] = {f32 ? (void **) &r->E32[c] : (void **) &r->E[c],
                        f32 ? (void **) &r->H32[c] : (void **) &r->H[c],
                        f32 ? (void **) &r->J32[c] : (void **) &r->J[c],
                        f32 ? (void **) &r->Hn32[c] : (void **) &r->Hn[c]};
      for (int q = 0 ; q < 4 && rc == MG_OK ; ++q) {
         rc = mg_dev_alloc (r, arrs[q], fb);
         if (rc == MG_OK)
            cudaMemsetAsync (*arrs[q], 0, fb, r->stream);
      }
   }
   for (int t = 0 ; t < 2 && rc == MG_OK ; ++t)
      for (int a = 0 ; a < 3 && rc == MG_OK ; ++a) {
         const size_t mb = 4*elt*(size_t) (params->n[(a + 1) % 3] + 2)*(params->n[(a + 2) % 3] + 2);
         void **mp = f32 ? (void **) &r->mur32[t][a] : (void **) &r->mur[t][a];
         rc = mg_dev_alloc (r, mp, mb);
         if (rc == MG_OK)
            cudaMemsetAsync (*mp, 0, mb, r->stream);
      }
   if (rc == MG_OK && f32) {
      const bool deflt = params->tile[0] == 0 && params->tile[1] == 0 && params->tile[2] == 0;
      const int T[3] = {deflt ? MG_TILE_X : params->tile[0], deflt ? MG_TILE_Y : params->tile[1],
                        deflt ? MG_TILE_Z : params->tile[2]};
      r->ntiles = 1;
      for (int a = 0 ; a < 3 ; ++a) {
         r->tdim[a] = T[a];
         r->tiles[a] = (params->n[a] + T[a] - 1)/T[a];
         r->ntiles *= r->tiles[a];
      }
      const size_t tb = sizeof (int)*(2*(size_t) r->ntiles + 4);
      rc = mg_dev_alloc (r, (void **) &r->tile_start, tb);
      if (rc == MG_OK) {
         cudaMemsetAsync (r->tile_start, 0, tb, r->stream);
         r->tile_list = r->tile_start + r->ntiles + 2;
      }
   }
   if (rc == MG_OK) rc = mg_dev_alloc (r, (void **) &r->dsc, sizeof (DevScalars));
   if (rc == MG_OK) rc = mg_dev_alloc (r, (void **) &r->ring, sizeof (double)*6*MG_RING);
   if (rc == MG_OK) {
      DevScalars s;
      memset (&s, 0, sizeof (s));
      s.time = r->time;
      cudaMemcpyAsync (r->dsc, &s, sizeof (s), cudaMemcpyHostToDevice, r->stream);
   }
   if (rc == MG_OK && params->capacity > 0)
      rc = f32 ? mg_ensure_capacity32 (r, params->capacity) : ensure_capacity (r, params->capacity);
   for (int e = 0 ; e < 4 && rc == MG_OK ; ++e)
      if (cudaEventCreate (&r->ev[e]) != cudaSuccess)
         rc = MG_ERR_CUDA;
   if (rc == MG_OK && cudaStreamSynchronize (r->stream) != cudaSuccess) {
      mg_set_error ("initialisation failed: %s", cudaGetErrorString (cudaGetLastError ()));
      rc = MG_ERR_CUDA;
   }
   if (rc != MG_OK) {
      char keep[1024];
      strncpy (keep, g_err, sizeof (keep) - 1);
      keep[sizeof (keep) - 1] = 0;
      mg_run_destroy (r);
      mg_set_error ("%s", keep);
      return rc;
   }
   *out = r;
   return MG_OK;
}

static void free_snapshot (mg_run_t *r);

extern "C" int mg_run_destroy (mg_run_t *r)
{
   if (!r)
      return MG_OK;
   cudaSetDevice (r->device);
   if (r->stream)
      cudaStreamSynchronize (r->stream);
   mg_drop_graphs (r);
   if (r->pev) {
      for (int q = 0 ; q < 2*MG_PROFILE_CHUNK ; ++q)
         if (r->pev[q]) cudaEventDestroy (r->pev[q]);
      free (r->pev);
   }
   for (int c = 0 ; c < 3 ; ++c) {
      if (r->E[c]) mg_dev_free (r, r->E[c]);
      if (r->H[c]) mg_dev_free (r, r->H[c]);
      if (r->J[c]) mg_dev_free (r, r->J[c]);
      if (r->Hn[c]) mg_dev_free (r, r->Hn[c]);
      if (r->Ealt[c]) mg_dev_free (r, r->Ealt[c]);
      if (r->Halt[c]) mg_dev_free (r, r->Halt[c]);
      if (r->Ealt32[c]) mg_dev_free (r, r->Ealt32[c]);
      if (r->Halt32[c]) mg_dev_free (r, r->Halt32[c]);
      if (r->E32[c]) mg_dev_free (r, r->E32[c]);
      if (r->H32[c]) mg_dev_free (r, r->H32[c]);
      if (r->J32[c]) mg_dev_free (r, r->J32[c]);
      if (r->Hn32[c]) mg_dev_free (r, r->Hn32[c]);
   }
   for (int t = 0 ; t < 2 ; ++t)
      for (int a = 0 ; a < 3 ; ++a)
         if (r->mur[t][a]) mg_dev_free (r, r->mur[t][a]);
   for (int t = 0 ; t < 2 ; ++t)
      for (int a = 0 ; a < 3 ; ++a)
         if (r->mur32[t][a]) mg_dev_free (r, r->mur32[t][a]);
   free_markers (r);
   mg_free_markers32 (r);
   if (r->dsc) mg_dev_free (r, r->dsc);
   if (r->ring) mg_dev_free (r, r->ring);
   if (r->stage) mg_dev_free (r, r->stage);
   if (r->sort_tmp) mg_dev_free (r, r->sort_tmp);
   if (r->tile_start) mg_dev_free (r, r->tile_start);
   if (r->probe_ijk) mg_dev_free (r, r->probe_ijk);
   if (r->probe_ring) mg_dev_free (r, r->probe_ring);
   if (r->probe_ptrs) mg_dev_free (r, r->probe_ptrs);
   mg_tfsf_free (r);
   free_snapshot (r);
   for (int q = 0 ; q < r->nmirrors ; ++q) {
      mg_dev_free (r, r->mirrors[q].E);
      mg_dev_free (r, r->mirrors[q].H);
   }
   for (int q = 0 ; q < 2 ; ++q)
      if (r->gauss_rho[q]) mg_dev_free (r, r->gauss_rho[q]);
   if (r->gauss_out) mg_dev_free (r, r->gauss_out);
   for (int e = 0 ; e < 4 ; ++e)
      if (r->ev[e]) cudaEventDestroy (r->ev[e]);
   if (r->xfer) {
      cudaStreamSynchronize (r->xfer);
      for (int b = 0 ; b < 2 ; ++b)
         for (int e = 0 ; e < 2 ; ++e)
            if (r->xev[b][e]) cudaEventDestroy (r->xev[b][e]);
      cudaStreamDestroy (r->xfer);
   }
   if (r->stream) {
      cudaStreamSynchronize (r->stream);          // the frees above reach the pool
      cudaStreamDestroy (r->stream);
   }
   free (r);
   return MG_OK;
}

// ---------------------------------------------------------------------------
// Transfers.
// ---------------------------------------------------------------------------
extern "C" int mg_run_set_fields (mg_run_t *r, const double *E, const double *H)
{
   CHECK_RUN (r);
   if (r->prm.precision != MG_FP64) {
      return mg_run_set_fields32 (r, E, H);
   }
   const long vol = (long) (r->g.n[0] + 1)*(r->g.n[1] + 1)*(r->g.n[2] + 1);
   const size_t bytes = (size_t) vol*3*sizeof (double);
   const void *host[2];
   double **dst[2];
   size_t sizes[2] = {bytes, bytes};
   int nf = 0;
   if (E) { host[nf] = E; dst[nf++] = r->E; }
   if (H) { host[nf] = H; dst[nf++] = r->H; }
   TRY (pipelined_h2d (r, nf, bytes, [&] (int q, char *buf) {
      k_fields_in<<<mg_blocks_for (vol, 256, 8), 256, 0, r->stream>>> (r->g, (const double *) buf,
                                                                       dst[q][0], dst[q][1], dst[q][2]);
   }, host, sizes));
   MG_CUDA (cudaStreamSynchronize (r->stream));
   r->inited = 0;
   return MG_OK;
}

// E and H over the checkpoint region into E, H (host memory, or device
// memory when dev: converted in place, no copy, nothing waited for).
int mg_fields_out (mg_run_t *r, double *E, double *H, bool dev)
{
   if (r->prm.precision != MG_FP64)
      return mg_fields_out32 (r, E, H, dev);
   const long vol = (long) (r->g.n[0] + 1)*(r->g.n[1] + 1)*(r->g.n[2] + 1);
   const size_t bytes = (size_t) vol*3*sizeof (double);
   double *dst[2] = {E, H};
   // Between mg_em_HHalfStep and mg_em_HStep the reference's H is H^n.
   double **src[2] = {r->E, (r->stage_no >= 1 && r->stage_no <= 3) ? r->Hn : r->H};
   if (dev) {
      for (int f = 0 ; f < 2 ; ++f) {
         if (!dst[f])
            continue;
         k_fields_out<<<mg_blocks_for (vol, 256, 8), 256, 0, r->stream>>> (r->g, dst[f], src[f][0], src[f][1],
                                                                           src[f][2], 0);
         MG_LAUNCH_CHECK ();
      }
      return MG_OK;
   }
   void *host[2];
   double **from[2];
   size_t sizes[2] = {bytes, bytes};
   int nf = 0;
   for (int f = 0 ; f < 2 ; ++f)
      if (dst[f]) {
         host[nf] = dst[f];
         from[nf++] = src[f];
      }
   return pipelined_d2h (r, nf, bytes, [&] (int q, char *buf) {
      k_fields_out<<<mg_blocks_for (vol, 256, 8), 256, 0, r->stream>>> (r->g, (double *) buf, from[q][0],
                                                                        from[q][1], from[q][2], 0);
   }, host, sizes);
}

extern "C" int mg_run_get_fields (mg_run_t *r, double *E, double *H)
{
   CHECK_RUN (r);
   return mg_fields_out (r, E, H, false);
}

extern "C" int mg_run_get_current (mg_run_t *r, double *J)
{
   CHECK_RUN (r);
   if (r->prm.precision != MG_FP64) {
      return mg_run_get_current32 (r, J);
   }
   const long vol = (long) (r->g.n[0] + 5)*(r->g.n[1] + 5)*(r->g.n[2] + 5);
   const size_t bytes = (size_t) vol*3*sizeof (double);
   TRY (mg_ensure_stage (r, bytes));
   k_fields_out<<<mg_blocks_for (vol, 256, 8), 256, 0, r->stream>>> (r->g, (double *) r->stage,
                                                                     r->J[0], r->J[1], r->J[2], 2);
   MG_LAUNCH_CHECK ();
   MG_CUDA (cudaMemcpyAsync (J, r->stage, bytes, cudaMemcpyDeviceToHost, r->stream));
   MG_CUDA (cudaStreamSynchronize (r->stream));
   return MG_OK;
}

static const long long CHUNK = 1LL << 22;   // markers per staged transfer
static const long long XCHUNK = 1LL << 20;  // markers per half of a pipelined transfer (64 MB)

extern "C" int mg_run_set_markers (mg_run_t *r, const mg_marker_t *m, long long n)
{
   CHECK_RUN (r);
   if (n < 0 || (n > 0 && !m)) {
      mg_set_error ("mg_run_set_markers: bad arguments");
      return MG_ERR_ARG;
   }
   if (r->prm.precision != MG_FP64) {
      return mg_run_set_markers32 (r, m, n);
   }
   TRY (ensure_capacity (r, n));
   const int chunks = (int) ((n + XCHUNK - 1)/XCHUNK);
   std::vector<const void *> host (chunks);
   std::vector<size_t> sizes (chunks);
   for (int q = 0 ; q < chunks ; ++q) {
      const long long at = q*XCHUNK, c = (n - at < XCHUNK) ? n - at : XCHUNK;
      host[q] = m + at;
      sizes[q] = (size_t) c*sizeof (mg_marker_t);
   }
   TRY (pipelined_h2d (r, chunks, (size_t) XCHUNK*sizeof (mg_marker_t), [&] (int q, char *buf) {
      const long long c = (long long) (sizes[q]/sizeof (mg_marker_t));
      k_markers_in<<<mg_blocks_for (c, 256, 8), 256, 0, r->stream>>> ((const mg_marker_t *) buf, c, r->m64,
                                                                       q*XCHUNK);
   }, host.data (), sizes.data ()));
   r->np = n;
   r->tiles_ok = 0;
   MG_CUDA (cudaMemsetAsync (&r->dsc->dead, 0, sizeof (long long), r->stream));
   MG_CUDA (cudaStreamSynchronize (r->stream));
   return MG_OK;
}

extern "C" int mg_run_marker_count (mg_run_t *r, long long *n)
{
   CHECK_RUN (r);
   if (!n) {
      mg_set_error ("mg_run_marker_count: null output");
      return MG_ERR_ARG;
   }
   long long dead = 0;
   MG_CUDA (cudaMemcpyAsync (&dead, &r->dsc->dead, sizeof (dead), cudaMemcpyDeviceToHost, r->stream));
   MG_CUDA (cudaStreamSynchronize (r->stream));
   *n = r->np - dead;
   return MG_OK;
}

extern "C" int mg_run_get_markers (mg_run_t *r, mg_marker_t *out, long long cap, long long *n)
{
   CHECK_RUN (r);
   return mg_markers_out (r, out, cap, n, false);
}

// The live markers, compacted, into out (host memory, or device memory when
// dev).
int mg_markers_out (mg_run_t *r, mg_marker_t *out, long long cap, long long *n, bool dev)
{
   if (r->prm.precision != MG_FP64)
      return mg_markers_out32 (r, out, cap, n, dev);
   long long live = 0;
   TRY (mg_run_marker_count (r, &live));
   if (n)
      *n = live;
   if (!out)
      return MG_OK;
   if (cap < live) {
      mg_set_error ("mg_run_get_markers: buffer holds %lld markers, %lld live", cap, live);
      return MG_ERR_CAPACITY;
   }
   if (live == r->np && !dev) {
      // No marker removed: nothing to compact, chunks go straight through
      // the pipelined copy.
      const int chunks = (int) ((r->np + XCHUNK - 1)/XCHUNK);
      std::vector<void *> host (chunks);
      std::vector<size_t> sizes (chunks);
      for (int q = 0 ; q < chunks ; ++q) {
         const long long at = q*XCHUNK, c = (r->np - at < XCHUNK) ? r->np - at : XCHUNK;
         host[q] = out + at;
         sizes[q] = (size_t) c*sizeof (mg_marker_t);
      }
      return pipelined_d2h (r, chunks, (size_t) XCHUNK*sizeof (mg_marker_t), [&] (int q, char *buf) {
         const long long c = (long long) (sizes[q]/sizeof (mg_marker_t));
         k_markers_out<<<mg_blocks_for (c, 256, 8), 256, 0, r->stream>>> (r->m64, q*XCHUNK, c,
                                                                         (mg_marker_t *) buf, nullptr);
      }, host.data (), sizes.data ());
   }
   const long long chunk = r->np < CHUNK ? r->np : CHUNK;
   const size_t need = (size_t) (chunk > 0 ? chunk : 1)*(sizeof (mg_marker_t) + sizeof (long long)) + 64;
   TRY (mg_ensure_stage (r, need));
   mg_marker_t *dst = (mg_marker_t *) r->stage;
   long long *slot = (long long *) ((char *) r->stage + (size_t) (chunk > 0 ? chunk : 1)*sizeof (mg_marker_t));
   long long *total_d = slot + (chunk > 0 ? chunk : 1);
   long long written = 0;
   for (long long at = 0 ; at < r->np ; at += CHUNK) {
      const long long c = (r->np - at < CHUNK) ? r->np - at : CHUNK;
      k_live_scan<<<1, 1024, 0, r->stream>>> (r->m64.qm, at, c, slot, total_d);
      k_markers_out<<<mg_blocks_for (c, 256, 8), 256, 0, r->stream>>> (r->m64, at, c, dst, slot);
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

// ---------------------------------------------------------------------------
// Asynchronous snapshot: the checkpoint state (fields over [0, n]^3 and the
// live markers, compacted) is converted into device buffers of the run on
// its own stream -- a step boundary -- and copied to the caller's host
// buffers on a second stream, so that later steps run while it travels.
// ---------------------------------------------------------------------------
static void free_snapshot (mg_run_t *r)
{
   if (r->snap_pending && r->snap_done)
      cudaEventSynchronize (r->snap_done);
   r->snap_pending = 0;
   if (r->snap_E) mg_dev_free (r, r->snap_E);
   if (r->snap_H) mg_dev_free (r, r->snap_H);
   if (r->snap_m) mg_dev_free (r, r->snap_m);
   r->snap_E = r->snap_H = nullptr;
   r->snap_m = nullptr;
   r->snap_cap = 0;
   if (r->snap_ready) cudaEventDestroy (r->snap_ready);
   if (r->snap_done) cudaEventDestroy (r->snap_done);
   if (r->snap_stream) cudaStreamDestroy (r->snap_stream);
   r->snap_ready = r->snap_done = nullptr;
   r->snap_stream = nullptr;
}

extern "C" int mg_run_snapshot_wait (mg_run_t *r)
{
   CHECK_RUN (r);
   if (!r->snap_pending)
      return MG_OK;
   MG_CUDA (cudaEventSynchronize (r->snap_done));
   r->snap_pending = 0;
   return MG_OK;
}

extern "C" int mg_run_snapshot (mg_run_t *r, double *E, double *H, mg_marker_t *m, long long cap,
                                long long *n)
{
   CHECK_RUN (r);
   TRY (mg_run_snapshot_wait (r));
   if (r->stage_no != 0) {
      mg_set_error ("mg_run_snapshot: a stage-by-stage step is in progress");
      return MG_ERR_STATE;
   }
   long long live = 0;
   TRY (mg_run_marker_count (r, &live));
   if (m && cap < live) {
      mg_set_error ("mg_run_snapshot: buffer holds %lld markers, %lld live", cap, live);
      return MG_ERR_CAPACITY;
   }
   const long vol = (long) (r->g.n[0] + 1)*(r->g.n[1] + 1)*(r->g.n[2] + 1);
   const size_t fbytes = (size_t) vol*3*sizeof (double);
   if (!r->snap_stream) {
      MG_CUDA (cudaStreamCreateWithFlags (&r->snap_stream, cudaStreamNonBlocking));
      MG_CUDA (cudaEventCreateWithFlags (&r->snap_ready, cudaEventDisableTiming));
      MG_CUDA (cudaEventCreateWithFlags (&r->snap_done, cudaEventDisableTiming));
   }
   if (!r->snap_E) {
      TRY (mg_dev_alloc (r, (void **) &r->snap_E, fbytes));
      TRY (mg_dev_alloc (r, (void **) &r->snap_H, fbytes));
   }
   if (m && live > r->snap_cap) {
      if (r->snap_m) {
         mg_dev_free (r, r->snap_m);
         r->dev_bytes -= (long long) r->snap_cap*sizeof (mg_marker_t);
         r->snap_m = nullptr;
         r->snap_cap = 0;
      }
      const long long c = live + live/8 + 1024;
      TRY (mg_dev_alloc (r, (void **) &r->snap_m, (size_t) c*sizeof (mg_marker_t)));
      r->snap_cap = c;
   }
   TRY (mg_fields_out (r, E ? r->snap_E : nullptr, H ? r->snap_H : nullptr, true));
   long long got = 0;
   if (m)
      TRY (mg_markers_out (r, r->snap_m, r->snap_cap, &got, true));
   MG_CUDA (cudaEventRecord (r->snap_ready, r->stream));
   MG_CUDA (cudaStreamWaitEvent (r->snap_stream, r->snap_ready, 0));
   if (E) MG_CUDA (cudaMemcpyAsync (E, r->snap_E, fbytes, cudaMemcpyDeviceToHost, r->snap_stream));
   if (H) MG_CUDA (cudaMemcpyAsync (H, r->snap_H, fbytes, cudaMemcpyDeviceToHost, r->snap_stream));
   if (m && got > 0)
      MG_CUDA (cudaMemcpyAsync (m, r->snap_m, (size_t) got*sizeof (mg_marker_t), cudaMemcpyDeviceToHost,
                                r->snap_stream));
   MG_CUDA (cudaEventRecord (r->snap_done, r->snap_stream));
   r->snap_pending = 1;
   if (n)
      *n = got;
   return MG_OK;
}

// ---------------------------------------------------------------------------
// Focused-laser mirrors (scpic/em_mirror.c, scpic/em_sources.c).
// ---------------------------------------------------------------------------
extern "C" int mg_run_add_mirror (mg_run_t *r, const mg_mirror_t *s)
{
   CHECK_RUN (r);
   if (!s || !s->E || !s->H || !(s->r0 > 0) || !(s->t0 > 0) || !(s->values[5] > 0)) {
      mg_set_error ("mg_run_add_mirror: need the profiles, units and a positive duration");
      return MG_ERR_ARG;
   }
   if (r->nmirrors >= MG_MIRRORS) {
      mg_set_error ("mg_run_add_mirror: at most %d mirrors", MG_MIRRORS);
      return MG_ERR_ARG;
   }
   if (r->g.n[1] < 10 || r->g.n[2] < 10) {
      mg_set_error ("mg_run_add_mirror: the source plane needs at least 10 cells along y and z");
      return MG_ERR_ARG;
   }
   // read_mirror_parameters (scpic/em_mirror.c:292-332), the values the play
   // needs; the backward delay subtracts the focus from the cell count, as
   // the reference does (:330).
   const double pi = 3.141592653589793238462643;
   const double e = 4.8032e-10, c = 2.9979e+10, m = 9.1094e-28, wpc = 1e7;   // misc_units.h:34-38
   const double *v = s->values;
   double A = v[0];
   if (A > 0)
      A = s->r0*e*sqrt (8*pi*A*wpc/c)/(m*c*c);
   else
      A *= (-2*pi);
   const double xf = v[2]*1e-4/s->r0;
   double dt = v[5]*1e-15/s->t0;
   const double T0 = v[6]*1e-15/s->t0;
   dt *= sqrt (2.0/log (2));
   MirrorDev d;
   d.A = A;
   d.dt = dt;
   d.T0 = T0;
   d.phi0 = v[7];
   d.forward = s->direction > 0;
   d.delay = d.forward ? xf - 5*r->g.h[0] : r->g.n[0] - 5*r->g.h[0] - xf;
   const size_t bytes = sizeof (double)*4*(size_t) (r->g.n[1] - 9)*(r->g.n[2] - 9);
   d.E = d.H = nullptr;
   TRY (mg_dev_alloc (r, (void **) &d.E, bytes));
   TRY (mg_dev_alloc (r, (void **) &d.H, bytes));
   MG_CUDA (cudaMemcpy (d.E, s->E, bytes, cudaMemcpyHostToDevice));
   MG_CUDA (cudaMemcpy (d.H, s->H, bytes, cudaMemcpyHostToDevice));
   r->mirrors[r->nmirrors++] = d;
   mg_drop_graphs (r);
   return MG_OK;
}

extern "C" int mg_run_clear_mirrors (mg_run_t *r)
{
   CHECK_RUN (r);
   for (int q = 0 ; q < r->nmirrors ; ++q) {
      mg_dev_free (r, r->mirrors[q].E);
      mg_dev_free (r, r->mirrors[q].H);
   }
   r->nmirrors = 0;
   mg_drop_graphs (r);
   return MG_OK;
}

extern "C" void *mg_host_alloc (size_t bytes)
{
   void *p = nullptr;
   if (cudaMallocHost (&p, bytes ? bytes : 1) != cudaSuccess) {
      mg_set_error ("mg_host_alloc: %zu bytes of pinned memory not available", bytes);
      return nullptr;
   }
   return p;
}

extern "C" void mg_host_free (void *p)
{
   if (p)
      cudaFreeHost (p);
}

extern "C" int mg_run_set_gauss_spot (mg_run_t *r, const mg_gauss_spot_t *s)
{
   CHECK_RUN (r);
   if (!s) {
      r->has_gspot = 0;
   } else {
      if (!(s->width > 0) || !(s->duration > 0)) {
         mg_set_error ("mg_run_set_gauss_spot: width %g and duration %g must be positive", s->width, s->duration);
         return MG_ERR_ARG;
      }
      GaussSpot &g = r->gspot;
      g.ey = ((s->ey > 0) - (s->ey < 0))*s->ampl;        // em_gaussSpot.c:70-71, 121-122
      g.ez = ((s->ez > 0) - (s->ez < 0))*s->ampl;
      g.omega = 2*3.14159265358979323846*s->frequency;   // em_gaussSpot.c:48
      g.y = s->y;
      g.z = s->z;
      g.width = s->width;
      g.duration = s->duration;
      g.front = s->front_offset;
      g.plateau = s->t_plateau;
      g.i = (int) (s->x/r->g.h[0] + 0.5);                  // em_gaussSpot.c:73
      r->has_gspot = 1;
   }
   mg_drop_graphs (r);
   return MG_OK;
}

extern "C" int mg_run_set_laser (mg_run_t *r, const mg_laser_t *l)
{
   CHECK_RUN (r);
   if (!l) {
      r->has_laser = 0;
   } else {
      // The E plane (plane - 1) and the transverse range must stay clear of
      // the two rim layers next to every wall: plane in [3, n-1], margin >= 2.
      if (l->plane < 3 || l->plane > r->g.n[0] - 1 || l->margin < 2 || !(l->waist > 0) ||
          !(l->duration > 0)) {
         mg_set_error ("mg_run_set_laser: plane %d (allowed 3..%d) / margin %d (>= 2) / waist %g / "
                       "duration %g out of range", l->plane, r->g.n[0] - 1, l->margin, l->waist,
                       l->duration);
         return MG_ERR_ARG;
      }
      r->laser = *l;
      r->has_laser = 1;
   }
   mg_drop_graphs (r);
   return MG_OK;
}

extern "C" int mg_run_set_time (mg_run_t *r, double t)
{
   CHECK_RUN (r);
   r->time = t;
   MG_CUDA (cudaMemcpyAsync (&r->dsc->time, &r->time, sizeof (double), cudaMemcpyHostToDevice, r->stream));
   MG_CUDA (cudaStreamSynchronize (r->stream));
   return MG_OK;
}

extern "C" int mg_run_get_time (mg_run_t *r, double *t)
{
   CHECK_RUN (r);
   MG_CUDA (cudaMemcpyAsync (&r->time, &r->dsc->time, sizeof (double), cudaMemcpyDeviceToHost, r->stream));
   MG_CUDA (cudaStreamSynchronize (r->stream));
   if (t)
      *t = r->time;
   return MG_OK;
}

// ---------------------------------------------------------------------------
// Stage API (core/main.c:353-478).  The order is checked like the
// reference's emStage flag (core/em.c:32).
// ---------------------------------------------------------------------------
static int expect_stage (mg_run_t *r, int want, const char *who)
{
   if (!r->inited) {
      mg_set_error ("%s: mg_run_init has not been called since the state was loaded", who);
      return MG_ERR_STATE;
   }
   if (r->stage_no != want) {
      mg_set_error ("%s: called at stage %d, expected stage %d", who, r->stage_no, want);
      return MG_ERR_STATE;
   }
   return MG_OK;
}

static bool is32 (const mg_run_t *r) { return r->prm.precision == MG_FP32_OFFSET; }

int mg_walls64 (mg_run_t *r);
int mg_walls32 (mg_run_t *r);

extern "C" int mg_run_init (mg_run_t *r)
{
   CHECK_RUN (r);
   TRY (is32 (r) ? mg_fields32_init (r) : mg_fields64_init (r));
   TRY (is32 (r) ? mg_walls32 (r) : mg_walls64 (r));
   if (is32 (r)) {
      // Order the markers by tile before the first step; the step graph
      // takes the tiled push only while that order is known.  sort_every < 0
      // keeps the upload order and the untiled push.
      mg_drop_graphs (r);
      if (r->prm.sort_every >= 0)
         TRY (mg_sort32 (r));
   } else if (r->prm.sort_every >= 0) {
      TRY (mg_sort64 (r));        // cell order for the gather's locality
   }
   MG_CUDA (cudaStreamSynchronize (r->stream));
   r->inited = 1;
   r->stage_no = 0;
   return MG_OK;
}

extern "C" int mg_em_HHalfStep (mg_run_t *r)
{
   CHECK_RUN (r);
   TRY (expect_stage (r, 0, __func__));
   // A stage-by-stage step keeps its probe samples and TF/SF record in row 0.
   if (r->nprobes > 0 || mg_tfsf_recording (r))
      MG_CUDA (cudaMemsetAsync (&r->dsc->step, 0, sizeof (int), r->stream));
   TRY (mg_tfsf_record (r));
   TRY (is32 (r) ? mg_fields32_h_half (r) : mg_fields64_h_half (r));
   // Probe samples (core/main.c:373 samples after em_energy; nothing in
   // between changes E or H^n).
   TRY (mg_probes_enqueue (r));
   r->stage_no = 1;
   return MG_OK;
}

extern "C" int mg_em_energy (mg_run_t *r, double *we, double *wm)
{
   CHECK_RUN (r);
   TRY (expect_stage (r, 1, __func__));
   TRY (is32 (r) ? mg_fields32_energy (r) : mg_fields64_energy (r));
   double acc[2];
   MG_CUDA (cudaMemcpyAsync (acc, r->dsc->acc, sizeof (acc), cudaMemcpyDeviceToHost, r->stream));
   MG_CUDA (cudaStreamSynchronize (r->stream));
   const double v = r->g.h[0]*r->g.h[1]*r->g.h[2];
   if (we) *we = 0.5*acc[0]*v;
   if (wm) *wm = 0.5*acc[1]*v;
   r->stage_no = 2;
   return MG_OK;
}

static int check_err (mg_run_t *r)
{
   int info[5];
   MG_CUDA (cudaMemcpyAsync (info, &r->dsc->err, sizeof (int)*5, cudaMemcpyDeviceToHost, r->stream));
   MG_CUDA (cudaStreamSynchronize (r->stream));
   if (info[0] & 4) {
      mg_set_error ("TF/SF frame %d is not on the device (mg_run_tfsf_put_frames)", info[1]);
      return MG_ERR_STATE;
   }
   if (info[0] & 8) {
      mg_set_error ("the tiled push gave up waiting for the TMA copy of a field tile (bounded wait); "
                    "the step is invalid");
      return MG_ERR_TIMEOUT;
   }
   if (info[0]) {
      mg_set_error ("marker %d left the mesh or moved more than one cell per step "
                    "(flags %d, cell %d %d %d); the step is invalid", info[1], info[0], info[2], info[3], info[4]);
      return MG_ERR_BOUNDS;
   }
   return MG_OK;
}

extern "C" int mg_plasma_move (mg_run_t *r)
{
   CHECK_RUN (r);
   if (r->stage_no == 1)
      r->stage_no = 2;       // the energy stage is optional
   TRY (expect_stage (r, 2, __func__));
   MG_CUDA (cudaMemsetAsync (r->dsc->acc + 2, 0, 3*sizeof (double), r->stream));
   TRY (is32 (r) ? mg_fields32_zero_j (r) : mg_fields64_zero_j (r));
   TRY (is32 (r) ? mg_push32 (r) : mg_push64 (r));
   TRY (check_err (r));
   r->stage_no = 3;
   return MG_OK;
}

extern "C" int mg_plasma_temperature (mg_run_t *r, double *wx, double *wy, double *wz)
{
   CHECK_RUN (r);
   double acc[3];
   MG_CUDA (cudaMemcpyAsync (acc, r->dsc->acc + 2, sizeof (acc), cudaMemcpyDeviceToHost, r->stream));
   MG_CUDA (cudaStreamSynchronize (r->stream));
   if (wx) *wx = acc[0];
   if (wy) *wy = acc[1];
   if (wz) *wz = acc[2];
   return MG_OK;
}

extern "C" int mg_em_HStep (mg_run_t *r)
{
   CHECK_RUN (r);
   TRY (expect_stage (r, 3, __func__));
   TRY (is32 (r) ? mg_fields32_h_step (r) : mg_fields64_h_step (r));
   r->stage_no = 4;
   return MG_OK;
}

extern "C" int mg_em_EStep_start (mg_run_t *r)
{
   CHECK_RUN (r);
   TRY (expect_stage (r, 4, __func__));
   TRY (is32 (r) ? mg_fields32_e_step (r) : mg_fields64_e_step (r));
   r->stage_no = 5;
   return MG_OK;
}

extern "C" int mg_jbc_finish (mg_run_t *r)
{
   CHECK_RUN (r);
   TRY (expect_stage (r, 5, __func__));
   TRY (is32 (r) ? mg_fields32_jbc (r) : mg_fields64_jbc (r));
   r->stage_no = 6;
   return MG_OK;
}

extern "C" int mg_em_EStep_finish (mg_run_t *r)
{
   CHECK_RUN (r);
   TRY (expect_stage (r, 6, __func__));
   TRY (is32 (r) ? mg_fields32_e_finish (r) : mg_fields64_e_finish (r));
   // Time advances at the end of the step (core/main.c:435).
   k_end_step<<<1, 1, 0, r->stream>>> (r->dsc, r->ring, r->g.h[0]*r->g.h[1]*r->g.h[2], r->g.tau);
   MG_LAUNCH_CHECK ();
   MG_CUDA (cudaStreamSynchronize (r->stream));
   r->time += r->g.tau;
   r->stage_no = 0;
   return MG_OK;
}

// Device buffers of the Gauss-law test: two densities and the residuals.
static int ensure_gauss (mg_run_t *r)
{
   if (r->gauss_rho[0])
      return MG_OK;
   const size_t fb = (size_t) r->g.total*sizeof (double);
   TRY (mg_dev_alloc (r, (void **) &r->gauss_rho[0], fb));
   TRY (mg_dev_alloc (r, (void **) &r->gauss_rho[1], fb));
   TRY (mg_dev_alloc (r, (void **) &r->gauss_out, 2*sizeof (double)));
   return MG_OK;
}

extern "C" int mg_plasma_rho (mg_run_t *r, double *rho)
{
   CHECK_RUN (r);
   TRY (ensure_gauss (r));
   double *d = r->gauss_rho[1];
   TRY (mg_gauss_rho (r, d));
   const long vol = (long) (r->g.n[0] + 5)*(r->g.n[1] + 5)*(r->g.n[2] + 5);
   TRY (mg_ensure_stage (r, vol*3*sizeof (double)));
   k_fields_out<<<mg_blocks_for (vol, 256, 8), 256, 0, r->stream>>> (r->g, (double *) r->stage, d, d, d, 2);
   MG_LAUNCH_CHECK ();
   // Take one component of the triplets on the host.
   double *tmp = (double *) malloc (vol*3*sizeof (double));
   MG_CUDA (cudaMemcpyAsync (tmp, r->stage, vol*3*sizeof (double), cudaMemcpyDeviceToHost, r->stream));
   MG_CUDA (cudaStreamSynchronize (r->stream));
   for (long t = 0 ; t < vol ; ++t)
      rho[t] = tmp[3*t];
   free (tmp);
   return MG_OK;
}

// ---------------------------------------------------------------------------
// Gauss-law test (core/plasma_gaussTest.c:89-149).
// ---------------------------------------------------------------------------
extern "C" int mg_gauss_before (mg_run_t *r)
{
   CHECK_RUN (r);
   TRY (ensure_gauss (r));
   TRY (mg_gauss_rho (r, r->gauss_rho[0]));
   MG_CUDA (cudaStreamSynchronize (r->stream));
   return MG_OK;
}

extern "C" int mg_gauss_after (mg_run_t *r, double out[2])
{
   CHECK_RUN (r);
   if (!r->gauss_rho[0]) {
      mg_set_error ("mg_gauss_after: mg_gauss_before has not been called");
      return MG_ERR_STATE;
   }
   TRY (mg_gauss_rho (r, r->gauss_rho[1]));
   TRY (mg_gauss_residual (r, r->gauss_rho[0], r->gauss_rho[1], r->gauss_out));
   double res[2];
   MG_CUDA (cudaMemcpyAsync (res, r->gauss_out, sizeof (res), cudaMemcpyDeviceToHost, r->stream));
   MG_CUDA (cudaStreamSynchronize (r->stream));
   if (out) {
      out[0] = res[0];
      out[1] = res[1];
   }
   return MG_OK;
}

// ---------------------------------------------------------------------------
// Whole steps.
// ---------------------------------------------------------------------------
// One step as three parts: fields before the push, the push, and the rest
// (core/main.c:353-478 order).  part < 0 enqueues all three.
int mg_enqueue_step64 (mg_run_t *r, int part)
{
   if (part < 0 && r->fo_graph) {        // field-only: one pass into Ealt, Halt
      TRY (mg_fields64_one_pass (r));
      k_end_step<<<1, 1, 0, r->stream>>> (r->dsc, r->ring, r->g.h[0]*r->g.h[1]*r->g.h[2], r->g.tau);
      MG_LAUNCH_CHECK ();
      return MG_OK;
   }
   if (part < 0 || part == 0) {
      TRY (mg_tfsf_record (r));
      TRY (mg_fields64_h_both (r));
      TRY (mg_probes_enqueue (r));
      if (r->np > 0)                       // without markers J stays zero
         TRY (mg_fields64_zero_j (r));
   }
   if (part < 0 || part == 1)
      TRY (mg_push64 (r));
   if (part < 0 || part == 2) {
      if (r->np > 0)
         TRY (mg_fields64_jbc_graph (r));
      TRY (mg_fields64_e_fused (r));
      k_end_step<<<1, 1, 0, r->stream>>> (r->dsc, r->ring, r->g.h[0]*r->g.h[1]*r->g.h[2], r->g.tau);
      MG_LAUNCH_CHECK ();
   }
   return MG_OK;
}

int mg_enqueue_step32 (mg_run_t *r, int part);

int mg_end_step (mg_run_t *r)
{
   k_end_step<<<1, 1, 0, r->stream>>> (r->dsc, r->ring, r->g.h[0]*r->g.h[1]*r->g.h[2], r->g.tau);
   MG_LAUNCH_CHECK ();
   return MG_OK;
}

static int count_kernels (cudaGraph_t graph)
{
   size_t n = 0;
   if (cudaGraphGetNodes (graph, nullptr, &n) != cudaSuccess)
      return 0;
   cudaGraphNode_t *nodes = (cudaGraphNode_t *) malloc (n*sizeof (cudaGraphNode_t));
   cudaGraphGetNodes (graph, nodes, &n);
   int k = 0;
   for (size_t q = 0 ; q < n ; ++q) {
      cudaGraphNodeType t;
      if (cudaGraphNodeGetType (nodes[q], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel)
         ++k;
   }
   free (nodes);
   return k;
}

void mg_drop_graphs (mg_run_t *r)
{
   for (int q = 0 ; q < 5 ; ++q) {
      if (r->gexec[q]) cudaGraphExecDestroy (r->gexec[q]);
      if (r->gr[q]) cudaGraphDestroy (r->gr[q]);
      r->gexec[q] = nullptr;
      r->gr[q] = nullptr;
   }
   r->graph_ok = 0;
   r->fo_graph = 0;
}

// A run stepped alone without markers, sources, probes or TF/SF takes the
// one-pass field step (both precisions).
static bool one_pass_ok (const mg_run_t *r)
{
   return r->np == 0 && !r->probe_ring && !r->has_laser && !r->has_gspot &&
          r->nmirrors == 0 && !r->tfsf && !r->in_batch;
}

template <typename T>
static void swap3 (T *a[3], T *b[3])
{
   for (int c = 0 ; c < 3 ; ++c) {
      T *t = a[c];
      a[c] = b[c];
      b[c] = t;
   }
}

static void swap_field_sets (mg_run_t *r)
{
   if (is32 (r)) {
      swap3 (r->E32, r->Ealt32);
      swap3 (r->H32, r->Halt32);
   } else {
      swap3 (r->E, r->Ealt);
      swap3 (r->H, r->Halt);
   }
}

static const void *field_set_id (const mg_run_t *r)
{
   return is32 (r) ? (const void *) r->E32[0] : (const void *) r->E[0];
}

// The second E and H arrays, equal to the current ones (nodes no step
// writes, the outer ghosts, must match in both sets).
template <typename T>
static int make_alt_set (mg_run_t *r, T *const E[3], T *const H[3], T *Ea[3], T *Ha[3])
{
   const size_t bytes = (size_t) r->g.total*sizeof (T);
   for (int c = 0 ; c < 3 ; ++c) {
      if (!Ea[c]) TRY (mg_dev_alloc (r, (void **) &Ea[c], bytes));
      if (!Ha[c]) TRY (mg_dev_alloc (r, (void **) &Ha[c], bytes));
      MG_CUDA (cudaMemcpyAsync (Ea[c], E[c], bytes, cudaMemcpyDeviceToDevice, r->stream));
      MG_CUDA (cudaMemcpyAsync (Ha[c], H[c], bytes, cudaMemcpyDeviceToDevice, r->stream));
   }
   return MG_OK;
}

// Graph 0: the whole step; graphs 1..3: its three parts (profiling mode, so
// that events can bracket the push on the run's stream).
static int build_graph (mg_run_t *r)
{
   if (r->graph_ok)
      return MG_OK;
   mg_drop_graphs (r);
   // A step graph without markers neither clears nor folds J and leaves
   // -tau J out of the E update: clear J once here.
   if (r->np == 0)
      for (int c = 0 ; c < 3 ; ++c) {
         void *J = is32 (r) ? (void *) r->J32[c] : (void *) r->J[c];
         const size_t elt = is32 (r) ? sizeof (float) : sizeof (double);
         MG_CUDA (cudaMemsetAsync (J, 0, (size_t) r->g.total*elt, r->stream));
      }
   // A plain-form run without markers, sources, probes or TF/SF steps its
   // fields in one pass between two sets of E and H arrays: graph 0 reads
   // the arrays current now and writes the others, graph 4 the reverse.
   r->fo_graph = one_pass_ok (r);
   if (r->fo_graph) {
      if (is32 (r))
         TRY (make_alt_set<float> (r, r->E32, r->H32, r->Ealt32, r->Halt32));
      else
         TRY (make_alt_set<double> (r, r->E, r->H, r->Ealt, r->Halt));
      r->fo_read0 = field_set_id (r);
   }
   for (int q = 0 ; q < (r->fo_graph ? 5 : 4) ; ++q) {
      if (q == 4)
         swap_field_sets (r);
      MG_CUDA (cudaStreamBeginCapture (r->stream, cudaStreamCaptureModeThreadLocal));
      const int part = q == 4 ? -1 : q - 1;
      int rc = is32 (r) ? mg_enqueue_step32 (r, part) : mg_enqueue_step64 (r, part);
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamEndCapture (r->stream, &g);
      if (q == 4)
         swap_field_sets (r);
      if (rc != MG_OK) {
         if (g) cudaGraphDestroy (g);
         return rc;
      }
      if (e != cudaSuccess) {
         mg_set_error ("graph capture failed: %s", cudaGetErrorString (e));
         return MG_ERR_CUDA;
      }
      r->gr[q] = g;
      MG_CUDA (cudaGraphInstantiate (&r->gexec[q], g, 0));
   }
   r->kernels_per_step = count_kernels (r->gr[0]);
   r->graph_ok = 1;
   return MG_OK;
}

// One whole step from its graph; the one-pass field-only pair alternates
// with the field arrays it writes.
static int launch_step_graph (mg_run_t *r)
{
   if (!r->fo_graph) {
      MG_CUDA (cudaGraphLaunch (r->gexec[0], r->stream));
      return MG_OK;
   }
   MG_CUDA (cudaGraphLaunch (field_set_id (r) == r->fo_read0 ? r->gexec[0] : r->gexec[4], r->stream));
   swap_field_sets (r);
   return MG_OK;
}

// Precision form: markers are re-sorted by tile and cell every sort_every
// steps (default 16) so that tiles stay compact and warps keep sharing cells;
// the sort runs between graph launches on the run's stream.
// The plain form is put in cell order every sort_every steps (default 24)
// for the gather's locality (mg_sort64): over the 2000-step laser-foil run
// the step takes 0.664, 0.644, 0.636, 0.634, 0.634 ms sorting every 8, 16,
// 24, 32, 48 steps (the push 0.362, 0.367, 0.371, 0.374, 0.380 ms).
static int maybe_sort (mg_run_t *r)
{
   if (r->prm.sort_every < 0)
      return MG_OK;
   const int every = r->prm.sort_every > 0 ? r->prm.sort_every : is32 (r) ? 16 : 24;
   if (r->steps_since_sort++ < every)
      return MG_OK;
   return is32 (r) ? mg_sort32 (r) : mg_sort64 (r);
}

static int run_steps (mg_run_t *r, int nsteps, double *host_rows, double *dev_rows, bool sync)
{
   if (!r->inited) {
      mg_set_error ("mg_run_step: mg_run_init has not been called since the state was loaded");
      return MG_ERR_STATE;
   }
   if (r->stage_no != 0) {
      mg_set_error ("mg_run_step: a stage-by-stage step is in progress (stage %d)", r->stage_no);
      return MG_ERR_STATE;
   }
   if (nsteps < 0) {
      mg_set_error ("mg_run_step: nsteps = %d", nsteps);
      return MG_ERR_ARG;
   }
   if (r->in_batch) {                     // stepped alone again
      mg_drop_graphs (r);
      r->in_batch = 0;
   }
   TRY (build_graph (r));
   if (r->profile && r->fo_graph && field_set_id (r) != r->fo_read0) {
      // The part graphs step the set they were captured on and do not
      // swap: capture them again on the current set.
      mg_drop_graphs (r);
      TRY (build_graph (r));
   }
   double push_sum = 0, step_sum = 0;
   for (int done = 0 ; done < nsteps ; ) {
      int chunk = (nsteps - done < MG_RING) ? nsteps - done : MG_RING;
      if (r->profile && chunk > MG_PROFILE_CHUNK)
         chunk = MG_PROFILE_CHUNK;
      MG_CUDA (cudaMemsetAsync (&r->dsc->step, 0, sizeof (int), r->stream));
      if (r->profile) {
         MG_CUDA (cudaEventRecord (r->ev[0], r->stream));
         for (int s = 0 ; s < chunk ; ++s) {
            TRY (maybe_sort (r));
            MG_CUDA (cudaGraphLaunch (r->gexec[1], r->stream));
            MG_CUDA (cudaEventRecord (r->pev[2*s], r->stream));
            MG_CUDA (cudaGraphLaunch (r->gexec[2], r->stream));
            MG_CUDA (cudaEventRecord (r->pev[2*s + 1], r->stream));
            MG_CUDA (cudaGraphLaunch (r->gexec[3], r->stream));
         }
         MG_CUDA (cudaEventRecord (r->ev[1], r->stream));
      } else {
         for (int s = 0 ; s < chunk ; ++s) {
            TRY (maybe_sort (r));
            TRY (launch_step_graph (r));
         }
      }
      if (host_rows)
         MG_CUDA (cudaMemcpyAsync (host_rows + 6*(size_t) done, r->ring, sizeof (double)*6*chunk,
                                   cudaMemcpyDeviceToHost, r->stream));
      if (dev_rows)
         MG_CUDA (cudaMemcpyAsync (dev_rows + 6*(size_t) done, r->ring, sizeof (double)*6*chunk,
                                   cudaMemcpyDeviceToDevice, r->stream));
      done += chunk;
      if (host_rows || sync || r->profile || done < nsteps)
         MG_CUDA (cudaStreamSynchronize (r->stream));
      if (r->profile) {
         float ms = 0;
         for (int s = 0 ; s < chunk ; ++s) {
            cudaEventElapsedTime (&ms, r->pev[2*s], r->pev[2*s + 1]);
            push_sum += ms;
         }
         cudaEventElapsedTime (&ms, r->ev[0], r->ev[1]);
         step_sum += ms;
      }
   }
   if (r->profile && nsteps > 0) {
      r->last_push_ms = push_sum/nsteps;
      r->last_step_ms = step_sum/nsteps;
   }
   r->time += nsteps*r->g.tau;
   if (sync)
      TRY (check_err (r));
   return MG_OK;
}

extern "C" int mg_run_step (mg_run_t *r, int nsteps, double *energies)
{
   CHECK_RUN (r);
   return run_steps (r, nsteps, energies, nullptr, true);
}

extern "C" int mg_run_step_async (mg_run_t *r, int nsteps, double *energies_dev)
{
   CHECK_RUN (r);
   return run_steps (r, nsteps, nullptr, energies_dev, false);
}

// ---------------------------------------------------------------------------
// Batches: one graph launch steps every run of the batch.
// ---------------------------------------------------------------------------
struct mg_batch {
   int              n;
   mg_run_t       **runs;
   int              device;
   cudaStream_t     stream;
   cudaGraph_t      graph;
   cudaGraphExec_t  exec;
};

extern "C" int mg_batch_destroy (mg_batch_t *b)
{
   if (!b)
      return MG_OK;
   cudaSetDevice (b->device);
   if (b->stream)
      cudaStreamSynchronize (b->stream);
   if (b->exec) cudaGraphExecDestroy (b->exec);
   if (b->graph) cudaGraphDestroy (b->graph);
   if (b->stream) cudaStreamDestroy (b->stream);
   free (b->runs);
   free (b);
   return MG_OK;
}

extern "C" int mg_batch_create (mg_run_t *const *runs, int n, mg_batch_t **out)
{
   if (!runs || n <= 0 || !out) {
      mg_set_error ("mg_batch_create: need at least one run");
      return MG_ERR_ARG;
   }
   *out = nullptr;
   for (int q = 0 ; q < n ; ++q) {
      if (!runs[q]) {
         mg_set_error ("mg_batch_create: run %d is null", q);
         return MG_ERR_ARG;
      }
      if (runs[q]->device != runs[0]->device) {
         mg_set_error ("mg_batch_create: runs on devices %d and %d", runs[0]->device, runs[q]->device);
         return MG_ERR_ARG;
      }
      if (!runs[q]->inited || runs[q]->stage_no != 0) {
         mg_set_error ("mg_batch_create: run %d is not initialised or is inside a staged step", q);
         return MG_ERR_STATE;
      }
   }
   MG_CUDA (cudaSetDevice (runs[0]->device));
   mg_batch_t *b = (mg_batch_t *) calloc (1, sizeof (mg_batch_t));
   b->n = n;
   b->device = runs[0]->device;
   b->runs = (mg_run_t **) malloc (sizeof (mg_run_t *)*n);
   memcpy (b->runs, runs, sizeof (mg_run_t *)*n);
   int rc = MG_OK;
   if (cudaStreamCreateWithFlags (&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
       cudaGraphCreate (&b->graph, 0) != cudaSuccess) {
      mg_set_error ("mg_batch_create: cannot create the stream or graph");
      rc = MG_ERR_CUDA;
   }
   for (int q = 0 ; q < n && rc == MG_OK ; ++q) {
      if (!runs[q]->in_batch) {           // batch branches take the per-axis walls
         mg_drop_graphs (runs[q]);
         runs[q]->in_batch = 1;
      }
      rc = build_graph (runs[q]);
      cudaGraphNode_t node;
      if (rc == MG_OK && cudaGraphAddChildGraphNode (&node, b->graph, nullptr, 0, runs[q]->gr[0]) != cudaSuccess) {
         mg_set_error ("mg_batch_create: cannot add run %d to the batch graph", q);
         rc = MG_ERR_CUDA;
      }
   }
   if (rc == MG_OK && cudaGraphInstantiate (&b->exec, b->graph, 0) != cudaSuccess) {
      mg_set_error ("mg_batch_create: graph instantiation failed");
      rc = MG_ERR_CUDA;
   }
   if (rc != MG_OK) {
      mg_batch_destroy (b);
      return rc;
   }
   *out = b;
   return MG_OK;
}

extern "C" int mg_batch_step (mg_batch_t *b, int nsteps, double *const *energies)
{
   if (!b || nsteps < 0) {
      mg_set_error ("mg_batch_step: bad arguments");
      return MG_ERR_ARG;
   }
   MG_CUDA (cudaSetDevice (b->device));
   for (int q = 0 ; q < b->n ; ++q) {
      mg_run_t *r = b->runs[q];
      if (!r->graph_ok || !r->inited || r->stage_no != 0) {
         mg_set_error ("mg_batch_step: run %d changed since the batch was built", q);
         return MG_ERR_STATE;
      }
   }
   // Everything a run enqueued before goes first.
   for (int q = 0 ; q < b->n ; ++q) {
      cudaEvent_t e = b->runs[q]->ev[2];
      MG_CUDA (cudaEventRecord (e, b->runs[q]->stream));
      MG_CUDA (cudaStreamWaitEvent (b->stream, e, 0));
   }
   int rc = MG_OK;
   for (int done = 0 ; done < nsteps && rc == MG_OK ; ) {
      const int chunk = (nsteps - done < MG_RING) ? nsteps - done : MG_RING;
      for (int q = 0 ; q < b->n ; ++q)
         MG_CUDA (cudaMemsetAsync (&b->runs[q]->dsc->step, 0, sizeof (int), b->stream));
      for (int s = 0 ; s < chunk && rc == MG_OK ; ++s) {
         // Sorts that are due go on the batch stream, between launches.
         for (int q = 0 ; q < b->n && rc == MG_OK ; ++q) {
            mg_run_t *r = b->runs[q];
            cudaStream_t own = r->stream;
            r->stream = b->stream;
            rc = maybe_sort (r);
            r->stream = own;
         }
         if (rc == MG_OK && cudaGraphLaunch (b->exec, b->stream) != cudaSuccess) {
            mg_set_error ("mg_batch_step: graph launch failed");
            rc = MG_ERR_CUDA;
         }
      }
      for (int q = 0 ; q < b->n && rc == MG_OK && energies ; ++q)
         if (energies[q])
            MG_CUDA (cudaMemcpyAsync (energies[q] + 6*(size_t) done, b->runs[q]->ring, sizeof (double)*6*chunk,
                                      cudaMemcpyDeviceToHost, b->stream));
      MG_CUDA (cudaStreamSynchronize (b->stream));
      done += chunk;
   }
   TRY (rc);
   for (int q = 0 ; q < b->n ; ++q) {
      b->runs[q]->time += nsteps*b->runs[q]->g.tau;
      TRY (check_err (b->runs[q]));
   }
   return MG_OK;
}

extern "C" int mg_run_step_gauss (mg_run_t *r, int nsteps, double *rows)
{
   CHECK_RUN (r);
   if (!r->inited || r->stage_no != 0) {
      mg_set_error ("mg_run_step_gauss: run not initialised or inside a staged step");
      return MG_ERR_STATE;
   }
   TRY (ensure_gauss (r));
   if (r->in_batch) {
      mg_drop_graphs (r);
      r->in_batch = 0;
   }
   TRY (build_graph (r));
   // gauss_start: the density at the start (plasma_gaussTest.c:77).
   TRY (mg_gauss_rho (r, r->gauss_rho[1]));
   for (int s = 0 ; s < nsteps ; ++s) {
      double *t = r->gauss_rho[0];
      r->gauss_rho[0] = r->gauss_rho[1];
      r->gauss_rho[1] = t;
      const double time = r->time;
      TRY (maybe_sort (r));
      MG_CUDA (cudaMemsetAsync (&r->dsc->step, 0, sizeof (int), r->stream));
      TRY (launch_step_graph (r));
      TRY (mg_gauss_rho (r, r->gauss_rho[1]));
      TRY (mg_gauss_residual (r, r->gauss_rho[0], r->gauss_rho[1], r->gauss_out));
      double res[2];
      MG_CUDA (cudaMemcpyAsync (res, r->gauss_out, sizeof (res), cudaMemcpyDeviceToHost, r->stream));
      MG_CUDA (cudaStreamSynchronize (r->stream));
      r->time += r->g.tau;
      if (rows) {
         rows[3*(size_t) s] = time;
         rows[3*(size_t) s + 1] = res[0];
         rows[3*(size_t) s + 2] = res[1];
      }
   }
   return check_err (r);
}

extern "C" int mg_run_synchronize (mg_run_t *r)
{
   CHECK_RUN (r);
   MG_CUDA (cudaStreamSynchronize (r->stream));
   return check_err (r);
}

extern "C" int mg_run_stream (mg_run_t *r, void **stream)
{
   CHECK_RUN (r);
   if (stream)
      *stream = (void *) r->stream;
   return MG_OK;
}

extern "C" int mg_run_kernels_per_step (mg_run_t *r, int *count)
{
   CHECK_RUN (r);
   TRY (build_graph (r));
   if (count)
      *count = r->kernels_per_step;
   return MG_OK;
}

extern "C" int mg_run_device_bytes (mg_run_t *r, long long *bytes)
{
   CHECK_RUN (r);
   if (bytes)
      *bytes = r->dev_bytes;
   return MG_OK;
}

extern "C" int mg_run_profile (mg_run_t *r, int enable)
{
   CHECK_RUN (r);
   if (enable && !r->pev) {
      r->pev = (cudaEvent_t *) calloc (2*MG_PROFILE_CHUNK, sizeof (cudaEvent_t));
      for (int q = 0 ; q < 2*MG_PROFILE_CHUNK ; ++q)
         MG_CUDA (cudaEventCreate (&r->pev[q]));
   }
   r->profile = enable;
   return MG_OK;
}

extern "C" int mg_run_last_timing (mg_run_t *r, double *push_ms, double *step_ms)
{
   CHECK_RUN (r);
   if (push_ms) *push_ms = r->last_push_ms;
   if (step_ms) *step_ms = r->last_step_ms;
   return MG_OK;
}

// ---------------------------------------------------------------------------
// Device placement.
// ---------------------------------------------------------------------------
int mg_place64 (mg_run_t *r, const mg_place_t *spec, long long at, long long count);
int mg_place32 (mg_run_t *r, const mg_place_t *spec, long long at, long long count);
int mg_ensure_capacity32 (mg_run_t *r, long long need);

int mg_ensure_capacity64 (mg_run_t *r, long long need)
{
   return ensure_capacity (r, need);
}

extern "C" int mg_run_place_uniform (mg_run_t *r, const mg_place_t *s)
{
   CHECK_RUN (r);
   if (!s || s->ppc <= 0) {
      mg_set_error ("mg_run_place_uniform: bad spec");
      return MG_ERR_ARG;
   }
   long long cells = 1;
   for (int a = 0 ; a < 3 ; ++a) {
      if (s->lo[a] < 0 || s->hi[a] > r->g.n[a] || s->hi[a] < s->lo[a]) {
         mg_set_error ("mg_run_place_uniform: box [%d,%d) outside axis %d of %d cells",
                       s->lo[a], s->hi[a], a, r->g.n[a]);
         return MG_ERR_ARG;
      }
      cells *= s->hi[a] - s->lo[a];
   }
   const long long count = cells*s->ppc;
   if (count == 0)
      return MG_OK;
   if (is32 (r)) {
      TRY (mg_ensure_capacity32 (r, r->np + count));
      TRY (mg_place32 (r, s, r->np, count));
   } else {
      TRY (ensure_capacity (r, r->np + count));
      TRY (mg_place64 (r, s, r->np, count));
   }
   r->np += count;
   r->inited = 0;
   r->tiles_ok = 0;
   return MG_OK;
}
