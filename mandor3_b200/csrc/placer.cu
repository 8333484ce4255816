// Device marker placement driven by the reference's ranmar generator
// (Marsaglia-Zaman lagged Fibonacci with lags 97 and 33 plus an arithmetic
// sequence, misc_ranmar.c:79-146).  The reference ships the generator but
// no placer that uses it; the placement rule here is this project's
// (documented in include/mandor_b200.h at mg_place_t).
//
// Every ranmar value is a multiple of 2^-24, so the generator runs in
// integers: F_n = (F_{n-97} - F_{n-33}) mod 2^24 and C_n = (C_0 - n CD) mod
// CM, output_n = (F_n - C_{n+1}) mod 2^24 scaled by 2^-24 -- bit-identical
// to the reference's doubles.  The Fibonacci part is linear over
// Z/2^24, so the state after L draws is A^L s_0 for the 97x97 companion
// matrix A; the host computes one start state per chunk by repeated
// squaring and every device thread then generates its own chunk.
#include <cuda_runtime.h>

#include <mutex>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "mg_internal.cuh"
#include "placer_math.cuh"

#define RM_LAG 97
#define RM_MASK 0xFFFFFFu
#define RM_CD 7654321LL
#define RM_CM 16777213LL
#define RM_C0 362436LL
#define MG_PLACE_STATIC_STATES 4096

namespace {

// ranmar_init (misc_ranmar.c:79-119) in integer form: F_{-1-s} = u[s].
static void rm_seed (int ij, int kl, uint32_t F[RM_LAG])
{
   int i = (ij/177)%177 + 2, j = ij%177 + 2, k = (kl/169)%178 + 1, l = kl%169;
   uint32_t u[RM_LAG];
   for (int ii = 0 ; ii < RM_LAG ; ii++) {
      uint32_t s = 0;
      for (int bit = 0 ; bit < 24 ; bit++) {
         int m = (((i*j)%179)*k)%179;
         i = j;
         j = k;
         k = m;
         l = (53*l + 1)%169;
         if ((l*m)%64 >= 32)
            s |= 1u << (23 - bit);
      }
      u[ii] = s;
   }
   // State vector s[q] = F_{q-97}, q = 0..96  (F_{-97} .. F_{-1}).
   for (int q = 0 ; q < RM_LAG ; ++q)
      F[q] = u[96 - q];
}

typedef uint32_t Mat[RM_LAG][RM_LAG];

// y = M x over Z/2^24.
static void mat_vec (const Mat &M, const uint32_t x[RM_LAG], uint32_t y[RM_LAG])
{
   for (int r = 0 ; r < RM_LAG ; ++r) {
      uint64_t acc = 0;
      for (int c = 0 ; c < RM_LAG ; ++c)
         acc += (uint64_t) M[r][c]*x[c];
      y[r] = (uint32_t) (acc & RM_MASK);
   }
}

static void mat_mul (const Mat &A, const Mat &B, Mat &C)
{
   for (int r = 0 ; r < RM_LAG ; ++r)
      for (int c = 0 ; c < RM_LAG ; ++c) {
         uint64_t acc = 0;
         for (int q = 0 ; q < RM_LAG ; ++q)
            acc += (uint64_t) A[r][q]*B[q][c];
         C[r][c] = (uint32_t) (acc & RM_MASK);
      }
}

// Companion matrix of one draw: new state s'[q] = s[q+1], s'[96] = s[0] - s[64].
static void mat_step (Mat &A)
{
   memset (&A, 0, sizeof (Mat));
   for (int q = 0 ; q < RM_LAG - 1 ; ++q)
      A[q][q + 1] = 1;
   A[96][0] = 1;
   A[96][64] = RM_MASK;           // -1 mod 2^24
}

struct PlaceArgs {
   mg_place_t s;
   double h[3];
   long long nmarkers;     // markers in the box
   long long per_thread;   // markers per thread
   long long at;           // first device slot
};

// One thread: markers [t*per, (t+1)*per) of the box, draws starting at
// skip + 7*t*per, whose generator state the host put in states[t].
__global__ void __launch_bounds__ (128)
k_place (PlaceArgs a, const uint32_t *states, Markers64 m)
{
   extern __shared__ uint32_t ring[];           // RM_LAG words per thread
   const long long t = blockIdx.x*(long long) blockDim.x + threadIdx.x;
   const long long first = t*a.per_thread;
   if (first >= a.nmarkers)
      return;
   uint32_t *F = ring + threadIdx.x*RM_LAG;
   for (int q = 0 ; q < RM_LAG ; ++q)
      F[q] = states[t*RM_LAG + q];               // F_{d-97} .. F_{d-1}
   long long d = a.s.skip + 7*first;             // absolute draw index
   int head = 0;                                 // slot of F_{d-97}
   const int ex = a.s.hi[0] - a.s.lo[0], ey = a.s.hi[1] - a.s.lo[1], ez = a.s.hi[2] - a.s.lo[2];
   long long last = first + a.per_thread;
   if (last > a.nmarkers)
      last = a.nmarkers;
   for (long long n = first ; n < last ; ++n) {
      double u[7];
      for (int q = 0 ; q < 7 ; ++q, ++d) {
         // F_d = F_{d-97} - F_{d-33}; F_{d-97} sits at slot head, F_{d-33}
         // at slot head + 64.
         int s33 = head + 64;
         if (s33 >= RM_LAG) s33 -= RM_LAG;
         const uint32_t f = (F[head] - F[s33]) & RM_MASK;
         F[head] = f;
         head = (head + 1 == RM_LAG) ? 0 : head + 1;
         long long c = (RM_C0 - ((d + 1) % RM_CM)*RM_CD) % RM_CM;
         if (c < 0) c += RM_CM;
         const uint32_t out = (f - (uint32_t) c) & RM_MASK;
         u[q] = (double) out*(1.0/16777216.0);
      }
      const long long cell = n / a.s.ppc;
      const int k = a.s.lo[2] + (int) (cell % ez);
      const int j = a.s.lo[1] + (int) ((cell / ez) % ey);
      const int i = a.s.lo[0] + (int) (cell / ((long long) ez*ey));
      (void) ex;
      const long long o = a.at + n;
      m.x[o] = (i + u[0])*a.h[0];
      m.y[o] = (j + u[1])*a.h[1];
      m.z[o] = (k + u[2])*a.h[2];
      double gx, gy, gz, gw;
      pm_box_muller (u[3], u[4], &gx, &gy);
      pm_box_muller (u[5], u[6], &gz, &gw);
      m.ux[o] = a.s.drift[0] + a.s.uth[0]*gx;
      m.uy[o] = a.s.drift[1] + a.s.uth[1]*gy;
      m.uz[o] = a.s.drift[2] + a.s.uth[2]*gz;
      m.rho[o] = (float) a.s.rho;
      m.qm[o] = (float) a.s.qDivM;
      m.id[o] = a.s.id0 + (int) n;
   }
}

} // namespace

// Powers A^(2^j) of the one-draw matrix, j < 63, computed once per process:
// any jump is then a product of at most 63 of them.
static Mat *g_pow2 = nullptr;
static std::once_flag g_pow2_once;

static void pow2_table ()
{
   g_pow2 = (Mat *) malloc (sizeof (Mat)*63);
   mat_step (g_pow2[0]);
   for (int j = 1 ; j < 63 ; ++j)
      mat_mul (g_pow2[j - 1], g_pow2[j - 1], g_pow2[j]);
}

// x <- A^e x with the cached powers (one 97x97 mat-vec per set bit of e).
static void jump_vec (long long e, uint32_t x[RM_LAG])
{
   uint32_t tmp[RM_LAG];
   for (int j = 0 ; e > 0 ; ++j, e >>= 1)
      if (e & 1) {
         mat_vec (g_pow2[j], x, tmp);
         memcpy (x, tmp, sizeof (tmp));
      }
}

// Host: generator states for `nthreads` chunks of `chunk_draws` draws
// starting at draw `skip`.  states[t] = (F_{d_t-97} .. F_{d_t-1}).
int mg_ranmar_states (int ij, int kl, long long skip, long long chunk_draws, int nthreads,
                      uint32_t *states)
{
   if (ij < 0 || ij > 31328 || kl < 0 || kl > 30081) {
      mg_set_error ("ranmar seeds must satisfy 0 <= ij <= 31328, 0 <= kl <= 30081 (misc_ranmar.c:81-84)");
      return MG_ERR_ARG;
   }
   std::call_once (g_pow2_once, pow2_table);
   uint32_t s[RM_LAG], tmp[RM_LAG];
   rm_seed (ij, kl, s);
   jump_vec (skip, s);
   // One chunk's jump as a matrix: the product of the cached powers.
   Mat *M = (Mat *) malloc (sizeof (Mat)), *T = (Mat *) malloc (sizeof (Mat));
   if (nthreads > 1) {
      bool first = true;
      long long e = chunk_draws;
      for (int j = 0 ; e > 0 ; ++j, e >>= 1) {
         if (!(e & 1))
            continue;
         if (first) {
            memcpy (M, &g_pow2[j], sizeof (Mat));
            first = false;
         } else {
            mat_mul (g_pow2[j], *M, *T);
            memcpy (M, T, sizeof (Mat));
         }
      }
   }
   for (int t = 0 ; t < nthreads ; ++t) {
      memcpy (states + (size_t) t*RM_LAG, s, sizeof (s));
      if (t + 1 < nthreads) {
         mat_vec (*M, s, tmp);
         memcpy (s, tmp, sizeof (s));
      }
   }
   free (M);
   free (T);
   return MG_OK;
}

int mg_place64 (mg_run_t *r, const mg_place_t *spec, long long at, long long count)
{
   PlaceArgs a;
   a.s = *spec;
   for (int q = 0 ; q < 3 ; ++q)
      a.h[q] = r->g.h[q];
   a.nmarkers = count;
   a.at = at;
   // Generator streams: 16 per SM, which keeps the host jump-ahead (one
   // 97x97 mat-vec per stream) at a few milliseconds; the markers are the
   // same for any stream count.
   int nthreads = mg_sm_count ()*16;
   if (count < nthreads) nthreads = (int) count;
   if (nthreads < 1) nthreads = 1;
   a.per_thread = (count + nthreads - 1)/nthreads;
   nthreads = (int) ((count + a.per_thread - 1)/a.per_thread);
   uint32_t *hs = (uint32_t *) malloc ((size_t) nthreads*RM_LAG*sizeof (uint32_t));
   int rc = mg_ranmar_states (spec->seed_ij, spec->seed_kl, spec->skip, 7*a.per_thread, nthreads, hs);
   if (rc != MG_OK) {
      free (hs);
      return rc;
   }
   uint32_t *ds = nullptr;
   const size_t ds_bytes = (size_t) nthreads*RM_LAG*sizeof (uint32_t);
   if (mg_dev_alloc (r, (void **) &ds, ds_bytes) != MG_OK) {
      free (hs);
      return MG_ERR_OOM;
   }
   cudaMemcpyAsync (ds, hs, ds_bytes, cudaMemcpyHostToDevice, r->stream);
   const int T = 128, B = (nthreads + T - 1)/T;
   const int smem = T*RM_LAG*sizeof (uint32_t);          // 49,664 bytes
   cudaFuncSetAttribute (k_place, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
   k_place<<<B, T, smem, r->stream>>> (a, ds, r->m64);
   cudaError_t e = cudaGetLastError ();
   cudaStreamSynchronize (r->stream);
   mg_dev_free (r, ds);
   r->dev_bytes -= ds_bytes;
   free (hs);
   if (e != cudaSuccess) {
      mg_set_error ("placer launch: %s", cudaGetErrorString (e));
      return MG_ERR_CUDA;
   }
   return MG_OK;
}

// ---------------------------------------------------------------------------
// Placement without allocation.
//
// mg_place_uniform_static writes the markers of one placement box into
// device arrays the caller owns, and allocates nothing: the generator start
// states live in a file-scope device array (MG_PLACE_STATIC_STATES states of
// 97 words, 1.59 MB, held by every GPU that loads the library until the
// process exits), and the host-side jump-ahead works in static host buffers.
// Every call overwrites the states it uses, so nothing needs clearing.
// Calls are serialised inside the process by a mutex; each call copies the
// start states from pageable static host memory and waits for its stream
// before returning, so the next call may reuse both buffers.  Work that
// touches the array concurrently from outside these calls would race on it.
// The array's device address is looked up once per device (first call with
// that device current) and kept: after cudaDeviceReset of that device the
// kept address is stale, so a process that resets a device must not call
// this entry point on it again.
// ---------------------------------------------------------------------------
static __device__ __align__ (256) uint32_t g_place_states[MG_PLACE_STATIC_STATES*RM_LAG];

namespace {

std::mutex g_place_mutex;
uint32_t   g_host_states[MG_PLACE_STATIC_STATES*RM_LAG];
Mat        g_mat[3];
uint32_t  *g_states_dev[64];          // cudaGetSymbolAddress of g_place_states per device

// Jump-ahead with the static matrices: R = A^e.
void mat_pow_static (long long e, Mat &R, Mat &base, Mat &tmp)
{
   mat_step (base);
   memset (&R, 0, sizeof (Mat));
   for (int q = 0 ; q < RM_LAG ; ++q)
      R[q][q] = 1;
   while (e > 0) {
      if (e & 1) {
         mat_mul (R, base, tmp);
         memcpy (&R, &tmp, sizeof (Mat));
      }
      e >>= 1;
      if (e) {
         mat_mul (base, base, tmp);
         memcpy (&base, &tmp, sizeof (Mat));
      }
   }
}

} // namespace

extern "C" int mg_place_uniform_static (const mg_place_t *spec, const double h[3],
                                        const mg_device_markers_t *out, long long capacity,
                                        int threads, void *stream)
{
   if (!spec || !h || !out || spec->ppc <= 0) {
      mg_set_error ("mg_place_uniform_static: null or empty argument");
      return MG_ERR_ARG;
   }
   long long cells = 1;
   for (int a = 0 ; a < 3 ; ++a) {
      if (spec->hi[a] < spec->lo[a]) {
         mg_set_error ("mg_place_uniform_static: empty box on axis %d", a);
         return MG_ERR_ARG;
      }
      cells *= spec->hi[a] - spec->lo[a];
   }
   const long long count = cells*spec->ppc;
   if (count > capacity) {
      mg_set_error ("mg_place_uniform_static: %lld markers do not fit the %lld-marker arrays",
                    count, capacity);
      return MG_ERR_CAPACITY;
   }
   if (threads < 0 || threads > MG_PLACE_STATIC_STATES) {
      mg_set_error ("mg_place_uniform_static: %d generator streams requested; the static scratch "
                    "holds at most %d", threads, MG_PLACE_STATIC_STATES);
      return MG_ERR_ARG;
   }
   if (spec->seed_ij < 0 || spec->seed_ij > 31328 || spec->seed_kl < 0 || spec->seed_kl > 30081) {
      mg_set_error ("ranmar seeds must satisfy 0 <= ij <= 31328, 0 <= kl <= 30081 (misc_ranmar.c:81-84)");
      return MG_ERR_ARG;
   }
   if (count == 0)
      return MG_OK;
   int dev = 0;
   if (cudaGetDevice (&dev) != cudaSuccess || dev < 0 || dev >= 64) {
      mg_set_error ("mg_place_uniform_static: no current CUDA device");
      return MG_ERR_CUDA;
   }
   std::lock_guard<std::mutex> lock (g_place_mutex);
   // First call on this device: resolve the device address of the static
   // scratch with the device current.
   if (!g_states_dev[dev]) {
      void *ptr = nullptr;
      cudaError_t e = cudaGetSymbolAddress (&ptr, g_place_states);
      if (e != cudaSuccess || !ptr) {
         mg_set_error ("mg_place_uniform_static: cudaGetSymbolAddress: %s", cudaGetErrorString (e));
         return MG_ERR_CUDA;
      }
      g_states_dev[dev] = (uint32_t *) ptr;
   }
   int nthreads = threads ? threads : MG_PLACE_STATIC_STATES;
   if (count < nthreads)
      nthreads = (int) count;
   PlaceArgs a;
   a.s = *spec;
   for (int q = 0 ; q < 3 ; ++q)
      a.h[q] = h[q];
   a.nmarkers = count;
   a.at = 0;
   a.per_thread = (count + nthreads - 1)/nthreads;
   nthreads = (int) ((count + a.per_thread - 1)/a.per_thread);

   uint32_t st[RM_LAG], tmp[RM_LAG];
   rm_seed (spec->seed_ij, spec->seed_kl, st);
   if (spec->skip > 0) {
      mat_pow_static (spec->skip, g_mat[0], g_mat[1], g_mat[2]);
      mat_vec (g_mat[0], st, tmp);
      memcpy (st, tmp, sizeof (st));
   }
   if (nthreads > 1)
      mat_pow_static (7*a.per_thread, g_mat[0], g_mat[1], g_mat[2]);
   for (int t = 0 ; t < nthreads ; ++t) {
      memcpy (g_host_states + (size_t) t*RM_LAG, st, sizeof (st));
      if (t + 1 < nthreads) {
         mat_vec (g_mat[0], st, tmp);
         memcpy (st, tmp, sizeof (st));
      }
   }
   cudaStream_t s = (cudaStream_t) stream;
   MG_CUDA (cudaMemcpyAsync (g_states_dev[dev], g_host_states, (size_t) nthreads*RM_LAG*sizeof (uint32_t),
                             cudaMemcpyHostToDevice, s));
   Markers64 m;
   m.x = out->x; m.y = out->y; m.z = out->z;
   m.ux = out->vx; m.uy = out->vy; m.uz = out->vz;
   m.rho = out->rho; m.qm = out->qDivM; m.id = out->id;
   const int T = 128, B = (nthreads + T - 1)/T;
   const int smem = T*RM_LAG*sizeof (uint32_t);
   MG_CUDA (cudaFuncSetAttribute (k_place, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
   k_place<<<B, T, smem, s>>> (a, g_states_dev[dev], m);
   MG_LAUNCH_CHECK ();
   // The host states buffer and the device scratch are reused by the next
   // call: wait here.
   MG_CUDA (cudaStreamSynchronize (s));
   return MG_OK;
}
