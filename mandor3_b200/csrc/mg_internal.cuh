// Internal definitions shared by the CUDA translation units of the B200
// particle-in-cell core.  Nothing here is part of the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mandor_b200.h"

// ---------------------------------------------------------------------------
// Device mesh layout.
//
// Every field component (Ex, Ey, Ez, Hx, Hy, Hz, Jx, Jy, Jz) is its own
// array ("structure of arrays") over nodes i in [-2, n0+2], j in [-2, n1+2],
// k in [-4, n2+2+pad]: two ghost layers on every side (the reference keeps
// one for E, H and two for J, core/main.c:108-115) and a z row padded so
// that k = 0 of every row starts on a 32-byte sector.  k is the fastest
// index, as in the reference's meshes (type_mesh.h:134-141).
// ---------------------------------------------------------------------------
#define MG_GX 2
#define MG_GZ_FRONT 4

// Precision-form tiles: markers are counting-sorted by (tile, cell) and the
// push stages one tile of fields and currents in shared memory at a time.
// The default tile; a run may pick 4x4x4 or 8x8x8 instead (tdim).
#define MG_TILE_X 8
#define MG_TILE_Y 8
#define MG_TILE_Z 4

struct Grid {
   int    n[3];
   long   sx, sy;          // strides of i and j (k stride is 1)
   long   origin;          // linear offset of node (0,0,0)
   long   total;           // elements per component array
   double h[3];
   double tau;
   int    bc[2][3];        // [min/max][axis]

   __host__ __device__ __forceinline__ long at (int i, int j, int k) const
   {
      return origin + i*sx + j*sy + k;
   }
};

// Nodes in front of k = 0 in a row: 4 for FP64 (k = 0 starts a 32-byte
// sector); 5 for FP32, so that the row offset of k = z0 - 1 is a multiple
// of 4 floats whenever z0 is, as a tensor-memory-access (TMA) tile copy
// starting there needs (16-byte aligned innermost coordinate).
#define MG_GZ_FRONT32 5

static inline Grid make_grid (const int n[3], const double h[3], double tau,
                              const int bc_min[3], const int bc_max[3], int front = MG_GZ_FRONT)
{
   Grid g;
   for (int a = 0 ; a < 3 ; ++a) {
      g.n[a] = n[a];
      g.h[a] = h[a];
      g.bc[0][a] = bc_min[a];
      g.bc[1][a] = bc_max[a];
   }
   g.tau = tau;
   long row = front + n[2] + 1 + MG_GX;
   row = (row + 3) & ~3L;                       // rows of a multiple of 4 elements
   g.sy = row;
   g.sx = row*(n[1] + 1 + 2*MG_GX);
   g.total = g.sx*(n[0] + 1 + 2*MG_GX);
   g.origin = MG_GX*g.sx + MG_GX*g.sy + front;
   return g;
}

// FP32-offset particle arrays.
struct Markers32 {
   int    *cell;           // packed cell ((i+1) << 20 | (j+1) << 10 | (k+1))
   float  *ox, *oy, *oz;   // offsets in [0,1) in units of h
   float  *ux, *uy, *uz;
   float  *rho, *qm;
   int    *id;
};

// Hard gauss-spot source, parameters as the kernel uses them
// (core/em_gaussSpot.c:64-123 conversions done).
struct GaussSpot {
   double ey, ez;          // signed amplitudes
   double omega;           // 2 pi frequency
   double y, z, width, duration, front, plateau;
   int    i;               // x-plane
};

// A focused-laser mirror (scpic/em_mirror.c) as the step plays it: the
// values read_mirror_parameters derives and the two device profiles.
struct MirrorDev {
   double A, dt, T0, delay, phi0;
   int    forward;
   double *E, *H;          // (n1-9)(n2-9) x {y_cos, y_sin, z_cos, z_sin}
};
#define MG_MIRRORS 8

// Device-side per-run scalars (one small allocation).
struct DevScalars {
   double time;            // t = n*tau of the step being advanced
   double acc[8];          // W_E, W_M, WTx, WTy, WTz of the current step
   long long dead;         // markers removed by open walls (not compacted)
   int    step;            // steps done since the energy ring was reset
   int    err;             // sticky error flags (1: start cell outside the
                           // ghost layers, 2: more than one cell per step)
   int    err_info[4];     // first offending marker index and cell
   int    tile_next;       // next tile to hand out in the tiled push
   int    tfsf_frame;      // TF/SF frame counter (steps since t = 0)
   float  rho_max;         // largest |rho| of the markers at the last sort
   Markers32 m32;          // the current marker buffer set (precision form),
                           // read by the kernels of the step graph
};

#define MG_RING 4096       // energy rows kept on the device between copies

// FP64 particle arrays (structure of arrays).
struct Markers64 {
   double *x, *y, *z, *ux, *uy, *uz;
   float  *rho, *qm;
   int    *id;
};


struct mg_run {
   mg_params_t prm;
   Grid        g;
   int         device;
   cudaStream_t stream;

   // fields
   double *E[3], *H[3], *J[3];
   double *Hn[3];          // H at t = n tau (H holds n-1/2, then n+1/2)
   // Second E and H arrays of the one-pass field-only step: the step reads
   // E, H (E32, H32) and writes Ealt, Halt (Ealt32, Halt32), then the
   // pointers swap.
   double *Ealt[3], *Halt[3];
   float  *Ealt32[3], *Halt32[3];
   const void *fo_read0;   // E[0] (E32[0]) the first field-only step graph reads
   int     fo_graph;       // the step graphs are the field-only pair
   double *mur[2][3];      // Mur history, 4 doubles per wall node
   float  *E32[3], *H32[3], *J32[3], *Hn32[3];
   float  *mur32[2][3];

   // markers
   long long  np, cap;
   Markers64  m64;
   Markers32  m32;         // current buffer set (precision form)
   Markers32  m32b;        // the other set: the sort scatters into it
   void      *sort_tmp;    // scratch for sorting / compaction
   size_t     sort_tmp_bytes;
   long long  steps_since_sort;
   int        tdim[3];     // tile size in cells (precision form)
   int        tiles[3];    // tiles per axis
   int        ntiles;
   int       *tile_start;  // ntiles + 2 marker offsets of the last sort:
                           // tile t holds [tile_start[t], tile_start[t+1]),
                           // then the markers outside the mesh, then the
                           // removed ones
   int       *tile_list;   // ntiles + 1: the tiles holding markers, then
                           // their count (after tile_start, same allocation)
   int        tiles_ok;    // tile_start describes the marker order

   // scalars and energy ring
   DevScalars *dsc;
   double     *ring;       // MG_RING rows of 6 doubles
   double      time;       // host mirror

   // laser
   int         has_laser;
   mg_laser_t  laser;
   int         has_gspot;
   GaussSpot   gspot;

   // asynchronous snapshot (mg_run_snapshot): device copy of the
   // checkpoint state, copied to the caller's buffers on its own stream
   double     *snap_E, *snap_H;
   mg_marker_t *snap_m;
   long long   snap_cap;
   cudaStream_t snap_stream;
   cudaEvent_t snap_ready, snap_done;
   // Host transfers: a copy stream beside the run's stream and, per half of
   // the staging buffer, "converted" and "copied" events, so that the
   // layout conversion of one chunk overlaps the copy of the previous one.
   cudaStream_t xfer;
   cudaEvent_t  xev[2][2];
   int         snap_pending;

   // focused-laser mirrors (mg_run_add_mirror)
   int         nmirrors;
   MirrorDev   mirrors[MG_MIRRORS];

   // TF/SF interface (tfsf.cu), null when off
   struct mg_tfsf_state *tfsf;

   // probes: nodes, per-step sample ring (MG_RING rows of nprobes x 7)
   int         nprobes;
   int        *probe_ijk;
   double     *probe_ring;
   void      **probe_ptrs;   // E and H^n component arrays (device copy)

   // Gauss-law test: densities before/after a step, residuals
   double     *gauss_rho[2];
   double     *gauss_out;

   // staging
   void       *stage;
   size_t      stage_bytes;

   // graph
   cudaGraph_t     gr[5];      // whole step, its three parts, the field-only step's mirror
   cudaGraphExec_t gexec[5];
   int             graph_ok;
   int             in_batch;       // step graph built for a batch branch (per-axis wall kernels)
   int             kernels_per_step;

   // stage ordering (like core/em.c:32's emStage)
   int         stage_no;
   int         inited;

   // profiling
   int         profile;
   cudaEvent_t ev[4];
   cudaEvent_t *pev;       // event pairs around the push, profiling mode
   double      last_push_ms, last_step_ms;

   long long   dev_bytes;
};

// Error handling -----------------------------------------------------------
void mg_set_error (const char *fmt, ...);

#define MG_CUDA(call)                                                        \
   do {                                                                      \
      cudaError_t e_ = (call);                                               \
      if (e_ != cudaSuccess) {                                               \
         mg_set_error ("%s:%d: %s: %s", __FILE__, __LINE__, #call,           \
                       cudaGetErrorString (e_));                             \
         return MG_ERR_CUDA;                                                 \
      }                                                                      \
   } while (0)

#define MG_LAUNCH_CHECK()                                                    \
   do {                                                                      \
      cudaError_t e_ = cudaGetLastError ();                                  \
      if (e_ != cudaSuccess) {                                               \
         mg_set_error ("%s:%d: kernel launch: %s", __FILE__, __LINE__,       \
                       cudaGetErrorString (e_));                             \
         return MG_ERR_CUDA;                                                 \
      }                                                                      \
   } while (0)

// Launch helpers shared between translation units ---------------------------
int mg_fields64_h_half (mg_run_t *r);
int mg_fields64_energy (mg_run_t *r);
int mg_fields64_h_step (mg_run_t *r);
int mg_fields64_e_step (mg_run_t *r);
int mg_fields64_jbc (mg_run_t *r);
int mg_fields64_jbc_graph (mg_run_t *r);
int mg_fields64_one_pass (mg_run_t *r);
int mg_fields32_one_pass (mg_run_t *r);
int mg_fields64_e_finish (mg_run_t *r);
int mg_fields64_init (mg_run_t *r);
int mg_fields64_zero_j (mg_run_t *r);
int mg_fields64_h_both (mg_run_t *r);
int mg_fields64_e_fused (mg_run_t *r);
int mg_push64 (mg_run_t *r);
int mg_gauss_rho (mg_run_t *r, double *rho);
int mg_probes_enqueue (mg_run_t *r);
int mg_sort64 (mg_run_t *r);
int mg_tile_list (mg_run_t *r, const long long *offset, int lc);
#define SCAN_CHUNK 4096
int mg_scan_counts (mg_run_t *r, const int *count, long long kp, long long len, long long *offset,
                    long long *bsum);

// Counter slot of a sort key: eight neighbouring keys sit in eight different
// regions of the counter array, so that nearly sorted markers do not queue
// their atomics on one 32-byte L2 sector.  kp: keys per region.
static __device__ __forceinline__ long long spread (long long key, long long kp)
{
   return (key & 7)*kp + (key >> 3);
}

// Runs of equal keys in a warp (markers arrive nearly sorted): the lane's
// run start and, for the run's first lane, the run length.
static __device__ __forceinline__ void key_runs (int key, int lane, int &start, int &len)
{
   const int prev = __shfl_up_sync (0xffffffffu, key, 1);
   const unsigned heads = __ballot_sync (0xffffffffu, lane == 0 || prev != key);
   const unsigned le = (lane == 31) ? 0xffffffffu : ((2u << lane) - 1);
   start = 31 - __clz (heads & le);
   const unsigned after = heads & ~le;
   len = (after ? __ffs (after) - 1 : 32) - lane;
}
int mg_tfsf_h (mg_run_t *r);
int mg_tfsf_e (mg_run_t *r);
int mg_tfsf_record (mg_run_t *r);
bool mg_tfsf_playing (const mg_run_t *r);
bool mg_tfsf_recording (const mg_run_t *r);
void mg_tfsf_free (mg_run_t *r);
int mg_gauss_residual (mg_run_t *r, const double *rho1, const double *rho2, double *out_dev);
int mg_end_step (mg_run_t *r);

int mg_fields32_h_half (mg_run_t *r);
int mg_fields32_energy (mg_run_t *r);
int mg_fields32_h_step (mg_run_t *r);
int mg_fields32_e_step (mg_run_t *r);
int mg_fields32_jbc (mg_run_t *r);
int mg_fields32_jbc_graph (mg_run_t *r);
int mg_fields32_e_finish (mg_run_t *r);
int mg_fields32_init (mg_run_t *r);
int mg_fields32_zero_j (mg_run_t *r);
int mg_fields32_h_both (mg_run_t *r);
int mg_fields32_e_fused (mg_run_t *r);
int mg_push32 (mg_run_t *r);
int mg_sort32 (mg_run_t *r);
int mg_walls32 (mg_run_t *r);
int mg_enqueue_step32 (mg_run_t *r, int part);
int mg_place32 (mg_run_t *r, const mg_place_t *spec, long long at, long long count);
int mg_ensure_capacity32 (mg_run_t *r, long long need);
int mg_publish_markers32 (mg_run_t *r);
void mg_free_markers32 (mg_run_t *r);
int mg_dev_alloc (mg_run_t *r, void **p, size_t bytes);
void mg_dev_free (mg_run_t *r, void *p);
int mg_ensure_stage (mg_run_t *r, size_t bytes);
void mg_drop_graphs (mg_run_t *r);
int mg_run_set_fields32 (mg_run_t *r, const double *E, const double *H);
int mg_fields_out32 (mg_run_t *r, double *E, double *H, bool dev);
int mg_fields_out (mg_run_t *r, double *E, double *H, bool dev);
int mg_markers_out (mg_run_t *r, mg_marker_t *out, long long cap, long long *n, bool dev);
int mg_run_get_current32 (mg_run_t *r, double *J);
int mg_run_set_markers32 (mg_run_t *r, const mg_marker_t *m, long long n);
int mg_markers_out32 (mg_run_t *r, mg_marker_t *m, long long cap, long long *n, bool dev);

// Grid sizing: a multiple of the SM count (148 on B200).
int mg_sm_count (void);
static inline int mg_blocks_for (long long work, int threads, int per_sm = 8)
{
   long long b = (work + threads - 1)/threads;
   long long cap = (long long) mg_sm_count ()*per_sm;
   if (b > cap) b = cap;
   if (b < 1) b = 1;
   return (int) b;
}
