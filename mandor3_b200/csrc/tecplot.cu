// Node-centred field dumps for tecplot.out (IO_tecplot.c:108-153) and the
// probe samples (core/diag_probe.c:409-446).  Dumps: over the
// nodes [0, n]^3, E-type meshes (E, J) as 0.5 (F[p] + F[p + d_c]) per
// component c, H as the 4-point average in the two other axes, summed in the
// reference's order; FP64 arithmetic in both precision forms.
#include <cuda_runtime.h>

#include "mg_internal.cuh"

#define TRY_P(x)                                                             \
   do {                                                                      \
      int rc_ = (x);                                                         \
      if (rc_ != MG_OK)                                                      \
         return rc_;                                                         \
   } while (0)

namespace {

template <typename T>
__global__ void k_tec (Grid g, const T *X, const T *Y, const T *Z, int h_type, double *out)
{
   const long nk = g.n[2] + 1, nj = g.n[1] + 1, ni = g.n[0] + 1;
   const long dx = g.sx, dy = g.sy, dz = 1;
   for (long t = blockIdx.x*(long) blockDim.x + threadIdx.x ; t < ni*nj*nk ; t += (long) gridDim.x*blockDim.x) {
      const int k = (int) (t % nk), j = (int) ((t/nk) % nj), i = (int) (t/(nk*nj));
      const long p = g.at (i, j, k);
      double *o = out + 3*t;
      if (!h_type) {
         o[0] = 0.5*((double) X[p] + (double) X[p + dx]);
         o[1] = 0.5*((double) Y[p] + (double) Y[p + dy]);
         o[2] = 0.5*((double) Z[p] + (double) Z[p + dz]);
      } else {
         o[0] = 0.25*((double) X[p] + (double) X[p + dy] + (double) X[p + dz] + (double) X[p + dy + dz]);
         o[1] = 0.25*((double) Y[p] + (double) Y[p + dx] + (double) Y[p + dz] + (double) Y[p + dx + dz]);
         o[2] = 0.25*((double) Z[p] + (double) Z[p + dx] + (double) Z[p + dy] + (double) Z[p + dx + dy]);
      }
   }
}

template <typename T>
int tec_out (mg_run_t *r, T *const c[3], int h_type, double *host)
{
   const long vol = (long) (r->g.n[0] + 1)*(r->g.n[1] + 1)*(r->g.n[2] + 1);
   const size_t bytes = (size_t) vol*3*sizeof (double);
   int rc = mg_ensure_stage (r, bytes);
   if (rc != MG_OK)
      return rc;
   k_tec<T><<<mg_blocks_for (vol, 256, 8), 256, 0, r->stream>>> (r->g, c[0], c[1], c[2], h_type,
                                                                   (double *) r->stage);
   MG_LAUNCH_CHECK ();
   MG_CUDA (cudaMemcpyAsync (host, r->stage, bytes, cudaMemcpyDeviceToHost, r->stream));
   MG_CUDA (cudaStreamSynchronize (r->stream));
   return MG_OK;
}

// Probe samples (core/diag_probe.c:409-446): for each probe node (i, j, k)
// the row {t, Ex, Ey, Ez, Hx, Hy, Hz} of E^n and H^n interpolated to the node
// as above, into row (step % MG_RING) of the ring.
template <typename T>
__global__ void k_probes (Grid g, T *const *E, T *const *H, const int *ijk, int n, const DevScalars *dsc,
                          double *ring)
{
   const int q = blockIdx.x*blockDim.x + threadIdx.x;
   if (q >= n)
      return;
   const long dx = g.sx, dy = g.sy, dz = 1;
   const long p = g.at (ijk[3*q], ijk[3*q + 1], ijk[3*q + 2]);
   double *o = ring + 7*((long) (dsc->step % MG_RING)*n + q);
   const T *Ex = E[0], *Ey = E[1], *Ez = E[2], *Hx = H[0], *Hy = H[1], *Hz = H[2];
   o[0] = dsc->time;
   o[1] = 0.5*((double) Ex[p] + (double) Ex[p + dx]);
   o[2] = 0.5*((double) Ey[p] + (double) Ey[p + dy]);
   o[3] = 0.5*((double) Ez[p] + (double) Ez[p + dz]);
   o[4] = 0.25*((double) Hx[p] + (double) Hx[p + dy] + (double) Hx[p + dz] + (double) Hx[p + dy + dz]);
   o[5] = 0.25*((double) Hy[p] + (double) Hy[p + dx] + (double) Hy[p + dz] + (double) Hy[p + dx + dz]);
   o[6] = 0.25*((double) Hz[p] + (double) Hz[p + dx] + (double) Hz[p + dy] + (double) Hz[p + dx + dy]);
}

} // namespace

// Probe samples of the current step (E^n and H^n, after the H half step).
int mg_probes_enqueue (mg_run_t *r)
{
   if (r->nprobes <= 0)
      return MG_OK;
   const int NT = 128, B = (r->nprobes + NT - 1)/NT;
   if (r->prm.precision == MG_FP64)
      k_probes<double><<<B, NT, 0, r->stream>>> (r->g, (double *const *) r->probe_ptrs,
                                                 (double *const *) r->probe_ptrs + 3, r->probe_ijk,
                                                 r->nprobes, r->dsc, r->probe_ring);
   else
      k_probes<float><<<B, NT, 0, r->stream>>> (r->g, (float *const *) r->probe_ptrs,
                                                (float *const *) r->probe_ptrs + 3, r->probe_ijk,
                                                r->nprobes, r->dsc, r->probe_ring);
   MG_LAUNCH_CHECK ();
   return MG_OK;
}

extern "C" int mg_run_set_probes (mg_run_t *r, const int *ijk, int n)
{
   if (!r || n < 0 || (n > 0 && !ijk)) {
      mg_set_error ("mg_run_set_probes: bad arguments");
      return MG_ERR_ARG;
   }
   MG_CUDA (cudaSetDevice (r->device));
   for (int q = 0 ; q < n ; ++q)
      for (int a = 0 ; a < 3 ; ++a)
         if (ijk[3*q + a] < 0 || ijk[3*q + a] >= r->g.n[a]) {
            mg_set_error ("mg_run_set_probes: probe %d node %d on axis %d outside [0, %d)", q, ijk[3*q + a],
                          a, r->g.n[a]);
            return MG_ERR_ARG;
         }
   if (r->probe_ijk) mg_dev_free (r, r->probe_ijk);
   if (r->probe_ring) mg_dev_free (r, r->probe_ring);
   if (r->probe_ptrs) mg_dev_free (r, r->probe_ptrs);
   r->probe_ijk = nullptr;
   r->probe_ring = nullptr;
   r->probe_ptrs = nullptr;
   r->nprobes = 0;
   mg_drop_graphs (r);
   if (n == 0)
      return MG_OK;
   TRY_P (mg_dev_alloc (r, (void **) &r->probe_ijk, sizeof (int)*3*n));
   TRY_P (mg_dev_alloc (r, (void **) &r->probe_ring, sizeof (double)*7*(size_t) n*MG_RING));
   TRY_P (mg_dev_alloc (r, (void **) &r->probe_ptrs, sizeof (void *)*6));
   void *ptrs[6];
   for (int c = 0 ; c < 3 ; ++c) {
      ptrs[c] = r->prm.precision == MG_FP64 ? (void *) r->E[c] : (void *) r->E32[c];
      ptrs[3 + c] = r->prm.precision == MG_FP64 ? (void *) r->Hn[c] : (void *) r->Hn32[c];
   }
   MG_CUDA (cudaMemcpy (r->probe_ijk, ijk, sizeof (int)*3*n, cudaMemcpyHostToDevice));
   MG_CUDA (cudaMemcpy (r->probe_ptrs, ptrs, sizeof (ptrs), cudaMemcpyHostToDevice));
   r->nprobes = n;
   return MG_OK;
}

extern "C" int mg_run_probe_samples (mg_run_t *r, int nsteps, double *out)
{
   if (!r || nsteps < 0 || nsteps > MG_RING || (nsteps > 0 && !out)) {
      mg_set_error ("mg_run_probe_samples: bad arguments (at most %d steps)", MG_RING);
      return MG_ERR_ARG;
   }
   if (r->nprobes == 0 || nsteps == 0)
      return MG_OK;
   MG_CUDA (cudaSetDevice (r->device));
   MG_CUDA (cudaMemcpyAsync (out, r->probe_ring, sizeof (double)*7*(size_t) r->nprobes*nsteps,
                             cudaMemcpyDeviceToHost, r->stream));
   MG_CUDA (cudaStreamSynchronize (r->stream));
   return MG_OK;
}

extern "C" int mg_tecplot_fields (mg_run_t *r, double *E, double *H)
{
   if (!r) {
      mg_set_error ("mg_tecplot_fields: null run");
      return MG_ERR_ARG;
   }
   MG_CUDA (cudaSetDevice (r->device));
   // Between mg_em_HHalfStep and mg_em_HStep H is the array of H^n.
   const bool hn = r->stage_no >= 1 && r->stage_no <= 3;
   int rc = MG_OK;
   if (r->prm.precision == MG_FP64) {
      if (E) rc = tec_out<double> (r, r->E, 0, E);
      if (H && rc == MG_OK) rc = tec_out<double> (r, hn ? r->Hn : r->H, 1, H);
   } else {
      if (E) rc = tec_out<float> (r, r->E32, 0, E);
      if (H && rc == MG_OK) rc = tec_out<float> (r, hn ? r->Hn32 : r->H32, 1, H);
   }
   return rc;
}

extern "C" int mg_tecplot_currents (mg_run_t *r, double *J)
{
   if (!r || !J) {
      mg_set_error ("mg_tecplot_currents: null argument");
      return MG_ERR_ARG;
   }
   MG_CUDA (cudaSetDevice (r->device));
   return r->prm.precision == MG_FP64 ? tec_out<double> (r, r->J, 0, J) : tec_out<float> (r, r->J32, 0, J);
}
