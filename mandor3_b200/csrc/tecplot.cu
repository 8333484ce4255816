// Node-centred field dumps for tecplot.out (IO_tecplot.c:108-153): over the
// nodes [0, n]^3, E-type meshes (E, J) as 0.5 (F[p] + F[p + d_c]) per
// component c, H as the 4-point average in the two other axes, summed in the
// reference's order; FP64 arithmetic in both precision forms.
#include <cuda_runtime.h>

#include "mg_internal.cuh"

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

} // namespace

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
