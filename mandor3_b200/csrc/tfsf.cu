// Total-field / scattered-field interface (core/em_TFSF.c): record and play.
//
// Geometry (TFSF_init, core/em_TFSF.c:480-558).  For each axis a with
// tangential axes ep = (a+1)%3, eq = (a+2)%3, each side top and each of the
// two tangential components comp, face f = 4a + 2 top + comp:
//   E face: the interface box flattened to x_a = side[top], E component
//           c = (a + 1 + comp) % 3 with its lower bound along c raised by one
//           (the E node shift);
//   H face: the same nodes shifted by top along a, component 3 - c - a;
//   source factor (1 - 2 top)(1 - 2 comp) tau/h_a.
// A face's values are unrolled with ep slowest and eq fastest.  A frame is
// the 12 E faces' values then the 12 H faces', each face over its region.
//
// Record (TFSF_turnRec :229-283, TFSF_writeMesh :565-594): at the start of
// each step E^n and H^(n-1/2) times the source factor, faces cut to the
// domain (E to [0, n-1], H to [1, n]), into a device ring of frames.
//
// Play (TFSF_turnPlay :329-460, :669-853): after the H step the H faces
// get the recorded E of frame n (backward: T - n); after the E step the E
// faces get the recorded H of frame n + 1 (backward: T - n, subtracted).
// The boundary-slab caching of each H half step already calls the E
// post-step on the slabs (core/em_caps.c:602-608), which switches the
// interface off for good once frame n + 1 is the last (:831-834), so a step
// plays only while n + 1 < T - 1.  Open faces (openFaces.cfg) are skipped.
// The frames live in a device ring filled by the host; each slot records
// the frame it holds and a step that finds another frame there sets error
// flag 4 instead of reading it.
//
// Faces that share a node and component (edges of the box) add their
// values in face order, one thread per node and component.
#include <cuda_runtime.h>

#include <unordered_map>
#include <vector>

#include "mg_internal.cuh"

#define TRY_T(x)                                                             \
   do {                                                                      \
      int rc_ = (x);                                                         \
      if (rc_ != MG_OK)                                                      \
         return rc_;                                                         \
   } while (0)

struct TfsfFace {
   int min[3], max[3], comp, ep, eq, used;
   double sf;
   long long vol, at;
};

struct mg_tfsf_state {
   mg_tfsf_t cfg;
   TfsfFace face[24];
   long long frame_size;
   // play
   double *ring;
   int *slot_frame;
   // per field (0: E faces, 1: H faces): node offset, component, up to four
   // source indices in a frame (-1: none)
   long long *add_off[2];
   int *add_comp[2];
   int4 *add_src[2];
   int add_n[2];
   // record: one entry per frame value
   long long *rec_off;
   int *rec_comp;            // 0..2: E, 3..5: H
   double *rec_sf;
   double *rec_ring;         // MG_RING frames
};

namespace {

template <typename T>
struct Fields6 { T *c[6]; };

template <typename T>
__global__ void k_tfsf_add (Fields6<T> F, const long long *off, const int *comp, const int4 *src, int n,
                            const double *ring, const int *slot_frame, int slots, long long frame_size,
                            int is_e, int mode, int last, DevScalars *dsc)
{
   const int t = blockIdx.x*blockDim.x + threadIdx.x;
   if (t >= n)
      return;
   const int tf = dsc->tfsf_frame;
   if (tf + 1 >= last - 1)
      return;
   const int fr = (mode == MG_TFSF_PLAY_FORWARD) ? (is_e ? tf + 1 : tf) : last - 1 - tf;
   const int slot = fr % slots;
   if (slot_frame[slot] != fr) {
      if (atomicOr (&dsc->err, 4) == 0)
         dsc->err_info[0] = fr;
      return;
   }
   const double *v = ring + slot*frame_size;
   T *f = F.c[comp[t]] + off[t];
   const int4 s = src[t];
   const int q[4] = {s.x, s.y, s.z, s.w};
   T x = *f;
   if (is_e && mode == MG_TFSF_PLAY_BACKWARD) {
      for (int a = 0 ; a < 4 ; ++a)
         if (q[a] >= 0)
            x -= (T) v[q[a]];
   } else {
      for (int a = 0 ; a < 4 ; ++a)
         if (q[a] >= 0)
            x += (T) v[q[a]];
   }
   *f = x;
}

template <typename T>
__global__ void k_tfsf_rec (Fields6<T> F, const long long *off, const int *comp, const double *sf, long long n,
                            double *ring, const DevScalars *dsc)
{
   const long long t = blockIdx.x*(long long) blockDim.x + threadIdx.x;
   if (t >= n)
      return;
   ring[(long long) (dsc->step % MG_RING)*n + t] = (double) F.c[comp[t]][off[t]]*sf[t];
}

template <typename T>
Fields6<T> fields6 (T *const *E, T *const *H)
{
   Fields6<T> f;
   for (int c = 0 ; c < 3 ; ++c) {
      f.c[c] = E[c];
      f.c[3 + c] = H[c];
   }
   return f;
}

bool is32 (const mg_run_t *r) { return r->prm.precision == MG_FP32_OFFSET; }

bool playing (const mg_run_t *r)
{
   return r->tfsf && r->tfsf->cfg.mode != MG_TFSF_RECORD;
}

void free_state (mg_run_t *r, mg_tfsf_state *s)
{
   if (!s)
      return;
   void *p[] = {s->ring, s->slot_frame, s->add_off[0], s->add_off[1], s->add_comp[0], s->add_comp[1],
                s->add_src[0], s->add_src[1], s->rec_off, s->rec_comp, s->rec_sf, s->rec_ring};
   for (void *q : p)
      if (q)
         mg_dev_free (r, q);
   delete s;
}

template <typename V>
int upload (mg_run_t *r, V **dst, const std::vector<V> &src)
{
   *dst = nullptr;
   if (src.empty())
      return MG_OK;
   TRY_T (mg_dev_alloc (r, (void **) dst, sizeof (V)*src.size()));
   MG_CUDA (cudaMemcpy (*dst, src.data(), sizeof (V)*src.size(), cudaMemcpyHostToDevice));
   return MG_OK;
}

// Face geometry of TFSF_init with the mode's cuts; -1 when a played face is
// closer than 5 cells to a wall (TFSF_turnPlay :341-357).
int geometry (const mg_run_t *r, const mg_tfsf_t &t, TfsfFace face[24], long long *frame_size)
{
   const int *side[2] = {t.lo, t.hi};
   const Grid &g = r->g;
   for (int a = 0 ; a < 3 ; ++a)
      for (int top = 0 ; top < 2 ; ++top)
         for (int comp = 0 ; comp < 2 ; ++comp)
            for (int fh = 0 ; fh < 2 ; ++fh) {
               TfsfFace &F = face[4*a + 2*top + comp + 12*fh];
               for (int b = 0 ; b < 3 ; ++b) {
                  F.min[b] = t.lo[b];
                  F.max[b] = t.hi[b];
               }
               F.min[a] = F.max[a] = side[top][a];
               const int ce = (a + 1 + comp) % 3;
               F.min[ce] += 1;
               if (fh) {
                  F.min[a] += top;
                  F.max[a] += top;
               }
               F.comp = fh ? 3 - ce - a : ce;
               F.ep = (a + 1) % 3;
               F.eq = (a + 2) % 3;
               F.sf = (1 - 2*top)*(1 - 2*comp)*(g.tau/g.h[a]);
               if (t.mode == MG_TFSF_RECORD)
                  for (int b = 0 ; b < 3 ; ++b) {
                     const int lo = fh ? 1 : 0, hi = fh ? g.n[b] : g.n[b] - 1;
                     F.min[b] = F.min[b] < lo ? lo : F.min[b];
                     F.max[b] = F.max[b] > hi ? hi : F.max[b];
                  }
               long long v = 1;
               for (int b = 0 ; b < 3 ; ++b)
                  v *= (F.max[b] >= F.min[b]) ? F.max[b] - F.min[b] + 1 : 0;
               F.vol = v;
               F.used = v > 0 && !(t.mode != MG_TFSF_RECORD && t.open[top][a]);
               if (F.used && t.mode != MG_TFSF_RECORD)
                  for (int b = 0 ; b < 3 ; ++b)
                     if (F.min[b] < 5 || F.max[b] > g.n[b] - 5)
                        return -1;
            }
   long long at = 0;
   for (int q = 0 ; q < 24 ; ++q) {
      face[q].at = at;
      at += face[q].vol;
   }
   *frame_size = at;
   return 0;
}

template <typename Fn>
void scan_face (const mg_run_t *r, const TfsfFace &F, Fn fn)
{
   int c[3] = {F.min[0], F.min[1], F.min[2]};
   long long idx = 0;
   for (c[F.ep] = F.min[F.ep] ; c[F.ep] <= F.max[F.ep] ; ++c[F.ep])
      for (c[F.eq] = F.min[F.eq] ; c[F.eq] <= F.max[F.eq] ; ++c[F.eq], ++idx)
         fn ((long long) r->g.at (c[0], c[1], c[2]), idx);
}

} // namespace

extern "C" int mg_run_set_tfsf (mg_run_t *r, const mg_tfsf_t *t)
{
   if (!r) {
      mg_set_error ("mg_run_set_tfsf: null run");
      return MG_ERR_ARG;
   }
   MG_CUDA (cudaSetDevice (r->device));
   free_state (r, r->tfsf);
   r->tfsf = nullptr;
   mg_drop_graphs (r);
   if (!t)
      return MG_OK;
   if (t->mode != MG_TFSF_PLAY_FORWARD && t->mode != MG_TFSF_RECORD && t->mode != MG_TFSF_PLAY_BACKWARD) {
      mg_set_error ("mg_run_set_tfsf: mode %d (0 play forward, 1 record, 2 play backward)", t->mode);
      return MG_ERR_ARG;
   }
   for (int a = 0 ; a < 3 ; ++a)
      if (t->hi[a] < t->lo[a]) {
         mg_set_error ("mg_run_set_tfsf: bad interface region");
         return MG_ERR_ARG;
      }
   if (t->mode != MG_TFSF_RECORD && (t->frames < 0 || t->ring < 2)) {
      mg_set_error ("mg_run_set_tfsf: play needs frames >= 0 and a ring of at least 2 slots");
      return MG_ERR_ARG;
   }
   mg_tfsf_state *s = new mg_tfsf_state ();
   s->cfg = *t;
   if (geometry (r, *t, s->face, &s->frame_size) != 0) {
      delete s;
      mg_set_error ("mg_run_set_tfsf: TFSF interface is too close to a boundary (less than 5 cell)");
      return MG_ERR_ARG;
   }
   int rc = MG_OK;
   if (t->mode == MG_TFSF_RECORD) {
      std::vector<long long> off;
      std::vector<int> comp;
      std::vector<double> sf;
      for (int q = 0 ; q < 24 ; ++q) {
         const TfsfFace &F = s->face[q];
         if (!F.used)
            continue;
         scan_face (r, F, [&] (long long o, long long) {
            off.push_back (o);
            comp.push_back (F.comp + (q < 12 ? 0 : 3));
            sf.push_back (F.sf);
         });
      }
      if (rc == MG_OK) rc = upload (r, &s->rec_off, off);
      if (rc == MG_OK) rc = upload (r, &s->rec_comp, comp);
      if (rc == MG_OK) rc = upload (r, &s->rec_sf, sf);
      if (rc == MG_OK && s->frame_size > 0)
         rc = mg_dev_alloc (r, (void **) &s->rec_ring, sizeof (double)*(size_t) MG_RING*s->frame_size);
   } else {
      for (int fh = 0 ; fh < 2 && rc == MG_OK ; ++fh) {
         std::unordered_map<long long, int> at;
         std::vector<long long> off;
         std::vector<int> comp;
         std::vector<int4> src;
         for (int q = 12*fh ; q < 12*fh + 12 ; ++q) {
            const TfsfFace &F = s->face[q];
            if (!F.used)
               continue;
            const long long base = s->face[(q + 12) % 24].at;
            scan_face (r, F, [&] (long long o, long long idx) {
               const long long key = (long long) F.comp*r->g.total + o;
               auto it = at.find (key);
               if (it == at.end ()) {
                  it = at.emplace (key, (int) off.size ()).first;
                  off.push_back (o);
                  comp.push_back (F.comp + 3*fh);
                  src.push_back (make_int4 (-1, -1, -1, -1));
               }
               int4 &e = src[it->second];
               int *slot = e.x < 0 ? &e.x : e.y < 0 ? &e.y : e.z < 0 ? &e.z : &e.w;
               *slot = (int) (base + idx);
            });
         }
         s->add_n[fh] = (int) off.size ();
         if (rc == MG_OK) rc = upload (r, &s->add_off[fh], off);
         if (rc == MG_OK) rc = upload (r, &s->add_comp[fh], comp);
         if (rc == MG_OK) rc = upload (r, &s->add_src[fh], src);
      }
      if (rc == MG_OK && s->frame_size > 0)
         rc = mg_dev_alloc (r, (void **) &s->ring, sizeof (double)*(size_t) t->ring*s->frame_size);
      if (rc == MG_OK)
         rc = mg_dev_alloc (r, (void **) &s->slot_frame, sizeof (int)*t->ring);
      if (rc == MG_OK && cudaMemset (s->slot_frame, 0xff, sizeof (int)*t->ring) != cudaSuccess)
         rc = MG_ERR_CUDA;
   }
   if (rc != MG_OK) {
      free_state (r, s);
      return rc;
   }
   // Frame counter from the run's time (:455): (int) (t/tau + 0.1).
   double time = 0;
   MG_CUDA (cudaMemcpy (&time, &r->dsc->time, sizeof (double), cudaMemcpyDeviceToHost));
   const int frame = (int) (time/r->g.tau + 0.1);
   MG_CUDA (cudaMemcpy (&r->dsc->tfsf_frame, &frame, sizeof (int), cudaMemcpyHostToDevice));
   r->tfsf = s;
   return MG_OK;
}

extern "C" int mg_run_tfsf_faces (mg_run_t *r, int *regions, long long *frame_size)
{
   if (!r || !r->tfsf) {
      mg_set_error ("mg_run_tfsf_faces: no TF/SF interface on this run");
      return MG_ERR_STATE;
   }
   for (int q = 0 ; q < 24 && regions ; ++q)
      for (int b = 0 ; b < 3 ; ++b) {
         regions[6*q + b] = r->tfsf->face[q].min[b];
         regions[6*q + 3 + b] = r->tfsf->face[q].max[b];
      }
   if (frame_size)
      *frame_size = r->tfsf->frame_size;
   return MG_OK;
}

extern "C" int mg_run_tfsf_put_frames (mg_run_t *r, int first, int count, const double *frames)
{
   if (!r || !playing (r) || first < 0 || count < 0 || (count > 0 && !frames) ||
       count > r->tfsf->cfg.ring) {
      mg_set_error ("mg_run_tfsf_put_frames: bad arguments (a playing interface, at most ring frames)");
      return MG_ERR_ARG;
   }
   MG_CUDA (cudaSetDevice (r->device));
   mg_tfsf_state *s = r->tfsf;
   for (int k = 0 ; k < count ; ++k) {
      const int fr = first + k, slot = fr % s->cfg.ring;
      if (s->frame_size > 0)
         MG_CUDA (cudaMemcpyAsync (s->ring + (size_t) slot*s->frame_size, frames + (size_t) k*s->frame_size,
                                   sizeof (double)*s->frame_size, cudaMemcpyHostToDevice, r->stream));
      MG_CUDA (cudaMemcpyAsync (s->slot_frame + slot, &fr, sizeof (int), cudaMemcpyHostToDevice, r->stream));
      MG_CUDA (cudaStreamSynchronize (r->stream));      // fr lives on this stack frame
   }
   return MG_OK;
}

extern "C" int mg_run_tfsf_recorded (mg_run_t *r, int nsteps, double *out)
{
   if (!r || !r->tfsf || r->tfsf->cfg.mode != MG_TFSF_RECORD || nsteps < 0 || nsteps > MG_RING ||
       (nsteps > 0 && !out)) {
      mg_set_error ("mg_run_tfsf_recorded: bad arguments (a recording interface, at most %d steps)", MG_RING);
      return MG_ERR_ARG;
   }
   if (nsteps == 0 || r->tfsf->frame_size == 0)
      return MG_OK;
   MG_CUDA (cudaSetDevice (r->device));
   MG_CUDA (cudaMemcpyAsync (out, r->tfsf->rec_ring, sizeof (double)*(size_t) nsteps*r->tfsf->frame_size,
                             cudaMemcpyDeviceToHost, r->stream));
   MG_CUDA (cudaStreamSynchronize (r->stream));
   return MG_OK;
}

// ---- step hooks ------------------------------------------------------------

void mg_tfsf_free (mg_run_t *r)
{
   free_state (r, r->tfsf);
   r->tfsf = nullptr;
}

bool mg_tfsf_playing (const mg_run_t *r) { return playing (r); }

bool mg_tfsf_recording (const mg_run_t *r)
{
   return r->tfsf && r->tfsf->cfg.mode == MG_TFSF_RECORD;
}

static int add (mg_run_t *r, int fh)
{
   if (!playing (r) || r->tfsf->add_n[fh] == 0)
      return MG_OK;
   const mg_tfsf_state *s = r->tfsf;
   const int NT = 128, B = (s->add_n[fh] + NT - 1)/NT;
   if (is32 (r))
      k_tfsf_add<float><<<B, NT, 0, r->stream>>> (
         fields6<float> (r->E32, r->H32), s->add_off[fh], s->add_comp[fh], s->add_src[fh], s->add_n[fh], s->ring,
         s->slot_frame, s->cfg.ring, s->frame_size, fh == 0, s->cfg.mode, s->cfg.frames, r->dsc);
   else
      k_tfsf_add<double><<<B, NT, 0, r->stream>>> (
         fields6<double> (r->E, r->H), s->add_off[fh], s->add_comp[fh], s->add_src[fh], s->add_n[fh], s->ring,
         s->slot_frame, s->cfg.ring, s->frame_size, fh == 0, s->cfg.mode, s->cfg.frames, r->dsc);
   MG_LAUNCH_CHECK ();
   return MG_OK;
}

// After the H step (core/em.c:125), before the sources.
int mg_tfsf_h (mg_run_t *r) { return add (r, 1); }

// After the E step and its walls (core/em.c:200), before the sources and
// the currents.
int mg_tfsf_e (mg_run_t *r) { return add (r, 0); }

// E^n and H^(n-1/2) at the start of the step (core/em.c:92).
int mg_tfsf_record (mg_run_t *r)
{
   if (!mg_tfsf_recording (r) || r->tfsf->frame_size == 0)
      return MG_OK;
   const mg_tfsf_state *s = r->tfsf;
   const int NT = 256;
   const int B = (int) ((s->frame_size + NT - 1)/NT);
   if (is32 (r))
      k_tfsf_rec<float><<<B, NT, 0, r->stream>>> (fields6<float> (r->E32, r->H32), s->rec_off, s->rec_comp,
                                                  s->rec_sf, s->frame_size, s->rec_ring, r->dsc);
   else
      k_tfsf_rec<double><<<B, NT, 0, r->stream>>> (fields6<double> (r->E, r->H), s->rec_off, s->rec_comp,
                                                   s->rec_sf, s->frame_size, s->rec_ring, r->dsc);
   MG_LAUNCH_CHECK ();
   return MG_OK;
}
