// FP64 Yee solver, field boundary conditions, current folding and energy
// reductions of the B200 PIC core.
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
// Arithmetic is compiled with --fmad=false so that every expression rounds
// exactly as the reference's C does.
#include <cuda_runtime.h>

#include "mg_internal.cuh"

namespace {

struct F3 {
   double *c[3];
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

// H += frac*tau*(-curl E) over the H box (core/em.c:67-76 expression order).
__global__ void k_h_advance (Grid g, F3 E, F3 H, Box b, double c1, double c2, double c3)
{
   const double *Ex = E.c[0], *Ey = E.c[1], *Ez = E.c[2];
   double *Hx = H.c[0], *Hy = H.c[1], *Hz = H.c[2];
   const long sx = g.sx, sy = g.sy;
   for (long t = blockIdx.x*(long) blockDim.x + threadIdx.x ; t < b.vol ; t += (long) gridDim.x*blockDim.x) {
      int i, j, k;
      box_index (t, b.lo, b.ext, i, j, k);
      const long o = g.at (i, j, k);
      const double ex = Ex[o], ey = Ey[o], ez = Ez[o];
      Hx[o] += c3*(ey - Ey[o - 1]) - c2*(ez - Ez[o - sy]);
      Hy[o] += c1*(ez - Ez[o - sx]) - c3*(ex - Ex[o - 1]);
      Hz[o] += c2*(ex - Ex[o - sy]) - c1*(ey - Ey[o - sx]);
   }
}

// E -= tau*(curl H) over the E box (core/em.c:155-162 expression order).
__global__ void k_e_advance (Grid g, F3 E, F3 H, Box b, double c1, double c2, double c3)
{
   double *Ex = E.c[0], *Ey = E.c[1], *Ez = E.c[2];
   const double *Hx = H.c[0], *Hy = H.c[1], *Hz = H.c[2];
   const long sx = g.sx, sy = g.sy;
   for (long t = blockIdx.x*(long) blockDim.x + threadIdx.x ; t < b.vol ; t += (long) gridDim.x*blockDim.x) {
      int i, j, k;
      box_index (t, b.lo, b.ext, i, j, k);
      const long o = g.at (i, j, k);
      const double hx = Hx[o], hy = Hy[o], hz = Hz[o];
      Ex[o] -= c3*(Hy[o + 1] - hy) - c2*(Hz[o + sy] - hz);
      Ey[o] -= c1*(Hz[o + sx] - hz) - c3*(Hx[o + 1] - hx);
      Ez[o] -= c2*(Hx[o + sy] - hx) - c1*(Hy[o + sx] - hy);
   }
}

// Wall kernels run over the two transverse axes, nodes [0, n+1] each (the
// flush extent of the reference's caps, core/em_caps.c:140-146).
struct Wall {
   int ea, ep, eq;
   int np_, nq_;           // extents n[ep]+2, n[eq]+2
   long s_a, s_p, s_q;     // strides along the three axes
};

static Wall make_wall (const Grid &g, int ea)
{
   Wall w;
   w.ea = ea;
   w.ep = (ea + 1) % 3;
   w.eq = (ea + 2) % 3;
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

// H wall operations (core/emCap_periodic.c:15-37, emCap_mirror.c:17-40,
// emCap_Mur.c:56-80).
__global__ void k_h_wall (Grid g, F3 H, Wall w, int op)
{
   long o;
   int p, q;
   const int N = g.n[w.ea];
   if (!wall_node (g, w, 0, o, p, q))
      return;
   double *Ha = H.c[w.ea], *Hp = H.c[w.ep], *Hq = H.c[w.eq];
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
__global__ void k_e_wall (Grid g, F3 E, Wall w, int op, double *mur, double alpha)
{
   long o;
   int p, q;
   const int N = g.n[w.ea];
   if (!wall_node (g, w, 0, o, p, q))
      return;
   double *Ea = E.c[w.ea], *Ep = E.c[w.ep], *Eq = E.c[w.eq];
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
      double *h = mur + 4*((long) p*w.nq_ + q);
      if (top)
         Ea[o + w.s_a] = Ea[o];
      else
         Ea[o] = Ea[o + w.s_a];
      const double ep = h[2] + alpha*(Ep[in] - h[0]);
      const double eq = h[3] + alpha*(Eq[in] - h[1]);
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
__global__ void k_mur_init (Grid g, F3 E, Wall w, int top, double *mur)
{
   long o;
   int p, q;
   const int N = g.n[w.ea];
   if (!wall_node (g, w, 0, o, p, q))
      return;
   if (top)
      o += N*w.s_a;
   const long in = top ? o - w.s_a : o + w.s_a;
   double *h = mur + 4*((long) p*w.nq_ + q);
   h[0] = E.c[w.ep][o];
   h[1] = E.c[w.eq][o];
   h[2] = E.c[w.ep][in];
   h[3] = E.c[w.eq][in];
   if (top)
      E.c[w.ea][o + w.s_a] = E.c[w.ea][o];
   else
      E.c[w.ea][o] = E.c[w.ea][o + w.s_a];
}

// Current folding, periodic pair of walls (plasma_currentWalls.c:53-75):
// five layers around the lower wall are added into their images at the upper
// wall and copied back; transverse extent [-2, n+2].
__global__ void k_j_periodic (Grid g, F3 J, int ea)
{
   const int ep = (ea == 0) ? 1 : 0, eq = (ea == 2) ? 1 : 2;
   const int np_ = g.n[ep] + 5, nq_ = g.n[eq] + 5;
   const long t = blockIdx.x*(long) blockDim.x + threadIdx.x;
   if (t >= (long) np_*nq_)
      return;
   const long s[3] = {g.sx, g.sy, 1};
   const int p = (int) (t / nq_) - 2, q = (int) (t % nq_) - 2;
   const long base = g.origin + p*s[ep] + q*s[eq];
   const long shift = (long) g.n[ea]*s[ea];
   for (int a = -2 ; a <= 2 ; ++a) {
      const long o = base + a*s[ea];
      for (int c = 0 ; c < 3 ; ++c) {
         const double v = J.c[c][o + shift] + J.c[c][o];
         J.c[c][o + shift] = v;
         J.c[c][o] = v;
      }
   }
}

// Current folding at a mirror or open wall (plasma_currentWalls.c:78-111).
__global__ void k_j_wall (Grid g, F3 J, int ea, int top)
{
   const int ep = (ea == 0) ? 1 : 0, eq = (ea == 2) ? 1 : 2;
   const int np_ = g.n[ep] + 5, nq_ = g.n[eq] + 5;
   const long t = blockIdx.x*(long) blockDim.x + threadIdx.x;
   if (t >= (long) np_*nq_)
      return;
   const long s[3] = {g.sx, g.sy, 1};
   const int p = (int) (t / nq_) - 2, q = (int) (t % nq_) - 2;
   const long o = g.origin + (top ? g.n[ea] : 0)*s[ea] + p*s[ep] + q*s[eq];
   const long st = s[ea];
   const long internal = (1 - top)*st, external = top*st, out = st*(2*top - 1);
   double *Ja = J.c[ea], *Jp = J.c[ep], *Jq = J.c[eq];
   Ja[o + internal] -= Ja[o + external];
   Jp[o - out] += Jp[o + out];
   Jq[o - out] += Jq[o + out];
   Ja[o + internal - out] -= Ja[o + external + out];
   Jp[o - 2*out] += Jp[o + 2*out];
   Jq[o - 2*out] += Jq[o + 2*out];
   Jp[o] = 0;
   Jq[o] = 0;
   Ja[o + external] = Ja[o + internal];
   Jp[o + out] = -Jp[o - out];
   Jq[o + out] = -Jq[o - out];
   Ja[o + external + out] = Ja[o + internal - out];
   Jp[o + 2*out] = -Jp[o - 2*out];
   Jq[o + 2*out] = -Jq[o - 2*out];
}

// E -= tau*J over [-1, n+1]^3 (core/em.c:167-184).
__global__ void k_e_sub_j (Grid g, F3 E, F3 J, Box b)
{
   const double tau = g.tau;
   for (long t = blockIdx.x*(long) blockDim.x + threadIdx.x ; t < b.vol ; t += (long) gridDim.x*blockDim.x) {
      int i, j, k;
      box_index (t, b.lo, b.ext, i, j, k);
      const long o = g.at (i, j, k);
      E.c[0][o] -= tau*J.c[0][o];
      E.c[1][o] -= tau*J.c[1][o];
      E.c[2][o] -= tau*J.c[2][o];
   }
}

__device__ __forceinline__ double warp_sum (double v)
{
   for (int d = 16 ; d > 0 ; d >>= 1)
      v += __shfl_xor_sync (0xffffffffu, v, d);
   return v;
}

// Field energy at t = n*tau (core/em.c:227-252): sums of squares of the
// staggered picks, reduced per block and added into acc[0], acc[1].
__global__ void k_energy (Grid g, F3 E, F3 H, Box b, DevScalars *dsc)
{
   __shared__ double sw[2][32];
   const long sx = g.sx, sy = g.sy;
   double we = 0, wb = 0;
   for (long t = blockIdx.x*(long) blockDim.x + threadIdx.x ; t < b.vol ; t += (long) gridDim.x*blockDim.x) {
      int i, j, k;
      box_index (t, b.lo, b.ext, i, j, k);
      const long o = g.at (i, j, k);
      const double ex = E.c[0][o + sx], ey = E.c[1][o + sy], ez = E.c[2][o + 1];
      const double hx = H.c[0][o + sy + 1], hy = H.c[1][o + sx + 1], hz = H.c[2][o + sx + sy];
      we += ex*ex + ey*ey + ez*ez;
      wb += hx*hx + hy*hy + hz*hz;
   }
   we = warp_sum (we);
   wb = warp_sum (wb);
   const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
   if (lane == 0) {
      sw[0][wid] = we;
      sw[1][wid] = wb;
   }
   __syncthreads ();
   if (wid == 0) {
      const int nw = blockDim.x >> 5;
      we = lane < nw ? sw[0][lane] : 0;
      wb = lane < nw ? sw[1][lane] : 0;
      we = warp_sum (we);
      wb = warp_sum (wb);
      if (lane == 0) {
         atomicAdd (&dsc->acc[0], we);
         atomicAdd (&dsc->acc[1], wb);
      }
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
__global__ void k_laser (Grid g, double *F, mg_laser_t l, const DevScalars *dsc,
                         int is_e)
{
   const int nj = g.n[1] - 2*l.margin + 1, nk = g.n[2] - 2*l.margin + 1;
   const long t = blockIdx.x*(long) blockDim.x + threadIdx.x;
   if (nj <= 0 || nk <= 0 || t >= (long) nj*nk)
      return;
   const int j = l.margin + (int) (t / nk), k = l.margin + (int) (t % nk);
   const double ymid = 0.5*g.n[1]*g.h[1], zmid = 0.5*g.n[2]*g.h[2];
   const double c1 = g.tau/g.h[0];
   const double time = dsc->time + (is_e ? 0.5*g.tau : 0.0);
   const double x = is_e ? (l.plane - 0.5)*g.h[0] : (l.plane - 1)*g.h[0];
   const int i = is_e ? l.plane - 1 : l.plane;
   const double v = laser_ey (l, x, (j - 0.5)*g.h[1], k*g.h[2], time, ymid, zmid);
   F[g.at (i, j, k)] += c1*v;
}

static F3 f3 (double *const c[3])
{
   F3 f;
   for (int a = 0 ; a < 3 ; ++a)
      f.c[a] = c[a];
   return f;
}

static int launch_box_h (mg_run_t *r, double frac)
{
   const Grid &g = r->g;
   int lo[3], hi[3];
   for (int a = 0 ; a < 3 ; ++a) {
      lo[a] = (g.bc[0][a] == MG_BC_MIRROR) ? 1 : 0;
      hi[a] = g.n[a];
   }
   Box b = make_box (lo, hi);
   const int T = 256;
   k_h_advance<<<mg_blocks_for (b.vol, T, 16), T, 0, r->stream>>> (
      g, f3 (r->E), f3 (r->H), b, frac*g.tau/g.h[0], frac*g.tau/g.h[1], frac*g.tau/g.h[2]);
   MG_LAUNCH_CHECK ();
   return MG_OK;
}

static int launch_walls (mg_run_t *r, int is_e)
{
   const Grid &g = r->g;
   for (int ea = 0 ; ea < 3 ; ++ea) {
      Wall w = make_wall (g, ea);
      const long nodes = (long) w.np_*w.nq_;
      const int T = 256, B = (int) ((nodes + T - 1)/T);
      const double alpha = (g.tau - g.h[ea])/(g.tau + g.h[ea]);
      for (int top = 0 ; top < 2 ; ++top) {
         const int bc = g.bc[top][ea];
         int op;
         if (bc == MG_BC_PERIODIC) {
            if (top)
               continue;
            op = OP_PERIODIC;
         } else if (bc == MG_BC_MIRROR) {
            op = top ? OP_MIRROR_MAX : OP_MIRROR_MIN;
         } else {
            op = top ? OP_OPEN_MAX : OP_OPEN_MIN;
         }
         if (is_e)
            k_e_wall<<<B, T, 0, r->stream>>> (g, f3 (r->E), w, op, r->mur[top][ea], alpha);
         else
            k_h_wall<<<B, T, 0, r->stream>>> (g, f3 (r->H), w, op);
         MG_LAUNCH_CHECK ();
      }
   }
   return MG_OK;
}

static int launch_laser (mg_run_t *r, int is_e)
{
   if (!r->has_laser)
      return MG_OK;
   const mg_laser_t &l = r->laser;
   const long nj = r->g.n[1] - 2*l.margin + 1, nk = r->g.n[2] - 2*l.margin + 1;
   if (nj <= 0 || nk <= 0)
      return MG_OK;
   const int T = 256, B = (int) ((nj*nk + T - 1)/T);
   k_laser<<<B, T, 0, r->stream>>> (r->g, is_e ? r->E[1] : r->H[2], l, r->dsc, is_e);
   MG_LAUNCH_CHECK ();
   return MG_OK;
}

} // namespace

int mg_fields64_h_half (mg_run_t *r)
{
   int rc = launch_box_h (r, 0.5);
   if (rc) return rc;
   return launch_walls (r, 0);
}

int mg_fields64_energy (mg_run_t *r)
{
   const int lo[3] = {0, 0, 0};
   const int hi[3] = {r->g.n[0] - 1, r->g.n[1] - 1, r->g.n[2] - 1};
   Box b = make_box (lo, hi);
   const int T = 256;
   k_energy<<<mg_blocks_for (b.vol, T, 4), T, 0, r->stream>>> (r->g, f3 (r->E), f3 (r->H), b, r->dsc);
   MG_LAUNCH_CHECK ();
   return MG_OK;
}

int mg_fields64_h_step (mg_run_t *r)
{
   int rc = launch_box_h (r, 0.5);
   if (rc) return rc;
   rc = launch_laser (r, 0);
   if (rc) return rc;
   return launch_walls (r, 0);
}

int mg_fields64_e_step (mg_run_t *r)
{
   const Grid &g = r->g;
   int lo[3], hi[3];
   for (int a = 0 ; a < 3 ; ++a) {
      lo[a] = (g.bc[0][a] == MG_BC_PERIODIC) ? 0 : 1;
      hi[a] = (g.bc[1][a] == MG_BC_PERIODIC) ? g.n[a] - 1 : g.n[a];
   }
   Box b = make_box (lo, hi);
   const int T = 256;
   k_e_advance<<<mg_blocks_for (b.vol, T, 16), T, 0, r->stream>>> (
      g, f3 (r->E), f3 (r->H), b, g.tau/g.h[0], g.tau/g.h[1], g.tau/g.h[2]);
   MG_LAUNCH_CHECK ();
   return launch_walls (r, 1);
}

int mg_fields64_jbc (mg_run_t *r)
{
   const Grid &g = r->g;
   for (int f = 0 ; f < 6 ; ++f) {
      const int ea = f >> 1, top = f & 1;
      const int ep = (ea == 0) ? 1 : 0, eq = (ea == 2) ? 1 : 2;
      const long nodes = (long) (g.n[ep] + 5)*(g.n[eq] + 5);
      const int T = 256, B = (int) ((nodes + T - 1)/T);
      if (g.bc[top][ea] == MG_BC_PERIODIC) {
         if (!top)
            k_j_periodic<<<B, T, 0, r->stream>>> (g, f3 (r->J), ea);
      } else {
         k_j_wall<<<B, T, 0, r->stream>>> (g, f3 (r->J), ea, top);
      }
      MG_LAUNCH_CHECK ();
   }
   return MG_OK;
}

int mg_fields64_e_finish (mg_run_t *r)
{
   int rc = launch_laser (r, 1);
   if (rc) return rc;
   const int lo[3] = {-1, -1, -1};
   const int hi[3] = {r->g.n[0] + 1, r->g.n[1] + 1, r->g.n[2] + 1};
   Box b = make_box (lo, hi);
   const int T = 256;
   k_e_sub_j<<<mg_blocks_for (b.vol, T, 16), T, 0, r->stream>>> (r->g, f3 (r->E), f3 (r->J), b);
   MG_LAUNCH_CHECK ();
   return MG_OK;
}

int mg_fields64_zero_j (mg_run_t *r)
{
   for (int c = 0 ; c < 3 ; ++c)
      MG_CUDA (cudaMemsetAsync (r->J[c], 0, r->g.total*sizeof (double), r->stream));
   return MG_OK;
}

// cap_init equivalent (core/em_caps.c:343-392), axis by axis.
int mg_fields64_init (mg_run_t *r)
{
   const Grid &g = r->g;
   for (int ea = 0 ; ea < 3 ; ++ea) {
      Wall w = make_wall (g, ea);
      const long nodes = (long) w.np_*w.nq_;
      const int T = 256, B = (int) ((nodes + T - 1)/T);
      if (g.bc[0][ea] == MG_BC_PERIODIC) {
         k_h_wall<<<B, T, 0, r->stream>>> (g, f3 (r->H), w, OP_PERIODIC);
         k_e_wall<<<B, T, 0, r->stream>>> (g, f3 (r->E), w, OP_PERIODIC, nullptr, 0.0);
         MG_LAUNCH_CHECK ();
         continue;
      }
      for (int top = 0 ; top < 2 ; ++top) {
         if (g.bc[top][ea] == MG_BC_MIRROR) {
            const int op = top ? OP_MIRROR_MAX : OP_MIRROR_MIN;
            k_h_wall<<<B, T, 0, r->stream>>> (g, f3 (r->H), w, op);
            k_e_wall<<<B, T, 0, r->stream>>> (g, f3 (r->E), w, op, nullptr, 0.0);
         } else if (g.bc[top][ea] == MG_BC_OPEN) {
            k_mur_init<<<B, T, 0, r->stream>>> (g, f3 (r->E), w, top, r->mur[top][ea]);
         }
         MG_LAUNCH_CHECK ();
      }
   }
   return MG_OK;
}
