/* Test infrastructure: the velocity pattern of the reference's Maxwell
 * quiet start (setup/tag_maxwell.c:84-158) built on the reference's own
 * sampler and mapper (setup/setup_denavit.c, setup/setup_distrMapper.c,
 * linked from the reference sources by oracle/Makefile).  The pattern loop
 * itself is restated here because tag_maxwell.c keeps it in a static
 * function; it is a few lines of arithmetic, in the reference's order.
 *
 *   maxwell_pattern.out nx ny nz layers omega_pe2 qDivM ux uy uz tune uniform
 *
 * prints one line "vx vy vz rho" (%.17g) per marker of the cell pattern. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "setup/setup_denavit.h"
#include "setup/setup_distrMapper.h"

static double f_maxwell (double x) { return exp (- x*x); }

int main (int argc, char **argv)
{
   if (argc != 12) {
      fprintf (stderr, "usage: %s nx ny nz layers omega_pe2 qDivM ux uy uz tune uniform\n", argv[0]);
      return 2;
   }
   const int nx = atoi (argv[1]), ny = atoi (argv[2]), nz = atoi (argv[3]), layers = atoi (argv[4]);
   const double w2 = atof (argv[5]), qDivM = atof (argv[6]);
   const double ux = atof (argv[7]), uy = atof (argv[8]), uz = atof (argv[9]);
   const int tune = atoi (argv[10]), uniform = atoi (argv[11]);
   const int PPC = nx*ny*nz*layers;
   const double pi = 3.141592653589793238462643;
   const double rho = w2*4*pi*pi/qDivM/(double) PPC;
   mapper_t *all = mapper_create (f_maxwell, -6.0, +6.0, 5000);
   mapper_t *pos = mapper_create (f_maxwell, 0, +6.0, 5000);
   double *vx_ = malloc (sizeof (double)*PPC), *vy_ = malloc (sizeof (double)*PPC),
          *vz_ = malloc (sizeof (double)*PPC), *r_ = malloc (sizeof (double)*PPC);
   for (int i = 0, p = 0 ; i < nx ; ++i)
      for (int j = 0 ; j < ny ; ++j)
         for (int k = 0 ; k < nz ; ++k)
            for (int l = 0 ; l < layers/2 ; ++l) {
               double vx, vy, vz, tmp;
               denavit_createQuartet (p/2, PPC/2, &tmp, &vx, &vy, &vz);
               if (uniform) {
                  vx = mapper_invoke (vx, pos);
                  vy = mapper_invoke (vy, all);
                  vz = mapper_invoke (vz, all);
                  r_[p] = 1.0;
               } else {
                  vx *= 1.6;
                  vy = 1.6*2*(vy - 0.5);
                  vz = 1.6*2*(vz - 0.5);
                  r_[p] = f_maxwell (vx)*f_maxwell (vy)*f_maxwell (vz);
               }
               vx_[p] = vx*ux; vy_[p] = vy*uy; vz_[p] = vz*uz;
               ++p;
               vx_[p] = - vx*ux; vy_[p] = - vy*uy; vz_[p] = - vz*uz;
               r_[p] = r_[p - 1];
               ++p;
            }
   double norm = 0;
   for (int p = 0 ; p < PPC ; ++p)
      norm += r_[p];
   norm = PPC*rho/norm;
   for (int p = 0 ; p < PPC ; ++p)
      r_[p] *= norm;
   if (tune) {
      double Wx = 0, Wy = 0, Wz = 0;
      for (int p = 0 ; p < PPC ; ++p) {
         Wx += vx_[p]*vx_[p]*r_[p];
         Wy += vy_[p]*vy_[p]*r_[p];
         Wz += vz_[p]*vz_[p]*r_[p];
      }
      Wx = ux*sqrt (rho*PPC*0.5/Wx);
      Wy = uy*sqrt (rho*PPC*0.5/Wy);
      Wz = uz*sqrt (rho*PPC*0.5/Wz);
      for (int p = 0 ; p < PPC ; ++p) {
         vx_[p] *= Wx;
         vy_[p] *= Wy;
         vz_[p] *= Wz;
      }
   }
   for (int p = 0 ; p < PPC ; ++p)
      printf ("%.17g %.17g %.17g %.17g\n", vx_[p], vy_[p], vz_[p], r_[p]);
   mapper_destroy (all);
   mapper_destroy (pos);
   return 0;
}
