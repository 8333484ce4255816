/* Test infrastructure: the reference's [DF:uniform] tag
 * (setup/tag_DF_uniform.c, linked unchanged from the reference sources by
 * oracle/Makefile) on a marker array of ours.  The tag draws from the C
 * library's rand () (3 draws per marker, vx then vy then vz, from the
 * default seed); `skip` draws are taken first, standing for the tags of a
 * deck that drew before it.  The plasma object and the particles-per-cell
 * count that setup/plasma.c and setup/tag_plasma.c would provide are
 * defined here (PPC fixed at 4).
 *
 *   df_uniform.out lambda_um markers skip deck
 *
 * deck: the tag's eight "@ value" lines; prints "vx vy vz rho qDivM"
 * (%.17g) per marker. */
#include <stdio.h>
#include <stdlib.h>

#include "type_marker.h"
#include "misc_units.h"

void tag_DF_uniform (FILE *fp);

const int plasma_nx = 1, plasma_ny = 1, plasma_nz = 1, plasma_layers = 4, plasma_PPC = 4;
const int memEstimateOnly = 0;

static marker_t *markers;
static long int count;

marker_t *plasma_getObject (int obj, long int *N)
{
   *N = obj == 0 ? count : 0;
   return obj == 0 ? markers : NULL;
}

int main (int argc, char **argv)
{
   if (argc != 5) {
      fprintf (stderr, "usage: %s lambda_um markers skip deck\n", argv[0]);
      return 2;
   }
   units_setLambda (atof (argv[1])*1.0e-4);            /* setup/tag_units.c: microns */
   count = atol (argv[2]);
   const long skip = atol (argv[3]);
   markers = (marker_t *) calloc (count > 0 ? count : 1, sizeof (marker_t));
   for (long q = 0 ; q < skip ; ++q)
      (void) rand ();
   FILE *fp = fopen (argv[4], "rt");
   if (!fp)
      return 3;
   tag_DF_uniform (fp);
   fclose (fp);
   for (long q = 0 ; q < count ; ++q)
      printf ("%.17g %.17g %.17g %.17g %.17g\n", markers[q].vx, markers[q].vy, markers[q].vz,
              (double) markers[q].rho, (double) markers[q].qDivM);
   return 0;
}
