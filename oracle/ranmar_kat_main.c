/* Driver for the reference ranmar generator (misc_ranmar.c:79-146), test
 * infrastructure only.  Usage:
 *   ranmar_kat.out                -> prints the six known-answer values
 *                                    (misc_ranmar.c:37-56) after 20000 draws
 *   ranmar_kat.out IJ KL N FILE   -> writes the first N draws of stream
 *                                    (IJ, KL) to FILE as raw doubles
 */
#include <stdio.h>
#include <stdlib.h>

#include "misc_ranmar.h"

int main (int argc, char **argv)
{
   if (argc == 5) {
      int ij = atoi (argv[1]), kl = atoi (argv[2]);
      long n = atol (argv[3]);
      double *v = (double *) malloc (sizeof (double)*(n > 0 ? n : 1));
      ranmar_init (ij, kl);
      for (long done = 0 ; done < n ; ) {
         int chunk = (n - done > 1000000) ? 1000000 : (int) (n - done);
         ranmar (v + done, chunk);
         done += chunk;
      }
      FILE *fp = fopen (argv[4], "wb");
      if (!fp)
         return 1;
      fwrite (v, sizeof (double), (size_t) n, fp);
      fclose (fp);
      free (v);
      return 0;
   }
   double temp[100];
   ranmar_init (1802, 9373);
   for (int i = 0 ; i < 200 ; i++)
      ranmar (temp, 100);
   ranmar (temp, 6);
   for (int i = 0 ; i < 6 ; i++)
      printf ("%.1f\n", 4096.0*4096.0*temp[i]);
   return 0;
}
