// FP64 instantiation of the field kernels (fields_tmpl.cuh): the
// reference's arithmetic, compiled with --fmad=false.
#include "fields_tmpl.cuh"

static FS<double> fs_of (mg_run_t *r)
{
   FS<double> fs;
   for (int c = 0 ; c < 3 ; ++c) {
      fs.E[c] = r->E[c];
      fs.H[c] = r->H[c];
      fs.Hn[c] = r->Hn[c];
      fs.J[c] = r->J[c];
      fs.mur[0][c] = r->mur[0][c];
      fs.mur[1][c] = r->mur[1][c];
   }
   return fs;
}

int mg_fields64_h_half (mg_run_t *r) { return fields_h_half<double> (r, fs_of (r)); }
int mg_fields64_energy (mg_run_t *r) { return fields_energy<double> (r, fs_of (r)); }
int mg_fields64_h_step (mg_run_t *r) { return fields_h_step<double> (r, fs_of (r)); }
int mg_fields64_h_both (mg_run_t *r) { return fields_h_both<double> (r, fs_of (r)); }
int mg_fields64_e_step (mg_run_t *r) { return fields_e_step<double> (r, fs_of (r)); }
int mg_fields64_jbc (mg_run_t *r) { return fields_jbc<double> (r, fs_of (r)); }
int mg_fields64_jbc_graph (mg_run_t *r) { return fields_jbc_graph<double> (r, fs_of (r)); }
int mg_fields64_e_finish (mg_run_t *r) { return fields_e_finish<double> (r, fs_of (r)); }
int mg_fields64_e_fused (mg_run_t *r) { return fields_e_fused<double> (r, fs_of (r)); }
int mg_fields64_zero_j (mg_run_t *r) { return fields_zero_j<double> (r, fs_of (r)); }
int mg_fields64_init (mg_run_t *r) { return fields_init<double> (r, fs_of (r)); }
int mg_fields64_one_pass (mg_run_t *r) { return fields_one_pass<double> (r, fs_of (r), r->Ealt, r->Halt); }
