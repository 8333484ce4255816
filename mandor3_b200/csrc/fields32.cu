// FP32 instantiation of the field kernels (fields_tmpl.cuh) for the
// precision form: FP32 E, H, J and Mur history, FP64 energy sums.
#include "fields_tmpl.cuh"

static FS<float> fs_of (mg_run_t *r)
{
   FS<float> fs;
   for (int c = 0 ; c < 3 ; ++c) {
      fs.E[c] = r->E32[c];
      fs.H[c] = r->H32[c];
      fs.Hn[c] = r->Hn32[c];
      fs.J[c] = r->J32[c];
      fs.mur[0][c] = r->mur32[0][c];
      fs.mur[1][c] = r->mur32[1][c];
   }
   return fs;
}

int mg_fields32_h_half (mg_run_t *r) { return fields_h_half<float> (r, fs_of (r)); }
int mg_fields32_energy (mg_run_t *r) { return fields_energy<float> (r, fs_of (r)); }
int mg_fields32_h_step (mg_run_t *r) { return fields_h_step<float> (r, fs_of (r)); }
int mg_fields32_h_both (mg_run_t *r) { return fields_h_both<float> (r, fs_of (r)); }
int mg_fields32_e_step (mg_run_t *r) { return fields_e_step<float> (r, fs_of (r)); }
int mg_fields32_jbc (mg_run_t *r) { return fields_jbc<float> (r, fs_of (r)); }
int mg_fields32_jbc_graph (mg_run_t *r) { return fields_jbc_graph<float> (r, fs_of (r)); }
int mg_fields32_e_finish (mg_run_t *r) { return fields_e_finish<float> (r, fs_of (r)); }
int mg_fields32_e_fused (mg_run_t *r) { return fields_e_fused<float> (r, fs_of (r)); }
int mg_fields32_zero_j (mg_run_t *r) { return fields_zero_j<float> (r, fs_of (r)); }
int mg_fields32_init (mg_run_t *r) { return fields_init<float> (r, fs_of (r)); }
int mg_fields32_one_pass (mg_run_t *r) { return fields_one_pass<float> (r, fs_of (r), r->Ealt32, r->Halt32); }
