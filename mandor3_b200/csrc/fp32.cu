// Precision form (int cell + FP32 offset): placeholder entry points until
// the form is built; every call fails loudly.
#include "mg_internal.cuh"

#define NOT_BUILT(name)                                                      \
   do {                                                                      \
      mg_set_error ("%s: the FP32-offset form is not available", name);      \
      return MG_ERR_ARG;                                                     \
   } while (0)

int mg_run_create32 (const mg_params_t *, mg_run_t **) { NOT_BUILT ("mg_run_create"); }
int mg_run_destroy32 (mg_run_t *) { NOT_BUILT ("mg_run_destroy"); }
int mg_run_set_fields32 (mg_run_t *, const double *, const double *) { NOT_BUILT ("set_fields"); }
int mg_run_get_fields32 (mg_run_t *, double *, double *) { NOT_BUILT ("get_fields"); }
int mg_run_get_current32 (mg_run_t *, double *) { NOT_BUILT ("get_current"); }
int mg_run_set_markers32 (mg_run_t *, const mg_marker_t *, long long) { NOT_BUILT ("set_markers"); }
int mg_run_get_markers32 (mg_run_t *, mg_marker_t *, long long, long long *) { NOT_BUILT ("get_markers"); }
int mg_plasma_rho32 (mg_run_t *, double *) { NOT_BUILT ("rho"); }
int mg_fields32_h_half (mg_run_t *) { NOT_BUILT ("h_half"); }
int mg_fields32_energy (mg_run_t *) { NOT_BUILT ("energy"); }
int mg_fields32_h_step (mg_run_t *) { NOT_BUILT ("h_step"); }
int mg_fields32_e_step (mg_run_t *) { NOT_BUILT ("e_step"); }
int mg_fields32_jbc (mg_run_t *) { NOT_BUILT ("jbc"); }
int mg_fields32_e_finish (mg_run_t *) { NOT_BUILT ("e_finish"); }
int mg_fields32_init (mg_run_t *) { NOT_BUILT ("init"); }
int mg_fields32_zero_j (mg_run_t *) { NOT_BUILT ("zero_j"); }
int mg_push32 (mg_run_t *) { NOT_BUILT ("push"); }
int mg_enqueue_step32 (mg_run_t *, int) { NOT_BUILT ("step"); }
int mg_place32 (mg_run_t *, const mg_place_t *, long long, long long) { NOT_BUILT ("place"); }
int mg_ensure_capacity32 (mg_run_t *, long long) { NOT_BUILT ("capacity"); }
int mg_walls32 (mg_run_t *) { NOT_BUILT ("walls"); }
