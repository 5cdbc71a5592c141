/*
 * lbm_oracle.h -- FP64 CPU restatement of the reference's family-B D3Q19
 * acoustic step.  TEST INFRASTRUCTURE ONLY: tests/, the smoke check and the
 * CPU-baseline leg of bench.py load it as the checker; the product library
 * never links it.
 *
 * Parity status: pinned.  On reference-native scenarios (NSCBC on x-,x+,y-,
 * y+,z+, ground wall at z-, sponge on the five open faces, Gaussian-pulse or
 * sine source on the 5x5x5 stencil, STL geometry) every population, the mask,
 * the sponge field and the probe series are bit-identical to the unmodified
 * reference (06_transient_localization_dx1.cpp, 08_city_scale_uav.cpp) run
 * through oracle/ref_harness.cpp; tests/test_oracle_pinning.py checks that and
 * the committed fixtures in tests/golden/.  The options the reference does not
 * have (other face types, sponge face sets, Ricker/table waveforms, trilinear
 * injection, several sources) follow the same code paths and are restated from
 * the reference pattern they extend.
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H

#include "nlos_lbm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_handle orc_handle;

orc_handle* orc_create(const lbm_config* cfg);
void orc_destroy(orc_handle* h);
int orc_set_geometry_triangles(orc_handle* h, const float* tris, int ntris, double scale, double sx,
                               double sy, double sz);
int orc_set_geometry_stl(orc_handle* h, const char* path, double scale, double sx, double sy, double sz);
int orc_set_mask(orc_handle* h, const unsigned char* mask);
/* Scheme A, before orc_init: per-column blend strengths and field-source
 * weights (nx*ny, x fastest), as lbm_set_blend_xy / lbm_set_field_weights_xy. */
int orc_set_blend_xy(orc_handle* h, const double* s_xy);
int orc_set_field_xy(orc_handle* h, const double* w_xy);
int orc_add_source(orc_handle* h, const lbm_source* src);
int orc_set_probes(orc_handle* h, const double* xyz, int n);
int orc_init(orc_handle* h);
void orc_apply_source(orc_handle* h, double t);
void orc_exchange_halos(orc_handle* h);
void orc_step_collision_bgk(orc_handle* h);
void orc_record_probes(orc_handle* h);
void orc_step(orc_handle* h, int nsteps);
void orc_set_threads(int n);
/* FP64 discrete adjoint of orc_step for L = 1/2 sum (probe - observed)^2 over
 * nsteps steps from the state after orc_init (no counterpart in the
 * reference); K: checkpoint interval (<= 0: sqrt(nsteps)).  grad_signal[s] =
 * dL/d(source value at step s), grad_pos = dL/d(rigid shift of the source
 * path).  Restores the initial state. */
int orc_adjoint_grad(orc_handle* h, int nsteps, const double* observed, int K, double* loss, double* grad_pos,
                     double* grad_signal, double* predicted);

void orc_get_dims(orc_handle* h, int* n3, int* n3_halo);
double orc_get_dt(orc_handle* h);
void orc_get_f(orc_handle* h, double* out);
void orc_set_f(orc_handle* h, const double* in);
void orc_set_density(orc_handle* h, const double* rho_prime);
void orc_get_mask(orc_handle* h, unsigned char* out);
void orc_get_rho(orc_handle* h, double* out);
void orc_get_sponge(orc_handle* h, double* out);
void orc_get_tau_a(orc_handle* h, double* out);
void orc_get_ground_height(orc_handle* h, double* out);
long orc_get_probes(orc_handle* h, double* out, long capacity);

#ifdef __cplusplus
}
#endif

#endif
