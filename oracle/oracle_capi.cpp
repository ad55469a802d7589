// C entry points over the CPU oracle (zsph_oracle.hpp) for ctypes callers in
// tests/ and bench.py's CPU-baseline leg.  Test infrastructure only: the
// product library never links this file.
//
// Arrays use the reference's particle layout
// (single_gpu_sph_src/header/data_structure.cuh:158-182): pos/vel/tmp_pos/
// tmp_vel are 3 values per particle, rhop/tmp_rhop 2, acc_drhodt and
// dofv_grandrho 4, type/table/index/hash one int, grid_start/grid_end one
// int per cell.
#include <omp.h>

#include <cmath>
#include <cstdio>

#include "zsph_oracle.hpp"

using namespace zsph_oracle;

extern "C" {

// JSON-level inputs (cpu_json_t fields that enter the derivation,
// single_gpu_sph_src/header/data_structure.cuh:6-32).
typedef struct {
  float g, rho0, dx, h_factor, r_factor, eta_factor, cs_factor, delta, alpha;
  float xmin, xmax, ymin, ymax, zmin, zmax, grid_layer_factor, grid_size_factor;
  float dt;
  int ptc_num;
} ocase_t;

// single_gpu_sph_src/lib/init.cu:153-251 (set_cpu_param + set_gpu_param) and
// single_gpu_sph_src/lib/check.cu:3-18 (check_dt).  Host math follows the
// reference's float arithmetic: sqrt and abs of a float resolve to the
// float overloads.  Returns 0, or 1 when dt > dt_max (where the reference
// calls exit(1)).
int oracle_params(const ocase_t* c, Params* p) {
  const float m = c->rho0 * c->dx * c->dx * c->dx;  // init.cu:157
  const float h = c->h_factor * c->dx;              // :160
  const float r = c->r_factor * c->h_factor * c->dx;
  const float eta = c->eta_factor * c->h_factor * c->dx;
  const float cs = c->cs_factor * std::sqrt(std::fabs(c->g) * (c->zmax - c->zmin));  // :163
  const float adh = 21.0f / (16.0f * 3.1415926f * h * h * h);                         // :166
  const float gs = c->r_factor * c->h_factor * c->dx / c->grid_size_factor;           // :177
  const float gxmin = c->xmin - gs * c->grid_layer_factor, gxmax = c->xmax + gs * c->grid_layer_factor;
  const float gymin = c->ymin - gs * c->grid_layer_factor, gymax = c->ymax + gs * c->grid_layer_factor;
  const float gzmin = c->zmin - gs * c->grid_layer_factor, gzmax = c->zmax + gs * c->grid_layer_factor;
  p->grid_xdim = (int)((gxmax - gxmin) / gs);  // :185-187
  p->grid_ydim = (int)((gymax - gymin) / gs);
  p->grid_zdim = (int)((gzmax - gzmin) / gs);
  p->grid_num = p->grid_xdim * p->grid_ydim * p->grid_zdim;
  p->grid_hash_min = 0;
  p->grid_hash_max = p->grid_num - 1;
  p->grid_size = gs;
  p->grid_factor = (int)c->grid_size_factor;
  p->grid_xmin = gxmin; p->grid_ymin = gymin; p->grid_zmin = gzmin;
  p->half_dt = c->dt / 2.0f;  // :223
  p->h = h; p->g = c->g; p->m = m; p->rho0 = c->rho0; p->adh = adh;
  p->h2 = h * h; p->eta2 = eta * eta; p->cs2 = cs * cs; p->alpha = c->alpha;
  p->delta_h_cs = c->delta * h * cs;       // :233
  p->h_cs_rho_m = h * cs * c->rho0 * m;    // :234
  p->ptc_num = c->ptc_num;
  p->dt = c->dt; p->cs = cs; p->eta = eta; p->r = r;
  p->dt_max = (float)(0.25 * (double)h / (double)std::sqrt(-c->g * (c->zmax - c->zmin)));  // check.cu:6
  return (c->dt <= p->dt_max) ? 0 : 1;  // check.cu:9-17
}

int oracle_sizeof_params(void) { return (int)sizeof(Params); }

void oracle_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int oracle_max_threads(void) { return omp_get_max_threads(); }

#define ORACLE_INSTANCE(SUF, T)                                                                       \
  void oracle_hash_##SUF(const Params* p, State<T>* s, Tmp<T>* t) { hash<T>(*p, *s, *t); }          \
  void oracle_sort_index_##SUF(const Params* p, Tmp<T>* t) { sort_index<T>(*p, *t); }               \
  void oracle_sort_data_##SUF(const Params* p, const State<T>* o, State<T>* w, Tmp<T>* t) {         \
    sort_data<T>(*p, *o, *w, *t);                                                                   \
  }                                                                                                 \
  void oracle_boundary_##SUF(const Params* p, State<T>* s, Tmp<T>* t, int wall_mode) {              \
    boundary<T>(*p, *s, *t, wall_mode);                                                             \
  }                                                                                                 \
  void oracle_governing_##SUF(const Params* p, const State<T>* s, Tmp<T>* t) { governing<T>(*p, *s, *t); } \
  void oracle_prediction_##SUF(const Params* p, State<T>* s, const Tmp<T>* t) { prediction<T>(*p, *s, *t); } \
  void oracle_correction_##SUF(const Params* p, State<T>* s, const Tmp<T>* t) { correction<T>(*p, *s, *t); } \
  void oracle_step_##SUF(const Params* p, State<T>* o, State<T>* w, Tmp<T>* t, int nsteps, int wall_mode) { \
    for (int k = 0; k < nsteps; ++k) step<T>(*p, *o, *w, *t, wall_mode);                            \
  }                                                                                                 \
  void oracle_neighbor_count_##SUF(const Params* p, const State<T>* s, const Tmp<T>* t, int ylast, int* out) { \
    neighbor_count<T>(*p, *s, *t, ylast, out);                                                      \
  }                                                                                                 \
  void oracle_boundary_simple_##SUF(const Params* p, State<T>* s, Tmp<T>* t, T* dofv) {             \
    boundary_simple<T>(*p, *s, dofv, *t);                                                           \
  }                                                                                                 \
  void oracle_governing_simple_##SUF(const Params* p, const State<T>* s, Tmp<T>* t, const T* dofv) { \
    governing_simple<T>(*p, *s, dofv, *t);                                                          \
  }                                                                                                 \
  void oracle_step_simple_##SUF(const Params* p, State<T>* o, State<T>* w, Tmp<T>* t, T* dofv, int nsteps) { \
    for (int k = 0; k < nsteps; ++k) step_simple<T>(*p, *o, *w, *t, dofv);                          \
  }                                                                                                 \
  void oracle_features_##SUF(const Params* p, const State<T>* s, const Tmp<T>* t, const float* scale,       \
                             const T* acc_prev, T* out) {                                           \
    features<T>(*p, *s, *t, scale, acc_prev, out);                                                  \
  }                                                                                                 \
  void oracle_step_rigid_##SUF(const Params* p, State<T>* o, State<T>* w, Tmp<T>* t, Rigid* b, int nsteps, \
                               int wall_mode) {                                                     \
    for (int k = 0; k < nsteps; ++k) step_rigid<T>(*p, *o, *w, *t, *b, wall_mode);                  \
  }                                                                                                 \
  void oracle_rigid_place_##SUF(const Params* p, State<T>* s, const Rigid* b) { rigid_place<T>(*p, *s, *b); } \
  void oracle_step_rigid_bodies_##SUF(const Params* p, State<T>* o, State<T>* w, Tmp<T>* t, Rigid* b, int nb,  \
                                      const Contact* ct, int nsteps, int wall_mode) {                  \
    for (int k = 0; k < nsteps; ++k) step_rigid_bodies<T>(*p, *o, *w, *t, b, nb, *ct, wall_mode);    \
  }

ORACLE_INSTANCE(f32, float)
ORACLE_INSTANCE(f64, double)

}  // extern "C"
