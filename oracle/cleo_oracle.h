/*
 * cleo_oracle.h — CPU restatement of CLEO's super-droplet hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker the parity tests, the smoke test and the
 * benchmark's CPU-baseline leg compare the CUDA path against. The product (cleo_b200/) never
 * links, loads or calls it.
 *
 * It mirrors the C ABI of include/cleo_b200.h on host memory: a context holding the SoA state,
 * stepped exactly like SDMMethods::run_step (libs/runcleo/sdmmethods.hpp:319-332) with the
 * reference's operation order, so that integer results (multiplicities, gridbox indexes, order)
 * are bit-identical and floating-point results differ only through libm.
 */
#ifndef CLEO_ORACLE_H_
#define CLEO_ORACLE_H_

#include "../include/cleo_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oc_ctx oc_ctx;

int oc_create(const cleo_b200_params* p, const cleo_b200_grid* g, size_t capacity, oc_ctx** out);
void oc_destroy(oc_ctx* c);
int oc_upload_supers(oc_ctx* c, const cleo_b200_supers* h, size_t n);
int oc_upload_state(oc_ctx* c, const cleo_b200_gbx_state* h);
int oc_step(oc_ctx* c, uint32_t t_mdl, uint32_t t_next);
int oc_status(oc_ctx* c, cleo_b200_error* err);
int oc_download_supers(oc_ctx* c, cleo_b200_supers* h, size_t* n_domain, size_t* n_total);
int oc_download_state(oc_ctx* c, cleo_b200_gbx_state* h);
int oc_download_budgets(oc_ctx* c, double* cond_mass, uint64_t* nr_iters);
int oc_monitors_begin(oc_ctx* c);
int oc_download_monitors(oc_ctx* c, cleo_b200_monitors* out, int reset);

/* Threads of the loops over gridboxes inside oc_step (OpenMP; 1 = sequential, the default).
 * Results do not depend on it. Returns the number set. */
int oc_set_num_threads(int n);

/* Batch of independent implicit-Euler condensation solves (host arrays). */
int oc_condensation_solve(const cleo_b200_params* p, size_t n, const double* radius,
                          const double* msol, const double* temp, const double* press,
                          const double* s_ratio, const double* delt, double* radius_out,
                          uint32_t* niters_out);

/* Same, but the Newton iteration starts from z0 = seed_rsqrd[i] (the branch decisions still use
 * the reference initial guess); used to check seeded solves. */
int oc_condensation_solve_seeded(const cleo_b200_params* p, size_t n, const double* radius,
                                 const double* msol, const double* temp, const double* press,
                                 const double* s_ratio, const double* delt,
                                 const double* seed_rsqrd, double* radius_out,
                                 uint32_t* niters_out);

/* The injected random stream (shared contract with the CUDA path and the reference harness). */
uint64_t oc_rng_u64(uint64_t seed, uint32_t t_sdm, uint32_t gbxindex, uint64_t slot);
double oc_rng_drand(uint64_t seed, uint32_t t_sdm, uint32_t gbxindex, uint64_t slot);
uint64_t oc_rng_urand(uint64_t seed, uint32_t t_sdm, uint32_t gbxindex, uint64_t slot,
                      uint64_t start, uint64_t end);

/* Terminal velocities and collision probabilities of single droplets / pairs (unit checks). */
double oc_terminal_velocity(int kind, double radius);
double oc_pair_probability(const cleo_b200_params* p, double r1, uint64_t xi1, double msol1,
                           double r2, uint64_t xi2, double msol2, double volume);

#ifdef __cplusplus
}
#endif

#endif /* CLEO_ORACLE_H_ */
