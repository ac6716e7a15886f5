/*
 * adrt_oracle.h -- TEST INFRASTRUCTURE: FP64 CPU restatement of the
 * reference's adding-doubling column solver (src/solver.cpp:348-722 and the
 * headers it includes).  It is the parity checker for the CUDA engine and is
 * never linked into, or called by, the product.  It is pinned against the
 * reference's own solver (oracle/_ref, compiled from the reference sources)
 * through the golden vectors in tests/golden/.
 */
#ifndef ADRT_ORACLE_H_
#define ADRT_ORACLE_H_

#include "../include/adrt_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Batched solve on host buffers; same description and layouts as the engine.
 * Returns 0, or -1 with oracle_last_error() set (validation failure). */
int oracle_solve_batch(const adrt_batch_desc* desc, const adrt_inputs* in,
                       const adrt_outputs* out, int nthreads);
int oracle_solve_batch_range(const adrt_batch_desc* desc, const adrt_inputs* in,
                             const adrt_outputs* out, int w0, int w1, int nthreads);
const char* oracle_last_error(void);

/* Pieces exposed for unit tests. */
void oracle_gauss_legendre(int n, double* nodes, double* weights);
double oracle_planck(double wnumlo, double wnumhi, double temp);
double oracle_planck_deriv(double wnumlo, double wnumhi, double temp);
int oracle_ipow0(double omega);
int oracle_num_doublings(double tau, double omega);

/* Algorithmic flop count of one wavenumber's solve, following the branch the
 * solver takes (delta-M, pure absorption, non-scattering adding shortcuts). */
double oracle_flops_batch(const adrt_batch_desc* desc, const adrt_inputs* in, int w0, int w1);

#ifdef __cplusplus
}
#endif
#endif
