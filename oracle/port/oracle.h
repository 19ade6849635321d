/*
 * oracle.h - CPU restatement of CIPHER's RHS evaluation and per-step
 * active-set update.  TEST INFRASTRUCTURE ONLY: tests, the smoke check and the
 * benchmark's CPU baseline call it; the product never does.
 */
#ifndef CIPHER_ORACLE_H
#define CIPHER_ORACLE_H

#include <stdint.h>
#include "cipher_problem.h"

double or_ipow(double base, unsigned e);
double or_tseries(double T, const cipher_tseries *s);
double or_tseries_dT(double T, const cipher_tseries *s);
int or_set_intersect(const uint16_t *a, int na, const uint16_t *b, int nb,
                     uint16_t *out, uint16_t *ina, uint16_t *inb);
int or_set_union(const uint16_t *a, int na, const uint16_t *b, int nb, uint16_t *out, int cap);
void or_invert(double *dst, double *src, int n);
void or_matvec(double *dst, const double *A, const double *x, int n);
void or_interpolant(int kind, const double *phi, int n, double *h);
void or_interpolant_dT(int kind, double *v, const double *phi, int n);
void or_simplex_projection(double *out, const double *in, int n);

cipher_aos_layout or_aos_layout(const cipher_problem *p);
const cipher_material *or_material(const cipher_problem *p, int phase);
double or_chemenergy(const cipher_problem *p, int phase, const double *y, const double *mu, double T);
void or_sitepot_explicit(const cipher_problem *p, int phase, const double *y, double T, double *out);
void or_sitepot_total(const cipher_problem *p, int phase, const double *y, double T, double *out);
void or_sitefrac(const cipher_problem *p, int phase, const double *pot, double T, double *y);
void or_sitefrac_tangent(const cipher_problem *p, int phase, const double *y, const double *pot, double T,
                         double *tpot, double *tex, double *tT);
void or_mobility(const cipher_problem *p, int phase, const double *y, double T, double *M);

/* public entry points (ctypes) */
int oracle_rhs(const cipher_problem *p, const cipher_mesh *m, double t,
               const double *Xlocal, double *F);
int oracle_poststep(const cipher_problem *p, const cipher_mesh *m, double *X);
int oracle_initial_state(const cipher_problem *p, const cipher_mesh *m, double *X);
int oracle_output_fields(const cipher_problem *p, const cipher_mesh *m, const double *X, const int32_t *kinds,
                         const int32_t *idx, int nf, double *out);

#endif
