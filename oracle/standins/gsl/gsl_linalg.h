// Test scaffolding for the oracle build only (not product code).
//
// GSL is absent here. The reference's potential/CCPotential_varBox.h includes <gsl/gsl_linalg.h> for its cell
// derivatives (dBi, EnergyDerivativeToBasisVectors), which the oracle never calls: the varBox potentials are checked at
// a fixed cell. These declarations let that header compile; the definitions in standins.cpp throw if ever reached.
#ifndef ORACLE_STANDIN_GSL_LINALG_H
#define ORACLE_STANDIN_GSL_LINALG_H

#include <cstddef>

struct gsl_matrix {
	size_t size1, size2, tda;
	double *data;
};
struct gsl_vector {
	size_t size, stride;
	double *data;
};
struct gsl_permutation {
	size_t size;
	size_t *data;
};

gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2);
void gsl_matrix_free(gsl_matrix *m);
double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j);
void gsl_matrix_set(gsl_matrix *m, size_t i, size_t j, double x);
gsl_vector *gsl_vector_alloc(size_t n);
void gsl_vector_free(gsl_vector *v);
double gsl_vector_get(const gsl_vector *v, size_t i);
void gsl_vector_set(gsl_vector *v, size_t i, double x);
void gsl_vector_set_zero(gsl_vector *v);
gsl_permutation *gsl_permutation_alloc(size_t n);
gsl_permutation *gsl_permutation_calloc(size_t n);
void gsl_permutation_free(gsl_permutation *p);
int gsl_linalg_LU_decomp(gsl_matrix *A, gsl_permutation *p, int *signum);
int gsl_linalg_LU_solve(const gsl_matrix *LU, const gsl_permutation *p, const gsl_vector *b, gsl_vector *x);
int gsl_linalg_LU_invert(const gsl_matrix *LU, const gsl_permutation *p, gsl_matrix *inverse);

#endif
