// Test scaffolding for the oracle build only (not product code).
//
// The reference's own ShiftedCCPotential (potential/CollectiveCoordinatePotential.h) is header-only, but
// linking it needs two out-of-line symbols whose real definitions live in translation units that depend on
// GSL, which is absent here:
//   - Potential::~Potential()   real one: potential/Potential.cpp:41-43 (an empty body);
//   - ::Volume(vecs, d)         real one: core/GeometryVector.cpp:63-77 (|det| through a GSL LU).
// This file supplies both, with the determinant written in closed form for d = 1..4. It also defines the
// few globals that core/etc.h declares extern and that inline code of the headers may name.
#include "GeometryVector.h"
#include "Potential.h"

#include <cmath>
#include <ctime>
#include <iostream>

Potential::~Potential() {}

static double det3(double a, double b, double c, double d, double e, double f, double g, double h, double i)
{
	return a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
}

double Volume(const GeometryVector *vecs, DimensionType dimension)
{
	if (!(dimension > 0))
		return 0.0;
	const double *r0 = vecs[0].x;
	if (dimension == 1)
		return std::abs(r0[0]);
	const double *r1 = vecs[1].x;
	if (dimension == 2)
		return std::abs(r0[0] * r1[1] - r0[1] * r1[0]);
	const double *r2 = vecs[2].x;
	if (dimension == 3)
		return std::abs(det3(r0[0], r0[1], r0[2], r1[0], r1[1], r1[2], r2[0], r2[1], r2[2]));
	const double *r3 = vecs[3].x;
	// Laplace expansion along the first row.
	double det = 0.0;
	for (int c = 0; c < 4; c++) {
		int cols[3], k = 0;
		for (int j = 0; j < 4; j++)
			if (j != c)
				cols[k++] = j;
		double minor = det3(r1[cols[0]], r1[cols[1]], r1[cols[2]], r2[cols[0]], r2[cols[1]], r2[cols[2]],
		                    r3[cols[0]], r3[cols[1]], r3[cols[2]]);
		det += ((c % 2) ? -1.0 : 1.0) * r0[c] * minor;
	}
	return std::abs(det);
}

size_t Verbosity = 0;
time_t ProgramStart = 0;
time_t TimeLimit = 0;
std::ostream logfile(nullptr);   // progress bars of the reference code go nowhere

// GeometryVector's binary I/O (core/GeometryVector.cpp) is named by the SpherePacking file readers that the
// multi-species potential's translation unit pulls in; the oracle never reads or writes a packing file, so these
// only write and read the d coordinates as raw doubles.
void GeometryVector::WriteBinary(std::ostream &ofile, DimensionType dimension) const
{
	ofile.write(reinterpret_cast<const char *>(this->x), sizeof(double) * dimension);
}

void GeometryVector::ReadBinary(std::istream &ifile, DimensionType dimension)
{
	ifile.read(reinterpret_cast<char *>(this->x), sizeof(double) * dimension);
}

// GSL stand-ins for potential/CCPotential_varBox.h (declared in standins/gsl/gsl_linalg.h). Only that header's cell
// derivatives call them, and the oracle never does: each throws, so a call by mistake fails loudly.
#include <gsl/gsl_linalg.h>

#include <stdexcept>

[[noreturn]] static void gsl_standin()
{
	throw std::logic_error("GSL stand-in reached: cell derivatives are not part of the oracle");
}

gsl_matrix *gsl_matrix_alloc(size_t, size_t) { gsl_standin(); }
void gsl_matrix_free(gsl_matrix *) { gsl_standin(); }
double gsl_matrix_get(const gsl_matrix *, size_t, size_t) { gsl_standin(); }
void gsl_matrix_set(gsl_matrix *, size_t, size_t, double) { gsl_standin(); }
gsl_vector *gsl_vector_alloc(size_t) { gsl_standin(); }
void gsl_vector_free(gsl_vector *) { gsl_standin(); }
double gsl_vector_get(const gsl_vector *, size_t) { gsl_standin(); }
void gsl_vector_set(gsl_vector *, size_t, double) { gsl_standin(); }
void gsl_vector_set_zero(gsl_vector *) { gsl_standin(); }
gsl_permutation *gsl_permutation_alloc(size_t) { gsl_standin(); }
gsl_permutation *gsl_permutation_calloc(size_t) { gsl_standin(); }
void gsl_permutation_free(gsl_permutation *) { gsl_standin(); }
int gsl_linalg_LU_decomp(gsl_matrix *, gsl_permutation *, int *) { gsl_standin(); }
int gsl_linalg_LU_solve(const gsl_matrix *, const gsl_permutation *, const gsl_vector *, gsl_vector *) { gsl_standin(); }
int gsl_linalg_LU_invert(const gsl_matrix *, const gsl_permutation *, gsl_matrix *) { gsl_standin(); }
