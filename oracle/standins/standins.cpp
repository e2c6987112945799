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
