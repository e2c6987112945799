// ORACLE — test infrastructure, not product code.
//
// A C interface over the reference's own MultiStealthyPotential (apps/CCOptimization/MultiStealthyPotential.{h,cpp},
// with core/SpherePacking.cpp), compiled from the reference tree into oracle/_ref/libccref.so. The tests and the
// golden generator call it as the checker of the product's cc_multi_* entry points.
#include "MultiStealthyPotential.h"
#include "RepulsiveCCPotential.h"

#include <cmath>
#include <cstring>
#include <iostream>
#include <vector>

extern "C" {

// Energy and Cartesian forces (N x d) of the reference's MultiStealthyPotential: nspecies species with M[s] Cartesian
// wavevectors kcart[s] (M[s] x d) and weights V[s]; particle i at fractional frac (N x d) in species species[i];
// radii (N) or NULL for the reference's defaults; u0, e0 as its members. Returns 0, or -1 if the reference threw.
int ccref_multi_eval(int d, const double *basis, int nspecies, const long *M, const double *const *kcart,
                     const double *const *V, double u0, double e0, long N, const double *frac, const int *species,
                     const double *radii, double *E, double *F)
{
	std::streambuf *saved = std::cout.rdbuf(nullptr);   // the reference reports set-up steps on stdout
	int rc = 0;
	try {
		std::vector<GeometryVector> a;
		double ml = 0.0;
		for (int i = 0; i < d; i++) {
			GeometryVector g(d);
			for (int j = 0; j < d; j++)
				g.x[j] = basis[i * d + j];
			ml = std::max(ml, std::sqrt(g.Modulus2()));
			a.push_back(g);
		}
		Configuration c(d, a.data(), 10.0 * ml);
		for (long i = 0; i < N; i++) {
			GeometryVector s(d);
			for (int e = 0; e < d; e++)
				s.x[e] = frac[i * d + e];
			c.Insert("A", s);
		}
		MultiStealthyPotential pot(d, e0);
		pot.u0 = u0;
		pot.SetNumSpecies(nspecies);
		for (int s = 0; s < nspecies; s++)
			for (long q = 0; q < M[s]; q++) {
				GeometryVector k(d);
				for (int e = 0; e < d; e++)
					k.x[e] = kcart[s][q * d + e];
				pot.AddConstraint(s, k, std::vector<double>{V[s][q]});
			}
		pot.SetConfiguration(c);
		for (long i = 0; i < N; i++)
			pot.SetSpeciesOfParticle(i, species[i]);
		if (radii)
			pot.SetSecureRadii(std::vector<double>(radii, radii + N));
		*E = pot.Energy();
		if (F) {
			std::vector<GeometryVector> f;
			pot.AllForce(f);
			for (long i = 0; i < N; i++)
				for (int e = 0; e < d; e++)
					F[i * d + e] = f[i].x[e];
		}
	} catch (...) {
		rc = -1;
	}
	std::cout.rdbuf(saved);
	return rc;
}

// Energy and Cartesian forces (N x d) of the reference's RepulsiveCCPotential (apps/CCOptimization/
// RepulsiveCCPotential.h:21-159): soft-core contact of strength e0 and distance sigma plus a ShiftedCCPotential
// (S0 == NULL) or a ShiftedCCPotential_S2 (targets S0, M values), constraints added through the collective-coordinate
// member's AddConstraint as GetCCO does (apps/CCOptimization/main.cpp:262-318). Returns 0, or -1 if the reference threw.
int ccref_repulsive_eval(int d, const double *basis, long M, const double *kcart, const double *V, const double *S0,
                         double e0, double sigma, long N, const double *frac, int nthreads, double *E, double *F)
{
	std::streambuf *saved = std::cout.rdbuf(nullptr);   // the reference reports set-up steps on stdout
	int rc = 0;
	try {
		std::vector<GeometryVector> a;
		double ml = 0.0;
		for (int i = 0; i < d; i++) {
			GeometryVector g(d);
			for (int j = 0; j < d; j++)
				g.x[j] = basis[i * d + j];
			ml = std::max(ml, std::sqrt(g.Modulus2()));
			a.push_back(g);
		}
		Configuration c(d, a.data(), 10.0 * ml);
		for (long i = 0; i < N; i++) {
			GeometryVector s(d);
			for (int e = 0; e < d; e++)
				s.x[e] = frac[i * d + e];
			c.Insert("A", s);
		}
		RepulsiveCCPotential pot(d, e0, sigma, S0 ? 1.0 : 0.0);
		pot.ParallelNumThread = nthreads;
		pot.CCPotential->ParallelNumThread = nthreads;
		for (long q = 0; q < M; q++) {
			GeometryVector k(d);
			for (int e = 0; e < d; e++)
				k.x[e] = kcart[q * d + e];
			std::vector<double> vals{V[q]};
			if (S0)
				vals.push_back(S0[q]);
			pot.CCPotential->AddConstraint(k, vals);
		}
		pot.SetConfiguration(c);
		*E = pot.Energy();
		if (F) {
			std::vector<GeometryVector> f;
			pot.AllForce(f);
			for (long i = 0; i < N; i++)
				for (int e = 0; e < d; e++)
					F[i * d + e] = f[i].x[e];
		}
	} catch (...) {
		rc = -1;
	}
	std::cout.rdbuf(saved);
	return rc;
}

}  // extern "C"
