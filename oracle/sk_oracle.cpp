// ORACLE — test infrastructure, not product code.
//
// The reference's own IsotropicStructureFactor and StructureFactor (pairstat/StructureFactor.cpp:56-260) are compiled
// from the reference tree into oracle/_ref/libccref.so (with a Boost.Math bessel stand-in), and so is its
// RandomGenerator (core/RandomGenerator.cpp, with the std::mt19937 stand-in for boost::mt19937). Two symbols they
// need live in translation units that need GSL or Boost.MultiIndex, absent here, and are restated below:
//   - HyperSphere_Volume (core/etc.cpp:50-73): c_n R^n with c_1 = 2, c_2 = pi, c_3 = 4 pi / 3, and
//     pi^(n/2) / Gamma(n/2 + 1) beyond;
//   - GetKs (core/PeriodicCellList.cpp:509-735): the grid enumeration of the half-space reciprocal lattice points
//     within CircularKMax (odometer order, axis 0 fastest), sorted by (|k|^2, k_x); for LinearKMax != CircularKMax
//     the multiples of the first point of each direction (directions compared as unit vectors, tolerance 1e-10),
//     each kept with SampleProbability drawn from RandomGenerator(98765); the 1D branches.
// ccref_getks and ccref_isotropic_sk give the tests a C interface to them.
#include "RandomGenerator.h"
#include "StructureFactor.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

double HyperSphere_Volume(DimensionType n, double R)
{
	double c;
	if (n == 1)
		c = 2.0;
	else if (n == 2)
		c = pi;
	else if (n == 3)
		c = 4.1887902047863909846;
	else
		c = std::pow(pi, n / 2.0) / std::tgamma(n / 2.0 + 1.0);
	return c * std::pow(R, static_cast<double>(n));
}

std::vector<GeometryVector> GetKs(const PeriodicCellList<Empty> &cell, double CircularKMax, double LinearKMax,
                                  double SampleProbability, bool, double CircularKMin)
{
	std::vector<GeometryVector> out;
	if (CircularKMax <= 0.0 || LinearKMax <= 0.0)
		return out;
	RandomGenerator gen(98765);
	auto keep = [&]() { return SampleProbability >= 1.0 || gen.RandomDouble() < SampleProbability; };
	const DimensionType dim = cell.GetDimension();
	if (dim == 1) {
		const GeometryVector b = cell.GetReciprocalBasisVector(0);
		if (CircularKMin <= 0.0) {
			for (double i = 1.0;; i += 1.0) {
				GeometryVector k = i * b;
				if (k.x[0] > LinearKMax)
					break;
				if (keep())
					out.push_back(k);
			}
			return out;
		}
		size_t inside = 0;
		for (double i = 1.0;; i += 1.0) {
			GeometryVector k = i * b;
			if (k.x[0] > CircularKMax)
				break;
			if (k.x[0] > CircularKMin && keep()) {
				out.push_back(k);
				inside++;
			}
		}
		if (inside == 0)
			return out;
		for (double i = 2.0;; i += 1.0)
			for (size_t j = 0; j < inside; j++) {
				GeometryVector k = i * out[j];
				if (k.x[0] > LinearKMax)
					return out;
				if (keep())
					out.push_back(k);
			}
	}
	std::vector<GeometryVector> b;
	std::vector<long> lim, n;
	size_t total = 1;
	for (DimensionType e = 0; e < dim; e++) {
		b.push_back(cell.GetReciprocalBasisVector(e));
		lim.push_back((long)std::ceil(CircularKMax * std::sqrt(cell.GetBasisVector(e).Modulus2()) / (2.0 * pi)));
		n.push_back(-lim.back());
		total *= (size_t)(2 * lim.back() + 1);
	}
	const double K2 = CircularKMax * CircularKMax, Kmin2 = CircularKMin * CircularKMin;
	std::vector<GeometryVector> ks;
	for (size_t it = 0; it < total; it++) {
		long first = 0;
		for (DimensionType e = 0; e < dim && first == 0; e++)
			first = n[e];
		if (first >= 0) {
			GeometryVector k(dim);
			for (DimensionType e = 0; e < dim; e++)
				k = k + (double)n[e] * b[e];
			const double k2 = k.Modulus2();
			if (k2 < K2 && k2 > Kmin2)
				ks.push_back(k);
		}
		for (DimensionType e = 0; e < dim; e++) {   // odometer, axis 0 fastest
			if (++n[e] <= lim[e])
				break;
			n[e] = -lim[e];
		}
	}
	std::sort(ks.begin(), ks.end(), [](const GeometryVector &l, const GeometryVector &r) {
		const double a = l.Modulus2(), c = r.Modulus2();
		if (a != c)
			return a < c;
		return l.x[0] < r.x[0];
	});
	if (LinearKMax == CircularKMax)
		return ks;
	std::vector<GeometryVector> dirs, firsts;
	for (const GeometryVector &k : ks) {
		GeometryVector u = (1.0 / std::sqrt(k.Modulus2())) * k;
		bool found = false;
		for (const GeometryVector &v : dirs)
			if ((u - v).Modulus2() < 1e-20) {
				found = true;
				break;
			}
		if (!found) {
			dirs.push_back(u);
			firsts.push_back(k);
		}
	}
	for (const GeometryVector &k : firsts)
		for (long i = 1;; i++) {
			GeometryVector t = static_cast<double>(i) * k;
			if (t.Modulus2() > LinearKMax * LinearKMax)
				break;
			if (keep())
				out.push_back(t);
		}
	return out;
}

namespace {

std::vector<GeometryVector> BasisOf(int d, const double *rows)
{
	std::vector<GeometryVector> v;
	for (int i = 0; i < d; i++) {
		GeometryVector g(d);
		for (int j = 0; j < d; j++)
			g.x[j] = rows[i * d + j];
		v.push_back(g);
	}
	return v;
}

}  // namespace

extern "C" {

// GetKs of a cell: Cartesian k (K x d) into out (cap rows); returns K (or -1 when cap is too small).
long ccref_getks(int d, const double *basis, double circ, double lin, double p, double kmin, long cap, double *out)
{
	std::vector<GeometryVector> a = BasisOf(d, basis);
	PeriodicCellList<Empty> cell(d, a.data(), 1.0);
	std::vector<GeometryVector> ks = GetKs(cell, circ, lin, p, false, kmin);
	if ((long)ks.size() > cap)
		return -1;
	for (size_t i = 0; i < ks.size(); i++)
		for (int j = 0; j < d; j++)
			out[i * d + j] = ks[i].x[j];
	return (long)ks.size();
}

// The reference's IsotropicStructureFactor over nconfigs configurations (bases nconfigs x d x d, N[j] particles at
// fractional frac[j]); rows of 4 into out (cap rows); returns the row count (or -1 when cap is too small).
long ccref_isotropic_sk(int d, long nconfigs, const double *bases, const long *N, const double *const *frac,
                        double circ, double lin, double kprec, double p, int option, double kmin, long cap, double *out)
{
	auto get = [&](size_t j) -> const Configuration {
		std::vector<GeometryVector> a = BasisOf(d, bases + j * d * d);
		double ml = 0.0;
		for (auto &v : a)
			ml = std::max(ml, std::sqrt(v.Modulus2()));
		Configuration c(d, a.data(), 10.0 * ml);
		for (long i = 0; i < N[j]; i++) {
			GeometryVector s(d);
			for (int e = 0; e < d; e++)
				s.x[e] = frac[j][i * d + e];
			c.Insert("A", s);
		}
		return c;
	};
	std::vector<GeometryVector> res;
	IsotropicStructureFactor(get, (size_t)nconfigs, circ, lin, res, kprec, p, (size_t)option, kmin);
	if ((long)res.size() > cap)
		return -1;
	for (size_t i = 0; i < res.size(); i++)
		for (int c = 0; c < 4; c++)
			out[i * 4 + c] = res[i].x[c];
	return (long)res.size();
}

}  // extern "C"
