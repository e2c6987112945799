// ORACLE — test infrastructure, not product code.
//
// A plain C interface over the reference's own collective-coordinate implementation, compiled from the
// reference tree by oracle/Makefile into oracle/_ref/libccref.so. Only the tests, the smoke check and the CPU
// baseline leg of bench.py load it, and only as the checker or the timed CPU reference.
//
// What is the reference's own code here (compiled unmodified from its headers/sources):
//   - ShiftedCCPotential: GetRho_Direct / Energy / Force / AllForce
//       (potential/CollectiveCoordinatePotential.h:1255-1286, :1351-1372, :1377-1394, :1434-1448);
//   - Configuration (PeriodicCellList<AtomName>): Insert with the double floor wrap and the Cartesian
//       coordinates sum_i s_i a_i (core/PeriodicCellList.h:517-538, :88-98), the reciprocal basis (:999-)
//       and the reciprocal-lattice cell list used for the k-set enumeration;
//   - LuksanPLIS (potential/LuksanPLIS.cpp), the L-BFGS the structure optimiser calls;
//   - ShiftedCCPotential_S2 and ShiftedCCPotential_S2_MultiConfig (potential/CollectiveCoordinatePotential.h:1642-1870)
//     and the named variable-cell classes of potential/CCPotential_Kernels.h with their constraint generation
//     (potential/CCPotential_varBox.h:129-202; its GSL-based cell derivatives link against throwing stand-ins).
// What is restated here, because its translation unit needs GSL/NLopt/Boost that this machine lacks:
//   - the Switch-0 objective (potential/StructureOptimization.cpp:339-350 FillParticles, :447-536 Objective)
//     and the three-pass driver (:1046-1090, RelaxStructure_NLOPT and RelaxStructure_NLOPT_Emin);
//   - the Type 0-3 k-set of GeneratePotential (apps/CollectiveCoordinateCLI/CollectiveCoordinateCLI.cpp:180-265);
//   - StructureFactor(config, k) (pairstat/StructureFactor.cpp:56-65).
#include "CollectiveCoordinatePotential.h"
#include "CCPotential_Kernels.h"
#include "LuksanPLIS.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <memory>
#include <vector>

namespace {

struct RefHandle {
	int d;
	std::vector<GeometryVector> basis;
	std::unique_ptr<Configuration> config;
	std::unique_ptr<ShiftedCCPotential> pot;
	std::unique_ptr<ShiftedCCPotential_ForMC> mc;   // ccref_mc_trymove's MC object, created at its first call
	int nthreads;
	// varBox potentials: the reference's own tildeV(k) and S0(k) at a wavevector (S0 NaN for the plain kinds)
	std::function<void(const GeometryVector &, double *, double *)> weights;
	ShiftedCCPotential_S2 *s2 = nullptr;
};

// Access to the protected weight and target functions of a varBox potential class.
template <class P> struct ProbeV : P {
	template <class... A> ProbeV(A... a) : P(a...) {}
	void eval(const GeometryVector &k, double *v, double *s0)
	{
		*v = this->tildeVk(k);
		*s0 = std::numeric_limits<double>::quiet_NaN();
	}
};
template <class P> struct ProbeVS : P {
	template <class... A> ProbeVS(A... a) : P(a...) {}
	void eval(const GeometryVector &k, double *v, double *s0)
	{
		*v = this->tildeVk(k);
		*s0 = this->S0k(k);
	}
};

GeometryVector MakeVec(int d, const double *x)
{
	GeometryVector v(d);
	for (int i = 0; i < d; i++)
		v.x[i] = x[i];
	return v;
}

std::unique_ptr<Configuration> EmptyConfig(RefHandle *h)
{
	double maxLength = 0.0;
	for (int i = 0; i < h->d; i++)
		maxLength = std::max(maxLength, std::sqrt(h->basis[i].Modulus2()));
	// One cell: the CC path never walks neighbours of the particles.
	return std::unique_ptr<Configuration>(new Configuration(h->d, h->basis.data(), 10.0 * maxLength));
}

void Fill(RefHandle *h, Configuration &c, long N, const double *frac, double rescale)
{
	c.RemoveParticles();
	for (long i = 0; i < N; i++) {
		GeometryVector rel(h->d);
		for (int j = 0; j < h->d; j++)
			rel.x[j] = frac[h->d * i + j] / rescale;
		c.Insert("A", rel);
	}
}

// --- restated Switch-0 objective (StructureOptimization.cpp:447-536), Pressure 0, no minimum distance ---
struct Aux {
	RefHandle *h;
	long N;
	double rescale;
	long evaluations;
	Configuration *work;
};

double Objective(unsigned n, const double *x, double *grad, void *data)
{
	Aux *aux = static_cast<Aux *>(data);
	RefHandle *h = aux->h;
	const int d = h->d;
	if (x[0] != x[0]) {
		if (grad)
			for (unsigned i = 0; i < n; i++)
				grad[i] = 0.0;
		return ::MaxEnergy;
	}
	Fill(h, *aux->work, aux->N, x, aux->rescale);
	const Configuration &list = *aux->work;
	double vol = list.PeriodicVolume();
	if (vol < std::pow(::LengthPrecision, static_cast<double>(d)))
		return ::MaxEnergy;
	h->pot->SetConfiguration(list);
	double result = h->pot->Energy() + 0.0 * vol;
	if (grad) {
		std::vector<GeometryVector> forces;
		h->pot->AllForce(forces);
		for (unsigned i = 0; i < n; i++)
			grad[i] = 0.0;
		for (long i = 0; i < aux->N; i++)
			for (int j = 0; j < d; j++)
				grad[i * d + j] = (-1.0) * forces[i].Dot(list.GetBasisVector(j)) / aux->rescale;
	}
	aux->evaluations++;
	return result;
}

}  // namespace

extern "C" {

// Build a potential over the cell `basis` (d rows of d doubles, row i = basis vector a_i). Constraints are given
// either as integer modes (k = sum_d m_d b_d over the reciprocal basis, as the reference's tests build lattice
// k-vectors) or as Cartesian k (kcart, M rows of d doubles); V holds the weights.
void *ccref_create(int d, const double *basis, long M, const int32_t *modes, const double *kcart, const double *V,
                   double shift, int nthreads)
{
	if (d < 1 || d > 4 || M < 0)
		return nullptr;
	RefHandle *h = new RefHandle();
	h->d = d;
	for (int i = 0; i < d; i++)
		h->basis.push_back(MakeVec(d, basis + d * i));
	h->config = EmptyConfig(h);
	h->pot.reset(new ShiftedCCPotential(d));
	h->nthreads = nthreads < 1 ? 1 : nthreads;
	h->pot->ParallelNumThread = h->nthreads;
	h->pot->Shift = shift;
	for (long m = 0; m < M; m++) {
		GeometryVector k(d);
		if (modes) {
			for (int e = 0; e < d; e++)
				k.AddFrom(static_cast<double>(modes[m * d + e]) * h->config->GetReciprocalBasisVector(e));
		} else {
			k = MakeVec(d, kcart + m * d);
		}
		h->pot->constraints.emplace_back(k, V[m]);
	}
	return h;
}

// The reference's ShiftedCCPotential_S2 (potential/CollectiveCoordinatePotential.h:1642-1749): E = sum_k V (|rho|^2 / N - S0)^2
// + Shift, constraints added through its AddConstraint(k, {V, S0}); evaluated with ccref_set_positions / ccref_eval.
void *ccref_create_s2(int d, const double *basis, long M, const int32_t *modes, const double *V, const double *S0,
                      double shift, int nthreads)
{
	if (d < 1 || d > 4 || M < 0)
		return nullptr;
	RefHandle *h = new RefHandle();
	h->d = d;
	for (int i = 0; i < d; i++)
		h->basis.push_back(MakeVec(d, basis + d * i));
	h->config = EmptyConfig(h);
	ShiftedCCPotential_S2 *s2 = new ShiftedCCPotential_S2(d);
	h->pot.reset(s2);
	h->nthreads = nthreads < 1 ? 1 : nthreads;
	h->pot->ParallelNumThread = h->nthreads;
	h->pot->Shift = shift;
	for (long m = 0; m < M; m++) {
		GeometryVector k(d);
		for (int e = 0; e < d; e++)
			k.AddFrom(static_cast<double>(modes[m * d + e]) * h->config->GetReciprocalBasisVector(e));
		s2->AddConstraint(k, std::vector<double>{V[m], S0[m]});
	}
	return h;
}

// The reference's ShiftedCCPotential_S2_MultiConfig (potential/CollectiveCoordinatePotential.h:1756-1870) over nsub
// sub-configurations, constraints and targets appended to its public lists as the CLI's Type 15 does
// (apps/CollectiveCoordinateCLI/CollectiveCoordinateCLI.cpp:524-540). N must be a multiple of nsub when positions are set.
void *ccref_create_s2_multiconfig(int d, const double *basis, long M, const int32_t *modes, const double *V,
                                  const double *S0, double shift, int nsub, int nthreads)
{
	if (d < 1 || d > 4 || M < 0 || nsub < 1)
		return nullptr;
	RefHandle *h = new RefHandle();
	h->d = d;
	for (int i = 0; i < d; i++)
		h->basis.push_back(MakeVec(d, basis + d * i));
	h->config = EmptyConfig(h);
	ShiftedCCPotential_S2_MultiConfig *mc = new ShiftedCCPotential_S2_MultiConfig(d, (size_t)nsub);
	h->pot.reset(mc);
	h->nthreads = nthreads < 1 ? 1 : nthreads;
	h->pot->ParallelNumThread = h->nthreads;
	h->pot->Shift = shift;
	for (long m = 0; m < M; m++) {
		GeometryVector k(d);
		for (int e = 0; e < d; e++)
			k.AddFrom(static_cast<double>(modes[m * d + e]) * h->config->GetReciprocalBasisVector(e));
		mc->constraints.emplace_back(k, V[m]);
		mc->S0.push_back(S0[m]);
	}
	return h;
}

// The named variable-cell potentials of potential/CCPotential_Kernels.h:190-191, 339-358 at the cell `basis`:
//   0 K2Potential, 1 KM3Potential (ShiftedCCPotential_varBox), 2 K2K2Potential, 3 K2K2Potential_noV0,
//   4 KM3K2Potential_noV0, 5 KM2K2Potential, 6 KM3K2Potential, 7 KM4K2Potential, 8 KM3KM2Potential,
//   9 KM3KMLogPotential, 10-12 KM2/KM3/KM4KnPotential(n), 13-15 KM2/KM3/KM4KlcPotential(n).
// Their constraints (k within rK, weights tildeV(k)) and shifts are generated by their own SetConfiguration, i.e. by
// ccref_set_positions.
void *ccref_create_varbox(int kind, int d, const double *basis, double rK, double n, int nthreads)
{
	if (d < 1 || d > 4 || kind < 0 || kind > 15)
		return nullptr;
	RefHandle *h = new RefHandle();
	h->d = d;
	for (int i = 0; i < d; i++)
		h->basis.push_back(MakeVec(d, basis + d * i));
	h->config = EmptyConfig(h);
	auto plain = [&](auto *q) {
		h->weights = [q](const GeometryVector &k, double *v, double *s0) { q->eval(k, v, s0); };
		h->pot.reset(q);
	};
	auto s2 = [&](auto *q) {
		plain(q);
		h->s2 = q;
	};
	switch (kind) {
	case 0: plain(new ProbeV<K2Potential>(d, rK)); break;
	case 1: plain(new ProbeV<KM3Potential>(d, rK)); break;
	case 2: s2(new ProbeVS<K2K2Potential>(d, rK)); break;
	case 3: s2(new ProbeVS<K2K2Potential_noV0>(d, rK)); break;
	case 4: s2(new ProbeVS<KM3K2Potential_noV0>(d, rK)); break;
	case 5: s2(new ProbeVS<KM2K2Potential>(d, rK)); break;
	case 6: s2(new ProbeVS<KM3K2Potential>(d, rK)); break;
	case 7: s2(new ProbeVS<KM4K2Potential>(d, rK)); break;
	case 8: s2(new ProbeVS<KM3KM2Potential>(d, rK)); break;
	case 9: s2(new ProbeVS<KM3KMLogPotential>(d, rK)); break;
	case 10: s2(new ProbeVS<KM2KnPotential>(d, n, rK)); break;
	case 11: s2(new ProbeVS<KM3KnPotential>(d, n, rK)); break;
	case 12: s2(new ProbeVS<KM4KnPotential>(d, n, rK)); break;
	case 13: s2(new ProbeVS<KM2KlcPotential>(d, n, rK)); break;
	case 14: s2(new ProbeVS<KM3KlcPotential>(d, n, rK)); break;
	default: s2(new ProbeVS<KM4KlcPotential>(d, n, rK)); break;
	}
	h->nthreads = nthreads < 1 ? 1 : nthreads;
	h->pot->ParallelNumThread = h->nthreads;
	return h;
}

// Constraint count, Shift and, for the S2 kinds, the length of the S0 list (-1 for the plain kinds).
void ccref_varbox_state(void *p, long *M, double *shift, long *nS0)
{
	RefHandle *h = static_cast<RefHandle *>(p);
	*M = (long)h->pot->constraints.size();
	*shift = h->pot->Shift;
	*nS0 = h->s2 ? (long)h->s2->S0.size() : -1;
}

// The constraints' Cartesian k (M x d) and weights V (M).
void ccref_constraints(void *p, double *k, double *V)
{
	RefHandle *h = static_cast<RefHandle *>(p);
	for (size_t m = 0; m < h->pot->constraints.size(); m++) {
		for (int e = 0; e < h->d; e++)
			k[m * h->d + e] = h->pot->constraints[m].k.x[e];
		V[m] = h->pot->constraints[m].V;
	}
}

// tildeV(k) and S0(k) of a varBox handle's class at M Cartesian wavevectors.
void ccref_varbox_weights(void *p, long M, const double *k, double *V, double *S0)
{
	RefHandle *h = static_cast<RefHandle *>(p);
	for (long m = 0; m < M; m++)
		h->weights(MakeVec(h->d, k + m * h->d), V + m, S0 + m);
}

void ccref_destroy(void *p) { delete static_cast<RefHandle *>(p); }

// Cartesian k of every constraint (M x d).
void ccref_kcart(void *p, double *out)
{
	RefHandle *h = static_cast<RefHandle *>(p);
	for (size_t m = 0; m < h->pot->constraints.size(); m++)
		for (int e = 0; e < h->d; e++)
			out[m * h->d + e] = h->pot->constraints[m].k.x[e];
}

double ccref_volume(void *p) { return static_cast<RefHandle *>(p)->config->PeriodicVolume(); }

// Reciprocal basis vectors (d x d, row e = b_e), as the reference computes them.
void ccref_reciprocal(void *p, double *out)
{
	RefHandle *h = static_cast<RefHandle *>(p);
	for (int e = 0; e < h->d; e++) {
		GeometryVector b = h->config->GetReciprocalBasisVector(e);
		for (int c = 0; c < h->d; c++)
			out[e * h->d + c] = b.x[c];
	}
}

// Insert N particles at fractional coordinates (N x d) and bind them (the reference's SetConfiguration).
void ccref_set_positions(void *p, long N, const double *frac)
{
	RefHandle *h = static_cast<RefHandle *>(p);
	Fill(h, *h->config, N, frac, 1.0);
	h->pot->SetConfiguration(*h->config);
}

// Energy() then AllForce(): E, Cartesian forces (N x d, may be null), rho (M each, may be null).
void ccref_eval(void *p, double *E, double *F, double *rhoRe, double *rhoIm)
{
	RefHandle *h = static_cast<RefHandle *>(p);
	*E = h->pot->Energy();
	if (F) {
		std::vector<GeometryVector> forces;
		h->pot->AllForce(forces);
		for (size_t i = 0; i < forces.size(); i++)
			for (int e = 0; e < h->d; e++)
				F[i * h->d + e] = forces[i].x[e];
	}
	// M values (a multi-configuration potential holds M per sub-configuration: the first sub-configuration's)
	const size_t M = std::min(h->pot->constraints.size(), h->pot->RhoReal.size());
	if (rhoRe)
		std::memcpy(rhoRe, h->pot->RhoReal.data(), sizeof(double) * M);
	if (rhoIm)
		std::memcpy(rhoIm, h->pot->RhoImag.data(), sizeof(double) * M);
}

// The reference's single-particle Force(i).
void ccref_force_one(void *p, long i, double *f)
{
	RefHandle *h = static_cast<RefHandle *>(p);
	GeometryVector r;
	h->pot->Force(r, static_cast<size_t>(i));
	for (int e = 0; e < h->d; e++)
		f[e] = r.x[e];
}

// Cartesian coordinates of the bound particles, as the reference derives them (N x d).
void ccref_cartesian(void *p, double *out)
{
	RefHandle *h = static_cast<RefHandle *>(p);
	for (size_t i = 0; i < h->config->NumParticle(); i++) {
		GeometryVector c = h->config->GetCartesianCoordinates(i);
		for (int e = 0; e < h->d; e++)
			out[i * h->d + e] = c.x[e];
	}
}

// Restated S(k) = |sum_j exp(i k.r_j)|^2 / N of pairstat/StructureFactor.cpp:56-65 on the bound particles, for
// K Cartesian wavevectors (K x d). Uses std::complex exp as the reference does.
void ccref_structure_factor(void *p, long K, const double *kcart, double *S)
{
	RefHandle *h = static_cast<RefHandle *>(p);
	const size_t np = h->config->NumParticle();
#pragma omp parallel for schedule(guided) num_threads(h->nthreads)
	for (long q = 0; q < K; q++) {
		GeometryVector k = MakeVec(h->d, kcart + q * h->d);
		std::complex<double> rho;
		for (size_t i = 0; i < np; i++)
			rho += std::exp(std::complex<double>(0, k.Dot(h->config->GetCartesianCoordinates(i))));
		S[q] = (rho.real() * rho.real() + rho.imag() * rho.imag()) / np;
	}
}

// The reference's ShiftedCCPotential_ForMC::TryMove (:1931-1950) on the bound configuration, for a move of one
// particle between two fractional positions (converted to Cartesian with the cell); accept = 1 also runs AcceptMove
// and keeps the ForMC object for later calls (its rho then follows the accepted moves, as in an MC run).
double ccref_mc_trymove(void *p, const double *s_prev, const double *s_after, int accept)
{
	RefHandle *h = static_cast<RefHandle *>(p);
	std::unique_ptr<ShiftedCCPotential_ForMC> &mc = h->mc;
	if (!mc) {
		h->pot->SetConfiguration(*h->config);
		mc.reset(new ShiftedCCPotential_ForMC(*h->pot));
		mc->SetConfiguration(*h->config);
		mc->GetRho();
	}
	GeometryVector a(h->d), b(h->d);
	for (int i = 0; i < h->d; i++) {
		a.AddFrom(s_prev[i] * h->basis[i]);
		b.AddFrom(s_after[i] * h->basis[i]);
	}
	const double dE = mc->TryMove(a, b);
	if (accept)
		mc->AcceptMove();
	return dE;
}

// Restated three-pass minimisation (RelaxStructure_NLOPT / _Emin, StructureOptimization.cpp:1046-1090) with the
// reference's LuksanPLIS as the inner L-BFGS. frac (N x d) is the start and receives the result.
// emin < 0: the plain three-pass driver (stop value -MaxEnergy in every pass); emin >= 0: the _Emin driver.
// fast: LuksanPLIS arithmetic mode (0 = NLopt's order). Returns the final energy; *evals gets the total count.
double ccref_minimize(void *p, long N, double *frac, double emin, long maxeval, int history, int fast, long *evals)
{
	RefHandle *h = static_cast<RefHandle *>(p);
	const int d = h->d;
	const double rescales[3] = {10000.0, 1.0, 0.01};
	const double fmin = emin >= 0 ? emin : -::MaxEnergy;
	long total = 0;
	std::vector<double> x(static_cast<size_t>(N) * d);
	std::unique_ptr<Configuration> work = EmptyConfig(h);
	for (int pass = 0; pass < 3; pass++) {
		Fill(h, *h->config, N, frac, 1.0);
		h->pot->SetConfiguration(*h->config);
		if (h->pot->Energy() < fmin)
			break;
		for (long i = 0; i < N; i++)
			for (int j = 0; j < d; j++)
				x[i * d + j] = h->config->GetRelativeCoordinates(i).x[j] * rescales[pass];
		Aux aux{h, N, rescales[pass], 0, work.get()};
		double minf = 0.0;
		LuksanPLIS(static_cast<int>(N * d), Objective, &aux, x.data(), &minf, fmin, static_cast<int>(maxeval), history,
		           nullptr, fast);
		total += aux.evaluations;
		// GetConfig: wrap the final iterate into the box again.
		Fill(h, *h->config, N, x.data(), rescales[pass]);
		for (long i = 0; i < N; i++)
			for (int j = 0; j < d; j++)
				frac[i * d + j] = h->config->GetRelativeCoordinates(i).x[j];
	}
	Fill(h, *h->config, N, frac, 1.0);
	h->pot->SetConfiguration(*h->config);
	if (evals)
		*evals = total;
	return h->pot->Energy();
}

// Restated GeneratePotential Type 0..3 (CollectiveCoordinateCLI.cpp:180-265): enumerate the reciprocal lattice with
// the reference's own cell list inside the CLI's radius, keep one of each +-k pair (first nonzero index > 0), sort by
// |k|^2, take ceil(chi*N*d) and complete the last shell (relative tolerance 1e-10), then apply the Type 1-3 weights.
// Writes up to cap modes (integer indices, cap x d) and weights; returns the count, or -1 if cap is too small.
long ccref_kset_cli(int d, const double *basis, long N, double chi, int type, long cap, int32_t *modes, double *V)
{
	RefHandle tmp;
	tmp.d = d;
	for (int i = 0; i < d; i++)
		tmp.basis.push_back(MakeVec(d, basis + d * i));
	std::unique_ptr<Configuration> config = EmptyConfig(&tmp);
	const size_t want = static_cast<size_t>(std::ceil(chi * N * d));
	const double maxk = (std::sqrt(static_cast<double>(d)) / 2) * std::pow((2 * static_cast<double>(d) * want), (1.0 / d)) *
	                    (2 * pi / std::pow(config->PeriodicVolume(), 1.0 / d));
	std::vector<GeometryVector> recip;
	for (int i = 0; i < d; i++)
		recip.push_back(config->GetReciprocalBasisVector(i));
	PeriodicCellList<Empty> lattice(d, &recip[0], std::sqrt(recip[0].Modulus2()) * 1.1, false);
	lattice.Insert(Empty(), GeometryVector(d));
	struct Entry {
		GeometryVector k;
		long n[4];
	};
	std::vector<Entry> found;
	lattice.IterateThroughNeighbors(GeometryVector(d), maxk,
	    [&](const GeometryVector &shift, const GeometryVector &, const signed long *ps, const size_t) {
		    int sign = 0;
		    for (int i = 0; i < d && sign == 0; i++)
			    sign = ps[i] > 0 ? 1 : (ps[i] < 0 ? -1 : 0);
		    if (sign > 0) {
			    Entry e;
			    e.k = shift;
			    for (int i = 0; i < 4; i++)
				    e.n[i] = i < d ? ps[i] : 0;
			    found.push_back(e);
		    }
	    });
	std::sort(found.begin(), found.end(), [](const Entry &a, const Entry &b) { return a.k.Modulus2() < b.k.Modulus2(); });
	size_t count = 0;
	double last = 0;
	while (count < found.size()) {
		const double k2 = found[count].k.Modulus2();
		if (!(count < want || std::abs((last - k2) / last) < 1e-10))
			break;
		last = k2;
		count++;
	}
	if (static_cast<long>(count) > cap)
		return -1;
	const double K2 = count < found.size() ? found[count].k.Modulus2() : 0.0;
	for (size_t m = 0; m < count; m++) {
		// The enumeration reports the lattice shift of the image; map it to the index of k = sum n_i b_i.
		GeometryVector check(d);
		for (int i = 0; i < d; i++)
			check.AddFrom(static_cast<double>(found[m].n[i]) * recip[i]);
		double s = (check.Dot(found[m].k) >= 0) ? 1.0 : -1.0;
		for (int i = 0; i < d; i++)
			modes[m * d + i] = static_cast<int32_t>(s * found[m].n[i]);
		double w = 1.0;
		if (type >= 1 && type <= 3) {
			double kk = std::sqrt(found[m].k.Modulus2() / K2);
			if (type == 1)
				w = std::acos(kk) - kk * std::sqrt(1 - found[m].k.Modulus2() / K2);
			else if (type == 2)
				w = std::pow(1.0 - kk, 6.0);
			else
				w = std::pow(1.0 - kk, 2.0);
		}
		V[m] = w;
	}
	return static_cast<long>(count);
}

}  // extern "C"
