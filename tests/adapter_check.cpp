// GPU adapter check, compiled against the reference's own headers (and the oracle's stand-ins) and linked with the
// reference build (oracle/_ref/libccref.so: LuksanPLIS, Potential::~Potential, Volume) and libccgpu.so.
//   1. GpuCCPotential (include/GpuCCPotential.h) against the reference's ShiftedCCPotential on the same
//      Configuration and constraints: Energy, AllForce, Force(i), EnergyAndAllForce, GetRho (1e-10 of the scales).
//   3. GpuMultiStealthyPotential (include/GpuMultiStealthyPotential.h) against the reference's MultiStealthyPotential
//      (compiled into oracle/_ref/libccref.so) on a skew 2D cell with three species and unequal radii: Energy and
//      AllForce (1e-10), and EnergyAndAllForce equal to Energy then AllForce bitwise.
//   2. The structure optimiser's Switch-0 objective (restated from potential/StructureOptimization.cpp:447-536) finds
//      CombinedEnergyForce by dynamic_cast and drives the reference's LuksanPLIS with the GPU adapter to the
//      stealthy ground state of a 2D N=100 chi=0.30 configuration (E/N < 1e-20).
//   4. GpuCCPotential_S2 against the reference's ShiftedCCPotential_S2 (constraints through AddConstraint(k, {V, S0}))
//      on a skew 2D cell: Energy and AllForce within 1e-10 of the S2 rounding scales, Force(i), EnergyAndAllForce
//      bitwise, and a changed S0 seen at the next evaluation.
//   5. GpuCCPotential_S2_MultiConfig against the reference's ShiftedCCPotential_S2_MultiConfig (3 sub-configurations,
//      skew 3D cell): Energy and AllForce within 1e-10 of the S2 rounding scales.
//   6. GpuRepulsiveCCPotential against the reference's RepulsiveCCPotential (GetCCO's potential) with the plain and
//      the S2 kernel on a skew 2D cell with contacts: Energy and AllForce within 1e-10 of max(1, |E|) and max(1, |F|).
// Prints one line per check and exits 0 only if all pass.
#include "GpuCCPotential.h"
#include "GpuMultiStealthyPotential.h"
#include "GpuRepulsiveCCPotential.h"
#include "LuksanPLIS.h"

#include <cmath>
#include <iostream>
#include <cstdio>
#include <random>
#include <vector>

static int failures = 0;
static void check(bool ok, const char *what, double a, double b)
{
	std::printf("%s %s: %.17g vs %.17g\n", ok ? "ok  " : "FAIL", what, a, b);
	if (!ok)
		failures++;
}

static Configuration make_config(int d, const std::vector<double> &rows, int n, std::mt19937_64 &rng)
{
	std::vector<GeometryVector> basis(d, GeometryVector(d));
	double maxlen = 0;
	for (int i = 0; i < d; i++) {
		for (int j = 0; j < d; j++)
			basis[i].x[j] = rows[i * d + j];
		maxlen = std::max(maxlen, std::sqrt(basis[i].Modulus2()));
	}
	Configuration c(d, basis.data(), 10 * maxlen);
	std::uniform_real_distribution<double> u(0, 1);
	for (int k = 0; k < n; k++) {
		GeometryVector s(d);
		for (int j = 0; j < d; j++)
			s.x[j] = u(rng);
		c.Insert("A", s);
	}
	return c;
}

struct Aux {
	Potential *pot;
	Configuration *work;
	int d;
	size_t n;
	double rescale;
};

// Switch-0 objective: x = rescale * relative coordinates; grad = -F . a_j / rescale; the combined call when offered
static double objective(unsigned nv, const double *x, double *grad, void *data)
{
	Aux *a = static_cast<Aux *>(data);
	a->work->RemoveParticles();
	for (size_t i = 0; i < a->n; i++) {
		GeometryVector r(a->d);
		for (int j = 0; j < a->d; j++)
			r.x[j] = x[a->d * i + j] / a->rescale;
		a->work->Insert("A", r);
	}
	a->pot->SetConfiguration(*a->work);
	CombinedEnergyForce *comb = grad ? dynamic_cast<CombinedEnergyForce *>(a->pot) : nullptr;
	std::vector<GeometryVector> f;
	const double E = comb ? comb->EnergyAndAllForce(f) : a->pot->Energy();
	if (grad) {
		if (!comb)
			a->pot->AllForce(f);
		for (unsigned i = 0; i < nv; i++)
			grad[i] = 0;
		for (size_t i = 0; i < a->n; i++)
			for (int j = 0; j < a->d; j++)
				grad[i * a->d + j] = -f[i].Dot(a->work->GetBasisVector(j)) / a->rescale;
	}
	return E;
}

int main()
{
	std::mt19937_64 rng(8080);
	// ---- 1. parity with the reference class on a skew 3D cell --------------------------------------------------
	{
		const int d = 3;
		Configuration c = make_config(d, {1.1, 0, 0, 0.3, 0.95, 0.1, 0.2, -0.25, 1.2}, 60, rng);
		ShiftedCCPotential ref(d);
		std::uniform_real_distribution<double> uv(-0.5, 1.5);
		for (int a = -3; a <= 3; a++)
			for (int b = -3; b <= 3; b++)
				for (int e = -3; e <= 3; e++) {
					GeometryVector k(d);
					k.AddFrom((double)a * c.GetReciprocalBasisVector(0));
					k.AddFrom((double)b * c.GetReciprocalBasisVector(1));
					k.AddFrom((double)e * c.GetReciprocalBasisVector(2));
					ref.constraints.emplace_back(k, uv(rng));
				}
		ref.Shift = 0.25;
		GpuCCPotential gpu(ref);
		ref.SetConfiguration(c);
		gpu.SetConfiguration(c);
		double sumV = 0, kmax = 0;
		for (auto &q : ref.constraints) {
			sumV += std::abs(q.V);
			kmax = std::max(kmax, std::sqrt(q.k.Modulus2()));
		}
		const double n = 60, vol = c.PeriodicVolume();
		const double sE = sumV * n * n / vol, sF = 4 * sumV * n * kmax / vol;
		const double Er = ref.Energy(), Eg = gpu.Energy();
		check(std::abs(Er - Eg) <= 1e-10 * std::abs(Er) + 1e-13 * sE, "Energy", Eg, Er);
		std::vector<GeometryVector> fr, fg, fc;
		ref.AllForce(fr);
		gpu.AllForce(fg);
		double worst = 0;
		for (size_t i = 0; i < fr.size(); i++)
			for (int j = 0; j < d; j++)
				worst = std::max(worst, std::abs(fr[i].x[j] - fg[i].x[j]));
		check(fg.size() == fr.size() && worst <= 1e-10 * sF, "AllForce max |dF| / scale", worst / sF, 1e-10);
		GeometryVector f1;
		gpu.Force(f1, 17);
		check(f1.x[0] == fg[17].x[0] && f1.x[2] == fg[17].x[2], "Force(i) == AllForce[i]", f1.x[0], fg[17].x[0]);
		const double Ec = gpu.EnergyAndAllForce(fc);
		bool same = Ec == Eg && fc.size() == fg.size();
		for (size_t i = 0; same && i < fc.size(); i++)
			for (int j = 0; j < d; j++)
				same = same && fc[i].x[j] == fg[i].x[j];
		check(same, "EnergyAndAllForce == Energy then AllForce (bitwise)", Ec, Eg);
		gpu.GetRho();
		ref.GetRho();
		double wr = 0;
		for (size_t q = 0; q < ref.RhoReal.size(); q++)
			wr = std::max(wr, std::abs(ref.RhoReal[q] - gpu.RhoReal[q]) + std::abs(ref.RhoImag[q] - gpu.RhoImag[q]));
		check(gpu.RhoValid && wr <= 1e-10 * n, "GetRho max |drho| / N", wr / n, 1e-10);
		// a changed constraint set is picked up at the next evaluation
		gpu.Shift = 1.5;
		ref.Shift = 1.5;
		check(std::abs(gpu.Energy() - ref.Energy()) <= 1e-10 * std::abs(Er) + 1e-13 * sE, "Shift change seen",
		      gpu.Energy(), ref.Energy());
	}
	// ---- 2. the optimiser's objective + LuksanPLIS to the ground state with the GPU adapter --------------------
	{
		const int d = 2, n = 100;
		Configuration c = make_config(d, {1, 0, 0, 1}, n, rng);
		GpuCCPotential gpu(d);
		// the CLI's Type 0 k-set (the library's generator reproduces GeneratePotential)
		std::vector<int32_t> modes(4096);
		std::vector<double> V(2048);
		int64_t M = 0;
		const double basis[4] = {1, 0, 0, 1};
		if (cc_kset_stealthy(d, basis, n, 0.30, 0, 2048, modes.data(), V.data(), &M) != CC_OK)
			return 2;
		for (int64_t q = 0; q < M; q++) {
			GeometryVector k(d);
			k.AddFrom((double)modes[q * d] * c.GetReciprocalBasisVector(0));
			k.AddFrom((double)modes[q * d + 1] * c.GetReciprocalBasisVector(1));
			gpu.constraints.emplace_back(k, V[q]);
		}
		Configuration work(c);
		Aux aux{&gpu, &work, d, (size_t)n, 1.0};
		std::vector<double> x(n * d);
		for (int i = 0; i < n; i++)
			for (int j = 0; j < d; j++)
				x[i * d + j] = c.GetRelativeCoordinates(i).x[j];
		double minf = 0;
		int evals = 0;
		const int st = LuksanPLIS(n * d, objective, &aux, x.data(), &minf, 1e-20 * n, 5000, 40, &evals, 0);
		std::printf("LuksanPLIS status %d after %d evaluations\n", st, evals);
		check(minf / n < 1e-20, "ground state E/N via Objective + LuksanPLIS + GpuCCPotential", minf / n, 1e-20);
	}
	// ---- 3. the multi-species potential with contact against the reference class ---------------------------------
	{
		const int d = 2, n = 90, S = 3;
		Configuration c = make_config(d, {10.0, 0.0, 3.0, 9.0}, n, rng);
		std::uniform_real_distribution<double> ur(0.25, 0.45);
		std::vector<double> radii(n);
		for (auto &r : radii)
			r = ur(rng);
		std::streambuf *saved = std::cout.rdbuf(nullptr);   // the reference reports its set-up on stdout
		MultiStealthyPotential ref(d, 1.0);
		GpuMultiStealthyPotential gpu(d, 1.0);
		ref.u0 = gpu.u0 = 1.5;
		ref.SetNumSpecies(S);
		gpu.SetNumSpecies(S);
		for (int s = 0; s < S; s++) {
			std::vector<int32_t> modes(2 * 512);
			std::vector<double> V(512);
			int64_t M = 0;
			const double basis[4] = {10.0, 0.0, 3.0, 9.0};
			if (cc_kset_stealthy(d, basis, n / S, 0.2 + 0.05 * s, 3, 512, modes.data(), V.data(), &M) != CC_OK)
				return 2;
			for (int64_t q = 0; q < M; q++) {
				GeometryVector k(d);
				k.AddFrom((double)modes[q * d] * c.GetReciprocalBasisVector(0));
				k.AddFrom((double)modes[q * d + 1] * c.GetReciprocalBasisVector(1));
				ref.AddConstraint(s, k, std::vector<double>{V[q]});
				gpu.AddConstraint(s, k, std::vector<double>{V[q]});
			}
		}
		ref.SetConfiguration(c);
		gpu.SetConfiguration(c);
		for (int i = 0; i < n; i++) {
			ref.SetSpeciesOfParticle(i, i % S);
			gpu.SetSpeciesOfParticle(i, i % S);
		}
		ref.SetSecureRadii(radii);
		gpu.SetSecureRadii(radii);
		std::cout.rdbuf(saved);
		const double Er = ref.Energy(), Eg = gpu.Energy();
		check(std::abs(Er - Eg) <= 1e-10 * std::abs(Er), "multi-species Energy", Eg, Er);
		std::vector<GeometryVector> fr, fg, fc;
		ref.AllForce(fr);
		gpu.AllForce(fg);
		double worst = 0, fmax = 1.0;
		for (size_t i = 0; i < fr.size(); i++)
			for (int j = 0; j < d; j++) {
				worst = std::max(worst, std::abs(fr[i].x[j] - fg[i].x[j]));
				fmax = std::max(fmax, std::abs(fr[i].x[j]));
			}
		check(fg.size() == fr.size() && worst <= 1e-10 * fmax, "multi-species AllForce max |dF| / max(1,|F|)",
		      worst / fmax, 1e-10);
		const double Ec = gpu.EnergyAndAllForce(fc);
		bool same = Ec == Eg && fc.size() == fg.size();
		for (size_t i = 0; same && i < fc.size(); i++)
			for (int j = 0; j < d; j++)
				same = same && fc[i].x[j] == fg[i].x[j];
		check(same, "multi-species EnergyAndAllForce == Energy then AllForce (bitwise)", Ec, Eg);
	}
	// ---- 4. the S2 form against the reference's ShiftedCCPotential_S2 --------------------------------------------
	{
		const int d = 2, n = 80;
		Configuration c = make_config(d, {9.0, 0.0, 2.0, 8.5}, n, rng);
		ShiftedCCPotential_S2 ref(d);
		GpuCCPotential_S2 gpu(d);
		std::uniform_real_distribution<double> uv(0.2, 2.0), us(0.0, 1.5);
		for (int a = -4; a <= 4; a++)
			for (int b = -4; b <= 4; b++) {
				if (a < 0 || (a == 0 && b <= 0))
					continue;
				GeometryVector k(d);
				k.AddFrom((double)a * c.GetReciprocalBasisVector(0));
				k.AddFrom((double)b * c.GetReciprocalBasisVector(1));
				const std::vector<double> vals{uv(rng), us(rng)};
				ref.AddConstraint(k, vals);
				gpu.AddConstraint(k, vals);
			}
		ref.Shift = gpu.Shift = -0.5;
		ref.SetConfiguration(c);
		gpu.SetConfiguration(c);
		ref.GetRho();
		double sE = 0, sF = 0;
		for (size_t q = 0; q < ref.constraints.size(); q++) {
			const double r2 = ref.RhoReal[q] * ref.RhoReal[q] + ref.RhoImag[q] * ref.RhoImag[q];
			const double dS = std::abs(r2 / n - ref.S0[q]) + 1;
			sE += std::abs(ref.constraints[q].V) * dS * dS;
			sF += 4.0 / n * std::abs(ref.constraints[q].V) * dS * (std::sqrt(r2) + 1) *
			      std::sqrt(ref.constraints[q].k.Modulus2());
		}
		const double Er = ref.Energy(), Eg = gpu.Energy();
		check(std::abs(Er - Eg) <= 1e-10 * sE, "S2 Energy", Eg, Er);
		std::vector<GeometryVector> fr, fg, fc;
		ref.AllForce(fr);
		gpu.AllForce(fg);
		double worst = 0;
		for (size_t i = 0; i < fr.size(); i++)
			for (int j = 0; j < d; j++)
				worst = std::max(worst, std::abs(fr[i].x[j] - fg[i].x[j]));
		check(fg.size() == fr.size() && worst <= 1e-10 * sF, "S2 AllForce max |dF| / scale", worst / sF, 1e-10);
		GeometryVector f1;
		gpu.Force(f1, 41);
		check(f1.x[0] == fg[41].x[0] && f1.x[1] == fg[41].x[1], "S2 Force(i) == AllForce[i]", f1.x[0], fg[41].x[0]);
		const double Ec = gpu.EnergyAndAllForce(fc);
		bool same = Ec == Eg && fc.size() == fg.size();
		for (size_t i = 0; same && i < fc.size(); i++)
			for (int j = 0; j < d; j++)
				same = same && fc[i].x[j] == fg[i].x[j];
		check(same, "S2 EnergyAndAllForce == Energy then AllForce (bitwise)", Ec, Eg);
		ref.S0[3] += 0.75;
		gpu.S0[3] += 0.75;
		ref.RhoValid = false;
		const double Er2 = ref.Energy(), Eg2 = gpu.Energy();
		check(Er2 != Er && std::abs(Er2 - Eg2) <= 1e-10 * sE, "S2 target change seen", Eg2, Er2);
	}
	// ---- 5. the multi-configuration S2 form against the reference's class ------------------------------------------
	{
		const int d = 3, nsub = 3, n = 3 * 40;
		Configuration c = make_config(d, {6.0, 0.0, 0.0, 1.0, 5.5, 0.0, -0.5, 0.75, 6.5}, n, rng);
		ShiftedCCPotential_S2_MultiConfig ref(d, nsub);
		GpuCCPotential_S2_MultiConfig gpu(d, nsub);
		std::uniform_real_distribution<double> uv(0.2, 2.0), us(0.0, 1.5);
		for (int a = -2; a <= 2; a++)
			for (int b = -2; b <= 2; b++)
				for (int e = -2; e <= 2; e++) {
					if (a < 0 || (a == 0 && (b < 0 || (b == 0 && e <= 0))))
						continue;
					GeometryVector k(d);
					k.AddFrom((double)a * c.GetReciprocalBasisVector(0));
					k.AddFrom((double)b * c.GetReciprocalBasisVector(1));
					k.AddFrom((double)e * c.GetReciprocalBasisVector(2));
					const double V = uv(rng), S0 = us(rng);
					ref.constraints.emplace_back(k, V);
					ref.S0.push_back(S0);
					gpu.constraints.emplace_back(k, V);
					gpu.S0.push_back(S0);
				}
		ref.SetConfiguration(c);
		gpu.SetConfiguration(c);
		const double Er = ref.Energy(), Eg = gpu.Energy();
		const int np = n / nsub;
		double sE = 0, sF = 0;
		for (size_t q = 0; q < ref.constraints.size(); q++) {
			double r2 = 0;
			for (int s = 0; s < nsub; s++) {
				const size_t at = (size_t)s * ref.constraints.size() + q;
				r2 += ref.RhoReal[at] * ref.RhoReal[at] + ref.RhoImag[at] * ref.RhoImag[at];
			}
			const double dS = std::abs(ref.Snow[q] - ref.S0[q]) + 1;
			sE += std::abs(ref.constraints[q].V) * dS * dS;
			sF += 4.0 / np * std::abs(ref.constraints[q].V) * dS * (std::sqrt(r2) + 1) *
			      std::sqrt(ref.constraints[q].k.Modulus2());
		}
		check(std::abs(Er - Eg) <= 1e-10 * sE, "S2 multi-configuration Energy", Eg, Er);
		std::vector<GeometryVector> fr, fg;
		ref.AllForce(fr);
		gpu.AllForce(fg);
		double worst = 0;
		for (size_t i = 0; i < fr.size(); i++)
			for (int j = 0; j < d; j++)
				worst = std::max(worst, std::abs(fr[i].x[j] - fg[i].x[j]));
		check(fg.size() == fr.size() && worst <= 1e-10 * sF, "S2 multi-configuration AllForce max |dF| / scale",
		      worst / sF, 1e-10);
		// NSubConfig is public: a new value applies from the next SetConfiguration on (the reference recomputes Np)
		ref.NSubConfig = gpu.NSubConfig = 2;
		ref.SetConfiguration(c);
		gpu.SetConfiguration(c);
		const double Er2 = ref.Energy(), Eg2 = gpu.Energy();
		check(Er2 != Er && std::abs(Er2 - Eg2) <= 1e-10 * sE, "S2 multi-configuration NSubConfig change seen", Eg2,
		      Er2);
	}
	// ---- 6. RepulsiveCCPotential, plain and S2 kernels -----------------------------------------------------------
	for (int withS0 = 0; withS0 < 2; withS0++) {
		const int d = 2, n = 90;
		Configuration c = make_config(d, {10.0, 0.0, 2.5, 9.0}, n, rng);
		std::streambuf *saved = std::cout.rdbuf(nullptr);   // the reference reports its set-up on stdout
		RepulsiveCCPotential ref(d, 1.25, 0.9, withS0 ? 1.0 : 0.0);
		GpuRepulsiveCCPotential gpu(d, 1.25, 0.9, withS0 ? 1.0 : 0.0);
		std::cout.rdbuf(saved);
		for (int a = 0; a <= 4; a++)
			for (int b = -4; b <= 4; b++) {
				if (a == 0 && b <= 0)
					continue;
				GeometryVector k(d);
				k.AddFrom((double)a * c.GetReciprocalBasisVector(0));
				k.AddFrom((double)b * c.GetReciprocalBasisVector(1));
				std::vector<double> vals{1.0 / (1.0 + a + std::abs(b))};
				if (withS0)
					vals.push_back(0.7);
				ref.CCPotential->AddConstraint(k, vals);
				gpu.CCPotential->AddConstraint(k, vals);
			}
		ref.SetConfiguration(c);
		gpu.SetConfiguration(c);
		const double Er = ref.Energy(), Eg = gpu.Energy();
		check(std::abs(Er - Eg) <= 1e-10 * std::max(1.0, std::abs(Er)),
		      withS0 ? "Repulsive (S2 kernel) Energy" : "Repulsive Energy", Eg, Er);
		// a nonzero Shift of the collective-coordinate part is in both energies
		ref.CCPotential->Shift = gpu.CCPotential->Shift = 0.375;
		const double Ers = ref.Energy(), Egs = gpu.Energy();
		check(std::abs(Ers - Egs) <= 1e-10 * std::max(1.0, std::abs(Ers)) && std::abs(Ers - Er - 0.375) <= 1e-12,
		      withS0 ? "Repulsive (S2 kernel) Energy with Shift" : "Repulsive Energy with Shift", Egs, Ers);
		std::vector<GeometryVector> fs;
		check(gpu.EnergyAndAllForce(fs) == Egs, "Repulsive EnergyAndAllForce equals Energy with Shift", Egs, Egs);
		ref.CCPotential->Shift = gpu.CCPotential->Shift = 0.0;
		std::vector<GeometryVector> fr, fg;
		ref.AllForce(fr);
		gpu.AllForce(fg);
		double worst = 0, fmax = 1.0;
		for (size_t i = 0; i < fr.size(); i++)
			for (int j = 0; j < d; j++) {
				worst = std::max(worst, std::abs(fr[i].x[j] - fg[i].x[j]));
				fmax = std::max(fmax, std::abs(fr[i].x[j]));
			}
		check(fg.size() == fr.size() && worst <= 1e-10 * fmax,
		      withS0 ? "Repulsive (S2 kernel) AllForce max |dF| / max(1,|F|)" : "Repulsive AllForce max |dF| / max(1,|F|)",
		      worst / fmax, 1e-10);
	}
	std::printf(failures ? "ADAPTER FAIL\n" : "ADAPTER OK\n");
	return failures ? 1 : 0;
}
