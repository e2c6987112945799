/* GpuRepulsiveCCPotential.h — drop-in GPU replacement for the reference's RepulsiveCCPotential, the potential of the
 * one-component optimiser GetCCO (header-only C++ adapter over the cc_multi_* entry points of libccgpu.so).
 *
 * Include it in code built against the reference (apps/CCOptimization/RepulsiveCCPotential.h and the potential/ and
 * core/ headers on the include path) and link libccgpu.so. The class derives from RepulsiveCCPotential
 * (apps/CCOptimization/RepulsiveCCPotential.h:21-159): e0, sigma and the collective-coordinate member CCPotential (a
 * ShiftedCCPotential, or a ShiftedCCPotential_S2 when constructed with S0 != 0, filled through its AddConstraint) are
 * the reference's own; Energy, Force, AllForce and EnergyAndAllForce run on the GPU as a one-species cc_multi with
 * radii sigma / 2:
 *   E = e0 sum_{i<j, images} [r < sigma] (1 - r / sigma)^2 + Phi_CC,
 * with the reference's forces and its rule for coincident particles.
 *
 * Contract kept from the reference:
 *   - every constraint k must lie on the reciprocal lattice of the cell (std::invalid_argument otherwise);
 *   - EnergyAndAllForce equals Energy() followed by AllForce() bitwise (one cached GPU evaluation, made again when the
 *     positions, constraints, targets, e0 or sigma changed);
 *   - SetConfiguration binds a Configuration the caller keeps alive (non-owning); positions changed inside it are seen
 *     at the next SetConfiguration, as the optimiser's objective calls it every step;
 *   - one object is not evaluated from several threads at once.
 */
#ifndef GPU_REPULSIVE_CC_POTENTIAL_H
#define GPU_REPULSIVE_CC_POTENTIAL_H

#include "CombinedEnergyForce.h"
#include "RepulsiveCCPotential.h"
#include "cc_gpu.h"

#include <cmath>
#include <stdexcept>
#include <string>
#include <typeinfo>
#include <vector>

class GpuRepulsiveCCPotential : public RepulsiveCCPotential, public CombinedEnergyForce
{
	cc_multi *handle_ = nullptr;
	std::vector<double> basis_, V_, S0_, frac_, forces_;
	std::vector<int32_t> modes_;
	double e0_ = 0.0, sigma_ = 0.0, energy_ = 0.0;
	bool s2_ = false, valid_ = false, positions_dirty_ = true;

	static void Check(int rc)
	{
		if (rc == CC_OK)
			return;
		const std::string msg = std::string("GpuRepulsiveCCPotential: ") + cc_last_error();
		if (rc == CC_ERR_ARG || rc == CC_ERR_NONLATTICE)
			throw std::invalid_argument(msg);
		if (rc == CC_ERR_STATE)
			throw std::logic_error(msg);
		throw std::runtime_error(msg);
	}

	void Evaluate()
	{
		if (!this->pConfig)
			throw std::logic_error("GpuRepulsiveCCPotential: no configuration bound");
		const Configuration &c = *this->pConfig;
		const int d = this->Dimension;
		const size_t n = c.NumParticle();
		std::vector<double> basis(d * d), V;
		std::vector<int32_t> modes;
		for (int i = 0; i < d; i++)
			for (int j = 0; j < d; j++)
				basis[i * d + j] = c.GetBasisVector(i).x[j];
		for (const auto &q : this->CCPotential->constraints) {
			for (int e = 0; e < d; e++) {
				const double x = q.k.Dot(c.GetBasisVector(e)) / (2.0 * M_PI), r = std::round(x);
				if (!(std::fabs(x - r) <= 1e-9 * std::max(1.0, std::fabs(r))))
					throw std::invalid_argument("GpuRepulsiveCCPotential: a constraint k is off the reciprocal lattice");
				modes.push_back((int32_t)r);
			}
			V.push_back(q.V);
		}
		// the two kernels the reference's constructor makes; another subclass put in CCPotential would have a form
		// of its own, which this adapter does not evaluate
		const ShiftedCCPotential &cc = *this->CCPotential;
		if (typeid(cc) != typeid(ShiftedCCPotential) && typeid(cc) != typeid(ShiftedCCPotential_S2))
			throw std::invalid_argument("GpuRepulsiveCCPotential: CCPotential must be a ShiftedCCPotential or a "
			                            "ShiftedCCPotential_S2");
		const ShiftedCCPotential_S2 *s2 = dynamic_cast<const ShiftedCCPotential_S2 *>(this->CCPotential.get());
		// the repulsion is on or off as the reference's constructor decided (WithRepulsion), not by the current e0
		const double e0 = this->WithRepulsion ? this->e0 : 0.0;
		const std::vector<double> S0 = s2 ? s2->S0 : std::vector<double>();
		if (s2 && S0.size() != V.size())
			throw std::invalid_argument("GpuRepulsiveCCPotential: the S2 kernel needs one S0 per constraint");
		if (!handle_ || basis != basis_ || modes != modes_ || V != V_ || S0 != S0_ || (s2 != nullptr) != s2_ ||
		    e0 != e0_ || this->sigma != sigma_) {
			cc_multi_destroy(handle_);
			handle_ = nullptr;
			const int64_t M = (int64_t)V.size();
			const int32_t *mp = modes.data();
			const double *vp = V.data(), *sp = s2 ? S0.data() : nullptr;
			Check(cc_multi_create_s2(d, basis.data(), 1, &M, &mp, &vp, &sp, 1.0, e0, &handle_));
			basis_.swap(basis);
			modes_.swap(modes);
			V_.swap(V);
			S0_ = S0;
			s2_ = s2 != nullptr;
			e0_ = e0;
			sigma_ = this->sigma;
			positions_dirty_ = true;
		}
		if (positions_dirty_ || !valid_) {
			frac_.resize(n * d);
			for (size_t i = 0; i < n; i++)
				for (int e = 0; e < d; e++)
					frac_[i * d + e] = c.GetRelativeCoordinates(i).x[e];
			const std::vector<int32_t> species(n, 0);
			const std::vector<double> radii(n, 0.5 * this->sigma);
			Check(cc_multi_set_configuration(handle_, (int64_t)n, frac_.data(), species.data(), radii.data()));
			forces_.resize(n * d);
			Check(cc_multi_energy_grad(handle_, &energy_, forces_.data()));
			positions_dirty_ = false;
			valid_ = true;
		}
	}

public:
	GpuRepulsiveCCPotential(DimensionType dim, double epsilon, double sigma, double S0 = 0.0)
	    : RepulsiveCCPotential(dim, epsilon, sigma, S0)
	{
	}
	GpuRepulsiveCCPotential(const GpuRepulsiveCCPotential &) = delete;
	GpuRepulsiveCCPotential &operator=(const GpuRepulsiveCCPotential &) = delete;
	~GpuRepulsiveCCPotential() override { cc_multi_destroy(handle_); }

	// Binds the configuration (non-owning) without the reference's CPU neighbour-list preparation.
	void SetConfiguration(const Configuration &c) override
	{
		this->pConfig = &c;
		this->CCPotential->SetConfiguration(c);
		positions_dirty_ = true;
		valid_ = false;
	}

	// The collective-coordinate part's Shift is added as the reference's CCPotential->Energy() adds it
	// (potential/CollectiveCoordinatePotential.h:1371, :1705).
	double Energy() override
	{
		Evaluate();
		return energy_ + this->CCPotential->Shift;
	}

	void AllForce(std::vector<GeometryVector> &results) override
	{
		Evaluate();
		const int d = this->Dimension;
		const size_t n = forces_.size() / d;
		results.assign(n, GeometryVector(d));
		for (size_t i = 0; i < n; i++)
			for (int e = 0; e < d; e++)
				results[i].x[e] = forces_[i * d + e];
	}

	void Force(GeometryVector &result, size_t i) override
	{
		Evaluate();
		const int d = this->Dimension;
		if (i >= forces_.size() / d)
			throw std::out_of_range("GpuRepulsiveCCPotential::Force: particle index out of range");
		result = GeometryVector(d);
		for (int e = 0; e < d; e++)
			result.x[e] = forces_[i * d + e];
	}

	double EnergyAndAllForce(std::vector<GeometryVector> &results) override
	{
		AllForce(results);
		return energy_ + this->CCPotential->Shift;
	}
};

#endif
