/* GpuMultiStealthyPotential.h — drop-in GPU replacement for the reference's MultiStealthyPotential (header-only C++
 * adapter over the cc_multi_* entry points of libccgpu.so).
 *
 * Include it in code built against the reference (apps/CCOptimization/MultiStealthyPotential.h and the potential/ and
 * core/ headers on the include path) and link libccgpu.so. The class derives from MultiStealthyPotential
 * (apps/CCOptimization/MultiStealthyPotential.h:115-481), so species, constraints, radii, u0 and e0 are set exactly as
 * on the reference object (SetNumSpecies, AddConstraint, SetConfiguration, SetSpeciesOfParticle, SetSecureRadii /
 * SetPacking, the public u0 / e0); Energy, Force, AllForce and EnergyAndAllForce run on the GPU:
 *   E   = u0 sum_s (N_s/N) Phi_s + e0 sum_{i<j, images} [r < R_i + R_j] (1 - r / (R_i + R_j))^2,
 * with the reference's forces, its default radii (0.5) and its rule for coincident particles.
 *
 * Contract kept from the reference:
 *   - every particle needs a species (std::runtime_error otherwise, as the reference);
 *   - every constraint k must lie on the reciprocal lattice of the cell (std::invalid_argument otherwise);
 *   - EnergyAndAllForce equals Energy() followed by AllForce() bitwise (both read one cached GPU evaluation, made again
 *     when the positions, species, radii, constraints, u0 or e0 changed);
 *   - one object is not evaluated from several threads at once.
 */
#ifndef GPU_MULTI_STEALTHY_POTENTIAL_H
#define GPU_MULTI_STEALTHY_POTENTIAL_H

#include "MultiStealthyPotential.h"
#include "cc_gpu.h"

#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

class GpuMultiStealthyPotential : public MultiStealthyPotential
{
	cc_multi *handle_ = nullptr;
	// what the handle was built from, and the inputs of the cached evaluation
	std::vector<double> basis_;
	std::vector<std::vector<int32_t> > modes_;
	std::vector<std::vector<double> > V_;
	double u0_ = 0.0, e0_ = 0.0;
	std::vector<double> frac_, radii_in_;
	std::vector<int32_t> species_;
	std::vector<double> forces_;
	double energy_ = 0.0;
	bool valid_ = false, positions_dirty_ = true;

	static void Check(int rc)
	{
		if (rc == CC_OK)
			return;
		const std::string msg = std::string("GpuMultiStealthyPotential: ") + cc_last_error();
		if (rc == CC_ERR_ARG || rc == CC_ERR_NONLATTICE)
			throw std::invalid_argument(msg);
		if (rc == CC_ERR_STATE)
			throw std::logic_error(msg);
		throw std::runtime_error(msg);
	}

	void Evaluate()
	{
		if (!this->pConfig)
			throw std::logic_error("GpuMultiStealthyPotential: no configuration bound");
		const Configuration &c = *this->pConfig;
		const int d = this->Dimension;
		const size_t n = c.NumParticle();
		// the handle: cell, per-species integer modes (n_e = k . a_e / 2 pi), weights, u0, e0
		std::vector<double> basis(d * d);
		for (int i = 0; i < d; i++)
			for (int j = 0; j < d; j++)
				basis[i * d + j] = c.GetBasisVector(i).x[j];
		const size_t S = this->species_constraints.size();
		std::vector<std::vector<int32_t> > modes(S);
		std::vector<std::vector<double> > V(S);
		for (size_t s = 0; s < S; s++)
			for (const auto &q : this->species_constraints[s].CCPotential->constraints) {
				for (int e = 0; e < d; e++) {
					const double x = q.k.Dot(c.GetBasisVector(e)) / (2.0 * M_PI), r = std::round(x);
					if (!(std::fabs(x - r) <= 1e-9 * std::max(1.0, std::fabs(r))))
						throw std::invalid_argument("GpuMultiStealthyPotential: a constraint k is off the reciprocal lattice");
					modes[s].push_back((int32_t)r);
				}
				V[s].push_back(q.V);
			}
		if (!handle_ || basis != basis_ || modes != modes_ || V != V_ || this->u0 != u0_ || this->e0 != e0_) {
			cc_multi_destroy(handle_);
			handle_ = nullptr;
			std::vector<int64_t> M(S);
			std::vector<const int32_t *> mp(S);
			std::vector<const double *> vp(S);
			for (size_t s = 0; s < S; s++) {
				M[s] = (int64_t)V[s].size();
				mp[s] = modes[s].data();
				vp[s] = V[s].data();
			}
			Check(cc_multi_create(d, basis.data(), (int)S, M.data(), mp.data(), vp.data(), this->u0, this->e0,
			                      &handle_));
			basis_.swap(basis);
			modes_.swap(modes);
			V_.swap(V);
			u0_ = this->u0;
			e0_ = this->e0;
			valid_ = false;
		}
		// positions, species and radii of this evaluation
		std::vector<int32_t> species(n);
		for (size_t i = 0; i < n; i++) {
			species[i] = this->idx2species.size() == n ? this->idx2species[i].species : -1;
			if (species[i] < 0)
				throw std::runtime_error("GpuMultiStealthyPotential: particle has no assigned species; assign every "
				                         "particle before evaluating.");
		}
		const bool own_radii = this->radii.size() == n && this->rc >= 0.0;
		std::vector<double> radii = own_radii ? this->radii : std::vector<double>();
		if (positions_dirty_ || species != species_ || radii != radii_in_ || !valid_) {
			frac_.resize(n * d);
			for (size_t i = 0; i < n; i++)
				for (int e = 0; e < d; e++)
					frac_[i * d + e] = c.GetRelativeCoordinates(i).x[e];
			Check(cc_multi_set_configuration(handle_, (int64_t)n, frac_.data(), species.data(),
			                                 own_radii ? radii.data() : nullptr));
			species_.swap(species);
			radii_in_.swap(radii);
			positions_dirty_ = false;
			forces_.resize(n * d);
			Check(cc_multi_energy_grad(handle_, &energy_, forces_.data()));
			valid_ = true;
		}
	}

public:
	GpuMultiStealthyPotential(DimensionType dimension, double epsilon) : MultiStealthyPotential(dimension, epsilon) {}
	GpuMultiStealthyPotential(const GpuMultiStealthyPotential &) = delete;
	GpuMultiStealthyPotential &operator=(const GpuMultiStealthyPotential &) = delete;
	~GpuMultiStealthyPotential() override { cc_multi_destroy(handle_); }

	void SetConfiguration(const Configuration &Position) override
	{
		MultiStealthyPotential::SetConfiguration(Position);
		positions_dirty_ = true;
	}

	double Energy() override
	{
		Evaluate();
		return energy_;
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
			throw std::out_of_range("GpuMultiStealthyPotential::Force: particle index out of range");
		result = GeometryVector(d);
		for (int e = 0; e < d; e++)
			result.x[e] = forces_[i * d + e];
	}

	double EnergyAndAllForce(std::vector<GeometryVector> &results) override
	{
		AllForce(results);
		return energy_;
	}
};

#endif
