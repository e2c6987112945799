/* GpuCCPotential.h — drop-in GPU replacements for the reference's ShiftedCCPotential, ShiftedCCPotential_S2 and
 * ShiftedCCPotential_S2_MultiConfig (header-only C++ adapter).
 *
 * Include it in code built against the reference (it needs potential/CollectiveCoordinatePotential.h and
 * potential/CombinedEnergyForce.h on the include path) and link libccgpu.so. GpuCCPotential derives from
 * ShiftedCCPotential (potential/CollectiveCoordinatePotential.h:53-1497), GpuCCPotential_S2 from ShiftedCCPotential_S2
 * (:1642-1749; its AddConstraint(k, {V, S0}) and public S0 list are the reference's), GpuCCPotential_S2_MultiConfig
 * from ShiftedCCPotential_S2_MultiConfig (:1756-1870; constraints and S0 pushed onto its public lists), all also from
 * CombinedEnergyForce (potential/CombinedEnergyForce.h), so the structure optimiser's Objective
 * (potential/StructureOptimization.cpp:447-536) finds EnergyAndAllForce by dynamic_cast and makes one GPU evaluation
 * per step; MD/MC drivers call Energy / AllForce / Force as before.
 *
 * Contract kept from the reference:
 *   - constraints / Shift (and S0 for the S2 form) are the public members of the reference class; a change is seen at
 *     the next evaluation; the S2 form needs one S0 per constraint;
 *     every k must lie on the reciprocal lattice of the bound cell (std::invalid_argument otherwise);
 *   - SetConfiguration binds a Configuration the caller keeps alive (non-owning), invalidating cached results;
 *   - EnergyAndAllForce equals Energy() followed by AllForce() bitwise (both read one cached GPU evaluation);
 *   - GetRho fills RhoReal / RhoImag and sets RhoValid (not for the multi-configuration form, whose rho is per
 *     sub-configuration: std::invalid_argument);
 *   - one object is not evaluated from several threads at once.
 * Errors of the C ABI become std::invalid_argument (CC_ERR_ARG, CC_ERR_NONLATTICE), std::logic_error (CC_ERR_STATE)
 * or std::runtime_error (the rest).
 */
#ifndef GPU_CC_POTENTIAL_H
#define GPU_CC_POTENTIAL_H

#include "CollectiveCoordinatePotential.h"
#include "CombinedEnergyForce.h"
#include "cc_gpu.h"

#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

template <class Base> class GpuCCAdapter : public Base, public CombinedEnergyForce
{
	cc_handle *handle_ = nullptr;
	std::vector<double> kcopy_, vcopy_, s0copy_, basis_;   // the constraint set and cell the handle was built from
	double shift_copy_ = 0.0;
	int nsub_copy_ = 1;   // sub-configurations applied to the handle (NSubConfig of the multi-configuration form)
	std::vector<double> frac_, forces_;
	double energy_ = 0.0;
	bool positions_dirty_ = true, result_valid_ = false;
	int precision_ = CC_PREC_FP64;

	static void Check(int rc)
	{
		if (rc == CC_OK)
			return;
		const std::string msg = std::string("GpuCCPotential: ") + cc_last_error();
		if (rc == CC_ERR_ARG || rc == CC_ERR_NONLATTICE)
			throw std::invalid_argument(msg);
		if (rc == CC_ERR_STATE)
			throw std::logic_error(msg);
		throw std::runtime_error(msg);
	}

	const Configuration &Bound() const { return *this->pConfig; }

	// the targets of the S2 form; none for the plain form
	static const std::vector<double> *Targets(const ShiftedCCPotential &) { return nullptr; }
	static const std::vector<double> *Targets(const ShiftedCCPotential_S2 &p) { return &p.S0; }
	static const std::vector<double> *Targets(const ShiftedCCPotential_S2_MultiConfig &p) { return &p.S0; }
	static int SubConfigs(const ShiftedCCPotential &) { return 1; }
	static int SubConfigs(const ShiftedCCPotential_S2_MultiConfig &p) { return (int)p.NSubConfig; }

	// (Re)create the handle when the constraints, Shift or the cell changed; upload positions when dirty.
	void Sync()
	{
		if (this->pConfig == nullptr)
			throw std::logic_error("GpuCCPotential: no configuration bound");
		const Configuration &c = Bound();
		const int d = this->Dimension;
		std::vector<double> basis(d * d), k, V;
		for (int i = 0; i < d; i++)
			for (int j = 0; j < d; j++)
				basis[i * d + j] = c.GetBasisVector(i).x[j];
		k.reserve(this->constraints.size() * d);
		for (const auto &q : this->constraints) {
			for (int j = 0; j < d; j++)
				k.push_back(q.k.x[j]);
			V.push_back(q.V);
		}
		const std::vector<double> *S0 = Targets(*this);
		if (S0 && S0->size() != V.size())
			throw std::invalid_argument("GpuCCPotential: the S2 form needs one S0 per constraint");
		if (!handle_ || k != kcopy_ || V != vcopy_ || basis != basis_ || this->Shift != shift_copy_ ||
		    (S0 && *S0 != s0copy_)) {
			cc_destroy(handle_);
			handle_ = nullptr;
			if (S0)
				Check(cc_create_s2_cartesian(d, basis.data(), (int64_t)V.size(), k.data(), V.data(), S0->data(),
				                             this->Shift, &handle_));
			else
				Check(cc_create_cartesian(d, basis.data(), (int64_t)V.size(), k.data(), V.data(), this->Shift,
				                          &handle_));
			nsub_copy_ = 1;   // a new handle starts with one configuration; NSubConfig is applied below
			if (S0)
				s0copy_ = *S0;
			kcopy_.swap(k);
			vcopy_.swap(V);
			basis_.swap(basis);
			shift_copy_ = this->Shift;
			positions_dirty_ = true;
		}
		// NSubConfig is a public member of the reference class: a change takes effect at the next evaluation
		if (SubConfigs(*this) != nsub_copy_) {
			Check(cc_set_subconfigurations(handle_, SubConfigs(*this)));
			nsub_copy_ = SubConfigs(*this);
			result_valid_ = false;
		}
		if (positions_dirty_) {
			const size_t n = c.NumParticle();
			frac_.resize(n * d);
			for (size_t i = 0; i < n; i++)
				for (int j = 0; j < d; j++)
					frac_[i * d + j] = c.GetRelativeCoordinates(i).x[j];
			Check(cc_set_positions(handle_, (int64_t)n, frac_.data()));
			positions_dirty_ = false;
			result_valid_ = false;
		}
	}

	void Evaluate()
	{
		Sync();
		if (result_valid_)
			return;
		forces_.assign(frac_.size(), 0.0);
		Check(cc_energy_grad(handle_, &energy_, forces_.empty() ? nullptr : forces_.data(), precision_));
		result_valid_ = true;
	}

public:
	explicit GpuCCAdapter(DimensionType dimension) : Base(dimension) {}
	explicit GpuCCAdapter(const Base &src) : Base(src) {}
	GpuCCAdapter(DimensionType dimension, size_t nsub) : Base(dimension, nsub) {}   // the multi-configuration form
	GpuCCAdapter(const GpuCCAdapter &) = delete;
	GpuCCAdapter &operator=(const GpuCCAdapter &) = delete;
	virtual ~GpuCCAdapter() { cc_destroy(handle_); }

	/* CC_PREC_FP64 (default, the reference's arithmetic to rounding) or CC_PREC_MIXED (the S2 form evaluates in FP64
	 * either way). */
	void SetPrecision(int precision)
	{
		precision_ = precision;
		result_valid_ = false;
	}

	virtual void SetConfiguration(const Configuration &Position)
	{
		Base::SetConfiguration(Position);
		positions_dirty_ = true;
		result_valid_ = false;
	}

	virtual void GetRho(void)
	{
		Sync();
		const size_t M = this->constraints.size();
		this->RhoReal.resize(M);
		this->RhoImag.resize(M);
		Check(cc_rho(handle_, this->RhoReal.data(), this->RhoImag.data(), precision_));
		this->RhoValid = true;
	}

	virtual double Energy()
	{
		Evaluate();
		return energy_;
	}

	virtual void AllForce(std::vector<GeometryVector> &results)
	{
		Evaluate();
		const int d = this->Dimension;
		const size_t n = frac_.size() / d;
		results.assign(n, GeometryVector(d));
		for (size_t i = 0; i < n; i++)
			for (int j = 0; j < d; j++)
				results[i].x[j] = forces_[i * d + j];
	}

	virtual void Force(GeometryVector &result, size_t i)
	{
		Evaluate();
		const int d = this->Dimension;
		if (i >= frac_.size() / d)
			throw std::out_of_range("GpuCCPotential: Force: particle index out of range");
		result = GeometryVector(d);
		for (int j = 0; j < d; j++)
			result.x[j] = forces_[i * d + j];
	}

	virtual double EnergyAndAllForce(std::vector<GeometryVector> &forces)
	{
		AllForce(forces);
		return energy_;
	}
};

class GpuCCPotential : public GpuCCAdapter<ShiftedCCPotential>
{
public:
	explicit GpuCCPotential(DimensionType dimension) : GpuCCAdapter<ShiftedCCPotential>(dimension) {}
	explicit GpuCCPotential(const ShiftedCCPotential &src) : GpuCCAdapter<ShiftedCCPotential>(src) {}
};

class GpuCCPotential_S2 : public GpuCCAdapter<ShiftedCCPotential_S2>
{
public:
	explicit GpuCCPotential_S2(DimensionType dimension) : GpuCCAdapter<ShiftedCCPotential_S2>(dimension) {}
	explicit GpuCCPotential_S2(const ShiftedCCPotential_S2 &src) : GpuCCAdapter<ShiftedCCPotential_S2>(src) {}
};

class GpuCCPotential_S2_MultiConfig : public GpuCCAdapter<ShiftedCCPotential_S2_MultiConfig>
{
public:
	GpuCCPotential_S2_MultiConfig(DimensionType dimension, size_t nsub)
	    : GpuCCAdapter<ShiftedCCPotential_S2_MultiConfig>(dimension, nsub)
	{
	}
	explicit GpuCCPotential_S2_MultiConfig(const ShiftedCCPotential_S2_MultiConfig &src)
	    : GpuCCAdapter<ShiftedCCPotential_S2_MultiConfig>(src)
	{
	}
};

#endif
