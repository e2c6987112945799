// cc_plan.h — host-side planning of the CC kernels: lattice-line segments, cell geometry, the stealthy k-set.
#pragma once
#include <cstdint>
#include <vector>

namespace cc {

// A piece of a lattice line of modes (see cc_kernels.cuh): modes (p0, p1, start + r) for r < len, d = 3;
// (p0, start + r) for d = 2; (start + r) for d = 1.
struct alignas(16) Seg {
	int p0, p1;
	int start;
	int len;
};

struct Plan {
	int d = 0;
	int L = 16;                   // slots per segment (8 or 16)
	int ngroups = 0;              // segments / 32
	int nslot = 0;                // ngroups * 32 * L
	std::vector<Seg> segs;        // ngroups * 32, padding segments have len 0
	std::vector<double> slotV;    // nslot: summed weight of the modes of each slot
	std::vector<int> mode_slot;   // M: slot of each input mode
	std::vector<double> modeV;    // M: input weights
	int64_t unique_modes = 0;
};

// Group M modes (M x d integers) into segments of at most L slots; L = 0 chooses 8 or 16 by a work estimate.
Plan build_plan(int d, int64_t M, const int32_t *modes, const double *V, int L);

// |det| of the basis (rows a_i) and the reciprocal basis rows b_e with b_e . a_i = 2 pi delta_ei.
bool cell_geometry(int d, const double *basis, double *volume, double *recip);

// n_e = k . a_e / (2 pi); false if some n_e is not within 1e-9 max(1, |n_e|) of an integer.
bool cartesian_to_modes(int d, const double *basis, int64_t M, const double *k, int32_t *modes);

// The CLI's stealthy k-set, GeneratePotential Type 0..3 (apps/CollectiveCoordinateCLI/CollectiveCoordinateCLI.cpp:
// 180-265): half-space reciprocal vectors within the CLI's enumeration radius, ordered by |k|^2 (ties by index), the
// first ceil(chi N d) plus the rest of the last shell, and the Type 1-3 weights.
bool stealthy_kset(int d, const double *basis, int64_t N, double chi, int type, std::vector<int32_t> &modes,
                   std::vector<double> &V);

}  // namespace cc
