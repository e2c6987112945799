// cc_plan.h — host-side planning of the CC kernels: lattice-line segments, phase-table specs, cell geometry and the
// stealthy k-set.
#pragma once
#include <cstdint>
#include <vector>

namespace cc {

// A piece of a lattice line of modes (see cc_kernels.cuh): modes (p0, p1, start + r) for r < len when d = 3;
// (p0, start + r) when d = 2; (start + r) when d = 1.
struct alignas(16) Seg {
	int p0, p1;
	int start;
	int len;
};

// One run of a per-particle phase table: entries off .. off+count-1 of a particle's row hold
// exp(2 pi i (m0 + stride k) s_axis), k = 0 .. count-1.
struct TabRun {
	int axis, stride, m0, count, off;
};

// The phase tables a group of segments needs, per particle. Axis e is looked up either in a FULL table (full[e] = 1:
// T(m) = row[offc[e] + m - lo[e]]) or as COARSE x FINE (full[e] = 0: T(m) = row[offc[e] + (m-lo[e])/8] *
// row[offf[e] + (m-lo[e])%8]). The last axis is always coarse x fine; its fine entry 1 is the recurrence step.
struct TabSpec {
	TabRun run[6];
	int nrun;
	int row;        // entries per particle
	int items;      // sum over runs of ceil(count / 8): table-building work items per particle
	int lo[3], full[3], offc[3], offf[3];
};

struct Plan {
	int d = 0;
	int L = 8;                        // slots per segment
	std::vector<Seg> segs;            // ngroups * 32: rho groups of 32 segments, padded with len = 0 segments
	int nslot = 0;                    // segs.size() * L; slot of (segment q, step r) = r * segs.size() + q
	std::vector<double> slotV;        // nslot: summed weight of the modes of each slot (0 for empty slots)
	std::vector<int> mode_slot;       // M: slot of each input mode
	std::vector<double> modeV;        // M: input weights
	int64_t unique_modes = 0;
	int64_t real_segs = 0;            // segments with len > 0
	std::vector<TabSpec> rspec;       // one table spec per rho group
	int rho_max_row = 0;
	int ngroups() const { return (int)rspec.size(); }
	// block groups of the split rho kernel: warp groups [bstart[b], bstart[b+1]) (at most kBlockGroups) that share
	// one table spec
	std::vector<int> bstart;
	std::vector<TabSpec> bspec;
	int block_max_row = 0;
	int nbgroups() const { return (int)bspec.size(); }
};

// A split of the segments for the force pass: segments [start[k], start[k+1]) share the table spec spec[k].
struct ForceSplits {
	std::vector<int> start;
	std::vector<TabSpec> spec;
	int max_row = 0;
	int count() const { return (int)spec.size(); }
};

constexpr int kGroupSegs = 32;     // segments per rho group (one per lane)
constexpr int kBlockGroups = 8;    // rho groups (warps) per block of the split rho kernel
constexpr int kMaxRow = 128;       // table entries per particle and group/split
constexpr int kFullMax = 48;       // prefix axes with a range up to this many indices get a full table

// Group M modes (M x d integers) into segments of L slots, in rho groups of 32 segments.
Plan build_plan(int d, int64_t M, const int32_t *modes, const double *V, int L);

// Cut the plan's segments into at least `want` force splits of similar size whose tables fit kMaxRow entries.
ForceSplits force_splits(const Plan &p, int want);

// |det| of the basis (rows a_i) and the reciprocal basis rows b_e with b_e . a_i = 2 pi delta_ei.
bool cell_geometry(int d, const double *basis, double *volume, double *recip);

// n_e = k . a_e / (2 pi); false if some n_e is not within 1e-9 max(1, |n_e|) of an integer.
bool cartesian_to_modes(int d, const double *basis, int64_t M, const double *k, int32_t *modes);

// The CLI's stealthy k-set, GeneratePotential Type 0..3 (apps/CollectiveCoordinateCLI/CollectiveCoordinateCLI.cpp:
// 180-265): half-space reciprocal vectors within the CLI's enumeration radius, ordered by |k|^2 (ties by index), the
// first ceil(chi N d) plus the rest of the last shell, and the Type 1-3 weights.
bool stealthy_kset(int d, const double *basis, int64_t N, double chi, int type, std::vector<int32_t> &modes,
                   std::vector<double> &V);

// The wavevectors of GetKs (core/PeriodicCellList.cpp:509-735) as integer modes, with |k| formed the way the
// reference forms it (k = sum_e n_e b_e summed in axis order, |k| = sqrt(k.k)):
//   d >= 2: the half-space lattice points with circ_kmin^2 < |k|^2 < circ_kmax^2, ordered by (|k|^2, k_x); when
//           lin_kmax differs from circ_kmax, instead every multiple i k (i >= 1, |i k| <= lin_kmax) of the first of
//           those points in each lattice direction;
//   d == 1: the multiples i b (b the reciprocal vector) up to lin_kmax, or, with circ_kmin > 0, the seeds in
//           (circ_kmin, circ_kmax] followed by their multiples, round by round, until one exceeds lin_kmax.
// With sample_prob < 1 each candidate of the multiples is kept when a Mersenne Twister seeded with 98765 draws below
// sample_prob (the reference's RandomGenerator: draw / 2^32). false for a degenerate cell, a 1D cell of non-positive
// length, or more than max_ks wavevectors.
// The reciprocal basis rows formed as the reference's cell forms them (core/PeriodicCellList.h:999-1030: projection
// on the Gram-Schmidt orthogonalised other basis vectors, scaled by 2 pi / (b_i . a_i)); same rounding as there.
void reciprocal_by_projection(int d, const double *basis, double *recip);

bool isotropic_ks(int d, const double *basis, double circ_kmax, double lin_kmax, double sample_prob, double circ_kmin,
                  std::vector<int32_t> &modes, std::vector<double> &kamp, size_t max_ks = 50000000);

}  // namespace cc
