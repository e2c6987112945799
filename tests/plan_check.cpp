// CPU check of the host planner's index arithmetic (modules_b200/csrc/cc_plan.cpp): reads k-sets from stdin as
//   d M   then M lines of d integers and a weight,
// builds the plan and verifies every index the kernels derive from it: slot <-> mode, segment lengths, rho groups
// (32 segments, padded) and force splits, each segment's seed-table entries and the recurrence step inside its
// group's/unit's table row (<= kMaxRow), and the table-building runs. Prints one line per k-set; exit 1 on a failure.
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cmath>
#include <vector>

#include "../modules_b200/csrc/cc_plan.h"

using namespace cc;

static int fails = 0;
#define CHECK(c)                                                                                       \
	do {                                                                                               \
		if (!(c)) {                                                                                    \
			if (fails++ < 20)                                                                          \
				std::printf("FAIL line %d: %s\n", __LINE__, #c);                                       \
		}                                                                                              \
	} while (0)

static void check_spec(int d, const TabSpec &t, const std::vector<Seg> &segs, int q0, int q1)
{
	CHECK(t.row > 0 && t.row <= kMaxRow);
	int items = 0, covered = 0;
	for (int r = 0; r < t.nrun; r++) {
		CHECK(t.run[r].off >= 0 && t.run[r].off + t.run[r].count <= t.row);
		CHECK(t.run[r].axis >= 0 && t.run[r].axis < d);
		items += (t.run[r].count + 7) / 8;
		covered += t.run[r].count;
	}
	CHECK(items == t.items && covered == t.row);
	CHECK(t.full[d - 1] == 0);
	CHECK(t.offf[d - 1] + 1 < t.row);
	for (int q = q0; q < q1; q++) {
		int v[3] = {segs[q].p0, segs[q].p1, 0};
		v[d - 1] = segs[q].start;
		for (int e = 0; e < d; e++) {
			const int m = v[e] - t.lo[e];
			CHECK(m >= 0);
			if (t.full[e]) {
				CHECK(t.offc[e] + m < t.row);
				bool in = false;   // the entry must be one the runs fill with index m0 + k = v[e]
				for (int r = 0; r < t.nrun; r++)
					if (t.run[r].axis == e && t.run[r].stride == 1 && t.run[r].off == t.offc[e])
						in = m < t.run[r].count && t.run[r].m0 + m == v[e];
				CHECK(in);
			} else {
				CHECK(t.offc[e] + (m >> 3) < t.offf[e]);
				CHECK(t.offf[e] + 7 < t.row);
				bool in = false;
				for (int r = 0; r < t.nrun; r++)
					if (t.run[r].axis == e && t.run[r].stride == 8 && t.run[r].off == t.offc[e])
						in = (m >> 3) < t.run[r].count && t.run[r].m0 + 8 * (m >> 3) + (m & 7) == v[e];
				CHECK(in);
			}
		}
	}
}

int main()
{
	int d;
	long M;
	while (std::scanf("%d %ld", &d, &M) == 2) {
		std::vector<int32_t> modes(M * d);
		std::vector<double> V(M);
		for (long m = 0; m < M; m++) {
			for (int e = 0; e < d; e++)
				if (std::scanf("%d", &modes[m * d + e]) != 1)
					return 2;
			if (std::scanf("%lf", &V[m]) != 1)
				return 2;
		}
		Plan p = build_plan(d, M, modes.data(), V.data(), 8);
		const int L = p.L;
		CHECK(p.nslot == (int)p.segs.size() * L);
		for (long m = 0; m < M; m++) {
			const int slot = p.mode_slot[m];
			CHECK(slot >= 0 && slot < p.nslot);
			const Seg &s = p.segs[slot % p.segs.size()];
			const int r = slot / (int)p.segs.size();
			CHECK(r < s.len);
			int v[3] = {s.p0, s.p1, 0};
			v[d - 1] = s.start + r;
			for (int e = 0; e < d; e++)
				CHECK(v[e] == modes[m * d + e]);
		}
		double sumV = 0, sumS = 0;
		for (long m = 0; m < M; m++)
			sumV += V[m];
		for (int q = 0; q < p.nslot; q++)
			sumS += p.slotV[q];
		CHECK(std::abs(sumV - sumS) <= 1e-9 * (1 + std::abs(sumV)));
		for (size_t q = 0; q < p.segs.size(); q++)
			CHECK(p.segs[q].len >= 0 && p.segs[q].len <= L);
		CHECK(p.segs.size() == (size_t)p.ngroups() * kGroupSegs);
		for (int g = 0; g < p.ngroups(); g++) {
			int q1 = g * kGroupSegs;
			while (q1 < (g + 1) * kGroupSegs && p.segs[q1].len > 0)
				q1++;
			for (int q = q1; q < (g + 1) * kGroupSegs; q++)
				CHECK(p.segs[q].len == 0);   // padding only at the end of a group
			CHECK(q1 > g * kGroupSegs);
			check_spec(d, p.rspec[g], p.segs, g * kGroupSegs, q1);
		}
		CHECK(p.bstart.size() == p.bspec.size() + 1 && p.bstart.front() == 0 && p.bstart.back() == p.ngroups());
		for (int b = 0; b < p.nbgroups(); b++) {
			CHECK(p.bstart[b + 1] > p.bstart[b] && p.bstart[b + 1] - p.bstart[b] <= kBlockGroups);
			std::vector<Seg> real;
			for (int q = p.bstart[b] * kGroupSegs; q < p.bstart[b + 1] * kGroupSegs; q++)
				if (p.segs[q].len > 0)
					real.push_back(p.segs[q]);
			check_spec(d, p.bspec[b], real, 0, (int)real.size());
		}
		int max_force_row = 0;
		for (int want : {1, 3, 8, 64, 1000}) {
			ForceSplits f = force_splits(p, want);
			CHECK(f.start.size() == f.spec.size() + 1 && f.start.front() == 0 && f.start.back() == (int)p.segs.size());
			for (int k = 0; k < f.count(); k++) {
				CHECK(f.start[k + 1] > f.start[k]);
				std::vector<Seg> real;
				for (int q = f.start[k]; q < f.start[k + 1]; q++)
					if (p.segs[q].len > 0)
						real.push_back(p.segs[q]);
				check_spec(d, f.spec[k], real, 0, (int)real.size());
			}
			max_force_row = std::max(max_force_row, f.max_row);
		}
		std::printf("d=%d M=%ld unique=%ld segs=%ld padded=%zu fill=%.3f groups=%d bgroups=%d rho_row=%d force_row=%d\n",
		            d, M, (long)p.unique_modes, (long)p.real_segs, p.segs.size(),
		            p.segs.empty() ? 1.0 : (double)p.unique_modes / p.nslot, p.ngroups(), p.nbgroups(), p.block_max_row,
		            max_force_row);
	}
	if (fails)
		std::printf("%d failures\n", fails);
	return fails ? 1 : 0;
}
