// cc_plan.cpp — host-side planning (see cc_plan.h).
#include "cc_plan.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <numeric>

namespace cc {

namespace {

const double kTwoPi = 6.283185307179586476925286766559;

// Lexicographic order on (prefix..., last).
struct ModeLess {
	const int32_t *m;
	int d;
	bool operator()(int64_t a, int64_t b) const
	{
		for (int e = 0; e < d; e++)
			if (m[a * d + e] != m[b * d + e])
				return m[a * d + e] < m[b * d + e];
		return false;
	}
};

int64_t count_segments(int d, const std::vector<std::array<int32_t, 3> > &u, int L)
{
	int64_t nseg = 0;
	int len = 0;
	for (size_t i = 0; i < u.size(); i++) {
		bool cont = i > 0 && len < L && u[i][d - 1] == u[i - 1][d - 1] + 1;
		for (int e = 0; e + 1 < d && cont; e++)
			cont = u[i][e] == u[i - 1][e];
		if (cont) {
			len++;
		} else {
			nseg++;
			len = 1;
		}
	}
	return (nseg + 31) / 32 * 32;
}

}  // namespace

Plan build_plan(int d, int64_t M, const int32_t *modes, const double *V, int L)
{
	Plan p;
	p.d = d;
	std::vector<int64_t> idx((size_t)M);
	std::iota(idx.begin(), idx.end(), 0);
	std::stable_sort(idx.begin(), idx.end(), ModeLess{modes, d});
	// unique modes in sorted order, with summed weights
	std::vector<std::array<int32_t, 3> > u;
	std::vector<double> uV;
	std::vector<int64_t> mode_u((size_t)M);
	for (size_t i = 0; i < idx.size(); i++) {
		const int64_t m = idx[i];
		std::array<int32_t, 3> key = {0, 0, 0};
		for (int e = 0; e < d; e++)
			key[e] = modes[m * d + e];
		if (u.empty() || key != u.back()) {
			u.push_back(key);
			uV.push_back(0.0);
		}
		uV.back() += V[m];
		mode_u[m] = (int64_t)u.size() - 1;
	}
	p.unique_modes = (int64_t)u.size();
	if (L == 0) {
		// seed (~45 FP64 instructions) + L recurrence steps (~7) per segment and particle
		const int64_t n8 = count_segments(d, u, 8), n16 = count_segments(d, u, 16);
		L = (n8 * (45 + 7 * 8) <= n16 * (45 + 7 * 16)) ? 8 : 16;
	}
	p.L = L;
	std::vector<int64_t> u_slot(u.size());
	int len = 0;
	for (size_t i = 0; i < u.size(); i++) {
		bool cont = i > 0 && len < L && u[i][d - 1] == u[i - 1][d - 1] + 1;
		for (int e = 0; e + 1 < d && cont; e++)
			cont = u[i][e] == u[i - 1][e];
		if (cont) {
			len++;
			p.segs.back().len = len;
		} else {
			Seg s;
			s.p0 = d >= 2 ? u[i][0] : 0;
			s.p1 = d >= 3 ? u[i][1] : 0;
			s.start = u[i][d - 1];
			s.len = 1;
			p.segs.push_back(s);
			len = 1;
		}
		u_slot[i] = (int64_t)(p.segs.size() - 1) * L + (len - 1);
	}
	while (p.segs.size() % 32)
		p.segs.push_back(Seg{0, 0, 0, 0});
	p.ngroups = (int)(p.segs.size() / 32);
	p.nslot = p.ngroups * 32 * L;
	p.slotV.assign((size_t)p.nslot, 0.0);
	for (size_t i = 0; i < u.size(); i++)
		p.slotV[(size_t)u_slot[i]] = uV[i];
	p.mode_slot.resize((size_t)M);
	p.modeV.assign(V, V + M);
	for (int64_t m = 0; m < M; m++)
		p.mode_slot[(size_t)m] = (int)u_slot[(size_t)mode_u[(size_t)m]];
	return p;
}

bool cell_geometry(int d, const double *a, double *volume, double *recip)
{
	double inv[9] = {0};
	double det;
	if (d == 1) {
		det = a[0];
		if (det == 0)
			return false;
		inv[0] = 1.0 / det;
	} else if (d == 2) {
		det = a[0] * a[3] - a[1] * a[2];
		if (det == 0)
			return false;
		inv[0] = a[3] / det;
		inv[1] = -a[1] / det;
		inv[2] = -a[2] / det;
		inv[3] = a[0] / det;
	} else {
		const double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
		det = a[0] * c00 + a[1] * c01 + a[2] * c02;
		if (det == 0)
			return false;
		// inverse = adjugate / det
		inv[0] = c00 / det;
		inv[3] = c01 / det;
		inv[6] = c02 / det;
		inv[1] = (a[2] * a[7] - a[1] * a[8]) / det;
		inv[4] = (a[0] * a[8] - a[2] * a[6]) / det;
		inv[7] = (a[1] * a[6] - a[0] * a[7]) / det;
		inv[2] = (a[1] * a[5] - a[2] * a[4]) / det;
		inv[5] = (a[2] * a[3] - a[0] * a[5]) / det;
		inv[8] = (a[0] * a[4] - a[1] * a[3]) / det;
	}
	if (!std::isfinite(det))
		return false;
	*volume = std::fabs(det);
	// b_e = 2 pi (row e of inv^T) = 2 pi (column e of inv)
	for (int e = 0; e < d; e++)
		for (int c = 0; c < d; c++)
			recip[e * d + c] = kTwoPi * inv[c * d + e];
	return true;
}

bool cartesian_to_modes(int d, const double *basis, int64_t M, const double *k, int32_t *modes)
{
	for (int64_t m = 0; m < M; m++)
		for (int e = 0; e < d; e++) {
			double x = 0;
			for (int c = 0; c < d; c++)
				x += k[m * d + c] * basis[e * d + c];
			x /= kTwoPi;
			const double r = std::nearbyint(x);
			if (!std::isfinite(x) || std::fabs(x - r) > 1e-9 * std::max(1.0, std::fabs(x)) || std::fabs(r) > 1e9)
				return false;
			modes[m * d + e] = (int32_t)r;
		}
	return true;
}

bool stealthy_kset(int d, const double *basis, int64_t N, double chi, int type, std::vector<int32_t> &modes,
                   std::vector<double> &V)
{
	double vol, recip[9];
	if (!cell_geometry(d, basis, &vol, recip))
		return false;
	const double want_d = std::ceil(chi * (double)N * d);
	if (!(want_d < 5e7))
		return false;
	const size_t want = (size_t)want_d;
	// the CLI's radius: half the diagonal of a cube of 2 d want reciprocal cells
	const double maxk = (std::sqrt((double)d) / 2) * std::pow(2 * (double)d * (double)want, 1.0 / d) *
	                    (kTwoPi / std::pow(vol, 1.0 / d));
	int64_t bound[3] = {0, 0, 0};
	double box = 1;
	for (int e = 0; e < d; e++) {
		double alen = 0;
		for (int c = 0; c < d; c++)
			alen += basis[e * d + c] * basis[e * d + c];
		bound[e] = (int64_t)std::floor(maxk * std::sqrt(alen) / kTwoPi) + 1;
		box *= 2.0 * bound[e] + 1;
	}
	if (box > 4e8)
		return false;
	struct Cand {
		double k2;
		int32_t n[3];
	};
	std::vector<Cand> c;
	int64_t n[3] = {0, 0, 0};
	const int64_t lo0 = 0;   // half space: the first index is >= 0
	for (n[0] = lo0; n[0] <= bound[0]; n[0]++)
		for (n[1] = (d >= 2 ? -bound[1] : 0); n[1] <= (d >= 2 ? bound[1] : 0); n[1]++)
			for (n[2] = (d >= 3 ? -bound[2] : 0); n[2] <= (d >= 3 ? bound[2] : 0); n[2]++) {
				int sign = 0;
				for (int e = 0; e < d && sign == 0; e++)
					sign = n[e] > 0 ? 1 : (n[e] < 0 ? -1 : 0);
				if (sign <= 0)
					continue;
				double k[3] = {0, 0, 0};
				for (int e = 0; e < d; e++)
					for (int cc = 0; cc < d; cc++)
						k[cc] += (double)n[e] * recip[e * d + cc];
				double k2 = 0;
				for (int cc = 0; cc < d; cc++)
					k2 += k[cc] * k[cc];
				if (!(k2 < maxk * maxk))   // the enumeration radius is exclusive
					continue;
				Cand x;
				x.k2 = k2;
				for (int e = 0; e < 3; e++)
					x.n[e] = (int32_t)n[e];
				c.push_back(x);
			}
	std::sort(c.begin(), c.end(), [](const Cand &a, const Cand &b) {
		if (a.k2 != b.k2)
			return a.k2 < b.k2;
		for (int e = 0; e < 3; e++)
			if (a.n[e] != b.n[e])
				return a.n[e] < b.n[e];
		return false;
	});
	size_t count = 0;
	double last = 0;
	while (count < c.size()) {
		if (!(count < want || std::fabs((last - c[count].k2) / last) < 1e-10))
			break;
		last = c[count].k2;
		count++;
	}
	const double K2 = count < c.size() ? c[count].k2 : 0.0;
	modes.resize(count * d);
	V.resize(count);
	for (size_t m = 0; m < count; m++) {
		for (int e = 0; e < d; e++)
			modes[m * d + e] = c[m].n[e];
		double w = 1.0;
		if (type >= 1 && type <= 3 && K2 > 0) {
			const double x = std::sqrt(c[m].k2 / K2);
			if (type == 1)
				w = std::acos(x) - x * std::sqrt(1 - c[m].k2 / K2);
			else if (type == 2)
				w = std::pow(1.0 - x, 6.0);
			else
				w = std::pow(1.0 - x, 2.0);
		}
		V[m] = w;
	}
	return true;
}

}  // namespace cc
