// cc_plan.cpp — host-side planning (see cc_plan.h).
#include "cc_plan.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <numeric>
#include <random>
#include <set>

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

// Index ranges of a set of segments, per axis (prefix axes: p0, p1; last axis: segment starts).
struct Ranges {
	int lo[3], hi[3];
	bool empty = true;
	void add(int d, const Seg &s)
	{
		int v[3] = {s.p0, s.p1, 0};
		v[d - 1] = s.start;
		for (int e = 0; e < d; e++) {
			if (empty || v[e] < lo[e])
				lo[e] = v[e];
			if (empty || v[e] > hi[e])
				hi[e] = v[e];
		}
		empty = false;
	}
};

TabSpec make_spec(int d, const Ranges &r)
{
	TabSpec t = {};
	int off = 0;
	for (int e = 0; e < d; e++) {
		const int range = r.hi[e] - r.lo[e] + 1;
		t.lo[e] = r.lo[e];
		if (e < d - 1 && range <= kFullMax) {
			t.full[e] = 1;
			t.offc[e] = off;
			t.run[t.nrun++] = TabRun{e, 1, r.lo[e], range, off};
			off += range;
		} else {
			const int nc = (range + 7) / 8;
			t.full[e] = 0;
			t.offc[e] = off;
			t.run[t.nrun++] = TabRun{e, 8, r.lo[e], nc, off};
			off += nc;
			t.offf[e] = off;
			t.run[t.nrun++] = TabRun{e, 1, 0, 8, off};
			off += 8;
		}
	}
	t.row = off;
	t.items = 0;
	for (int i = 0; i < t.nrun; i++)
		t.items += (t.run[i].count + 7) / 8;
	return t;
}

int spec_row(int d, const Ranges &r) { return make_spec(d, r).row; }

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
	if (L <= 0)
		L = 8;
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
	// rho groups: up to 32 consecutive segments whose tables fit kMaxRow entries, padded to 32
	std::vector<Seg> raw;
	raw.swap(p.segs);
	p.real_segs = (int64_t)raw.size();
	std::vector<int64_t> where(raw.size());
	size_t i0 = 0;
	while (i0 < raw.size()) {
		Ranges r;
		size_t j = i0;
		while (j < raw.size() && (int)(j - i0) < kGroupSegs) {
			Ranges t = r;
			t.add(d, raw[j]);
			if (j > i0 && spec_row(d, t) > kMaxRow)
				break;
			r = t;
			j++;
		}
		for (size_t k = i0; k < j; k++) {
			where[k] = (int64_t)p.segs.size();
			p.segs.push_back(raw[k]);
		}
		while (p.segs.size() % kGroupSegs)
			p.segs.push_back(Seg{0, 0, 0, 0});
		p.rspec.push_back(make_spec(d, r));
		p.rho_max_row = std::max(p.rho_max_row, p.rspec.back().row);
		i0 = j;
	}
	// slot of (segment q, step r) = r * nseg + q: a warp's 32 segments are contiguous for every r
	const int64_t nseg = (int64_t)p.segs.size();
	for (size_t i = 0; i < u.size(); i++) {
		const int64_t seg = u_slot[i] / L, r = u_slot[i] % L;
		u_slot[i] = r * nseg + where[(size_t)seg];
	}
	// block groups: up to kBlockGroups consecutive rho groups whose joint tables fit kMaxRow entries
	{
		const int ng = p.ngroups();
		int g = 0;
		while (g < ng) {
			Ranges r;
			int h = g;
			while (h < ng && h - g < kBlockGroups) {
				Ranges t = r;
				for (int q = h * kGroupSegs; q < (h + 1) * kGroupSegs; q++)
					if (p.segs[q].len > 0)
						t.add(d, p.segs[q]);
				if (h > g && spec_row(d, t) > kMaxRow)
					break;
				r = t;
				h++;
			}
			p.bstart.push_back(g);
			p.bspec.push_back(make_spec(d, r));
			p.block_max_row = std::max(p.block_max_row, p.bspec.back().row);
			g = h;
		}
		p.bstart.push_back(ng);
	}
	p.nslot = (int)p.segs.size() * L;
	p.slotV.assign((size_t)p.nslot, 0.0);
	for (size_t i = 0; i < u.size(); i++)
		p.slotV[(size_t)u_slot[i]] = uV[i];
	p.mode_slot.resize((size_t)M);
	p.modeV.assign(V, V + M);
	for (int64_t m = 0; m < M; m++)
		p.mode_slot[(size_t)m] = (int)u_slot[(size_t)mode_u[(size_t)m]];
	return p;
}

ForceSplits force_splits(const Plan &p, int want)
{
	ForceSplits f;
	const int nseg = (int)p.segs.size();
	want = std::max(1, std::min(want, std::max(1, (int)p.real_segs)));
	const int64_t target = (p.real_segs + want - 1) / want;   // real segments per split
	int i = 0;
	while (i < nseg) {
		Ranges r;
		int j = i, real = 0;
		while (j < nseg) {
			if (p.segs[j].len == 0) {   // padding: no table entries
				j++;
				continue;
			}
			if (real >= target)
				break;
			Ranges t = r;
			t.add(p.d, p.segs[j]);
			if (real > 0 && spec_row(p.d, t) > kMaxRow)
				break;
			r = t;
			real++;
			j++;
		}
		if (real == 0)   // trailing padding only: attach to the previous split
		{
			if (!f.start.empty()) {
				i = nseg;
				break;
			}
			Seg z = {0, 0, 0, 1};
			r.add(p.d, z);
		}
		f.start.push_back(i);
		f.spec.push_back(make_spec(p.d, r));
		f.max_row = std::max(f.max_row, f.spec.back().row);
		i = j;
	}
	f.start.push_back(nseg);
	return f;
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

namespace {

int64_t gcd64(int64_t a, int64_t b)
{
	a = a < 0 ? -a : a;
	b = b < 0 ? -b : b;
	while (b) {
		const int64_t t = a % b;
		a = b;
		b = t;
	}
	return a;
}

// Cartesian k = sum_e n_e b_e, accumulated axis by axis from zero (as GeometryVector sums), and k.k.
void lattice_k(int d, const double *recip, const int64_t *n, double *k)
{
	for (int x = 0; x < d; x++)
		k[x] = 0.0;
	for (int e = 0; e < d; e++)
		for (int x = 0; x < d; x++)
			k[x] = k[x] + (double)n[e] * recip[e * d + x];
}

double mod2(int d, const double *k)
{
	double s = 0.0;
	for (int x = 0; x < d; x++)
		s += k[x] * k[x];
	return s;
}

double dot(int d, const double *u, const double *v)
{
	double s = 0.0;
	for (int x = 0; x < d; x++)
		s += u[x] * v[x];
	return s;
}

// Reciprocal basis formed as the reference's cell forms it (core/PeriodicCellList.h:999-1030): b_i = a_i minus its
// projections on the Gram-Schmidt orthogonalised other basis vectors, scaled by 2 pi / (b_i . a_i). Same algebra as
// cell_geometry's inverse, but the same rounding as the reference, so lattice vectors of equal length compare equal
// (and order) exactly as there.
void reciprocal_by_projection_impl(int d, const double *a, double *recip)
{
	for (int i = 0; i < d; i++) {
		double r[3], ortho[2][3];
		int no = 0;
		for (int x = 0; x < d; x++)
			r[x] = a[i * d + x];
		for (int j = 0; j < d; j++) {
			if (j == i)
				continue;
			double t[3];
			for (int x = 0; x < d; x++)
				t[x] = a[j * d + x];
			for (int o = 0; o < no; o++) {
				const double c = dot(d, t, ortho[o]) / mod2(d, ortho[o]);
				for (int x = 0; x < d; x++)
					t[x] -= ortho[o][x] * c;
			}
			for (int x = 0; x < d; x++)
				ortho[no][x] = t[x];
			no++;
		}
		for (int o = 0; o < no; o++) {
			const double c = dot(d, ortho[o], r) / mod2(d, ortho[o]);
			for (int x = 0; x < d; x++)
				r[x] -= ortho[o][x] * c;
		}
		const double sc = 2.0 * M_PI / dot(d, r, a + i * d);
		for (int x = 0; x < d; x++)
			recip[i * d + x] = r[x] * sc;
	}
}

}  // namespace

void reciprocal_by_projection(int d, const double *basis, double *recip)
{
	reciprocal_by_projection_impl(d, basis, recip);
}

bool isotropic_ks(int d, const double *basis, double circ_kmax, double lin_kmax, double sample_prob, double circ_kmin,
                  std::vector<int32_t> &modes, std::vector<double> &kamp, size_t max_ks)
{
	modes.clear();
	kamp.clear();
	double vol = 0.0, recip[9];
	if (d < 1 || d > 3 || !cell_geometry(d, basis, &vol, recip))
		return false;
	if (!(circ_kmax > 0.0) || !(lin_kmax > 0.0))
		return true;
	reciprocal_by_projection_impl(d, basis, recip);
	std::mt19937 rng(98765u);
	auto keep = [&]() { return sample_prob >= 1.0 || (double)rng() / 4294967296.0 < sample_prob; };
	auto push = [&](int64_t n0, int64_t n1, int64_t n2, double amp) {
		const int64_t n[3] = {n0, n1, n2};
		for (int e = 0; e < d; e++) {
			if (n[e] > INT32_MAX || n[e] < INT32_MIN)
				return false;
			modes.push_back((int32_t)n[e]);
		}
		kamp.push_back(amp);
		return kamp.size() <= max_ks;
	};
	if (d == 1) {
		const double b = recip[0];
		if (!(b > 0.0))
			return false;
		if (circ_kmin <= 0.0) {
			for (int64_t i = 1;; i++) {
				const double kx = (double)i * b;
				if (kx > lin_kmax)
					break;
				if (keep() && !push(i, 0, 0, std::sqrt(kx * kx)))
					return false;
			}
			return true;
		}
		std::vector<int64_t> seed;
		std::vector<double> seedk;
		for (int64_t i = 1;; i++) {
			const double kx = (double)i * b;
			if (kx > circ_kmax)
				break;
			if (kx > circ_kmin && keep()) {
				if (!push(i, 0, 0, std::sqrt(kx * kx)))
					return false;
				seed.push_back(i);
				seedk.push_back(kx);
			}
		}
		if (seed.empty())
			return true;
		for (int64_t i = 2;; i++) {
			for (size_t j = 0; j < seed.size(); j++) {
				const double kx = (double)i * seedk[j];
				if (kx > lin_kmax)
					return true;
				if (keep() && !push(i * seed[j], 0, 0, std::sqrt(kx * kx)))
					return false;
			}
		}
	}
	// d >= 2: half-space points of the circle, by (|k|^2, k_x)
	int64_t lim[3] = {0, 0, 0};
	for (int e = 0; e < d; e++) {
		double a2 = 0.0;
		for (int x = 0; x < d; x++)
			a2 += basis[e * d + x] * basis[e * d + x];
		lim[e] = (int64_t)std::ceil(circ_kmax * std::sqrt(a2) / (2.0 * M_PI));
		if (lim[e] > 100000)
			return false;
	}
	struct P {
		int64_t n[3];
		double k2, kx;
	};
	std::vector<P> circle;
	const double K2 = circ_kmax * circ_kmax, Kmin2 = circ_kmin * circ_kmin;
	// the reference's odometer order (axis 0 fastest): std::sort below then orders ties as the reference's does
	int64_t n[3] = {0, 0, 0};
	for (n[2] = (d == 3 ? -lim[2] : 0); n[2] <= (d == 3 ? lim[2] : 0); n[2]++)
		for (n[1] = -lim[1]; n[1] <= lim[1]; n[1]++)
			for (n[0] = -lim[0]; n[0] <= lim[0]; n[0]++) {
				int first = 0;
				for (int e = 0; e < d && first == 0; e++)
					first = n[e] > 0 ? 1 : n[e] < 0 ? -1 : 0;
				if (first < 0)
					continue;   // the inverted half (k = 0 fails the k^2 > kmin^2 test below)
				double k[3];
				lattice_k(d, recip, n, k);
				const double k2 = mod2(d, k);
				if (k2 < K2 && k2 > Kmin2) {
					circle.push_back({{n[0], n[1], n[2]}, k2, k[0]});
					if (circle.size() > max_ks)
						return false;
				}
			}
	std::sort(circle.begin(), circle.end(), [](const P &a, const P &b) {
		if (a.k2 != b.k2)
			return a.k2 < b.k2;
		return a.kx < b.kx;
	});
	if (lin_kmax == circ_kmax) {
		for (const P &q : circle)
			if (!push(q.n[0], q.n[1], q.n[2], std::sqrt(q.k2)))
				return false;
		return true;
	}
	// the first point of each lattice direction (directions compared as primitive integer vectors)
	std::set<std::array<int64_t, 3> > seen;
	std::vector<P> first;
	for (const P &q : circle) {
		int64_t g = 0;
		for (int e = 0; e < d; e++)
			g = gcd64(g, q.n[e]);
		std::array<int64_t, 3> key = {q.n[0] / g, q.n[1] / g, d == 3 ? q.n[2] / g : 0};
		if (!seen.insert(key).second)
			continue;
		first.push_back(q);
	}
	const double L2 = lin_kmax * lin_kmax;
	for (const P &q : first) {
		double k[3];
		lattice_k(d, recip, q.n, k);
		for (int64_t i = 1;; i++) {
			double t[3];
			for (int x = 0; x < d; x++)
				t[x] = (double)i * k[x];
			const double t2 = mod2(d, t);
			if (t2 > L2)
				break;
			if (keep() && !push(i * q.n[0], i * q.n[1], i * q.n[2], std::sqrt(t2)))
				return false;
		}
	}
	return true;
}

}  // namespace cc
