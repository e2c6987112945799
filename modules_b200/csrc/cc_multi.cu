// cc_multi.cu — the multi-species stealthy potential with soft-core contact repulsion on one GPU
// (MultiStealthyPotential, apps/CCOptimization/MultiStealthyPotential.h:115-481 and .cpp:139-985):
//
//   E   = u0 sum_s (N_s / N) Phi_s  +  e0 sum_{i<j} sum_{images} [r < sigma_ij] (1 - r / sigma_ij)^2,
//   F_i = u0 (N_s / N) F_i^{CC,s}   +  e0 sum_{j != i} sum_{images} (2 / sigma)(1 / r - 1 / sigma)(r_i - r_j),
//
// with Phi_s the collective-coordinate energy of species s over its own particles and constraint set (a cc_handle
// per species, evaluated by the rho / reduce / force kernels), sigma_ij = R_i + R_j, and the reference's rule for two
// coincident particles (r < 1e-15: a unit push along the first axis, away from the higher index).
//
// The contact sum runs on the GPU, one thread per particle, over a cell grid in fractional coordinates built on the
// host: n_e = max(1, floor(h_e / rc)) cells along axis e (h_e the spacing of the lattice planes of that axis) and a
// reach of ceil(n_e rc / h_e) cells on each side, so every periodic image of every neighbour within rc is visited
// exactly once, also in cells smaller than 2 rc where a neighbour (or the particle itself) has several images.
#include "../../include/cc_gpu.h"
#include "cc_error.h"
#include "cc_plan.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace {

struct ContactArgs {
	const double *frac;      // N x D fractional, in [0,1)
	const double *radii;     // N
	const int *cell;         // N x D cell coordinates
	const int *cell_start;   // ncell + 1
	const int *items;        // N particle indices sorted by cell (increasing within a cell)
	int N;
	int n[3], reach[3];
	double basis[9];         // rows a_e (Cartesian)
	double e0;
	double *E_out;           // N: contact energy of the pairs (i, j > i), before e0
	double *F_out;           // N x D: e0 times the contact force
};

__device__ __forceinline__ int floor_div(int q, int n) { return q >= 0 ? q / n : -((-q + n - 1) / n); }

template <int D> __global__ void __launch_bounds__(128) cc_contact_kernel(ContactArgs a)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= a.N)
		return;
	double si[D];
	int ci[D];
#pragma unroll
	for (int e = 0; e < D; e++) {
		si[e] = a.frac[(size_t)i * D + e];
		ci[e] = a.cell[(size_t)i * D + e];
	}
	const double Ri = a.radii[i];
	double E = 0.0, f[D];
#pragma unroll
	for (int x = 0; x < D; x++)
		f[x] = 0.0;
	int span[3] = {1, 1, 1}, noff = 1;
#pragma unroll
	for (int e = 0; e < D; e++) {
		span[e] = 2 * a.reach[e] + 1;
		noff *= span[e];
	}
	for (int t = 0; t < noff; t++) {
		int rem = t, lin = 0, stride = 1, m[D];
#pragma unroll
		for (int e = 0; e < D; e++) {
			const int o = rem % span[e] - a.reach[e];
			rem /= span[e];
			const int q = ci[e] + o;
			m[e] = floor_div(q, a.n[e]);
			lin += (q - m[e] * a.n[e]) * stride;
			stride *= a.n[e];
		}
		for (int p = a.cell_start[lin]; p < a.cell_start[lin + 1]; p++) {
			const int j = a.items[p];
			if (j == i)
				continue;   // no self interaction, with any image
			double ds[D], sh[D];
#pragma unroll
			for (int e = 0; e < D; e++)
				ds[e] = (a.frac[(size_t)j * D + e] + (double)m[e]) - si[e];
			double r2 = 0.0;
#pragma unroll
			for (int x = 0; x < D; x++) {
				double c = 0.0;
#pragma unroll
				for (int e = 0; e < D; e++)
					c += ds[e] * a.basis[e * D + x];
				sh[x] = c;   // Cartesian displacement from i to this image of j
				r2 += c * c;
			}
			const double r = sqrt(r2);
			const double sig = Ri + a.radii[j];
			if (i < j) {
				const double rs = r / sig;
				if (rs < 1.0)
					E += (1.0 - rs) * (1.0 - rs);
			}
			if (r < 1e-15) {
				// coincident: a unit push along the first axis, away from the higher index
				const double c = 2.0 / sig;
				f[0] -= c * ((i > j) ? -1.0 : 1.0);
#pragma unroll
				for (int x = 1; x < D; x++)
					f[x] -= c * sh[x];
			} else if (r < sig) {
				const double c = 2.0 / sig * (1.0 / r - 1.0 / sig);
#pragma unroll
				for (int x = 0; x < D; x++)
					f[x] += c * (-1.0 * sh[x]);
			}
		}
	}
	a.E_out[i] = E;
#pragma unroll
	for (int x = 0; x < D; x++)
		a.F_out[(size_t)i * D + x] = f[x] * a.e0;
}

template <class T> int grow_dev(T **p, size_t &cap, size_t n)
{
	n = std::max<size_t>(n, 1);
	if (n <= cap)
		return CC_OK;
	cudaFree(*p);
	*p = nullptr;
	cap = 0;
	cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), n * sizeof(T));
	if (e != cudaSuccess)
		return cc::set_error(CC_ERR_OOM, (std::string("cudaMalloc: ") + cudaGetErrorString(e)).c_str());
	cap = n;
	return CC_OK;
}

}  // namespace

struct cc_multi {
	int d = 0;
	double basis[9] = {0}, recip[9] = {0}, volume = 0;
	double u0 = 1.0, e0 = 1.0;
	bool repulsion = true;
	std::vector<cc_handle *> species;
	int64_t N = -1;
	std::vector<std::vector<int64_t> > members;   // particle indices of each species, increasing
	std::vector<int32_t> spec;
	std::vector<double> radii;
	double rc = 0.0;
	int n[3] = {1, 1, 1}, reach[3] = {0, 0, 0};
	cudaStream_t stream = nullptr;
	double *d_frac = nullptr, *d_radii = nullptr, *d_E = nullptr, *d_F = nullptr;
	int *d_cell = nullptr, *d_start = nullptr, *d_items = nullptr;
	size_t cap_frac = 0, cap_radii = 0, cap_E = 0, cap_F = 0, cap_cell = 0, cap_start = 0, cap_items = 0;
	std::vector<double> h_E, h_F, h_fs;
};

namespace {

// S0: per species the S2 targets (ShiftedCCPotential_S2 for that species' collective-coordinate part), or null
int multi_create(int d, const double *basis, int nspecies, const int64_t *M, const int32_t *const *modes,
                 const double *const *V, const double *const *S0, double u0, double e0, cc_multi **out)
{
	if (!out)
		return cc::set_error(CC_ERR_ARG, "out is null");
	*out = nullptr;
	if (d < 1 || d > 3 || !basis || nspecies < 1 || !M || !std::isfinite(u0) || !std::isfinite(e0))
		return cc::set_error(CC_ERR_ARG, "invalid multi-species arguments");
	cc_multi *m = new cc_multi();
	m->d = d;
	std::memcpy(m->basis, basis, sizeof(double) * d * d);
	if (!cc::cell_geometry(d, m->basis, &m->volume, m->recip)) {
		delete m;
		return cc::set_error(CC_ERR_ARG, "degenerate cell basis");
	}
	m->u0 = u0;
	m->e0 = e0;
	m->repulsion = std::abs(e0) > 1e-10;   // as the reference's WithRepulsion
	for (int s = 0; s < nspecies; s++) {
		cc_handle *h = nullptr;
		const int32_t *ms = M[s] > 0 ? modes[s] : nullptr;
		const double *vs = M[s] > 0 ? V[s] : nullptr;
		const int rc = (S0 && S0[s]) ? cc_create_s2(d, basis, M[s], ms, vs, S0[s], 0.0, &h)
		                             : cc_create(d, basis, M[s], ms, vs, 0.0, &h);
		if (rc != CC_OK) {
			cc_multi_destroy(m);
			return rc;
		}
		m->species.push_back(h);
	}
	if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) {
		cc_multi_destroy(m);
		return cc::set_error(CC_ERR_CUDA, "cudaStreamCreate failed");
	}
	m->members.resize(nspecies);
	*out = m;
	return CC_OK;
}

}  // namespace

extern "C" {

int cc_multi_create(int d, const double *basis, int nspecies, const int64_t *M, const int32_t *const *modes,
                    const double *const *V, double u0, double e0, cc_multi **out)
{
	return multi_create(d, basis, nspecies, M, modes, V, nullptr, u0, e0, out);
}

int cc_multi_create_s2(int d, const double *basis, int nspecies, const int64_t *M, const int32_t *const *modes,
                       const double *const *V, const double *const *S0, double u0, double e0, cc_multi **out)
{
	return multi_create(d, basis, nspecies, M, modes, V, S0, u0, e0, out);
}

int cc_multi_destroy(cc_multi *m)
{
	if (!m)
		return CC_OK;
	if (m->stream)
		cudaStreamSynchronize(m->stream);
	for (cc_handle *h : m->species)
		cc_destroy(h);
	cudaFree(m->d_frac);
	cudaFree(m->d_radii);
	cudaFree(m->d_E);
	cudaFree(m->d_F);
	cudaFree(m->d_cell);
	cudaFree(m->d_start);
	cudaFree(m->d_items);
	if (m->stream)
		cudaStreamDestroy(m->stream);
	delete m;
	return CC_OK;
}

int cc_multi_set_configuration(cc_multi *m, int64_t N, const double *frac, const int32_t *species, const double *radii)
{
	if (!m)
		return cc::set_error(CC_ERR_ARG, "null handle");
	if (N < 0 || N > (1 << 30) || (N > 0 && (!frac || !species)))
		return cc::set_error(CC_ERR_ARG, "invalid particle count or null positions / species");
	const int d = m->d, S = (int)m->species.size();
	std::vector<double> s((size_t)N * d);
	for (int64_t i = 0; i < N * d; i++) {
		const double x = frac[i];
		if (!std::isfinite(x))
			return cc::set_error(CC_ERR_ARG, "non-finite fractional coordinate");
		double v = x - std::floor(x);
		s[i] = v - std::floor(v);   // Configuration::Insert's wrap
	}
	std::vector<std::vector<int64_t> > members(S);
	for (int64_t i = 0; i < N; i++) {
		if (species[i] < 0 || species[i] >= S)
			return cc::set_error(CC_ERR_ARG, "every particle needs a species in 0..nspecies-1");
		members[species[i]].push_back(i);
	}
	// radii: the reference's default is 0.5 with rc = 1; SetSecureRadii takes rc = 2.01 max R
	std::vector<double> R((size_t)N, 0.5);
	double rc = 1.0;
	if (radii) {
		double rmax = 0.0;
		for (int64_t i = 0; i < N; i++) {
			if (!std::isfinite(radii[i]) || radii[i] <= 0.0)
				return cc::set_error(CC_ERR_ARG, "radii must be finite and positive");
			R[i] = radii[i];
			rmax = std::max(rmax, radii[i]);
		}
		rc = N > 0 ? 2.01 * rmax : 0.0;
	}
	// species potentials: each species' particles in increasing index order
	for (int sp = 0; sp < S; sp++) {
		std::vector<double> fs(members[sp].size() * d);
		for (size_t k = 0; k < members[sp].size(); k++)
			for (int e = 0; e < d; e++)
				fs[k * d + e] = s[(size_t)members[sp][k] * d + e];
		if (int rc2 = cc_set_positions(m->species[sp], (int64_t)members[sp].size(), fs.data()))
			return rc2;
	}
	// contact cell grid
	int ncell = 1;
	for (int e = 0; e < d; e++) {
		double b2 = 0.0;
		for (int x = 0; x < d; x++)
			b2 += m->recip[e * d + x] * m->recip[e * d + x];
		const double h = 2.0 * M_PI / std::sqrt(b2);   // spacing of the lattice planes of axis e
		const double nmax = std::max(1.0, std::ceil(2.0 * std::pow((double)std::max<int64_t>(N, 1), 1.0 / d)));
		const int ne = rc > 0 ? (int)std::min(nmax, std::max(1.0, std::floor(h / rc))) : 1;
		m->n[e] = ne;
		m->reach[e] = rc > 0 ? (int)std::ceil((double)ne * rc / h * (1.0 + 1e-9)) : 0;
		if (m->reach[e] > 64)
			return cc::set_error(CC_ERR_ARG, "contact radius spans more than 64 cell images along an axis");
		ncell *= ne;
	}
	std::vector<int> cell((size_t)N * d), lin((size_t)N), start((size_t)ncell + 1, 0), items((size_t)N);
	for (int64_t i = 0; i < N; i++) {
		int l = 0, stride = 1;
		for (int e = 0; e < d; e++) {
			int c = (int)std::floor(s[(size_t)i * d + e] * m->n[e]);
			c = std::min(std::max(c, 0), m->n[e] - 1);
			cell[(size_t)i * d + e] = c;
			l += c * stride;
			stride *= m->n[e];
		}
		lin[i] = l;
		start[l + 1]++;
	}
	for (int c = 0; c < ncell; c++)
		start[c + 1] += start[c];
	{
		std::vector<int> fill(start.begin(), start.end() - 1);
		for (int64_t i = 0; i < N; i++)
			items[fill[lin[i]]++] = (int)i;
	}
	int rc3;
	if ((rc3 = grow_dev(&m->d_frac, m->cap_frac, (size_t)N * d)) || (rc3 = grow_dev(&m->d_radii, m->cap_radii, (size_t)N)) ||
	    (rc3 = grow_dev(&m->d_E, m->cap_E, (size_t)N)) || (rc3 = grow_dev(&m->d_F, m->cap_F, (size_t)N * d)) ||
	    (rc3 = grow_dev(&m->d_cell, m->cap_cell, (size_t)N * d)) ||
	    (rc3 = grow_dev(&m->d_start, m->cap_start, (size_t)ncell + 1)) ||
	    (rc3 = grow_dev(&m->d_items, m->cap_items, (size_t)N)))
		return rc3;
	cudaError_t e = cudaSuccess;
	if (N > 0) {
		if (e == cudaSuccess)
			e = cudaMemcpyAsync(m->d_frac, s.data(), sizeof(double) * N * d, cudaMemcpyHostToDevice, m->stream);
		if (e == cudaSuccess)
			e = cudaMemcpyAsync(m->d_radii, R.data(), sizeof(double) * N, cudaMemcpyHostToDevice, m->stream);
		if (e == cudaSuccess)
			e = cudaMemcpyAsync(m->d_cell, cell.data(), sizeof(int) * N * d, cudaMemcpyHostToDevice, m->stream);
		if (e == cudaSuccess)
			e = cudaMemcpyAsync(m->d_items, items.data(), sizeof(int) * N, cudaMemcpyHostToDevice, m->stream);
	}
	if (e == cudaSuccess)
		e = cudaMemcpyAsync(m->d_start, start.data(), sizeof(int) * (ncell + 1), cudaMemcpyHostToDevice, m->stream);
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(m->stream);
	if (e != cudaSuccess)
		return cc::set_error(CC_ERR_CUDA, (std::string("multi-species upload: ") + cudaGetErrorString(e)).c_str());
	m->N = N;
	m->members.swap(members);
	m->radii.swap(R);
	m->rc = rc;
	return CC_OK;
}

int cc_multi_energy_grad(cc_multi *m, double *E, double *F)
{
	if (!m || !E)
		return cc::set_error(CC_ERR_ARG, "null handle or E");
	if (m->N < 0)
		return cc::set_error(CC_ERR_STATE, "configuration not set");
	const int64_t N = m->N;
	const int d = m->d, S = (int)m->species.size();
	// contact part on the GPU (launched first: it overlaps the host side of the species evaluations)
	const bool contact = m->repulsion && N > 0;
	if (contact) {
		ContactArgs a;
		a.frac = m->d_frac;
		a.radii = m->d_radii;
		a.cell = m->d_cell;
		a.cell_start = m->d_start;
		a.items = m->d_items;
		a.N = (int)N;
		for (int e = 0; e < 3; e++) {
			a.n[e] = m->n[e];
			a.reach[e] = m->reach[e];
		}
		for (int k = 0; k < 9; k++)
			a.basis[k] = m->basis[k];
		a.e0 = m->e0;
		a.E_out = m->d_E;
		a.F_out = m->d_F;
		const unsigned grid = (unsigned)((N + 127) / 128);
		if (d == 1)
			cc_contact_kernel<1><<<grid, 128, 0, m->stream>>>(a);
		else if (d == 2)
			cc_contact_kernel<2><<<grid, 128, 0, m->stream>>>(a);
		else
			cc_contact_kernel<3><<<grid, 128, 0, m->stream>>>(a);
		cudaError_t e = cudaGetLastError();
		if (e != cudaSuccess)
			return cc::set_error(CC_ERR_CUDA, (std::string("contact kernel: ") + cudaGetErrorString(e)).c_str());
	}
	// species potentials
	double CC = 0.0;
	if (F)
		std::fill(F, F + N * d, 0.0);
	for (int sp = 0; sp < S; sp++) {
		const std::vector<int64_t> &mem = m->members[sp];
		double Es = 0.0;
		m->h_fs.resize(std::max<size_t>(mem.size() * d, 1));
		if (int rc = cc_energy_grad(m->species[sp], &Es, F ? m->h_fs.data() : nullptr, CC_PREC_FP64))
			return rc;
		const double ns = (double)mem.size();
		CC += (ns / (double)N) * Es;
		if (F) {
			const double w = m->u0 * ns / (double)N;
			for (size_t k = 0; k < mem.size(); k++)
				for (int x = 0; x < d; x++)
					F[(size_t)mem[k] * d + x] = m->h_fs[k * d + x] * w;
		}
	}
	double CP = 0.0;
	if (contact) {
		m->h_E.resize((size_t)N);
		m->h_F.resize((size_t)N * d);
		cudaError_t e = cudaMemcpyAsync(m->h_E.data(), m->d_E, sizeof(double) * N, cudaMemcpyDeviceToHost, m->stream);
		if (e == cudaSuccess && F)
			e = cudaMemcpyAsync(m->h_F.data(), m->d_F, sizeof(double) * N * d, cudaMemcpyDeviceToHost, m->stream);
		if (e == cudaSuccess)
			e = cudaStreamSynchronize(m->stream);
		if (e != cudaSuccess)
			return cc::set_error(CC_ERR_CUDA, (std::string("contact result: ") + cudaGetErrorString(e)).c_str());
		for (int64_t i = 0; i < N; i++)
			CP += m->h_E[i];
		if (F)   // contact force + species force, as the reference adds them
			for (int64_t i = 0; i < N * d; i++)
				F[i] = m->h_F[i] + F[i];
	}
	*E = m->u0 * CC + m->e0 * CP;
	return CC_OK;
}

}  // extern "C"
