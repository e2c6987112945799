// cc_capi.cu — the C ABI of libccgpu.so (declared in include/cc_gpu.h): handles, k-set planning, launches.
//
// A handle holds the constraint set of one ShiftedCCPotential (potential/CollectiveCoordinatePotential.h:84-117)
// planned into lattice-line segments (see cc_kernels.cuh), the cell (volume, reciprocal basis) and the device
// buffers of the bound positions. One evaluation is two kernel launches on the handle's stream:
//   cc_rho_kernel   -> rho per slot, u = V conj(rho), the energy (and rho in mode order on request);
//   cc_force_kernel -> Cartesian forces and/or the gradient in fractional coordinates.
// There is no CPU path: without a CUDA device every call that computes returns CC_ERR_NOGPU.
#include "../../include/cc_gpu.h"
#include "cc_internal.h"
#include "cc_kernels.cuh"
#include "cc_lbfgs.cuh"
#include "cc_multi_launch.h"
#include "cc_nufft.cuh"
#include "cc_plan.h"

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <array>
#include <atomic>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

namespace {
thread_local std::string g_err = "";
}  // namespace

namespace cci {

int fail(int code, const std::string &msg)
{
	g_err = msg;
	return code;
}

std::atomic<unsigned long long> g_alloc_gen{1};

}  // namespace cci

namespace cc {
// Error reporting for the library's other translation units: sets the message cc_last_error() returns.
int set_error(int code, const char *msg)
{
	g_err = msg;
	return code;
}
}  // namespace cc

using namespace cci;

int cci::check_prec(int precision)
{
	if (precision != CC_PREC_FP64 && precision != CC_PREC_MIXED)
		return fail(CC_ERR_ARG, "precision must be CC_PREC_FP64 or CC_PREC_MIXED");
	return CC_OK;
}

int cci::sm_count()
{
	static int n = 0;
	if (n == 0) {
		int dev = 0;
		cudaGetDevice(&dev);
		if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
			n = 148;
	}
	return n;
}

int cci::get_splits(DevKSet &k, int want, const DevSplits **out)
{
	for (const DevSplits &f : k.splits)
		if (f.want == want) {
			*out = &f;
			return CC_OK;
		}
	DevSplits f;
	f.want = want;
	f.host = cc::force_splits(k.plan, want);
	int rc;
	if ((rc = upload(&f.kstart, f.host.start)) || (rc = upload(&f.kspec, f.host.spec)))
		return rc;
	k.splits.push_back(f);
	*out = &k.splits.back();
	return CC_OK;
}


int cci::upload_kset(DevKSet &k, const cc::Plan &plan)
{
	k.release();
	k.plan = plan;
	int rc;
	const size_t nslot = plan.slotV.size(), M = plan.mode_slot.size();
	const size_t nred = (nslot + 31) / 32;
	if ((rc = upload(&k.segs, plan.segs)) || (rc = upload(&k.rspec, plan.rspec)) || (rc = upload(&k.slotV, plan.slotV)) ||
	    (rc = upload(&k.bstart, plan.bstart)) || (rc = upload(&k.bspec, plan.bspec)) ||
	    (rc = upload(&k.mode_slot, plan.mode_slot)) || (rc = dev_alloc(&k.rho_slot, nslot)) ||
	    (rc = dev_alloc(&k.u_slot, nslot)) || (rc = dev_alloc(&k.rho_mode, M)) || (rc = dev_alloc(&k.eblock, nred)) ||
	    (rc = dev_alloc(&k.ticket, 1)))
		return rc;
	CC_CUDA(cudaMemset(k.ticket, 0, sizeof(unsigned)));
	return CC_OK;
}

namespace {

// ---------------------------------------------------------------------------------------------------------------
// launch configuration
// ---------------------------------------------------------------------------------------------------------------
struct Launch {
	int nsplit, per_split, csize, chunk;   // rho: particle splits (a multiple of the cluster size)
	int want_force;                       // force: requested number of segment splits
};


// Record a timing event; inside a stream capture it must be an external record node to carry a timestamp.
cudaError_t record_timing(cudaEvent_t e, cudaStream_t st)
{
	cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
	if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusActive)
		return cudaEventRecordWithFlags(e, st, cudaEventRecordExternal);
	return cudaEventRecord(e, st);
}


int rho_wave(int d, bool mixed, int csize, size_t smem);   // resident rho blocks (clusters of csize) on the device
int force_wave(int d, bool mixed, size_t smem);            // resident force blocks on the device

// Per-block fixed cost of each kernel (table build, barriers, split reduction) expressed in particle-k pairs of its
// main loop, from block-level timelines of the 3D N=2000 and 2D N=20000 workloads on B200.
constexpr double kRhoFixedPairs = 17000.0;
constexpr double kForceFixedPairs = 4600.0;

// Estimated time of `blocks` equal blocks sharing `pairs`, `wave` of them resident at once.
double grid_cost(int64_t blocks, int wave, double pairs, double fixed_pairs)
{
	const int64_t waves = (blocks + wave - 1) / wave;
	return (double)waves * (1.0 + pairs / (double)blocks / fixed_pairs);
}

Launch choose_launch(const cc::Plan &p, int64_t N, bool mixed)
{
	Launch l;
	const size_t esz = mixed ? sizeof(float2) : sizeof(double2);
	l.chunk = (int)std::max<size_t>(8, std::min<size_t>(64, kRhoTabBudget / (esz * std::max(1, p.block_max_row | 1))));
	const double pairs = (double)std::max<int64_t>(N, 1) * (double)std::max<int64_t>(p.real_segs, 1) * p.L;
	// rho: particle splits (a multiple of the cluster size, at least 2 particles each) with the least estimated time
	// over whole waves of resident blocks
	const int ng = std::max(1, p.nbgroups());
	const size_t rsm = mixed ? rho_smem<float2>(p.block_max_row, l.chunk, p.L)
	                         : rho_smem<double2>(p.block_max_row, l.chunk, p.L);
	const int maxns = (int)std::max<int64_t>(1, std::min<int64_t>(N / 2, 4096));
	double best = 1e300;
	l.csize = 1;
	l.nsplit = 1;
	for (int cs = 8; cs >= 1; cs >>= 1) {
		const int wave = std::max(cs, rho_wave(p.d, mixed, cs, rsm));
		for (int ns = cs; ns <= maxns; ns += cs) {
			// smaller clusters leave more partial rows to the reduce kernel
			const double c = grid_cost((int64_t)ns * ng, wave, pairs, kRhoFixedPairs) * (cs == 8 ? 1.0 : 1.15);
			if (c < best) {
				best = c;
				l.csize = cs;
				l.nsplit = ns;
			}
			if ((int64_t)ns * ng > 4LL * wave)
				break;
		}
	}
	l.per_split = (int)std::max<int64_t>(1, (N + l.nsplit - 1) / l.nsplit);
	// no cluster of splits left without particles (N = 2000 over 192 splits of 11 fills only 182: 184 splits, one
	// cluster wave fewer to place)
	l.nsplit = (int)std::min<int64_t>(l.nsplit, ((N + l.per_split - 1) / l.per_split + l.csize - 1) / l.csize * l.csize);
	// force: segment splits of every group of 32 particles, chosen the same way
	const int64_t pg = std::max<int64_t>(1, (N + 31) / 32);
	// (the tables of a split usually stay within 64 entries per particle)
	const size_t fsm = mixed ? force_smem<float2>(64, p.d) : force_smem<double2>(64, p.d);
	const int fwave = std::max(1, force_wave(p.d, mixed, fsm));
	const int maxnk = (int)std::max<int64_t>(1, std::min<int64_t>(p.real_segs, 1024));
	best = 1e300;
	l.want_force = 1;
	for (int nk = 1; nk <= maxnk; nk++) {
		const double c = grid_cost(pg * nk, fwave, pairs, kForceFixedPairs);
		if (c < best) {
			best = c;
			l.want_force = nk;
		}
		if (pg * nk > 4LL * fwave)
			break;
	}
	return l;
}

// ---------------------------------------------------------------------------------------------------------------
// kernel dispatch
// ---------------------------------------------------------------------------------------------------------------

// Launch with programmatic stream serialization: the kernel may be scheduled while the previous kernel on the stream
// drains; it calls cudaGridDependencySynchronize() before it reads that kernel's results.
template <typename Kern, typename Arg>
cudaError_t launch_pdl(Kern kern, dim3 grid, dim3 block, size_t smem, cudaStream_t st, const Arg &a)
{
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = grid;
	cfg.blockDim = block;
	cfg.dynamicSmemBytes = smem;
	cfg.stream = st;
	cudaLaunchAttribute attr[1];
	attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
	attr[0].val.programmaticStreamSerializationAllowed = 1;
	cfg.attrs = attr;
	cfg.numAttrs = 1;
	return cudaLaunchKernelEx(&cfg, kern, a);
}
template <int D, int L, bool MIXED> cudaError_t rho_attr()
{
	typedef typename std::conditional<MIXED, float2, double2>::type C;
	static cudaError_t e = cudaFuncSetAttribute(cc::cc_rho_kernel<D, L, MIXED>,
	                                            cudaFuncAttributeMaxDynamicSharedMemorySize,
	                                            (int)rho_smem<C>(cc::kMaxRow, 64, L));
	return e;
}
template <int D, int L, bool MIXED> cudaError_t force_attr()
{
	typedef typename std::conditional<MIXED, float2, double2>::type C;
	static cudaError_t e = cudaFuncSetAttribute(cc::cc_force_kernel<D, L, MIXED>,
	                                            cudaFuncAttributeMaxDynamicSharedMemorySize,
	                                            (int)force_smem<C>(cc::kMaxRow, D));
	return e;
}

// Resident blocks of one wave, from the occupancy calculator (cached per device, kernel, cluster size and smem).
struct WaveKey {
	int dev, kind, d, mixed, csize;
	size_t smem;
	bool operator==(const WaveKey &o) const
	{
		return dev == o.dev && kind == o.kind && d == o.d && mixed == o.mixed && csize == o.csize && smem == o.smem;
	}
};
std::mutex g_wave_mu;
std::vector<std::pair<WaveKey, int> > g_waves;

template <int D, bool MIXED> int rho_wave_t(int csize, size_t smem)
{
	if (rho_attr<D, 8, MIXED>() != cudaSuccess)
		return sm_count() * 3;
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = dim3(1, csize);
	cfg.blockDim = dim3(cc::kRhoThreads);
	cfg.dynamicSmemBytes = smem;
	cudaLaunchAttribute at[1];
	at[0].id = cudaLaunchAttributeClusterDimension;
	at[0].val.clusterDim.x = 1;
	at[0].val.clusterDim.y = csize;
	at[0].val.clusterDim.z = 1;
	cfg.attrs = at;
	cfg.numAttrs = 1;
	int n = 0;
	if (cudaOccupancyMaxActiveClusters(&n, cc::cc_rho_kernel<D, 8, MIXED>, &cfg) != cudaSuccess || n <= 0) {
		cudaGetLastError();
		return sm_count() * 3;
	}
	return n * csize;
}
template <int D, bool MIXED> int force_wave_t(size_t smem)
{
	int n = 0;
	if (force_attr<D, 8, MIXED>() != cudaSuccess ||
	    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, cc::cc_force_kernel<D, 8, MIXED>, cc::kForceThreads, smem) !=
	        cudaSuccess ||
	    n <= 0) {
		cudaGetLastError();
		n = 2;
	}
	return n * sm_count();
}

int cached_wave(int kind, int d, bool mixed, int csize, size_t smem)
{
	int dev = 0;
	cudaGetDevice(&dev);
	const WaveKey k = {dev, kind, d, mixed ? 1 : 0, csize, smem};
	{
		std::lock_guard<std::mutex> g(g_wave_mu);
		for (auto &e : g_waves)
			if (e.first == k)
				return e.second;
	}
	int w;
	if (kind == 0)
		w = d == 1 ? (mixed ? rho_wave_t<1, true>(csize, smem) : rho_wave_t<1, false>(csize, smem))
		  : d == 2 ? (mixed ? rho_wave_t<2, true>(csize, smem) : rho_wave_t<2, false>(csize, smem))
		           : (mixed ? rho_wave_t<3, true>(csize, smem) : rho_wave_t<3, false>(csize, smem));
	else
		w = d == 1 ? (mixed ? force_wave_t<1, true>(smem) : force_wave_t<1, false>(smem))
		  : d == 2 ? (mixed ? force_wave_t<2, true>(smem) : force_wave_t<2, false>(smem))
		           : (mixed ? force_wave_t<3, true>(smem) : force_wave_t<3, false>(smem));
	std::lock_guard<std::mutex> g(g_wave_mu);
	g_waves.push_back(std::make_pair(k, w));
	return w;
}

int rho_wave(int d, bool mixed, int csize, size_t smem) { return cached_wave(0, d, mixed, csize, smem); }
int force_wave(int d, bool mixed, size_t smem) { return cached_wave(1, d, mixed, 1, smem); }

template <int D, int L, bool MIXED> int launch_rho_t(const cc::RhoArgs &a, int ngroups, int nsplit, int csize, int row,
                                                     cudaStream_t st)
{
	typedef typename std::conditional<MIXED, float2, double2>::type C;
	auto kern = cc::cc_rho_kernel<D, L, MIXED>;
	if (cudaError_t e = rho_attr<D, L, MIXED>())
		return fail(CC_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = dim3(ngroups, nsplit);
	cfg.blockDim = dim3(cc::kRhoThreads);
	cfg.dynamicSmemBytes = rho_smem<C>(row, a.chunk, L);
	cfg.stream = st;
	cudaLaunchAttribute attrs[2];
	attrs[0].id = cudaLaunchAttributeClusterDimension;
	attrs[0].val.clusterDim.x = 1;
	attrs[0].val.clusterDim.y = csize;
	attrs[0].val.clusterDim.z = 1;
	attrs[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
	attrs[1].val.programmaticStreamSerializationAllowed = 1;
	cfg.attrs = attrs;
	cfg.numAttrs = 2;
	CC_CUDA(cudaLaunchKernelEx(&cfg, kern, a));
	return CC_OK;
}

template <int D, int L, bool MIXED> int launch_force_t(const cc::ForceArgs &a, int64_t N, int row, cudaStream_t st)
{
	typedef typename std::conditional<MIXED, float2, double2>::type C;
	auto kern = cc::cc_force_kernel<D, L, MIXED>;
	if (cudaError_t e = force_attr<D, L, MIXED>())
		return fail(CC_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
	CC_CUDA(launch_pdl(kern, dim3((unsigned)((N + 31) / 32), a.nksplit), dim3(cc::kForceThreads), force_smem<C>(row, D),
	                   st, a));
	return CC_OK;
}

template <int D> int launch_rho_d(const cc::RhoArgs &a, bool mixed, int ngroups, int nsplit, int csize, int row,
                                  cudaStream_t st)
{
	return mixed ? launch_rho_t<D, 8, true>(a, ngroups, nsplit, csize, row, st)
	             : launch_rho_t<D, 8, false>(a, ngroups, nsplit, csize, row, st);
}
template <int D> int launch_force_d(const cc::ForceArgs &a, bool mixed, int64_t N, int row, cudaStream_t st)
{
	return mixed ? launch_force_t<D, 8, true>(a, N, row, st) : launch_force_t<D, 8, false>(a, N, row, st);
}

int launch_rho(int d, const cc::RhoArgs &a, bool mixed, int ngroups, int nsplit, int csize, int row, cudaStream_t st)
{
	switch (d) {
	case 1: return launch_rho_d<1>(a, mixed, ngroups, nsplit, csize, row, st);
	case 2: return launch_rho_d<2>(a, mixed, ngroups, nsplit, csize, row, st);
	default: return launch_rho_d<3>(a, mixed, ngroups, nsplit, csize, row, st);
	}
}
int launch_force(int d, const cc::ForceArgs &a, bool mixed, int64_t N, int row, cudaStream_t st)
{
	switch (d) {
	case 1: return launch_force_d<1>(a, mixed, N, row, st);
	case 2: return launch_force_d<2>(a, mixed, N, row, st);
	default: return launch_force_d<3>(a, mixed, N, row, st);
	}
}

// force splits for `want`, uploaded once and cached on the k-set

// ---------------------------------------------------------------------------------------------------------------
// buffers
// ---------------------------------------------------------------------------------------------------------------
int ensure_particles(cc_handle *h, int64_t N)
{
	const size_t need = (size_t)std::max<int64_t>(N, 1);
	if (need > h->ncap) {
		cudaFree(h->d_frac);
		cudaFree(h->d_F);
		cudaFree(h->d_gfrac);
		cudaFree(h->d_fcounters);
		h->d_frac = h->d_F = h->d_gfrac = nullptr;
		h->d_fcounters = nullptr;
		h->ncap = 0;
		h->N = -1;   // the bound positions do not survive a reallocation
		h->lastF_valid = false;
		int rc;
		if ((rc = dev_alloc(&h->d_frac, need * h->d)) || (rc = dev_alloc(&h->d_F, need * h->d)) ||
		    (rc = dev_alloc(&h->d_gfrac, need * h->d)) || (rc = dev_alloc(&h->d_fcounters, (need + 31) / 32)))
			return rc;
		CC_CUDA(cudaMemset(h->d_fcounters, 0, ((need + 31) / 32) * sizeof(unsigned)));
		h->ncap = need;
	}
	const size_t pin = need * h->d + 2;
	if (pin > h->pin_cap) {
		cudaFreeHost(h->h_pin);
		h->h_pin = nullptr;
		h->pin_cap = 0;
		h->lastF_valid = false;
		h->d_pin = nullptr;
		g_alloc_gen++;
		cudaError_t e = cudaHostAlloc(reinterpret_cast<void **>(&h->h_pin), pin * sizeof(double), cudaHostAllocMapped);
		if (e != cudaSuccess)
			return fail(CC_ERR_OOM, std::string("cudaHostAlloc: ") + cudaGetErrorString(e));
		e = cudaHostGetDevicePointer(reinterpret_cast<void **>(&h->d_pin), h->h_pin, 0);
		if (e != cudaSuccess)
			return fail(CC_ERR_CUDA, std::string("cudaHostGetDevicePointer: ") + cudaGetErrorString(e));
		h->pin_cap = pin;
	}
	return CC_OK;
}

// Pinned input staging of n doubles, free for writing: the previous copy out of it has completed.
int input_staging(cc_handle *h, size_t n)
{
	if (!h->ev_in)
		CC_CUDA(cudaEventCreateWithFlags(&h->ev_in, cudaEventDisableTiming));
	if (h->in_pending) {
		CC_CUDA(cudaEventSynchronize(h->ev_in));
		h->in_pending = false;
	}
	n = std::max<size_t>(n, 1);
	if (n > h->in_cap) {
		g_alloc_gen++;
		cudaFreeHost(h->h_in);
		h->h_in = nullptr;
		h->d_in = nullptr;
		h->in_cap = 0;
		cudaError_t e = cudaHostAlloc(reinterpret_cast<void **>(&h->h_in), n * sizeof(double), cudaHostAllocMapped);
		if (e != cudaSuccess)
			return fail(CC_ERR_OOM, std::string("cudaHostAlloc: ") + cudaGetErrorString(e));
		e = cudaHostGetDevicePointer(reinterpret_cast<void **>(&h->d_in), h->h_in, 0);
		if (e != cudaSuccess) {
			cudaFreeHost(h->h_in);
			h->h_in = nullptr;
			h->d_in = nullptr;
			return fail(CC_ERR_CUDA, std::string("cudaHostGetDevicePointer: ") + cudaGetErrorString(e));
		}
		h->in_cap = n;
	}
	return CC_OK;
}

// Copy n staged doubles to d_frac on the handle's stream; the staging is reusable once ev_in has passed.
int upload_staged(cc_handle *h, size_t n)
{
	h->upload_pending = false;
	if (n == 0)
		return CC_OK;
	CC_CUDA(cudaMemcpyAsync(h->d_frac, h->h_in, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
	CC_CUDA(cudaEventRecord(h->ev_in, h->stream));
	h->in_pending = true;
	return CC_OK;
}

// Positions staged by cc_set_positions are copied to the device by the first call that reads them.
int flush_upload(cc_handle *h)
{
	if (!h->upload_pending || h->N <= 0)
		return CC_OK;
	return upload_staged(h, (size_t)h->N * h->d);
}

// Wrap into [0,1) as Configuration::Insert does (core/PeriodicCellList.h:517-538: floor twice). Values already in
// [0,1) are returned unchanged, which is what the two floors give for them. Returns false on a non-finite value.
inline bool wrap_unit(double x, double *out)
{
	if (x >= 0.0 && x < 1.0) {
		*out = x;
		return true;
	}
	if (!std::isfinite(x))
		return false;
	double s = x - std::floor(x);
	s -= std::floor(s);
	*out = s;
	return true;
}

int ensure_partial(DevKSet &k, size_t elems)
{
	if (elems <= k.partial_cap)
		return CC_OK;
	cudaFree(k.partial);
	k.partial = nullptr;
	k.partial_cap = 0;
	int rc = dev_alloc(&k.partial, elems);
	if (rc)
		return rc;
	k.partial_cap = elems;
	return CC_OK;
}

int ensure_partialG(cc_handle *h, size_t elems)
{
	if (elems <= h->partialG_cap)
		return CC_OK;
	cudaFree(h->d_partialG);
	h->d_partialG = nullptr;
	h->partialG_cap = 0;
	int rc = dev_alloc(&h->d_partialG, elems);
	if (rc)
		return rc;
	h->partialG_cap = elems;
	return CC_OK;
}

// rho pass of k-set `k` over N device positions: rho per slot, u, and the energy into d_E.
// energy_in_force: a force pass follows and sums the energy partials (one reduce-block ticket less on the path).
// rho_out / u_out: where the reduce writes rho and u per slot (the k-set's own buffers when null; the S2 form's
// per-slot targets then apply).
int run_rho(cc_handle *h, DevKSet &k, int64_t N, const double *d_frac, double *d_E, bool want_rho_mode, bool mixed,
            const Launch &l, cudaStream_t st, cudaEvent_t after_rho = nullptr, bool energy_in_force = false,
            double2 *rho_out = nullptr, double2 *u_out = nullptr)
{
	const cc::Plan &p = k.plan;
	if (p.nslot == 0) {
		cc::cc_set_scalar_kernel<<<1, 1, 0, st>>>(d_E, h->shift);
		CC_CUDA(cudaGetLastError());
		return CC_OK;
	}
	const int nsplit = N > 0 ? l.nsplit : 1;
	const int csize = N > 0 ? l.csize : 1;
	const int rows = nsplit / csize;
	if (int rc = ensure_partial(k, (size_t)rows * p.nslot))
		return rc;
	cc::RhoArgs a = {};
	a.frac = d_frac;
	a.N = (int)N;
	a.per_split = N > 0 ? l.per_split : 0;
	a.chunk = l.chunk;
	a.segs = k.segs;
	a.bstart = k.bstart;
	a.bspec = k.bspec;
	a.nseg = (int)p.segs.size();
	a.nslot = p.nslot;
	a.partial = k.partial;
	a.skip = h->d_skip;
	a.frac_copy = (&k == &h->main) ? h->rho_copy : nullptr;
	a.early = (h->early_call && &k == &h->main && !a.skip && !a.frac_copy) ? 1 : 0;
	if (int rc = launch_rho(h->d, a, mixed, p.nbgroups(), nsplit, csize, p.block_max_row, st))
		return rc;
	if (after_rho)
		CC_CUDA(record_timing(after_rho, st));
	cc::ReduceArgs r = {};
	r.partial = k.partial;
	r.nsplit = rows;
	r.nslot = p.nslot;
	r.slotV = k.slotV;
	r.rho_offset = h->rho_offset;
	r.rho_slot = k.rho_slot;
	r.u_slot = k.u_slot;
	r.eblock = k.eblock;
	r.ticket = k.ticket;
	r.inv_vol = 1.0 / h->volume;
	r.shift = h->shift;
	r.E_out = d_E;
	r.finalize = energy_in_force ? 0 : 1;
	r.skip = h->d_skip;
	if (rho_out) {
		r.rho_slot = rho_out;
		r.u_slot = u_out;
	} else if (h->d_slotS0 && &k == &h->main) {
		r.slotS0 = h->d_slotS0;
		r.npart = (double)N;
		r.inv_vol = 1.0;
	}
	CC_CUDA(launch_pdl(cc::cc_reduce_kernel, dim3((p.nslot + 31) / 32), dim3(cc::kRedThreads), 0, st, r));
	if (want_rho_mode && !p.mode_slot.empty()) {
		const int M = (int)p.mode_slot.size();
		cc::cc_gather_rho_kernel<<<(M + 255) / 256, 256, 0, st>>>(k.rho_slot, k.mode_slot, M, k.rho_mode);
		CC_CUDA(cudaGetLastError());
	}
	return CC_OK;
}

// d_E: when not null, the force kernel also writes the energy (run_rho was called with energy_in_force).
// u_in / fscale_in: the slot coefficients and force scale to use instead of the handle's (one sub-configuration of
// the multi-configuration S2 form).
int run_force(cc_handle *h, int64_t N, const double *d_frac, double *d_F, double *d_gfrac, bool mixed,
              const Launch &l, cudaStream_t st, double *d_E = nullptr, const double2 *u_in = nullptr,
              double fscale_in = 0.0)
{
	const cc::Plan &p = h->main.plan;
	if (N == 0)
		return CC_OK;
	if (p.nslot == 0) {
		if (d_F)
			CC_CUDA(cudaMemsetAsync(d_F, 0, sizeof(double) * N * h->d, st));
		if (d_gfrac)
			CC_CUDA(cudaMemsetAsync(d_gfrac, 0, sizeof(double) * N * h->d, st));
		return CC_OK;
	}
	const DevSplits *f = nullptr;
	if (int rc = get_splits(h->main, l.want_force, &f))
		return rc;
	const int nk = f->host.count();
	if (nk > 1) {
		int rc = ensure_partialG(h, (size_t)nk * N * h->d);
		if (rc)
			return rc;
	}
	cc::ForceArgs a = {};
	a.frac = d_frac;
	a.N = (int)N;
	a.segs = h->main.segs;
	a.kstart = f->kstart;
	a.kspec = f->kspec;
	a.nksplit = nk;
	a.u_slot = h->main.u_slot;
	a.nseg = (int)p.segs.size();
	a.partialG = h->d_partialG;
	a.counters = h->d_fcounters;
	for (int i = 0; i < 9; i++)
		a.recip[i] = h->recip[i];
	a.fscale = 2.0 / h->volume;
	a.F_out = d_F;
	a.gfrac_out = d_gfrac;
	a.eblock = h->main.eblock;
	a.neblock = (p.nslot + 31) / 32;   // the reduce kernel's grid
	a.inv_vol = 1.0 / h->volume;
	a.shift = h->shift;
	a.E_out = d_E;
	a.skip = h->d_skip;
	if (h->d_slotS0) {   // F = (4 / N) sum_k Im(u z) k with u = V dS conj(rho)
		a.fscale = 4.0 / (double)N;
		a.inv_vol = 1.0;
	}
	if (u_in) {
		a.u_slot = u_in;
		a.fscale = fscale_in;
	}
	return launch_force(h->d, a, mixed, N, f->host.max_row, st);
}

// Grow a device buffer to n elements (contents not kept).
template <class T> int grow(T **p, size_t &cap, size_t n)
{
	if (n <= cap)
		return CC_OK;
	cudaFree(*p);
	*p = nullptr;
	cap = 0;
	if (int rc = dev_alloc(p, n))
		return rc;
	cap = n;
	return CC_OK;
}

// ---------------------------------------------------------------------------------------------------------------
// non-uniform FFT path
// ---------------------------------------------------------------------------------------------------------------
// Gauss-Legendre nodes and weights on [-1, 1]: Newton's method on the three-term Legendre recurrence from the
// asymptotic first guesses cos(pi (i + 3/4) / (q + 1/2)).
void gauss_legendre(int q, std::vector<double> &x, std::vector<double> &w)
{
	x.assign(q, 0.0);
	w.assign(q, 0.0);
	for (int i = 0; i < q; i++) {
		double z = std::cos(M_PI * (i + 0.75) / (q + 0.5)), dp = 1.0;
		for (int it = 0; it < 100; it++) {
			double p0 = 1.0, p1 = z;
			for (int k = 2; k <= q; k++) {
				const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
				p0 = p1;
				p1 = p2;
			}
			dp = q * (z * p1 - p0) / (z * z - 1.0);
			const double dz = p1 / dp;
			z -= dz;
			if (std::fabs(dz) < 1e-16)
				break;
		}
		x[i] = z;
		w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
	}
}

// Smallest n >= lo whose only prime factors are 2, 3, 5 and 7 (sizes cuFFT transforms fastest), even.
int fft_size(int lo)
{
	for (int n = std::max(lo, 2);; n++) {
		if (n & 1)
			continue;
		int r = n;
		for (int p : {2, 3, 5, 7})
			while (r % p == 0)
				r /= p;
		if (r == 1)
			return n;
	}
}

template <class T> int nu_alloc(cc_handle *h, T **p, size_t n)
{
	if (int rc = dev_alloc(p, n))
		return rc;
	h->nu_bufs.push_back(*p);
	return CC_OK;
}

int nufft_setup(cc_handle *h)
{
	if (h->nu_ready)
		return CC_OK;
	const int d = h->d;
	const int64_t M = (int64_t)h->V.size();
	// unique modes (sorted) with summed weights, and each input mode's unique index
	std::vector<int64_t> order((size_t)M);
	for (int64_t m = 0; m < M; m++)
		order[m] = m;
	auto less = [&](int64_t a, int64_t b) {
		for (int e = 0; e < d; e++)
			if (h->modes[a * d + e] != h->modes[b * d + e])
				return h->modes[a * d + e] < h->modes[b * d + e];
		return a < b;
	};
	std::sort(order.begin(), order.end(), less);
	std::vector<int32_t> um;
	std::vector<double> uV;
	std::vector<int> mode_u((size_t)std::max<int64_t>(M, 1), 0);
	int K[3] = {0, 0, 0};
	for (int64_t k = 0; k < M; k++) {
		const int64_t m = order[k];
		const bool same = k > 0 && std::equal(h->modes.begin() + m * d, h->modes.begin() + (m + 1) * d,
		                                      h->modes.begin() + order[k - 1] * d);
		if (!same) {
			for (int e = 0; e < d; e++) {
				um.push_back(h->modes[m * d + e]);
				K[e] = std::max(K[e], std::abs(h->modes[m * d + e]));
			}
			uV.push_back(0.0);
		}
		uV.back() += h->V[m];
		mode_u[m] = (int)uV.size() - 1;
	}
	const int U = (int)uV.size();
	cc::NufftDev &a = h->nu;
	a = cc::NufftDev();
	a.beta = cc::kNufftBetaPerW * cc::kNufftW;
	int64_t ngrid = 1;
	for (int e = 0; e < 3; e++) {
		a.nf[e] = 1;
		a.K[e] = 0;
	}
	for (int e = 0; e < d; e++) {
		a.K[e] = K[e];
		a.nf[e] = fft_size(std::max(2 * (2 * K[e] + 1), 2 * cc::kNufftW));
		ngrid *= a.nf[e];
	}
	if (ngrid > ((int64_t)1 << 28))
		return fail(CC_ERR_ARG, "the k-set's fine grid is too large for the NUFFT path");
	// phihat_e(n) = 2 int_0^{w/2} phi(t) cos(2 pi n t / nf_e) dt by Gauss-Legendre quadrature
	std::vector<double> gx, gw;
	gauss_legendre(4 * cc::kNufftW + 40, gx, gw);
	for (int e = 0; e < d; e++) {
		std::vector<double> ph((size_t)(2 * K[e] + 1));
		for (int n = -K[e]; n <= K[e]; n++) {
			double acc = 0.0;
			for (size_t q = 0; q < gx.size(); q++) {
				const double t = 0.25 * cc::kNufftW * (gx[q] + 1.0), wt = 0.25 * cc::kNufftW * gw[q];
				const double z = 1.0 - (2.0 * t / cc::kNufftW) * (2.0 * t / cc::kNufftW);
				const double phi = z > 0 ? std::exp(a.beta * (std::sqrt(z) - 1.0)) : 0.0;
				acc += wt * phi * std::cos(2.0 * M_PI * n * t / a.nf[e]);
			}
			ph[n + K[e]] = 2.0 * acc;
		}
		double *dp = nullptr;
		if (int rc = nu_alloc(h, &dp, ph.size()))
			return rc;
		CC_CUDA(cudaMemcpy(dp, ph.data(), ph.size() * sizeof(double), cudaMemcpyHostToDevice));
		a.phihat[e] = dp;
	}
	int32_t *d_um = nullptr;
	double *d_uV = nullptr;
	unsigned long long *gi = nullptr;
	double *gr = nullptr, *epart = nullptr, *gim = nullptr;
	double2 *spec = nullptr, *coef = nullptr, *rho_u = nullptr, *u_u = nullptr;
	const int64_t nspec = ngrid / a.nf[d - 1] * (a.nf[d - 1] / 2 + 1);
	const int nblk = std::max(1, (U + 255) / 256);
	int rc;
	if ((rc = nu_alloc(h, &d_um, (size_t)std::max(U, 1) * d)) || (rc = nu_alloc(h, &d_uV, (size_t)std::max(U, 1))) ||
	    (rc = nu_alloc(h, &gi, (size_t)ngrid)) || (rc = nu_alloc(h, &gr, (size_t)ngrid)) ||
	    (rc = nu_alloc(h, &spec, (size_t)nspec)) || (rc = nu_alloc(h, &coef, (size_t)nspec * d)) ||
	    (rc = nu_alloc(h, &gim, (size_t)ngrid * d)) ||
	    (rc = nu_alloc(h, &rho_u, (size_t)std::max(U, 1))) || (rc = nu_alloc(h, &u_u, (size_t)std::max(U, 1))) ||
	    (rc = nu_alloc(h, &epart, (size_t)nblk)) || (rc = nu_alloc(h, &h->d_nu_mode_u, mode_u.size())))
		return rc;
	if (U > 0) {
		CC_CUDA(cudaMemcpy(d_um, um.data(), um.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
		CC_CUDA(cudaMemcpy(d_uV, uV.data(), uV.size() * sizeof(double), cudaMemcpyHostToDevice));
	}
	CC_CUDA(cudaMemcpy(h->d_nu_mode_u, mode_u.data(), mode_u.size() * sizeof(int), cudaMemcpyHostToDevice));
	a.U = U;
	a.umodes = d_um;
	a.uV = d_uV;
	a.gi = gi;
	a.gr = gr;
	a.spec = spec;
	a.coef = coef;
	a.gim = gim;
	a.rho_u = rho_u;
	a.u_u = u_u;
	a.epart = epart;
	int dims[3] = {a.nf[0], a.nf[1], a.nf[2]};
	if (cufftPlanMany(&h->nu_p1, d, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_D2Z, 1) != CUFFT_SUCCESS)
		return fail(CC_ERR_CUDA, "cufftPlanMany (D2Z) failed");
	h->nu_p1_ok = true;
	if (cufftPlanMany(&h->nu_p2, d, dims, nullptr, 1, (int)nspec, nullptr, 1, (int)ngrid, CUFFT_Z2D, d) !=
	    CUFFT_SUCCESS)
		return fail(CC_ERR_CUDA, "cufftPlanMany (Z2D) failed");
	h->nu_p2_ok = true;
	h->nu_ngrid = ngrid;
	h->nu_nspec = nspec;
	h->nu_rho_blocks = nblk;
	h->nu_ready = true;
	return CC_OK;
}

template <int D>
int run_nufft_t(cc_handle *h, int64_t N, const double *d_frac, double *d_E, double *d_F, double *d_gfrac,
                bool want_rho_mode, cudaStream_t st)
{
	cc::NufftDev a = h->nu;
	a.skip = h->d_skip;
	const int64_t ngrid = h->nu_ngrid;
	CC_CUDA(cudaMemsetAsync(a.gi, 0, sizeof(unsigned long long) * ngrid, st));
	if (N > 0) {
		cc::nufft_spread_kernel<D><<<(unsigned)((N + cc::kNufftPerBlock - 1) / cc::kNufftPerBlock), cc::kNufftThreads,
		                             0, st>>>(a, d_frac, (int)N);
		CC_CUDA(cudaGetLastError());
	}
	cc::nufft_fix_to_double_kernel<<<(unsigned)((ngrid + 255) / 256), 256, 0, st>>>(a, ngrid);
	CC_CUDA(cudaGetLastError());
	if (cufftSetStream(h->nu_p1, st) != CUFFT_SUCCESS ||
	    cufftExecD2Z(h->nu_p1, a.gr, reinterpret_cast<cufftDoubleComplex *>(const_cast<double2 *>(a.spec))) !=
	        CUFFT_SUCCESS)
		return fail(CC_ERR_CUDA, "cufftExecD2Z failed");
	cc::nufft_rho_kernel<D><<<h->nu_rho_blocks, 256, 0, st>>>(a, h->rho_offset);
	CC_CUDA(cudaGetLastError());
	cc::nufft_energy_kernel<<<1, 32, 0, st>>>(a, h->nu_rho_blocks, 1.0 / h->volume, h->shift, d_E);
	CC_CUDA(cudaGetLastError());
	const int M = (int)h->V.size();
	if (want_rho_mode && M > 0) {
		cc::nufft_gather_rho_kernel<<<(M + 255) / 256, 256, 0, st>>>(a.rho_u, h->d_nu_mode_u, M, h->main.rho_mode);
		CC_CUDA(cudaGetLastError());
	}
	if (!(d_F || d_gfrac) || N == 0)
		return CC_OK;
	CC_CUDA(cudaMemsetAsync(a.coef, 0, sizeof(double2) * h->nu_nspec * D, st));
	cc::nufft_coef_kernel<D><<<h->nu_rho_blocks, 256, 0, st>>>(a, h->nu_nspec);
	CC_CUDA(cudaGetLastError());
	// complex-to-real (the input spectra are overwritten; they are rebuilt every evaluation)
	if (cufftSetStream(h->nu_p2, st) != CUFFT_SUCCESS ||
	    cufftExecZ2D(h->nu_p2, reinterpret_cast<cufftDoubleComplex *>(a.coef), a.gim) != CUFFT_SUCCESS)
		return fail(CC_ERR_CUDA, "cufftExecZ2D failed");
	cc::NufftOut o;
	for (int i = 0; i < 9; i++)
		o.recip[i] = h->recip[i];
	o.fscale = 2.0 / h->volume;
	o.F_out = d_F;
	o.gfrac_out = d_gfrac;
	cc::nufft_interp_kernel<D><<<(unsigned)((N + cc::kNufftPerBlock - 1) / cc::kNufftPerBlock), cc::kNufftThreads, 0,
	                             st>>>(a, d_frac, (int)N, ngrid, o);
	CC_CUDA(cudaGetLastError());
	return CC_OK;
}

int run_nufft(cc_handle *h, int64_t N, const double *d_frac, double *d_E, double *d_F, double *d_gfrac,
              bool want_rho_mode, cudaStream_t st)
{
	if (int rc = nufft_setup(h))
		return rc;
	switch (h->d) {
	case 1: return run_nufft_t<1>(h, N, d_frac, d_E, d_F, d_gfrac, want_rho_mode, st);
	case 2: return run_nufft_t<2>(h, N, d_frac, d_E, d_F, d_gfrac, want_rho_mode, st);
	default: return run_nufft_t<3>(h, N, d_frac, d_E, d_F, d_gfrac, want_rho_mode, st);
	}
}

int check_handle(const cc_handle *h)
{
	if (!h)
		return fail(CC_ERR_ARG, "null handle");
	return CC_OK;
}

int device_ok()
{
	int n = 0;
	if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0)
		return fail(CC_ERR_NOGPU, "no CUDA device is visible; libccgpu has no CPU path");
	return CC_OK;
}

int create_common(int d, const double *basis, int64_t M, const int32_t *modes, const double *V, double shift,
                  cc_handle **out)
{
	if (!out)
		return fail(CC_ERR_ARG, "out is null");
	*out = nullptr;
	if (d < 1 || d > 3)
		return fail(CC_ERR_ARG, "dimension must be 1, 2 or 3");
	if (!basis || M < 0 || (M > 0 && (!modes || !V)))
		return fail(CC_ERR_ARG, "null basis/modes/V or negative M");
	if (M > (int64_t)1 << 30)
		return fail(CC_ERR_ARG, "too many constraints");
	int rc = device_ok();
	if (rc)
		return rc;
	cc_handle *h = new cc_handle();
	h->d = d;
	for (int i = 0; i < d * d; i++)
		h->basis[i] = basis[i];
	if (!cc::cell_geometry(d, h->basis, &h->volume, h->recip)) {
		delete h;
		return fail(CC_ERR_ARG, "degenerate cell basis");
	}
	h->shift = shift;
	h->modes.assign(modes, modes + M * d);
	h->V.assign(V, V + M);
	for (int64_t m = 0; m < M; m++)
		if (!std::isfinite(V[m])) {
			delete h;
			return fail(CC_ERR_ARG, "non-finite weight V");
		}
	cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
	if (e != cudaSuccess) {
		delete h;
		return fail(CC_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
	}
	cc::Plan plan = cc::build_plan(d, M, modes, V, 8);
	if ((rc = upload_kset(h->main, plan)) || (rc = dev_alloc(&h->d_E, 2))) {
		cc_destroy(h);
		return rc;
	}
	*out = h;
	return CC_OK;
}

cudaEvent_t next_event(cc_handle *h)
{
	if (h->ev_used == h->ev.size()) {
		cudaEvent_t e;
		if (cudaEventCreate(&e) != cudaSuccess)
			return nullptr;
		h->ev.push_back(e);
	}
	return h->ev[h->ev_used++];
}

// CC_PATH_AUTO: the NUFFT path when its estimated time, with a 20 % margin, is below the direct path's. Direct:
// N x slots at 700 G pairs/s; NUFFT: 3.9e-12 s per particle and kernel point (spread + interpolation, W^d points),
// 7.2e-12 s per fine-grid point and transform, 80 us of launches and transforms at small sizes. Fitted to B200
// timings of single evaluations (L2 flushed, FP64 energy + forces): 2D N=1e5 M=40002 0.165 ms NUFFT against 5.1 ms
// direct; 2D N=2e4 M=8002 0.083 against 0.26; 3D N=2e4 M=12055 0.31 against 0.44; 3D N=1e5 M=60020 1.21 against
// 9.3; 3D N=2000 M=2724 0.13 against 0.034.
bool nufft_preferred(cc_handle *h, int64_t N)
{
	if (h->main.plan.nslot == 0 || N < 1024 || h->d_slotS0)
		return false;
	const int d = h->d;
	if (h->nu_grid_est < 0) {
		double grid = 1.0;
		for (int e = 0; e < d; e++) {
			int K = 0;
			for (size_t m = e; m < h->modes.size(); m += d)
				K = std::max(K, std::abs(h->modes[m]));
			grid *= fft_size(std::max(2 * (2 * K + 1), 2 * cc::kNufftW));
		}
		h->nu_grid_est = grid;
	}
	const double grid = h->nu_grid_est;
	double w = 1.0;
	for (int e = 0; e < d; e++)
		w *= cc::kNufftW;
	if (grid > (double)((int64_t)1 << 28))
		return false;
	const double direct = (double)N * (double)h->main.plan.real_segs * h->main.plan.L / 7e11;
	const double nufft = 3.9e-12 * (double)N * w + 7.2e-12 * grid * (1 + d) + 8e-5;
	return 1.2 * nufft < direct;
}

// ShiftedCCPotential_S2_MultiConfig (potential/CollectiveCoordinatePotential.h:1756-1870): particles
// [c Np, (c + 1) Np) form sub-configuration c; per c a rho pass into its own rho / u slab, one combination over the
// sub-configurations (the mean S(k), the energy and u_c), then per c a force pass with scale 4 / Np / nsub. FP64.
int eval_multiconfig(cc_handle *h, int64_t N, const double *d_frac, double *d_E, double *d_F, double *d_gfrac,
                     cudaStream_t st)
{
	const int nsub = h->nsub, d = h->d;
	const int64_t Np = N / nsub;
	DevKSet &k = h->main;
	const cc::Plan &p = k.plan;
	if (p.nslot == 0) {
		cc::cc_set_scalar_kernel<<<1, 1, 0, st>>>(d_E, h->shift);
		CC_CUDA(cudaGetLastError());
		if (N > 0 && d_F)
			CC_CUDA(cudaMemsetAsync(d_F, 0, sizeof(double) * N * d, st));
		if (N > 0 && d_gfrac)
			CC_CUDA(cudaMemsetAsync(d_gfrac, 0, sizeof(double) * N * d, st));
		return CC_OK;
	}
	const size_t slab = (size_t)nsub * p.nslot;
	const int nb = (p.nslot + cc::kS2mThreads - 1) / cc::kS2mThreads;
	if (int rc = grow(&h->d_msub, h->msub_cap, 2 * slab))
		return rc;
	if (int rc = grow(&h->d_mpart, h->mpart_cap, (size_t)nb + 1))
		return rc;
	double2 *rho = h->d_msub, *u = h->d_msub + slab;
	const Launch l = choose_launch(p, Np, false);
	double *copy = h->rho_copy;   // graph path: the rho passes store the positions for the force passes
	for (int c = 0; c < nsub; c++) {
		h->rho_copy = copy ? copy + (size_t)c * Np * d : nullptr;
		const int rc = run_rho(h, k, Np, d_frac + (size_t)c * Np * d, h->d_mpart + nb, false, false, l, st, nullptr,
		                       false, rho + (size_t)c * p.nslot, u + (size_t)c * p.nslot);
		if (rc) {
			h->rho_copy = copy;
			return rc;
		}
	}
	h->rho_copy = copy;
	if (copy)
		d_frac = copy;
	cc::cc_s2multi_kernel<<<nb, cc::kS2mThreads, 0, st>>>(rho, u, p.nslot, nsub, k.slotV, h->d_slotS0,
	                                                       (double)Np * (double)nsub, h->d_mpart);
	CC_CUDA(cudaGetLastError());
	cc::cc_mc_sum_kernel<<<1, 32, 0, st>>>(h->d_mpart, nb, 1.0, d_E, h->shift);
	CC_CUDA(cudaGetLastError());
	if (!(d_F || d_gfrac) || Np == 0)
		return CC_OK;
	const double fscale = 4.0 / (double)Np / (double)nsub;
	for (int c = 0; c < nsub; c++) {
		const size_t off = (size_t)c * Np * d;
		if (int rc = run_force(h, Np, d_frac + off, d_F ? d_F + off : nullptr, d_gfrac ? d_gfrac + off : nullptr,
		                       false, l, st, nullptr, u + (size_t)c * p.nslot, fscale))
			return rc;
	}
	return CC_OK;
}

int eval_device(cc_handle *h, int64_t N, const double *d_frac, double *d_E, double *d_F, double *d_gfrac,
                bool want_rho_mode, int precision, cudaStream_t st)
{
	if (h->nsub > 1) {
		if (N % h->nsub)
			return fail(CC_ERR_ARG, "the particle count is not a multiple of the number of sub-configurations");
		if (want_rho_mode)
			return fail(CC_ERR_ARG, "rho per constraint is per sub-configuration in the multi-configuration form");
		return eval_multiconfig(h, N, d_frac, d_E, d_F, d_gfrac, st);
	}
	const bool mixed = precision == CC_PREC_MIXED && !h->d_slotS0;   // the S2 form evaluates in FP64
	const Launch l = choose_launch(h->main.plan, N, mixed);
	cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr, e3 = nullptr;
	if (h->timing && h->ev_used + 4 <= 4 * 100000) {
		e0 = next_event(h);
		e1 = next_event(h);
		e2 = next_event(h);
		e3 = next_event(h);
		if (!(e0 && e1 && e2 && e3))
			return fail(CC_ERR_CUDA, "cudaEventCreate failed");
		CC_CUDA(record_timing(e0, st));
	}
	if ((h->use_nufft || (h->auto_path && nufft_preferred(h, N))) && h->main.plan.nslot > 0) {
		// non-uniform FFT path (FP64 whatever the precision): reported as the force interval
		if (e1)
			CC_CUDA(record_timing(e1, st));
		if (e2)
			CC_CUDA(record_timing(e2, st));
		int rc = run_nufft(h, N, d_frac, d_E, d_F, d_gfrac, want_rho_mode, st);
		if (e3)
			CC_CUDA(record_timing(e3, st));
		return rc;
	}
	// with forces (and a constraint set and particles), the force kernel finishes the energy
	const bool e_in_force = (d_F || d_gfrac) && N > 0 && h->main.plan.nslot > 0;
	int rc = run_rho(h, h->main, N, d_frac, d_E, want_rho_mode, mixed, l, st, e1, e_in_force);
	if (h->rho_copy)   // the rho kernel has stored the positions in device memory for the force kernel
		d_frac = h->rho_copy;
	if (rc)
		return rc;
	if (e2)
		CC_CUDA(record_timing(e2, st));
	if (d_F || d_gfrac)
		rc = run_force(h, N, d_frac, d_F, d_gfrac, mixed, l, st, e_in_force ? d_E : nullptr);
	if (e3)
		CC_CUDA(record_timing(e3, st));
	return rc;
}

// cc_energy_grad as one CUDA graph: the rho / reduce / force kernels (the rho kernel reading the staged positions from
// mapped pinned memory) writing E and F into mapped pinned memory. A key is captured on its second consecutive use
// with no allocation in between (the first, direct evaluation makes every allocation the launch needs); *done tells
// whether the graph ran.
int launch_eval_graph(cc_handle *h, int64_t N, int precision, int forces, bool *done)
{
	*done = false;
	const unsigned long long gen = g_alloc_gen.load();
	for (size_t i = 0; i < h->graphs.size(); i++) {
		cc_handle::EvalGraph &g = h->graphs[i];
		if (g.N != N || g.precision != precision || g.forces != forces)
			continue;
		if (g.gen != gen) {
			cudaGraphExecDestroy(g.exec);
			h->graphs.erase(h->graphs.begin() + i);
			break;
		}
		CC_CUDA(cudaGraphLaunch(g.exec, h->stream));
		CC_CUDA(cudaEventRecord(h->ev_in, h->stream));
		h->in_pending = true;
		h->upload_pending = false;
		*done = true;
		return CC_OK;
	}
	if (!(h->last_N == N && h->last_precision == precision && h->last_forces == forces && h->last_gen == gen))
		return CC_OK;
	if (h->in_pending) {   // the staging buffer is read by the graph's first node
		CC_CUDA(cudaEventSynchronize(h->ev_in));
		h->in_pending = false;
	}
	cudaGraph_t graph = nullptr;
	CC_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
	// Positions from the mapped staging buffer: on the three-kernel path the rho kernel reads them there and stores
	// them into d_frac for the force kernel; on the NUFFT path a kernel copies them first. Either way the first
	// kernel of the evaluation reads host memory, and no copy node sits in front of the programmatic dependent launches.
	const bool nufft = h->use_nufft || (h->auto_path && nufft_preferred(h, N));
	cudaError_t ce = cudaSuccess;
	int rc;
	if (nufft) {
		const int64_t nv = N * h->d;
		cc::cc_upload_kernel<<<(unsigned)((nv + 255) / 256), 256, 0, h->stream>>>(h->d_in, h->d_frac, nv);
		ce = cudaGetLastError();
		rc = ce == cudaSuccess ? eval_device(h, N, h->d_frac, h->d_pin, forces ? h->d_pin + 2 : nullptr, nullptr, false,
		                                     precision, h->stream)
		                       : CC_ERR_CUDA;
	} else {
		h->rho_copy = h->d_frac;
		rc = eval_device(h, N, h->d_in, h->d_pin, forces ? h->d_pin + 2 : nullptr, nullptr, false, precision,
		                 h->stream);
		h->rho_copy = nullptr;
	}
	const cudaError_t ee = cudaStreamEndCapture(h->stream, &graph);
	if (rc != CC_OK || ce != cudaSuccess || ee != cudaSuccess || g_alloc_gen.load() != gen) {
		if (graph)
			cudaGraphDestroy(graph);
		cudaGetLastError();
		return CC_OK;   // not capturable now: the caller evaluates directly
	}
	cudaGraphExec_t exec = nullptr;
	const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
	cudaGraphDestroy(graph);
	if (ie != cudaSuccess) {
		cudaGetLastError();
		return CC_OK;
	}
	if (h->graphs.size() >= 4) {
		cudaGraphExecDestroy(h->graphs.front().exec);
		h->graphs.erase(h->graphs.begin());
	}
	h->graphs.push_back({N, precision, forces, gen, exec});
	CC_CUDA(cudaGraphLaunch(exec, h->stream));
	CC_CUDA(cudaEventRecord(h->ev_in, h->stream));
	h->in_pending = true;
	h->upload_pending = false;
	*done = true;
	return CC_OK;
}

template <typename T> __global__ void fma_probe_kernel(T *out, int iters, T a, T b)
{
	T x[8];
#pragma unroll
	for (int k = 0; k < 8; k++)
		x[k] = (T)(threadIdx.x + k) * (T)1e-3;
	for (int i = 0; i < iters; i++) {
#pragma unroll
		for (int k = 0; k < 8; k++)
			x[k] = fma(x[k], a, b);
	}
	T s = 0;
#pragma unroll
	for (int k = 0; k < 8; k++)
		s += x[k];
	if (s == (T)-1.2345)
		out[0] = s;
}

template <typename T> int probe_peak(double *tflops)
{
	T *out = nullptr;
	if (int rc = dev_alloc(&out, 1))
		return rc;
	const int blocks = sm_count() * 8, threads = 256, iters = 1 << 14;
	cudaEvent_t a, b;
	CC_CUDA(cudaEventCreate(&a));
	CC_CUDA(cudaEventCreate(&b));
	float best = 1e30f;
	for (int rep = 0; rep < 6; rep++) {
		CC_CUDA(cudaEventRecord(a));
		fma_probe_kernel<T><<<blocks, threads>>>(out, iters, (T)0.9999999, (T)1e-7);
		CC_CUDA(cudaEventRecord(b));
		CC_CUDA(cudaEventSynchronize(b));
		float ms = 0;
		CC_CUDA(cudaEventElapsedTime(&ms, a, b));
		if (rep > 0)
			best = std::min(best, ms);
	}
	cudaEventDestroy(a);
	cudaEventDestroy(b);
	cudaFree(out);
	*tflops = 2.0 * 8.0 * iters * (double)blocks * threads / (best * 1e-3) / 1e12;
	return CC_OK;
}

}  // namespace

// The handle operations the library's other translation units use (cc_internal.h).
int cci::handle_check(const cc_handle *h) { return check_handle(h); }
int cci::handle_reserve(cc_handle *h, int64_t N) { return ensure_particles(h, N); }
int cci::handle_eval(cc_handle *h, int64_t N, const double *d_frac, double *d_E, double *d_F, double *d_gfrac,
                     bool want_rho_mode, int precision, cudaStream_t st)
{
	return eval_device(h, N, d_frac, d_E, d_F, d_gfrac, want_rho_mode, precision, st);
}

// ===============================================================================================================
// C ABI
// ===============================================================================================================
extern "C" {

const char *cc_last_error(void) { return g_err.c_str(); }

int cc_device_available(void)
{
	int n = 0;
	return (cudaGetDeviceCount(&n) == cudaSuccess && n > 0) ? 1 : 0;
}

int cc_create(int d, const double *basis, int64_t M, const int32_t *modes, const double *V, double shift,
              cc_handle **out)
{
	return create_common(d, basis, M, modes, V, shift, out);
}

int cc_create_cartesian(int d, const double *basis, int64_t M, const double *k, const double *V, double shift,
                        cc_handle **out)
{
	if (d < 1 || d > 3 || !basis || M < 0 || (M > 0 && !k))
		return fail(CC_ERR_ARG, "invalid arguments");
	std::vector<int32_t> modes((size_t)M * d);
	if (!cc::cartesian_to_modes(d, basis, M, k, modes.data()))
		return fail(CC_ERR_NONLATTICE, "a Cartesian k is not on the reciprocal lattice of the cell");
	return create_common(d, basis, M, modes.data(), V, shift, out);
}

int cc_create_s2(int d, const double *basis, int64_t M, const int32_t *modes, const double *V, const double *S0,
                 double shift, cc_handle **out)
{
	if (!out)
		return fail(CC_ERR_ARG, "out is null");
	*out = nullptr;
	if (M > 0 && !S0)
		return fail(CC_ERR_ARG, "null S0");
	for (int64_t m = 0; m < M; m++)
		if (!std::isfinite(S0[m]))
			return fail(CC_ERR_ARG, "non-finite target S0");
	cc_handle *h = nullptr;
	if (int rc = create_common(d, basis, M, modes, V, shift, &h))
		return rc;
	const cc::Plan &p = h->main.plan;
	// A repeated mode shares one slot: over its copies sum_m V_m (S - S0_m)^2 = W (S - T)^2 + C with W = sum V_m (the
	// slot's weight), T = sum V_m S0_m / W and C = sum V_m S0_m^2 - W T^2, which joins the shift. Copies whose weights
	// sum to zero (but are not all zero) have no such form.
	std::vector<double> slotS0((size_t)p.nslot, 0.0), vs0((size_t)p.nslot, 0.0), vs02((size_t)p.nslot, 0.0);
	std::vector<int> copies((size_t)p.nslot, 0);
	std::vector<char> nonzero((size_t)p.nslot, 0);
	for (int64_t m = 0; m < M; m++) {
		const size_t q = (size_t)p.mode_slot[(size_t)m];
		slotS0[q] = S0[m];
		vs0[q] += V[m] * S0[m];
		vs02[q] += V[m] * S0[m] * S0[m];
		copies[q]++;
		nonzero[q] |= V[m] != 0.0;
	}
	double extra = 0.0;
	for (size_t q = 0; q < (size_t)p.nslot; q++) {
		if (copies[q] < 2)
			continue;
		const double W = p.slotV[q];
		if (W == 0.0) {
			if (nonzero[q]) {
				cc_destroy(h);
				return fail(CC_ERR_ARG, "repeated S2 modes whose weights sum to zero");
			}
			slotS0[q] = 0.0;
			continue;
		}
		slotS0[q] = vs0[q] / W;
		extra += vs02[q] - W * slotS0[q] * slotS0[q];
	}
	h->shift += extra;
	if (int rc = upload(&h->d_slotS0, slotS0)) {
		cc_destroy(h);
		return rc;
	}
	*out = h;
	return CC_OK;
}

int cc_create_s2_multiconfig(int d, const double *basis, int64_t M, const int32_t *modes, const double *V,
                             const double *S0, double shift, int nsub, cc_handle **out)
{
	if (nsub < 1)
		return fail(CC_ERR_ARG, "the number of sub-configurations must be positive");
	if (int rc = cc_create_s2(d, basis, M, modes, V, S0, shift, out))
		return rc;
	(*out)->nsub = nsub;
	return CC_OK;
}

int cc_set_subconfigurations(cc_handle *h, int nsub)
{
	if (int rc = check_handle(h))
		return rc;
	if (nsub < 1 || (nsub > 1 && !h->d_slotS0 && !h->V.empty()))
		return fail(CC_ERR_ARG, "sub-configurations belong to an S2 handle; their count must be positive");
	if (h->N > 0 && h->N % nsub)
		return fail(CC_ERR_ARG, "the particle count is not a multiple of the number of sub-configurations");
	h->nsub = nsub;
	g_alloc_gen++;   // captured evaluations hold the old form
	return CC_OK;
}

int cc_create_s2_cartesian(int d, const double *basis, int64_t M, const double *k, const double *V, const double *S0,
                           double shift, cc_handle **out)
{
	if (d < 1 || d > 3 || !basis || M < 0 || (M > 0 && !k))
		return fail(CC_ERR_ARG, "invalid arguments");
	std::vector<int32_t> modes((size_t)M * d);
	if (!cc::cartesian_to_modes(d, basis, M, k, modes.data()))
		return fail(CC_ERR_NONLATTICE, "a Cartesian k is not on the reciprocal lattice of the cell");
	return cc_create_s2(d, basis, M, modes.data(), V, S0, shift, out);
}

int cc_destroy(cc_handle *h)
{
	if (!h)
		return CC_OK;
	if (h->stream)
		cudaStreamSynchronize(h->stream);
	if (h->sched_batch)
		cc_batch_destroy(h->sched_batch);
	h->lb.release();
	h->main.release();
	h->sk.release();
	cudaFree(h->d_frac);
	cudaFree(h->d_F);
	cudaFree(h->d_gfrac);
	cudaFree(h->d_partialG);
	cudaFree(h->d_fcounters);
	cudaFree(h->d_E);
	cudaFree(h->d_slotS0);
	cudaFree(h->d_msub);
	cudaFree(h->d_mpart);
	cudaFreeHost(h->h_pin);
	cudaFreeHost(h->h_in);
	if (h->ev_in)
		cudaEventDestroy(h->ev_in);
	cudaFree(h->d_modes);
	cudaFree(h->d_modeV);
	cudaFree(h->d_rho_trial);
	cudaFree(h->d_rho_cur);
	cudaFree(h->d_mc_part);
	for (cudaEvent_t e : h->ev)
		cudaEventDestroy(e);
	for (auto &g : h->graphs)
		cudaGraphExecDestroy(g.exec);
	if (h->nu_p1_ok)
		cufftDestroy(h->nu_p1);
	if (h->nu_p2_ok)
		cufftDestroy(h->nu_p2);
	for (void *b : h->nu_bufs)
		cudaFree(b);
	if (h->copy_stream)
		cudaStreamSynchronize(h->copy_stream);
	cudaFree(h->d_many_in);
	cudaFree(h->d_many_F);
	cudaFree(h->d_many_E);
	cudaFree(h->d_many_bad);
	for (cudaEvent_t e : h->many_ev)
		cudaEventDestroy(e);
	if (h->copy_stream)
		cudaStreamDestroy(h->copy_stream);
	if (h->stream)
		cudaStreamDestroy(h->stream);
	delete h;
	return CC_OK;
}

int cc_info(const cc_handle *h, int64_t *M, int *d, double *volume, int32_t *modes)
{
	if (int rc = check_handle(h))
		return rc;
	if (M)
		*M = (int64_t)h->V.size();
	if (d)
		*d = h->d;
	if (volume)
		*volume = h->volume;
	if (modes)
		std::memcpy(modes, h->modes.data(), h->modes.size() * sizeof(int32_t));
	return CC_OK;
}

int cc_set_rho_offset(cc_handle *h, double offset)
{
	if (int rc = check_handle(h))
		return rc;
	if (!std::isfinite(offset))
		return fail(CC_ERR_ARG, "offset must be finite");
	h->rho_offset = offset;
	h->lastF_valid = false;
	g_alloc_gen++;   // captured evaluations hold the old offset
	return CC_OK;
}

int cc_set_positions(cc_handle *h, int64_t N, const double *frac)
{
	if (int rc = check_handle(h))
		return rc;
	if (N < 0 || (N > 0 && !frac) || N > ((int64_t)1 << 31) - 64)
		return fail(CC_ERR_ARG, "invalid particle count or null positions");
	if (N % h->nsub)
		return fail(CC_ERR_ARG, "the particle count is not a multiple of the number of sub-configurations");
	if (int rc = ensure_particles(h, N))
		return rc;
	const int d = h->d;
	if (int rc = input_staging(h, (size_t)N * d))
		return rc;
	double *in = h->h_in;
	// positions already in [0,1) (the usual case) are copied as they are, in the same pass that checks them (an
	// integer flag the compiler vectorises); NaN fails both comparisons
	long bad = 0;
	const int64_t nv = N * d;
	for (int64_t i = 0; i < nv; i++) {
		const double x = frac[i];
		in[i] = x;
		bad |= (long)!(x >= 0.0) | (long)!(x < 1.0);
	}
	if (bad) {
		for (int64_t i = 0; i < N * d; i++)
			if (!wrap_unit(frac[i], in + i)) {
				h->upload_pending = false;
				h->N = -1;
				return fail(CC_ERR_ARG, "non-finite fractional coordinate");
			}
	}
	h->upload_pending = true;
	h->N = N;
	h->lastF_valid = false;
	h->mc_valid = false;
	return CC_OK;
}

int cc_energy_grad(cc_handle *h, double *E, double *F, int precision)
{
	if (int rc = check_handle(h))
		return rc;
	if (int rc = check_prec(precision))
		return rc;
	if (h->N < 0)
		return fail(CC_ERR_STATE, "positions not set");
	if (!E)
		return fail(CC_ERR_ARG, "E is null");
	const int64_t N = h->N;
	const int forces = (F && N > 0) ? 1 : 0;
	h->lastF_valid = false;
	// E and F are written by the kernels straight into the mapped pinned result buffer
	bool done = false;
	if (!h->timing && !h->d_skip && N > 0 && h->main.plan.nslot > 0)
		if (int rc = launch_eval_graph(h, N, precision, forces, &done))
			return rc;
	if (!done) {
		if (int rc = flush_upload(h))
			return rc;
		if (int rc = eval_device(h, N, h->d_frac, h->d_pin, forces ? h->d_pin + 2 : nullptr, nullptr, false,
		                         precision, h->stream))
			return rc;
		h->last_N = N;
		h->last_precision = precision;
		h->last_forces = forces;
		h->last_gen = g_alloc_gen.load();
	}
	CC_CUDA(cudaStreamSynchronize(h->stream));
	h->in_pending = false;   // ev_in was recorded on this stream: the staging buffer is free again
	*E = h->h_pin[0];
	if (F && N > 0) {
		std::memcpy(F, h->h_pin + 2, sizeof(double) * N * h->d);
		h->lastF_valid = true;
	}
	return CC_OK;
}

int cc_energy_grad_device(cc_handle *h, int64_t N, const double *d_frac, double *d_E, double *d_F, double *d_gfrac,
                          int precision, void *stream)
{
	if (int rc = check_handle(h))
		return rc;
	if (int rc = check_prec(precision))
		return rc;
	if (N < 0 || (N > 0 && !d_frac) || !d_E)
		return fail(CC_ERR_ARG, "invalid device arguments");
	if ((size_t)std::max<int64_t>(N, 1) > h->ncap)
		if (int rc = ensure_particles(h, N))
			return rc;
	cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : h->stream;
	h->early_call = h->independent;
	const int rc = eval_device(h, N, d_frac, d_E, d_F, d_gfrac, false, precision, st);
	h->early_call = false;
	return rc;
}

// Positions of cc_energy_grad_many brought into [0, 1) with cc_set_positions' operations (so the results are the
// same bitwise); a non-finite coordinate is replaced by 0, so that no kernel sees it, and reported through *bad.
static __global__ void cc_wrap_many_kernel(double *x, int64_t n, int *bad)
{
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
		const double v = x[i];
		if (v >= 0.0 && v < 1.0)
			continue;
		if (!isfinite(v)) {
			x[i] = 0.0;
			*bad = 1;
			continue;
		}
		double w = v - floor(v);
		w -= floor(w);
		x[i] = w;
	}
}

constexpr int64_t kManyChunk = 64;   // configurations per host<->device copy of cc_energy_grad_many

static int many_buffers(cc_handle *h, int64_t P, size_t total, int64_t nch)
{
	if (total > h->many_cap) {
		cudaFree(h->d_many_in);
		cudaFree(h->d_many_F);
		h->d_many_in = h->d_many_F = nullptr;
		h->many_cap = 0;
		if (int rc = dev_alloc(&h->d_many_in, total))
			return rc;
		if (int rc = dev_alloc(&h->d_many_F, total))
			return rc;
		h->many_cap = total;
	}
	if ((size_t)P > h->many_ecap) {
		cudaFree(h->d_many_E);
		h->d_many_E = nullptr;
		h->many_ecap = 0;
		if (int rc = dev_alloc(&h->d_many_E, (size_t)P))
			return rc;
		h->many_ecap = (size_t)P;
	}
	if (!h->d_many_bad)
		if (int rc = dev_alloc(&h->d_many_bad, 1))
			return rc;
	if (!h->copy_stream)
		CC_CUDA(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
	while ((int64_t)h->many_ev.size() < 2 * nch) {
		cudaEvent_t e = nullptr;
		CC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
		h->many_ev.push_back(e);
	}
	return CC_OK;
}

int cc_energy_grad_many(cc_handle *h, int64_t P, int64_t N, const double *frac, double *E, double *F, int precision)
{
	if (int rc = check_handle(h))
		return rc;
	if (int rc = check_prec(precision))
		return rc;
	if (P < 0 || N < 0 || N > ((int64_t)1 << 31) - 64 || (P > 0 && (!E || (N > 0 && !frac))))
		return fail(CC_ERR_ARG, "invalid configuration count, particle count or buffers");
	if (N % h->nsub)
		return fail(CC_ERR_ARG, "the particle count is not a multiple of the number of sub-configurations");
	if (P == 0)
		return CC_OK;
	const size_t per = (size_t)N * h->d, total = (size_t)P * per;
	const int64_t nch = (P + kManyChunk - 1) / kManyChunk;
	if ((size_t)std::max<int64_t>(N, 1) > h->ncap)
		if (int rc = ensure_particles(h, N))
			return rc;
	if (int rc = many_buffers(h, P, total, nch))
		return rc;
	cudaStream_t st = h->stream, cp = h->copy_stream;
	CC_CUDA(cudaMemsetAsync(h->d_many_bad, 0, sizeof(int), st));
	// the copy stream starts after the handle's earlier work (which may still read these buffers)
	CC_CUDA(cudaEventRecord(h->many_ev[1], st));
	CC_CUDA(cudaStreamWaitEvent(cp, h->many_ev[1], 0));
	int rc = CC_OK;
	for (int64_t c = 0; c < nch && rc == CC_OK; c++) {
		const int64_t p0 = c * kManyChunk, p1 = std::min(P, p0 + kManyChunk);
		const size_t n = (size_t)(p1 - p0) * per;
		cudaEvent_t in = h->many_ev[2 * c], done = h->many_ev[2 * c + 1];
		if (n)
			CC_CUDA(cudaMemcpyAsync(h->d_many_in + p0 * per, frac + p0 * per, n * sizeof(double), cudaMemcpyHostToDevice,
			                        cp));
		CC_CUDA(cudaEventRecord(in, cp));
		CC_CUDA(cudaStreamWaitEvent(st, in, 0));
		if (n) {
			const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 4 * 148);
			cc_wrap_many_kernel<<<blocks, 256, 0, st>>>(h->d_many_in + p0 * per, (int64_t)n, h->d_many_bad);
			CC_CUDA(cudaGetLastError());
		}
		for (int64_t p = p0; p < p1 && rc == CC_OK; p++) {
			// after the chunk's first evaluation (which waits for the wrap kernel) the positions are complete before
			// the kernel just before each rho kernel: the rho kernels may overlap the previous evaluation
			h->early_call = p > p0;
			rc = eval_device(h, N, h->d_many_in + p * per, h->d_many_E + p, (F && N > 0) ? h->d_many_F + p * per : nullptr,
			                 nullptr, false, precision, st);
			h->early_call = false;
		}
		CC_CUDA(cudaEventRecord(done, st));
	}
	// Results go out after every evaluation is enqueued: a copy into pageable memory returns only when it is done,
	// and must not hold back the enqueueing of later chunks.
	for (int64_t c = 0; c < nch && rc == CC_OK; c++) {
		const int64_t p0 = c * kManyChunk, p1 = std::min(P, p0 + kManyChunk);
		const size_t n = (size_t)(p1 - p0) * per;
		CC_CUDA(cudaStreamWaitEvent(cp, h->many_ev[2 * c + 1], 0));
		if (F && n)
			CC_CUDA(cudaMemcpyAsync(F + p0 * per, h->d_many_F + p0 * per, n * sizeof(double), cudaMemcpyDeviceToHost, cp));
	}
	int bad = 0;
	if (rc == CC_OK) {
		CC_CUDA(cudaMemcpyAsync(E, h->d_many_E, (size_t)P * sizeof(double), cudaMemcpyDeviceToHost, cp));
		CC_CUDA(cudaMemcpyAsync(&bad, h->d_many_bad, sizeof(int), cudaMemcpyDeviceToHost, cp));
	}
	CC_CUDA(cudaStreamSynchronize(cp));
	CC_CUDA(cudaStreamSynchronize(st));
	if (rc != CC_OK)
		return rc;
	if (bad)
		return fail(CC_ERR_ARG, "non-finite fractional coordinate");
	return CC_OK;
}

int cc_rho(cc_handle *h, double *re, double *im, int precision)
{
	if (int rc = check_handle(h))
		return rc;
	if (int rc = check_prec(precision))
		return rc;
	if (h->N < 0)
		return fail(CC_ERR_STATE, "positions not set");
	if (h->nsub > 1)
		return fail(CC_ERR_ARG, "rho per constraint is per sub-configuration in the multi-configuration form");
	if (int rc = flush_upload(h))
		return rc;
	const int64_t N = h->N;
	const size_t M = h->V.size();
	if ((h->use_nufft || (h->auto_path && nufft_preferred(h, N))) && h->main.plan.nslot > 0) {
		if (int rc = run_nufft(h, N, h->d_frac, h->d_E, nullptr, nullptr, true, h->stream))
			return rc;
	} else {
		const Launch l = choose_launch(h->main.plan, N, precision == CC_PREC_MIXED);
		if (int rc = run_rho(h, h->main, N, h->d_frac, h->d_E, true, precision == CC_PREC_MIXED, l, h->stream))
			return rc;
	}
	if (M == 0)
		return CC_OK;
	std::vector<double2> tmp(M);
	CC_CUDA(cudaMemcpyAsync(tmp.data(), h->main.rho_mode, sizeof(double2) * M, cudaMemcpyDeviceToHost, h->stream));
	CC_CUDA(cudaStreamSynchronize(h->stream));
	for (size_t m = 0; m < M; m++) {
		if (re)
			re[m] = tmp[m].x;
		if (im)
			im[m] = tmp[m].y;
	}
	return CC_OK;
}

int cc_force_one(cc_handle *h, int64_t i, double *f)
{
	if (int rc = check_handle(h))
		return rc;
	if (h->N < 0)
		return fail(CC_ERR_STATE, "positions not set");
	if (i < 0 || i >= h->N || !f)
		return fail(CC_ERR_ARG, "particle index out of range");
	if (!h->lastF_valid) {
		std::vector<double> F((size_t)h->N * h->d);
		double E;
		if (int rc = cc_energy_grad(h, &E, F.data(), CC_PREC_FP64))
			return rc;
	}
	for (int e = 0; e < h->d; e++)
		f[e] = h->h_pin[2 + (size_t)i * h->d + e];
	return CC_OK;
}

int cc_structure_factor(cc_handle *h, int64_t K, const int32_t *modes, double *S, int precision)
{
	if (int rc = check_handle(h))
		return rc;
	if (int rc = check_prec(precision))
		return rc;
	if (h->N < 0)
		return fail(CC_ERR_STATE, "positions not set");
	if (K < 0 || (K > 0 && (!modes || !S)))
		return fail(CC_ERR_ARG, "invalid k list");
	if (K == 0)
		return CC_OK;
	const int64_t N = h->N;
	if (N == 0) {
		for (int64_t q = 0; q < K; q++)
			S[q] = std::nan("");
		return CC_OK;
	}
	std::vector<int32_t> key(modes, modes + K * h->d);
	if (key != h->sk_modes || h->sk.segs == nullptr) {
		std::vector<double> ones((size_t)K, 1.0);
		cc::Plan plan = cc::build_plan(h->d, K, modes, ones.data(), 8);
		if (int rc = upload_kset(h->sk, plan))
			return rc;
		h->sk_modes = key;
	}
	if (int rc = flush_upload(h))
		return rc;
	const Launch l = choose_launch(h->sk.plan, N, precision == CC_PREC_MIXED);
	const double save_off = h->rho_offset;
	h->rho_offset = 0.0;   // S(k) of the particles themselves (StructureFactor has no fixed-particle offset)
	int rc = run_rho(h, h->sk, N, h->d_frac, h->d_E + 1, true, precision == CC_PREC_MIXED, l, h->stream);
	h->rho_offset = save_off;
	if (rc)
		return rc;
	std::vector<double2> tmp((size_t)K);
	CC_CUDA(cudaMemcpyAsync(tmp.data(), h->sk.rho_mode, sizeof(double2) * K, cudaMemcpyDeviceToHost, h->stream));
	CC_CUDA(cudaStreamSynchronize(h->stream));
	for (int64_t q = 0; q < K; q++)
		S[q] = (tmp[q].x * tmp[q].x + tmp[q].y * tmp[q].y) / (double)N;
	return CC_OK;
}

int cc_objective(cc_handle *h, int64_t N, const double *x, double rescale, double *f, double *grad, int precision)
{
	if (int rc = check_handle(h))
		return rc;
	if (!x || !f || N < 0 || !(rescale != 0.0))
		return fail(CC_ERR_ARG, "invalid objective arguments");
	const int d = h->d;
	// A NaN first variable is the reference's NotANumberFound (StructureOptimization.cpp:460-461), which its Objective
	// does not catch: a status of its own, so a caller can stop its optimiser as the reference's does.
	if (N > 0 && x[0] != x[0])
		return fail(CC_ERR_NAN, "NotANumberFound: the first variable is NaN");
	if (int rc = ensure_particles(h, N))
		return rc;
	if (int rc = input_staging(h, (size_t)N * d))
		return rc;
	for (int64_t i = 0; i < N * d; i++)
		if (!std::isfinite(x[i]) || !wrap_unit(x[i] / rescale, h->h_in + i))
			return fail(CC_ERR_ARG, "non-finite variable");
	if (int rc = upload_staged(h, (size_t)N * d))
		return rc;
	h->N = N;
	h->lastF_valid = false;
	if (int rc = eval_device(h, N, h->d_frac, h->d_E, nullptr, grad ? h->d_gfrac : nullptr, false, precision,
	                         h->stream))
		return rc;
	CC_CUDA(cudaMemcpyAsync(h->h_pin, h->d_E, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
	if (grad && N > 0)
		CC_CUDA(cudaMemcpyAsync(h->h_pin + 2, h->d_gfrac, sizeof(double) * N * d, cudaMemcpyDeviceToHost,
		                        h->stream));
	CC_CUDA(cudaStreamSynchronize(h->stream));
	*f = h->h_pin[0];
	if (grad)
		for (int64_t i = 0; i < N * d; i++)
			grad[i] = h->h_pin[2 + i] / rescale;
	return CC_OK;
}

int cc_mc_try_move(cc_handle *h, const double *s_prev, const double *s_after, double *dE)
{
	if (int rc = check_handle(h))
		return rc;
	if (!s_prev || !s_after || !dE)
		return fail(CC_ERR_ARG, "null move arguments");
	if (h->d_slotS0)
		return fail(CC_ERR_ARG, "single-particle moves evaluate the plain collective-coordinate form only");
	if (h->N < 0)
		return fail(CC_ERR_STATE, "positions not set");
	const int M = (int)h->V.size(), d = h->d;
	for (int c = 0; c < d; c++)
		if (!std::isfinite(s_prev[c]) || !std::isfinite(s_after[c]))
			return fail(CC_ERR_ARG, "non-finite move");
	h->mc_pending = false;
	if (M == 0) {
		*dE = 0.0;
		return CC_OK;
	}
	const int nb = (M + cc::kMcThreads - 1) / cc::kMcThreads;
	if (!h->d_modes) {
		int rc;
		if ((rc = upload(&h->d_modes, h->modes)) || (rc = upload(&h->d_modeV, h->V)) ||
		    (rc = dev_alloc(&h->d_rho_trial, M)) || (rc = dev_alloc(&h->d_rho_cur, M)) ||
		    (rc = dev_alloc(&h->d_mc_part, nb + 1)))
			return rc;
	}
	if (!h->mc_valid) {
		// rho of the bound positions in mode order (FP64), as the cached RhoReal / RhoImag of the reference
		if (int rc = flush_upload(h))
			return rc;
		const Launch l = choose_launch(h->main.plan, h->N, false);
		if (int rc = run_rho(h, h->main, h->N, h->d_frac, h->d_E, true, false, l, h->stream))
			return rc;
		CC_CUDA(cudaMemcpyAsync(h->d_rho_cur, h->main.rho_mode, sizeof(double2) * M, cudaMemcpyDeviceToDevice,
		                        h->stream));
		h->mc_valid = true;
	}
	double sp[3] = {0, 0, 0}, sa[3] = {0, 0, 0};
	for (int c = 0; c < d; c++) {
		sp[c] = s_prev[c];
		sa[c] = s_after[c];
	}
	cc::cc_mc_kernel<<<nb, cc::kMcThreads, 0, h->stream>>>(h->d_modes, d, h->d_modeV, h->d_rho_cur, M, sp[0], sp[1],
	                                                        sp[2], sa[0], sa[1], sa[2], h->d_rho_trial, h->d_mc_part);
	cc::cc_mc_sum_kernel<<<1, 32, 0, h->stream>>>(h->d_mc_part, nb, 1.0 / h->volume, h->d_mc_part + nb);
	CC_CUDA(cudaGetLastError());
	CC_CUDA(cudaMemcpyAsync(h->h_pin, h->d_mc_part + nb, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
	CC_CUDA(cudaStreamSynchronize(h->stream));
	*dE = h->h_pin[0];
	h->mc_pending = true;
	return CC_OK;
}

int cc_mc_accept_move(cc_handle *h)
{
	if (int rc = check_handle(h))
		return rc;
	if (!h->mc_pending)
		return fail(CC_ERR_STATE, "no trial move to accept");
	std::swap(h->d_rho_cur, h->d_rho_trial);
	h->mc_pending = false;
	return CC_OK;
}

int cc_set_path(cc_handle *h, int path)
{
	if (int rc = check_handle(h))
		return rc;
	if (path != CC_PATH_SPLIT && path != CC_PATH_NUFFT && path != CC_PATH_AUTO)
		return fail(CC_ERR_ARG, "path must be CC_PATH_SPLIT, CC_PATH_NUFFT or CC_PATH_AUTO");
	if (h->d_slotS0 && path == CC_PATH_NUFFT)
		return fail(CC_ERR_ARG, "the NUFFT path evaluates the plain collective-coordinate form only");
	h->use_nufft = path == CC_PATH_NUFFT;
	h->auto_path = path == CC_PATH_AUTO;
	g_alloc_gen++;   // captured evaluations hold the old path
	return CC_OK;
}

int cc_check_device_error(cc_handle *h)
{
	if (int rc = check_handle(h))
		return rc;
	CC_CUDA(cudaDeviceSynchronize());
	return CC_OK;
}

int cc_set_timing(cc_handle *h, int on)
{
	if (int rc = check_handle(h))
		return rc;
	h->timing = on != 0;
	if (on)
		h->ev_used = 0;   // switching on starts a new record; switching off keeps it for cc_get_timing
	return CC_OK;
}

int cc_set_independent_positions(cc_handle *h, int on)
{
	if (int rc = check_handle(h))
		return rc;
	h->independent = on != 0;
	return CC_OK;
}

int cc_get_timing(cc_handle *h, double *rho_ms, double *reduce_ms, double *force_ms, int64_t *evals)
{
	if (int rc = check_handle(h))
		return rc;
	CC_CUDA(cudaDeviceSynchronize());
	double r = 0, q = 0, f = 0;
	for (size_t i = 0; i + 4 <= h->ev_used; i += 4) {
		float a = 0, b = 0, c = 0;
		CC_CUDA(cudaEventElapsedTime(&a, h->ev[i], h->ev[i + 1]));
		CC_CUDA(cudaEventElapsedTime(&b, h->ev[i + 1], h->ev[i + 2]));
		CC_CUDA(cudaEventElapsedTime(&c, h->ev[i + 2], h->ev[i + 3]));
		r += a;
		q += b;
		f += c;
	}
	if (rho_ms)
		*rho_ms = r;
	if (reduce_ms)
		*reduce_ms = q;
	if (force_ms)
		*force_ms = f;
	if (evals)
		*evals = (int64_t)(h->ev_used / 4);
	h->ev_used = 0;
	return CC_OK;
}

int cc_plan_info(const cc_handle *h, int64_t N, int *L, int64_t *nseg, int *nsplit, int *nksplit)
{
	if (int rc = check_handle(h))
		return rc;
	const Launch l = choose_launch(h->main.plan, N, false);
	if (L)
		*L = h->main.plan.L;
	if (nseg)
		*nseg = h->main.plan.real_segs;
	if (nsplit)
		*nsplit = l.nsplit;
	if (nksplit)
		*nksplit = (int)cc::force_splits(h->main.plan, l.want_force).count();
	return CC_OK;
}

int cc_eval_path(cc_handle *h, int64_t N, int precision, int *path)
{
	if (int rc = check_handle(h))
		return rc;
	if (int rc = check_prec(precision))
		return rc;
	if (!path || N < 0)
		return fail(CC_ERR_ARG, "invalid cc_eval_path arguments");
	if (h->nsub <= 1 && (h->use_nufft || (h->auto_path && nufft_preferred(h, N))) && h->main.plan.nslot > 0)
		*path = CC_PATH_NUFFT;
	else
		*path = CC_PATH_SPLIT;
	return CC_OK;
}

int cc_probe_fma_peak(int precision, double *tflops)
{
	if (int rc = check_prec(precision))
		return rc;
	if (!tflops)
		return fail(CC_ERR_ARG, "tflops is null");
	if (int rc = device_ok())
		return rc;
	return precision == CC_PREC_FP64 ? probe_peak<double>(tflops) : probe_peak<float>(tflops);
}

}  // extern "C"

extern "C" {

int cc_kset_stealthy(int d, const double *basis, int64_t N, double chi, int type, int64_t cap, int32_t *modes,
                     double *V, int64_t *M)
{
	if (d < 1 || d > 3 || !basis || N < 0 || !(chi >= 0) || type < 0 || type > 3 || !M || cap < 0 ||
	    (cap > 0 && (!modes || !V)))
		return fail(CC_ERR_ARG, "invalid k-set arguments");
	std::vector<int32_t> mv;
	std::vector<double> vv;
	if (!cc::stealthy_kset(d, basis, N, chi, type, mv, vv))
		return fail(CC_ERR_ARG, "degenerate cell basis or k-set too large");
	*M = (int64_t)vv.size();
	if (*M > cap)
		return fail(CC_ERR_ARG, "cap too small for the k-set");
	std::memcpy(modes, mv.data(), mv.size() * sizeof(int32_t));
	std::memcpy(V, vv.data(), vv.size() * sizeof(double));
	return CC_OK;
}


int cc_kset_isotropic(int d, const double *basis, double circular_kmax, double linear_kmax, double sample_probability,
                      double circular_kmin, int64_t cap, int32_t *modes, double *kamp, int64_t *K)
{
	if (d < 1 || d > 3 || !basis || !K || cap < 0 || (cap > 0 && (!modes || !kamp)) || std::isnan(circular_kmax) ||
	    std::isnan(linear_kmax) || std::isnan(sample_probability) || std::isnan(circular_kmin))
		return fail(CC_ERR_ARG, "invalid wavevector-list arguments");
	std::vector<int32_t> mv;
	std::vector<double> kv;
	if (!cc::isotropic_ks(d, basis, circular_kmax, linear_kmax, sample_probability, circular_kmin, mv, kv))
		return fail(CC_ERR_ARG, "degenerate cell, non-positive 1D cell or too many wavevectors");
	*K = (int64_t)kv.size();
	if (*K > cap)
		return fail(CC_ERR_ARG, "cap too small for the wavevector list");
	std::memcpy(modes, mv.data(), mv.size() * sizeof(int32_t));
	std::memcpy(kamp, kv.data(), kv.size() * sizeof(double));
	return CC_OK;
}

int cc_isotropic_structure_factor(int d, int64_t nconfigs, const double *bases, const int64_t *N,
                                  const double *const *frac, double circular_kmax, double linear_kmax,
                                  double k_precision, double sample_probability, int option, double circular_kmin,
                                  double *results, int64_t cap, int64_t *count)
{
	if (d < 1 || d > 3 || nconfigs < 1 || !bases || !N || !frac || !count || cap < 0 || (cap > 0 && !results))
		return fail(CC_ERR_ARG, "invalid isotropic S(k) arguments");
	if (option < 0 || option > 2)
		return fail(CC_ERR_ARG, "option must be 0 (average over wavevectors), 1 (over k-space volume) or 2 (per wavevector)");
	if (std::isnan(k_precision) || k_precision < 0.0 || std::isnan(sample_probability) || std::isnan(circular_kmin))
		return fail(CC_ERR_ARG, "k_precision must be >= 0 (0: the first reciprocal vector's length)");
	*count = 0;
	// the reference returns no result for these
	if (!(circular_kmax > 0.0) || !(linear_kmax > 0.0) || circular_kmin > circular_kmax)
		return CC_OK;
	const int dd = d * d;
	double vol0 = 0.0, recip0[9];
	if (!cc::cell_geometry(d, bases, &vol0, recip0))
		return fail(CC_ERR_ARG, "degenerate cell basis");
	if (k_precision == 0.0) {
		cc::reciprocal_by_projection(d, bases, recip0);   // the reference's |b_0|
		double b2 = 0.0;
		for (int x = 0; x < d; x++)
			b2 += recip0[x] * recip0[x];
		k_precision = std::sqrt(b2);
	}
	struct Bin {
		double n = 0, k1 = 0, k2 = 0, s1 = 0, s2 = 0;
	};
	const size_t nbin = (size_t)std::floor(linear_kmax / k_precision) + 1;
	if (!(linear_kmax / k_precision < 1e9))
		return fail(CC_ERR_ARG, "linear_kmax / k_precision is too large");
	std::vector<Bin> bins(option == 2 ? 0 : nbin);
	double ident[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
	double I[9];
	for (int i = 0; i < d; i++)
		for (int j = 0; j < d; j++)
			I[i * d + j] = ident[i * 3 + j];
	// S(k) depends only on the integer modes and the fractional positions: one handle serves every configuration
	cc_handle *h = nullptr;
	if (int rc = cc_create(d, I, 0, nullptr, nullptr, 0.0, &h))
		return rc;
	std::vector<int32_t> modes;
	std::vector<double> kamp, S;
	int rc = CC_OK;
	for (int64_t j = 0; j < nconfigs && rc == CC_OK; j++) {
		const double *bj = bases + (size_t)j * dd;
		const bool same = j > 0 && std::equal(bj, bj + dd, bases + (size_t)(j - 1) * dd);
		if (!same) {
			if (!cc::isotropic_ks(d, bj, circular_kmax, linear_kmax, sample_probability, circular_kmin, modes, kamp)) {
				rc = fail(CC_ERR_ARG, "degenerate cell, non-positive 1D cell or too many wavevectors");
				break;
			}
			if (option == 2) {
				if (j == 0)
					bins.assign(kamp.size(), Bin());
				else if (kamp.size() != bins.size()) {
					rc = fail(CC_ERR_ARG, "per-wavevector S(k) needs the same number of wavevectors in every cell");
					break;
				}
			}
		}
		const int64_t K = (int64_t)kamp.size();
		if (K == 0)
			continue;
		if (N[j] < 0 || (N[j] > 0 && !frac[j])) {
			rc = fail(CC_ERR_ARG, "invalid particle count or null positions");
			break;
		}
		S.resize((size_t)K);
		if ((rc = cc_set_positions(h, N[j], frac[j])) || (rc = cc_structure_factor(h, K, modes.data(), S.data(), CC_PREC_FP64)))
			break;
		for (int64_t i = 0; i < K; i++) {
			size_t b = (size_t)i;
			if (option != 2) {
				b = (size_t)std::floor(kamp[i] / k_precision);
				if (b >= bins.size())
					continue;
			}
			Bin &q = bins[b];
			q.n += 1.0;
			q.k1 += kamp[i];
			q.k2 += kamp[i] * kamp[i];
			q.s1 += S[i];
			q.s2 += S[i] * S[i];
		}
	}
	cc_destroy(h);
	if (rc)
		return rc;
	// rows (k, S, dk, dS) as IsotropicStructureFactor (pairstat/StructureFactor.cpp:199-256)
	auto ball = [d](double r) {
		const double c = d == 1 ? 2.0 : d == 2 ? M_PI : 4.1887902047863909846;
		return c * std::pow(r, (double)d);
	};
	const double omega = std::pow(2.0 * M_PI, (double)d) / vol0 / (double)nconfigs;
	std::vector<std::array<double, 4> > rows;
	for (const Bin &q : bins) {
		if (!(q.n > 0.0))
			continue;
		std::array<double, 4> r;
		r[0] = q.k1 / q.n;
		const double kv = (q.k2 / q.n - r[0] * r[0]) / q.n;
		r[2] = kv > 0 ? std::sqrt(kv) : 0.0;
		const double mean = q.s1 / q.n, sv = q.s2 / q.n - mean * mean;
		if (option == 0 || r[0] > circular_kmax) {
			r[1] = mean;
			r[3] = std::sqrt((sv > 0 ? sv : 0.0) / q.n);
		} else if (option == 1) {
			const double vd = 0.5 * (ball(r[0] + 0.5 * k_precision) - ball(r[0] - 0.5 * k_precision));
			r[1] = q.s1 * omega / vd;
			r[2] = 0.5 * k_precision;
			r[3] = (omega / vd) * std::sqrt((sv > 0 ? sv : 0.0) / q.n);
		} else {
			r[1] = mean;
			r[3] = q.n;
		}
		rows.push_back(r);
	}
	if (option == 2)   // by |k|; equal |k| keep the order the reference's sort gives them on the same sequence
		std::sort(rows.begin(), rows.end(),
		          [](const std::array<double, 4> &a, const std::array<double, 4> &b) { return a[0] < b[0]; });
	*count = (int64_t)rows.size();
	if (*count > cap)
		return fail(CC_ERR_ARG, "cap too small for the S(k) rows");
	for (size_t i = 0; i < rows.size(); i++)
		for (int c = 0; c < 4; c++)
			results[i * 4 + c] = rows[i][c];
	return CC_OK;
}

}  // extern "C"
