// cc_serve.cu — a ground-state server with continuous batching (cc_serve in include/cc_gpu.h).
//
// Requests (a stealthy CC configuration each: d, N, chi, weight type, start positions, arrival time) are minimised
// to their ground state on one GPU. The server works in rounds:
//   1. admit arrived requests, in arrival order, while a slot is free and the request's device memory fits the HBM
//      budget (a request waiting for memory may be passed by later ones until it has waited max_bypass_s; one that can
//      never be served is rejected with a status of its own). Its k-set is planned on the host; its k-set arrays,
//      partial sums and L-BFGS state are allocated from the server's own stream-ordered pool, which holds the
//      budget, and stay resident until it finishes;
//   2. run `iters_per_round` L-BFGS iterations for every admitted request at once: per iteration ONE launch of the
//      fused batch kernel evaluating every request (cc_multi_launch.h; requests of any dimension in one work queue)
//      and one launch each of the batched L-BFGS kernels (cc_lbfgs.cuh);
//   3. read every request's status (one gather kernel, one copy), retire finished requests (time-to-ground-state =
//      completion - arrival) and free their memory.
// Requests that arrive while others are on the GPU join at the next round, so their work overlaps; an instance's
// iterates do not depend on the rest of the batch (every sum has a fixed per-instance order), so a request's result
// is the same alone and in the mix.
#include "../../include/cc_gpu.h"
#include "cc_multi_launch.h"
#include "cc_lbfgs.cuh"
#include "cc_plan.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace {

thread_local std::string s_err;

int sfail(int code, const std::string &m)
{
	s_err = m;
	return code;
}

#define SV_CUDA(call)                                                                                         \
	do {                                                                                                      \
		cudaError_t e_ = (call);                                                                              \
		if (e_ != cudaSuccess)                                                                                \
			return sfail(CC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));                    \
	} while (0)

struct Carve {
	size_t used = 0;
	size_t take(size_t bytes)
	{
		const size_t off = used;
		used += (bytes + 255) / 256 * 256;
		return off;
	}
};

struct Slot {
	int req = -1;
	int d = 0;
	int64_t N = 0;
	size_t bytes = 0;
	unsigned char *mem = nullptr;
	cc::RhoArgs ra;
	cc::ReduceArgs rr;
	cc::ForceArgs fa;
	int blocks[3], shape[3];   // rho / reduce / force blocks and grid shapes of the multi-instance launches
	int rho_row, force_row;
	cc::LbInst li;
};

// Particles per rho block of a served request: the largest power of two in [kServeMinPerSplit, kBatchPerSplit] whose
// blocks hold at most kServeRhoPairs particle-slot pairs (particles x the widest block group's slots). Serving runs
// light loads, where an iteration lasts about one block's time: smaller rho tiles cut it for the large requests.
constexpr int kServeMinPerSplit = 16;
constexpr int64_t kServeRhoPairs = 1 << 14;
int serve_per_split(const cc::Plan &p)
{
	int max_wg = 1;
	for (int g = 0; g < p.nbgroups(); g++)
		max_wg = std::max(max_wg, p.bstart[g + 1] - p.bstart[g]);
	const int64_t bslots = (int64_t)max_wg * 32 * p.L;
	int per = cc::kBatchPerSplit;
	while (per > kServeMinPerSplit && (int64_t)per * bslots > kServeRhoPairs)
		per /= 2;
	return per;
}

// Offsets of a request's arrays in its one allocation (see open_slot).
struct SlotOffsets {
	size_t segs, slotV, bstart, bspec, kstart, kspec, part, rho, u, ep, tk, pg, fc, x, g, d, xt, gt, S, Y, lp, st;
};

int fill_slot(const cc_request &r, int idx, int m, const cc::Plan &p, const cc::ForceSplits &fs, double vol,
              const double *recip, int per_split, int nsplit, int nchunks, int pgroups, int nks, cudaStream_t st,
              const SlotOffsets &off, Slot &s);

// Plan and allocate a request; returns CC_OK and fills the slot.
int open_slot(const cc_request &r, int idx, int m, int nblk_cap, cudaMemPool_t pool, cudaStream_t st, Slot &s)
{
	const int d = r.d;
	const double side = std::pow((double)r.N, 1.0 / d);   // unit density
	double basis[9] = {0};
	for (int e = 0; e < d; e++)
		basis[e * d + e] = side;
	std::vector<int32_t> modes;
	std::vector<double> V;
	if (!cc::stealthy_kset(d, basis, r.N, r.chi, r.vtype, modes, V) || V.empty())
		return sfail(CC_ERR_ARG, "request k-set is empty or invalid");
	cc::Plan p = cc::build_plan(d, (int64_t)V.size(), modes.data(), V.data(), 8);
	const int want = (int)std::max<int64_t>(1, (p.real_segs + cc::kBatchSegsPerSplit - 1) / cc::kBatchSegsPerSplit);
	cc::ForceSplits fs = cc::force_splits(p, want);
	double vol = 0, recip[9] = {0};
	cc::cell_geometry(d, basis, &vol, recip);
	const int64_t N = r.N;
	const int n = (int)(N * d);
	const int per_split = serve_per_split(p);
	const int nsplit = (int)((N + per_split - 1) / per_split);
	// reduce items of kWideSlots slots each in the fused launch (their energy terms are the force items' eblock)
	const int nchunks = (p.nslot + cc::kWideSlots - 1) / cc::kWideSlots, pgroups = (int)((N + 31) / 32);
	const int nks = fs.count();
	Carve c;
	const size_t o_segs = c.take(sizeof(cc::Seg) * p.segs.size()), o_slotV = c.take(sizeof(double) * p.nslot),
	             o_bstart = c.take(sizeof(int) * p.bstart.size()), o_bspec = c.take(sizeof(cc::TabSpec) * p.bspec.size()),
	             o_kstart = c.take(sizeof(int) * fs.start.size()), o_kspec = c.take(sizeof(cc::TabSpec) * fs.spec.size()),
	             o_part = c.take(sizeof(double2) * (size_t)nsplit * p.nslot), o_rho = c.take(sizeof(double2) * p.nslot),
	             o_u = c.take(sizeof(double2) * p.nslot), o_ep = c.take(sizeof(double) * nchunks),
	             o_tk = c.take(sizeof(unsigned)), o_pg = c.take(sizeof(double) * (size_t)nks * n),
	             o_fc = c.take(sizeof(unsigned) * pgroups),
	             o_x = c.take(8 * n), o_g = c.take(8 * n), o_d = c.take(8 * n), o_xt = c.take(8 * n), o_gt = c.take(8 * n),
	             o_S = c.take(8 * (size_t)n * m), o_Y = c.take(8 * (size_t)n * m),
	             o_lp = c.take(8 * (size_t)nblk_cap * cc::lb_ndots(m)), o_st = c.take(sizeof(cc::LbState));
	s.bytes = c.used;
	{
		const cudaError_t ae = cudaMallocFromPoolAsync(reinterpret_cast<void **>(&s.mem), c.used, pool, st);
		if (ae != cudaSuccess) {
			cudaGetLastError();   // an allocation failure is not sticky: clear it and reject this request alone
			s.mem = nullptr;
			return sfail(ae == cudaErrorMemoryAllocation ? CC_ERR_OOM : CC_ERR_CUDA,
			             std::string("request memory: ") + cudaGetErrorString(ae));
		}
	}
	if (int rc = fill_slot(r, idx, m, p, fs, vol, recip, per_split, nsplit, nchunks, pgroups, nks, st,
	                       {o_segs, o_slotV, o_bstart, o_bspec, o_kstart, o_kspec, o_part, o_rho, o_u, o_ep, o_tk,
	                        o_pg, o_fc, o_x, o_g, o_d, o_xt, o_gt, o_S, o_Y, o_lp, o_st},
	                       s)) {
		cudaFreeAsync(s.mem, st);
		s.mem = nullptr;
		return rc;
	}
	return CC_OK;
}

// Upload a request's plan and start and fill its kernel arguments (its memory is allocated).
int fill_slot(const cc_request &r, int idx, int m, const cc::Plan &p, const cc::ForceSplits &fs, double vol,
              const double *recip, int per_split, int nsplit, int nchunks, int pgroups, int nks, cudaStream_t st,
              const SlotOffsets &off, Slot &s)
{
	const size_t o_segs = off.segs, o_slotV = off.slotV, o_bstart = off.bstart, o_bspec = off.bspec,
	             o_kstart = off.kstart, o_kspec = off.kspec, o_part = off.part, o_rho = off.rho, o_u = off.u,
	             o_ep = off.ep, o_tk = off.tk, o_pg = off.pg, o_fc = off.fc, o_x = off.x, o_g = off.g, o_d = off.d,
	             o_xt = off.xt, o_gt = off.gt, o_S = off.S, o_Y = off.Y, o_lp = off.lp, o_st = off.st;
	const int d = r.d;
	const int64_t N = r.N;
	const int n = (int)(N * d);
	unsigned char *b = s.mem;
	SV_CUDA(cudaMemcpyAsync(b + o_segs, p.segs.data(), sizeof(cc::Seg) * p.segs.size(), cudaMemcpyHostToDevice, st));
	SV_CUDA(cudaMemcpyAsync(b + o_slotV, p.slotV.data(), sizeof(double) * p.nslot, cudaMemcpyHostToDevice, st));
	SV_CUDA(cudaMemcpyAsync(b + o_bstart, p.bstart.data(), sizeof(int) * p.bstart.size(), cudaMemcpyHostToDevice, st));
	SV_CUDA(cudaMemcpyAsync(b + o_bspec, p.bspec.data(), sizeof(cc::TabSpec) * p.bspec.size(), cudaMemcpyHostToDevice,
	                        st));
	SV_CUDA(cudaMemcpyAsync(b + o_kstart, fs.start.data(), sizeof(int) * fs.start.size(), cudaMemcpyHostToDevice, st));
	SV_CUDA(cudaMemcpyAsync(b + o_kspec, fs.spec.data(), sizeof(cc::TabSpec) * fs.spec.size(), cudaMemcpyHostToDevice,
	                        st));
	SV_CUDA(cudaMemsetAsync(b + o_tk, 0, sizeof(unsigned), st));
	SV_CUDA(cudaMemsetAsync(b + o_fc, 0, sizeof(unsigned) * pgroups, st));
	std::vector<double> x0(n);
	for (int k = 0; k < n; k++) {
		double v = r.frac0[k] - std::floor(r.frac0[k]);
		x0[k] = v - std::floor(v);
	}
	SV_CUDA(cudaMemcpyAsync(b + o_x, x0.data(), 8 * n, cudaMemcpyHostToDevice, st));
	SV_CUDA(cudaMemcpyAsync(b + o_xt, x0.data(), 8 * n, cudaMemcpyHostToDevice, st));
	SV_CUDA(cudaMemsetAsync(b + o_g, 0, 8 * n, st));
	SV_CUDA(cudaMemsetAsync(b + o_d, 0, 8 * n, st));
	cc::LbState s0;
	std::memset(&s0, 0, sizeof(s0));
	s0.E = INFINITY;
	s0.gamma = 1.0;
	s0.stopval = 1e-20 * (double)N;
	s0.ftol = 1e-15;
	s0.max_evals = r.max_evals > 0 ? r.max_evals : 100000;
	s0.m = m;
	s0.newslot = -1;
	SV_CUDA(cudaMemcpyAsync(b + o_st, &s0, sizeof(s0), cudaMemcpyHostToDevice, st));
	// host buffers above are pageable: the copies complete before the call returns
	SV_CUDA(cudaStreamSynchronize(st));
	s.req = idx;
	s.d = d;
	s.N = N;
	cc::LbInst &l = s.li;
	l.n = n;
	l.m = m;
	l.x = reinterpret_cast<double *>(b + o_x);
	l.g = reinterpret_cast<double *>(b + o_g);
	l.d = reinterpret_cast<double *>(b + o_d);
	l.xt = reinterpret_cast<double *>(b + o_xt);
	l.gt = reinterpret_cast<double *>(b + o_gt);
	l.S = reinterpret_cast<double *>(b + o_S);
	l.Y = reinterpret_cast<double *>(b + o_Y);
	l.part = reinterpret_cast<double *>(b + o_lp);
	l.st = reinterpret_cast<cc::LbState *>(b + o_st);
	const int *status = &l.st->status;
	cc::RhoArgs &ra = s.ra;
	ra = cc::RhoArgs();
	ra.frac = l.xt;
	ra.N = (int)N;
	ra.per_split = per_split;
	ra.chunk = cc::kBatchChunk;
	ra.segs = reinterpret_cast<const cc::Seg *>(b + o_segs);
	ra.bstart = reinterpret_cast<const int *>(b + o_bstart);
	ra.bspec = reinterpret_cast<const cc::TabSpec *>(b + o_bspec);
	ra.nseg = (int)p.segs.size();
	ra.nslot = p.nslot;
	ra.partial = reinterpret_cast<double2 *>(b + o_part);
	ra.skip = status;
	cc::ReduceArgs &rr = s.rr;
	rr = cc::ReduceArgs();
	rr.partial = ra.partial;
	rr.nsplit = nsplit;
	rr.nslot = p.nslot;
	rr.slotV = reinterpret_cast<const double *>(b + o_slotV);
	rr.rho_offset = 0.0;
	rr.rho_slot = reinterpret_cast<double2 *>(b + o_rho);
	rr.u_slot = reinterpret_cast<double2 *>(b + o_u);
	rr.eblock = reinterpret_cast<double *>(b + o_ep);
	rr.ticket = reinterpret_cast<unsigned *>(b + o_tk);
	rr.inv_vol = 1.0 / vol;
	rr.shift = 0.0;
	rr.E_out = &l.st->Et;
	rr.finalize = 0;   // the force kernel sums the energy terms
	rr.skip = status;
	cc::ForceArgs &fa = s.fa;
	fa = cc::ForceArgs();
	fa.frac = l.xt;
	fa.N = (int)N;
	fa.segs = ra.segs;
	fa.kstart = reinterpret_cast<const int *>(b + o_kstart);
	fa.kspec = reinterpret_cast<const cc::TabSpec *>(b + o_kspec);
	fa.nksplit = nks;
	fa.u_slot = rr.u_slot;
	fa.nseg = ra.nseg;
	fa.partialG = reinterpret_cast<double *>(b + o_pg);
	fa.counters = reinterpret_cast<unsigned *>(b + o_fc);
	for (int k = 0; k < 9; k++)
		fa.recip[k] = recip[k];
	fa.fscale = 2.0 / vol;
	fa.F_out = nullptr;
	fa.gfrac_out = l.gt;
	fa.eblock = rr.eblock;
	fa.neblock = nchunks;
	fa.inv_vol = rr.inv_vol;
	fa.shift = 0.0;
	fa.E_out = &l.st->Et;
	fa.skip = status;
	s.blocks[0] = p.nbgroups() * nsplit;
	s.blocks[1] = nchunks;
	s.blocks[2] = pgroups * nks;
	s.shape[0] = p.nbgroups();
	s.shape[1] = nchunks;
	s.shape[2] = pgroups;
	s.rho_row = std::max(1, p.block_max_row);
	s.force_row = std::max(1, fs.max_row);
	return CC_OK;
}

// a request's reduce and force items in one fused launch
int sl_items(const Slot &s) { return s.blocks[1] + s.blocks[2]; }

// device bytes a request will need (the same carve as open_slot, with the k-set size estimated from chi N d)
size_t estimate_bytes(const cc_request &r, int m, int nblk_cap)
{
	const double M = std::ceil(r.chi * (double)r.N * r.d) * 1.1 + 64;
	const double nseg = M / 4 + 64, nslot = nseg * 8;
	const double n = (double)r.N * r.d;
	const double nsplit = std::ceil(r.N / (double)kServeMinPerSplit), nks = std::ceil(nseg / cc::kBatchSegsPerSplit) + 2;
	const double bytes = 16 * nseg + 8 * nslot + 2 * 768 * (nseg / 256 + nks + 2) + 16 * nsplit * nslot + 32 * nslot +
	                     8 * nks * n + 8 * n * (5 + 2 * m) + 8.0 * nblk_cap * cc::lb_ndots(m) + 16384;
	return (size_t)bytes;
}

}  // namespace

extern "C" const char *cc_serve_last_error(void) { return s_err.c_str(); }

extern "C" int cc_serve(const cc_request *reqs, int count, const cc_serve_opts *opts, cc_request_result *out,
                        double *wall_s)
{
	if (!reqs || count < 1 || !out)
		return sfail(CC_ERR_ARG, "invalid serve arguments");
	cc_serve_opts o = {};
	o.hbm_budget = (size_t)16 << 30;
	o.max_slots = 256;
	o.iters_per_round = 16;
	o.history = 40;
	o.max_bypass_s = 1.0;
	if (opts)
		o = *opts;
	if (o.max_slots < 1 || o.iters_per_round < 1 || o.history < 1 || o.history > cc::kLbMaxHist ||
	    !(o.max_bypass_s >= 0.0))
		return sfail(CC_ERR_ARG, "invalid serve options");
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
		return sfail(CC_ERR_NOGPU, "no CUDA device is visible");
	const int m = o.history;
	const int nblk_cap = cc::kLbMaxBlocks;
	cudaStream_t st;
	SV_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
	// The requests' memory comes from a pool of the server's own that keeps what it holds (release threshold: all)
	// and holds the HBM budget from the start (as far as the device has it free): admitting and retiring requests then
	// makes no allocation call into the CUDA driver, whose calls took up to ~1 s under contention on shared hosts.
	int dev = 0;
	SV_CUDA(cudaGetDevice(&dev));
	cudaMemPoolProps pprops = {};
	pprops.allocType = cudaMemAllocationTypePinned;
	pprops.location.type = cudaMemLocationTypeDevice;
	pprops.location.id = dev;
	cudaMemPool_t pool = nullptr;
	SV_CUDA(cudaMemPoolCreate(&pool, &pprops));
	{
		uint64_t keep = UINT64_MAX;
		SV_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
		size_t free_b = 0, total_b = 0;
		SV_CUDA(cudaMemGetInfo(&free_b, &total_b));
		const size_t margin = (size_t)1 << 30;
		const size_t reserve = std::min(o.hbm_budget, free_b > margin ? free_b - margin : 0);
		if (reserve > 0) {
			void *p = nullptr;
			if (cudaMallocFromPoolAsync(&p, reserve, pool, st) == cudaSuccess)
				cudaFreeAsync(p, st);
			else
				cudaGetLastError();   // no reservation: the pool grows on demand
			SV_CUDA(cudaStreamSynchronize(st));
		}
	}
	// device descriptor arrays sized for max_slots; one work queue (6 words) per dimension
	cc::RhoArgs *d_ra = nullptr;
	cc::ReduceArgs *d_rr = nullptr;
	cc::ForceArgs *d_fa = nullptr;
	cc::LbInst *d_li = nullptr;
	int *d_pre = nullptr, *d_shape = nullptr, *d_dim = nullptr;
	unsigned *d_queue = nullptr, *d_count = nullptr;
	cc::LbBrief *d_brief = nullptr;
	SV_CUDA(cudaMalloc(&d_ra, sizeof(cc::RhoArgs) * o.max_slots));
	SV_CUDA(cudaMalloc(&d_rr, sizeof(cc::ReduceArgs) * o.max_slots));
	SV_CUDA(cudaMalloc(&d_fa, sizeof(cc::ForceArgs) * o.max_slots));
	SV_CUDA(cudaMalloc(&d_li, sizeof(cc::LbInst) * o.max_slots));
	SV_CUDA(cudaMalloc(&d_pre, sizeof(int) * 4 * (o.max_slots + 1)));
	SV_CUDA(cudaMalloc(&d_shape, sizeof(int) * 3 * o.max_slots));
	SV_CUDA(cudaMalloc(&d_dim, sizeof(int) * o.max_slots));
	SV_CUDA(cudaMalloc(&d_queue, sizeof(unsigned) * 2));
	SV_CUDA(cudaMalloc(&d_count, sizeof(unsigned) * (3 * o.max_slots + 1)));
	SV_CUDA(cudaMalloc(&d_brief, sizeof(cc::LbBrief) * o.max_slots));
	SV_CUDA(cudaMemset(d_queue, 0, sizeof(unsigned) * 2));
	// the fused launch's completion counts are zero between launches (its items reset them); the error word after
	// the counts of the current round's requests must start at zero too
	SV_CUDA(cudaMemset(d_count, 0, sizeof(unsigned) * (3 * o.max_slots + 1)));
	const auto t0 = std::chrono::steady_clock::now();
	auto now = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
	int done = 0;
	// a request the server cannot serve gets a status of its own; the others carry on
	auto reject = [&](int idx, int code) {
		cc_request_result &res = out[idx];
		res.E = NAN;
		res.evals = 0;
		res.status = code;
		res.t_admit = res.t_done = now();
		done++;
	};
	std::vector<int> order;
	order.reserve(count);
	for (int i = 0; i < count; i++) {
		const cc_request &r = reqs[i];
		bool ok = r.d >= 1 && r.d <= 3 && r.N >= 1 && r.N <= (1 << 24) && r.frac0 && r.chi > 0 && r.vtype >= 0 &&
		          r.vtype <= 3 && std::isfinite(r.arrival_s) && r.max_evals >= 0;
		for (int64_t k = 0; ok && k < r.N * r.d; k++)
			ok = std::isfinite(r.frac0[k]);
		if (ok)
			order.push_back(i);
		else
			reject(i, CC_ERR_ARG);
	}
	std::stable_sort(order.begin(), order.end(),
	                 [&](int a, int b) { return reqs[a].arrival_s < reqs[b].arrival_s; });
	std::vector<Slot> active;
	std::vector<int> pending;   // arrived and not yet admitted, in arrival order
	size_t used = 0;
	size_t next = 0;
	int rc = CC_OK;
	std::vector<cc::LbBrief> hs(o.max_slots);
	while (done < count && rc == CC_OK) {
		// 1. admission: every arrived request that fits, in arrival order; one that does not fit yet may be passed
		// by later ones until it has waited max_bypass_s
		const double t = now();
		while (next < order.size() && reqs[order[next]].arrival_s <= t)
			pending.push_back(order[next++]);
		std::vector<int> waiting;
		bool hold = false;
		for (int idx : pending) {
			if (hold || (int)active.size() >= o.max_slots) {
				waiting.push_back(idx);
				continue;
			}
			const cc_request &r = reqs[idx];
			const size_t need = estimate_bytes(r, m, nblk_cap);
			if (need > o.hbm_budget) {
				reject(idx, CC_ERR_OOM);
				continue;
			}
			if (used + need > o.hbm_budget) {
				waiting.push_back(idx);
				hold = now() - r.arrival_s > o.max_bypass_s;
				continue;
			}
			Slot s;
			const int orc = open_slot(r, idx, m, nblk_cap, pool, st, s);
			if (orc != CC_OK) {
				reject(idx, orc);
				continue;
			}
			used += s.bytes;
			out[idx].t_admit = now();
			active.push_back(s);
		}
		pending.swap(waiting);
		if (active.empty()) {
			if (!pending.empty()) {   // nothing runs and a request still waits: it cannot be placed at all
				reject(pending.front(), CC_ERR_OOM);
				pending.erase(pending.begin());
				continue;
			}
			if (next < order.size()) {
				const double wait = reqs[order[next]].arrival_s - now();
				if (wait > 0)
					std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.01)));
			}
			continue;
		}
		// 2. descriptors of the active set, requests by decreasing work (the fused launch's work queue then hands out
		// the longest items first)
		std::stable_sort(active.begin(), active.end(), [](const Slot &x, const Slot &y) {
			return (double)x.N * x.rr.nslot > (double)y.N * y.rr.nslot;
		});
		const int A = (int)active.size();
		std::vector<cc::LbInst> li(A);
		std::vector<cc::RhoArgs> ra(A);
		std::vector<cc::ReduceArgs> rr(A);
		std::vector<cc::ForceArgs> fa(A);
		std::vector<int> pre(4 * (A + 1), 0), shape(3 * A, 0), dim(A, 0);
		int rho_row = 1, force_row = 1, maxd = 1, maxn = 0;
		for (int k = 0; k < A; k++) {
			const Slot &sl = active[k];
			li[k] = sl.li;
			ra[k] = sl.ra;
			rr[k] = sl.rr;
			fa[k] = sl.fa;
			for (int ph = 0; ph < 3; ph++) {
				pre[ph * (A + 1) + k + 1] = pre[ph * (A + 1) + k] + sl.blocks[ph];
				shape[ph * A + k] = sl.shape[ph];
			}
			dim[k] = sl.d;
			rho_row = std::max(rho_row, sl.rho_row);
			force_row = std::max(force_row, sl.force_row);
			maxd = std::max(maxd, sl.d);
			maxn = std::max(maxn, sl.li.n);
		}
		for (int k = 0; k < A; k++)   // each request's reduce and force items, consecutive in the queue
			pre[3 * (A + 1) + k + 1] = pre[3 * (A + 1) + k] + sl_items(active[k]);
		SV_CUDA(cudaMemcpyAsync(d_ra, ra.data(), sizeof(cc::RhoArgs) * A, cudaMemcpyHostToDevice, st));
		SV_CUDA(cudaMemcpyAsync(d_rr, rr.data(), sizeof(cc::ReduceArgs) * A, cudaMemcpyHostToDevice, st));
		SV_CUDA(cudaMemcpyAsync(d_fa, fa.data(), sizeof(cc::ForceArgs) * A, cudaMemcpyHostToDevice, st));
		SV_CUDA(cudaMemcpyAsync(d_li, li.data(), sizeof(cc::LbInst) * A, cudaMemcpyHostToDevice, st));
		SV_CUDA(cudaMemcpyAsync(d_pre, pre.data(), sizeof(int) * pre.size(), cudaMemcpyHostToDevice, st));
		SV_CUDA(cudaMemcpyAsync(d_shape, shape.data(), sizeof(int) * shape.size(), cudaMemcpyHostToDevice, st));
		SV_CUDA(cudaMemcpyAsync(d_dim, dim.data(), sizeof(int) * A, cudaMemcpyHostToDevice, st));
		// the descriptor vectors are pageable: the copies complete before the iterations read them
		cc::MBatchArgs ma;
		ma.rho = d_ra;
		ma.red = d_rr;
		ma.force = d_fa;
		ma.dim = d_dim;
		ma.pre = d_pre;
		ma.shape = d_shape;
		ma.B = A;
		for (int ph = 0; ph < 3; ph++)
			ma.total[ph] = pre[ph * (A + 1) + A];
		ma.want_stage = 1;
		ma.queue = d_queue;
		ma.count = d_count;
		ma.spins = 0;
		ma.phantom = 0;
		const int nblk = cc::lb_blocks(maxn, nblk_cap);
		// every iteration: one fused evaluation of all admitted requests, then their L-BFGS step
		for (int it = 0; it < o.iters_per_round && rc == CC_OK; it++) {
			if ((rc = cc::launch_mbatch(0, ma, rho_row, force_row, maxd, st))) {
				s_err = std::string("serve: ") + cc_last_error();
				break;
			}
			if (cc::lb_step(d_li, A, nblk, maxn, st, A == 1 ? &li[0] : nullptr) != cudaSuccess)
				rc = sfail(CC_ERR_CUDA, "serve: kernel launch failed");
		}
		if (rc)
			break;
		// 3. retire finished requests
		// every slot's status, energy and evaluation count: one gather kernel, one copy (d_li holds this round's slots)
		cc::lb_brief_kernel<<<(A + 127) / 128, 128, 0, st>>>(d_li, A, d_brief);
		SV_CUDA(cudaGetLastError());
		SV_CUDA(cudaMemcpyAsync(hs.data(), d_brief, sizeof(cc::LbBrief) * A, cudaMemcpyDeviceToHost, st));
		unsigned wait_err = 0;
		SV_CUDA(cudaMemcpyAsync(&wait_err, d_count + 3 * A, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
		SV_CUDA(cudaStreamSynchronize(st));
		if (wait_err) {
			rc = sfail(CC_ERR_TIMEOUT, "serve: a bounded wait of the fused evaluation kernel ran out");
			break;
		}
		const double tdone = now();
		std::vector<Slot> keep;
		for (int a = 0; a < A; a++) {
			if (hs[a].status == cc::kLbRunning) {
				keep.push_back(active[a]);
				continue;
			}
			cc_request_result &res = out[active[a].req];
			if (double *fo = reqs[active[a].req].frac_out)
				SV_CUDA(cudaMemcpyAsync(fo, active[a].li.x, sizeof(double) * active[a].li.n, cudaMemcpyDeviceToHost,
				                        st));
			res.E = hs[a].E;
			res.evals = hs[a].evals;
			res.status = hs[a].status;
			res.t_done = tdone;
			cudaFreeAsync(active[a].mem, st);
			used -= active[a].bytes;
			done++;
		}
		active.swap(keep);
	}
	for (Slot &s : active)
		cudaFreeAsync(s.mem, st);
	cudaStreamSynchronize(st);
	if (wall_s)
		*wall_s = now();
	cudaFree(d_ra);
	cudaFree(d_rr);
	cudaFree(d_fa);
	cudaFree(d_li);
	cudaFree(d_pre);
	cudaFree(d_shape);
	cudaFree(d_dim);
	cudaFree(d_queue);
	cudaFree(d_count);
	cudaFree(d_brief);
	cudaMemPoolDestroy(pool);
	cudaStreamDestroy(st);
	return rc;
}
