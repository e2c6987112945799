// cc_serve.cu — a ground-state server with continuous batching (cc_serve in include/cc_gpu.h).
//
// Requests (a stealthy CC configuration each: d, N, chi, weight type, start positions, arrival time) are minimised
// to their ground state on one GPU. The server works in rounds:
//   1. admit every request that has arrived, in arrival order, while a slot is free and the request's device memory
//      fits the HBM budget (its k-set is planned on the host, its k-set arrays, phase tables, partial sums and L-BFGS
//      state are allocated from a stream-ordered pool and stay resident until it finishes);
//   2. run `iters_per_round` L-BFGS iterations for every admitted request at once: per iteration one cooperative batch
//      evaluation per dimension (cc_batch.cuh) and one launch each of the batched L-BFGS kernels (cc_lbfgs.cuh);
//   3. retire finished requests (time-to-ground-state = completion - arrival) and free their memory.
// Requests that arrive while others are on the GPU join at the next round, so their work overlaps; an instance's
// iterates do not depend on the rest of the batch (every sum has a fixed per-instance order), so a request's result
// is the same alone and in the mix.
#include "../../include/cc_gpu.h"
#include "cc_batch.cuh"
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
	cc::BInst bi;
	cc::LbInst li;
};

template <int D> int grid_for()
{
	static int per_sm = -1;
	if (per_sm < 0) {
		if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cc::cc_batch_kernel<D, 8, false>, cc::kFusedThreads,
		                                                  0) != cudaSuccess)
			per_sm = 0;
	}
	int sms = 148, dev = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
	return per_sm * sms;
}

int launch_batch(int D, cc::BatchArgs &a, cudaStream_t st)
{
	void *args[] = {&a};
	const void *k = D == 1 ? (const void *)cc::cc_batch_kernel<1, 8, false>
	                       : D == 2 ? (const void *)cc::cc_batch_kernel<2, 8, false>
	                                : (const void *)cc::cc_batch_kernel<3, 8, false>;
	const int grid = D == 1 ? grid_for<1>() : D == 2 ? grid_for<2>() : grid_for<3>();
	if (grid < 1)
		return sfail(CC_ERR_CUDA, "batch kernel cannot be resident");
	SV_CUDA(cudaLaunchCooperativeKernel(k, dim3(grid), dim3(cc::kFusedThreads), args, 0, st));
	return CC_OK;
}

// Plan and allocate a request; returns CC_OK and fills the slot.
int open_slot(const cc_request &r, int idx, int m, int nblk_cap, cudaStream_t st, Slot &s)
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
	cc::TabSpec g = cc::global_spec(p);
	double vol = 0, recip[9] = {0};
	cc::cell_geometry(d, basis, &vol, recip);
	const int64_t N = r.N;
	const int n = (int)(N * d);
	const int Npad = (int)((N + 31) / 32 * 32);
	const int nsplit = (int)((N + cc::kBatchSplit - 1) / cc::kBatchSplit);
	const int nks = std::max(1, (int)(p.segs.size() + cc::kBatchSegs - 1) / cc::kBatchSegs);
	Carve c;
	const size_t o_segs = c.take(sizeof(cc::Seg) * p.segs.size()), o_slotV = c.take(sizeof(double) * p.nslot),
	             o_tabP = c.take(sizeof(double2) * (size_t)(g.row | 1) * Npad),
	             o_tabE = c.take(sizeof(double2) * (size_t)g.row * Npad),
	             o_part = c.take(sizeof(double2) * (size_t)nsplit * p.nslot), o_u = c.take(sizeof(double2) * p.nslot),
	             o_ep = c.take(sizeof(double) * ((p.nslot + 255) / 256)),
	             o_pg = c.take(sizeof(double) * (size_t)nks * n), o_fc = c.take(sizeof(unsigned) * ((N + 31) / 32)),
	             o_x = c.take(8 * n), o_g = c.take(8 * n), o_d = c.take(8 * n), o_xt = c.take(8 * n), o_gt = c.take(8 * n),
	             o_S = c.take(8 * (size_t)n * m), o_Y = c.take(8 * (size_t)n * m),
	             o_lp = c.take(8 * (size_t)nblk_cap * cc::lb_ndots(m)), o_st = c.take(sizeof(cc::LbState));
	s.bytes = c.used;
	SV_CUDA(cudaMallocAsync(reinterpret_cast<void **>(&s.mem), c.used, st));
	unsigned char *b = s.mem;
	SV_CUDA(cudaMemcpyAsync(b + o_segs, p.segs.data(), sizeof(cc::Seg) * p.segs.size(), cudaMemcpyHostToDevice, st));
	SV_CUDA(cudaMemcpyAsync(b + o_slotV, p.slotV.data(), sizeof(double) * p.nslot, cudaMemcpyHostToDevice, st));
	SV_CUDA(cudaMemsetAsync(b + o_fc, 0, sizeof(unsigned) * ((N + 31) / 32), st));
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
	l.x = reinterpret_cast<double *>(b + o_x);
	l.g = reinterpret_cast<double *>(b + o_g);
	l.d = reinterpret_cast<double *>(b + o_d);
	l.xt = reinterpret_cast<double *>(b + o_xt);
	l.gt = reinterpret_cast<double *>(b + o_gt);
	l.S = reinterpret_cast<double *>(b + o_S);
	l.Y = reinterpret_cast<double *>(b + o_Y);
	l.part = reinterpret_cast<double *>(b + o_lp);
	l.st = reinterpret_cast<cc::LbState *>(b + o_st);
	cc::BInst &in = s.bi;
	std::memset(&in, 0, sizeof(in));
	in.frac = l.xt;
	in.E_out = &l.st->Et;
	in.gfrac_out = l.gt;
	in.F_out = nullptr;
	in.status = &l.st->status;
	in.N = (int)N;
	in.Npad = Npad;
	in.segs = reinterpret_cast<const cc::Seg *>(b + o_segs);
	in.ngroups = p.ngroups();
	in.nseg = (int)p.segs.size();
	in.nslot = p.nslot;
	in.slotV = reinterpret_cast<const double *>(b + o_slotV);
	in.rho_offset = 0.0;
	in.inv_vol = 1.0 / vol;
	in.shift = 0.0;
	in.spec = g;
	in.tabP = b + o_tabP;
	in.tabE = b + o_tabE;
	in.nsplit = nsplit;
	in.partial = reinterpret_cast<double2 *>(b + o_part);
	in.u_slot = reinterpret_cast<double2 *>(b + o_u);
	in.epart = reinterpret_cast<double *>(b + o_ep);
	in.nechunk = (p.nslot + 255) / 256;
	in.nks = nks;
	in.partialG = reinterpret_cast<double *>(b + o_pg);
	in.fcounters = reinterpret_cast<unsigned *>(b + o_fc);
	for (int k = 0; k < 9; k++)
		in.recip[k] = recip[k];
	in.fscale = 2.0 / vol;
	return CC_OK;
}

// device bytes a request will need (the same carve as open_slot, with the k-set size estimated from chi N d)
size_t estimate_bytes(const cc_request &r, int m, int nblk_cap)
{
	const double M = std::ceil(r.chi * (double)r.N * r.d) * 1.1 + 64;
	const double nseg = M / 4 + 64, nslot = nseg * 8;
	const double n = (double)r.N * r.d, Npad = (double)((r.N + 31) / 32 * 32);
	const double row = 128;
	const double nsplit = std::ceil(r.N / (double)cc::kBatchSplit), nks = std::ceil(nseg / cc::kBatchSegs);
	const double bytes = 16 * nseg + 8 * nslot + 2 * 16 * row * Npad + 16 * nsplit * nslot + 16 * nslot +
	                     8 * nks * n + 8 * n * (5 + 2 * m) + 8.0 * nblk_cap * cc::lb_ndots(m) + 8192;
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
	if (opts)
		o = *opts;
	if (o.max_slots < 1 || o.iters_per_round < 1 || o.history < 1 || o.history > cc::kLbMaxHist)
		return sfail(CC_ERR_ARG, "invalid serve options");
	for (int i = 0; i < count; i++)
		if (reqs[i].d < 1 || reqs[i].d > 3 || reqs[i].N < 1 || reqs[i].N > (1 << 24) || !reqs[i].frac0 ||
		    !(reqs[i].chi > 0) || (reqs[i].vtype < 0 || reqs[i].vtype > 3))
			return sfail(CC_ERR_ARG, "invalid request");
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
		return sfail(CC_ERR_NOGPU, "no CUDA device is visible");
	const int m = o.history;
	const int nblk_cap = 32;
	cudaStream_t st;
	SV_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
	// device descriptor arrays sized for max_slots
	cc::BInst *d_bi = nullptr;
	cc::LbInst *d_li = nullptr;
	int *d_pre = nullptr;
	unsigned *d_bar = nullptr;
	SV_CUDA(cudaMalloc(&d_bi, sizeof(cc::BInst) * o.max_slots));
	SV_CUDA(cudaMalloc(&d_li, sizeof(cc::LbInst) * o.max_slots));
	SV_CUDA(cudaMalloc(&d_pre, sizeof(int) * 4 * (o.max_slots + 1) * 3));
	SV_CUDA(cudaMalloc(&d_bar, 16));
	SV_CUDA(cudaMemset(d_bar, 0, 16));
	std::vector<int> order(count);
	for (int i = 0; i < count; i++)
		order[i] = i;
	std::stable_sort(order.begin(), order.end(),
	                 [&](int a, int b) { return reqs[a].arrival_s < reqs[b].arrival_s; });
	std::vector<Slot> active;
	size_t used = 0;
	int next = 0, done = 0;
	int rc = CC_OK;
	std::vector<cc::LbState> hs(o.max_slots);
	const auto t0 = std::chrono::steady_clock::now();
	auto now = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
	while (done < count && rc == CC_OK) {
		// 1. admission
		const double t = now();
		while (next < count && reqs[order[next]].arrival_s <= t && (int)active.size() < o.max_slots) {
			const cc_request &r = reqs[order[next]];
			const size_t need = estimate_bytes(r, m, nblk_cap);
			if (!active.empty() && used + need > o.hbm_budget)
				break;
			Slot s;
			if ((rc = open_slot(r, order[next], m, nblk_cap, st, s)))
				break;
			used += s.bytes;
			out[order[next]].t_admit = now();
			active.push_back(s);
			next++;
		}
		if (rc)
			break;
		if (active.empty()) {
			if (next < count) {
				const double wait = reqs[order[next]].arrival_s - now();
				if (wait > 0)
					std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.01)));
			}
			continue;
		}
		// 2. descriptors of the active set, grouped by dimension
		const int A = (int)active.size();
		std::vector<cc::LbInst> li(A);
		int maxn = 0;
		for (int a = 0; a < A; a++) {
			li[a] = active[a].li;
			maxn = std::max(maxn, li[a].n);
		}
		std::vector<cc::BInst> bi;
		std::vector<int> pre;
		struct G {
			int D, off, B, pre_off;
		};
		std::vector<G> groups;
		for (int D = 1; D <= 3; D++) {
			G g = {D, (int)bi.size(), 0, (int)pre.size()};
			for (int a = 0; a < A; a++)
				if (active[a].d == D) {
					bi.push_back(active[a].bi);
					g.B++;
				}
			if (!g.B)
				continue;
			std::vector<int> p4(4 * (g.B + 1), 0);
			for (int k = 0; k < g.B; k++) {
				const cc::BInst &in = bi[g.off + k];
				const int c[4] = {(in.N * in.spec.items + cc::kFusedThreads - 1) / cc::kFusedThreads,
				                  in.ngroups * in.nsplit, in.nechunk, ((in.N + 31) / 32) * in.nks};
				for (int ph = 0; ph < 4; ph++)
					p4[ph * (g.B + 1) + k + 1] = p4[ph * (g.B + 1) + k] + c[ph];
			}
			pre.insert(pre.end(), p4.begin(), p4.end());
			groups.push_back(g);
		}
		SV_CUDA(cudaMemcpyAsync(d_bi, bi.data(), sizeof(cc::BInst) * bi.size(), cudaMemcpyHostToDevice, st));
		SV_CUDA(cudaMemcpyAsync(d_li, li.data(), sizeof(cc::LbInst) * A, cudaMemcpyHostToDevice, st));
		SV_CUDA(cudaMemcpyAsync(d_pre, pre.data(), sizeof(int) * pre.size(), cudaMemcpyHostToDevice, st));
		const int nblk = std::max(1, std::min(nblk_cap, maxn / 2048));
		for (int it = 0; it < o.iters_per_round && rc == CC_OK; it++) {
			for (const G &g : groups) {
				cc::BatchArgs ba;
				ba.inst = d_bi + g.off;
				ba.B = g.B;
				for (int k = 0; k < 4; k++)
					ba.pre[k] = d_pre + g.pre_off + k * (g.B + 1);
				ba.bar = d_bar;
				if ((rc = launch_batch(g.D, ba, st)))
					break;
			}
			if (rc)
				break;
			cc::lb_dots_kernel<<<dim3(nblk, A), cc::kLbThreads, 0, st>>>(d_li, nblk);
			cc::lb_solve_kernel<<<A, cc::kLbSolveThreads, 0, st>>>(d_li, nblk);
			cc::lb_update_kernel<<<dim3((maxn + cc::kLbThreads - 1) / cc::kLbThreads, A), cc::kLbThreads, 0, st>>>(
			    d_li);
			if (cudaGetLastError() != cudaSuccess)
				rc = sfail(CC_ERR_CUDA, "serve: kernel launch failed");
		}
		if (rc)
			break;
		// 3. retire finished requests
		for (int a = 0; a < A; a++)
			SV_CUDA(cudaMemcpyAsync(&hs[a], active[a].li.st, offsetof(cc::LbState, w), cudaMemcpyDeviceToHost, st));
		SV_CUDA(cudaStreamSynchronize(st));
		unsigned bar[3];
		SV_CUDA(cudaMemcpy(bar, d_bar, sizeof(bar), cudaMemcpyDeviceToHost));
		if (bar[2]) {
			rc = sfail(CC_ERR_TIMEOUT, "serve: a grid barrier wait ran out");
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
	cudaFree(d_bi);
	cudaFree(d_li);
	cudaFree(d_pre);
	cudaFree(d_bar);
	cudaStreamDestroy(st);
	return rc;
}
