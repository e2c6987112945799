// cc_minimize.cu — the device-resident L-BFGS of one configuration (cc_minimize, cc_lbfgs_defaults in
// include/cc_gpu.h), which replaces the reference's Switch-0 RelaxStructure_NLOPT loop
// (potential/StructureOptimization.cpp:881-1090). Positions, gradient, the history pairs and every dot product stay on
// the device; blocks of iterations (one evaluation of the handle and the L-BFGS kernels of cc_lbfgs.cuh each) are
// captured in CUDA graphs, and the host reads one status word per block. The precision schedule (mixed, then FP64)
// runs through a batch of one (cc_batch.cu).
#include "cc_internal.h"

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

using namespace cci;

extern "C" {

int cc_lbfgs_defaults(cc_lbfgs_opts *o)
{
	if (!o)
		return fail(CC_ERR_ARG, "opts is null");
	o->history = 40;
	o->max_evals = 100000;
	o->stopval = -1e300;
	o->gtol = 0.0;
	o->ftol = 1e-15;
	o->precision = CC_PREC_FP64;
	o->switch_energy_per_particle = 1e-12;
	o->iters_per_check = 32;
	return CC_OK;
}

namespace {

// one iteration: evaluation at x_trial, dot products, solve, update
int lb_iteration(cc_handle *h, int64_t N, LbBuffers &b, int n, int nblk, int prec, cudaStream_t st)
{
	if (int rc = handle_eval(h, N, b.xt, &b.st->Et, nullptr, b.gt, false, prec, st))
		return rc;
	CC_CUDA(cc::lb_step(b.inst, 1, nblk, n, st, &b.host_inst));
	CC_CUDA(cudaGetLastError());
	return CC_OK;
}

int lb_graph(cc_handle *h, int64_t N, LbBuffers &b, int n, int nblk, int prec, int iters, cudaGraphExec_t *out)
{
	cudaGraph_t g = nullptr;
	CC_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
	int rc = CC_OK;
	for (int i = 0; i < iters && rc == CC_OK; i++)
		rc = lb_iteration(h, N, b, n, nblk, prec, h->stream);
	cudaError_t e = cudaStreamEndCapture(h->stream, &g);
	if (rc)
		return rc;
	if (e != cudaSuccess)
		return fail(CC_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
	e = cudaGraphInstantiate(out, g, 0);
	cudaGraphDestroy(g);
	if (e != cudaSuccess)
		return fail(CC_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
	return CC_OK;
}

}  // namespace

int cc_minimize(cc_handle *h, int64_t N, double *frac, const cc_lbfgs_opts *opts, cc_lbfgs_result *result)
{
	if (int rc = handle_check(h))
		return rc;
	cc_lbfgs_opts o;
	cc_lbfgs_defaults(&o);
	if (opts)
		o = *opts;
	if (N < 1 || !frac || o.history < 1 || o.history > cc::kLbMaxHist || o.iters_per_check < 1 ||
	    (o.precision != CC_PREC_FP64 && o.precision != CC_PREC_MIXED && o.precision != CC_PREC_SCHEDULE))
		return fail(CC_ERR_ARG, "invalid minimisation arguments");
	if ((int64_t)N * h->d > (1 << 30))
		return fail(CC_ERR_ARG, "too many variables");
	if (h->d_slotS0)   // the S2 form evaluates in FP64 only
		o.precision = CC_PREC_FP64;
	if (o.precision == CC_PREC_SCHEDULE && h->main.plan.nslot > 0) {
		// the precision schedule is per instance: run it as a batch of one (kept by the handle for this N)
		int rc2 = CC_OK;
		if (!h->sched_batch || h->sched_N != N) {
			if (h->sched_batch)
				cc_batch_destroy(h->sched_batch);
			h->sched_batch = nullptr;
			h->sched_N = -1;
			if ((rc2 = cc_batch_create(1, &h, &N, &h->sched_batch)) != CC_OK)
				return rc2;
			h->sched_N = N;
		}
		rc2 = cc_batch_minimize(h->sched_batch, &frac, &o, result);
		if (rc2 == CC_OK)
			rc2 = cc_set_positions(h, N, frac);
		return rc2;
	}
	const int d = h->d, n = (int)(N * d), m = o.history;
	const int nblk = cc::lb_blocks(n, 148);
	LbBuffers &b = h->lb;
	int rc;
	if (h->lb_n < n || h->lb_m < m || h->lb_nblk < nblk) {
		const int cn = std::max(n, h->lb_n), cm = std::max(m, h->lb_m), cb = std::max(nblk, h->lb_nblk);
		b.release();
		h->lb_n = h->lb_m = h->lb_nblk = 0;
		if ((rc = dev_alloc(&b.x, cn)) || (rc = dev_alloc(&b.g, cn)) || (rc = dev_alloc(&b.d, cn)) ||
		    (rc = dev_alloc(&b.xt, cn)) || (rc = dev_alloc(&b.gt, cn)) || (rc = dev_alloc(&b.S, (size_t)cm * cn)) ||
		    (rc = dev_alloc(&b.Y, (size_t)cm * cn)) || (rc = dev_alloc(&b.part, (size_t)cb * cc::lb_ndots(cm))) ||
		    (rc = dev_alloc(&b.st, 1)) || (rc = dev_alloc(&b.inst, 1))) {
			b.release();
			return rc;
		}
		h->lb_n = cn;
		h->lb_m = cm;
		h->lb_nblk = cb;
	}
	if ((rc = handle_reserve(h, N)))
		return rc;
	auto cleanup = [&](int code) {
		h->d_skip = nullptr;
		return code;
	};
	std::vector<double> x0((size_t)n);
	for (int i = 0; i < n; i++) {
		if (!std::isfinite(frac[i]))
			return cleanup(fail(CC_ERR_ARG, "non-finite start"));
		double v = frac[i] - std::floor(frac[i]);
		x0[i] = v - std::floor(v);
	}
	CC_CUDA(cudaMemcpy(b.x, x0.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
	CC_CUDA(cudaMemcpy(b.xt, x0.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
	CC_CUDA(cudaMemset(b.g, 0, sizeof(double) * n));
	CC_CUDA(cudaMemset(b.d, 0, sizeof(double) * n));
	cc::LbInst inst;
	inst.n = n;
	inst.m = m;
	inst.x = b.x;
	inst.g = b.g;
	inst.d = b.d;
	inst.xt = b.xt;
	inst.gt = b.gt;
	inst.S = b.S;
	inst.Y = b.Y;
	inst.part = b.part;
	inst.st = b.st;
	CC_CUDA(cudaMemcpy(b.inst, &inst, sizeof(inst), cudaMemcpyHostToDevice));
	b.host_inst = inst;
	// warm-up evaluations allocate the evaluation's work buffers before any capture
	const bool sched = o.precision == CC_PREC_SCHEDULE;
	const int prec0 = (o.precision == CC_PREC_FP64) ? CC_PREC_FP64 : CC_PREC_MIXED;
	if ((rc = handle_eval(h, N, b.xt, b.part, nullptr, b.gt, false, prec0, h->stream)) ||
	    (sched && (rc = handle_eval(h, N, b.xt, b.part, nullptr, b.gt, false, CC_PREC_FP64, h->stream))))
		return cleanup(rc);
	CC_CUDA(cudaStreamSynchronize(h->stream));
	// state: a virtual previous point of infinite energy, so the first evaluation is always accepted
	cc::LbState s0;
	std::memset(&s0, 0, sizeof(s0));
	s0.E = INFINITY;
	s0.gamma = 1.0;
	s0.stopval = o.stopval == CC_STOPVAL_GROUND_STATE ? 1e-20 * (double)N : o.stopval;
	s0.gtol = o.gtol;
	s0.ftol = o.ftol;
	s0.max_evals = o.max_evals;
	s0.m = m;
	s0.newslot = -1;
	CC_CUDA(cudaMemcpy(b.st, &s0, sizeof(s0), cudaMemcpyHostToDevice));
	h->d_skip = &b.st->status;
	cudaGraphExec_t gexec[2] = {nullptr, nullptr};
	auto destroy_graphs = [&]() {
		for (auto &ge : gexec)
			if (ge)
				cudaGraphExecDestroy(ge);
	};
	if ((rc = lb_graph(h, N, b, n, nblk, prec0, o.iters_per_check, &gexec[0])) ||
	    (sched && (rc = lb_graph(h, N, b, n, nblk, CC_PREC_FP64, o.iters_per_check, &gexec[1])))) {
		destroy_graphs();
		return cleanup(rc);
	}
	int stage = 0;
	cc::LbState hs;
	const int64_t max_rounds = o.max_evals / o.iters_per_check + 2;
	for (int64_t round = 0; round < max_rounds; round++) {
		cudaError_t e = cudaGraphLaunch(gexec[stage], h->stream);
		if (e == cudaSuccess)
			e = cudaMemcpyAsync(&hs, b.st, sizeof(hs), cudaMemcpyDeviceToHost, h->stream);
		if (e == cudaSuccess)
			e = cudaStreamSynchronize(h->stream);
		if (e != cudaSuccess) {
			destroy_graphs();
			return cleanup(fail(CC_ERR_CUDA, std::string("minimisation: ") + cudaGetErrorString(e)));
		}
		if (hs.status != cc::kLbRunning)
			break;
		if (sched && stage == 0 && std::isfinite(hs.E) && hs.E <= o.switch_energy_per_particle * (double)N)
			stage = 1;
	}
	destroy_graphs();
	h->d_skip = nullptr;
	// result: the last accepted point, wrapped into [0,1), and its FP64 energy
	CC_CUDA(cudaMemcpy(x0.data(), b.x, sizeof(double) * n, cudaMemcpyDeviceToHost));
	for (int i = 0; i < n; i++) {
		double v = x0[i] - std::floor(x0[i]);
		frac[i] = v - std::floor(v);
	}
	if ((rc = cc_set_positions(h, N, frac)))
		return rc;
	double E = 0.0;
	if ((rc = cc_energy_grad(h, &E, nullptr, CC_PREC_FP64)))
		return rc;
	if (result) {
		result->E = E;
		result->evals = hs.evals;
		result->iters = hs.iters;
		result->status = hs.status == cc::kLbRunning ? cc::kLbMaxEval : hs.status;
	}
	return CC_OK;
}

}  // extern "C"
