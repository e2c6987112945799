// cc_batch.cu — batches of independent configurations (cc_batch_* in include/cc_gpu.h).
//
// A batch evaluates many configurations of uneven size and dimension together: ONE launch of the fused batch kernel
// (cc_mbatch_kernel, cc_kernels.cuh) per energy + gradient step, whose work queue holds the rho blocks, split-reduction
// chunks and force blocks of every instance; per-instance completion counts order the three phases of an instance.
// Its batched L-BFGS (cc_batch_minimize) keeps every instance's positions, gradient and history on the device and
// captures blocks of iterations (one fused evaluation and the L-BFGS kernels each) in CUDA graphs. The reference
// evaluates one configuration per Objective call (potential/StructureOptimization.cpp:447-578).
#include "cc_internal.h"
#include "cc_multi_launch.h"

#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

using namespace cci;

namespace {

// carve 256-byte aligned pieces out of one device allocation
struct Arena {
	unsigned char *base = nullptr;
	size_t used = 0, cap = 0;
	size_t take(size_t bytes)
	{
		const size_t off = used;
		used += (bytes + 255) / 256 * 256;
		return off;
	}
	template <class T> T *at(size_t off) { return reinterpret_cast<T *>(base + off); }
};

using cc::kBatchChunk;
using cc::kBatchPerSplit;
using cc::kBatchSegsPerSplit;

// an instance's evaluation buffers in the batch arena
struct BatchBufs {
	size_t o_part, o_rho, o_u, o_eb, o_tk, o_pg, o_fc;
};

// tile shapes the autotuner times: particles per rho block, segments per force block
constexpr int kTuneSplits[] = {32, 64, 128, 256, 512, 1024};
constexpr int kTuneSegs[] = {32, 64, 128, 256, 512, 1024};

// dynamic shared memory the fused kernel is allowed (its largest table rows in FP64, any dimension)
size_t mbatch_smem_cap()
{
	return std::max(rho_smem<double2>(cc::kMaxRow, kBatchChunk, 8), force_smem<double2>(cc::kMaxRow, 3));
}

template <int MODE> int mbatch_launch_t(const cc::MBatchArgs &a, size_t smem, cudaStream_t st)
{
	static const cudaError_t attr = cudaFuncSetAttribute(
	    cc::cc_mbatch_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mbatch_smem_cap());
	if (attr != cudaSuccess)
		return fail(CC_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(attr));
	// resident blocks per SM for this shared memory size (looked up once per size)
	static std::mutex mu;
	static std::map<size_t, int> per_sm;
	int resident = 0;
	{
		std::lock_guard<std::mutex> lk(mu);
		auto it = per_sm.find(smem);
		if (it == per_sm.end()) {
			int n = 0;
			CC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, cc::cc_mbatch_kernel<MODE>, cc::kMBatchThreads,
			                                                      smem));
			it = per_sm.emplace(smem, std::max(1, n)).first;
		}
		resident = it->second * sm_count();
	}
	const int total = a.total[0] + a.total[1] + a.total[2];
	if (total <= 0)
		return CC_OK;
	CC_CUDA(launch_pdl_n(cc::cc_mbatch_kernel<MODE>, dim3(std::min(total, resident)), dim3(cc::kMBatchThreads), smem,
	                     st, a));
	return CC_OK;
}

}  // namespace

int cc::launch_mbatch(int mode, const MBatchArgs &a, int rho_row, int force_row, int maxd, cudaStream_t st)
{
	if (a.B < 1)
		return CC_OK;
	const size_t smem = std::max(rho_smem<double2>(rho_row, kBatchChunk, 8), force_smem<double2>(force_row, maxd));
	switch (mode) {
	case 0: return mbatch_launch_t<0>(a, smem, st);
	case 1: return mbatch_launch_t<1>(a, smem, st);
	default: return mbatch_launch_t<2>(a, smem, st);
	}
}

struct cc_batch {
	std::vector<cc_handle *> h;
	std::vector<int64_t> N;
	std::vector<int> order;                  // instances by decreasing work: their order in the fused launch
	Arena arena;
	std::vector<size_t> off_frac, off_F, off_E;
	std::vector<BatchBufs> bufs;
	int per_split = 0, segs_per_split = 0;   // the tile shape in use
	cudaStream_t stream = nullptr;
	// the fused launch's descriptors in `order`: set 0 evaluates the batch positions into the batch outputs, set 1 a
	// minimisation's trial points into its L-BFGS buffers
	cc::RhoArgs *d_rho[2] = {nullptr, nullptr};
	cc::ReduceArgs *d_red[2] = {nullptr, nullptr};
	cc::ForceArgs *d_force[2] = {nullptr, nullptr};
	int *d_dim = nullptr;                    // B
	int *d_pre = nullptr;                    // 4 x (B + 1): rho, reduce, force, reduce + force items per instance
	int *d_shape = nullptr;                  // 3 x B
	unsigned *d_queue = nullptr;             // 2 words
	unsigned *d_count = nullptr;             // 3 x B completion counts + 1 error word
	int total[3] = {0, 0, 0};
	int rho_row = 1, force_row = 1, maxd = 1;
	unsigned wait_spins = 0, wait_phantom = 0;   // cc_batch_set_wait_test
	std::vector<cc::RhoArgs> rho;            // host copies of set 0 (in `order`)
	std::vector<cc::ReduceArgs> red;
	std::vector<cc::ForceArgs> force;
	// L-BFGS state of cc_batch_minimize, kept between calls (grow-only): a minimisation makes no allocation call
	// into the CUDA driver once the batch has run one
	unsigned char *lb_base = nullptr;
	size_t lb_cap = 0;
	cc::LbInst *d_lb = nullptr;              // the instances in `order`
	cc::LbBrief *d_brief = nullptr;
	int d_lb_cap = 0;
};

namespace {

cc::MBatchArgs batch_args(const cc_batch *b, int set, int want_stage)
{
	cc::MBatchArgs a;
	a.rho = b->d_rho[set];
	a.red = b->d_red[set];
	a.force = b->d_force[set];
	a.dim = b->d_dim;
	a.pre = b->d_pre;
	a.shape = b->d_shape;
	a.B = (int)b->order.size();
	for (int k = 0; k < 3; k++)
		a.total[k] = b->total[k];
	a.want_stage = want_stage;
	a.queue = b->d_queue;
	a.count = b->d_count;
	a.spins = b->wait_spins;
	a.phantom = b->wait_phantom;
	return a;
}

// (Re)build the evaluation descriptors (set 0) for a tile shape: per_split particles per rho block and force splits
// of about segs_per_split segments; the arena holds the buffers of every candidate shape.
int batch_build(cc_batch *b, int per_split, int segs_per_split)
{
	const int B = (int)b->order.size();
	std::vector<int> pre(4 * (B + 1), 0), shape(3 * B, 0), dim(B, 0);
	b->rho.clear();
	b->red.clear();
	b->force.clear();
	b->rho_row = b->force_row = 1;
	b->maxd = 1;
	for (int k = 0; k < B; k++) {
		const int i = b->order[k];
		cc_handle *h = b->h[i];
		const cc::Plan &p = h->main.plan;
		const BatchBufs &q = b->bufs[i];
		const int64_t n = b->N[i];
		const int nsplit = (int)((n + per_split - 1) / per_split);
		// reduce items of kWideSlots slots each (their energy terms are the force items' eblock entries)
		const int nchunks = (p.nslot + cc::kWideSlots - 1) / cc::kWideSlots, pgroups = (int)((n + 31) / 32);
		const DevSplits *f = nullptr;
		const int want = (int)std::max<int64_t>(1, (p.real_segs + segs_per_split - 1) / segs_per_split);
		if (int rc = get_splits(h->main, want, &f))
			return rc;
		cc::RhoArgs ra = {};
		ra.frac = b->arena.at<double>(b->off_frac[i]);
		ra.N = (int)n;
		ra.per_split = per_split;
		ra.chunk = kBatchChunk;
		ra.segs = h->main.segs;
		ra.bstart = h->main.bstart;
		ra.bspec = h->main.bspec;
		ra.nseg = (int)p.segs.size();
		ra.nslot = p.nslot;
		ra.partial = b->arena.at<double2>(q.o_part);
		cc::ReduceArgs rr = {};
		rr.partial = ra.partial;
		rr.nsplit = nsplit;
		rr.nslot = p.nslot;
		rr.slotV = h->main.slotV;
		rr.rho_offset = h->rho_offset;
		rr.rho_slot = b->arena.at<double2>(q.o_rho);
		rr.u_slot = b->arena.at<double2>(q.o_u);
		rr.eblock = b->arena.at<double>(q.o_eb);
		rr.ticket = b->arena.at<unsigned>(q.o_tk);
		rr.inv_vol = 1.0 / h->volume;
		rr.shift = h->shift;
		rr.E_out = b->arena.at<double>(b->off_E[i]);
		rr.finalize = 0;   // the force items sum the energy terms
		cc::ForceArgs fa = {};
		fa.frac = ra.frac;
		fa.N = ra.N;
		fa.segs = h->main.segs;
		fa.kstart = f->kstart;
		fa.kspec = f->kspec;
		fa.nksplit = f->host.count();
		fa.u_slot = rr.u_slot;
		fa.nseg = ra.nseg;
		fa.partialG = b->arena.at<double>(q.o_pg);
		fa.counters = b->arena.at<unsigned>(q.o_fc);
		for (int c = 0; c < 9; c++)
			fa.recip[c] = h->recip[c];
		fa.fscale = 2.0 / h->volume;
		fa.F_out = b->arena.at<double>(b->off_F[i]);
		fa.gfrac_out = nullptr;
		fa.eblock = rr.eblock;
		fa.neblock = nchunks;
		fa.inv_vol = rr.inv_vol;
		fa.shift = rr.shift;
		fa.E_out = rr.E_out;
		b->rho.push_back(ra);
		b->red.push_back(rr);
		b->force.push_back(fa);
		const int c[3] = {p.nbgroups() * nsplit, nchunks, pgroups * fa.nksplit};
		const int sh[3] = {p.nbgroups(), nchunks, pgroups};
		for (int ph = 0; ph < 3; ph++) {
			pre[ph * (B + 1) + k + 1] = pre[ph * (B + 1) + k] + c[ph];
			shape[ph * B + k] = sh[ph];
		}
		dim[k] = h->d;
		b->rho_row = std::max(b->rho_row, p.block_max_row);
		b->force_row = std::max(b->force_row, f->host.max_row);
		b->maxd = std::max(b->maxd, h->d);
	}
	for (int ph = 0; ph < 3; ph++)
		b->total[ph] = pre[ph * (B + 1) + B];
	for (int k = 0; k < B; k++)   // each instance's reduce and force items, consecutive in the queue
		pre[3 * (B + 1) + k + 1] = pre[3 * (B + 1) + k] + (pre[(B + 1) + k + 1] - pre[(B + 1) + k]) +
		                           (pre[2 * (B + 1) + k + 1] - pre[2 * (B + 1) + k]);
	int rc;
	if ((rc = upload_into(b->d_rho[0], b->rho)) || (rc = upload_into(b->d_red[0], b->red)) ||
	    (rc = upload_into(b->d_force[0], b->force)) || (rc = upload_into(b->d_pre, pre)) ||
	    (rc = upload_into(b->d_shape, shape)) || (rc = upload_into(b->d_dim, dim)))
		return rc;
	b->per_split = per_split;
	b->segs_per_split = segs_per_split;
	return CC_OK;
}

// One fused launch evaluating every instance (descriptor set `set`). Precision CC_PREC_SCHEDULE evaluates each
// instance at the precision of its stage word; CC_PREC_FP64 / CC_PREC_MIXED skip instances whose stage word (set 1
// only) differs from 1 / 0.
int batch_eval(cc_batch *b, int set, int precision, cudaStream_t st)
{
	const int mode = precision == CC_PREC_SCHEDULE ? 2 : precision == CC_PREC_MIXED ? 1 : 0;
	return cc::launch_mbatch(mode, batch_args(b, set, mode == 1 ? 0 : 1), b->rho_row, b->force_row, b->maxd, st);
}

// A bounded wait of the fused kernel that ran out leaves the error word set: report it (after a synchronisation of
// the batch's stream) and clear it.
int batch_check_wait(cc_batch *b)
{
	unsigned err = 0;
	const unsigned *w = b->d_count + 3 * b->order.size();
	CC_CUDA(cudaMemcpy(&err, w, sizeof(unsigned), cudaMemcpyDeviceToHost));
	if (err) {
		CC_CUDA(cudaMemset(const_cast<unsigned *>(w), 0, sizeof(unsigned)));
		return fail(CC_ERR_TIMEOUT, "a bounded wait of the fused batch kernel ran out");
	}
	return CC_OK;
}

}  // namespace

extern "C" {

int cc_batch_create(int count, cc_handle *const *handles, const int64_t *N, cc_batch **out)
{
	if (!out || count < 1 || !handles || !N)
		return fail(CC_ERR_ARG, "invalid batch arguments");
	*out = nullptr;
	for (int i = 0; i < count; i++) {
		if (!handles[i] || N[i] < 1 || N[i] > (1 << 26) || handles[i]->main.plan.nslot == 0)
			return fail(CC_ERR_ARG, "every instance needs a handle with constraints and 1 <= N <= 2^26");
		if (handles[i]->d_slotS0)
			return fail(CC_ERR_ARG, "batches hold the plain collective-coordinate form only");
	}
	cc_batch *b = new cc_batch();
	b->h.assign(handles, handles + count);
	b->N.assign(N, N + count);
	// per instance: buffers sized for every tile shape the autotuner may choose (the most particle splits and force
	// splits among the candidates), carved out of one arena
	b->off_frac.resize(count);
	b->off_F.resize(count);
	b->off_E.resize(count);
	b->bufs.resize(count);
	for (int i = 0; i < count; i++) {
		cc_handle *h = handles[i];
		const cc::Plan &p = h->main.plan;
		const int64_t n = N[i];
		BatchBufs &q = b->bufs[i];
		int max_nks = 1;
		for (int segs : kTuneSegs) {
			const DevSplits *f = nullptr;
			const int want = (int)std::max<int64_t>(1, (p.real_segs + segs - 1) / segs);
			if (int rc = get_splits(h->main, want, &f)) {
				delete b;
				return rc;
			}
			max_nks = std::max(max_nks, f->host.count());
		}
		const int max_nsplit = (int)((n + kTuneSplits[0] - 1) / kTuneSplits[0]);
		const int nchunks = (p.nslot + 31) / 32, pgroups = (int)((n + 31) / 32);
		b->off_frac[i] = b->arena.take(sizeof(double) * n * h->d);
		b->off_F[i] = b->arena.take(sizeof(double) * n * h->d);
		b->off_E[i] = b->arena.take(sizeof(double));
		q.o_part = b->arena.take(sizeof(double2) * (size_t)max_nsplit * p.nslot);
		q.o_rho = b->arena.take(sizeof(double2) * p.nslot);
		q.o_u = b->arena.take(sizeof(double2) * p.nslot);
		q.o_eb = b->arena.take(sizeof(double) * nchunks);
		q.o_tk = b->arena.take(sizeof(unsigned));
		q.o_pg = b->arena.take(sizeof(double) * (size_t)max_nks * n * h->d);
		q.o_fc = b->arena.take(sizeof(unsigned) * pgroups);
	}
	int rc;
	if ((rc = dev_alloc(&b->arena.base, b->arena.used))) {
		cc_batch_destroy(b);
		return rc;
	}
	b->arena.cap = b->arena.used;
	if (cudaMemset(b->arena.base, 0, b->arena.used) != cudaSuccess ||
	    cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
		cc_batch_destroy(b);
		return fail(CC_ERR_CUDA, "batch initialisation failed");
	}
	// instances by decreasing work: the work queue hands out the longest items first
	b->order.resize(count);
	for (int i = 0; i < count; i++)
		b->order[i] = i;
	std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) {
		return (double)N[x] * handles[x]->main.plan.real_segs > (double)N[y] * handles[y]->main.plan.real_segs;
	});
	const int B = count;
	if ((rc = dev_alloc(&b->d_rho[0], B)) || (rc = dev_alloc(&b->d_red[0], B)) || (rc = dev_alloc(&b->d_force[0], B)) ||
	    (rc = dev_alloc(&b->d_rho[1], B)) || (rc = dev_alloc(&b->d_red[1], B)) || (rc = dev_alloc(&b->d_force[1], B)) ||
	    (rc = dev_alloc(&b->d_pre, 4 * (B + 1))) || (rc = dev_alloc(&b->d_shape, 3 * B)) ||
	    (rc = dev_alloc(&b->d_dim, B)) || (rc = dev_alloc(&b->d_queue, 2)) || (rc = dev_alloc(&b->d_count, 3 * B + 1)) ||
	    (rc = (cudaMemset(b->d_queue, 0, 2 * sizeof(unsigned)) == cudaSuccess &&
	                   cudaMemset(b->d_count, 0, (3 * B + 1) * sizeof(unsigned)) == cudaSuccess
	               ? CC_OK
	               : fail(CC_ERR_CUDA, "batch initialisation failed")))) {
		cc_batch_destroy(b);
		return rc;
	}
	if ((rc = batch_build(b, kBatchPerSplit, kBatchSegsPerSplit))) {
		cc_batch_destroy(b);
		return rc;
	}
	*out = b;
	return CC_OK;
}

int cc_batch_autotune(cc_batch *b, int reps, int *per_split, int *segs_per_split)
{
	if (!b || reps < 1)
		return fail(CC_ERR_ARG, "invalid autotune arguments");
	cudaEvent_t e0, e1;
	CC_CUDA(cudaEventCreate(&e0));
	CC_CUDA(cudaEventCreate(&e1));
	float best = 1e30f;
	int bp = b->per_split, bs = b->segs_per_split, rc = CC_OK;
	for (int ps : kTuneSplits)
		for (int sg : kTuneSegs) {
			if ((rc = batch_build(b, ps, sg)) || (rc = batch_eval(b, 0, CC_PREC_FP64, b->stream)))
				break;
			if (cudaEventRecord(e0, b->stream) != cudaSuccess) {
				rc = fail(CC_ERR_CUDA, "cudaEventRecord failed");
				break;
			}
			for (int r = 0; r < reps && rc == CC_OK; r++)
				rc = batch_eval(b, 0, CC_PREC_FP64, b->stream);
			if (rc)
				break;
			float ms = 0.0f;
			if (cudaEventRecord(e1, b->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
			    cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
				rc = fail(CC_ERR_CUDA, "autotune timing failed");
				break;
			}
			if (ms < best) {
				best = ms;
				bp = ps;
				bs = sg;
			}
		}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	if (rc)
		return rc;
	if ((rc = batch_check_wait(b)))
		return rc;
	if ((rc = batch_build(b, bp, bs)))
		return rc;
	if (per_split)
		*per_split = bp;
	if (segs_per_split)
		*segs_per_split = bs;
	return CC_OK;
}

int cc_batch_destroy(cc_batch *b)
{
	if (!b)
		return CC_OK;
	if (b->stream)
		cudaStreamSynchronize(b->stream);
	for (int w = 0; w < 2; w++) {
		cudaFree(b->d_rho[w]);
		cudaFree(b->d_red[w]);
		cudaFree(b->d_force[w]);
	}
	cudaFree(b->d_dim);
	cudaFree(b->d_pre);
	cudaFree(b->d_shape);
	cudaFree(b->d_queue);
	cudaFree(b->d_count);
	cudaFree(b->arena.base);
	cudaFree(b->lb_base);
	cudaFree(b->d_lb);
	cudaFree(b->d_brief);
	if (b->stream)
		cudaStreamDestroy(b->stream);
	delete b;
	return CC_OK;
}

int cc_batch_set_positions(cc_batch *b, const double *const *frac)
{
	if (!b || !frac)
		return fail(CC_ERR_ARG, "invalid batch arguments");
	for (size_t i = 0; i < b->h.size(); i++) {
		const size_t n = (size_t)b->N[i] * b->h[i]->d;
		std::vector<double> w(n);
		for (size_t k = 0; k < n; k++) {
			if (!std::isfinite(frac[i][k]))
				return fail(CC_ERR_ARG, "non-finite fractional coordinate");
			double v = frac[i][k] - std::floor(frac[i][k]);
			w[k] = v - std::floor(v);
		}
		CC_CUDA(cudaMemcpyAsync(b->arena.at<double>(b->off_frac[i]), w.data(), sizeof(double) * n,
		                        cudaMemcpyHostToDevice, b->stream));
		CC_CUDA(cudaStreamSynchronize(b->stream));
	}
	return CC_OK;
}

int cc_batch_set_wait_test(cc_batch *b, unsigned polls, int phantom)
{
	if (!b || phantom < 0)
		return fail(CC_ERR_ARG, "invalid wait test arguments");
	b->wait_spins = polls;
	b->wait_phantom = (unsigned)phantom;
	return CC_OK;
}

int cc_batch_eval_device(cc_batch *b, int precision, void *stream)
{
	if (!b)
		return fail(CC_ERR_ARG, "null batch");
	if (int rc = check_prec(precision))
		return rc;
	return batch_eval(b, 0, precision, stream ? static_cast<cudaStream_t>(stream) : b->stream);
}

int cc_batch_energy_grad(cc_batch *b, double *E, double *const *F, int precision)
{
	if (!b || !E)
		return fail(CC_ERR_ARG, "invalid batch arguments");
	if (int rc = cc_batch_eval_device(b, precision, b->stream))
		return rc;
	CC_CUDA(cudaStreamSynchronize(b->stream));
	if (int rc = batch_check_wait(b))
		return rc;
	for (size_t i = 0; i < b->h.size(); i++) {
		CC_CUDA(cudaMemcpy(&E[i], b->arena.at<double>(b->off_E[i]), sizeof(double), cudaMemcpyDeviceToHost));
		if (F && F[i])
			CC_CUDA(cudaMemcpy(F[i], b->arena.at<double>(b->off_F[i]), sizeof(double) * b->N[i] * b->h[i]->d,
			                   cudaMemcpyDeviceToHost));
	}
	return CC_OK;
}

int cc_batch_minimize(cc_batch *b, double *const *frac, const cc_lbfgs_opts *opts, cc_lbfgs_result *results)
{
	if (!b || !frac)
		return fail(CC_ERR_ARG, "invalid batch arguments");
	cc_lbfgs_opts o;
	cc_lbfgs_defaults(&o);
	if (opts)
		o = *opts;
	if (o.history < 1 || o.history > cc::kLbMaxHist || o.iters_per_check < 1 ||
	    (o.precision != CC_PREC_FP64 && o.precision != CC_PREC_MIXED && o.precision != CC_PREC_SCHEDULE))
		return fail(CC_ERR_ARG, "invalid minimisation options");
	const int count = (int)b->h.size(), m = o.history;
	for (int i = 0; i < count; i++) {
		const size_t n = (size_t)b->N[i] * b->h[i]->d;
		for (size_t k = 0; k < n; k++)
			if (!std::isfinite(frac[i][k]))
				return fail(CC_ERR_ARG, "non-finite start");
	}
	int maxn = 0;
	for (int i = 0; i < count; i++)
		maxn = std::max(maxn, (int)(b->N[i] * b->h[i]->d));
	const int nblk = cc::lb_blocks(maxn, cc::kLbMaxBlocks);
	// L-BFGS buffers of every instance in one allocation
	Arena ar;
	std::vector<size_t> ox(count), og(count), od(count), oxt(count), ogt(count), oS(count), oY(count), op(count),
	    ost(count);
	for (int i = 0; i < count; i++) {
		const size_t n = (size_t)b->N[i] * b->h[i]->d;
		ox[i] = ar.take(8 * n);
		og[i] = ar.take(8 * n);
		od[i] = ar.take(8 * n);
		oxt[i] = ar.take(8 * n);
		ogt[i] = ar.take(8 * n);
		oS[i] = ar.take(8 * n * m);
		oY[i] = ar.take(8 * n * m);
		op[i] = ar.take(8 * (size_t)nblk * cc::lb_ndots(m));
		ost[i] = ar.take(sizeof(cc::LbState));
	}
	int rc;
	if (b->lb_cap < ar.used) {
		cudaFree(b->lb_base);
		b->lb_base = nullptr;
		b->lb_cap = 0;
		if ((rc = dev_alloc(&b->lb_base, ar.used)))
			return rc;
		b->lb_cap = ar.used;
	}
	if (b->d_lb_cap < count) {
		cudaFree(b->d_lb);
		cudaFree(b->d_brief);
		b->d_lb = nullptr;
		b->d_brief = nullptr;
		b->d_lb_cap = 0;
		if ((rc = dev_alloc(&b->d_lb, (size_t)count)) || (rc = dev_alloc(&b->d_brief, count)))
			return rc;
		b->d_lb_cap = count;
	}
	ar.base = b->lb_base;
	std::vector<cc::LbInst> lbi(count);   // by instance index
	cc::LbState s0;
	std::memset(&s0, 0, sizeof(s0));
	s0.E = INFINITY;
	s0.gamma = 1.0;
	s0.gtol = o.gtol;
	s0.ftol = o.ftol;
	s0.max_evals = o.max_evals;
	s0.m = m;
	s0.newslot = -1;
	for (int i = 0; i < count; i++) {
		const size_t n = (size_t)b->N[i] * b->h[i]->d;
		cc::LbInst &l = lbi[i];
		l.n = (int)n;
		l.m = m;
		l.x = ar.at<double>(ox[i]);
		l.g = ar.at<double>(og[i]);
		l.d = ar.at<double>(od[i]);
		l.xt = ar.at<double>(oxt[i]);
		l.gt = ar.at<double>(ogt[i]);
		l.S = ar.at<double>(oS[i]);
		l.Y = ar.at<double>(oY[i]);
		l.part = ar.at<double>(op[i]);
		l.st = ar.at<cc::LbState>(ost[i]);
		std::vector<double> x0(n);
		for (size_t k = 0; k < n; k++) {
			double v = frac[i][k] - std::floor(frac[i][k]);
			x0[k] = v - std::floor(v);
		}
		CC_CUDA(cudaMemcpy(l.x, x0.data(), 8 * n, cudaMemcpyHostToDevice));
		CC_CUDA(cudaMemcpy(l.xt, x0.data(), 8 * n, cudaMemcpyHostToDevice));
		CC_CUDA(cudaMemset(l.g, 0, 8 * n));
		CC_CUDA(cudaMemset(l.d, 0, 8 * n));
		s0.stopval = o.stopval == CC_STOPVAL_GROUND_STATE ? 1e-20 * (double)b->N[i] : o.stopval;
		s0.sched = o.precision == CC_PREC_SCHEDULE;
		s0.stage = o.precision == CC_PREC_FP64 ? 1 : 0;
		s0.switch_E = o.switch_energy_per_particle * (double)b->N[i];
		CC_CUDA(cudaMemcpy(l.st, &s0, sizeof(s0), cudaMemcpyHostToDevice));
	}
	// the L-BFGS instances in the launch order, and the minimisation descriptors (set 1): evaluate at x_trial into
	// the L-BFGS buffers, skip finished instances
	std::vector<cc::LbInst> lbo(count);
	std::vector<cc::RhoArgs> ra = b->rho;
	std::vector<cc::ReduceArgs> rr = b->red;
	std::vector<cc::ForceArgs> fa = b->force;
	for (int k = 0; k < count; k++) {
		const int i = b->order[k];
		lbo[k] = lbi[i];
		const int *status = &lbi[i].st->status, *stage = &lbi[i].st->stage;
		ra[k].frac = lbi[i].xt;
		ra[k].skip = status;
		ra[k].stage = stage;
		rr[k].E_out = &lbi[i].st->Et;
		rr[k].skip = status;
		rr[k].stage = stage;
		fa[k].frac = lbi[i].xt;
		fa[k].E_out = &lbi[i].st->Et;
		fa[k].gfrac_out = lbi[i].gt;
		fa[k].F_out = nullptr;
		fa[k].skip = status;
		fa[k].stage = stage;
	}
	if ((rc = upload_into(b->d_lb, lbo)) || (rc = upload_into(b->d_rho[1], ra)) || (rc = upload_into(b->d_red[1], rr)) ||
	    (rc = upload_into(b->d_force[1], fa)))
		return rc;
	cudaStream_t st = b->stream;
	const bool sched = o.precision == CC_PREC_SCHEDULE;
	// schedule: each instance at its stage's precision while some instance is in the mixed stage; then FP64 only
	auto iterations = [&](int prec) -> int {
		for (int it = 0; it < o.iters_per_check; it++) {
			if (int r2 = batch_eval(b, 1, prec, st))
				return r2;
			CC_CUDA(cc::lb_step(b->d_lb, count, nblk, maxn, st, count == 1 ? &lbo[0] : nullptr));
			CC_CUDA(cudaGetLastError());
		}
		return CC_OK;
	};
	auto make_graph = [&](int prec, cudaGraphExec_t *out) -> int {
		cudaGraph_t g = nullptr;
		CC_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
		const int r2 = iterations(prec);
		cudaError_t e = cudaStreamEndCapture(st, &g);
		if (r2)
			return r2;
		if (e != cudaSuccess)
			return fail(CC_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
		e = cudaGraphInstantiate(out, g, 0);
		cudaGraphDestroy(g);
		if (e != cudaSuccess)
			return fail(CC_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
		return CC_OK;
	};
	cudaGraphExec_t gexec[2] = {nullptr, nullptr};
	auto destroy_graphs = [&]() {
		for (auto &ge : gexec)
			if (ge)
				cudaGraphExecDestroy(ge);
	};
	// kernel attributes and occupancy are looked up outside the capture: one eager evaluation of every mode in use
	if ((rc = batch_eval(b, 0, o.precision, st)) || (sched && (rc = batch_eval(b, 0, CC_PREC_FP64, st))))
		return rc;
	CC_CUDA(cudaStreamSynchronize(st));
	if ((rc = make_graph(o.precision, &gexec[0])) || (sched && (rc = make_graph(CC_PREC_FP64, &gexec[1])))) {
		destroy_graphs();
		return rc;
	}
	std::vector<cc::LbBrief> hs(count);   // in launch order
	int stage = 0;
	const int64_t max_rounds = o.max_evals / o.iters_per_check + 2;
	for (int64_t round = 0; round < max_rounds; round++) {
		cudaError_t e = cudaGraphLaunch(gexec[stage], st);
		if (e == cudaSuccess)
			e = cudaStreamSynchronize(st);
		if (e != cudaSuccess) {
			destroy_graphs();
			return fail(CC_ERR_CUDA, std::string("batch minimisation: ") + cudaGetErrorString(e));
		}
		if ((rc = batch_check_wait(b))) {
			destroy_graphs();
			return rc;
		}
		bool running = false, any_mixed = false;
		cc::lb_brief_kernel<<<(count + 127) / 128, 128, 0, st>>>(b->d_lb, count, b->d_brief);
		e = cudaGetLastError();
		if (e == cudaSuccess)
			e = cudaMemcpyAsync(hs.data(), b->d_brief, sizeof(cc::LbBrief) * count, cudaMemcpyDeviceToHost, st);
		if (e == cudaSuccess)
			e = cudaStreamSynchronize(st);
		if (e != cudaSuccess) {
			destroy_graphs();
			return fail(CC_ERR_CUDA, std::string("batch minimisation status: ") + cudaGetErrorString(e));
		}
		for (int k = 0; k < count; k++) {
			running |= hs[k].status == cc::kLbRunning;
			any_mixed |= hs[k].status == cc::kLbRunning && hs[k].stage == 0;
		}
		if (!running)
			break;
		if (sched && stage == 0 && !any_mixed)
			stage = 1;
	}
	destroy_graphs();
	// results: positions wrapped into [0,1), FP64 energies of the results (one batched evaluation)
	std::vector<const double *> fr(count);
	for (int i = 0; i < count; i++) {
		const size_t n = (size_t)b->N[i] * b->h[i]->d;
		CC_CUDA(cudaMemcpy(frac[i], lbi[i].x, 8 * n, cudaMemcpyDeviceToHost));
		for (size_t k = 0; k < n; k++) {
			double v = frac[i][k] - std::floor(frac[i][k]);
			frac[i][k] = v - std::floor(v);
		}
		fr[i] = frac[i];
	}
	if ((rc = cc_batch_set_positions(b, fr.data())))
		return rc;
	std::vector<double> E(count);
	if ((rc = cc_batch_energy_grad(b, E.data(), nullptr, CC_PREC_FP64)))
		return rc;
	if (results)
		for (int k = 0; k < count; k++) {
			const int i = b->order[k];
			results[i].E = E[i];
			results[i].evals = hs[k].evals;
			results[i].iters = hs[k].iters;
			results[i].status = hs[k].status == cc::kLbRunning ? cc::kLbMaxEval : hs[k].status;
		}
	return CC_OK;
}

}  // extern "C"
