// cc_internal.h — what the library's translation units share behind the C ABI: the error channel, device buffer
// helpers, the device copy of a planned k-set, and the handle itself. Not part of the ABI (include/cc_gpu.h is).
#pragma once
#include "../../include/cc_gpu.h"
#include "cc_kernels.cuh"
#include "cc_lbfgs.cuh"
#include "cc_nufft.cuh"
#include "cc_plan.h"

#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <atomic>
#include <string>
#include <utility>
#include <vector>

namespace cci {

// Sets the message cc_last_error() returns (this thread) and returns code.
int fail(int code, const std::string &msg);

#define CC_CUDA(call)                                                                                         \
	do {                                                                                                      \
		cudaError_t e_ = (call);                                                                              \
		if (e_ != cudaSuccess)                                                                                \
			return ::cci::fail(CC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));             \
	} while (0)

// ---------------------------------------------------------------------------------------------------------------
// device-side k-set: a Plan uploaded
// ---------------------------------------------------------------------------------------------------------------
struct DevSplits {
	int want = 0;
	cc::ForceSplits host;
	int *kstart = nullptr;
	cc::TabSpec *kspec = nullptr;
};

struct DevKSet {
	cc::Plan plan;
	cc::Seg *segs = nullptr;
	cc::TabSpec *rspec = nullptr;
	int *bstart = nullptr;
	cc::TabSpec *bspec = nullptr;
	double *slotV = nullptr;
	int *mode_slot = nullptr;
	double2 *rho_slot = nullptr;
	double2 *u_slot = nullptr;
	double2 *rho_mode = nullptr;
	double *eblock = nullptr;       // one per reduce block
	unsigned *ticket = nullptr;
	double2 *partial = nullptr;     // partial rows * nslot
	size_t partial_cap = 0;         // in double2 elements
	std::vector<DevSplits> splits;  // force splits per requested count

	void release()
	{
		cudaFree(segs);
		cudaFree(rspec);
		cudaFree(bstart);
		cudaFree(bspec);
		cudaFree(slotV);
		cudaFree(mode_slot);
		cudaFree(rho_slot);
		cudaFree(u_slot);
		cudaFree(rho_mode);
		cudaFree(eblock);
		cudaFree(ticket);
		cudaFree(partial);
		for (DevSplits &f : splits) {
			cudaFree(f.kstart);
			cudaFree(f.kspec);
		}
		*this = DevKSet();
	}
};

// Bumped by every device or pinned allocation of the library and by changes of by-value kernel parameters: a
// captured evaluation graph whose generation differs may hold stale pointers and is captured again.
extern std::atomic<unsigned long long> g_alloc_gen;

template <class T> int dev_alloc(T **p, size_t n)
{
	g_alloc_gen++;
	*p = nullptr;
	if (n == 0)
		n = 1;
	cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), n * sizeof(T));
	if (e != cudaSuccess)
		return fail(e == cudaErrorMemoryAllocation ? CC_ERR_OOM : CC_ERR_CUDA,
		            std::string("cudaMalloc: ") + cudaGetErrorString(e));
	return CC_OK;
}

template <class T> int upload(T **p, const std::vector<T> &v)
{
	if (int rc = dev_alloc(p, v.size()))
		return rc;
	if (!v.empty())
		CC_CUDA(cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
	return CC_OK;
}

template <class T> int upload_into(T *p, const std::vector<T> &v)
{
	if (!v.empty())
		CC_CUDA(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
	return CC_OK;
}


// Upload a plan into a device k-set (releases what it held).
int upload_kset(DevKSet &k, const cc::Plan &plan);

// The device splits of the force pass into about `want` segment ranges (uploaded on first use, kept by the k-set).
int get_splits(DevKSet &k, int want, const DevSplits **out);

// Device state of cc_minimize (L-BFGS of one configuration), kept by the handle between calls (grow-only).
struct LbBuffers {
	double *x = nullptr, *g = nullptr, *d = nullptr, *xt = nullptr, *gt = nullptr, *S = nullptr, *Y = nullptr;
	double *part = nullptr;
	cc::LbState *st = nullptr;
	cc::LbInst *inst = nullptr;
	cc::LbInst host_inst{};   // the host copy of *inst (passed in the L-BFGS kernels' parameters)
	void release()
	{
		cudaFree(x);
		cudaFree(g);
		cudaFree(d);
		cudaFree(xt);
		cudaFree(gt);
		cudaFree(S);
		cudaFree(Y);
		cudaFree(part);
		cudaFree(st);
		cudaFree(inst);
		*this = LbBuffers();
	}
};



// Streaming multiprocessors of the current device.
int sm_count();

// CC_ERR_ARG unless precision is CC_PREC_FP64 or CC_PREC_MIXED.
int check_prec(int precision);

}  // namespace cci

struct cc_handle;

namespace cci {

// CC_ERR_ARG for a null handle.
int handle_check(const cc_handle *h);
// The handle's per-particle buffers for N particles (positions, forces, gradients; grow-only).
int handle_reserve(cc_handle *h, int64_t N);
// One evaluation of the handle at device positions d_frac (N x d), enqueued on st: E (device), and F (Cartesian) and /
// or gfrac (fractional gradient) where not null; want_rho_mode also fills rho in constraint order.
int handle_eval(cc_handle *h, int64_t N, const double *d_frac, double *d_E, double *d_F, double *d_gfrac,
                bool want_rho_mode, int precision, cudaStream_t st);

constexpr size_t kRhoTabBudget = 48 * 1024;   // shared memory for one chunk of rho tables

template <typename C> size_t rho_smem(int row, int chunk, int L)
{
	return std::max((size_t)chunk * (row | 1) * sizeof(C), (size_t)cc::kRhoWarps * 32 * L * sizeof(double2));
}
template <typename C> size_t force_smem(int row, int d) { return cc::force_smem_bytes<C>(row, d, 8); }

// Launch with programmatic stream serialization: the kernel may be scheduled while the previous kernel on the stream
// drains; it calls cudaGridDependencySynchronize() before it reads that kernel's results.
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl_n(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args... args)
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
	return cudaLaunchKernelEx(&cfg, kern, args...);
}

}  // namespace cci

struct cc_handle {
	int d = 0;
	double basis[9] = {0};
	double recip[9] = {0};
	double volume = 0;
	double shift = 0;
	double rho_offset = 0;
	std::vector<int32_t> modes;
	std::vector<double> V;
	cci::DevKSet main;
	cci::DevKSet sk;                     // k-set of the last cc_structure_factor call
	std::vector<int32_t> sk_modes;
	cudaStream_t stream = nullptr;
	int64_t N = -1;                 // bound particle count, -1 before cc_set_positions
	size_t ncap = 0;                // capacity of the per-particle buffers
	double *d_frac = nullptr, *d_F = nullptr, *d_gfrac = nullptr, *d_partialG = nullptr;
	size_t partialG_cap = 0;
	unsigned *d_fcounters = nullptr;
	double *d_E = nullptr;
	double *h_pin = nullptr;        // pinned results: E at [0], N*d forces or gradients from [2]
	size_t pin_cap = 0;
	double *h_in = nullptr;         // pinned staging of the wrapped positions (N*d), mapped
	double *d_in = nullptr;         // device view of h_in (read by the first kernel of the host-path graph)
	double *rho_copy = nullptr;     // while the host-path graph is captured on the three-kernel path: the rho kernel
	                                // reads the positions from d_in and stores them here (d_frac) for the force kernel
	size_t in_cap = 0;
	cudaEvent_t ev_in = nullptr;    // recorded after the last copy out of h_in
	bool in_pending = false;
	bool lastF_valid = false;       // h_pin + 2 holds the forces of the bound positions
	bool upload_pending = false;    // h_in holds positions not yet copied to d_frac
	double *d_pin = nullptr;        // device view of h_pin (mapped pinned memory): kernels write E and F there
	// captured evaluations of cc_energy_grad (upload + kernels writing into h_pin), per (N, precision, forces)
	struct EvalGraph {
		int64_t N;
		int precision, forces;
		unsigned long long gen;
		cudaGraphExec_t exec;
	};
	std::vector<EvalGraph> graphs;
	int64_t last_N = -1;            // key and generation of the last direct cc_energy_grad (captured when repeated)
	int last_precision = -1, last_forces = -1;
	unsigned long long last_gen = 0;
	// S2 form (cc_create_s2): per-slot targets S0, E = sum V (|rho|^2 / N - S0)^2 + shift; split path only
	double *d_slotS0 = nullptr;
	// S2 over nsub sub-configurations (cc_create_s2_multiconfig): rho and u per sub-configuration, block partials
	int nsub = 1;
	double2 *d_msub = nullptr;      // [2][nsub][nslot]: rho, then u
	double *d_mpart = nullptr;      // energy partials of the combination, then one scratch word
	size_t msub_cap = 0, mpart_cap = 0;
	bool use_nufft = false;         // cc_set_path(CC_PATH_NUFFT)
	bool auto_path = true;          // CC_PATH_AUTO (default): the NUFFT path where its estimated time is lower
	double nu_grid_est = -1.0;      // fine-grid points the NUFFT path would use (computed once)
	// non-uniform FFT path (cc_nufft.cuh), set up at its first use
	bool nu_ready = false;
	cc::NufftDev nu = {};
	int64_t nu_ngrid = 0, nu_nspec = 0;
	int nu_rho_blocks = 0;
	int *d_nu_mode_u = nullptr;
	std::vector<void *> nu_bufs;    // device buffers owned by the NUFFT set-up
	cufftHandle nu_p1 = 0, nu_p2 = 0;
	bool nu_p1_ok = false, nu_p2_ok = false;
	// Monte Carlo: rho in mode order of the bound positions, the trial rho and the device modes
	int32_t *d_modes = nullptr;
	double *d_modeV = nullptr;
	double2 *d_rho_trial = nullptr, *d_rho_cur = nullptr;
	double *d_mc_part = nullptr;
	bool mc_valid = false, mc_pending = false;
	const int *d_skip = nullptr;    // evaluations do nothing while *d_skip != 0 (set by cc_minimize)
	bool timing = false;            // cc_set_timing
	bool independent = false;       // cc_set_independent_positions
	// cc_energy_grad_many: every configuration of a call resident at once, so that its copies overlap the evaluations
	double *d_many_in = nullptr, *d_many_F = nullptr, *d_many_E = nullptr;
	int *d_many_bad = nullptr;          // set by the wrap kernel on a non-finite coordinate
	size_t many_cap = 0, many_ecap = 0; // doubles of d_many_in / d_many_F and of d_many_E
	cudaStream_t copy_stream = nullptr;
	std::vector<cudaEvent_t> many_ev;   // two per chunk: positions in, results done
	bool early_call = false;        // set for the duration of a cc_energy_grad_device call when independent
	// cc_minimize's state, kept between calls so that a minimisation makes no allocation call into the CUDA driver
	// once the handle has run one of its size: FP64 / mixed buffers (capacities n variables, m pairs, nblk dot
	// blocks) and the batch of one that runs the precision schedule (for sched_N particles)
	cci::LbBuffers lb;
	int lb_n = 0, lb_m = 0, lb_nblk = 0;
	cc_batch *sched_batch = nullptr;
	int64_t sched_N = -1;
	std::vector<cudaEvent_t> ev;    // 3 events per timed evaluation
	size_t ev_used = 0;
};

