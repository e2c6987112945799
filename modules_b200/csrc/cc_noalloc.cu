// cc_noalloc.cu — cc_energy_noalloc: the rho + energy pass for callers that cannot allocate GPU memory.
//
// Who needs it: host programs whose memory manager has already reserved the device's memory (a caching allocator or
// a serving engine with a fixed HBM budget) and does not allow a library to allocate on the side, and loops that must
// not pay for cudaMalloc, which can synchronise the whole device.
// Such callers cannot create a cc_handle, because cc_create allocates the planned k-set and work buffers.
//
// This entry point takes every input and output in the caller's own device memory and computes
//   rho(k_m) = sum_j exp(2 pi i n_m . s_j)   and   E = sum_m V_m |rho(k_m)|^2 / volume + shift
// with a variant of the rho kernel of cc_kernels.cuh in which every mode is its own one-slot segment (no host-side
// plan, so the call allocates nothing on the host either). Its only scratch memory (per-split partial sums and the
// completion tickets) is the file-scope array g_noalloc_scratch below: CC_NOALLOC_SCRATCH_BYTES (16 MiB) of device
// memory that every GPU which loads this library holds until the process exits.
#include "../../include/cc_gpu.h"
#include "cc_kernels.cuh"

#include <cuda_runtime.h>

#include <atomic>

namespace {

constexpr size_t kScratchBytes = CC_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;
constexpr int kWarpsNA = 8;
constexpr int kChunkNA = 64;

// The scratch array. In host code this name is only a stand-in for the symbol, not a device address: host code
// gets the address with cudaGetSymbolAddress (once per device, see scratch_on_device).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Cached device addresses, one per device. Concurrent first calls from several host threads may each look the
// address up and store the same value; the atomics make that well defined.
std::atomic<void *> g_scratch_ptr[kMaxDevices];

thread_local const char *g_na_err = "";

// Device address of g_noalloc_scratch on the current device; looked up on the first call per device.
int scratch_on_device(int dev, void **out)
{
	if (dev < 0 || dev >= kMaxDevices)
		return CC_ERR_ARG;
	void *p = g_scratch_ptr[dev].load(std::memory_order_relaxed);
	if (!p) {
		if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p)
			return CC_ERR_CUDA;
		g_scratch_ptr[dev].store(p, std::memory_order_relaxed);
	}
	*out = p;
	return CC_OK;
}

struct ModesArgs {
	const double *frac;     // N x D
	int N, per_split, nsplit;
	const int32_t *modes;   // M x D
	const double *V;        // M
	int M, ngroups;
	double2 *partial;       // [nsplit][ngroups*32]  (scratch)
	unsigned *tickets;      // [ngroups + 1]         (scratch, zero on entry)
	double2 *rho;           // M, or nullptr
	double *E;
	double inv_vol, shift;
};

// One lane per mode, a block = 32 modes x kWarpsNA warps striding over the block's particle range; the last block of
// each group of 32 modes sums the splits in split order; the last group sums the energy over modes in mode order.
template <int D>
__global__ void __launch_bounds__(kWarpsNA * 32) cc_rho_modes_kernel(ModesArgs a)
{
	__shared__ double sh_s[kChunkNA * D];
	__shared__ double2 sh_red[kWarpsNA * 32];
	__shared__ int sh_last;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const int group = blockIdx.x, split = blockIdx.y;
	const int m = group * 32 + lane;
	cc::Seg sg = {0, 0, 0, 0};
	if (m < a.M) {
		if (D >= 2)
			sg.p0 = a.modes[(size_t)m * D];
		if (D >= 3)
			sg.p1 = a.modes[(size_t)m * D + 1];
		sg.start = a.modes[(size_t)m * D + D - 1];
		sg.len = 1;
	}
	const int j0 = split * a.per_split;
	const int j1 = min(a.N, j0 + a.per_split);
	double2 acc = make_double2(0.0, 0.0);
	for (int cj = j0; cj < j1; cj += kChunkNA) {
		const int cnt = min(kChunkNA, j1 - cj);
		__syncthreads();
		for (int i = threadIdx.x; i < cnt * D; i += kWarpsNA * 32)
			sh_s[i] = a.frac[(size_t)cj * D + i];
		__syncthreads();
		for (int i = warp; i < cnt; i += kWarpsNA) {
			double s[D];
#pragma unroll
			for (int e = 0; e < D; e++)
				s[e] = sh_s[i * D + e];
			const double2 z = cc::expi2pi(cc::seg_phase<D>(sg, s));
			acc.x += z.x;
			acc.y += z.y;
		}
	}
	__syncthreads();
	sh_red[warp * 32 + lane] = acc;
	__syncthreads();
	if (warp == 0) {
		double2 t = sh_red[lane];
		for (int w = 1; w < kWarpsNA; w++) {
			t.x += sh_red[w * 32 + lane].x;
			t.y += sh_red[w * 32 + lane].y;
		}
		a.partial[(size_t)split * a.ngroups * 32 + group * 32 + lane] = t;
	}
	__threadfence();
	__syncthreads();
	if (threadIdx.x == 0)
		sh_last = (atomicAdd(&a.tickets[group], 1u) == (unsigned)(a.nsplit - 1));
	__syncthreads();
	if (!sh_last)
		return;
	__threadfence();
	if (warp == 0) {
		double2 t = __ldcg(&a.partial[group * 32 + lane]);
		for (int sp = 1; sp < a.nsplit; sp++) {
			const double2 v = __ldcg(&a.partial[(size_t)sp * a.ngroups * 32 + group * 32 + lane]);
			t.x += v.x;
			t.y += v.y;
		}
		// the group's final rho stays in split 0's row for the energy pass
		a.partial[group * 32 + lane] = t;
		if (a.rho && m < a.M)
			a.rho[m] = t;
	}
	__threadfence();
	__syncthreads();
	if (threadIdx.x == 0)
		sh_last = (atomicAdd(&a.tickets[a.ngroups], 1u) == (unsigned)(a.ngroups - 1));
	__syncthreads();
	if (!sh_last)
		return;
	__threadfence();
	double e = 0.0;
	for (int q = threadIdx.x; q < a.M; q += kWarpsNA * 32) {
		const double2 r = __ldcg(&a.partial[q]);
		e += a.V[q] * (r.x * r.x + r.y * r.y);
	}
	double *sh_e = reinterpret_cast<double *>(sh_red);
	__syncthreads();
	sh_e[threadIdx.x] = e;
	__syncthreads();
	for (int stride = kWarpsNA * 16; stride > 0; stride >>= 1) {
		if (threadIdx.x < stride)
			sh_e[threadIdx.x] += sh_e[threadIdx.x + stride];
		__syncthreads();
	}
	if (threadIdx.x == 0)
		*a.E = sh_e[0] * a.inv_vol + a.shift;
}

template <int D> void launch_modes(const ModesArgs &a, cudaStream_t st)
{
	cc_rho_modes_kernel<D><<<dim3(a.ngroups, a.nsplit), kWarpsNA * 32, 0, st>>>(a);
}

double det_abs(int d, const double *b)
{
	double det;
	if (d == 1)
		det = b[0];
	else if (d == 2)
		det = b[0] * b[3] - b[1] * b[2];
	else
		det = b[0] * (b[4] * b[8] - b[5] * b[7]) - b[1] * (b[3] * b[8] - b[5] * b[6]) + b[2] * (b[3] * b[7] - b[4] * b[6]);
	return det < 0 ? -det : det;
}

}  // namespace

extern "C" const char *cc_noalloc_last_error(void) { return g_na_err; }

extern "C" int cc_energy_noalloc(int d, const double *basis, int64_t M, const int32_t *d_modes, const double *d_V,
                                 double shift, int64_t N, const double *d_frac, double *d_E, double *d_rho,
                                 void *stream)
{
	if (d < 1 || d > 3 || !basis || M < 0 || N < 0 || !d_E || (M > 0 && (!d_modes || !d_V)) || (N > 0 && !d_frac)) {
		g_na_err = "cc_energy_noalloc: invalid arguments";
		return CC_ERR_ARG;
	}
	if (M > CC_NOALLOC_MAX_MODES) {
		g_na_err = "cc_energy_noalloc: more modes than CC_NOALLOC_MAX_MODES";
		return CC_ERR_ARG;
	}
	if (N > CC_NOALLOC_MAX_PARTICLES) {
		g_na_err = "cc_energy_noalloc: more particles than CC_NOALLOC_MAX_PARTICLES";
		return CC_ERR_ARG;
	}
	const double vol = det_abs(d, basis);
	if (!(vol > 0) || vol != vol) {
		g_na_err = "cc_energy_noalloc: degenerate cell basis";
		return CC_ERR_ARG;
	}
	int dev = 0;
	if (cudaGetDevice(&dev) != cudaSuccess) {
		g_na_err = "cc_energy_noalloc: no CUDA device";
		return CC_ERR_NOGPU;
	}
	void *scratch = nullptr;
	if (int rc = scratch_on_device(dev, &scratch)) {
		g_na_err = "cc_energy_noalloc: cudaGetSymbolAddress of the scratch array failed";
		return rc;
	}
	cudaStream_t st = static_cast<cudaStream_t>(stream);
	const int ngroups = (int)((M + 31) / 32);
	// tickets first, then the partials, 256-byte aligned
	const size_t tick_bytes = ((size_t)(ngroups + 1) * sizeof(unsigned) + 255) / 256 * 256;
	const size_t row_bytes = (size_t)ngroups * 32 * sizeof(double2);
	int nsplit = 1;
	if (N > 0 && ngroups > 0) {
		int sms = 148;
		cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
		const int64_t want = (int64_t)(sms * 4 + ngroups - 1) / ngroups;
		const int64_t fit = (int64_t)((kScratchBytes - tick_bytes) / row_bytes);
		const int64_t most = (N + 2 * kWarpsNA - 1) / (2 * kWarpsNA);
		int64_t ns = want < fit ? want : fit;
		ns = ns < most ? ns : most;
		nsplit = (int)(ns < 1 ? 1 : ns);
	}
	ModesArgs a;
	a.frac = d_frac;
	a.N = (int)N;
	a.per_split = N > 0 ? (int)((N + nsplit - 1) / nsplit) : 0;
	a.nsplit = N > 0 ? (int)((N + a.per_split - 1) / a.per_split) : 1;
	a.modes = d_modes;
	a.V = d_V;
	a.M = (int)M;
	a.ngroups = ngroups;
	a.tickets = static_cast<unsigned *>(scratch);
	a.partial = reinterpret_cast<double2 *>(static_cast<unsigned char *>(scratch) + tick_bytes);
	a.rho = reinterpret_cast<double2 *>(d_rho);
	a.E = d_E;
	a.inv_vol = 1.0 / vol;
	a.shift = shift;
	// every call shares the scratch array: the tickets must start at zero
	if (cudaMemsetAsync(scratch, 0, tick_bytes, st) != cudaSuccess) {
		g_na_err = "cc_energy_noalloc: cudaMemsetAsync of the tickets failed";
		return CC_ERR_CUDA;
	}
	if (ngroups == 0) {
		// no modes: one block with M = 0 writes E = shift
		a.ngroups = 1;
		a.nsplit = 1;
		a.per_split = 0;
	}
	if (d == 1)
		launch_modes<1>(a, st);
	else if (d == 2)
		launch_modes<2>(a, st);
	else
		launch_modes<3>(a, st);
	if (cudaGetLastError() != cudaSuccess) {
		g_na_err = "cc_energy_noalloc: kernel launch failed";
		return CC_ERR_CUDA;
	}
	return CC_OK;
}
