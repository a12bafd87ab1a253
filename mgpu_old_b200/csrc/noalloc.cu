// sortArrayNoAlloc: sortArray for callers that cannot allocate device memory.
//
// Some callers must not let a library allocate on the GPU: programs that hand
// all of a GPU's memory to their own allocator or budget up front (a
// database engine or an inference server that reserves HBM at start-up and
// fails any allocation outside it), and latency-critical loops where a
// cudaMalloc or cudaFree would synchronize the device and stall every other
// stream. sortArray cannot serve them, because its engine allocates its
// scratch (control block, per-pass range counts, a mapped error word).
//
// This entry point needs no engine and allocates nothing. Its scratch is the
// file-scope array below: a control block plus the per-pass range counts and
// offsets, about 2 MiB, which each GPU that loads this module holds until the
// process exits. It accepts up to SORT_NOALLOC_MAX_ELEMENTS elements. The
// caller passes the key and value buffers in a sortData_d, exactly as for
// sortArray.

// The library is built with hidden visibility; the C ABI is all it exports.
#pragma GCC visibility push(default)
#include "../../include/mgpusort.h"
#include "../../include/mgpusort_b200.h"
#pragma GCC visibility pop
#include "sort_kernels.h"

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <utility>

namespace {

constexpr size_t kControlWords =
	(sizeof(mgpusort::Control) + 255) / 256 * 256 / sizeof(unsigned long long);
constexpr size_t kPassWords =
	(mgpusort::kPassScratchWords * sizeof(unsigned) + 7) / sizeof(unsigned long long);
constexpr size_t kScratchWords = kControlWords + kPassWords;

} // namespace

// The scratch: [Control, padded to 256 bytes][pass scratch].
static __device__ __align__(256) unsigned long long g_noAllocScratch[kScratchWords];

namespace {

constexpr int kMaxDevices = 64;

// Host-side view of one device's scratch. `scratch` is the device address of
// g_noAllocScratch on that device: in host code the array's own name is only
// a stand-in for the symbol, never an address a kernel may be given.
struct DeviceScratch {
	bool ready;
	unsigned long long* scratch;
	int numSMs;
};

DeviceScratch g_devices[kMaxDevices];
std::mutex g_lock;

// First call on a device (that device current): resolve the array's device
// address, configure the kernels and clear the whole array once.
sortStatus_t set_up(int device, DeviceScratch* s) {
	int major = 0, minor = 0;
	if(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device)
		!= cudaSuccess ||
		cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device)
		!= cudaSuccess) {
		cudaGetLastError();
		return SORT_STATUS_INVALID_CONTEXT;
	}
	if(major != 10 || minor != 0) return SORT_STATUS_UNSUPPORTED_DEVICE;
	void* p = nullptr;
	cudaError_t e = cudaGetSymbolAddress(&p, g_noAllocScratch);
	if(e != cudaSuccess || !p) {
		cudaGetLastError();
		return SORT_STATUS_DEVICE_ERROR;
	}
	if(mgpusort::configure_kernels() != cudaSuccess) {
		cudaGetLastError();
		return SORT_STATUS_KERNEL_ERROR;
	}
	int sms = 0;
	if(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)
		!= cudaSuccess || cudaMemset(p, 0, sizeof(g_noAllocScratch)) != cudaSuccess
		|| cudaDeviceSynchronize() != cudaSuccess) {
		cudaGetLastError();
		return SORT_STATUS_DEVICE_ERROR;
	}
	s->scratch = static_cast<unsigned long long*>(p);
	s->numSMs = sms;
	s->ready = true;
	return SORT_STATUS_SUCCESS;
}

void swap_buffers(sortData_d* d) {
	std::swap(d->keys[0], d->keys[1]);
	for(int i = 0; i < 6; ++i) std::swap(d->values[i][0], d->values[i][1]);
	d->parity ^= 1;
}

} // namespace

extern "C" sortStatus_t SORTAPI sortArrayNoAlloc(sortData_t d, CUstream cuStream) {
	if(!d) return SORT_STATUS_INVALID_VALUE;
	const int numBits = d->endBit - d->firstBit;
	if(!numBits) return SORT_STATUS_SUCCESS;
	if(numBits < 0 || numBits > 32 || d->firstBit < 0 || d->endBit > 32)
		return SORT_STATUS_INVALID_VALUE;
	if(d->numElements > d->maxElements || d->numElements < 0)
		return SORT_STATUS_INVALID_VALUE;
	if(d->valueCount < -1 || d->valueCount > 6) return SORT_STATUS_INVALID_VALUE;
	const int n = d->numElements;
	const bool indexMode = d->valueCount == -1;
	const int numArrays = indexMode ? 1 : d->valueCount;
	if(!d->keys[0] || !d->keys[1]) return SORT_STATUS_INVALID_VALUE;
	for(int i = 0; i < numArrays; ++i)
		if(!d->values[i][0] || !d->values[i][1]) return SORT_STATUS_INVALID_VALUE;
	if(n > SORT_NOALLOC_MAX_ELEMENTS) return SORT_STATUS_CONFIG_NOT_SUPPORTED;
	if(!n) return SORT_STATUS_SUCCESS;

	// The same plan as sortArray.
	int widths[mgpusort::kMaxPasses];
	const int passes = sortPlanPasses(d->firstBit, d->endBit, 0, widths);
	if(passes <= 0) return SORT_STATUS_INTERNAL_ERROR;
	mgpusort::PassPlan plan;
	std::memset(&plan, 0, sizeof(plan));
	plan.numPasses = passes;
	for(int p = 0, bit = d->firstBit, bin = 0; p < passes; ++p) {
		plan.shift[p] = bit;
		plan.width[p] = widths[p];
		plan.binBase[p] = bin;
		bit += widths[p];
		bin += 1 << widths[p];
		plan.totalBins = bin;
	}

	std::lock_guard<std::mutex> guard(g_lock);
	int device = 0;
	if(cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) {
		cudaGetLastError();
		return SORT_STATUS_INVALID_CONTEXT;
	}
	DeviceScratch& s = g_devices[device];
	if(!s.ready) {
		sortStatus_t st = set_up(device, &s);
		if(st != SORT_STATUS_SUCCESS) return st;
	}
	mgpusort::Control* ctrl = reinterpret_cast<mgpusort::Control*>(s.scratch);
	unsigned* passScratch = reinterpret_cast<unsigned*>(s.scratch + kControlWords);
	cudaStream_t stream = reinterpret_cast<cudaStream_t>(cuStream);

	// The array keeps the previous call's contents. The control block (its
	// error word) must start at zero; every pass rewrites the pass scratch
	// before reading it.
	if(cudaMemsetAsync(ctrl, 0, sizeof(mgpusort::Control), stream) != cudaSuccess) {
		cudaGetLastError();
		return SORT_STATUS_DEVICE_ERROR;
	}
	bool bulk = true;
	for(int i = 0; i < 2; ++i) bulk = bulk && (d->keys[i] & 15) == 0;
	for(int i = 0; i < numArrays; ++i)
		for(int j = 0; j < 2; ++j) bulk = bulk && (d->values[i][j] & 15) == 0;

	// The passes ping-pong between the two buffers of a local copy of the
	// caller's struct; the caller's struct takes the swaps only once every
	// pass has been launched, so a launch failure leaves it as it was.
	sortData_d work = *d;
	cudaError_t ce = cudaSuccess;
	for(int p = 0; p < passes; ++p) {
		const int vm = (indexMode && p == 0) ? mgpusort::kValueIndex : numArrays;
		mgpusort::PassBuffers buf = {};
		buf.keysIn = reinterpret_cast<const unsigned*>(work.keys[0]);
		buf.keysOut = reinterpret_cast<unsigned*>(work.keys[1]);
		for(int i = 0; i < 6; ++i) {
			buf.valsIn[i] = reinterpret_cast<const unsigned*>(work.values[i][0]);
			buf.valsOut[i] = reinterpret_cast<unsigned*>(work.values[i][1]);
		}
		ce = mgpusort::launch_pass(buf, vm, n, p, plan, ctrl, passScratch, bulk, -1,
			nullptr, s.numSMs, stream);
		if(ce != cudaSuccess) {
			cudaGetLastError();
			return SORT_STATUS_LAUNCH_ERROR;
		}
		swap_buffers(&work);
	}
	for(int p = 0; p < passes; ++p) swap_buffers(d);

	// Wait for the sort and read its device error word.
	unsigned err = 0;
	if(cudaMemcpyAsync(&err, &ctrl->error, sizeof(err), cudaMemcpyDeviceToHost,
		stream) != cudaSuccess || cudaStreamSynchronize(stream) != cudaSuccess) {
		cudaGetLastError();
		return SORT_STATUS_DEVICE_ERROR;
	}
	return err ? SORT_STATUS_KERNEL_ERROR : SORT_STATUS_SUCCESS;
}
