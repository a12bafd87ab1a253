// Burrows-Wheeler block sort: the C API of include/mgpubwt.h on this
// library's radix sort.
//
// Follows the reference's bwtSortBlock (bwt/src/mgpubwt/mgpubwt.cpp:213-371):
//  1. Rotation i of the block is keyed by its first 4 * S symbols, S =
//     ceil(gpuKeySize / 4), as S big-endian 32-bit key streams (stream s
//     holds symbols 4s .. 4s + 3), gathered on the device from the block
//     written twice in a row (so no rotation needs a modulo).
//  2. LSD over streams, least significant first: sortArray sorts stream s
//     (its top 8 * min(gpuKeySize - 4s, 4) bits) and carries the streams
//     still to be sorted plus the rotation indices as value arrays
//     (mgpubwt.cpp:256-291). Every sort is stable, so the indices end up
//     ordered by the first gpuKeySize symbols, ties in index order.
//  3. A head flag marks each sorted rotation whose first gpuKeySize symbols
//     differ from its predecessor's; the groups of two or more tied
//     rotations are finished on the host by comparing the remaining
//     count - gpuKeySize symbols (mgpubwt.cpp:318-348), with a stable sort,
//     so that rotations equal as whole strings stay in index order.
// Blocks shorter than 3000 bytes are sorted on the host only
// (mgpubwt.cpp:217-221, TinyBlockCutoff in bwtsort.h).

// The library is built with hidden visibility; the C ABI is all it exports.
#pragma GCC visibility push(default)
#include "../../include/mgpubwt.h"
#include "../../include/mgpusort.h"
#include "../../include/mgpusort_b200.h"
#pragma GCC visibility pop

#include <cuda_runtime.h>

#include "sort_common.cuh"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <thread>
#include <vector>

namespace {

constexpr int kTinyBlock = 3000;
constexpr int kMaxKeyBytes = 24;
constexpr int kMaxStreams = kMaxKeyBytes / 4;
constexpr int kThreads = 256;

const char* const kStatusNames[] = {
	"BWT_STATUS_SUCCESS",
	"BWT_STATUS_NOT_INITIALIZED",
	"BWT_STATUS_DEVICE_ALLOC_FAILED",
	"BWT_STATUS_INVALID_CONTEXT",
	"BWT_STATUS_KERNEL_NOT_FOUND",
	"BWT_STATUS_KERNEL_ERROR",
	"BWT_STATUS_LAUNCH_ERROR",
	"BWT_STATUS_INVALID_VALUE",
	"BWT_STATUS_DEVICE_ERROR",
	"BWT_STATUS_NOT_IMPLEMENTED",
	"BWT_STATUS_UNSUPPORTED_DEVICE",
	"BWT_STATUS_SORT_ERROR",
};

struct GatherArgs {
	const unsigned char* sym;       // the block twice, plus padding
	int count;
	int numStreams;
	unsigned* streams[kMaxStreams];
	unsigned* indices;
};

// Key streams and initial indices of every rotation.
__global__ void __launch_bounds__(kThreads) bwt_gather_keys(const GatherArgs a) {
	for(int i = blockIdx.x * kThreads + threadIdx.x; i < a.count;
		i += gridDim.x * kThreads) {
		const unsigned char* p = a.sym + i;
		for(int s = 0; s < a.numStreams; ++s)
			a.streams[s][i] = ((unsigned)p[4 * s] << 24) | ((unsigned)p[4 * s + 1] << 16)
				| ((unsigned)p[4 * s + 2] << 8) | (unsigned)p[4 * s + 3];
		a.indices[i] = (unsigned)i;
	}
}

// flags[i] = 1 where the first keyBytes symbols of the i-th sorted rotation
// differ from those of the (i - 1)-th (and at i = 0).
__global__ void __launch_bounds__(kThreads) bwt_head_flags(const unsigned char* sym,
	const unsigned* sorted, int count, int keyBytes, unsigned char* flags) {
	for(int i = blockIdx.x * kThreads + threadIdx.x; i < count;
		i += gridDim.x * kThreads) {
		unsigned char head = 1;
		if(i > 0) {
			const unsigned char* x = sym + sorted[i - 1];
			const unsigned char* y = sym + sorted[i];
			head = 0;
			for(int k = 0; k < keyBytes; ++k)
				if(x[k] != y[k]) { head = 1; break; }
		}
		flags[i] = head;
	}
}

// Orders rotation starts by the `len` symbols from `sym + start`.
struct RotationLess {
	const unsigned char* sym;
	int len;
	bool operator()(int a, int b) const {
		return std::memcmp(sym + a, sym + b, len) < 0;
	}
};

void host_block_sort(const unsigned char* block, int count, void* transform,
	int* indices, int* segCount, float* avSegSize) {
	std::vector<unsigned char> sym(2 * (size_t)count);
	if(count) {
		std::memcpy(sym.data(), block, count);
		std::memcpy(sym.data() + count, block, count);
	}
	std::vector<int> order(count);
	for(int i = 0; i < count; ++i) order[i] = i;
	std::stable_sort(order.begin(), order.end(), RotationLess{sym.data(), count});
	if(segCount) *segCount = count ? 1 : 0;
	if(avSegSize) *avSegSize = (float)count;
	if(indices && count) std::memcpy(indices, order.data(), sizeof(int) * count);
	if(transform) {
		unsigned char* out = static_cast<unsigned char*>(transform);
		for(int i = 0; i < count; ++i) out[i] = sym[order[i] + count - 1];
	}
}

size_t round_up(size_t x, size_t m) { return (x + m - 1) / m * m; }

} // namespace

struct bwtEngine_d {
	sortEngine_t sort = nullptr;
	cudaStream_t stream = nullptr;
	int numSMs = 0;
	unsigned char* dSym = nullptr;
	size_t symBytes = 0;
	unsigned* dArrays = nullptr;     // (kMaxStreams + 1) x 2 arrays
	size_t arrayElements = 0;
	unsigned char* dFlags = nullptr;
	size_t flagBytes = 0;
	std::vector<unsigned char> sym;
	std::vector<int> order;
	std::vector<unsigned char> flags;
};

namespace {

template<typename T>
bool grow(T*& p, size_t& have, size_t want) {
	if(have >= want) return true;
	if(p) cudaFree(p);
	p = nullptr;
	have = 0;
	if(cudaMalloc(&p, want * sizeof(T)) != cudaSuccess) {
		cudaGetLastError();
		p = nullptr;
		return false;
	}
	have = want;
	return true;
}

} // namespace

extern "C" {

const char* BWTAPI bwtStatusString(bwtStatus_t status) {
	const int n = (int)(sizeof(kStatusNames) / sizeof(kStatusNames[0]));
	if((int)status < 0 || (int)status >= n) return nullptr;
	return kStatusNames[status];
}

bwtStatus_t BWTAPI bwtCreateEngine(const char* kernelPath, bwtEngine_t* engine) {
	if(!engine) return BWT_STATUS_INVALID_VALUE;
	*engine = nullptr;
	bwtEngine_d* e = new bwtEngine_d;
	const sortStatus_t st = sortCreateEngine(kernelPath, &e->sort);
	if(st != SORT_STATUS_SUCCESS) {
		delete e;
		if(st == SORT_STATUS_UNSUPPORTED_DEVICE) return BWT_STATUS_UNSUPPORTED_DEVICE;
		if(st == SORT_STATUS_INVALID_CONTEXT) return BWT_STATUS_INVALID_CONTEXT;
		return BWT_STATUS_SORT_ERROR;
	}
	int device = 0;
	if(cudaGetDevice(&device) != cudaSuccess ||
		cudaDeviceGetAttribute(&e->numSMs, cudaDevAttrMultiProcessorCount, device)
		!= cudaSuccess ||
		cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
		cudaGetLastError();
		sortReleaseEngine(e->sort);
		delete e;
		return BWT_STATUS_DEVICE_ERROR;
	}
	*engine = e;
	return BWT_STATUS_SUCCESS;
}

bwtStatus_t BWTAPI bwtDestroyEngine(bwtEngine_t engine) {
	if(!engine) return BWT_STATUS_SUCCESS;
	if(engine->stream) cudaStreamSynchronize(engine->stream);
	if(engine->dSym) cudaFree(engine->dSym);
	if(engine->dArrays) cudaFree(engine->dArrays);
	if(engine->dFlags) cudaFree(engine->dFlags);
	if(engine->stream) cudaStreamDestroy(engine->stream);
	sortReleaseEngine(engine->sort);
	delete engine;
	return BWT_STATUS_SUCCESS;
}

bwtStatus_t BWTAPI bwtSortBlock(bwtEngine_t engine, const void* block, int count,
	int gpuKeySize, void* transform, int* indices, int* segCount, float* avSegSize) {
	if(count < 0 || (count > 0 && !block)) return BWT_STATUS_INVALID_VALUE;
	const unsigned char* bytes = static_cast<const unsigned char*>(block);
	if(count < kTinyBlock) {
		host_block_sort(bytes, count, transform, indices, segCount, avSegSize);
		return BWT_STATUS_SUCCESS;
	}
	if(!engine || gpuKeySize < 1 || gpuKeySize > kMaxKeyBytes)
		return BWT_STATUS_INVALID_VALUE;
	if(count > (1 << 28)) return BWT_STATUS_INVALID_VALUE;
	const int numStreams = (gpuKeySize + 3) / 4;

	// The block twice in a row, padded so that every key read stays inside.
	std::vector<unsigned char>& sym = engine->sym;
	sym.assign(2 * (size_t)count + 32, 0);
	std::memcpy(sym.data(), bytes, count);
	std::memcpy(sym.data() + count, bytes, count);

	const size_t stride = round_up((size_t)count, 2048);
	if(!grow(engine->dSym, engine->symBytes, sym.size()) ||
		!grow(engine->dArrays, engine->arrayElements, stride * 2 * (kMaxStreams + 1)) ||
		!grow(engine->dFlags, engine->flagBytes, (size_t)count))
		return BWT_STATUS_DEVICE_ALLOC_FAILED;
	cudaStream_t stream = engine->stream;
	auto array = [&](int a, int half) { return engine->dArrays + stride * (2 * a + half); };

	if(cudaMemcpyAsync(engine->dSym, sym.data(), sym.size(), cudaMemcpyHostToDevice,
		stream) != cudaSuccess) {
		cudaGetLastError();
		return BWT_STATUS_DEVICE_ERROR;
	}
	GatherArgs g;
	std::memset(&g, 0, sizeof(g));
	g.sym = engine->dSym;
	g.count = count;
	g.numStreams = numStreams;
	for(int s = 0; s < numStreams; ++s) g.streams[s] = array(s, 0);
	g.indices = array(kMaxStreams, 0);
	const int grid = std::max(1, std::min(engine->numSMs * 8,
		(count + kThreads - 1) / kThreads));
	if(mgpusort::launch_plain(bwt_gather_keys, grid, kThreads, 0, stream, g) != cudaSuccess)
		return BWT_STATUS_LAUNCH_ERROR;

	// Most significant stream last; the parity says which half of every
	// array still carried holds its current contents (mgpusort.cpp:519-526).
	sortData_d d;
	std::memset(&d, 0, sizeof(d));
	d.maxElements = count;
	d.numElements = count;
	for(int cur = numStreams - 1; cur >= 0; --cur) {
		const int p = d.parity;
		d.keys[0] = reinterpret_cast<CUdeviceptr>(array(cur, p));
		d.keys[1] = reinterpret_cast<CUdeviceptr>(array(cur, 1 - p));
		for(int v = 0; v < 6; ++v) d.values[v][0] = d.values[v][1] = 0;
		for(int s = 0; s < cur; ++s) {
			d.values[s][0] = reinterpret_cast<CUdeviceptr>(array(s, p));
			d.values[s][1] = reinterpret_cast<CUdeviceptr>(array(s, 1 - p));
		}
		d.values[cur][0] = reinterpret_cast<CUdeviceptr>(array(kMaxStreams, p));
		d.values[cur][1] = reinterpret_cast<CUdeviceptr>(array(kMaxStreams, 1 - p));
		d.valueCount = cur + 1;
		const int curBytes = std::min(gpuKeySize - 4 * cur, 4);
		d.firstBit = 32 - 8 * curBytes;
		d.endBit = 32;
		if(sortArrayAsync(engine->sort, &d, reinterpret_cast<CUstream>(stream))
			!= SORT_STATUS_SUCCESS)
			return BWT_STATUS_SORT_ERROR;
	}
	const unsigned* sorted = reinterpret_cast<const unsigned*>(d.values[0][0]);

	if(mgpusort::launch_plain(bwt_head_flags, grid, kThreads, 0, stream,
		static_cast<const unsigned char*>(engine->dSym), sorted, count, gpuKeySize,
		engine->dFlags) != cudaSuccess)
		return BWT_STATUS_LAUNCH_ERROR;

	std::vector<int>& order = engine->order;
	std::vector<unsigned char>& flags = engine->flags;
	order.resize(count);
	flags.resize((size_t)count + 1);
	if(cudaMemcpyAsync(order.data(), sorted, sizeof(int) * (size_t)count,
		cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
		cudaMemcpyAsync(flags.data(), engine->dFlags, count, cudaMemcpyDeviceToHost,
		stream) != cudaSuccess ||
		cudaStreamSynchronize(stream) != cudaSuccess) {
		cudaGetLastError();
		return BWT_STATUS_DEVICE_ERROR;
	}
	if(sortSynchronize(engine->sort) != SORT_STATUS_SUCCESS) return BWT_STATUS_SORT_ERROR;
	flags[count] = 1;

	// Finish every group of tied rotations on the host, the groups spread
	// over the host's threads.
	const RotationLess rest{sym.data() + gpuKeySize, count - gpuKeySize};
	std::vector<std::pair<int, int>> tied;
	long long grouped = 0;
	int start = 0;
	for(int i = 1; i <= count; ++i) {
		if(!flags[i]) continue;
		if(i - start >= 2) {
			tied.emplace_back(start, i);
			grouped += i - start;
		}
		start = i;
	}
	const int groups = (int)tied.size();
	std::atomic<int> nextGroup(0);
	auto finish = [&] {
		for(int g; (g = nextGroup.fetch_add(1)) < groups;)
			std::stable_sort(order.begin() + tied[g].first, order.begin() + tied[g].second,
				rest);
	};
	const int workers = (int)std::min<long long>(
		std::max(1u, std::thread::hardware_concurrency()), 1 + grouped / 4096);
	std::vector<std::thread> pool;
	for(int t = 1; t < workers; ++t) pool.emplace_back(finish);
	finish();
	for(auto& th : pool) th.join();
	if(segCount) *segCount = groups;
	if(avSegSize) *avSegSize = groups ? (float)((double)grouped / groups) : 0.0f;
	if(indices) std::memcpy(indices, order.data(), sizeof(int) * (size_t)count);
	if(transform) {
		unsigned char* out = static_cast<unsigned char*>(transform);
		for(int i = 0; i < count; ++i) out[i] = sym[(size_t)order[i] + count - 1];
	}
	return BWT_STATUS_SUCCESS;
}

} // extern "C"
