// Host engine and C ABI of libmgpusort_b200.so.
//
// Follows the reference's host engine, sort/src/mgpusort/mgpusort.cpp: the
// engine handle with its reference count (:200-261), sortData_d buffer
// management (:655-734), the LSD pass loop with ping-pong swaps and parity
// (:541-601), sortArray / sortArrayEx argument handling (:607-648) and the
// sortHost / sortDevice conveniences (:740-806). The per-pass kernel chain
// (:356-530) is replaced by three launches per pass (count, scan, sort over
// a range partition; sort_kernels.cu), plus one upsweep per sort for
// earlyExit.

// The library is built with hidden visibility; the C ABI is all it exports.
#pragma GCC visibility push(default)
#include "../../include/mgpusort.h"
#include "../../include/mgpusort_b200.h"
#pragma GCC visibility pop
#include "engine_internal.h"
#include "sort_kernels.h"
#include "tile_config.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <utility>
#include <vector>

// The struct layout callers compiled against (inc/mgpusort.h:63-147):
// five ints, two bools, an int, then the pointer unions at offset 32.
static_assert(offsetof(sortData_d, maxElements) == 0, "sortData_d layout");
static_assert(offsetof(sortData_d, numElements) == 4, "sortData_d layout");
static_assert(offsetof(sortData_d, valueCount) == 8, "sortData_d layout");
static_assert(offsetof(sortData_d, firstBit) == 12, "sortData_d layout");
static_assert(offsetof(sortData_d, endBit) == 16, "sortData_d layout");
static_assert(offsetof(sortData_d, preserveEndKeys) == 20, "sortData_d layout");
static_assert(offsetof(sortData_d, earlyExit) == 21, "sortData_d layout");
static_assert(offsetof(sortData_d, parity) == 24, "sortData_d layout");
static_assert(offsetof(sortData_d, keys) == 32, "sortData_d layout");
static_assert(offsetof(sortData_d, values1) == 48, "sortData_d layout");
static_assert(offsetof(sortData_d, values6) == 128, "sortData_d layout");
static_assert(offsetof(sortData_d, pKeys) == 32, "sortData_d layout");
static_assert(sizeof(sortData_d) == 144, "sortData_d layout");

namespace {

const char* const kStatusNames[] = {
	"SORT_STATUS_SUCCESS",
	"SORT_STATUS_NOT_INITIALIZED",
	"SORT_STATUS_DEVICE_ALLOC_FAILED",
	"SORT_STATUS_HOST_ALLOC_FAILED",
	"SORT_STATUS_CONFIG_NOT_SUPPORTED",
	"SORT_STATUS_CONTEXT_MISMATCH",
	"SORT_STATUS_INVALID_CONTEXT",
	"SORT_STATUS_KERNEL_NOT_FOUND",
	"SORT_STATUS_KERNEL_ERROR",
	"SORT_STATUS_LAUNCH_ERROR",
	"SORT_STATUS_INVALID_VALUE",
	"SORT_STATUS_DEVICE_ERROR",
	"SORT_STATUS_INTERNAL_ERROR",
	"SORT_STATUS_UNSUPPORTED_DEVICE"
};

// Buffer capacity granularity of library allocations, as in the reference
// (mgpusort.cpp:663, 696).
constexpr int kAllocRound = 2048;

int round_up(int x, int m) { return (int)(((long long)x + m - 1) / m * m); }

} // namespace

// Everything the kernel arguments of one sort call depend on. Two calls with
// equal keys launch the same kernels with the same arguments (the engine's
// scratch is fixed while a key is cached), so a launch sequence captured as
// a CUDA graph can be replayed for the second and later ones.
struct GraphKey {
	int kind;                   // 0: one array, 1: segmented
	int bitPass;
	int keyType;
	int numElements;
	int valueCount;
	int firstBit;
	int endBit;
	int numSegments;
	const int* offsets;
	CUdeviceptr keys[2];
	CUdeviceptr values[6][2];
};

struct CachedGraph {
	GraphKey key;
	cudaGraphExec_t exec;
	int swaps;                  // buffer swaps the sequence makes
	unsigned long long used;
};

constexpr size_t kGraphCacheSize = 8;

struct sortEngine_d {
	long refs = 1;
	int device = 0;
	int numSMs = 0;
	mgpusort::Control* ctrl = nullptr;
	// Per-pass scratch: range digit counts, their prefixes, digit totals.
	unsigned* scratch = nullptr;
	// Segmented-sort scratch, grown on demand.
	void* segScratch = nullptr;
	size_t segScratchBytes = 0;
	// Onesweep lookback buffers (two, for alternate executed passes), grown
	// on demand: osStatusBytes each.
	void* osStatus[2] = {nullptr, nullptr};
	size_t osStatusBytes = 0;
	// Pass method of sortArray: range partition (count, scan and sort
	// launches per pass) or onesweep (one launch per pass, decoupled
	// lookback). MGPU_SORT_PASS=onesweep in the environment at engine
	// creation selects the latter.
	bool onesweep = false;
	// sortArray of more than the small-array limit and at most this many
	// elements (keys only, index mode, one value array) runs every pass in
	// one cooperative launch. MGPU_SORT_COOP_MAX in the environment at engine
	// creation overrides the built-in limit (0: never).
	int coopMax = 0;
	// Host-mapped error word written by kernels, read without synchronizing.
	volatile unsigned* hostError = nullptr;
	unsigned* hostErrorDev = nullptr;
	// Pinned host copy of the trivial-pass flags (earlyExit read-back).
	unsigned* hostTrivial = nullptr;
	cudaEvent_t done = nullptr;
	bool dirty = false;
	int failTile = -1;
	// Kernel timing (benchmarks): one event pair per timed launch.
	struct TimedLaunch { cudaEvent_t start, stop; int kind; };
	bool timing = false;
	std::vector<TimedLaunch> timed;
	size_t timedUsed = 0;
	// CUDA graphs of launch sequences that repeat (sortEnableGraphs).
	bool graphs = true;
	cudaStream_t captureStream = nullptr;
	std::vector<CachedGraph> graphCache;
	std::vector<GraphKey> seenOnce;
	unsigned long long graphClock = 0;
	int graphReplays = 0;
};

namespace {

enum { kTimedUpsweep = 0, kTimedPass = 1 };

// Opens a timed launch of `kind` on `stream`; returns its slot or -1.
int timing_begin(sortEngine_d* e, int kind, cudaStream_t stream) {
	if(!e->timing) return -1;
	if(e->timedUsed == e->timed.size()) {
		sortEngine_d::TimedLaunch t = {nullptr, nullptr, kind};
		if(cudaEventCreate(&t.start) != cudaSuccess) return -1;
		if(cudaEventCreate(&t.stop) != cudaSuccess) {
			cudaEventDestroy(t.start);
			return -1;
		}
		e->timed.push_back(t);
	}
	int slot = (int)e->timedUsed++;
	e->timed[slot].kind = kind;
	cudaEventRecord(e->timed[slot].start, stream);
	return slot;
}

void timing_end(sortEngine_d* e, int slot, cudaStream_t stream) {
	if(slot >= 0) cudaEventRecord(e->timed[slot].stop, stream);
}

// Release everything an engine holds; tolerates a partly built engine.
void destroy_engine(sortEngine_d* e) {
	if(!e) return;
	if(e->done) cudaEventSynchronize(e->done);
	for(auto& t : e->timed) {
		cudaEventDestroy(t.start);
		cudaEventDestroy(t.stop);
	}
	for(auto& g : e->graphCache) cudaGraphExecDestroy(g.exec);
	if(e->captureStream) cudaStreamDestroy(e->captureStream);
	if(e->ctrl) cudaFree(e->ctrl);
	if(e->scratch) cudaFree(e->scratch);
	if(e->segScratch) cudaFree(e->segScratch);
	if(e->osStatus[0]) cudaFree(e->osStatus[0]);
	if(e->hostError) cudaFreeHost(const_cast<unsigned*>(e->hostError));
	if(e->hostTrivial) cudaFreeHost(e->hostTrivial);
	if(e->done) cudaEventDestroy(e->done);
	delete e;
}

// sortArray's plan: the fewest passes of at most MGPU_SORT_MAX_DIGIT_BITS
// (8) bits, widths balanced (wider passes first), least significant digit
// first.
int plan_widths_default(int numBits, int* widths) {
	constexpr int kWidth = MGPU_SORT_MAX_DIGIT_BITS;
	static_assert(kWidth >= 1 && kWidth <= 8, "digits of 1..8 bits");
	int passes = (numBits + kWidth - 1) / kWidth;
	for(int p = 0; p < passes; ++p)
		widths[p] = numBits / passes + (p < numBits % passes ? 1 : 0);
	return passes;
}

// sortArrayEx's plan, as the reference builds it (mgpusort.cpp:626-646 and
// the table walk of :574-576): ceil(bits / bitPass) passes, `split` of them
// one bit narrower, the narrower ones first.
int plan_widths_reference(int numBits, int bitPass, int* widths) {
	if(bitPass <= 0 || bitPass > 6) bitPass = 6;
	if(bitPass > numBits) bitPass = numBits;
	int passes = (numBits + bitPass - 1) / bitPass;
	int split = passes * bitPass - numBits;
	for(int p = 0; p < passes; ++p) widths[p] = bitPass - (p < split ? 1 : 0);
	return passes;
}

bool make_plan(int firstBit, int numBits, int bitPass, mgpusort::PassPlan* plan) {
	int widths[mgpusort::kMaxPasses];
	int passes = bitPass ? plan_widths_reference(numBits, bitPass, widths)
		: plan_widths_default(numBits, widths);
	if(passes > mgpusort::kMaxPasses) return false;
	std::memset(plan, 0, sizeof(*plan));
	plan->numPasses = passes;
	int bit = firstBit, bin = 0;
	for(int p = 0; p < passes; ++p) {
		plan->shift[p] = bit;
		plan->width[p] = widths[p];
		plan->binBase[p] = bin;
		bit += widths[p];
		bin += 1 << widths[p];
	}
	plan->totalBins = bin;
	return bin <= mgpusort::kMaxBins;
}

bool aligned16(CUdeviceptr p) { return (p & 15) == 0; }

// Checks the status of a launch sequence. With MGPU_SORT_VERBOSE set in the
// environment, a failed launch also names its CUDA error on stderr.
sortStatus_t launch_status(cudaError_t e) {
	if(e == cudaSuccess) return SORT_STATUS_SUCCESS;
	if(std::getenv("MGPU_SORT_VERBOSE"))
		std::fprintf(stderr, "mgpusort: launch failed: %s (%s)\n", cudaGetErrorName(e),
			cudaGetErrorString(e));
	return SORT_STATUS_LAUNCH_ERROR;
}

sortStatus_t take_device_error(sortEngine_d* e) {
	unsigned err = *e->hostError;
	if(!err) return SORT_STATUS_SUCCESS;
	*e->hostError = 0;
	e->dirty = true;
	return SORT_STATUS_KERNEL_ERROR;
}

void swap_buffers(sortData_d* d) {
	std::swap(d->keys[0], d->keys[1]);
	for(int i = 0; i < 6; ++i) std::swap(d->values[i][0], d->values[i][1]);
	d->parity ^= 1;
}

GraphKey graph_key(int kind, const sortData_d* d, int bitPass, int keyType,
	const int* offsets, int numSegments) {
	GraphKey k;
	std::memset(&k, 0, sizeof(k));
	k.kind = kind;
	k.bitPass = bitPass;
	k.keyType = keyType;
	k.numElements = d->numElements;
	k.valueCount = d->valueCount;
	k.firstBit = d->firstBit;
	k.endBit = d->endBit;
	k.numSegments = numSegments;
	k.offsets = offsets;
	const int arrays = d->valueCount == -1 ? 1 : d->valueCount;
	for(int j = 0; j < 2; ++j) {
		k.keys[j] = d->keys[j];
		for(int i = 0; i < arrays; ++i) k.values[i][j] = d->values[i][j];
	}
	return k;
}

bool same_key(const GraphKey& a, const GraphKey& b) {
	return std::memcmp(&a, &b, sizeof(GraphKey)) == 0;
}

void drop_graphs(sortEngine_d* e) {
	for(auto& g : e->graphCache) cudaGraphExecDestroy(g.exec);
	e->graphCache.clear();
	e->seenOnce.clear();
}

// Makes the onesweep lookback buffers hold `bytes` bytes each. Growing them
// moves them, so every cached graph (which holds their old address) is
// dropped first.
sortStatus_t ensure_onesweep_status(sortEngine_d* e, size_t bytes) {
	if(bytes <= e->osStatusBytes) return SORT_STATUS_SUCCESS;
	drop_graphs(e);
	if(e->osStatus[0]) {
		// Earlier sorts may still read the old buffers.
		if(e->done) cudaEventSynchronize(e->done);
		cudaFree(e->osStatus[0]);
	}
	e->osStatus[0] = e->osStatus[1] = nullptr;
	e->osStatusBytes = 0;
	void* p = nullptr;
	if(cudaMalloc(&p, 2 * bytes) != cudaSuccess) {
		cudaGetLastError();
		return SORT_STATUS_DEVICE_ALLOC_FAILED;
	}
	e->osStatus[0] = p;
	e->osStatus[1] = static_cast<char*>(p) + bytes;
	e->osStatusBytes = bytes;
	return SORT_STATUS_SUCCESS;
}

// Runs a launch sequence seq(d, stream, &swaps) on `stream`. A sequence whose
// key was launched before is captured once into a CUDA graph on the
// engine's capture stream and replayed from then on (one graph launch
// instead of one launch per kernel); a key seen for the first time runs
// directly, so one-off calls pay no capture. On replay the host side makes
// the buffer swaps the sequence made when it was captured. If capture or
// instantiation fails the sequence runs directly.
template<typename Seq>
sortStatus_t run_sequence(sortEngine_d* e, sortData_d* d, const GraphKey& key,
	bool graphOk, cudaStream_t stream, Seq seq) {
	int swaps = 0;
	if(!graphOk || !e->graphs) return seq(d, stream, &swaps);
	++e->graphClock;
	for(auto& g : e->graphCache) {
		if(!same_key(g.key, key)) continue;
		if(cudaGraphLaunch(g.exec, stream) != cudaSuccess) {
			cudaGetLastError();
			return SORT_STATUS_LAUNCH_ERROR;
		}
		for(int i = 0; i < g.swaps; ++i) swap_buffers(d);
		g.used = e->graphClock;
		++e->graphReplays;
		return SORT_STATUS_SUCCESS;
	}
	bool seen = false;
	for(auto& k : e->seenOnce) seen = seen || same_key(k, key);
	if(!seen) {
		if(e->seenOnce.size() >= kGraphCacheSize) e->seenOnce.erase(e->seenOnce.begin());
		e->seenOnce.push_back(key);
		return seq(d, stream, &swaps);
	}

	// Second sighting: capture. The capture stream first waits for the
	// caller's stream (no work is captured from it; the graph launch below
	// is what orders after it).
	sortData_d shadow = *d;
	cudaGraph_t graph = nullptr;
	cudaGraphExec_t exec = nullptr;
	sortStatus_t st = SORT_STATUS_INTERNAL_ERROR;
	if(cudaStreamBeginCapture(e->captureStream, cudaStreamCaptureModeThreadLocal)
		== cudaSuccess) {
		st = seq(&shadow, e->captureStream, &swaps);
		const cudaError_t ce = cudaStreamEndCapture(e->captureStream, &graph);
		if(ce != cudaSuccess) st = SORT_STATUS_INTERNAL_ERROR;
	}
	if(st == SORT_STATUS_SUCCESS && graph &&
		cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess)
		exec = nullptr;
	if(graph) cudaGraphDestroy(graph);
	if(st != SORT_STATUS_SUCCESS || !exec) {
		cudaGetLastError();
		if(exec) cudaGraphExecDestroy(exec);
		return seq(d, stream, &swaps);
	}
	if(e->graphCache.size() >= kGraphCacheSize) {
		auto lru = std::min_element(e->graphCache.begin(), e->graphCache.end(),
			[](const CachedGraph& a, const CachedGraph& b) { return a.used < b.used; });
		cudaGraphExecDestroy(lru->exec);
		e->graphCache.erase(lru);
	}
	e->graphCache.push_back(CachedGraph{key, exec, swaps, e->graphClock});
	if(cudaGraphLaunch(exec, stream) != cudaSuccess) {
		cudaGetLastError();
		return SORT_STATUS_LAUNCH_ERROR;
	}
	for(int i = 0; i < swaps; ++i) swap_buffers(d);
	return SORT_STATUS_SUCCESS;
}

// Small arrays: one CTA sorts the whole array through every pass of the plan
// in shared memory (one launch). The result is written where the multi-pass
// sequence would leave it (buffer numPasses & 1, in place when even) and the
// struct takes the same swaps, so buffers and parity are as for any size.
sortStatus_t small_sequence(sortEngine_d* e, sortData_d* sd, cudaStream_t st, int* swaps,
	const mgpusort::PassPlan& plan, int n, bool indexMode, int numArrays, int keyType) {
	const int out = plan.numPasses & 1;
	mgpusort::PassBuffers buf = {};
	buf.keysIn = reinterpret_cast<const unsigned*>(sd->keys[0]);
	buf.keysOut = reinterpret_cast<unsigned*>(sd->keys[out]);
	for(int i = 0; i < 6; ++i) {
		buf.valsIn[i] = reinterpret_cast<const unsigned*>(sd->values[i][0]);
		buf.valsOut[i] = reinterpret_cast<unsigned*>(sd->values[i][out]);
	}
	const int slot = timing_begin(e, kTimedPass, st);
	cudaError_t ce = mgpusort::launch_small_array(buf,
		indexMode ? mgpusort::kValueIndex : numArrays, plan, n, st);
	timing_end(e, slot, st);
	e->failTile = -1;
	if(ce != cudaSuccess) { e->dirty = true; return launch_status(ce); }
	for(int p = 0; p < plan.numPasses; ++p) {
		swap_buffers(sd);
		++*swaps;
	}
	ce = mgpusort::launch_key_transform(reinterpret_cast<unsigned*>(sd->keys[0]), n,
		keyType, false, st);
	return launch_status(ce);
}

// Mid-size arrays: every pass in one cooperative launch (count, scan and
// sort phases separated by grid-wide barriers). Pass p writes buffer
// (p + 1) & 1, so the result lies where the multi-pass sequence leaves it
// and the struct takes the same swaps.
sortStatus_t coop_sequence(sortEngine_d* e, sortData_d* sd, cudaStream_t st, int* swaps,
	const mgpusort::PassPlan& plan, int n, bool indexMode, int numArrays, bool bulk,
	int keyType) {
	mgpusort::PassBuffers buf = {};
	buf.keysIn = reinterpret_cast<const unsigned*>(sd->keys[0]);
	buf.keysOut = reinterpret_cast<unsigned*>(sd->keys[1]);
	buf.valsIn[0] = reinterpret_cast<const unsigned*>(sd->values[0][0]);
	buf.valsOut[0] = reinterpret_cast<unsigned*>(sd->values[0][1]);
	const int slot = timing_begin(e, kTimedPass, st);
	cudaError_t ce = mgpusort::launch_coop_sort(buf,
		indexMode ? mgpusort::kValueIndex : numArrays, n, plan, e->ctrl, e->scratch, bulk,
		e->hostErrorDev, e->numSMs, st);
	timing_end(e, slot, st);
	if(ce != cudaSuccess) { e->dirty = true; return launch_status(ce); }
	for(int p = 0; p < plan.numPasses; ++p) {
		swap_buffers(sd);
		++*swaps;
	}
	ce = mgpusort::launch_key_transform(reinterpret_cast<unsigned*>(sd->keys[0]), n,
		keyType, false, st);
	return launch_status(ce);
}

// The onesweep launch sequence of one sort: the upsweep (every pass's digit
// offsets; clears the first lookback buffer and the tile counters), the
// earlyExit read-back of single-digit passes, then one launch per executed
// pass, and the key transform back.
sortStatus_t onesweep_sequence(sortEngine_d* e, sortData_d* sd, cudaStream_t st,
	int* swaps, const mgpusort::PassPlan& plan, int n, bool indexMode, int numArrays,
	bool bulk, size_t statusBytes, int keyType) {
	int slot = timing_begin(e, kTimedUpsweep, st);
	cudaError_t ce = mgpusort::launch_onesweep_upsweep(
		reinterpret_cast<const unsigned*>(sd->keys[0]), n, plan, e->ctrl, e->osStatus[0],
		statusBytes, e->hostErrorDev, e->numSMs, st);
	timing_end(e, slot, st);
	if(ce != cudaSuccess) { e->dirty = true; return launch_status(ce); }
	bool skip[mgpusort::kMaxPasses] = {};
	if(sd->earlyExit) {
		if(cudaMemcpyAsync(e->hostTrivial, e->ctrl->trivial,
			sizeof(unsigned) * plan.numPasses, cudaMemcpyDeviceToHost, st)
			!= cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) {
			e->dirty = true;
			return SORT_STATUS_DEVICE_ERROR;
		}
		for(int p = 0; p < plan.numPasses; ++p) skip[p] = e->hostTrivial[p] != 0;
	}
	int exec = 0;
	for(int p = 0; p < plan.numPasses; ++p) {
		if(skip[p]) continue;
		const int vm = (indexMode && exec == 0) ? mgpusort::kValueIndex : numArrays;
		mgpusort::PassBuffers buf = {};
		buf.keysIn = reinterpret_cast<const unsigned*>(sd->keys[0]);
		buf.keysOut = reinterpret_cast<unsigned*>(sd->keys[1]);
		for(int i = 0; i < 6; ++i) {
			buf.valsIn[i] = reinterpret_cast<const unsigned*>(sd->values[i][0]);
			buf.valsOut[i] = reinterpret_cast<unsigned*>(sd->values[i][1]);
		}
		slot = timing_begin(e, kTimedPass, st);
		ce = mgpusort::launch_onesweep_pass(buf, vm, n, p, exec, plan, e->ctrl,
			e->osStatus, bulk, e->failTile, e->hostErrorDev, e->numSMs, st);
		timing_end(e, slot, st);
		e->failTile = -1;
		if(ce != cudaSuccess) { e->dirty = true; return launch_status(ce); }
		swap_buffers(sd);
		++*swaps;
		++exec;
	}
	if(indexMode && exec == 0) {
		// Every pass was skipped: the identity order still needs its indices.
		ce = mgpusort::launch_iota(reinterpret_cast<unsigned*>(sd->values1[0]), n, st);
		if(ce != cudaSuccess) return launch_status(ce);
	}
	ce = mgpusort::launch_key_transform(reinterpret_cast<unsigned*>(sd->keys[0]), n,
		keyType, false, st);
	return launch_status(ce);
}

// The whole sort of one sortData_d: validation, upsweep, the pass loop.
// bitPass 0 selects sortArray's plan, 1..6 sortArrayEx's. Signed and float
// keys (keyType) are mapped to their uint32 image in place before the first
// pass and back after the last.
sortStatus_t sort_impl(sortEngine_d* e, sortData_d* d, int bitPass,
	cudaStream_t stream, int keyType = mgpusort::kKeyUint32) {
	if(!e || !d) return SORT_STATUS_INVALID_VALUE;
	sortStatus_t pending = take_device_error(e);
	if(pending != SORT_STATUS_SUCCESS) return pending;

	const int numBits = d->endBit - d->firstBit;
	if(!numBits) return SORT_STATUS_SUCCESS;   // mgpusort.cpp:610
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
	if(!n) return SORT_STATUS_SUCCESS;

	mgpusort::PassPlan plan;
	if(!make_plan(d->firstBit, numBits, bitPass, &plan))
		return SORT_STATUS_INTERNAL_ERROR;

	if(e->dirty) {
		if(cudaMemsetAsync(e->ctrl, 0, sizeof(mgpusort::Control), stream)
			!= cudaSuccess) return SORT_STATUS_DEVICE_ERROR;
		e->dirty = false;
	}

	bool bulk = true;
	for(int i = 0; i < 2; ++i) bulk = bulk && aligned16(d->keys[i]);
	for(int i = 0; i < numArrays; ++i)
		for(int j = 0; j < 2; ++j) bulk = bulk && aligned16(d->values[i][j]);

	// Onesweep: lookback buffers for this size (index mode and one value
	// array share a tile size, so the first mode decides).
	const int firstMode = indexMode ? mgpusort::kValueIndex : numArrays;
	const size_t statusBytes = mgpusort::onesweep_status_bytes(n, firstMode);
	if(e->onesweep && n > mgpusort::small_array_max_elements()) {
		const sortStatus_t gs = ensure_onesweep_status(e, statusBytes);
		if(gs != SORT_STATUS_SUCCESS) return gs;
	}

	auto seq = [&](sortData_d* sd, cudaStream_t st, int* swaps) -> sortStatus_t {
		cudaError_t ce = mgpusort::launch_key_transform(
			reinterpret_cast<unsigned*>(sd->keys[0]), n, keyType, true, st);
		if(ce != cudaSuccess) return launch_status(ce);
		if(n <= mgpusort::small_array_max_elements())
			return small_sequence(e, sd, st, swaps, plan, n, indexMode, numArrays, keyType);
		if(n <= e->coopMax && numArrays <= 1 && !sd->earlyExit && e->failTile < 0
			&& !e->onesweep)
			return coop_sequence(e, sd, st, swaps, plan, n, indexMode, numArrays, bulk,
				keyType);
		if(e->onesweep) return onesweep_sequence(e, sd, st, swaps, plan, n, indexMode,
			numArrays, bulk, statusBytes, keyType);

		// earlyExit: one upsweep builds every pass's digit histogram, one
		// read-back of the per-pass "single digit" flags, then those passes
		// are skipped (the reference reads its detect counters back per pass
		// for the same purpose, mgpusort.cpp:434-451). Without earlyExit a
		// single-digit pass runs as a straight copy.
		bool skip[mgpusort::kMaxPasses] = {};
		int slot = -1;
		if(sd->earlyExit) {
			slot = timing_begin(e, kTimedUpsweep, st);
			ce = mgpusort::launch_upsweep(
				reinterpret_cast<const unsigned*>(sd->keys[0]), n, plan, e->ctrl,
				e->hostErrorDev, e->numSMs, st);
			timing_end(e, slot, st);
			if(ce != cudaSuccess) { e->dirty = true; return launch_status(ce); }
			if(cudaMemcpyAsync(e->hostTrivial, e->ctrl->trivial,
				sizeof(unsigned) * plan.numPasses, cudaMemcpyDeviceToHost, st)
				!= cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) {
				e->dirty = true;
				return SORT_STATUS_DEVICE_ERROR;
			}
			for(int p = 0; p < plan.numPasses; ++p) skip[p] = e->hostTrivial[p] != 0;
		}

		bool firstExecuted = true;
		for(int p = 0; p < plan.numPasses; ++p) {
			if(skip[p]) continue;
			const int vm = (indexMode && firstExecuted) ? mgpusort::kValueIndex
				: numArrays;
			mgpusort::PassBuffers buf = {};
			buf.keysIn = reinterpret_cast<const unsigned*>(sd->keys[0]);
			buf.keysOut = reinterpret_cast<unsigned*>(sd->keys[1]);
			for(int i = 0; i < 6; ++i) {
				buf.valsIn[i] = reinterpret_cast<const unsigned*>(sd->values[i][0]);
				buf.valsOut[i] = reinterpret_cast<unsigned*>(sd->values[i][1]);
			}
			slot = timing_begin(e, kTimedUpsweep, st);
			ce = mgpusort::launch_pass_count(buf, vm, n, p, plan, e->scratch,
				e->numSMs, st);
			timing_end(e, slot, st);
			if(ce != cudaSuccess) { e->dirty = true; return launch_status(ce); }
			slot = timing_begin(e, kTimedPass, st);
			ce = mgpusort::launch_pass_sort(buf, vm, n, p, plan, e->ctrl, e->scratch,
				bulk, e->failTile, e->hostErrorDev, e->numSMs, st);
			timing_end(e, slot, st);
			e->failTile = -1;
			if(ce != cudaSuccess) { e->dirty = true; return launch_status(ce); }
			swap_buffers(sd);
			++*swaps;
			firstExecuted = false;
		}
		if(indexMode && firstExecuted) {
			// Every pass was skipped: the identity order still needs its
			// indices.
			ce = mgpusort::launch_iota(reinterpret_cast<unsigned*>(sd->values1[0]), n,
				st);
			if(ce != cudaSuccess) return launch_status(ce);
		}
		ce = mgpusort::launch_key_transform(reinterpret_cast<unsigned*>(sd->keys[0]), n,
			keyType, false, st);
		return launch_status(ce);
	};

	// earlyExit decides on the host mid-sequence; timing and fault
	// injection are per call: those run directly.
	const bool graphOk = !d->earlyExit && !e->timing && e->failTile < 0;
	const sortStatus_t rs = run_sequence(e, d,
		graph_key(0, d, bitPass, keyType, nullptr, 0), graphOk, stream, seq);
	if(rs != SORT_STATUS_SUCCESS) return rs;
	cudaEventRecord(e->done, stream);
	return SORT_STATUS_SUCCESS;
}

// Checks shared by the sort entry points: bit range, sizes, value mode and
// buffers. Returns SUCCESS with *work = false when there is nothing to do.
sortStatus_t validate(const sortData_d* d, bool* work) {
	*work = false;
	const int numBits = d->endBit - d->firstBit;
	if(!numBits) return SORT_STATUS_SUCCESS;
	if(numBits < 0 || numBits > 32 || d->firstBit < 0 || d->endBit > 32)
		return SORT_STATUS_INVALID_VALUE;
	if(d->numElements > d->maxElements || d->numElements < 0)
		return SORT_STATUS_INVALID_VALUE;
	if(d->valueCount < -1 || d->valueCount > 6) return SORT_STATUS_INVALID_VALUE;
	const int numArrays = d->valueCount == -1 ? 1 : d->valueCount;
	if(!d->keys[0] || !d->keys[1]) return SORT_STATUS_INVALID_VALUE;
	for(int i = 0; i < numArrays; ++i)
		if(!d->values[i][0] || !d->values[i][1]) return SORT_STATUS_INVALID_VALUE;
	*work = d->numElements > 0;
	return SORT_STATUS_SUCCESS;
}

// Makes the segmented scratch hold `bytes` bytes. The old scratch may still
// be in use by this engine's last sort: wait for it before the memory goes
// back. Growth is geometric, so a stream of growing batches reallocates only
// a few times.
sortStatus_t ensure_seg_scratch(sortEngine_d* e, size_t bytes) {
	if(bytes <= e->segScratchBytes) return SORT_STATUS_SUCCESS;
	drop_graphs(e);
	if(e->segScratch) {
		if(e->done) cudaEventSynchronize(e->done);
		cudaFree(e->segScratch);
	}
	e->segScratch = nullptr;
	const size_t grown = std::max(bytes, 2 * e->segScratchBytes);
	e->segScratchBytes = 0;
	if(cudaMalloc(&e->segScratch, grown) != cudaSuccess) {
		cudaGetLastError();
		e->segScratch = nullptr;
		return SORT_STATUS_DEVICE_ALLOC_FAILED;
	}
	e->segScratchBytes = grown;
	return SORT_STATUS_SUCCESS;
}

sortStatus_t segmented_impl(sortEngine_d* e, sortData_d* d, const int* offsets,
	int numSegments, cudaStream_t stream) {
	if(!e || !d || !offsets || numSegments < 1) return SORT_STATUS_INVALID_VALUE;
	sortStatus_t pending = take_device_error(e);
	if(pending != SORT_STATUS_SUCCESS) return pending;
	bool work = false;
	sortStatus_t st = validate(d, &work);
	if(st != SORT_STATUS_SUCCESS || !work) return st;
	const int n = d->numElements;
	const bool indexMode = d->valueCount == -1;
	const int numArrays = indexMode ? 1 : d->valueCount;

	mgpusort::PassPlan plan;
	if(!make_plan(d->firstBit, d->endBit - d->firstBit, 0, &plan))
		return SORT_STATUS_INTERNAL_ERROR;

	const sortStatus_t gs = ensure_seg_scratch(e, mgpusort::seg_scratch_bytes(n, numSegments));
	if(gs != SORT_STATUS_SUCCESS) return gs;
	if(e->dirty) {
		if(cudaMemsetAsync(e->ctrl, 0, sizeof(mgpusort::Control), stream)
			!= cudaSuccess) return SORT_STATUS_DEVICE_ERROR;
		e->dirty = false;
	}
	bool bulk = true;
	for(int i = 0; i < 2; ++i) bulk = bulk && aligned16(d->keys[i]);
	for(int i = 0; i < numArrays; ++i)
		for(int j = 0; j < 2; ++j) bulk = bulk && aligned16(d->values[i][j]);

	const int firstMode = indexMode ? mgpusort::kValueIndex : numArrays;
	auto seq = [&](sortData_d* sd, cudaStream_t st, int* swaps) -> sortStatus_t {
		cudaError_t ce = mgpusort::launch_seg_plan(offsets, numSegments, n, firstMode,
			e->segScratch, e->ctrl, e->hostErrorDev, st);
		if(ce != cudaSuccess) { e->dirty = true; return launch_status(ce); }

		// Segments of up to 4096 elements: every pass in shared memory,
		// straight into the buffers that hold the result after all passes'
		// swaps.
		const int last = plan.numPasses & 1;
		mgpusort::PassBuffers small = {};
		small.keysIn = reinterpret_cast<const unsigned*>(sd->keys[0]);
		small.keysOut = reinterpret_cast<unsigned*>(sd->keys[last]);
		for(int i = 0; i < 6; ++i) {
			small.valsIn[i] = reinterpret_cast<const unsigned*>(sd->values[i][0]);
			small.valsOut[i] = reinterpret_cast<unsigned*>(sd->values[i][last]);
		}
		int slot = timing_begin(e, kTimedUpsweep, st);
		ce = mgpusort::launch_seg_small(small, firstMode, plan, offsets, numSegments, n,
			e->segScratch, e->numSMs, st);
		timing_end(e, slot, st);
		if(ce != cudaSuccess) { e->dirty = true; return launch_status(ce); }

		for(int p = 0; p < plan.numPasses; ++p) {
			const int vm = (indexMode && p == 0) ? mgpusort::kValueIndex : numArrays;
			mgpusort::PassBuffers buf = {};
			buf.keysIn = reinterpret_cast<const unsigned*>(sd->keys[0]);
			buf.keysOut = reinterpret_cast<unsigned*>(sd->keys[1]);
			for(int i = 0; i < 6; ++i) {
				buf.valsIn[i] = reinterpret_cast<const unsigned*>(sd->values[i][0]);
				buf.valsOut[i] = reinterpret_cast<unsigned*>(sd->values[i][1]);
			}
			slot = timing_begin(e, kTimedPass, st);
			ce = mgpusort::launch_seg_pass(buf, vm, p, plan, offsets, numSegments, n,
				e->segScratch, e->ctrl, bulk, e->hostErrorDev, e->numSMs, st);
			timing_end(e, slot, st);
			if(ce != cudaSuccess) { e->dirty = true; return launch_status(ce); }
			swap_buffers(sd);
			++*swaps;
		}
		return SORT_STATUS_SUCCESS;
	};
	const sortStatus_t rs = run_sequence(e, d,
		graph_key(1, d, 0, 0, offsets, numSegments), !e->timing, stream, seq);
	if(rs != SORT_STATUS_SUCCESS) return rs;
	cudaEventRecord(e->done, stream);
	return SORT_STATUS_SUCCESS;
}

} // namespace

sortStatus_t engine_reserve_segmented(sortEngine_t engine, int n, int numSegments) {
	if(!engine || n < 0 || numSegments < 1) return SORT_STATUS_INVALID_VALUE;
	return ensure_seg_scratch(engine, mgpusort::seg_scratch_bytes(n, numSegments));
}

extern "C" {

const char* SORTAPI sortStatusString(sortStatus_t status) {
	int code = (int)status;
	if(code < 0 || code >= (int)(sizeof(kStatusNames) / sizeof(kStatusNames[0])))
		return nullptr;
	return kStatusNames[code];
}

sortStatus_t SORTAPI sortCreateEngine(const char* kernelPath,
	sortEngine_t* engine) {
	(void)kernelPath;
	if(!engine) return SORT_STATUS_INVALID_VALUE;
	*engine = nullptr;
	int device = 0;
	if(cudaGetDevice(&device) != cudaSuccess) {
		cudaGetLastError();
		return SORT_STATUS_INVALID_CONTEXT;
	}
	cudaDeviceProp prop;
	if(cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
		cudaGetLastError();
		return SORT_STATUS_INVALID_CONTEXT;
	}
	if(prop.major != 10 || prop.minor != 0) return SORT_STATUS_UNSUPPORTED_DEVICE;

	sortEngine_d* e = new sortEngine_d;
	e->device = device;
	e->numSMs = prop.multiProcessorCount;
	if(const char* m = std::getenv("MGPU_SORT_PASS"))
		e->onesweep = std::strcmp(m, "onesweep") == 0;
	e->coopMax = mgpusort::coop_max_elements();
	if(const char* m = std::getenv("MGPU_SORT_COOP_MAX")) e->coopMax = std::atoi(m);
	sortStatus_t status = SORT_STATUS_SUCCESS;
	void* p = nullptr;
	if(mgpusort::configure_kernels() != cudaSuccess)
		status = SORT_STATUS_KERNEL_ERROR;
	else if(cudaMalloc(&p, sizeof(mgpusort::Control)) != cudaSuccess)
		status = SORT_STATUS_DEVICE_ALLOC_FAILED;
	else {
		e->ctrl = static_cast<mgpusort::Control*>(p);
		if(cudaMemset(e->ctrl, 0, sizeof(mgpusort::Control)) != cudaSuccess)
			status = SORT_STATUS_DEVICE_ERROR;
		else if(cudaMalloc(&p, mgpusort::pass_scratch_bytes()) != cudaSuccess)
			status = SORT_STATUS_DEVICE_ALLOC_FAILED;
		else e->scratch = static_cast<unsigned*>(p);
	}
	if(status == SORT_STATUS_SUCCESS) {
		void* h = nullptr;
		if(cudaHostAlloc(&h, sizeof(unsigned), cudaHostAllocMapped) != cudaSuccess)
			status = SORT_STATUS_HOST_ALLOC_FAILED;
		else {
			e->hostError = static_cast<unsigned*>(h);
			*e->hostError = 0;
			void* dp = nullptr;
			if(cudaHostGetDevicePointer(&dp, h, 0) != cudaSuccess)
				status = SORT_STATUS_HOST_ALLOC_FAILED;
			e->hostErrorDev = static_cast<unsigned*>(dp);
		}
	}
	if(status == SORT_STATUS_SUCCESS) {
		void* h = nullptr;
		if(cudaHostAlloc(&h, sizeof(unsigned) * mgpusort::kMaxPasses,
			cudaHostAllocDefault) != cudaSuccess)
			status = SORT_STATUS_HOST_ALLOC_FAILED;
		e->hostTrivial = static_cast<unsigned*>(h);
	}
	if(status == SORT_STATUS_SUCCESS &&
		(cudaEventCreateWithFlags(&e->done, cudaEventDisableTiming) != cudaSuccess ||
		cudaStreamCreateWithFlags(&e->captureStream, cudaStreamNonBlocking) != cudaSuccess))
		status = SORT_STATUS_DEVICE_ERROR;
	if(status != SORT_STATUS_SUCCESS) {
		cudaGetLastError();
		destroy_engine(e);
		return status;
	}
	*engine = e;
	return SORT_STATUS_SUCCESS;
}

sortStatus_t SORTAPI sortLoadKernel(sortEngine_t engine, int numSortThreads,
	int valuesPerThread, bool useTransList, int valueCount) {
	(void)useTransList;
	if(!engine) return SORT_STATUS_INVALID_VALUE;
	// The reference's checks (mgpusort.cpp:148-153).
	if(numSortThreads != 128 && numSortThreads != 256)
		return SORT_STATUS_INVALID_VALUE;
	if(valuesPerThread != 4 && valuesPerThread != 8)
		return SORT_STATUS_INVALID_VALUE;
	if(valueCount < -1 || valueCount > 6) return SORT_STATUS_INVALID_VALUE;
	return mgpusort::configure_kernels() == cudaSuccess ? SORT_STATUS_SUCCESS
		: SORT_STATUS_KERNEL_ERROR;
}

sortStatus_t SORTAPI sortIncEngine(sortEngine_t engine) {
	if(!engine) return SORT_STATUS_INVALID_VALUE;
	++engine->refs;
	return SORT_STATUS_SUCCESS;
}

sortStatus_t SORTAPI sortReleaseEngine(sortEngine_t engine) {
	if(engine && !--engine->refs) destroy_engine(engine);
	return SORT_STATUS_SUCCESS;
}

sortStatus_t SORTAPI sortCreateData(sortEngine_t engine, int maxElements,
	int valueCount, sortData_t* data) {
	if(!data || valueCount > 6 || valueCount < -1 || maxElements < 0)
		return SORT_STATUS_INVALID_VALUE;
	sortData_d* d = new sortData_d;
	std::memset(d, 0, sizeof(*d));
	d->maxElements = round_up(maxElements, kAllocRound);
	d->numElements = maxElements;
	d->valueCount = valueCount;
	d->firstBit = 0;
	d->endBit = 32;
	sortStatus_t status = sortAllocData(engine, d);
	if(status != SORT_STATUS_SUCCESS) {
		sortFreeData(d);
		delete d;
		*data = nullptr;
		return status;
	}
	*data = d;
	return SORT_STATUS_SUCCESS;
}

sortStatus_t SORTAPI sortDestroyData(sortData_t data) {
	if(!data) return SORT_STATUS_SUCCESS;
	sortFreeData(data);
	delete data;
	return SORT_STATUS_SUCCESS;
}

sortStatus_t SORTAPI sortAllocData(sortEngine_t engine, sortData_t data) {
	(void)engine;
	if(!data || data->valueCount > 6 || data->valueCount < -1 ||
		data->maxElements < 0) return SORT_STATUS_INVALID_VALUE;
	const size_t elems = (size_t)round_up(data->maxElements, kAllocRound);
	const int count = data->valueCount == -1 ? 1 : data->valueCount;
	// keys[0], keys[1], values1[0], values1[1], ... are consecutive.
	CUdeviceptr* slots = data->keys;
	CUdeviceptr fresh[14] = {};
	for(int i = 0; i < 2 + 2 * count; ++i) {
		if(slots[i]) continue;
		void* p = nullptr;
		if(elems && cudaMalloc(&p, elems * sizeof(unsigned)) != cudaSuccess) {
			cudaGetLastError();
			for(int j = 0; j < i; ++j)
				if(fresh[j]) cudaFree(reinterpret_cast<void*>(fresh[j]));
			return SORT_STATUS_DEVICE_ALLOC_FAILED;
		}
		fresh[i] = reinterpret_cast<CUdeviceptr>(p);
	}
	for(int i = 0; i < 2 + 2 * count; ++i)
		if(fresh[i]) slots[i] = fresh[i];
	data->parity = 0;
	return SORT_STATUS_SUCCESS;
}

sortStatus_t SORTAPI sortFreeData(sortData_d* data) {
	if(!data) return SORT_STATUS_INVALID_VALUE;
	for(int i = 0; i < 2; ++i) {
		if(data->keys[i]) cudaFree(reinterpret_cast<void*>(data->keys[i]));
		for(int j = 0; j < 6; ++j)
			if(data->values[j][i])
				cudaFree(reinterpret_cast<void*>(data->values[j][i]));
	}
	std::memset(data, 0, sizeof(*data));
	return SORT_STATUS_SUCCESS;
}

sortStatus_t SORTAPI sortArray(sortEngine_t engine, sortData_t data) {
	return sort_impl(engine, data, 0, cudaStreamLegacy);
}

sortStatus_t SORTAPI sortArrayEx(sortEngine_t engine, sortData_t data,
	int numSortThreads, int valuesPerThread, int bitPass, bool useTransList) {
	(void)useTransList;
	if(!data) return SORT_STATUS_INVALID_VALUE;
	// mgpusort.cpp:621-626.
	if((numSortThreads != 128 && numSortThreads != 256) || valuesPerThread != 8)
		return SORT_STATUS_INVALID_VALUE;
	if(data->numElements > data->maxElements) return SORT_STATUS_INVALID_VALUE;
	if(bitPass <= 0 || bitPass > 6) bitPass = 6;
	return sort_impl(engine, data, bitPass, cudaStreamLegacy);
}

sortStatus_t SORTAPI sortArrayAsync(sortEngine_t engine, sortData_t data,
	CUstream stream) {
	return sort_impl(engine, data, 0, reinterpret_cast<cudaStream_t>(stream));
}

sortStatus_t SORTAPI sortArrayTyped(sortEngine_t engine, sortData_t data,
	int keyType, CUstream stream) {
	if(keyType != mgpusort::kKeyUint32 && keyType != mgpusort::kKeyInt32 &&
		keyType != mgpusort::kKeyFloat32) return SORT_STATUS_INVALID_VALUE;
	return sort_impl(engine, data, 0, reinterpret_cast<cudaStream_t>(stream), keyType);
}

sortStatus_t SORTAPI sortSelectKey(sortEngine_t engine, sortData_t data, int k,
	unsigned int* value) {
	if(!engine || !data || !value || k < 0 || k >= data->numElements)
		return SORT_STATUS_INVALID_VALUE;
	sortStatus_t st = sort_impl(engine, data, 0, cudaStreamLegacy);
	if(st != SORT_STATUS_SUCCESS) return st;
	const unsigned* keys = reinterpret_cast<const unsigned*>(data->keys[0]);
	if(cudaMemcpy(value, keys + k, sizeof(unsigned), cudaMemcpyDeviceToHost)
		!= cudaSuccess) {
		cudaGetLastError();
		return SORT_STATUS_DEVICE_ERROR;
	}
	return take_device_error(engine);
}

sortStatus_t SORTAPI sortSegmentedArray(sortEngine_t engine, sortData_t data,
	const int* segmentOffsets, int numSegments, CUstream stream) {
	return segmented_impl(engine, data, segmentOffsets, numSegments,
		stream ? reinterpret_cast<cudaStream_t>(stream) : cudaStreamLegacy);
}

sortStatus_t SORTAPI sortSynchronize(sortEngine_t engine) {
	if(!engine) return SORT_STATUS_INVALID_VALUE;
	if(cudaEventSynchronize(engine->done) != cudaSuccess) {
		cudaGetLastError();
		return SORT_STATUS_DEVICE_ERROR;
	}
	return take_device_error(engine);
}

int SORTAPI sortPlanPasses(int firstBit, int endBit, int bitPass,
	int* widths) {
	const int numBits = endBit - firstBit;
	if(firstBit < 0 || endBit > 32 || numBits < 0 || !widths) return -1;
	if(!numBits) return 0;
	if(bitPass < 0 || bitPass > 6) return -1;
	return bitPass ? plan_widths_reference(numBits, bitPass, widths)
		: plan_widths_default(numBits, widths);
}

sortStatus_t SORTAPI sortEnableGraphs(sortEngine_t engine, int enable) {
	if(!engine) return SORT_STATUS_INVALID_VALUE;
	engine->graphs = enable != 0;
	if(!engine->graphs) drop_graphs(engine);
	return SORT_STATUS_SUCCESS;
}

sortStatus_t SORTAPI sortGraphStats(sortEngine_t engine, int* replays, int* cached) {
	if(!engine) return SORT_STATUS_INVALID_VALUE;
	if(replays) *replays = engine->graphReplays;
	if(cached) *cached = (int)engine->graphCache.size();
	return SORT_STATUS_SUCCESS;
}

sortStatus_t SORTAPI sortInjectFault(sortEngine_t engine, int tile) {
	if(!engine || tile < -1) return SORT_STATUS_INVALID_VALUE;
	engine->failTile = tile;
	return SORT_STATUS_SUCCESS;
}

sortStatus_t SORTAPI sortEnableKernelTiming(sortEngine_t engine, int enable) {
	if(!engine) return SORT_STATUS_INVALID_VALUE;
	engine->timing = enable != 0;
	return SORT_STATUS_SUCCESS;
}

sortStatus_t SORTAPI sortReadKernelTiming(sortEngine_t engine,
	double* upsweepMs, int* upsweepLaunches, double* passMs, int* passLaunches) {
	if(!engine) return SORT_STATUS_INVALID_VALUE;
	double ms[2] = {0, 0};
	int launches[2] = {0, 0};
	sortStatus_t status = SORT_STATUS_SUCCESS;
	for(size_t i = 0; i < engine->timedUsed; ++i) {
		auto& t = engine->timed[i];
		float f = 0;
		if(cudaEventSynchronize(t.stop) != cudaSuccess ||
			cudaEventElapsedTime(&f, t.start, t.stop) != cudaSuccess) {
			cudaGetLastError();
			status = SORT_STATUS_DEVICE_ERROR;
			continue;
		}
		ms[t.kind] += f;
		++launches[t.kind];
	}
	engine->timedUsed = 0;
	if(upsweepMs) *upsweepMs = ms[kTimedUpsweep];
	if(upsweepLaunches) *upsweepLaunches = launches[kTimedUpsweep];
	if(passMs) *passMs = ms[kTimedPass];
	if(passLaunches) *passLaunches = launches[kTimedPass];
	return status;
}

sortStatus_t SORTAPI sortHost(sortEngine_t engine, unsigned int* keys,
	unsigned int* values, int numElements, int numBits) {
	if(!engine || !keys || numElements < 0 || numBits < 0 || numBits > 32)
		return SORT_STATUS_INVALID_VALUE;
	if(!numElements) return SORT_STATUS_SUCCESS;
	sortData_d d;
	std::memset(&d, 0, sizeof(d));
	d.maxElements = numElements;
	d.numElements = numElements;
	d.valueCount = values ? 1 : 0;
	d.endBit = numBits;
	sortStatus_t status = sortAllocData(engine, &d);
	if(status != SORT_STATUS_SUCCESS) return status;
	const size_t bytes = sizeof(unsigned) * (size_t)numElements;
	if(cudaMemcpy(reinterpret_cast<void*>(d.keys[0]), keys, bytes,
		cudaMemcpyHostToDevice) != cudaSuccess ||
		(values && cudaMemcpy(reinterpret_cast<void*>(d.values1[0]), values,
			bytes, cudaMemcpyHostToDevice) != cudaSuccess))
		status = SORT_STATUS_DEVICE_ERROR;
	if(status == SORT_STATUS_SUCCESS) status = sortArray(engine, &d);
	if(status == SORT_STATUS_SUCCESS) {
		if(cudaMemcpy(keys, reinterpret_cast<void*>(d.keys[0]), bytes,
			cudaMemcpyDeviceToHost) != cudaSuccess ||
			(values && cudaMemcpy(values, reinterpret_cast<void*>(d.values1[0]),
				bytes, cudaMemcpyDeviceToHost) != cudaSuccess))
			status = SORT_STATUS_DEVICE_ERROR;
	}
	if(status == SORT_STATUS_SUCCESS) status = sortSynchronize(engine);
	cudaGetLastError();
	sortFreeData(&d);
	return status;
}

sortStatus_t SORTAPI sortDevice(sortEngine_t engine, CUdeviceptr keys,
	CUdeviceptr values, int numElements, int numBits) {
	if(!engine || !keys || numElements < 0 || numBits < 0 || numBits > 32)
		return SORT_STATUS_INVALID_VALUE;
	if(!numElements) return SORT_STATUS_SUCCESS;
	sortData_d d;
	std::memset(&d, 0, sizeof(d));
	d.keys[0] = keys;
	d.values1[0] = values;
	d.maxElements = numElements;
	d.numElements = numElements;
	d.valueCount = values ? 1 : 0;
	d.endBit = numBits;
	sortStatus_t status = sortAllocData(engine, &d);
	if(status != SORT_STATUS_SUCCESS) return status;
	status = sortArray(engine, &d);
	const size_t bytes = sizeof(unsigned) * (size_t)numElements;
	if(status == SORT_STATUS_SUCCESS && d.keys[0] != keys) {
		// An odd number of passes: the result is in the library's buffer.
		if(cudaMemcpyAsync(reinterpret_cast<void*>(keys),
			reinterpret_cast<void*>(d.keys[0]), bytes, cudaMemcpyDeviceToDevice,
			cudaStreamLegacy) != cudaSuccess ||
			(values && cudaMemcpyAsync(reinterpret_cast<void*>(values),
				reinterpret_cast<void*>(d.values1[0]), bytes,
				cudaMemcpyDeviceToDevice, cudaStreamLegacy) != cudaSuccess))
			status = SORT_STATUS_DEVICE_ERROR;
	}
	if(status == SORT_STATUS_SUCCESS) {
		if(cudaStreamSynchronize(cudaStreamLegacy) != cudaSuccess)
			status = SORT_STATUS_DEVICE_ERROR;
		else status = take_device_error(engine);
	}
	cudaGetLastError();
	// Free only the library's buffers.
	for(int i = 0; i < 2; ++i) {
		if(d.keys[i] == keys) d.keys[i] = 0;
		if(d.values1[i] == values) d.values1[i] = 0;
	}
	sortFreeData(&d);
	return status;
}

} // extern "C"
