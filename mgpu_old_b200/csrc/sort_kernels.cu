// Radix sort kernels for sm_100a.
//
// A sort over the bit range [firstBit, endBit) runs as
//   1. one upsweep launch that reads every key once and builds the digit
//      histograms of all passes, then (last CTA) their exclusive scans;
//   2. one onesweep launch per pass (least significant digit first). Each CTA
//      takes the next tile id from an atomic counter, stages its tile of keys
//      (and value arrays) in shared memory with bulk copies, ranks the keys
//      stably by digit, finds the tile's global digit offsets with a
//      decoupled lookback over the tiles before it, reorders the tile in
//      shared memory into digit runs and writes each run contiguously.
//
// This replaces the reference's per-pass count / hist1 / hist2 / hist3 / sort
// kernel chain (sort/src/mgpusort/mgpusort.cpp:421-516; kernels
// sort/src/kernels/count.cu, hist1.cu, hist2.cu, hist3.cu, sort.cu) with two
// kernels and one read of the keys for all counting. The ordering contract is
// the same: every pass is a stable partition by its digit, so the passes
// compose into a stable sort by the whole bit field.

#include "sort_kernels.h"
#include "sort_device.cuh"

#include <algorithm>

namespace mgpusort {

////////////////////////////////////////////////////////////////////////////////
// Upsweep: digit histograms of every pass in one read of the keys.

constexpr int kUpThreads = 512;
constexpr int kUpKeysPerThread = 16;
constexpr int kUpChunk = kUpThreads * kUpKeysPerThread;

struct UpsweepArgs {
	const unsigned* keys;
	int n;
	int vecOk;
	PassPlan plan;
	Control* ctrl;
	volatile unsigned* hostError;
};

// Count nValid (a prefix of) keys into a shared histogram. Runs of equal
// digits in a thread's keys are merged into one atomic, which keeps skewed
// digits (e.g. all-zero high bytes) from serialising on one counter.
__device__ __forceinline__ void count_digits(unsigned* hist,
	const unsigned (&k)[kUpKeysPerThread], int nValid, int shift,
	unsigned mask) {
	unsigned cur = (k[0] >> shift) & mask;
	unsigned run = 0;
#pragma unroll
	for(int i = 0; i < kUpKeysPerThread; ++i) {
		if(i < nValid) {
			unsigned d = (k[i] >> shift) & mask;
			if(d != cur) {
				atomicAdd(&hist[cur], run);
				cur = d;
				run = 1;
			} else ++run;
		}
	}
	if(run) atomicAdd(&hist[cur], run);
}

__global__ void __launch_bounds__(kUpThreads, 3) upsweep_kernel(
	const UpsweepArgs a) {

	__shared__ unsigned sHist[kMaxBins];
	__shared__ unsigned sScan[kUpThreads / 32];
	__shared__ unsigned sLast;

	const int tid = threadIdx.x;
	const int lane = tid & 31;
	const int warp = tid >> 5;
	const int totalBins = a.plan.totalBins;
	const int numPasses = a.plan.numPasses;

	for(int i = tid; i < totalBins; i += kUpThreads) sHist[i] = 0;
	__syncthreads();

	auto count_all = [&](const unsigned (&k)[kUpKeysPerThread], int nValid) {
		for(int p = 0; p < numPasses; ++p)
			count_digits(sHist + a.plan.binBase[p], k, nValid, a.plan.shift[p],
				(1u << a.plan.width[p]) - 1);
	};

	// Full chunks with 16-byte loads, the next chunk's loads in flight while
	// the current one is counted.
	const long long fullChunks = a.vecOk ? a.n / kUpChunk : 0;
	long long c = blockIdx.x;
	uint4 next[kUpKeysPerThread / 4];
	if(c < fullChunks) {
		const uint4* src = reinterpret_cast<const uint4*>(a.keys + c * kUpChunk);
#pragma unroll
		for(int i = 0; i < kUpKeysPerThread / 4; ++i)
			next[i] = ld_stream_u4(src + i * kUpThreads + tid);
	}
	for(; c < fullChunks; c += gridDim.x) {
		unsigned k[kUpKeysPerThread];
#pragma unroll
		for(int i = 0; i < kUpKeysPerThread / 4; ++i) {
			k[4 * i + 0] = next[i].x;
			k[4 * i + 1] = next[i].y;
			k[4 * i + 2] = next[i].z;
			k[4 * i + 3] = next[i].w;
		}
		if(c + gridDim.x < fullChunks) {
			const uint4* src = reinterpret_cast<const uint4*>(
				a.keys + (c + gridDim.x) * kUpChunk);
#pragma unroll
			for(int i = 0; i < kUpKeysPerThread / 4; ++i)
				next[i] = ld_stream_u4(src + i * kUpThreads + tid);
		}
		count_all(k, kUpKeysPerThread);
	}

	// The rest (a ragged tail, or everything when the keys are not 16-byte
	// aligned) with plain loads. Element (i, j) of this thread sits at
	// base + (i*NT + tid)*4 + j, increasing in (i, j): the valid elements
	// form a prefix.
	for(long long r = fullChunks + blockIdx.x; r * kUpChunk < a.n; r += gridDim.x) {
		const long long base = r * kUpChunk;
		unsigned k[kUpKeysPerThread];
		int nValid = 0;
#pragma unroll
		for(int i = 0; i < kUpKeysPerThread / 4; ++i)
#pragma unroll
			for(int j = 0; j < 4; ++j) {
				long long idx = base + (long long)(i * kUpThreads + tid) * 4 + j;
				bool valid = idx < a.n;
				k[4 * i + j] = valid ? a.keys[idx] : 0u;
				nValid += valid;
			}
		count_all(k, nValid);
	}
	__syncthreads();

	for(int i = tid; i < totalBins; i += kUpThreads) {
		unsigned c = sHist[i];
		if(c) atomicAdd(&a.ctrl->hist[i], c);
	}
	__threadfence();
	__syncthreads();
	if(tid == 0) {
		unsigned ticket = atomicAdd(&a.ctrl->ticket, 1u);
		sLast = (ticket == gridDim.x - 1);
	}
	__syncthreads();
	if(!sLast) return;

	// Last CTA: every other CTA's histogram is in ctrl->hist.
	__threadfence();
	for(int p = 0; p < numPasses; ++p) {
		const int bins = 1 << a.plan.width[p];
		unsigned* hist = a.ctrl->hist + a.plan.binBase[p];
		unsigned c = 0;
		if(tid < bins) c = ld_relaxed_u32(hist + tid);
		unsigned incl = warp_inclusive_scan(c, lane);
		if(lane == 31) sScan[warp] = incl;
		int nonEmpty = __syncthreads_count(c != 0);
		unsigned prefix = 0;
		for(int w = 0; w < warp; ++w) prefix += sScan[w];
		if(tid < bins) {
			a.ctrl->offsets[a.plan.binBase[p] + tid] = prefix + incl - c;
			hist[tid] = 0;
		}
		if(tid == 0) a.ctrl->trivial[p] = nonEmpty <= 1;
		__syncthreads();
	}
	if(tid == 0) a.ctrl->ticket = 0;
}

////////////////////////////////////////////////////////////////////////////////
// Onesweep pass.

struct PassArgs {
	PassBuffers buf;
	const unsigned* digitOffsets;   // exclusive global start of each digit
	const unsigned* trivial;        // nonzero: one digit only, pass = copy
	unsigned* tileCounter;
	unsigned long long* status;     // [numTiles][256] lookback words
	unsigned* devError;
	volatile unsigned* hostError;
	int n;
	int numTiles;
	int shift;
	int width;
	unsigned epoch;
	int useBulk;
	int failTile;                   // tile that skips publishing; -1: none
};

// Lookback word: epoch (30 bits) | flag (2 bits) | count (32 bits). A word
// whose epoch is not the current pass's is treated as not yet published, so
// the status array never needs clearing between passes.
constexpr unsigned long long kFlagAggregate = 1ull << 32;
constexpr unsigned long long kFlagInclusive = 2ull << 32;

template<int VM> struct PassConfig {
	static constexpr int kThreads = 256;
	static constexpr int kItems = 16;
	static constexpr int kMinBlocks = 4;
};

template<int VM> struct PassLayout {
	static constexpr int NT = PassConfig<VM>::kThreads;
	static constexpr int IPT = PassConfig<VM>::kItems;
	static constexpr int TILE = NT * IPT;
	static constexpr int NW = NT / 32;
	// Value staging buffers: index mode writes its generated indices into
	// one, value arrays are double-buffered.
	static constexpr int NSTAGE = VM >= 2 ? 2 : (VM == 0 ? 0 : 1);
	// Word offsets into dynamic shared memory.
	static constexpr int kKeys = 0;
	static constexpr int kVals = kKeys + TILE;
	static constexpr int kWarpHist = kVals + NSTAGE * TILE;
	static constexpr int kDigStart = kWarpHist + NW * kDigitBins;
	static constexpr int kScatter = kDigStart + kDigitBins;
	static constexpr int kScan = kScatter + kDigitBins;
	static constexpr int kBar = kScan + 32;          // 8-byte aligned: even
	static constexpr int kTile = kBar + 2 * 4;
	static constexpr int kWords = kTile + 4;
	static constexpr size_t kBytes = sizeof(unsigned) * kWords;
	static_assert(kBar % 2 == 0, "mbarriers need 8-byte alignment");
};

// Identity pass (all keys share the digit): copy the tile through.
template<int VM>
__device__ __forceinline__ void copy_tile(const PassArgs& a, long long start,
	int count) {
	constexpr int NT = PassLayout<VM>::NT;
	const int tid = threadIdx.x;
	for(int i = tid; i < count; i += NT) {
		a.buf.keysOut[start + i] = a.buf.keysIn[start + i];
		if constexpr(VM == kValueIndex)
			a.buf.valsOut[0][start + i] = (unsigned)(start + i);
#pragma unroll
		for(int v = 0; v < (VM > 0 ? VM : 0); ++v)
			a.buf.valsOut[v][start + i] = a.buf.valsIn[v][start + i];
	}
}

// Lanes of the warp whose 8-bit digit equals this lane's, from one ballot per
// digit bit (a lane keeps the ballot where its bit is set, the complement
// where it is clear).
__device__ __forceinline__ unsigned match_digit8(unsigned d) {
	unsigned peers = 0xffffffffu;
#pragma unroll
	for(int b = 0; b < 8; ++b) {
		const bool set = (d >> b) & 1u;
		const unsigned bal = __ballot_sync(0xffffffffu, set);
		peers &= set ? bal : ~bal;
	}
	return peers;
}

// Decoupled lookback of one digit: sum the counts of the tiles before `tile`
// back to the nearest one that published an inclusive prefix. Reads up to
// four predecessors per step so that a walk over published aggregates costs
// one memory round trip per four tiles.
__device__ __forceinline__ unsigned lookback_digit(
	const unsigned long long* status, int tile, int digit, unsigned epoch,
	bool* timedOut) {
	unsigned excl = 0;
	int j = tile - 1;
	WaitBudget budget;
	while(true) {
		unsigned long long w[4];
#pragma unroll
		for(int k = 0; k < 4; ++k)
			w[k] = j - k >= 0
				? ld_relaxed_u64(status + (size_t)(j - k) * kDigitBins + digit) : 0ull;
		int consumed = 0;
		bool done = false, stalled = false;
#pragma unroll
		for(int k = 0; k < 4; ++k) {
			if(done || stalled) continue;
			const unsigned long long flag = w[k] & (3ull << 32);
			if(j - k < 0 || (w[k] >> 34) != epoch || !flag) {
				stalled = true;
				continue;
			}
			excl += (unsigned)w[k];
			++consumed;
			if(flag == kFlagInclusive) done = true;
		}
		if(done) break;
		j -= consumed;
		if(consumed) budget = WaitBudget();
		else if(!budget.poll()) {
			*timedOut = true;
			break;
		}
	}
	return excl;
}

template<int VM>
__global__ void __launch_bounds__(PassLayout<VM>::NT, PassConfig<VM>::kMinBlocks)
onesweep_kernel(const PassArgs a) {

	using L = PassLayout<VM>;
	constexpr int NT = L::NT;
	constexpr int IPT = L::IPT;
	constexpr int TILE = L::TILE;
	constexpr int NW = L::NW;
	constexpr int NV = VM > 0 ? VM : 0;
	// Value arrays (or generated indices) reordered in shared memory before
	// the lookback; the rest stream through the staging buffers after it.
	constexpr int NPRE = VM == kValueIndex ? 1 : (NV < 2 ? NV : 2);

	extern __shared__ __align__(128) unsigned smem[];
	unsigned* sKeys = smem + L::kKeys;
	unsigned* sVals = smem + L::kVals;
	unsigned* sWarpHist = smem + L::kWarpHist;
	unsigned* sDigStart = smem + L::kDigStart;
	int* sScatter = reinterpret_cast<int*>(smem + L::kScatter);
	unsigned* sScan = smem + L::kScan;
	uint64_t* sBar = reinterpret_cast<uint64_t*>(smem + L::kBar);
	unsigned* sTile = smem + L::kTile;

	const int tid = threadIdx.x;
	const int lane = tid & 31;
	const int warp = tid >> 5;

	if(tid == 0) {
		unsigned t = atomicAdd(a.tileCounter, 1u);
		// Every CTA of this launch has drawn its id once this one has the
		// last: re-arm the counter for the next launch.
		if(t == (unsigned)a.numTiles - 1) *a.tileCounter = 0;
		sTile[0] = t;
		sTile[1] = *a.trivial;
		if(a.useBulk) {
			mbar_init(&sBar[0], 1);
			mbar_init(&sBar[1], 1);
			mbar_init(&sBar[2], 1);
			fence_mbar_init();
		}
	}
	for(int i = tid; i < NW * kDigitBins; i += NT) sWarpHist[i] = 0;
	__syncthreads();

	const int tile = (int)sTile[0];
	const long long tileStart = (long long)tile * TILE;
	const int count = (int)min((long long)TILE, (long long)a.n - tileStart);

	if(sTile[1]) {
		copy_tile<VM>(a, tileStart, count);
		return;
	}

	const bool bulk = a.useBulk && count == TILE;
	if(bulk && tid == 0) {
		mbar_arrive_expect_tx(&sBar[0], TILE * 4);
		bulk_load(sKeys, a.buf.keysIn + tileStart, TILE * 4, &sBar[0]);
		if constexpr(NV >= 1) {
			mbar_arrive_expect_tx(&sBar[1], TILE * 4);
			bulk_load(sVals, a.buf.valsIn[0] + tileStart, TILE * 4, &sBar[1]);
		}
		if constexpr(NV >= 2) {
			mbar_arrive_expect_tx(&sBar[2], TILE * 4);
			bulk_load(sVals + TILE, a.buf.valsIn[1] + tileStart, TILE * 4,
				&sBar[2]);
		}
	}

	// Keys in warp-striped order: item i of lane l in warp w is tile element
	// w*32*IPT + i*32 + l, so (item, lane) order is input order per warp.
	const int warpBase = warp * 32 * IPT;
	unsigned keys[IPT];
	if(bulk) {
		if(!mbar_wait_bounded(&sBar[0], 0))
			report_error(a.devError, a.hostError, kErrBarrierTimeout);
#pragma unroll
		for(int i = 0; i < IPT; ++i) keys[i] = sKeys[warpBase + i * 32 + lane];
	} else {
#pragma unroll
		for(int i = 0; i < IPT; ++i) {
			int idx = warpBase + i * 32 + lane;
			keys[i] = idx < count ? a.buf.keysIn[tileStart + idx] : 0xffffffffu;
		}
	}

	const unsigned mask = (1u << a.width) - 1;
	const int shift = a.shift;
	// Padding of a partial tile gets digit 255: it ranks after every real
	// key (it is last in input order and 255 is the last bin) and is never
	// stored.
	auto digit_of = [&](int i) -> unsigned {
		int idx = warpBase + i * 32 + lane;
		return idx < count ? (keys[i] >> shift) & mask : (kDigitBins - 1);
	};

	// Stable rank within the warp: peers with the same digit are ranked by
	// lane, items in order. The highest peer adds the group to the warp's
	// running count of the digit; the atomic's old value, broadcast, is the
	// group's base. The shuffle orders each item's update before the next.
	unsigned* myHist = sWarpHist + warp * kDigitBins;
	const unsigned ltMask = lanemask_lt();
	unsigned rank[IPT];
#pragma unroll
	for(int i = 0; i < IPT; ++i) {
		const unsigned d = digit_of(i);
		const unsigned peers = match_digit8(d);
		const int leader = 31 - __clz(peers);
		unsigned base = 0;
		if(lane == leader) base = atomicAdd(&myHist[d], (unsigned)__popc(peers));
		base = __shfl_sync(0xffffffffu, base, leader);
		rank[i] = base + __popc(peers & ltMask);
	}
	__syncthreads();

	// Per digit: exclusive offsets of the warps, and the tile's count.
	unsigned total = 0;
	if(tid < kDigitBins) {
#pragma unroll
		for(int w = 0; w < NW; ++w) {
			unsigned c = sWarpHist[w * kDigitBins + tid];
			sWarpHist[w * kDigitBins + tid] = total;
			total += c;
		}
	}
	const unsigned incl = warp_inclusive_scan(total, lane);
	if(lane == 31 && tid < kDigitBins) sScan[warp] = incl;
	__syncthreads();

	// Publish this tile's digit counts as soon as they are known.
	const unsigned long long epochBits = (unsigned long long)a.epoch << 34;
	unsigned digStart = 0;
	unsigned mine = 0;
	if(tid < kDigitBins) {
		unsigned prefix = 0;
		for(int w = 0; w < warp; ++w) prefix += sScan[w];
		digStart = prefix + incl - total;
		sDigStart[tid] = digStart;
		mine = total;
		if(tid == kDigitBins - 1) mine -= TILE - count;
		if(tid <= (int)mask && tile != a.failTile) {
			unsigned long long* st = a.status + (size_t)tile * kDigitBins + tid;
			st_relaxed_u64(st, epochBits | (tile == 0 ? kFlagInclusive : kFlagAggregate)
				| mine);
		}
	}
	__syncthreads();

	// Reorder the tile in shared memory into digit runs: keys, then the
	// value arrays whose tiles are already staged (or generated indices).
#pragma unroll
	for(int i = 0; i < IPT; ++i) {
		const unsigned d = digit_of(i);
		rank[i] += sDigStart[d] + sWarpHist[warp * kDigitBins + d];
		sKeys[rank[i]] = keys[i];
	}
	if constexpr(VM == kValueIndex) {
#pragma unroll
		for(int i = 0; i < IPT; ++i)
			sVals[rank[i]] = (unsigned)(tileStart + warpBase + i * 32 + lane);
	}
#pragma unroll
	for(int v = 0; v < (VM > 0 ? NPRE : 0); ++v) {
		unsigned vals[IPT];
		if(bulk) {
			if(!mbar_wait_bounded(&sBar[1 + v], 0))
				report_error(a.devError, a.hostError, kErrBarrierTimeout);
#pragma unroll
			for(int i = 0; i < IPT; ++i) vals[i] = sVals[v * TILE + warpBase + i * 32 + lane];
		} else {
#pragma unroll
			for(int i = 0; i < IPT; ++i) {
				int idx = warpBase + i * 32 + lane;
				vals[i] = idx < count ? a.buf.valsIn[v][tileStart + idx] : 0u;
			}
		}
		__syncthreads();
#pragma unroll
		for(int i = 0; i < IPT; ++i) sVals[v * TILE + rank[i]] = vals[i];
	}

	// Global offsets: the digit's start over the whole array plus the counts
	// of the tiles before this one.
	if(tid <= (int)mask) {
		unsigned excl = 0;
		if(tile == a.failTile) {
			// Injected fault (tests only): this tile never publishes, so the
			// tiles after it run their bounded waits out.
			if(tid == 0) report_error(a.devError, a.hostError, kErrInjected);
		} else if(tile > 0) {
			bool timedOut = false;
			excl = lookback_digit(a.status, tile, tid, a.epoch, &timedOut);
			if(timedOut) report_error(a.devError, a.hostError, kErrLookbackTimeout);
			st_relaxed_u64(a.status + (size_t)tile * kDigitBins + tid,
				epochBits | kFlagInclusive | (excl + mine));
		}
		sScatter[tid] = (int)(a.digitOffsets[tid] + excl - digStart);
	}
	__syncthreads();

	// Write each run to its global position: element p of the reordered tile
	// goes to scatter[digit] + p, consecutive p -> consecutive addresses.
#pragma unroll
	for(int j = 0; j < IPT; ++j) {
		const int p = j * NT + tid;
		if(p < count) {
			const unsigned k = sKeys[p];
			const int dst = sScatter[(k >> shift) & mask] + p;
			a.buf.keysOut[dst] = k;
			if constexpr(VM == kValueIndex) a.buf.valsOut[0][dst] = sVals[p];
#pragma unroll
			for(int v = 0; v < (VM > 0 ? NPRE : 0); ++v)
				a.buf.valsOut[v][dst] = sVals[v * TILE + p];
		}
	}

	// Remaining value arrays stream through the two staging buffers.
#pragma unroll
	for(int v = NPRE; v < NV; ++v) {
		const int stage = v & 1;
		unsigned* buf = sVals + stage * TILE;
		// Everyone is done with this staging buffer (its last reader was the
		// store of array v - 2): refill it.
		__syncthreads();
		if(bulk && tid == 0) {
			fence_proxy_async_smem();
			mbar_arrive_expect_tx(&sBar[1 + stage], TILE * 4);
			bulk_load(buf, a.buf.valsIn[v] + tileStart, TILE * 4, &sBar[1 + stage]);
		}
		unsigned vals[IPT];
		if(bulk) {
			if(!mbar_wait_bounded(&sBar[1 + stage], (v >> 1) & 1))
				report_error(a.devError, a.hostError, kErrBarrierTimeout);
#pragma unroll
			for(int i = 0; i < IPT; ++i) vals[i] = buf[warpBase + i * 32 + lane];
		} else {
#pragma unroll
			for(int i = 0; i < IPT; ++i) {
				int idx = warpBase + i * 32 + lane;
				vals[i] = idx < count ? a.buf.valsIn[v][tileStart + idx] : 0u;
			}
		}
		__syncthreads();
#pragma unroll
		for(int i = 0; i < IPT; ++i) buf[rank[i]] = vals[i];
		__syncthreads();
#pragma unroll
		for(int j = 0; j < IPT; ++j) {
			const int p = j * NT + tid;
			if(p < count) {
				const int dst = sScatter[(sKeys[p] >> shift) & mask] + p;
				a.buf.valsOut[v][dst] = buf[p];
			}
		}
	}
}

__global__ void iota_kernel(unsigned* out, int n) {
	for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
		i += (long long)gridDim.x * blockDim.x)
		out[i] = (unsigned)i;
}

////////////////////////////////////////////////////////////////////////////////
// Host launchers.

template<int VM>
static cudaError_t set_pass_attributes() {
	return cudaFuncSetAttribute(onesweep_kernel<VM>,
		cudaFuncAttributeMaxDynamicSharedMemorySize,
		(int)PassLayout<VM>::kBytes);
}

cudaError_t configure_kernels() {
	cudaError_t e = cudaSuccess;
	cudaError_t r;
	if((r = set_pass_attributes<-1>()) != cudaSuccess) e = r;
	if((r = set_pass_attributes<0>()) != cudaSuccess) e = r;
	if((r = set_pass_attributes<1>()) != cudaSuccess) e = r;
	if((r = set_pass_attributes<2>()) != cudaSuccess) e = r;
	if((r = set_pass_attributes<3>()) != cudaSuccess) e = r;
	if((r = set_pass_attributes<4>()) != cudaSuccess) e = r;
	if((r = set_pass_attributes<5>()) != cudaSuccess) e = r;
	if((r = set_pass_attributes<6>()) != cudaSuccess) e = r;
	return e;
}

int pass_tile_elements(int valueMode) {
	switch(valueMode) {
		case -1: return PassLayout<-1>::TILE;
		case 0: return PassLayout<0>::TILE;
		case 1: return PassLayout<1>::TILE;
		case 2: return PassLayout<2>::TILE;
		case 3: return PassLayout<3>::TILE;
		case 4: return PassLayout<4>::TILE;
		case 5: return PassLayout<5>::TILE;
		default: return PassLayout<6>::TILE;
	}
}

size_t pass_status_bytes(int n, int valueMode) {
	int tile = pass_tile_elements(valueMode);
	size_t tiles = n > 0 ? ((size_t)n + tile - 1) / tile : 0;
	return tiles * kDigitBins * sizeof(unsigned long long);
}

cudaError_t launch_upsweep(const unsigned* keys, int n, const PassPlan& plan,
	Control* ctrl, volatile unsigned* hostError, int numSMs,
	cudaStream_t stream) {
	UpsweepArgs a;
	a.keys = keys;
	a.n = n;
	a.vecOk = ((reinterpret_cast<size_t>(keys) & 15) == 0);
	a.plan = plan;
	a.ctrl = ctrl;
	a.hostError = hostError;
	long long chunks = ((long long)n + kUpChunk - 1) / kUpChunk;
	int grid = (int)std::min<long long>(chunks, (long long)numSMs * 3);
	if(grid < 1) grid = 1;
	upsweep_kernel<<<grid, kUpThreads, 0, stream>>>(a);
	return cudaGetLastError();
}

template<int VM>
static void launch_pass_vm(const PassArgs& a, cudaStream_t stream) {
	using L = PassLayout<VM>;
	onesweep_kernel<VM><<<a.numTiles, L::NT, L::kBytes, stream>>>(a);
}

cudaError_t launch_pass(const PassBuffers& buf, int valueMode, int n,
	int pass, const PassPlan& plan, Control* ctrl,
	unsigned long long* status, unsigned epoch, bool useBulk, int failTile,
	volatile unsigned* hostError, cudaStream_t stream) {
	PassArgs a;
	a.buf = buf;
	a.digitOffsets = ctrl->offsets + plan.binBase[pass];
	a.trivial = ctrl->trivial + pass;
	a.tileCounter = ctrl->tileCounter + pass;
	a.status = status;
	a.devError = &ctrl->error;
	a.hostError = hostError;
	a.n = n;
	const int tile = pass_tile_elements(valueMode);
	a.numTiles = (int)(((long long)n + tile - 1) / tile);
	a.shift = plan.shift[pass];
	a.width = plan.width[pass];
	a.epoch = epoch;
	a.useBulk = useBulk ? 1 : 0;
	a.failTile = failTile;
	switch(valueMode) {
		case -1: launch_pass_vm<-1>(a, stream); break;
		case 0: launch_pass_vm<0>(a, stream); break;
		case 1: launch_pass_vm<1>(a, stream); break;
		case 2: launch_pass_vm<2>(a, stream); break;
		case 3: launch_pass_vm<3>(a, stream); break;
		case 4: launch_pass_vm<4>(a, stream); break;
		case 5: launch_pass_vm<5>(a, stream); break;
		case 6: launch_pass_vm<6>(a, stream); break;
		default: return cudaErrorInvalidValue;
	}
	return cudaGetLastError();
}

cudaError_t launch_iota(unsigned* out, int n, cudaStream_t stream) {
	if(n <= 0) return cudaSuccess;
	int grid = (int)std::min<long long>(((long long)n + 255) / 256, 4096);
	iota_kernel<<<grid, 256, 0, stream>>>(out, n);
	return cudaGetLastError();
}

} // namespace mgpusort
