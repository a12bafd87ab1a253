// Radix sort kernels for sm_100a.
//
// A sort over the bit range [firstBit, endBit) runs one pass per digit,
// least significant first. Each pass is three launches over a partition of
// the array into R ranges of consecutive tiles (R = resident CTAs of the
// sort kernel):
//   1. count_kernel: each range's digit histogram (one read of the keys);
//   2. scan_kernel: per digit, the exclusive prefix over ranges and the
//      digit's total;
//   3. sort_kernel: CTA r starts every digit at (keys with smaller digits in
//      the whole array) + (keys with this digit in ranges before r) and
//      walks its tiles in order: bulk-copy the tile into shared memory, rank
//      its keys stably by digit, reorder it into digit runs, store each run
//      contiguously, advance the digit offsets. No tile waits for another.
// With earlyExit an upsweep launch first builds every pass's histogram in one
// read so that single-digit passes can be skipped.
//
// This replaces the reference's per-pass count / hist1 / hist2 / hist3 / sort
// kernel chain (sort/src/mgpusort/mgpusort.cpp:421-516; kernels
// sort/src/kernels/count.cu, hist1.cu, hist2.cu, hist3.cu, sort.cu). The
// ordering contract is the same: every pass is a stable partition by its
// digit, so the passes compose into a stable sort by the whole bit field.

#include "sort_kernels.h"
#include "sort_device.cuh"
#include "sort_common.cuh"
#include "tile_config.h"

#include <algorithm>

namespace mgpusort {

////////////////////////////////////////////////////////////////////////////////
// Upsweep: digit histograms of every pass in one read of the keys.

constexpr int kUpThreads = 1024;
constexpr int kUpKeysPerThread = 16;
constexpr int kUpChunk = kUpThreads * kUpKeysPerThread;

struct UpsweepArgs {
	const unsigned* keys;
	int n;
	int vecOk;
	PassPlan plan;
	Control* ctrl;
	volatile unsigned* hostError;
	// Onesweep sorts: the first executed pass's lookback buffer, cleared here
	// (statusWords words), and the tile counters, zeroed here.
	unsigned* status0;
	size_t statusWords;
};

// Shared memory of the upsweep: every bin of every pass has one counter per
// lane (word bin * 32 + lane), so the 32 atomics of a warp instruction fall
// in 32 different banks whatever the digits; warps share the columns.
__host__ __device__ constexpr size_t upsweep_smem_bytes(int totalBins) {
	return sizeof(unsigned) * 32 * (size_t)totalBins;
}

__global__ void __launch_bounds__(kUpThreads, 1) upsweep_kernel(const UpsweepArgs a) {
	extern __shared__ __align__(128) unsigned sHist[];
	__shared__ unsigned sScan[kUpThreads / 32];
	__shared__ unsigned sLast;

	const int tid = threadIdx.x;
	const int lane = tid & 31;
	const int warp = tid >> 5;
	const int totalBins = a.plan.totalBins;
	const int numPasses = a.plan.numPasses;

	for(int i = tid; i < totalBins * 32; i += kUpThreads) sHist[i] = 0;
	if(a.status0) {
		for(size_t i = (size_t)blockIdx.x * kUpThreads + tid; i < a.statusWords;
			i += (size_t)gridDim.x * kUpThreads)
			a.status0[i] = 0;
		if(blockIdx.x == 0 && tid < kMaxPasses) a.ctrl->tileCounter[tid] = 0;
	}
	__syncthreads();

	unsigned* myCol = sHist + lane;
	auto count_all = [&](const unsigned (&k)[kUpKeysPerThread], int nValid) {
#pragma unroll 1
		for(int p = 0; p < numPasses; ++p) {
			const int shift = a.plan.shift[p];
			const unsigned mask = (1u << a.plan.width[p]) - 1;
			unsigned* col = myCol + a.plan.binBase[p] * 32;
#pragma unroll
			for(int i = 0; i < kUpKeysPerThread; ++i)
				if(i < nValid) atomicAdd(&col[((k[i] >> shift) & mask) * 32], 1u);
		}
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

	// Column sums: warp w sums bins w, w + 32, ...; lane l reads column l.
	for(int b = warp; b < totalBins; b += kUpThreads / 32) {
		unsigned v = sHist[b * 32 + lane];
#pragma unroll
		for(int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
		if(lane == 0 && v) atomicAdd(&a.ctrl->hist[b], v);
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
		unsigned v = 0;
		if(tid < bins) v = ld_relaxed_u32(hist + tid);
		unsigned incl = warp_inclusive_scan(v, lane);
		if(lane == 31) sScan[warp] = incl;
		int nonEmpty = __syncthreads_count(v != 0);
		unsigned prefix = 0;
		for(int w = 0; w < warp; ++w) prefix += sScan[w];
		if(tid < bins) {
			a.ctrl->offsets[a.plan.binBase[p] + tid] = prefix + incl - v;
			hist[tid] = 0;
		}
		if(tid == 0) a.ctrl->trivial[p] = nonEmpty <= 1;
		__syncthreads();
	}
	if(tid == 0) a.ctrl->ticket = 0;
}

////////////////////////////////////////////////////////////////////////////////
// One pass = count + scan + sort over a range partition.
//
// The tiles of a pass are split into R ranges of consecutive tiles, one per
// CTA of the sort kernel. count_kernel builds each range's digit histogram
// (one read of the keys); scan_kernel turns them, per digit, into the
// exclusive prefix over ranges and the digit's total; sort_kernel CTA r
// starts each digit at (keys with smaller digits in the whole array) + (keys
// with this digit in ranges before r) and walks its tiles in order: stable
// rank of the tile, reorder into digit runs in shared memory, run-wise
// stores, then advance each digit's offset by the tile's count. No tile
// waits for another tile, and each CTA copies its next tile in while it sorts
// the current one. This is the reference's count -> histogram scan -> sort
// structure (sort/src/mgpusort/mgpusort.cpp:421-516) with per-range instead
// of per-block counts.

// Consecutive tiles [first_tile(r), first_tile(r + 1)) form range r.
struct RangeSplit {
	int numTiles;
	int numRanges;
	int tilesLo;    // tiles per range; the first `extra` ranges have one more
	int extra;
	__host__ __device__ __forceinline__ int first_tile(int r) const {
		return r * tilesLo + (r < extra ? r : extra);
	}
};

constexpr int kCountThreads = 512;

struct CountArgs {
	const unsigned* keys;
	int n;
	int tile;                       // elements per tile of the sort kernel
	int shift;
	int width;
	int vecOk;
	RangeSplit split;
	unsigned* rangeCounts;          // [256][R], digit-major
};

// Each lane owns one copy of the histogram, interleaved so that bin b of
// lane l is word b * 32 + l: every atomic of a warp falls in its own bank,
// and lanes never share a counter (warps do, through the atomic).
// The digit counts of range r (one CTA of NT threads; sHist holds
// kDigitBins * 32 words). NC: the keys are not written by the running grid.
template<bool NC, int NT = kCountThreads>
__device__ __forceinline__ void count_range(const CountArgs& a, int r, unsigned* sHist) {
	const int tid = threadIdx.x;
	const int lane = tid & 31;
	const unsigned mask = (1u << a.width) - 1;
	const int shift = a.shift;

	for(int i = tid; i < kDigitBins * 32; i += NT) sHist[i] = 0;
	__syncthreads();

	const long long begin = (long long)a.split.first_tile(r) * a.tile;
	const long long end = min((long long)a.n,
		(long long)a.split.first_tile(r + 1) * a.tile);
	unsigned* myCol = sHist + lane;
	auto add = [&](unsigned k) { atomicAdd(&myCol[((k >> shift) & mask) * 32], 1u); };
	long long done = begin;
	if(a.vecOk) {
		// begin is a multiple of the tile size (a multiple of 4): 16-byte
		// aligned.
		const uint4* src = reinterpret_cast<const uint4*>(a.keys + begin);
		const int nvec = (int)((end - begin) / 4);
		// Software pipelined: the next U loads are in flight while the
		// current U are counted.
		constexpr int U = 4;
		int i = tid;
		uint4 q[U];
		bool have = i + (U - 1) * NT < nvec;
		if(have) {
#pragma unroll
			for(int u = 0; u < U; ++u) q[u] = ld_in_u4<NC>(src + i + u * NT);
		}
		while(have) {
			uint4 cur[U];
#pragma unroll
			for(int u = 0; u < U; ++u) cur[u] = q[u];
			const int inext = i + U * NT;
			const bool haveNext = inext + (U - 1) * NT < nvec;
			if(haveNext) {
#pragma unroll
				for(int u = 0; u < U; ++u) q[u] = ld_in_u4<NC>(src + inext + u * NT);
			}
#pragma unroll
			for(int u = 0; u < U; ++u) {
				add(cur[u].x);
				add(cur[u].y);
				add(cur[u].z);
				add(cur[u].w);
			}
			i = inext;
			have = haveNext;
		}
		for(; i < nvec; i += NT) {
			const uint4 q = ld_in_u4<NC>(src + i);
			add(q.x);
			add(q.y);
			add(q.z);
			add(q.w);
		}
		done = begin + 4ll * nvec;
	}
	for(long long e = done + tid; e < end; e += NT) add(a.keys[e]);
	__syncthreads();

	// Sum the 32 copies of each bin: warp w sums bins w, w + 16, ...; lane l
	// reads copy l of the bin, a warp reduction adds them up.
	for(int b = tid >> 5; b < kDigitBins; b += NT / 32) {
		unsigned c = sHist[b * 32 + lane];
#pragma unroll
		for(int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
		if(lane == 0) a.rangeCounts[(size_t)b * a.split.numRanges + r] = c;
	}
}

__global__ void __launch_bounds__(kCountThreads) count_kernel(const CountArgs a) {
	__shared__ unsigned sHist[kDigitBins * 32];
	wait_for_predecessor();
	allow_successor();
	count_range<true>(a, blockIdx.x, sHist);
}

struct ScanArgs {
	const unsigned* rangeCounts;    // [256][R]
	unsigned* rangeOffsets;         // [256][R]: exclusive over ranges
	unsigned* totals;               // [256]
	int numRanges;
};

// One CTA per digit, one thread per range (R <= kMaxRanges = 1024): the
// exclusive scan of the digit's range counts and the digit's total.
// Digit d's column: one thread per range (numRanges <= blockDim.x).
__device__ __forceinline__ void scan_digit(const ScanArgs& a, int d, unsigned* sWarp) {
	const int t = threadIdx.x;
	const int lane = t & 31;
	const int warp = t >> 5;
	const int R = a.numRanges;
	const unsigned v = t < R ? a.rangeCounts[(size_t)d * R + t] : 0u;
	const unsigned incl = warp_inclusive_scan(v, lane);
	if(lane == 31) sWarp[warp] = incl;
	__syncthreads();
	if(warp == 0) {
		const int nw = blockDim.x >> 5;
		const unsigned w = lane < nw ? sWarp[lane] : 0u;
		const unsigned wi = warp_inclusive_scan(w, lane);
		sWarp[lane] = wi - w;
		if(lane == 31) a.totals[d] = wi;
	}
	__syncthreads();
	if(t < R) a.rangeOffsets[(size_t)d * R + t] = sWarp[warp] + incl - v;
}

__global__ void __launch_bounds__(1024) scan_kernel(const ScanArgs a) {
	__shared__ unsigned sWarp[32];
	wait_for_predecessor();
	allow_successor();
	scan_digit(a, blockIdx.x, sWarp);
}

struct SortArgs {
	PassBuffers buf;
	const unsigned* rangeOffsets;   // [256][R]
	const unsigned* totals;         // [256]
	unsigned* devError;
	volatile unsigned* hostError;
	RangeSplit split;
	int n;
	int shift;
	int width;
	int useBulk;
	int failTile;                   // tile whose CTA runs a wait out; -1: none
};

// mbarriers of a sort CTA: keys, up to six value arrays, the fault wait.
constexpr int kNumBars = 8;
constexpr int kFaultBar = 7;

// Tile shapes (tile_config.h, chosen by the autotuner and later sweeps).
// What the measurements showed: larger tiles give each digit longer runs
// per tile, so fewer partially written sectors reach DRAM; for indices and
// one value array two CTAs of 256 x 32 per SM are best (fewer, longer warps:
// less per-tile work per key than 384 x 20; 256 x 20 with three CTAs per SM
// was 29% slower at 64 Mi uniform keys: more ranges, more write fronts; one
// CTA per SM lost the overlap of one CTA's ranking with the other's
// stores). Several value
// arrays multiply the write fronts (ranges x digits x arrays), and a front
// is revisited only once per tile of its range, so partial sectors leave L2
// before they are completed: one CTA of 768 x 8 per SM halves the ranges.
//
// Value mode kKeysLarge is the keys-only pass of sortArray on at least
// MGPU_SORT_KEYS_LARGE_ELEMENTS keys: a tile shape of its own (the keys-only
// shape that is fastest at 1 Mi keys is not the fastest at 64 Mi).
constexpr int kKeysLarge = -2;
__host__ __device__ constexpr bool keys_only(int vm) { return vm == 0 || vm == kKeysLarge; }
// Value modes kSegOne (one value array) and kSegIndex (index mode) are those
// of the segmented sort's range passes, which keep a tile shape of their own
// (MGPU_SORT_SEG_SINGLE_*): their ranges are short, and the one-array
// sortArray shape measured slower there.
constexpr int kSegOne = -3;
constexpr int kSegIndex = -4;
__host__ __device__ constexpr bool seg_single(int vm) { return vm == kSegOne || vm == kSegIndex; }
__host__ __device__ constexpr bool is_index(int vm) { return vm == kValueIndex || vm == kSegIndex; }
__host__ __device__ constexpr int value_arrays(int vm) {
	return vm == kSegOne ? 1 : (vm > 0 ? vm : 0);
}

template<int VM> struct SortConfig {
	static constexpr bool kBig = VM == kKeysLarge;
	static constexpr bool kSeg = seg_single(VM);
	static constexpr int kThreads = VM >= 2 ? MGPU_SORT_MULTI_THREADS
		: kBig ? MGPU_SORT_KEYS_LARGE_THREADS : kSeg ? MGPU_SORT_SEG_SINGLE_THREADS
		: VM == 0 ? MGPU_SORT_KEYS_THREADS : MGPU_SORT_SINGLE_THREADS;
	static constexpr int kItems = VM >= 2 ? MGPU_SORT_MULTI_ITEMS
		: kBig ? MGPU_SORT_KEYS_LARGE_ITEMS : kSeg ? MGPU_SORT_SEG_SINGLE_ITEMS
		: VM == 0 ? MGPU_SORT_KEYS_ITEMS : MGPU_SORT_SINGLE_ITEMS;
	static constexpr int kMinBlocks = VM >= 2 ? MGPU_SORT_MULTI_MIN_BLOCKS
		: kBig ? MGPU_SORT_KEYS_LARGE_MIN_BLOCKS : kSeg ? MGPU_SORT_SEG_SINGLE_MIN_BLOCKS
		: VM == 0 ? MGPU_SORT_KEYS_MIN_BLOCKS : MGPU_SORT_SINGLE_MIN_BLOCKS;
	// Digit bits resolved by ballots in the warp ranking (match_digit8);
	// sortArray on at least kLargeElements keys uses kBallotBitsLarge.
	static constexpr int kBallotBits = VM >= 2 ? MGPU_SORT_MULTI_BALLOT_BITS
		: keys_only(VM) ? MGPU_SORT_KEYS_BALLOT_BITS : MGPU_SORT_SINGLE_BALLOT_BITS;
	static constexpr int kBallotBitsLarge = VM >= 2 ? MGPU_SORT_MULTI_BALLOT_BITS
		: keys_only(VM) ? MGPU_SORT_KEYS_BALLOT_BITS : MGPU_SORT_SINGLE_LARGE_BALLOT_BITS;
	static constexpr int kLargeElements = MGPU_SORT_SINGLE_LARGE_ELEMENTS;
	// Items of a thread whose peers are found before their counter updates.
	static constexpr int kRankBatch = VM >= 2 ? MGPU_SORT_MULTI_RANK_BATCH
		: keys_only(VM) ? MGPU_SORT_KEYS_RANK_BATCH
		: kSeg ? MGPU_SORT_SEG_SINGLE_RANK_BATCH : MGPU_SORT_SINGLE_RANK_BATCH;
	// Key tiles staged per CTA: with two, the next tile's keys are copied in
	// while this tile is sorted.
	static constexpr int kKeySlots = VM <= 1 ? 2 : 1;
};

template<int VM> struct SortLayout {
	static constexpr int NT = SortConfig<VM>::kThreads;
	static constexpr int IPT = SortConfig<VM>::kItems;
	static constexpr int TILE = NT * IPT;
	static constexpr int NW = NT / 32;
	static constexpr int KSLOTS = SortConfig<VM>::kKeySlots;
	static constexpr int NV = value_arrays(VM);
	// Vector stores (keys only, index mode, one value array): the reordered
	// tile leaves up to 3 unused words before each digit's run, so that a
	// run's shared-memory position and its global position agree mod 4.
	static constexpr bool VEC = MGPU_SORT_VECTOR_STORES != 0 && VM <= 1;
	static constexpr int PAD = VEC ? 3 * kDigitBins : 0;
	// Words per reordered buffer (a key slot, the value buffer).
	static constexpr int TILEP = TILE + PAD;
	// Keys only: no value buffer. One value array (or the generated
	// indices): one buffer, reordered in place. Two or more: a buffer of
	// source positions, then one staging buffer per value array.
	static constexpr int NVBUF = keys_only(VM) ? 0 : (NV >= 2 ? 1 + NV : 1);
	// Per digit: the scatter offset (one word), or with vector stores the
	// pair {global - shared offset, run start | run end << 16}.
	static constexpr int kTableWords = VEC ? 2 * kDigitBins : kDigitBins;
	// Word offsets into dynamic shared memory.
	static constexpr int kKeys = 0;
	static constexpr int kVals = kKeys + KSLOTS * TILEP;
	static constexpr int kWarpHist = kVals + NVBUF * TILEP;
	static constexpr int kRunning = kWarpHist + NW * kDigitBins;
	static constexpr int kScatter = kRunning + kDigitBins;
	static constexpr int kScan = kScatter + kTableWords;
	static constexpr int kBar = kScan + 32;          // 8-byte aligned: even
	static constexpr int kWords = kBar + 2 * kNumBars;
	static constexpr size_t kBytes = sizeof(unsigned) * kWords;
	static_assert(kBar % 2 == 0, "mbarriers need 8-byte alignment");
	static_assert(TILE % 4 == 0 && TILEP % 4 == 0, "16-byte aligned buffers");
	static_assert(NT >= kDigitBins && NT % 32 == 0,
		"the digit starts take one thread per digit");
	static_assert(TILEP < 65536, "ranks and run bounds are packed in 16 bits");
};

// Stable warp rank of one item with digit d and peers (match_digit8): the
// group of peers starts at the warp's running count of the digit, which the
// highest peer then advances by the group's size. Returns
// (digit << 16) | rank within the warp.
__device__ __forceinline__ unsigned count_item(unsigned d, unsigned peers,
	unsigned* warpHist, int lane, unsigned ltMask) {
	// Every peer reads the count; the highest peer then adds the group.
	const unsigned base = warpHist[d];
	__syncwarp();
	if((peers >> lane) == 1u) warpHist[d] = base + __popc(peers);
	__syncwarp();
	return (d << 16) | (base + __popc(peers & ltMask));
}

// Rank the staged tile's keys (warp-striped: item i of lane l in warp w is
// tile element w*32*IPT + i*32 + l, so (item, lane) order is input order per
// warp). In a partial tile the elements past `count` get digit 255: they
// rank after every real key and are never stored.
// Items are taken CH at a time: the peers of all CH are found first (the
// match steps of different items are independent), then the CH counter
// updates run in item order.
template<int IPT, bool FULL, bool BYTE, int BB, int CH>
__device__ __forceinline__ void rank_tile(const unsigned* sKeys, unsigned* myHist,
	int warpBase, int lane, int count, const DigitOf<BYTE>& digit, unsigned ltMask,
	const unsigned (&nClear)[4], unsigned (&rank)[IPT]) {
#pragma unroll
	for(int c = 0; c < IPT; c += CH) {
		unsigned d[CH], peers[CH];
#pragma unroll
		for(int j = 0; j < CH; ++j) {
			if(c + j < IPT) {
				const int idx = warpBase + (c + j) * 32 + lane;
				d[j] = digit(sKeys[idx]);
				if(!FULL && idx >= count) d[j] = kDigitBins - 1;
				peers[j] = match_digit8<BB>(d[j], nClear);
			}
		}
#pragma unroll
		for(int j = 0; j < CH; ++j) {
			if(c + j < IPT) rank[c + j] = count_item(d[j], peers[j], myHist, lane, ltMask);
		}
	}
}

// Shared-memory arrays of the sort kernels.
template<int VM> struct SortSmem {
	using L = SortLayout<VM>;
	unsigned* smem;
	unsigned* vals;
	unsigned* warpHist;
	unsigned* running;
	int* scatter;
	unsigned* scan;
	// mbarriers: one key slot: [0] keys, [1 + v] value array v; two key
	// slots: [0..1] keys, [2] value buffer. [kFaultBar] is the injected-fault
	// wait (never completed).
	uint64_t* bar;
	__device__ __forceinline__ explicit SortSmem(unsigned* base)
		: smem(base), vals(base + L::kVals),
		  warpHist(base + L::kWarpHist), running(base + L::kRunning),
		  scatter(reinterpret_cast<int*>(base + L::kScatter)), scan(base + L::kScan),
		  bar(reinterpret_cast<uint64_t*>(base + L::kBar)) { }
	__device__ __forceinline__ unsigned* keys(int slot) const {
		return smem + L::kKeys + slot * L::TILEP;
	}
	// Vector stores: per digit {global - shared offset, start | end << 16}.
	__device__ __forceinline__ int2* runs() const {
		return reinterpret_cast<int2*>(scatter);
	}
	// Several value arrays: the source positions and staging buffer v.
	__device__ __forceinline__ unsigned* positions() const { return vals; }
	__device__ __forceinline__ unsigned* staged(int v) const {
		return vals + (1 + v) * L::TILE;
	}
};

// Once per CTA: mbarriers and zeroed warp histograms.
template<int VM>
__device__ __forceinline__ void sort_setup(const SortSmem<VM>& sm) {
	using L = SortLayout<VM>;
	if(threadIdx.x == 0) {
		for(int i = 0; i < kNumBars; ++i) mbar_init(&sm.bar[i], 1);
		fence_mbar_init();
	}
	for(int i = threadIdx.x; i < L::NW * kDigitBins; i += L::NT) sm.warpHist[i] = 0;
}

// Identity pass over [begin, end) (every key has the same digit): a
// streaming copy of the keys and value arrays (index mode: the positions).
// With 16-byte aligned buffers the aligned middle moves in 16-byte vectors,
// every array's load of a step in flight before its stores.
template<int VM, bool NC = true>
__device__ __forceinline__ void copy_range(const SortArgs& a, long long begin,
	long long end, long long indexBase) {
	constexpr int NV = SortLayout<VM>::NV;
	constexpr int NT = SortLayout<VM>::NT;
	auto copy_one = [&](long long i) {
		a.buf.keysOut[i] = a.buf.keysIn[i];
		if constexpr(is_index(VM)) a.buf.valsOut[0][i] = (unsigned)(i - indexBase);
#pragma unroll
		for(int v = 0; v < NV; ++v) a.buf.valsOut[v][i] = a.buf.valsIn[v][i];
	};
	long long head = end;
	long long vecEnd = end;
	if(a.useBulk) {
		head = min(end, (begin + 3) & ~3ll);
		vecEnd = head + ((end - head) & ~3ll);
	}
	for(long long i = begin + threadIdx.x; i < head; i += NT) copy_one(i);
	if(head < vecEnd) {
		const long long v0 = head >> 2;
		const long long nvec = (vecEnd - head) >> 2;
		for(long long j = threadIdx.x; j < nvec; j += NT) {
			const long long e = (v0 + j) << 2;
			uint4 k = ld_in_u4<NC>(reinterpret_cast<const uint4*>(a.buf.keysIn) + v0 + j);
			uint4 vals[NV > 0 ? NV : 1];
#pragma unroll
			for(int v = 0; v < NV; ++v)
				vals[v] = ld_in_u4<NC>(reinterpret_cast<const uint4*>(a.buf.valsIn[v]) + v0 + j);
			reinterpret_cast<uint4*>(a.buf.keysOut)[v0 + j] = k;
			if constexpr(is_index(VM)) {
				const unsigned x = (unsigned)(e - indexBase);
				reinterpret_cast<uint4*>(a.buf.valsOut[0])[v0 + j] =
					make_uint4(x, x + 1, x + 2, x + 3);
			}
#pragma unroll
			for(int v = 0; v < NV; ++v)
				reinterpret_cast<uint4*>(a.buf.valsOut[v])[v0 + j] = vals[v];
		}
	}
	for(long long i = vecEnd + threadIdx.x; i < end; i += NT) copy_one(i);
}

// Once the warps of a tile have counted their digits (sm.warpHist): per
// digit the start of its run in the reordered tile, and for every warp the
// position where its part of the run begins (run start + counts of the
// warps before it), written over the warp counts. Each digit's running
// offset advances by the tile's real count (padding is only ever in digit
// 255 and is not counted).
//
// Without gaps the runs are packed (run start = exclusive prefix of the
// digit counts) and element p of the reordered tile belongs at
// scatter[digit] + p globally. With gaps (vector stores) run d starts at the
// first position at or after the end of run d - 1 that is congruent mod 4
// to its global start running[d]; as run d - 1 itself started congruent to
// running[d - 1], the gap before run d is
//   (running[d] - running[d - 1] - count[d - 1]) mod 4,
// known from digit d - 1 alone, so the starts are one prefix sum of
// count + gap. The runs table then holds per digit the global - shared
// offset and the run's [start, end) over its real elements. One barrier
// inside; the caller synchronizes before reading the results.
template<int VM>
__device__ __forceinline__ void tile_digit_starts(const SortSmem<VM>& sm, int count,
	bool gaps) {
	using L = SortLayout<VM>;
	constexpr int NW = L::NW;
	const int tid = threadIdx.x;
	const int lane = tid & 31;
	const int warp = tid >> 5;
	unsigned c[NW];
	unsigned tileTotal = 0;
	unsigned g = 0;
	if(tid < kDigitBins) {
#pragma unroll
		for(int w = 0; w < NW; ++w) {
			c[w] = sm.warpHist[w * kDigitBins + tid];
			tileTotal += c[w];
		}
		g = sm.running[tid];
	}
	unsigned gap = 0;
	if constexpr(L::VEC) {
		// End of run d - 1 mod 4: from the neighbouring lane, or for the
		// first lane of a warp from shared memory.
		unsigned prevEnd = __shfl_up_sync(0xffffffffu, g + tileTotal, 1);
		if(lane == 0 && tid > 0 && tid < kDigitBins) {
			unsigned t = 0;
#pragma unroll
			for(int w = 0; w < NW; ++w) t += sm.warpHist[w * kDigitBins + tid - 1];
			prevEnd = sm.running[tid - 1] + t;
		}
		if(tid == 0) prevEnd = 0;
		if(gaps && tid < kDigitBins) gap = (g - prevEnd) & 3u;
	}
	const unsigned incl = warp_inclusive_scan(tileTotal + gap, lane);
	if(lane == 31 && tid < kDigitBins) sm.scan[warp] = incl;
	__syncthreads();
	if(tid < kDigitBins) {
		unsigned prefix = 0;
		for(int w = 0; w < warp; ++w) prefix += sm.scan[w];
		const unsigned digStart = prefix + incl - tileTotal;
		unsigned run = digStart;
#pragma unroll
		for(int w = 0; w < NW; ++w) {
			sm.warpHist[w * kDigitBins + tid] = run;
			run += c[w];
		}
		const unsigned mine = tileTotal - (tid == kDigitBins - 1 ? L::TILE - count : 0);
		if constexpr(L::VEC)
			sm.runs()[tid] = make_int2((int)(g - digStart),
				(int)(digStart | ((digStart + mine) << 16)));
		else
			sm.scatter[tid] = (int)(g - digStart);
		sm.running[tid] = g + mine;
	}
}

// Stores a reordered tile laid out with gaps (tile_digit_starts): thread t
// takes the aligned 4-element chunks t, t + NT, ... of shared memory. A chunk
// inside one digit run (its first key's run covers all four positions) goes
// out as one 16-byte store per array, at a 16-byte aligned global address
// since shared and global positions of a run agree mod 4; a chunk at a run
// boundary stores each element that lies inside its own digit's run. Gap
// words hold stale data and lie in no run, so they are never stored. Without
// 16-byte aligned buffers the tile has no gaps and every element is stored
// on its own.
template<int VM, bool BYTE>
__device__ __forceinline__ void store_runs(const SortArgs& a, const SortSmem<VM>& sm,
	const unsigned* sKeys, int count, const DigitOf<BYTE>& digit) {
	using L = SortLayout<VM>;
	constexpr int NT = L::NT;
	const int2* runs = sm.runs();
	const unsigned* sVals = sm.vals;
	const int tid = threadIdx.x;
	auto store_one = [&](int q, unsigned k, unsigned v) {
		const int2 r = runs[digit(k)];
		if(q >= (r.y & 0xffff) && q < (int)((unsigned)r.y >> 16)) {
			a.buf.keysOut[q + r.x] = k;
			if constexpr(!keys_only(VM)) a.buf.valsOut[0][q + r.x] = v;
		}
	};
	if(a.useBulk) {
		// The last run ends after every other.
		const int len = (int)((unsigned)runs[kDigitBins - 1].y >> 16);
		for(int q = tid * 4; q < len; q += NT * 4) {
			const uint4 k = *reinterpret_cast<const uint4*>(sKeys + q);
			uint4 v = make_uint4(0u, 0u, 0u, 0u);
			if constexpr(!keys_only(VM)) v = *reinterpret_cast<const uint4*>(sVals + q);
			const int2 r = runs[digit(k.x)];
			if(q >= (r.y & 0xffff) && q + 4 <= (int)((unsigned)r.y >> 16)) {
				*reinterpret_cast<uint4*>(a.buf.keysOut + q + r.x) = k;
				if constexpr(!keys_only(VM))
					*reinterpret_cast<uint4*>(a.buf.valsOut[0] + q + r.x) = v;
			} else {
				store_one(q, k.x, v.x);
				store_one(q + 1, k.y, v.y);
				store_one(q + 2, k.z, v.z);
				store_one(q + 3, k.w, v.w);
			}
		}
	} else {
		for(int p = tid; p < count; p += NT) {
			const unsigned k = sKeys[p];
			const int dst = runs[digit(k)].x + p;
			a.buf.keysOut[dst] = k;
			if constexpr(!keys_only(VM)) a.buf.valsOut[0][dst] = sVals[p];
		}
	}
}

// Sort the tiles of [begin, end) in order, from digit offsets already in
// sm.running (element p of digit d's run in a tile goes to running[d] + p,
// then running[d] advances by the tile's count). Keys only, index mode or
// one value array. Each tile: stable warp ranks, digit starts, reorder into
// digit runs in shared memory, run-wise stores. The next tile's keys are
// copied in while a tile is sorted (two key slots), its value array as soon
// as this tile has stored its own. Index mode writes position - indexBase.
// Requires sort_setup and a barrier before.
template<int VM, bool BYTE, int BB>
__device__ void sort_range_single(const SortArgs& a, const SortSmem<VM>& sm,
	long long begin, long long end, long long indexBase, unsigned& phase) {
	static_assert(VM <= 1, "one value array at most");

	using L = SortLayout<VM>;
	constexpr int NT = L::NT;
	constexpr int IPT = L::IPT;
	constexpr int CH = SortConfig<VM>::kRankBatch;
	constexpr int TILE = L::TILE;
	constexpr int NW = L::NW;
	constexpr int NV = L::NV;
	constexpr int KSLOTS = L::KSLOTS;
	constexpr unsigned kTileBytes = TILE * 4;

	unsigned* sVals = sm.vals;
	unsigned* sWarpHist = sm.warpHist;
	int* sScatter = sm.scatter;
	uint64_t* sBar = sm.bar;

	const int tid = threadIdx.x;
	const int lane = tid & 31;
	const int warp = tid >> 5;
	const int warpBase = warp * 32 * IPT;

	// Full tiles at 16-byte aligned offsets are staged with bulk copies.
	auto tile_is_bulk = [&](long long t) {
		return a.useBulk && (t & 3) == 0 && t + TILE <= end;
	};

	if(tid == 0 && begin < end && tile_is_bulk(begin)) {
		fence_proxy_async_smem();
		stage_tile(sm.keys(0), a.buf.keysIn + begin, kTileBytes, &sBar[0]);
		if constexpr(NV >= 1) stage_tile(sVals, a.buf.valsIn[0] + begin, kTileBytes, &sBar[2]);
	}

	const DigitOf<BYTE> digit(a.shift, a.width);
	const unsigned ltMask = lanemask_lt();
	unsigned nClear[4];
#pragma unroll
	for(int k = 0; k < 4; ++k) nClear[k] = ((lane >> k) & 1) ? 0u : 0xffffffffu;
	int slot = 0;

	// Tiles lie on a grid of 4-element (16-byte) aligned starts: when begin
	// is not aligned, the first tile is shorter and every later one can be
	// staged with bulk copies.
	for(long long tileStart = begin; tileStart < end;) {
		unsigned* sKeys = sm.keys(slot);
		const long long next = (tileStart & ~3ll) + TILE;
		const int count = (int)(min(next, end) - tileStart);
		const bool bulk = tile_is_bulk(tileStart);

		// The next tile's keys go into the other slot (free since the end of
		// the previous iteration) while this one is sorted.
		if(KSLOTS == 2 && tid == 0 && next < end && tile_is_bulk(next)) {
			fence_proxy_async_smem();
			stage_tile(sm.keys(slot ^ 1), a.buf.keysIn + next, kTileBytes, &sBar[slot ^ 1]);
		}

		unsigned* myHist = sWarpHist + warp * kDigitBins;
		unsigned rank[IPT];
		if(bulk) {
			if(!mbar_wait_bounded(&sBar[slot], (phase >> slot) & 1u))
				report_error(a.devError, a.hostError, kErrBarrierTimeout);
			phase ^= 1u << slot;
			rank_tile<IPT, true, BYTE, BB, CH>(sKeys, myHist, warpBase, lane, count, digit,
				ltMask, nClear, rank);
		} else {
			// Plain loads (a partial tile, or data that is not 16-byte
			// aligned): stage the keys and the first value array by hand.
			for(int i = tid; i < TILE; i += NT) {
				sKeys[i] = i < count ? a.buf.keysIn[tileStart + i] : 0xffffffffu;
				if constexpr(NV >= 1)
					sVals[i] = i < count ? a.buf.valsIn[0][tileStart + i] : 0u;
			}
			__syncthreads();
			rank_tile<IPT, false, BYTE, BB, CH>(sKeys, myHist, warpBase, lane, count, digit,
				ltMask, nClear, rank);
		}
		__syncthreads();

		tile_digit_starts<VM>(sm, count, a.useBulk);

		// Every warp's keys leave shared memory for registers before the tile
		// is reordered in place.
		unsigned keys[IPT];
#pragma unroll
		for(int i = 0; i < IPT; ++i) keys[i] = sKeys[warpBase + i * 32 + lane];
		__syncthreads();

		// Reorder the tile into digit runs in shared memory: keys in place,
		// then the first value array (or the generated indices).
#pragma unroll
		for(int i = 0; i < IPT; ++i) {
			rank[i] = (rank[i] & 0xffffu) + sWarpHist[warp * kDigitBins + (rank[i] >> 16)];
			sKeys[rank[i]] = keys[i];
		}
		if constexpr(is_index(VM)) {
#pragma unroll
			for(int i = 0; i < IPT; ++i)
				sVals[rank[i]] = (unsigned)(tileStart - indexBase + warpBase + i * 32 + lane);
		}
		if constexpr(NV >= 1) {
			unsigned vals[IPT];
			if(bulk) {
				if(!mbar_wait_bounded(&sBar[2], (phase >> 2) & 1u))
					report_error(a.devError, a.hostError, kErrBarrierTimeout);
				phase ^= 1u << 2;
			}
#pragma unroll
			for(int i = 0; i < IPT; ++i) vals[i] = sVals[warpBase + i * 32 + lane];
			__syncthreads();
#pragma unroll
			for(int i = 0; i < IPT; ++i) sVals[rank[i]] = vals[i];
		}
		if(a.failTile >= 0 && tileStart / TILE == a.failTile && tid == 0) {
			// Injected fault (tests only): wait on a barrier that nothing
			// completes, so the bounded wait runs out and is reported.
			if(!mbar_wait_bounded(&sBar[kFaultBar], 0))
				report_error(a.devError, a.hostError, kErrInjected);
		}
		__syncthreads();

		// Write each run to its global position: consecutive positions of
		// the reordered tile, consecutive addresses.
		if constexpr(L::VEC) {
			store_runs<VM, BYTE>(a, sm, sKeys, count, digit);
		} else if(count == TILE) {
#pragma unroll
			for(int j = 0; j < IPT; ++j) {
				const int p = j * NT + tid;
				const unsigned k = sKeys[p];
				const int dst = sScatter[digit(k)] + p;
				a.buf.keysOut[dst] = k;
				if constexpr(!keys_only(VM)) a.buf.valsOut[0][dst] = sVals[p];
			}
		} else {
#pragma unroll
			for(int j = 0; j < IPT; ++j) {
				const int p = j * NT + tid;
				if(p < count) {
					const unsigned k = sKeys[p];
					const int dst = sScatter[digit(k)] + p;
					a.buf.keysOut[dst] = k;
					if constexpr(!keys_only(VM)) a.buf.valsOut[0][dst] = sVals[p];
				}
			}
		}

		for(int i = tid; i < NW * kDigitBins; i += NT) sWarpHist[i] = 0;
		__syncthreads();

		// This tile's buffers are free: request the next tile's first value
		// array, and with one key slot its keys.
		if(tid == 0 && next < end && tile_is_bulk(next)) {
			fence_proxy_async_smem();
			if(KSLOTS == 1) stage_tile(sKeys, a.buf.keysIn + next, kTileBytes, &sBar[0]);
			if constexpr(NV >= 1)
				stage_tile(sVals, a.buf.valsIn[0] + next, kTileBytes, &sBar[2]);
		}
		slot = KSLOTS == 2 ? slot ^ 1 : 0;
		tileStart = next;
	}
}

// The same range sort with two or more value arrays. Keys are ranked and
// reordered as above; the reorder also records, for every position of the
// reordered tile, the element's position in the input tile. Each thread then
// holds, for its IPT output positions, the global destination and the source
// position in registers, and every value array is written straight from its
// staging buffer: valsOut[v][dst] = staged_v[src]. Each array has its own
// staging buffer, so all of a tile's arrays are in flight at once: they are
// requested as soon as the previous tile has written its own (the first
// tile's with its keys) and arrive while the keys are ranked. The next
// tile's keys are requested as soon as this tile's keys are stored. Tiles
// without bulk copies gather their values from global memory (a window of
// one tile).
template<int VM, bool BYTE, int BB>
__device__ void sort_range_multi(const SortArgs& a, const SortSmem<VM>& sm,
	long long begin, long long end, unsigned& phase) {

	using L = SortLayout<VM>;
	constexpr int NT = L::NT;
	constexpr int IPT = L::IPT;
	constexpr int CH = SortConfig<VM>::kRankBatch;
	constexpr int TILE = L::TILE;
	constexpr int NV = L::NV;
	constexpr unsigned kTileBytes = TILE * 4;
	static_assert(NV >= 2 && NV < kFaultBar && L::KSLOTS == 1, "multi-array layout");

	unsigned* sKeys = sm.keys(0);
	unsigned* sPos = sm.positions();
	unsigned* sWarpHist = sm.warpHist;
	int* sScatter = sm.scatter;
	uint64_t* sBar = sm.bar;

	const int tid = threadIdx.x;
	const int lane = tid & 31;
	const int warp = tid >> 5;
	const int warpBase = warp * 32 * IPT;

	auto tile_is_bulk = [&](long long t) {
		return a.useBulk && (t & 3) == 0 && t + TILE <= end;
	};
	auto wait_bar = [&](int b) {
		if(!mbar_wait_bounded(&sBar[b], (phase >> b) & 1u))
			report_error(a.devError, a.hostError, kErrBarrierTimeout);
		phase ^= 1u << b;
	};
	// Value array v of the tile at t into staging buffer v (mbarrier 1 + v).
	auto stage_values = [&](long long t) {
#pragma unroll
		for(int v = 0; v < NV; ++v)
			stage_tile(sm.staged(v), a.buf.valsIn[v] + t, kTileBytes, &sBar[1 + v]);
	};

	if(tid == 0 && begin < end && tile_is_bulk(begin)) {
		fence_proxy_async_smem();
		stage_tile(sKeys, a.buf.keysIn + begin, kTileBytes, &sBar[0]);
		stage_values(begin);
	}

	const DigitOf<BYTE> digit(a.shift, a.width);
	const unsigned ltMask = lanemask_lt();
	unsigned nClear[4];
#pragma unroll
	for(int k = 0; k < 4; ++k) nClear[k] = ((lane >> k) & 1) ? 0u : 0xffffffffu;

	for(long long tileStart = begin; tileStart < end;) {
		const long long next = (tileStart & ~3ll) + TILE;
		const int count = (int)(min(next, end) - tileStart);
		const bool bulk = tile_is_bulk(tileStart);
		const bool nextBulk = next < end && tile_is_bulk(next);

		unsigned* myHist = sWarpHist + warp * kDigitBins;
		unsigned rank[IPT];
		if(bulk) {
			wait_bar(0);
			rank_tile<IPT, true, BYTE, BB, CH>(sKeys, myHist, warpBase, lane, count, digit,
				ltMask, nClear, rank);
		} else {
			for(int i = tid; i < TILE; i += NT)
				sKeys[i] = i < count ? a.buf.keysIn[tileStart + i] : 0xffffffffu;
			__syncthreads();
			rank_tile<IPT, false, BYTE, BB, CH>(sKeys, myHist, warpBase, lane, count, digit,
				ltMask, nClear, rank);
		}
		__syncthreads();
		tile_digit_starts<VM>(sm, count, false);

		unsigned keys[IPT];
#pragma unroll
		for(int i = 0; i < IPT; ++i) keys[i] = sKeys[warpBase + i * 32 + lane];
		__syncthreads();

		// Reorder the keys in place; record each element's input position.
#pragma unroll
		for(int i = 0; i < IPT; ++i) {
			const unsigned pos = (rank[i] & 0xffffu)
				+ sWarpHist[warp * kDigitBins + (rank[i] >> 16)];
			sKeys[pos] = keys[i];
			sPos[pos] = (unsigned)(warpBase + i * 32 + lane);
		}
		if(a.failTile >= 0 && tileStart / TILE == a.failTile && tid == 0) {
			// Injected fault (tests only): wait on a barrier that nothing
			// completes, so the bounded wait runs out and is reported.
			if(!mbar_wait_bounded(&sBar[kFaultBar], 0))
				report_error(a.devError, a.hostError, kErrInjected);
		}
		__syncthreads();

		// Destinations and sources of this thread's output positions; the
		// keys are stored run-wise.
		int dst[IPT];
		unsigned src[IPT];
#pragma unroll
		for(int j = 0; j < IPT; ++j) {
			const int p = j * NT + tid;
			dst[j] = -1;
			src[j] = 0;
			if(p < count) {
				const unsigned k = sKeys[p];
				dst[j] = sScatter[digit(k)] + p;
				src[j] = sPos[p];
				a.buf.keysOut[dst[j]] = k;
			}
		}
		for(int i = tid; i < L::NW * kDigitBins; i += NT) sWarpHist[i] = 0;
		__syncthreads();

		// The key buffer is free: the next tile's keys head there.
		if(tid == 0 && nextBulk) {
			fence_proxy_async_smem();
			stage_tile(sKeys, a.buf.keysIn + next, kTileBytes, &sBar[0]);
		}

#pragma unroll
		for(int v = 0; v < NV; ++v) {
			if(bulk) {
				wait_bar(1 + v);
				const unsigned* buf = sm.staged(v);
#pragma unroll
				for(int j = 0; j < IPT; ++j)
					if(dst[j] >= 0) a.buf.valsOut[v][dst[j]] = buf[src[j]];
			} else {
				const unsigned* in = a.buf.valsIn[v] + tileStart;
#pragma unroll
				for(int j = 0; j < IPT; ++j)
					if(dst[j] >= 0) a.buf.valsOut[v][dst[j]] = in[src[j]];
			}
		}
		__syncthreads();

		// Every staging buffer is free: the next tile's value arrays.
		if(tid == 0 && nextBulk) {
			fence_proxy_async_smem();
			stage_values(next);
		}
		tileStart = next;
	}
}

template<int VM, bool BYTE, int BB>
__device__ __forceinline__ void sort_range(const SortArgs& a, const SortSmem<VM>& sm,
	long long begin, long long end, long long indexBase, unsigned& phase) {
	if constexpr(VM >= 2) sort_range_multi<VM, BYTE, BB>(a, sm, begin, end, phase);
	else sort_range_single<VM, BYTE, BB>(a, sm, begin, end, indexBase, phase);
}

// Range r of one pass (the CTA of sort_kernel, or of the cooperative sort):
// where each digit's keys start in the output, then a copy if the pass has
// a single digit, else the tiles of the range. NC: the input was not written
// by the running grid.
template<int VM, bool BYTE, int BB, bool NC>
__device__ __forceinline__ void sort_one_range(const SortArgs& a, unsigned* smem, int r) {
	using L = SortLayout<VM>;
	const SortSmem<VM> sm(smem);
	const int tid = threadIdx.x;
	const int lane = tid & 31;
	const int warp = tid >> 5;
	const int R = a.split.numRanges;
	const long long begin = (long long)a.split.first_tile(r) * L::TILE;
	const long long end = min((long long)a.n, (long long)a.split.first_tile(r + 1) * L::TILE);

	// Each digit starts at the keys with smaller digits in the whole array
	// plus the keys with this digit in the ranges before this one.
	const unsigned total = tid < kDigitBins ? a.totals[tid] : 0u;
	const unsigned inclTotal = warp_inclusive_scan(total, lane);
	if(lane == 31 && tid < kDigitBins) sm.scan[warp] = inclTotal;
	const int nonEmpty = __syncthreads_count(tid < kDigitBins && total != 0);
	if(tid < kDigitBins) {
		unsigned prefix = 0;
		for(int w = 0; w < warp; ++w) prefix += sm.scan[w];
		sm.running[tid] = prefix + inclTotal - total + a.rangeOffsets[(size_t)tid * R + r];
	}
	if(nonEmpty <= 1) {
		copy_range<VM, NC>(a, begin, end, 0);
		return;
	}
	sort_setup<VM>(sm);
	__syncthreads();
	unsigned phase = 0;
	sort_range<VM, BYTE, BB>(a, sm, begin, end, 0, phase);
}

// One pass over a whole array: CTA r sorts range r of the split.
template<int VM, bool BYTE, int BB>
__global__ void __launch_bounds__(SortLayout<VM>::NT, SortConfig<VM>::kMinBlocks)
sort_kernel(const SortArgs a) {
	using L = SortLayout<VM>;
	extern __shared__ __align__(128) unsigned smem[];
	// The successor (the next pass's count) is released when this grid
	// exits, not here: released early, its CTAs cost more than the launch
	// latency they hide.
	wait_for_predecessor();
	sort_one_range<VM, BYTE, BB, true>(a, smem, blockIdx.x);
}

////////////////////////////////////////////////////////////////////////////////
// Segmented sort: many independent segments of one array, one pass plan.
//
// seg_plan_kernel classifies the segments (device offsets) once per sort:
// segments of at most kSegSmallMax elements go to a kernel that sorts each
// one in shared memory through every pass (tiny ones with a small tile);
// larger ones are cut into ranges of consecutive tiles. Each pass then runs
// seg_count (range digit counts), seg_scan (per segment: digit starts and
// range offsets, plus whether the segment has a single digit) and seg_sort
// (the range sort loop of the one-array path). All of them are persistent
// over device-side work lists, so the launch shapes do not depend on the
// segment sizes.

// Segmented-plan counters (ints): [0] tiny segments, [1] small, [2] large,
// [3] ranges; from kSegWork, work counters the persistent kernels draw their
// next item from: per pass p, [kSegWork + 2p] (count) and [kSegWork + 2p + 1]
// (sort); then the tiny and small lists' (kSegWorkSmall, + 1). The plan
// kernel zeroes them at the start of every sort.
constexpr int kSegWork = 8;
constexpr int kSegWorkSmall = kSegWork + 2 * kMaxPasses;
constexpr int kSegCounters = kSegWorkSmall + 2;

constexpr int kSegTinyMax = 512;
constexpr int kSegSmallMax = 4096;
constexpr int kSegMaxRangesPerSegment = 64;
constexpr int kSegTilesPerRange = MGPU_SORT_SEG_TILES_PER_RANGE;
constexpr int kPlanThreads = 1024;

// counters: [0] tiny segments, [1] small, [2] large, [3] ranges, [4] error.
struct SegPlanArgs {
	const int* offsets;
	int numSegments;
	int n;
	int tile;
	int* tinyList;
	int* smallList;
	int* largeList;
	int* largeRangeFirst;
	int* largeRangeCount;
	int* rangeBegin;
	int* rangeEnd;
	int* rangeSeg;
	int* counters;
	unsigned* devError;
	volatile unsigned* hostError;
};

__device__ __forceinline__ void seg_classify(const SegPlanArgs& a, int s, int& tiny,
	int& small, int& large, int& ranges) {
	const int len = a.offsets[s + 1] - a.offsets[s];
	tiny = small = large = ranges = 0;
	// A one-element segment still moves to the result buffers (and gets its
	// index in index mode).
	if(len <= 0) return;
	if(len <= kSegTinyMax) tiny = 1;
	else if(len <= kSegSmallMax) small = 1;
	else {
		large = 1;
		const int base = a.offsets[s] & ~3;
		const int tiles = (a.offsets[s + 1] - base + a.tile - 1) / a.tile;
		ranges = min(kSegMaxRangesPerSegment,
			(tiles + kSegTilesPerRange - 1) / kSegTilesPerRange);
	}
}

// Exclusive scan over the 1024 threads of the plan kernel.
__device__ __forceinline__ int block_exclusive_scan(int x, int* sScan, int& total) {
	const int lane = threadIdx.x & 31;
	const int warp = threadIdx.x >> 5;
	int incl = (int)warp_inclusive_scan((unsigned)x, lane);
	__syncthreads();
	if(lane == 31) sScan[warp] = incl;
	__syncthreads();
	if(warp == 0) {
		int w = sScan[lane];
		int wi = (int)warp_inclusive_scan((unsigned)w, lane);
		sScan[lane] = wi - w;
		if(lane == 31) sScan[32] = wi;
	}
	__syncthreads();
	total = sScan[32];
	return sScan[warp] + incl - x;
}

__global__ void __launch_bounds__(kPlanThreads) seg_plan_kernel(const SegPlanArgs a) {
	__shared__ int sScan[33];
	const int tid = threadIdx.x;
	const int S = a.numSegments;
	const int chunk = (S + kPlanThreads - 1) / kPlanThreads;
	const int s0 = min(S, tid * chunk);
	const int s1 = min(S, s0 + chunk);

	// Offsets must start at 0, never decrease and end at n.
	bool bad = false;
	for(int s = s0; s < s1; ++s) bad |= a.offsets[s + 1] < a.offsets[s];
	if(tid == 0) bad |= a.offsets[0] != 0 || a.offsets[S] != a.n;
	if(__syncthreads_or(bad)) {
		if(tid == 0) {
			for(int i = 0; i < 5; ++i) a.counters[i] = 0;
			report_error(a.devError, a.hostError, kErrBadSegments);
		}
		return;
	}
	for(int i = kSegWork + tid; i < kSegCounters; i += kPlanThreads) a.counters[i] = 0;

	int nt = 0, ns = 0, nl = 0, nr = 0;
	for(int s = s0; s < s1; ++s) {
		int t, sm, l, r;
		seg_classify(a, s, t, sm, l, r);
		nt += t;
		ns += sm;
		nl += l;
		nr += r;
	}
	int totT, totS, totL, totR;
	int bt = block_exclusive_scan(nt, sScan, totT);
	int bs = block_exclusive_scan(ns, sScan, totS);
	int bl = block_exclusive_scan(nl, sScan, totL);
	int br = block_exclusive_scan(nr, sScan, totR);
	for(int s = s0; s < s1; ++s) {
		int t, sm, l, r;
		seg_classify(a, s, t, sm, l, r);
		if(t) a.tinyList[bt++] = s;
		if(sm) a.smallList[bs++] = s;
		if(l) {
			a.largeList[bl] = s;
			a.largeRangeFirst[bl] = br;
			a.largeRangeCount[bl] = r;
			++bl;
			// Split the segment's tiles evenly over its r ranges. Tiles lie on
			// the 4-element aligned grid from the segment's aligned-down start
			// (the same grid the sort kernel walks), so the first tile may be
			// shorter.
			const int begin = a.offsets[s];
			const int end = a.offsets[s + 1];
			const long long base = begin & ~3;
			const int tiles = (int)((end - base + a.tile - 1) / a.tile);
			const int lo = tiles / r;
			const int extra = tiles % r;
			for(int k = 0; k < r; ++k) {
				const int t0 = k * lo + min(k, extra);
				const int t1 = (k + 1) * lo + min(k + 1, extra);
				a.rangeBegin[br] = (int)max((long long)begin, base + (long long)t0 * a.tile);
				a.rangeEnd[br] = (int)min((long long)end, base + (long long)t1 * a.tile);
				a.rangeSeg[br] = s;
				++br;
			}
		}
	}
	if(tid == 0) {
		a.counters[0] = totT;
		a.counters[1] = totS;
		a.counters[2] = totL;
		a.counters[3] = totR;
	}
}

struct SegCountArgs {
	const unsigned* keys;
	const int* rangeBegin;
	const int* rangeEnd;
	int* counters;
	int work;                       // counters[work]: next range to count
	int shift;
	int width;
	int vecOk;
	unsigned* counts;               // [R][256], range-major
};

__global__ void __launch_bounds__(kCountThreads) seg_count_kernel(const SegCountArgs a) {
	__shared__ unsigned sHist[kDigitBins * 32];
	const int tid = threadIdx.x;
	const int lane = tid & 31;
	const unsigned mask = (1u << a.width) - 1;
	const int shift = a.shift;
	__shared__ int sNext;
	const int R = a.counters[3];
	unsigned* myCol = sHist + lane;
	auto add = [&](unsigned k) { atomicAdd(&myCol[((k >> shift) & mask) * 32], 1u); };

	// Ranges differ in size: each CTA draws the next one when done.
	for(;;) {
		if(tid == 0) sNext = atomicAdd(&a.counters[a.work], 1);
		for(int i = tid; i < kDigitBins * 32; i += kCountThreads) sHist[i] = 0;
		__syncthreads();
		const int r = sNext;
		if(r >= R) break;
		const int begin = a.rangeBegin[r];
		const int end = a.rangeEnd[r];
		int e = begin;
		if(a.vecOk) {
			// Plain loads up to a 16-byte boundary, then 16-byte loads.
			const int head = min(end, (begin + 3) & ~3);
			for(int i = begin + tid; i < head; i += kCountThreads) add(a.keys[i]);
			const uint4* src = reinterpret_cast<const uint4*>(a.keys + head);
			const int nvec = max(0, (end - head) / 4);
			// Four independent 16-byte loads in flight per thread.
			constexpr int U = 4;
			int i = tid;
			for(; i + (U - 1) * kCountThreads < nvec; i += U * kCountThreads) {
				uint4 q[U];
#pragma unroll
				for(int u = 0; u < U; ++u) q[u] = ld_stream_u4(src + i + u * kCountThreads);
#pragma unroll
				for(int u = 0; u < U; ++u) {
					add(q[u].x);
					add(q[u].y);
					add(q[u].z);
					add(q[u].w);
				}
			}
			for(; i < nvec; i += kCountThreads) {
				const uint4 q = ld_stream_u4(src + i);
				add(q.x);
				add(q.y);
				add(q.z);
				add(q.w);
			}
			e = head + 4 * nvec;
		}
		for(int i = e + tid; i < end; i += kCountThreads) add(a.keys[i]);
		__syncthreads();
		for(int b = tid >> 5; b < kDigitBins; b += kCountThreads / 32) {
			unsigned c = sHist[b * 32 + lane];
#pragma unroll
			for(int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
			if(lane == 0) a.counts[(size_t)r * kDigitBins + b] = c;
		}
		__syncthreads();
	}
}

struct SegScanArgs {
	const int* offsets;
	const int* largeList;
	const int* largeRangeFirst;
	const int* largeRangeCount;
	const int* counters;
	const unsigned* counts;         // [R][256]
	unsigned* rangeStart;           // [R][256]: first output position per digit
	unsigned* rangeTrivial;         // [R]: the segment has a single digit
};

// One CTA per large segment: digit d of range r starts at segment start +
// keys of the segment with smaller digits + keys with digit d in the
// segment's earlier ranges.
__global__ void __launch_bounds__(256) seg_scan_kernel(const SegScanArgs a) {
	__shared__ unsigned sScan[8];
	const int d = threadIdx.x;
	const int lane = d & 31;
	const int warp = d >> 5;
	const int L = a.counters[2];
	for(int i = blockIdx.x; i < L; i += gridDim.x) {
		const int s = a.largeList[i];
		const int r0 = a.largeRangeFirst[i];
		const int nr = a.largeRangeCount[i];
		unsigned run = 0;
		for(int k = 0; k < nr; ++k) {
			const size_t at = (size_t)(r0 + k) * kDigitBins + d;
			const unsigned c = a.counts[at];
			a.rangeStart[at] = run;
			run += c;
		}
		const unsigned incl = warp_inclusive_scan(run, lane);
		if(lane == 31) sScan[warp] = incl;
		const int nonEmpty = __syncthreads_count(run != 0);
		unsigned prefix = 0;
		for(int w = 0; w < warp; ++w) prefix += sScan[w];
		const unsigned base = (unsigned)a.offsets[s] + prefix + incl - run;
		for(int k = 0; k < nr; ++k) {
			const size_t at = (size_t)(r0 + k) * kDigitBins + d;
			a.rangeStart[at] += base;
		}
		if(d < nr) a.rangeTrivial[r0 + d] = nonEmpty <= 1;
		for(int k = d + 256; k < nr; k += 256) a.rangeTrivial[r0 + k] = nonEmpty <= 1;
		__syncthreads();
	}
}

struct SegSortArgs {
	SortArgs sort;                  // buffers, digit, bulk flag, errors
	const int* offsets;
	const int* rangeBegin;
	const int* rangeEnd;
	const int* rangeSeg;
	int* counters;
	int work;                       // counters[work]: next range to sort
	const unsigned* rangeStart;
	const unsigned* rangeTrivial;
};

template<int VM, bool BYTE>
__global__ void __launch_bounds__(SortLayout<VM>::NT, SortConfig<VM>::kMinBlocks)
seg_sort_kernel(const SegSortArgs a) {
	extern __shared__ __align__(128) unsigned smem[];
	const SortSmem<VM> sm(smem);
	const int tid = threadIdx.x;
	__shared__ int sNext;
	const int R = a.counters[3];
	sort_setup<VM>(sm);
	unsigned phase = 0;
	// Ranges differ in size: each CTA draws the next one when done.
	for(;;) {
		if(tid == 0) sNext = atomicAdd(&a.counters[a.work], 1);
		__syncthreads();
		const int r = sNext;
		if(r >= R) break;
		const long long begin = a.rangeBegin[r];
		const long long end = a.rangeEnd[r];
		const long long segStart = a.offsets[a.rangeSeg[r]];
		if(tid < kDigitBins) sm.running[tid] = a.rangeStart[(size_t)r * kDigitBins + tid];
		const bool trivial = a.rangeTrivial[r] != 0;
		__syncthreads();
		if(trivial) copy_range<VM>(a.sort, begin, end, segStart);
		else sort_range<VM, BYTE, SortConfig<VM>::kBallotBits>(a.sort, sm, begin, end, segStart,
			phase);
		__syncthreads();
	}
}

// Segments of at most TILE elements, sorted whole in shared memory: keys
// and their segment-local positions go through every pass, then keys are
// written out and each value array is permuted through shared memory by
// the final positions (index mode writes the positions).
constexpr int kSmallThreads = 256;
constexpr int kSmallBallotBits = MGPU_SORT_SMALL_BALLOT_BITS;
constexpr int kSmallRankBatch = MGPU_SORT_SMALL_RANK_BATCH;

struct SmallSortArgs {
	PassBuffers buf;                // in: [0] arrays; out: the result arrays
	PassPlan plan;
	const int* offsets;
	const int* list;
	int* counters;
	int listIndex;                  // counters[listIndex] = list length
	int work;                       // counters[work]: next list entry
	int numArrays;                  // value arrays to permute (0 in index mode)
	int indexMode;
};

// One segment [begin, begin + len) of at most kSmallThreads * IPT elements,
// sorted whole in shared memory: keys and their segment-local positions go
// through every pass, then keys are written out and each value array is
// permuted through shared memory by the final positions (index mode writes
// the positions). Ends with a barrier.
template<int IPT, int NT = kSmallThreads>
__device__ __forceinline__ void small_sort_segment(const SmallSortArgs& a, int begin,
	int len, unsigned* sKeys, unsigned* sIdx, unsigned* sWarpHist, unsigned* sScan,
	unsigned ltMask, const unsigned (&nClear)[4]) {
	static_assert(NT >= kDigitBins && NT % 32 == 0 && NT <= 1024, "one thread per digit");
	constexpr int TILE = NT * IPT;
	constexpr int NW = NT / 32;
	const int tid = threadIdx.x;
	const int lane = tid & 31;
	const int warp = tid >> 5;
	const int warpBase = warp * 32 * IPT;

	for(int j = tid; j < TILE; j += NT) {
		sKeys[j] = j < len ? a.buf.keysIn[begin + j] : 0xffffffffu;
		sIdx[j] = j;
	}
	for(int j = tid; j < NW * kDigitBins; j += NT) sWarpHist[j] = 0;
	__syncthreads();

	for(int p = 0; p < a.plan.numPasses; ++p) {
		const DigitOf<false> digit(a.plan.shift[p], a.plan.width[p]);
		unsigned rank[IPT];
		rank_tile<IPT, false, false, kSmallBallotBits,
			(IPT < kSmallRankBatch ? IPT : kSmallRankBatch)>(sKeys, sWarpHist + warp * kDigitBins, warpBase,
			lane, len, digit, ltMask, nClear, rank);
		__syncthreads();
		// Thread d < 256: digit d's count over the warps, its start, and
		// each warp's run start.
		unsigned c[NW];
		unsigned tileTotal = 0;
		if(tid < kDigitBins) {
#pragma unroll
			for(int w = 0; w < NW; ++w) {
				c[w] = sWarpHist[w * kDigitBins + tid];
				tileTotal += c[w];
			}
		}
		const unsigned incl = warp_inclusive_scan(tileTotal, lane);
		if(lane == 31 && tid < kDigitBins) sScan[warp] = incl;
		__syncthreads();
		if(tid < kDigitBins) {
			unsigned prefix = 0;
			for(int w = 0; w < warp; ++w) prefix += sScan[w];
			unsigned run = prefix + incl - tileTotal;
#pragma unroll
			for(int w = 0; w < NW; ++w) {
				sWarpHist[w * kDigitBins + tid] = run;
				run += c[w];
			}
		}
		unsigned keys[IPT], idx[IPT];
#pragma unroll
		for(int j = 0; j < IPT; ++j) {
			keys[j] = sKeys[warpBase + j * 32 + lane];
			idx[j] = sIdx[warpBase + j * 32 + lane];
		}
		__syncthreads();
#pragma unroll
		for(int j = 0; j < IPT; ++j) {
			const unsigned pos = (rank[j] & 0xffffu)
				+ sWarpHist[warp * kDigitBins + (rank[j] >> 16)];
			sKeys[pos] = keys[j];
			sIdx[pos] = idx[j];
		}
		__syncthreads();
		for(int j = tid; j < NW * kDigitBins; j += NT) sWarpHist[j] = 0;
		__syncthreads();
	}

	for(int j = tid; j < len; j += NT) {
		a.buf.keysOut[begin + j] = sKeys[j];
		if(a.indexMode) a.buf.valsOut[0][begin + j] = sIdx[j];
	}
	for(int v = 0; v < a.numArrays; ++v) {
		// Stage the segment's values (the input may be the output buffer).
		__syncthreads();
		for(int j = tid; j < len; j += NT) sKeys[j] = a.buf.valsIn[v][begin + j];
		__syncthreads();
		for(int j = tid; j < len; j += NT) a.buf.valsOut[v][begin + j] = sKeys[sIdx[j]];
	}
	__syncthreads();
}

// Segments of at most kSmallThreads * MAXIPT elements, persistent over a
// list (each CTA draws the next entry when done). Each segment is sorted in
// the smallest tile of 2, 4, 8 or 16 keys per thread that holds it, so the
// ranking work follows the segment's size.
template<int MAXIPT>
__global__ void __launch_bounds__(kSmallThreads) small_sort_kernel(const SmallSortArgs a) {
	constexpr int NT = kSmallThreads;
	constexpr int NW = NT / 32;
	__shared__ unsigned sKeys[NT * MAXIPT];
	__shared__ unsigned sIdx[NT * MAXIPT];
	__shared__ unsigned sWarpHist[NW * kDigitBins];
	__shared__ unsigned sScan[32];
	__shared__ int sNext;

	const int tid = threadIdx.x;
	const int lane = tid & 31;
	const unsigned ltMask = lanemask_lt();
	unsigned nClear[4];
#pragma unroll
	for(int k = 0; k < 4; ++k) nClear[k] = ((lane >> k) & 1) ? 0u : 0xffffffffu;
	const int count = a.counters[a.listIndex];

	for(;;) {
		if(tid == 0) sNext = atomicAdd(&a.counters[a.work], 1);
		__syncthreads();
		const int i = sNext;
		if(i >= count) break;
		const int s = a.list[i];
		const int begin = a.offsets[s];
		const int len = a.offsets[s + 1] - begin;
		if constexpr(MAXIPT >= 16) {
			if(len > 8 * NT) {
				small_sort_segment<16>(a, begin, len, sKeys, sIdx, sWarpHist, sScan,
					ltMask, nClear);
				continue;
			}
		}
		if constexpr(MAXIPT >= 8) {
			if(len > 4 * NT) {
				small_sort_segment<8>(a, begin, len, sKeys, sIdx, sWarpHist, sScan,
					ltMask, nClear);
				continue;
			}
		}
		if constexpr(MAXIPT >= 4) {
			if(len > 2 * NT) {
				small_sort_segment<4>(a, begin, len, sKeys, sIdx, sWarpHist, sScan,
					ltMask, nClear);
				continue;
			}
		}
		small_sort_segment<2>(a, begin, len, sKeys, sIdx, sWarpHist, sScan, ltMask, nClear);
	}
}

// A whole array of at most NT * IPT elements, sorted by one CTA of NT
// threads through every pass in shared memory (sortArray on small arrays:
// one launch). Dynamic shared memory: keys and positions (NT * IPT words
// each), the warp histograms, the scan words.
template<int NT, int IPT>
__host__ __device__ constexpr size_t small_array_smem_bytes() {
	return sizeof(unsigned) * (2 * (size_t)NT * IPT + (NT / 32) * kDigitBins + 32);
}

template<int NT, int IPT>
__global__ void __launch_bounds__(NT) small_array_kernel(const SmallSortArgs a, int n) {
	extern __shared__ __align__(128) unsigned smem[];
	unsigned* sKeys = smem;
	unsigned* sIdx = sKeys + NT * IPT;
	unsigned* sWarpHist = sIdx + NT * IPT;
	unsigned* sScan = sWarpHist + (NT / 32) * kDigitBins;
	const int lane = threadIdx.x & 31;
	const unsigned ltMask = lanemask_lt();
	unsigned nClear[4];
#pragma unroll
	for(int k = 0; k < 4; ++k) nClear[k] = ((lane >> k) & 1) ? 0u : 0xffffffffu;
	small_sort_segment<IPT, NT>(a, 0, n, sKeys, sIdx, sWarpHist, sScan, ltMask, nClear);
}

int small_array_max_elements() { return MGPU_SORT_SMALL_ARRAY_MAX; }

template<int NT, int IPT>
static cudaError_t launch_small_shape(const SmallSortArgs& a, int n, cudaStream_t stream) {
	return launch_plain(small_array_kernel<NT, IPT>, 1, NT,
		(int)small_array_smem_bytes<NT, IPT>(), stream, a, n);
}

static cudaError_t configure_small_array_kernels() {
	cudaError_t e = cudaSuccess;
	cudaError_t r;
	const cudaFuncAttribute m = cudaFuncAttributeMaxDynamicSharedMemorySize;
#define MGPU_SMALL_SHAPE(nt, ipt) \
	if((r = cudaFuncSetAttribute(small_array_kernel<nt, ipt>, m, \
		(int)small_array_smem_bytes<nt, ipt>())) != cudaSuccess) e = r;
	MGPU_SMALL_SHAPE(256, 2)
	MGPU_SMALL_SHAPE(256, 4)
	MGPU_SMALL_SHAPE(256, 8)
	MGPU_SMALL_SHAPE(256, 16)
	MGPU_SMALL_SHAPE(512, 4)
	MGPU_SMALL_SHAPE(1024, 4)
#undef MGPU_SMALL_SHAPE
	return e;
}

// The CTA grows with the array (up to MGPU_SORT_SMALL_ARRAY_THREADS threads)
// before the keys per thread do: more warps rank in parallel, and each
// warp's chain of counter updates stays short.
cudaError_t launch_small_array(const PassBuffers& buf, int valueMode, const PassPlan& plan,
	int n, cudaStream_t stream) {
	if(n <= 0 || n > kSegSmallMax || n > MGPU_SORT_SMALL_ARRAY_MAX) return cudaErrorInvalidValue;
	SmallSortArgs a = {};
	a.buf = buf;
	a.plan = plan;
	a.numArrays = valueMode > 0 ? valueMode : 0;
	a.indexMode = valueMode == kValueIndex;
	constexpr int kMaxThreads = MGPU_SORT_SMALL_ARRAY_THREADS;
	if(n <= 512) return launch_small_shape<256, 2>(a, n, stream);
	if(n <= 1024) return launch_small_shape<256, 4>(a, n, stream);
	if(kMaxThreads >= 512 && n <= 2048) return launch_small_shape<512, 4>(a, n, stream);
	if(kMaxThreads >= 1024) return launch_small_shape<1024, 4>(a, n, stream);
	if(kMaxThreads >= 512) return launch_small_shape<512, 8>(a, n, stream);
	if(n <= 2048) return launch_small_shape<256, 8>(a, n, stream);
	return launch_small_shape<256, 16>(a, n, stream);
}

__global__ void iota_kernel(unsigned* out, int n) {
	for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
		i += (long long)gridDim.x * blockDim.x)
		out[i] = (unsigned)i;
}

////////////////////////////////////////////////////////////////////////////////
// Host launchers.

template<int VM>
static cudaError_t set_sort_attributes() {
	const int bytes = (int)SortLayout<VM>::kBytes;
	const cudaFuncAttribute attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
	constexpr int bb = SortConfig<VM>::kBallotBits;
	constexpr int bbLarge = SortConfig<VM>::kBallotBitsLarge;
	cudaError_t e = cudaFuncSetAttribute(sort_kernel<VM, false, bb>, attr, bytes);
	if(e == cudaSuccess) e = cudaFuncSetAttribute(sort_kernel<VM, true, bb>, attr, bytes);
	if constexpr(bbLarge != bb) {
		if(e == cudaSuccess) e = cudaFuncSetAttribute(sort_kernel<VM, false, bbLarge>, attr, bytes);
		if(e == cudaSuccess) e = cudaFuncSetAttribute(sort_kernel<VM, true, bbLarge>, attr, bytes);
	}
	return e;
}

// The segmented passes' kernels of a value mode (kSegIndex, 0, kSegOne, 2..6).
template<int VM>
static cudaError_t set_seg_attributes() {
	const int bytes = (int)SortLayout<VM>::kBytes;
	const cudaFuncAttribute attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
	cudaError_t e = cudaFuncSetAttribute(seg_sort_kernel<VM, false>, attr, bytes);
	if(e == cudaSuccess) e = cudaFuncSetAttribute(seg_sort_kernel<VM, true>, attr, bytes);
	return e;
}

cudaError_t configure_kernels() {
	cudaError_t e = cudaSuccess;
	cudaError_t r;
#if MGPU_SORT_SEG_SHARED_CARVEOUT
	{
		const cudaFuncAttribute c = cudaFuncAttributePreferredSharedMemoryCarveout;
		const int v = (int)cudaSharedmemCarveoutMaxShared;
		if((r = cudaFuncSetAttribute(seg_plan_kernel, c, v)) != cudaSuccess) e = r;
		if((r = cudaFuncSetAttribute(seg_count_kernel, c, v)) != cudaSuccess) e = r;
		if((r = cudaFuncSetAttribute(seg_scan_kernel, c, v)) != cudaSuccess) e = r;
		if((r = cudaFuncSetAttribute(small_sort_kernel<kSegTinyMax / kSmallThreads>, c, v))
			!= cudaSuccess) e = r;
		if((r = cudaFuncSetAttribute(small_sort_kernel<kSegSmallMax / kSmallThreads>, c, v))
			!= cudaSuccess) e = r;
	}
#endif
	if((r = set_sort_attributes<-1>()) != cudaSuccess) e = r;
	if((r = set_sort_attributes<0>()) != cudaSuccess) e = r;
	if((r = set_sort_attributes<kKeysLarge>()) != cudaSuccess) e = r;
	if((r = set_sort_attributes<1>()) != cudaSuccess) e = r;
	if((r = set_sort_attributes<2>()) != cudaSuccess) e = r;
	if((r = set_sort_attributes<3>()) != cudaSuccess) e = r;
	if((r = set_sort_attributes<4>()) != cudaSuccess) e = r;
	if((r = set_sort_attributes<5>()) != cudaSuccess) e = r;
	if((r = set_sort_attributes<6>()) != cudaSuccess) e = r;
	if((r = set_seg_attributes<kSegIndex>()) != cudaSuccess) e = r;
	if((r = set_seg_attributes<0>()) != cudaSuccess) e = r;
	if((r = set_seg_attributes<kSegOne>()) != cudaSuccess) e = r;
	if((r = set_seg_attributes<2>()) != cudaSuccess) e = r;
	if((r = set_seg_attributes<3>()) != cudaSuccess) e = r;
	if((r = set_seg_attributes<4>()) != cudaSuccess) e = r;
	if((r = set_seg_attributes<5>()) != cudaSuccess) e = r;
	if((r = set_seg_attributes<6>()) != cudaSuccess) e = r;
	if((r = configure_onesweep_kernels()) != cudaSuccess) e = r;
	if((r = configure_coop_kernels()) != cudaSuccess) e = r;
	if((r = configure_small_array_kernels()) != cudaSuccess) e = r;
	if((r = cudaFuncSetAttribute(upsweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
		(int)upsweep_smem_bytes(kMaxBins))) != cudaSuccess) e = r;
	return e;
}

int pass_tile_elements(int valueMode) {
	switch(valueMode) {
		case kKeysLarge: return SortLayout<kKeysLarge>::TILE;
		case kSegOne: return SortLayout<kSegOne>::TILE;
		case kSegIndex: return SortLayout<kSegIndex>::TILE;
		case -1: return SortLayout<-1>::TILE;
		case 0: return SortLayout<0>::TILE;
		case 1: return SortLayout<1>::TILE;
		default: return SortLayout<2>::TILE;
	}
}

size_t pass_scratch_bytes() {
	return sizeof(unsigned) * kPassScratchWords;
}

cudaError_t launch_upsweep(const unsigned* keys, int n, const PassPlan& plan,
	Control* ctrl, volatile unsigned* hostError, int numSMs,
	cudaStream_t stream) {
	return launch_onesweep_upsweep(keys, n, plan, ctrl, nullptr, 0, hostError, numSMs,
		stream);
}

cudaError_t launch_onesweep_upsweep(const unsigned* keys, int n, const PassPlan& plan,
	Control* ctrl, void* status0, size_t statusBytes, volatile unsigned* hostError,
	int numSMs, cudaStream_t stream) {
	UpsweepArgs a;
	a.keys = keys;
	a.n = n;
	a.vecOk = ((reinterpret_cast<size_t>(keys) & 15) == 0);
	a.plan = plan;
	a.ctrl = ctrl;
	a.hostError = hostError;
	a.status0 = static_cast<unsigned*>(status0);
	a.statusWords = statusBytes / sizeof(unsigned);
	long long chunks = ((long long)n + kUpChunk - 1) / kUpChunk;
	int grid = (int)std::min<long long>(chunks, (long long)numSMs);
	if(grid < 1) grid = 1;
	return launch_plain(upsweep_kernel, grid, kUpThreads, upsweep_smem_bytes(plan.totalBins),
		stream, a);
}

// CTAs of the sort kernel that fit on one SM (occupancy), once per mode.
template<int VM>
static int sort_ctas_per_sm() {
	static int perSM = 0;
	if(!perSM) {
		int v = 0;
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v,
			sort_kernel<VM, false, SortConfig<VM>::kBallotBits>,
			SortLayout<VM>::NT, SortLayout<VM>::kBytes);
		perSM = v > 0 ? v : 1;
	}
	return perSM;
}

template<int VM>
static RangeSplit split_for(int n, int numSMs) {
	using L = SortLayout<VM>;
	RangeSplit split;
	split.numTiles = (int)(((long long)n + L::TILE - 1) / L::TILE);
	long long ranges = std::min<long long>(split.numTiles,
		(long long)numSMs * sort_ctas_per_sm<VM>());
	ranges = std::min<long long>(ranges, kMaxRanges);
	split.numRanges = (int)std::max<long long>(ranges, 1);
	split.tilesLo = split.numTiles / split.numRanges;
	split.extra = split.numTiles % split.numRanges;
	return split;
}

// The tile class of a sortArray pass: keys-only passes over at least
// MGPU_SORT_KEYS_LARGE_ELEMENTS keys take the large-array shape.
static int pass_class(int valueMode, int n) {
	return valueMode == 0 && (long long)n >= MGPU_SORT_KEYS_LARGE_ELEMENTS ? kKeysLarge
		: valueMode;
}

static RangeSplit split_for_mode(int valueMode, int n, int numSMs) {
	switch(valueMode) {
		case kKeysLarge: return split_for<kKeysLarge>(n, numSMs);
		case -1: return split_for<-1>(n, numSMs);
		case 0: return split_for<0>(n, numSMs);
		case 1: return split_for<1>(n, numSMs);
		case 2: return split_for<2>(n, numSMs);
		case 3: return split_for<3>(n, numSMs);
		case 4: return split_for<4>(n, numSMs);
		case 5: return split_for<5>(n, numSMs);
		default: return split_for<6>(n, numSMs);
	}
}

cudaError_t launch_pass_count(const PassBuffers& buf, int valueMode, int n,
	int pass, const PassPlan& plan, unsigned* scratch, int numSMs,
	cudaStream_t stream) {
	const int cls = pass_class(valueMode, n);
	const RangeSplit split = split_for_mode(cls, n, numSMs);
	unsigned* rangeCounts = scratch;
	CountArgs c;
	c.keys = buf.keysIn;
	c.n = n;
	c.tile = pass_tile_elements(cls);
	c.shift = plan.shift[pass];
	c.width = plan.width[pass];
	c.vecOk = (reinterpret_cast<size_t>(buf.keysIn) & 15) == 0;
	c.split = split;
	c.rangeCounts = rangeCounts;
	// Small sorts: count and scan take the sort kernel's carveout, so that
	// no SM has to change its L1/shared split (which it can only do when
	// idle) between the kernels of a pass. Larger sorts leave the count
	// kernel its default, larger L1.
	const int carveout = (long long)n <= MGPU_SORT_CARVEOUT_MAX_ELEMENTS
		? (int)cudaSharedmemCarveoutMaxShared : -1;
	cudaError_t e = launch_dependent(count_kernel, split.numRanges, kCountThreads, 0,
		stream, c, carveout);
	if(e != cudaSuccess) return e;

	ScanArgs s;
	s.rangeCounts = rangeCounts;
	s.rangeOffsets = scratch + (size_t)kDigitBins * kMaxRanges;
	s.totals = scratch + 2 * (size_t)kDigitBins * kMaxRanges;
	s.numRanges = split.numRanges;
	return launch_dependent(scan_kernel, kDigitBins, (split.numRanges + 31) / 32 * 32, 0,
		stream, s, carveout);
}

template<int VM, int BB>
static cudaError_t launch_sort_bb(const SortArgs& a, cudaStream_t stream) {
	using L = SortLayout<VM>;
	if(a.width == 8 && (a.shift & 7) == 0)
		return launch_dependent(sort_kernel<VM, true, BB>, a.split.numRanges, L::NT,
			L::kBytes, stream, a);
	return launch_dependent(sort_kernel<VM, false, BB>, a.split.numRanges, L::NT,
		L::kBytes, stream, a);
}

template<int VM>
static cudaError_t launch_sort_vm(const SortArgs& a, cudaStream_t stream) {
	using C = SortConfig<VM>;
	if constexpr(C::kBallotBitsLarge != C::kBallotBits) {
		if(a.n >= C::kLargeElements) return launch_sort_bb<VM, C::kBallotBitsLarge>(a, stream);
	}
	return launch_sort_bb<VM, C::kBallotBits>(a, stream);
}

cudaError_t launch_pass_sort(const PassBuffers& buf, int valueMode, int n,
	int pass, const PassPlan& plan, Control* ctrl, unsigned* scratch,
	bool useBulk, int failTile, volatile unsigned* hostError, int numSMs,
	cudaStream_t stream) {
	SortArgs a;
	a.buf = buf;
	a.rangeOffsets = scratch + (size_t)kDigitBins * kMaxRanges;
	a.totals = scratch + 2 * (size_t)kDigitBins * kMaxRanges;
	a.devError = &ctrl->error;
	a.hostError = hostError;
	const int cls = pass_class(valueMode, n);
	a.split = split_for_mode(cls, n, numSMs);
	a.n = n;
	a.shift = plan.shift[pass];
	a.width = plan.width[pass];
	a.useBulk = useBulk ? 1 : 0;
	a.failTile = failTile;
	switch(cls) {
		case kKeysLarge: return launch_sort_vm<kKeysLarge>(a, stream);
		case -1: return launch_sort_vm<-1>(a, stream);
		case 0: return launch_sort_vm<0>(a, stream);
		case 1: return launch_sort_vm<1>(a, stream);
		case 2: return launch_sort_vm<2>(a, stream);
		case 3: return launch_sort_vm<3>(a, stream);
		case 4: return launch_sort_vm<4>(a, stream);
		case 5: return launch_sort_vm<5>(a, stream);
		case 6: return launch_sort_vm<6>(a, stream);
		default: return cudaErrorInvalidValue;
	}
}

cudaError_t launch_pass(const PassBuffers& buf, int valueMode, int n,
	int pass, const PassPlan& plan, Control* ctrl, unsigned* scratch,
	bool useBulk, int failTile, volatile unsigned* hostError, int numSMs,
	cudaStream_t stream) {
	cudaError_t e = launch_pass_count(buf, valueMode, n, pass, plan, scratch,
		numSMs, stream);
	if(e != cudaSuccess) return e;
	return launch_pass_sort(buf, valueMode, n, pass, plan, ctrl, scratch, useBulk,
		failTile, hostError, numSMs, stream);
}

////////////////////////////////////////////////////////////////////////////////
// Cooperative sort: every pass of a mid-size sort in one launch.
//
// A pass of the range partition is three dependent launches (count, scan,
// sort); for arrays of a few million keys each launch's fixed latency
// (prologue, first copy, drain) costs more than its work. Here one grid of
// co-resident CTAs (a cooperative launch: all CTAs run at once) runs the
// same three phases per pass with grid-wide barriers between them: CTA r
// counts range r, CTA r scans the columns of digits r, r + R, ..., CTA r
// sorts range r. Barriers are bounded waits: a CTA that gives up reports
// kErrBarrierTimeout and returns. Keys and values written by one pass are
// read by the next through L2 (coherent loads, bulk copies after a proxy
// fence), never through the non-coherent path.

struct CoopArgs {
	unsigned* keys[2];              // [0]: input of pass 0; passes alternate
	unsigned* vals[2];
	PassPlan plan;
	RangeSplit split;
	unsigned* rangeCounts;          // [256][R]
	unsigned* rangeOffsets;         // [256][R]
	unsigned* totals;               // [256]
	unsigned* barrier;              // arrivals, zero at launch
	unsigned* devError;
	volatile unsigned* hostError;
	int n;
	int vecOk;
	int useBulk;
	int indexFirst;                 // the first pass writes indices (index mode)
};

// Grid-wide barrier number `gen` (1, 2, ...): every CTA adds one arrival and
// waits for gen x gridDim.x of them. Thread 0's fences make the CTA's
// earlier global writes visible before its arrival and order its later
// loads and bulk copies after the other CTAs' writes. False if the wait ran
// out (reported).
__device__ __forceinline__ bool grid_barrier(const CoopArgs& a, unsigned gen) {
	__shared__ int sOk;
	__syncthreads();
	if(threadIdx.x == 0) {
		int ok = 1;
		__threadfence();
		atomicAdd(a.barrier, 1u);
		const unsigned target = gen * gridDim.x;
		WaitBudget budget;
		while(ld_relaxed_u32(a.barrier) < target) {
			if(!budget.poll()) {
				report_error(a.devError, a.hostError, kErrBarrierTimeout);
				ok = 0;
				break;
			}
		}
		__threadfence();
		asm volatile("fence.proxy.async.global;" ::: "memory");
		sOk = ok;
	}
	__syncthreads();
	return sOk != 0;
}

template<int VM, int BB>
__global__ void __launch_bounds__(SortLayout<VM>::NT, SortConfig<VM>::kMinBlocks)
coop_sort_kernel(const CoopArgs a) {
	static_assert(VM == 0 || VM == 1, "keys only or one value array");
	using L = SortLayout<VM>;
	static_assert(L::kWords >= kDigitBins * 32 + 32, "count and scan fit the sort's memory");
	extern __shared__ __align__(128) unsigned smem[];
	const int r = blockIdx.x;
	const int R = a.split.numRanges;
	unsigned gen = 0;
	for(int p = 0; p < a.plan.numPasses; ++p) {
		const int src = p & 1;
		CountArgs c;
		c.keys = a.keys[src];
		c.n = a.n;
		c.tile = L::TILE;
		c.shift = a.plan.shift[p];
		c.width = a.plan.width[p];
		c.vecOk = a.vecOk;
		c.split = a.split;
		c.rangeCounts = a.rangeCounts;
		count_range<false, L::NT>(c, r, smem);
		if(!grid_barrier(a, ++gen)) return;

		ScanArgs sc;
		sc.rangeCounts = a.rangeCounts;
		sc.rangeOffsets = a.rangeOffsets;
		sc.totals = a.totals;
		sc.numRanges = R;
		for(int d = r; d < kDigitBins; d += gridDim.x) {
			scan_digit(sc, d, smem);
			__syncthreads();
		}
		if(!grid_barrier(a, ++gen)) return;

		SortArgs sa;
		sa.buf.keysIn = a.keys[src];
		sa.buf.keysOut = a.keys[src ^ 1];
		for(int i = 0; i < 6; ++i) {
			sa.buf.valsIn[i] = i ? nullptr : a.vals[src];
			sa.buf.valsOut[i] = i ? nullptr : a.vals[src ^ 1];
		}
		sa.rangeOffsets = a.rangeOffsets;
		sa.totals = a.totals;
		sa.devError = a.devError;
		sa.hostError = a.hostError;
		sa.split = a.split;
		sa.n = a.n;
		sa.shift = a.plan.shift[p];
		sa.width = a.plan.width[p];
		sa.useBulk = a.useBulk;
		sa.failTile = -1;
		if(VM == 1 && a.indexFirst && p == 0)
			sort_one_range<kValueIndex, false, BB, false>(sa, smem, r);
		else
			sort_one_range<VM, false, BB, false>(sa, smem, r);
		if(p + 1 < a.plan.numPasses && !grid_barrier(a, ++gen)) return;
	}
}

template<int VM>
static int coop_ctas_per_sm() {
	static int perSM = 0;
	if(!perSM) {
		int v = 0;
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v,
			coop_sort_kernel<VM, SortConfig<VM>::kBallotBits>, SortLayout<VM>::NT,
			SortLayout<VM>::kBytes);
		perSM = v > 0 ? v : 0;
	}
	return perSM;
}

template<int VM>
static cudaError_t launch_coop_vm(CoopArgs& a, int numSMs, cudaStream_t stream) {
	using L = SortLayout<VM>;
	const int perSM = coop_ctas_per_sm<VM>();
	if(perSM <= 0) return cudaErrorCooperativeLaunchTooLarge;
	RangeSplit split;
	split.numTiles = (int)(((long long)a.n + L::TILE - 1) / L::TILE);
	long long ranges = std::min<long long>(split.numTiles, (long long)numSMs * perSM);
	// One scan thread per range.
	ranges = std::min<long long>(ranges, std::min(L::NT, kMaxRanges));
	split.numRanges = (int)std::max<long long>(ranges, 1);
	split.tilesLo = split.numTiles / split.numRanges;
	split.extra = split.numTiles % split.numRanges;
	a.split = split;
	cudaLaunchAttribute attr[1];
	attr[0].id = cudaLaunchAttributeCooperative;
	attr[0].val.cooperative = 1;
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = dim3(split.numRanges);
	cfg.blockDim = dim3(L::NT);
	cfg.dynamicSmemBytes = L::kBytes;
	cfg.stream = stream;
	cfg.attrs = attr;
	cfg.numAttrs = 1;
	return cudaLaunchKernelEx(&cfg, coop_sort_kernel<VM, SortConfig<VM>::kBallotBits>, a);
}

cudaError_t configure_coop_kernels() {
	cudaError_t e = cudaSuccess;
	cudaError_t r;
	const cudaFuncAttribute m = cudaFuncAttributeMaxDynamicSharedMemorySize;
	if((r = cudaFuncSetAttribute(coop_sort_kernel<0, SortConfig<0>::kBallotBits>, m,
		(int)SortLayout<0>::kBytes)) != cudaSuccess) e = r;
	if((r = cudaFuncSetAttribute(coop_sort_kernel<1, SortConfig<1>::kBallotBits>, m,
		(int)SortLayout<1>::kBytes)) != cudaSuccess) e = r;
	return e;
}

int coop_max_elements() {
	return MGPU_SORT_COOP_MAX_ELEMENTS;
}

cudaError_t launch_coop_sort(const PassBuffers& buf, int valueMode, int n,
	const PassPlan& plan, Control* ctrl, unsigned* scratch, bool useBulk,
	volatile unsigned* hostError, int numSMs, cudaStream_t stream) {
	if(valueMode < -1 || valueMode > 1 || n <= 0) return cudaErrorInvalidValue;
	cudaError_t e = cudaMemsetAsync(&ctrl->coopBarrier, 0, sizeof(unsigned), stream);
	if(e != cudaSuccess) return e;
	CoopArgs a;
	a.keys[0] = const_cast<unsigned*>(buf.keysIn);
	a.keys[1] = buf.keysOut;
	a.vals[0] = const_cast<unsigned*>(buf.valsIn[0]);
	a.vals[1] = buf.valsOut[0];
	a.plan = plan;
	a.rangeCounts = scratch;
	a.rangeOffsets = scratch + (size_t)kDigitBins * kMaxRanges;
	a.totals = scratch + 2 * (size_t)kDigitBins * kMaxRanges;
	a.barrier = &ctrl->coopBarrier;
	a.devError = &ctrl->error;
	a.hostError = hostError;
	a.n = n;
	a.vecOk = (reinterpret_cast<size_t>(buf.keysIn) & 15) == 0
		&& (reinterpret_cast<size_t>(buf.keysOut) & 15) == 0;
	a.useBulk = useBulk ? 1 : 0;
	a.indexFirst = valueMode == kValueIndex ? 1 : 0;
	if(valueMode == 0) return launch_coop_vm<0>(a, numSMs, stream);
	return launch_coop_vm<1>(a, numSMs, stream);
}

// Segmented scratch: [counters][lists 5 x S][range table 4 x Rmax]
// [counts Rmax x 256][rangeStart Rmax x 256], in 32-bit words.
struct SegScratch {
	int* counters;
	int* tinyList;
	int* smallList;
	int* largeList;
	int* largeRangeFirst;
	int* largeRangeCount;
	int* rangeBegin;
	int* rangeEnd;
	int* rangeSeg;
	unsigned* rangeTrivial;
	unsigned* counts;
	unsigned* rangeStart;
};

// The smallest tile of any value mode: the most ranges a plan can cut.
constexpr int kMinTile = std::min({SortLayout<kSegIndex>::TILE, SortLayout<kSegOne>::TILE,
	SortLayout<0>::TILE, SortLayout<2>::TILE, SortLayout<3>::TILE, SortLayout<4>::TILE,
	SortLayout<5>::TILE, SortLayout<6>::TILE});

// Ranges of a plan: a large segment (more than 4096 elements) of t tiles gets
// min(64, ceil(t / 4)) ranges, and t <= len / tile + 2 (aligned-down start,
// partial end), so it gets at most len / (4 tile) + 1.25. Summed over at most
// n / 4096 large segments that is below n / kMinTile + numSegments (tile >=
// kMinTile) whenever 0.25 n / 4096 <= 0.75 n / kMinTile, i.e. kMinTile <= 12288.
static_assert(kMinTile <= 12288, "the range bound of seg_max_ranges");

static size_t seg_max_ranges(int n, int numSegments) {
	return (size_t)n / kMinTile + (size_t)numSegments + 1;
}

size_t seg_scratch_bytes(int n, int numSegments) {
	const size_t S = (size_t)numSegments;
	const size_t R = seg_max_ranges(n, numSegments);
	return sizeof(unsigned) * (kSegCounters + 5 * S + 4 * R + 2 * R * kDigitBins) + 256;
}

static SegScratch seg_scratch(void* base, int n, int numSegments) {
	const size_t S = (size_t)numSegments;
	const size_t R = seg_max_ranges(n, numSegments);
	unsigned* w = static_cast<unsigned*>(base);
	SegScratch x;
	x.counters = reinterpret_cast<int*>(w); w += kSegCounters;
	x.tinyList = reinterpret_cast<int*>(w); w += S;
	x.smallList = reinterpret_cast<int*>(w); w += S;
	x.largeList = reinterpret_cast<int*>(w); w += S;
	x.largeRangeFirst = reinterpret_cast<int*>(w); w += S;
	x.largeRangeCount = reinterpret_cast<int*>(w); w += S;
	x.rangeBegin = reinterpret_cast<int*>(w); w += R;
	x.rangeEnd = reinterpret_cast<int*>(w); w += R;
	x.rangeSeg = reinterpret_cast<int*>(w); w += R;
	x.rangeTrivial = w; w += R;
	x.counts = w; w += R * kDigitBins;
	x.rangeStart = w;
	return x;
}

// The tile class of a segmented pass: index mode and one value array take
// the segmented sort's own shape.
static int seg_class(int valueMode) {
	return valueMode == 1 ? kSegOne : valueMode == kValueIndex ? kSegIndex : valueMode;
}

cudaError_t launch_seg_plan(const int* offsets, int numSegments, int n,
	int valueMode, void* scratch, Control* ctrl, volatile unsigned* hostError,
	cudaStream_t stream) {
	const SegScratch x = seg_scratch(scratch, n, numSegments);
	SegPlanArgs a;
	a.offsets = offsets;
	a.numSegments = numSegments;
	a.n = n;
	a.tile = pass_tile_elements(seg_class(valueMode));
	a.tinyList = x.tinyList;
	a.smallList = x.smallList;
	a.largeList = x.largeList;
	a.largeRangeFirst = x.largeRangeFirst;
	a.largeRangeCount = x.largeRangeCount;
	a.rangeBegin = x.rangeBegin;
	a.rangeEnd = x.rangeEnd;
	a.rangeSeg = x.rangeSeg;
	a.counters = x.counters;
	a.devError = &ctrl->error;
	a.hostError = hostError;
	return launch_plain(seg_plan_kernel, 1, kPlanThreads, 0, stream, a);
}

cudaError_t launch_seg_small(const PassBuffers& buf, int valueMode,
	const PassPlan& plan, const int* offsets, int numSegments, int n,
	void* scratch, int numSMs, cudaStream_t stream) {
	const SegScratch x = seg_scratch(scratch, n, numSegments);
	SmallSortArgs a;
	a.buf = buf;
	a.plan = plan;
	a.offsets = offsets;
	a.counters = x.counters;
	a.numArrays = valueMode > 0 ? valueMode : 0;
	a.indexMode = valueMode == kValueIndex;
	a.list = x.tinyList;
	a.listIndex = 0;
	a.work = kSegWorkSmall;
	cudaError_t e = launch_plain(small_sort_kernel<kSegTinyMax / kSmallThreads>, numSMs * 8,
		kSmallThreads, 0, stream, a);
	if(e != cudaSuccess) return e;
	a.list = x.smallList;
	a.listIndex = 1;
	a.work = kSegWorkSmall + 1;
	return launch_plain(small_sort_kernel<kSegSmallMax / kSmallThreads>, numSMs * 4,
		kSmallThreads, 0, stream, a);
}

template<int VM>
static int seg_sort_ctas_per_sm() {
	static int perSM = 0;
	if(!perSM) {
		int v = 0;
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, seg_sort_kernel<VM, false>,
			SortLayout<VM>::NT, SortLayout<VM>::kBytes);
		perSM = v > 0 ? v : 1;
	}
	return perSM;
}

template<int VM>
static cudaError_t launch_seg_sort_vm(const SegSortArgs& a, int numSMs, cudaStream_t stream) {
	using L = SortLayout<VM>;
	const int grid = numSMs * seg_sort_ctas_per_sm<VM>();
	if(a.sort.width == 8 && (a.sort.shift & 7) == 0)
		return launch_plain(seg_sort_kernel<VM, true>, grid, L::NT, L::kBytes, stream, a);
	return launch_plain(seg_sort_kernel<VM, false>, grid, L::NT, L::kBytes, stream, a);
}

cudaError_t launch_seg_pass(const PassBuffers& buf, int valueMode, int pass,
	const PassPlan& plan, const int* offsets, int numSegments, int n,
	void* scratch, Control* ctrl, bool useBulk, volatile unsigned* hostError,
	int numSMs, cudaStream_t stream) {
	const SegScratch x = seg_scratch(scratch, n, numSegments);
	SegCountArgs c;
	c.keys = buf.keysIn;
	c.rangeBegin = x.rangeBegin;
	c.rangeEnd = x.rangeEnd;
	c.counters = x.counters;
	c.shift = plan.shift[pass];
	c.width = plan.width[pass];
	c.vecOk = (reinterpret_cast<size_t>(buf.keysIn) & 15) == 0;
	c.counts = x.counts;
	c.work = kSegWork + 2 * pass;
	cudaError_t e = launch_plain(seg_count_kernel, numSMs * 4, kCountThreads, 0, stream, c);
	if(e != cudaSuccess) return e;

	SegScanArgs q;
	q.offsets = offsets;
	q.largeList = x.largeList;
	q.largeRangeFirst = x.largeRangeFirst;
	q.largeRangeCount = x.largeRangeCount;
	q.counters = x.counters;
	q.counts = x.counts;
	q.rangeStart = x.rangeStart;
	q.rangeTrivial = x.rangeTrivial;
	e = launch_plain(seg_scan_kernel, numSMs * 8, 256, 0, stream, q);
	if(e != cudaSuccess) return e;

	SegSortArgs a;
	a.sort.buf = buf;
	a.sort.rangeOffsets = nullptr;
	a.sort.totals = nullptr;
	a.sort.devError = &ctrl->error;
	a.sort.hostError = hostError;
	a.sort.n = n;
	a.sort.shift = plan.shift[pass];
	a.sort.width = plan.width[pass];
	a.sort.useBulk = useBulk ? 1 : 0;
	a.sort.failTile = -1;
	a.offsets = offsets;
	a.rangeBegin = x.rangeBegin;
	a.rangeEnd = x.rangeEnd;
	a.rangeSeg = x.rangeSeg;
	a.counters = x.counters;
	a.work = kSegWork + 2 * pass + 1;
	a.rangeStart = x.rangeStart;
	a.rangeTrivial = x.rangeTrivial;
	switch(seg_class(valueMode)) {
		case kSegIndex: return launch_seg_sort_vm<kSegIndex>(a, numSMs, stream);
		case kSegOne: return launch_seg_sort_vm<kSegOne>(a, numSMs, stream);
		case 0: return launch_seg_sort_vm<0>(a, numSMs, stream);
		case 2: return launch_seg_sort_vm<2>(a, numSMs, stream);
		case 3: return launch_seg_sort_vm<3>(a, numSMs, stream);
		case 4: return launch_seg_sort_vm<4>(a, numSMs, stream);
		case 5: return launch_seg_sort_vm<5>(a, numSMs, stream);
		case 6: return launch_seg_sort_vm<6>(a, numSMs, stream);
		default: return cudaErrorInvalidValue;
	}
}

cudaError_t launch_iota(unsigned* out, int n, cudaStream_t stream) {
	if(n <= 0) return cudaSuccess;
	int grid = (int)std::min<long long>(((long long)n + 255) / 256, 4096);
	return launch_plain(iota_kernel, grid, 256, 0, stream, out, n);
}

// Order-preserving uint32 image of signed and float keys (the transform of
// the reference's sort/src/kernels/common.cu:159-186, written from its
// definition): int32 flips the sign bit; float32 flips the sign bit of
// non-negative values and every bit of negative ones, so unsigned order is
// -NaN < -inf < ... < -0.0 < +0.0 < ... < +inf < +NaN. The inverse undoes
// it: an image with the top bit set came from a non-negative value.
__global__ void key_transform_kernel(unsigned* keys, int n, int keyType, int forward) {
	for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
		i += (long long)gridDim.x * blockDim.x) {
		unsigned k = keys[i];
		if(keyType == kKeyInt32) k ^= 0x80000000u;
		else {
			const bool top = (k >> 31) != 0;
			k ^= (forward ? top : !top) ? 0xffffffffu : 0x80000000u;
		}
		keys[i] = k;
	}
}

cudaError_t launch_key_transform(unsigned* keys, int n, int keyType, bool forward,
	cudaStream_t stream) {
	if(n <= 0 || keyType == kKeyUint32) return cudaSuccess;
	int grid = (int)std::min<long long>(((long long)n + 255) / 256, 4096);
	return launch_plain(key_transform_kernel, grid, 256, 0, stream, keys, n, keyType,
		forward ? 1 : 0);
}

} // namespace mgpusort
