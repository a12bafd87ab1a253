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

// Each bin of the upsweep's shared histogram has kUpCopies counters, one per
// lane class (lane % kUpCopies), in consecutive words: lanes of a warp that
// hit the same bin in one instruction mostly update different words (in
// different banks), which keeps skewed digits from serialising the atomics.
constexpr int kUpCopies = 4;

__device__ __forceinline__ void count_digits(unsigned* hist,
	const unsigned (&k)[kUpKeysPerThread], int nValid, int shift,
	unsigned mask, int copy) {
#pragma unroll
	for(int i = 0; i < kUpKeysPerThread; ++i)
		if(i < nValid)
			atomicAdd(&hist[((k[i] >> shift) & mask) * kUpCopies + copy], 1u);
}

__global__ void __launch_bounds__(kUpThreads, 3) upsweep_kernel(
	const UpsweepArgs a) {

	__shared__ unsigned sHist[kMaxBins * kUpCopies];
	__shared__ unsigned sScan[kUpThreads / 32];
	__shared__ unsigned sLast;

	const int tid = threadIdx.x;
	const int lane = tid & 31;
	const int warp = tid >> 5;
	const int copy = lane & (kUpCopies - 1);
	const int totalBins = a.plan.totalBins;
	const int numPasses = a.plan.numPasses;

	for(int i = tid; i < totalBins * kUpCopies; i += kUpThreads) sHist[i] = 0;
	__syncthreads();

	auto count_all = [&](const unsigned (&k)[kUpKeysPerThread], int nValid) {
		for(int p = 0; p < numPasses; ++p)
			count_digits(sHist + a.plan.binBase[p] * kUpCopies, k, nValid,
				a.plan.shift[p], (1u << a.plan.width[p]) - 1, copy);
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
		unsigned c = 0;
#pragma unroll
		for(int j = 0; j < kUpCopies; ++j) c += sHist[i * kUpCopies + j];
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

constexpr int kTileElements = 4096;
constexpr int kCountThreads = 512;

struct CountArgs {
	const unsigned* keys;
	int n;
	int shift;
	int width;
	int vecOk;
	RangeSplit split;
	unsigned* rangeCounts;          // [256][R], digit-major
};

__global__ void __launch_bounds__(kCountThreads) count_kernel(const CountArgs a) {
	__shared__ unsigned sHist[kDigitBins * kUpCopies];
	const int tid = threadIdx.x;
	const int copy = tid & (kUpCopies - 1);
	const int r = blockIdx.x;
	const unsigned mask = (1u << a.width) - 1;
	const int shift = a.shift;

	for(int i = tid; i < kDigitBins * kUpCopies; i += kCountThreads) sHist[i] = 0;
	__syncthreads();

	const long long begin = (long long)a.split.first_tile(r) * kTileElements;
	const long long end = min((long long)a.n,
		(long long)a.split.first_tile(r + 1) * kTileElements);
	auto add = [&](unsigned k) {
		atomicAdd(&sHist[((k >> shift) & mask) * kUpCopies + copy], 1u);
	};
	long long done = begin;
	if(a.vecOk) {
		// begin is a multiple of the tile size: 16-byte aligned.
		const uint4* src = reinterpret_cast<const uint4*>(a.keys + begin);
		const int nvec = (int)((end - begin) / 4);
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
		done = begin + 4ll * nvec;
	}
	for(long long e = done + tid; e < end; e += kCountThreads) add(a.keys[e]);
	__syncthreads();

	if(tid < kDigitBins) {
		unsigned c = 0;
#pragma unroll
		for(int j = 0; j < kUpCopies; ++j) c += sHist[tid * kUpCopies + j];
		a.rangeCounts[(size_t)tid * a.split.numRanges + r] = c;
	}
}

struct ScanArgs {
	const unsigned* rangeCounts;    // [256][R]
	unsigned* rangeOffsets;         // [256][R]: exclusive over ranges
	unsigned* totals;               // [256]
	int numRanges;
};

// One warp per digit: exclusive scan of the digit's range counts.
__global__ void __launch_bounds__(256) scan_kernel(const ScanArgs a) {
	const int lane = threadIdx.x & 31;
	const int d = blockIdx.x * 8 + (threadIdx.x >> 5);
	const unsigned* in = a.rangeCounts + (size_t)d * a.numRanges;
	unsigned* out = a.rangeOffsets + (size_t)d * a.numRanges;
	unsigned carry = 0;
	for(int base = 0; base < a.numRanges; base += 32) {
		const int r = base + lane;
		const unsigned v = r < a.numRanges ? in[r] : 0u;
		const unsigned incl = warp_inclusive_scan(v, lane);
		if(r < a.numRanges) out[r] = carry + incl - v;
		carry += __shfl_sync(0xffffffffu, incl, 31);
	}
	if(lane == 0) a.totals[d] = carry;
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

template<int VM> struct SortConfig {
	static constexpr int kThreads = 256;
	static constexpr int kItems = 16;
	static constexpr int kMinBlocks = 3;
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
	static constexpr int NV = VM > 0 ? VM : 0;
	// One value buffer holds the first value array (or the generated
	// indices); with more arrays, each further one is copied into the stream
	// buffer while the one before it is reordered in the value buffer.
	static constexpr int NVBUF = VM == 0 ? 0 : 1;
	static constexpr int NSTREAM = NV >= 2 ? 1 : 0;
	// Word offsets into dynamic shared memory.
	static constexpr int kKeys = 0;
	static constexpr int kVals = kKeys + KSLOTS * TILE;
	static constexpr int kStream = kVals + NVBUF * TILE;
	static constexpr int kWarpHist = kStream + NSTREAM * TILE;
	static constexpr int kDigStart = kWarpHist + NW * kDigitBins;
	static constexpr int kCount = kDigStart + kDigitBins;
	static constexpr int kRunning = kCount + kDigitBins;
	static constexpr int kScatter = kRunning + kDigitBins;
	static constexpr int kScan = kScatter + kDigitBins;
	static constexpr int kBar = kScan + 32;          // 8-byte aligned: even
	static constexpr int kWords = kBar + 2 * 6;       // 6 mbarriers
	static constexpr size_t kBytes = sizeof(unsigned) * kWords;
	static_assert(kBar % 2 == 0, "mbarriers need 8-byte alignment");
	static_assert(TILE == kTileElements, "count and sort kernels share tiles");
};

// Peers of an 8-bit digit: the lanes of the warp whose digit equals this
// lane's. From the eight ballots of the digit bits, lane l builds two
// entries of two 16-entry tables: the lanes whose low nibble is l & 15 and
// the lanes whose high nibble is l & 15 (nClear[k] is all ones where bit k of
// l & 15 is clear, so ballot ^ nClear[k] is the set of lanes agreeing with
// that bit). A lane's peers are the AND of the low-table entry for its low
// nibble and the high-table entry for its high nibble, fetched by shuffle.
__device__ __forceinline__ unsigned match_digit8(unsigned d,
	const unsigned (&nClear)[4]) {
	unsigned bal[8];
#pragma unroll
	for(int b = 0; b < 8; ++b) bal[b] = __ballot_sync(0xffffffffu, d & (1u << b));
	unsigned lo = bal[0] ^ nClear[0];
	unsigned hi = bal[4] ^ nClear[0];
#pragma unroll
	for(int k = 1; k < 4; ++k) {
		lo &= bal[k] ^ nClear[k];
		hi &= bal[4 + k] ^ nClear[k];
	}
	return __shfl_sync(0xffffffffu, lo, d & 15u) & __shfl_sync(0xffffffffu, hi, d >> 4);
}

// Stable warp rank of one item: the highest peer adds the group's size to
// the warp's running count of the digit; the old count, broadcast, is the
// group's base. Returns (digit << 16) | rank within the warp.
__device__ __forceinline__ unsigned rank_item(unsigned d, unsigned* warpHist,
	int lane, unsigned ltMask, const unsigned (&nClear)[4]) {
	const unsigned peers = match_digit8(d, nClear);
	const int leader = 31 - __clz(peers);
	unsigned base = 0;
	if(lane == leader) base = atomicAdd(&warpHist[d], (unsigned)__popc(peers));
	base = __shfl_sync(0xffffffffu, base, leader);
	// Orders this item's counter update before the next item's.
	__syncwarp();
	return (d << 16) | (base + __popc(peers & ltMask));
}

__device__ __forceinline__ void stage_tile(unsigned* dst, const unsigned* src,
	unsigned bytes, uint64_t* bar) {
	mbar_arrive_expect_tx(bar, bytes);
	bulk_load(dst, src, bytes, bar);
}

// Rank the staged tile's keys (warp-striped: item i of lane l in warp w is
// tile element w*32*IPT + i*32 + l, so (item, lane) order is input order per
// warp). In a partial tile the elements past `count` get digit 255: they
// rank after every real key and are never stored.
template<int IPT, bool FULL>
__device__ __forceinline__ void rank_tile(const unsigned* sKeys, unsigned* myHist,
	int warpBase, int lane, int count, int shift, unsigned mask, unsigned ltMask,
	const unsigned (&nClear)[4], unsigned (&rank)[IPT]) {
#pragma unroll
	for(int i = 0; i < IPT; ++i) {
		const int idx = warpBase + i * 32 + lane;
		unsigned d = (sKeys[idx] >> shift) & mask;
		if(!FULL && idx >= count) d = kDigitBins - 1;
		rank[i] = rank_item(d, myHist, lane, ltMask, nClear);
	}
}

template<int VM>
__global__ void __launch_bounds__(SortLayout<VM>::NT, SortConfig<VM>::kMinBlocks)
sort_kernel(const SortArgs a) {

	using L = SortLayout<VM>;
	constexpr int NT = L::NT;
	constexpr int IPT = L::IPT;
	constexpr int TILE = L::TILE;
	constexpr int NW = L::NW;
	constexpr int NV = L::NV;
	constexpr int KSLOTS = L::KSLOTS;
	constexpr unsigned kTileBytes = TILE * 4;

	extern __shared__ __align__(128) unsigned smem[];
	unsigned* sVals = smem + L::kVals;
	unsigned* sStream = smem + L::kStream;
	unsigned* sWarpHist = smem + L::kWarpHist;
	unsigned* sRunning = smem + L::kRunning;
	int* sScatter = reinterpret_cast<int*>(smem + L::kScatter);
	unsigned* sScan = smem + L::kScan;
	// mbarriers: [0..1] key slots, [2] value buffer, [3] stream buffer,
	// [5] injected-fault wait (never completed).
	uint64_t* sBar = reinterpret_cast<uint64_t*>(smem + L::kBar);

	const int tid = threadIdx.x;
	const int lane = tid & 31;
	const int warp = tid >> 5;
	const int warpBase = warp * 32 * IPT;
	const int r = blockIdx.x;
	const int t0 = a.split.first_tile(r);
	const int t1 = a.split.first_tile(r + 1);
	const int R = a.split.numRanges;

	// Each digit starts at the keys with smaller digits in the whole array
	// plus the keys with this digit in the ranges before this one.
	const unsigned total = tid < kDigitBins ? a.totals[tid] : 0u;
	const unsigned inclTotal = warp_inclusive_scan(total, lane);
	if(lane == 31 && tid < kDigitBins) sScan[warp] = inclTotal;
	const int nonEmpty = __syncthreads_count(tid < kDigitBins && total != 0);
	if(tid < kDigitBins) {
		unsigned prefix = 0;
		for(int w = 0; w < warp; ++w) prefix += sScan[w];
		sRunning[tid] = prefix + inclTotal - total + a.rangeOffsets[(size_t)tid * R + r];
	}

	if(nonEmpty <= 1) {
		// Every key has the same digit: the pass is the identity.
		const long long b = (long long)t0 * TILE;
		const long long e = min((long long)a.n, (long long)t1 * TILE);
		for(long long i = b + tid; i < e; i += NT) {
			a.buf.keysOut[i] = a.buf.keysIn[i];
			if constexpr(VM == kValueIndex) a.buf.valsOut[0][i] = (unsigned)i;
#pragma unroll
			for(int v = 0; v < NV; ++v) a.buf.valsOut[v][i] = a.buf.valsIn[v][i];
		}
		return;
	}

	auto tile_is_bulk = [&](int t) {
		return a.useBulk && (long long)(t + 1) * TILE <= a.n;
	};

	if(tid == 0) {
		for(int i = 0; i < 6; ++i) mbar_init(&sBar[i], 1);
		fence_mbar_init();
		if(t0 < t1 && tile_is_bulk(t0)) {
			stage_tile(smem + L::kKeys, a.buf.keysIn + (size_t)t0 * TILE, kTileBytes,
				&sBar[0]);
			if constexpr(NV >= 1)
				stage_tile(sVals, a.buf.valsIn[0] + (size_t)t0 * TILE, kTileBytes, &sBar[2]);
		}
	}
	for(int i = tid; i < NW * kDigitBins; i += NT) sWarpHist[i] = 0;
	__syncthreads();

	const unsigned mask = (1u << a.width) - 1;
	const int shift = a.shift;
	const unsigned ltMask = lanemask_lt();
	unsigned nClear[4];
#pragma unroll
	for(int k = 0; k < 4; ++k) nClear[k] = ((lane >> k) & 1) ? 0u : 0xffffffffu;
	unsigned phase = 0;    // bit s: key slot s; bit 2: value buffer; bit 3: stream
	int slot = 0;

	for(int tile = t0; tile < t1; ++tile) {
		unsigned* sKeys = smem + L::kKeys + slot * TILE;
		const long long tileStart = (long long)tile * TILE;
		const int count = (int)min((long long)TILE, (long long)a.n - tileStart);
		const bool bulk = tile_is_bulk(tile);
		const int next = tile + 1;

		// The next tile's keys go into the other slot (free since the end of
		// the previous iteration) while this one is sorted.
		if(KSLOTS == 2 && tid == 0 && next < t1 && tile_is_bulk(next)) {
			fence_proxy_async_smem();
			stage_tile(smem + L::kKeys + (slot ^ 1) * TILE,
				a.buf.keysIn + (size_t)next * TILE, kTileBytes, &sBar[slot ^ 1]);
		}

		unsigned* myHist = sWarpHist + warp * kDigitBins;
		unsigned rank[IPT];
		if(bulk) {
			if(!mbar_wait_bounded(&sBar[slot], (phase >> slot) & 1u))
				report_error(a.devError, a.hostError, kErrBarrierTimeout);
			phase ^= 1u << slot;
			rank_tile<IPT, true>(sKeys, myHist, warpBase, lane, count, shift, mask,
				ltMask, nClear, rank);
		} else {
			// Plain loads (a partial tile, or buffers that are not 16-byte
			// aligned): stage the keys and the first value array by hand.
			for(int i = tid; i < TILE; i += NT) {
				sKeys[i] = i < count ? a.buf.keysIn[tileStart + i] : 0xffffffffu;
				if constexpr(NV >= 1)
					sVals[i] = i < count ? a.buf.valsIn[0][tileStart + i] : 0u;
			}
			__syncthreads();
			rank_tile<IPT, false>(sKeys, myHist, warpBase, lane, count, shift, mask,
				ltMask, nClear, rank);
		}
		__syncthreads();

		// Per digit: the tile's count, its exclusive digit start, and for every
		// warp the position where its run of the digit begins in the reordered
		// tile (digit start + counts of the warps before it).
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
			const unsigned digStart = prefix + incl - tileTotal;
			unsigned run = digStart;
#pragma unroll
			for(int w = 0; w < NW; ++w) {
				sWarpHist[w * kDigitBins + tid] = run;
				run += c[w];
			}
			// Global position of element p of digit tid's run: scatter + p.
			// Padding is only ever in digit 255 and is not counted.
			const unsigned mine = tileTotal - (tid == kDigitBins - 1 ? TILE - count : 0);
			const unsigned g = sRunning[tid];
			sScatter[tid] = (int)(g - digStart);
			sRunning[tid] = g + mine;
		}

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
		if constexpr(VM == kValueIndex) {
#pragma unroll
			for(int i = 0; i < IPT; ++i)
				sVals[rank[i]] = (unsigned)(tileStart + warpBase + i * 32 + lane);
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
		if constexpr(NV >= 2) {
			// The second value array heads for the stream buffer now.
			if(bulk && tid == 0) {
				fence_proxy_async_smem();
				stage_tile(sStream, a.buf.valsIn[1] + tileStart, kTileBytes, &sBar[3]);
			}
		}
		if(tile == a.failTile && tid == 0) {
			// Injected fault (tests only): wait on a barrier that nothing
			// completes, so the bounded wait runs out and is reported.
			if(!mbar_wait_bounded(&sBar[5], 0))
				report_error(a.devError, a.hostError, kErrInjected);
		}
		__syncthreads();

		// Write each run to its global position: element p of the reordered
		// tile goes to scatter[digit] + p; consecutive p, consecutive addresses.
		if(count == TILE) {
#pragma unroll
			for(int j = 0; j < IPT; ++j) {
				const int p = j * NT + tid;
				const unsigned k = sKeys[p];
				const int dst = sScatter[(k >> shift) & mask] + p;
				a.buf.keysOut[dst] = k;
				if constexpr(VM != 0) a.buf.valsOut[0][dst] = sVals[p];
			}
		} else {
#pragma unroll
			for(int j = 0; j < IPT; ++j) {
				const int p = j * NT + tid;
				if(p < count) {
					const unsigned k = sKeys[p];
					const int dst = sScatter[(k >> shift) & mask] + p;
					a.buf.keysOut[dst] = k;
					if constexpr(VM != 0) a.buf.valsOut[0][dst] = sVals[p];
				}
			}
		}

		// Value arrays 2..V: array v arrives in the stream buffer (requested
		// while array v - 1 was reordered), is read out, array v + 1 is
		// requested into the stream buffer, and array v is reordered in the
		// value buffer and stored.
#pragma unroll
		for(int v = 1; v < NV; ++v) {
			unsigned vals[IPT];
			if(bulk) {
				if(!mbar_wait_bounded(&sBar[3], (phase >> 3) & 1u))
					report_error(a.devError, a.hostError, kErrBarrierTimeout);
				phase ^= 1u << 3;
#pragma unroll
				for(int i = 0; i < IPT; ++i) vals[i] = sStream[warpBase + i * 32 + lane];
			} else {
#pragma unroll
				for(int i = 0; i < IPT; ++i) {
					const int idx = warpBase + i * 32 + lane;
					vals[i] = idx < count ? a.buf.valsIn[v][tileStart + idx] : 0u;
				}
			}
			// Everyone has read the stream buffer and finished the stores
			// that read the value buffer.
			__syncthreads();
			if(bulk && tid == 0 && v + 1 < NV) {
				fence_proxy_async_smem();
				stage_tile(sStream, a.buf.valsIn[v + 1] + tileStart, kTileBytes, &sBar[3]);
			}
#pragma unroll
			for(int i = 0; i < IPT; ++i) sVals[rank[i]] = vals[i];
			__syncthreads();
#pragma unroll
			for(int j = 0; j < IPT; ++j) {
				const int p = j * NT + tid;
				if(p < count) {
					const int dst = sScatter[(sKeys[p] >> shift) & mask] + p;
					a.buf.valsOut[v][dst] = sVals[p];
				}
			}
		}

		for(int i = tid; i < NW * kDigitBins; i += NT) sWarpHist[i] = 0;
		__syncthreads();

		// This tile's buffers are free: request the next tile's first value
		// array, and with one key slot its keys.
		if(tid == 0 && next < t1 && tile_is_bulk(next)) {
			fence_proxy_async_smem();
			if(KSLOTS == 1)
				stage_tile(sKeys, a.buf.keysIn + (size_t)next * TILE, kTileBytes, &sBar[0]);
			if constexpr(NV >= 1)
				stage_tile(sVals, a.buf.valsIn[0] + (size_t)next * TILE, kTileBytes,
					&sBar[2]);
		}
		slot = KSLOTS == 2 ? slot ^ 1 : 0;
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
static cudaError_t set_sort_attributes() {
	return cudaFuncSetAttribute(sort_kernel<VM>,
		cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SortLayout<VM>::kBytes);
}

cudaError_t configure_kernels() {
	cudaError_t e = cudaSuccess;
	cudaError_t r;
	if((r = set_sort_attributes<-1>()) != cudaSuccess) e = r;
	if((r = set_sort_attributes<0>()) != cudaSuccess) e = r;
	if((r = set_sort_attributes<1>()) != cudaSuccess) e = r;
	if((r = set_sort_attributes<2>()) != cudaSuccess) e = r;
	if((r = set_sort_attributes<3>()) != cudaSuccess) e = r;
	if((r = set_sort_attributes<4>()) != cudaSuccess) e = r;
	if((r = set_sort_attributes<5>()) != cudaSuccess) e = r;
	if((r = set_sort_attributes<6>()) != cudaSuccess) e = r;
	return e;
}

int pass_tile_elements(int valueMode) {
	(void)valueMode;
	return kTileElements;
}

size_t pass_scratch_bytes() {
	return sizeof(unsigned) * kPassScratchWords;
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

// CTAs of the sort kernel that fit on one SM (occupancy), once per mode.
template<int VM>
static int sort_ctas_per_sm() {
	static int perSM = 0;
	if(!perSM) {
		int v = 0;
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, sort_kernel<VM>,
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

static RangeSplit split_for_mode(int valueMode, int n, int numSMs) {
	switch(valueMode) {
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
	const RangeSplit split = split_for_mode(valueMode, n, numSMs);
	unsigned* rangeCounts = scratch;
	CountArgs c;
	c.keys = buf.keysIn;
	c.n = n;
	c.shift = plan.shift[pass];
	c.width = plan.width[pass];
	c.vecOk = (reinterpret_cast<size_t>(buf.keysIn) & 15) == 0;
	c.split = split;
	c.rangeCounts = rangeCounts;
	count_kernel<<<split.numRanges, kCountThreads, 0, stream>>>(c);

	ScanArgs s;
	s.rangeCounts = rangeCounts;
	s.rangeOffsets = scratch + (size_t)kDigitBins * kMaxRanges;
	s.totals = scratch + 2 * (size_t)kDigitBins * kMaxRanges;
	s.numRanges = split.numRanges;
	scan_kernel<<<kDigitBins / 8, 256, 0, stream>>>(s);
	return cudaGetLastError();
}

template<int VM>
static void launch_sort_vm(const SortArgs& a, cudaStream_t stream) {
	using L = SortLayout<VM>;
	sort_kernel<VM><<<a.split.numRanges, L::NT, L::kBytes, stream>>>(a);
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
	a.split = split_for_mode(valueMode, n, numSMs);
	a.n = n;
	a.shift = plan.shift[pass];
	a.width = plan.width[pass];
	a.useBulk = useBulk ? 1 : 0;
	a.failTile = failTile;
	switch(valueMode) {
		case -1: launch_sort_vm<-1>(a, stream); break;
		case 0: launch_sort_vm<0>(a, stream); break;
		case 1: launch_sort_vm<1>(a, stream); break;
		case 2: launch_sort_vm<2>(a, stream); break;
		case 3: launch_sort_vm<3>(a, stream); break;
		case 4: launch_sort_vm<4>(a, stream); break;
		case 5: launch_sort_vm<5>(a, stream); break;
		case 6: launch_sort_vm<6>(a, stream); break;
		default: return cudaErrorInvalidValue;
	}
	return cudaGetLastError();
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

cudaError_t launch_iota(unsigned* out, int n, cudaStream_t stream) {
	if(n <= 0) return cudaSuccess;
	int grid = (int)std::min<long long>(((long long)n + 255) / 256, 4096);
	iota_kernel<<<grid, 256, 0, stream>>>(out, n);
	return cudaGetLastError();
}

} // namespace mgpusort
