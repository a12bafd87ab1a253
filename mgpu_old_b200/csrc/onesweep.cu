// Onesweep radix sort passes for sm_100a: one launch per digit pass.
//
// A sort runs one upsweep launch, which reads the keys once and builds the
// digit histogram of every pass and its exclusive scan (the global start of
// every digit in every pass), and then one launch per pass. Each CTA of a
// pass sorts one tile, which it draws from a counter in launch order:
//
//   1. bulk-copy the tile's keys (and values) into shared memory;
//   2. count the tile's digits, per warp, into shared memory;
//   3. publish the tile's digit counts to the pass's lookback buffer (tile 0
//      publishes them as inclusive prefixes at once);
//   4. rank every key stably within the tile (warp peers by ballots and
//      match.any, warp counters pre-offset by the tile's digit starts, so a
//      rank is the key's position in the tile sorted by digit);
//   5. decoupled lookback: for each digit, walk back over the predecessors'
//      published words, a window at a time, summing digit counts until a
//      tile that published its inclusive prefix; publish this tile's own
//      inclusive prefix;
//   6. reorder keys and values into digit runs in shared memory and store
//      each run at the digit's global start + the count of that digit in
//      earlier tiles.
//
// No key is read twice per pass and no tile waits for anything but the
// published words of tiles drawn before it, which are held by CTAs that are
// already running. Every wait is bounded (sort_device.cuh: WaitBudget).
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

namespace {

// A lookback word of (tile, digit), 64 bits: 0 until the tile publishes it,
// then a flag (bits 62-63: 1 aggregate, 2 inclusive prefix), a span (bits
// 32-61) and a count (bits 0-31). An aggregate with span s is the digit's
// count over tiles [tile - s + 1, tile]; an inclusive prefix is its count
// over tiles [0, tile]. A tile first publishes its own count (span 1), widens
// its aggregate as its lookback walks back over its predecessors, and ends
// with its inclusive prefix, so a later walker jumps over every tile an
// earlier one has already summed.
constexpr unsigned long long kLbAggregate = 1ull << 62;
constexpr unsigned long long kLbInclusive = 2ull << 62;

__device__ __forceinline__ unsigned long long lookback_word(unsigned count, unsigned span,
	bool inclusive) {
	return (inclusive ? kLbInclusive : kLbAggregate) | ((unsigned long long)span << 32) | count;
}

__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
	asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" :: "l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
	unsigned long long v;
	asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
	return v;
}

} // namespace

// Tile shapes of the onesweep kernels per value mode (tile_config.h).
template<int VM> struct OsConfig {
	// Ranking threads (the block has one more warp, for the lookback).
	static constexpr int kThreads = VM >= 2 ? MGPU_OS_MULTI_THREADS
		: VM == 0 ? MGPU_OS_KEYS_THREADS : MGPU_OS_SINGLE_THREADS;
	static constexpr int kItems = VM >= 2 ? MGPU_OS_MULTI_ITEMS
		: VM == 0 ? MGPU_OS_KEYS_ITEMS : MGPU_OS_SINGLE_ITEMS;
	static constexpr int kMinBlocks = VM >= 2 ? MGPU_OS_MULTI_MIN_BLOCKS
		: VM == 0 ? MGPU_OS_KEYS_MIN_BLOCKS : MGPU_OS_SINGLE_MIN_BLOCKS;
	static constexpr int kBallotBits = VM >= 2 ? MGPU_OS_MULTI_BALLOT_BITS
		: VM == 0 ? MGPU_OS_KEYS_BALLOT_BITS : MGPU_OS_SINGLE_BALLOT_BITS;
	static constexpr int kRankBatch = VM >= 2 ? MGPU_OS_MULTI_RANK_BATCH
		: VM == 0 ? MGPU_OS_KEYS_RANK_BATCH : MGPU_OS_SINGLE_RANK_BATCH;
	// Staging slots: with two, a CTA copies its next tile in while it
	// reorders and stores the current one. Several value arrays take one.
	static constexpr int kSlots = VM >= 2 ? 1 : VM == 0 ? MGPU_OS_KEYS_SLOTS
		: MGPU_OS_SINGLE_SLOTS;
};

template<int VM> struct OsLayout {
	static constexpr int NTR = OsConfig<VM>::kThreads;     // ranking threads
	static constexpr int NT = NTR + 32;                     // + the lookback warp
	static constexpr int LBW = NTR / 32;                    // its warp index
	static constexpr int IPT = OsConfig<VM>::kItems;
	static constexpr int TILE = NTR * IPT;
	static constexpr int NW = NTR / 32;                     // ranking warps
	static constexpr int NV = VM > 0 ? VM : 0;
	static constexpr int SLOTS = OsConfig<VM>::kSlots;
	// Per slot: the keys, then keys only: nothing; index mode or one value
	// array: one buffer, reordered in place; two or more: source positions
	// and one staging buffer per value array.
	static constexpr int NVBUF = VM == 0 ? 0 : (NV >= 2 ? 1 + NV : 1);
	static constexpr int kSlotWords = (1 + NVBUF) * TILE;
	// Word offsets into dynamic shared memory.
	static constexpr int kSlot0 = 0;
	static constexpr int kHist = SLOTS * kSlotWords;        // [NW][256]
	static constexpr int kOfs = kHist + NW * kDigitBins;    // [256] global offset - tile start
	static constexpr int kReal = kOfs + kDigitBins;         // [256] the tile's digit counts
	static constexpr int kStart = kReal + kDigitBins;       // [256] digit starts in the tile
	static constexpr int kScan = kStart + kDigitBins;       // [32]
	static constexpr int kTile = kScan + 32;                // [2] drawn tiles
	static constexpr int kBar = kTile + 2;                  // 8-byte aligned
	static constexpr int kNumBars = 8;                      // keys, 6 value arrays, fault
	static constexpr int kFaultBar = 7;
	static constexpr int kWords = kBar + 2 * kNumBars * SLOTS;
	static constexpr size_t kBytes = sizeof(unsigned) * kWords;
	static_assert(kBar % 2 == 0, "mbarriers need 8-byte alignment");
	static_assert(NTR >= kDigitBins && NTR % 32 == 0, "one ranking thread per digit");
	static_assert(TILE % 4 == 0, "tiles start on 16-byte boundaries");
	static_assert(TILE <= 65536, "ranks are packed in 16 bits");
	static_assert(kBytes <= 227 * 1024, "shared memory of one CTA");
};

struct OsArgs {
	PassBuffers buf;
	const unsigned* digitStart;     // [256] the pass's exclusive digit offsets
	const unsigned* trivial;        // the pass has a single digit: copy
	unsigned long long* status;     // [tiles][256] this pass's lookback words
	unsigned long long* statusNext; // the next executed pass's, cleared here
	unsigned* tileCounter;
	unsigned* devError;
	volatile unsigned* hostError;
	int n;
	int numTiles;
	int shift;
	int width;
	int useBulk;
	int failTile;
};

// Stable rank of a warp's items within the tile. myHist[d] holds, for this
// warp, the tile position of its next key with digit d (the digit's start in
// the tile plus the counts of earlier warps). Items are taken CH at a time:
// the peers of all CH are found first (independent match steps), then the
// counter updates run in item order; the lowest peer of a group advances the
// counter by the group's size.
// Ranks are below 2^16 and kept two to a register: item i's rank is the
// halfword i & 1 of rank[i / 2].
template<int IPT> struct PackedRanks {
	unsigned r[(IPT + 1) / 2];
	__device__ __forceinline__ void set(int i, unsigned v) {
		if(i & 1) r[i >> 1] |= v << 16;
		else r[i >> 1] = v;
	}
	__device__ __forceinline__ unsigned get(int i) const {
		return (i & 1) ? r[i >> 1] >> 16 : r[i >> 1] & 0xffffu;
	}
};

template<int IPT, int BB, int CH, bool BYTE>
__device__ __forceinline__ void os_rank(const unsigned (&keys)[IPT], const DigitOf<BYTE>& digit,
	unsigned* myHist, unsigned ltMask, const unsigned (&nClear)[4], PackedRanks<IPT>& rank) {
#pragma unroll
	for(int c = 0; c < IPT; c += CH) {
		unsigned d[CH], peers[CH];
#pragma unroll
		for(int j = 0; j < CH; ++j) {
			if(c + j < IPT) {
				d[j] = digit(keys[c + j]);
				peers[j] = match_digit8<BB>(d[j], nClear);
			}
		}
#pragma unroll
		for(int j = 0; j < CH; ++j) {
			if(c + j < IPT) {
				const unsigned below = __popc(peers[j] & ltMask);
				const unsigned base = myHist[d[j]];
				__syncwarp();
				if(!below) myHist[d[j]] = base + __popc(peers[j]);
				__syncwarp();
				rank.set(c + j, base + below);
			}
		}
	}
}

// The lookback warp of a tile: lane l finds, for digits l, l + 32, ...,
// l + 224 (those of the pass), the digit's count over tiles [0, tile). The
// walks of four digits run in lockstep, so that their loads are in flight
// together. A walk reads its predecessor's word, adds its count and either
// stops (an inclusive prefix) or jumps back over the word's span; after every
// jump the tile widens its own aggregate. A word not yet published is polled
// again (bounded: on time-out the error is reported and the walk ends). Then
// the tile's inclusive prefixes are published and the global offsets of its
// digits written to ofs.
constexpr int kLbGroup = 4;

__device__ __forceinline__ void os_lookback_warp(const OsArgs& a, int tile, unsigned bins,
	const unsigned* sReal, const unsigned* sStart, int* sOfs) {
	const int lane = threadIdx.x & 31;
	unsigned long long* row = a.status + (size_t)tile * kDigitBins;
#pragma unroll 1
	for(int g = 0; g < 8; g += kLbGroup) {
		int j[kLbGroup];
		unsigned excl[kLbGroup];
		unsigned pending = 0;
#pragma unroll
		for(int k = 0; k < kLbGroup; ++k) {
			j[k] = tile - 1;
			excl[k] = 0;
			if(tile > 0 && lane + 32 * (g + k) < (int)bins) pending |= 1u << k;
		}
		WaitBudget budget;
		while(__any_sync(0xffffffffu, pending != 0)) {
			unsigned long long w[kLbGroup];
#pragma unroll
			for(int k = 0; k < kLbGroup; ++k)
				w[k] = (pending >> k) & 1u ? ld_relaxed_u64(
					a.status + (size_t)j[k] * kDigitBins + lane + 32 * (g + k)) : 0ull;
			bool progress = false;
#pragma unroll
			for(int k = 0; k < kLbGroup; ++k) {
				if(((pending >> k) & 1u) && w[k]) {
					const int d = lane + 32 * (g + k);
					progress = true;
					excl[k] += (unsigned)w[k];
					if(w[k] & kLbInclusive) {
						pending &= ~(1u << k);
					} else {
						j[k] -= (int)((w[k] >> 32) & 0x3fffffffu);
						st_relaxed_u64(row + d, lookback_word(excl[k] + sReal[d],
							(unsigned)(tile - j[k]), false));
					}
				}
			}
			if(pending && !progress && !budget.poll()) {
				report_error(a.devError, a.hostError, kErrBarrierTimeout);
				pending = 0;
			}
		}
#pragma unroll
		for(int k = 0; k < kLbGroup; ++k) {
			const int d = lane + 32 * (g + k);
			if(d < (int)bins) {
				if(tile > 0) st_relaxed_u64(row + d, lookback_word(excl[k] + sReal[d], 0, true));
				sOfs[d] = (int)(a.digitStart[d] + excl[k] - sStart[d]);
			}
		}
	}
}

// Barrier of the ranking warps only (named barrier 1; the lookback warp
// does not take part).
template<int NTR>
__device__ __forceinline__ void bar_sync_rankers() {
	asm volatile("bar.sync 1, %0;" :: "n"(NTR) : "memory");
}

// Identity pass (a single digit): the tile's keys and values move unchanged
// (index mode: their positions).
template<int VM>
__device__ __forceinline__ void os_copy_tile(const OsArgs& a, long long start, int count) {
	using L = OsLayout<VM>;
	for(int i = threadIdx.x; i < count; i += L::NT) {
		const long long e = start + i;
		a.buf.keysOut[e] = a.buf.keysIn[e];
		if constexpr(VM == kValueIndex) a.buf.valsOut[0][e] = (unsigned)e;
#pragma unroll
		for(int v = 0; v < L::NV; ++v) a.buf.valsOut[v][e] = a.buf.valsIn[v][e];
	}
}

// The bulk copies of one tile into a slot's buffers (one thread): keys and
// every value array, each completing on its own mbarrier of the slot.
template<int VM>
__device__ __forceinline__ void os_stage(const OsArgs& a, unsigned* slot, uint64_t* bars,
	long long tileStart) {
	using L = OsLayout<VM>;
	constexpr unsigned kTileBytes = L::TILE * 4;
	fence_proxy_async_smem();
	stage_tile(slot, a.buf.keysIn + tileStart, kTileBytes, &bars[0]);
	if constexpr(L::NV == 1)
		stage_tile(slot + L::TILE, a.buf.valsIn[0] + tileStart, kTileBytes, &bars[1]);
	if constexpr(L::NV >= 2) {
#pragma unroll
		for(int v = 0; v < L::NV; ++v)
			stage_tile(slot + (2 + v) * L::TILE, a.buf.valsIn[v] + tileStart, kTileBytes,
				&bars[1 + v]);
	}
}

// Persistent CTAs: each draws tiles from the pass's counter, in order, until
// none are left, and sorts them one at a time. Ranking warps count and rank
// the keys while the lookback warp walks back for the tile's digit offsets.
// With two staging slots the next tile is drawn, and its bulk copies issued,
// as soon as this tile's inclusive prefixes are out: they land while this
// tile is reordered and stored. A tile waits only on tiles drawn before it,
// whose CTAs publish their counts without waiting on anything, so the pass
// cannot deadlock.
template<int VM, bool BYTE, int BB>
__global__ void __launch_bounds__(OsLayout<VM>::NT, OsConfig<VM>::kMinBlocks)
onesweep_kernel(const OsArgs a) {
	using L = OsLayout<VM>;
	constexpr int NT = L::NT;
	constexpr int NTR = L::NTR;
	constexpr int IPT = L::IPT;
	constexpr int TILE = L::TILE;
	constexpr int NW = L::NW;
	constexpr int NV = L::NV;
	constexpr int SLOTS = L::SLOTS;
	constexpr int CH = OsConfig<VM>::kRankBatch;
	extern __shared__ __align__(128) unsigned smem[];
	unsigned* sHist = smem + L::kHist;
	int* sOfs = reinterpret_cast<int*>(smem + L::kOfs);
	unsigned* sReal = smem + L::kReal;
	unsigned* sStart = smem + L::kStart;
	unsigned* sScan = smem + L::kScan;
	unsigned* sTile = smem + L::kTile;
	uint64_t* sBar = reinterpret_cast<uint64_t*>(smem + L::kBar);

	const int tid = threadIdx.x;
	const int lane = tid & 31;
	const int warp = tid >> 5;
	const bool ranker = warp < NW;
	const int warpBase = warp * 32 * IPT;

	auto tile_bulk = [&](int t) {
		return a.useBulk && (long long)(t + 1) * TILE <= (long long)a.n;
	};
	// The next tile into slot s (one thread).
	auto draw_next = [&](int s) {
		const int t = (int)atomicAdd(a.tileCounter, 1u);
		sTile[s] = t;
		if(t < a.numTiles && tile_bulk(t))
			os_stage<VM>(a, smem + L::kSlot0 + s * L::kSlotWords, sBar + s * L::kNumBars,
				(long long)t * TILE);
	};

	// Shared-memory set-up touches no global memory: it overlaps the previous
	// launch's tail.
	for(int i = tid; i < NW * kDigitBins; i += NT) sHist[i] = 0;
	if(tid == 0) {
		for(int b = 0; b < L::kNumBars * SLOTS; ++b) mbar_init(&sBar[b], 1);
		fence_mbar_init();
	}
	wait_for_predecessor();
	const bool trivial = *a.trivial != 0;
	if(tid == 0) {
		if(trivial) sTile[0] = atomicAdd(a.tileCounter, 1u);
		else draw_next(0);
	}
	__syncthreads();

	if(trivial) {
		for(int t = (int)sTile[0]; t < a.numTiles;) {
			const long long start = (long long)t * TILE;
			if(tid < kDigitBins && a.statusNext)
				a.statusNext[(size_t)t * kDigitBins + tid] = 0;
			os_copy_tile<VM>(a, start, (int)min((long long)TILE, (long long)a.n - start));
			__syncthreads();
			if(tid == 0) sTile[0] = atomicAdd(a.tileCounter, 1u);
			__syncthreads();
			t = (int)sTile[0];
		}
		return;
	}

	const DigitOf<BYTE> digit(a.shift, a.width);
	const unsigned bins = 1u << a.width;
	const unsigned padDigit = bins - 1;
	const unsigned ltMask = lanemask_lt();
	unsigned nClear[4];
#pragma unroll
	for(int k = 0; k < 4; ++k) nClear[k] = ((lane >> k) & 1) ? 0u : 0xffffffffu;
	unsigned* myHist = sHist + (ranker ? warp : 0) * kDigitBins;

	int slot = 0;
	unsigned phase = 0;        // bit s: parity of slot s's barriers
	for(;;) {
		const int tile = (int)sTile[slot];
		if(tile >= a.numTiles) break;
		unsigned* sKeys = smem + L::kSlot0 + slot * L::kSlotWords;
		unsigned* sVals = sKeys + TILE;
		uint64_t* bars = sBar + slot * L::kNumBars;
		const long long tileStart = (long long)tile * TILE;
		const int count = (int)min((long long)TILE, (long long)a.n - tileStart);
		const bool bulk = tile_bulk(tile);
		const unsigned par = (phase >> slot) & 1u;

		if(tid < kDigitBins && a.statusNext)
			a.statusNext[(size_t)tile * kDigitBins + tid] = 0;
		if(!bulk) {
			// A partial tile, or buffers that are not 16-byte aligned: plain
			// loads. Positions past the end hold 0xffffffff, whose digit is the
			// largest, so they rank after every real key and are never stored.
			for(int i = tid; i < TILE; i += NT) {
				sKeys[i] = i < count ? a.buf.keysIn[tileStart + i] : 0xffffffffu;
				if constexpr(NV == 1) sVals[i] = i < count ? a.buf.valsIn[0][tileStart + i] : 0u;
			}
			__syncthreads();
		}

		// Keys to registers (warp-striped: item i of lane l of warp w is tile
		// element w*32*IPT + i*32 + l, so (item, lane) order is input order);
		// each warp counts its digits.
		unsigned keys[IPT];
		if(ranker) {
			if(bulk && !mbar_wait_bounded(&bars[0], par))
				report_error(a.devError, a.hostError, kErrBarrierTimeout);
#pragma unroll
			for(int i = 0; i < IPT; ++i) {
				keys[i] = sKeys[warpBase + i * 32 + lane];
				atomicAdd(&myHist[digit(keys[i])], 1u);
			}
		}
		__syncthreads();

		// Per digit: the tile's count, published at once (tile 0: as its
		// inclusive prefix); the digit's start in the tile (scan over
		// digits); each warp's first position.
		unsigned total = 0;
		unsigned c[NW];
		if(tid < kDigitBins) {
#pragma unroll
			for(int w = 0; w < NW; ++w) {
				c[w] = sHist[w * kDigitBins + tid];
				total += c[w];
			}
			const unsigned real = total - (tid == (int)padDigit ? (unsigned)(TILE - count) : 0u);
			sReal[tid] = real;
			if(tid < (int)bins)
				st_relaxed_u64(a.status + (size_t)tile * kDigitBins + tid,
					lookback_word(real, 1, tile == 0));
		}
		const unsigned incl = warp_inclusive_scan(total, lane);
		if(lane == 31 && warp < kDigitBins / 32) sScan[warp] = incl;
		__syncthreads();
		if(tid < kDigitBins) {
			unsigned prefix = 0;
#pragma unroll
			for(int w = 0; w < kDigitBins / 32; ++w)
				if(w < warp) prefix += sScan[w];
			const unsigned start = prefix + incl - total;
			sStart[tid] = start;
			unsigned run = start;
#pragma unroll
			for(int w = 0; w < NW; ++w) {
				sHist[w * kDigitBins + tid] = run;
				run += c[w];
			}
		}
		__syncthreads();

		PackedRanks<IPT> rank;
		if(ranker) {
			os_rank<IPT, BB, CH, BYTE>(keys, digit, myHist, ltMask, nClear, rank);
		} else {
			os_lookback_warp(a, tile, bins, sReal, sStart, sOfs);
			if(a.failTile == tile && lane == 0) {
				// Injected fault (tests only): wait on a barrier that nothing
				// completes, so the bounded wait runs out and is reported.
				if(!mbar_wait_bounded(&sBar[L::kFaultBar], 0))
					report_error(a.devError, a.hostError, kErrInjected);
			}
			// The next tile: drawn now, its copies into the other slot (free:
			// its tile was stored in the previous iteration).
			if(SLOTS == 2 && lane == 0) draw_next(slot ^ 1);
		}
		__syncthreads();

		// Reorder into digit runs in shared memory; the warp counters are free
		// again. One value array is reordered in place after the keys: read
		// into registers, a barrier, written.
		if(ranker) {
#pragma unroll
			for(int i = 0; i < IPT; ++i) sKeys[rank.get(i)] = keys[i];
			if constexpr(VM == kValueIndex) {
#pragma unroll
				for(int i = 0; i < IPT; ++i)
					sVals[rank.get(i)] = (unsigned)(tileStart + warpBase + i * 32 + lane);
			} else if constexpr(NV == 1) {
				if(bulk && !mbar_wait_bounded(&bars[1], par))
					report_error(a.devError, a.hostError, kErrBarrierTimeout);
				unsigned vals[IPT];
#pragma unroll
				for(int i = 0; i < IPT; ++i) vals[i] = sVals[warpBase + i * 32 + lane];
				bar_sync_rankers<NTR>();
#pragma unroll
				for(int i = 0; i < IPT; ++i) sVals[rank.get(i)] = vals[i];
			} else if constexpr(NV >= 2) {
				unsigned* sPos = sVals;
#pragma unroll
				for(int i = 0; i < IPT; ++i)
					sPos[rank.get(i)] = (unsigned)(warpBase + i * 32 + lane);
			}
		}
		for(int i = tid; i < NW * kDigitBins; i += NT) sHist[i] = 0;
		__syncthreads();

		if(ranker) {
			if constexpr(NV <= 1) {
				// Element p of the reordered tile goes to ofs[digit] + p:
				// consecutive p, consecutive addresses within a run.
#pragma unroll
				for(int j = 0; j < IPT; ++j) {
					const int p = j * NTR + tid;
					if(count == TILE || p < count) {
						const unsigned k = sKeys[p];
						const int dst = sOfs[digit(k)] + p;
						a.buf.keysOut[dst] = k;
						if constexpr(VM != 0) a.buf.valsOut[0][dst] = sVals[p];
					}
				}
			} else {
				// Several value arrays: each thread keeps its destinations and
				// source positions; every array is written from its own staging
				// buffer (or gathered from global memory on the plain-load path).
				const unsigned* sPos = sVals;
				int dst[IPT];
				unsigned src[IPT];
#pragma unroll
				for(int j = 0; j < IPT; ++j) {
					const int p = j * NTR + tid;
					dst[j] = -1;
					src[j] = 0;
					if(count == TILE || p < count) {
						const unsigned k = sKeys[p];
						dst[j] = sOfs[digit(k)] + p;
						src[j] = sPos[p];
						a.buf.keysOut[dst[j]] = k;
					}
				}
#pragma unroll
				for(int v = 0; v < NV; ++v) {
					if(bulk) {
						if(!mbar_wait_bounded(&bars[1 + v], par))
							report_error(a.devError, a.hostError, kErrBarrierTimeout);
						const unsigned* buf = sVals + (1 + v) * TILE;
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
			}
		}
		if(bulk) phase ^= 1u << slot;
		if constexpr(SLOTS == 1) {
			// One slot: the next tile is drawn and copied in once this one is
			// stored.
			__syncthreads();
			if(tid == 0) draw_next(0);
			__syncthreads();
		} else {
			slot ^= 1;
		}
	}
}

////////////////////////////////////////////////////////////////////////////////
// Host side.

template<int VM>
static cudaError_t set_os_attributes() {
	const int bytes = (int)OsLayout<VM>::kBytes;
	const cudaFuncAttribute attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
	constexpr int bb = OsConfig<VM>::kBallotBits;
	cudaError_t e = cudaFuncSetAttribute(onesweep_kernel<VM, false, bb>, attr, bytes);
	if(e == cudaSuccess) e = cudaFuncSetAttribute(onesweep_kernel<VM, true, bb>, attr, bytes);
	return e;
}

cudaError_t configure_onesweep_kernels() {
	cudaError_t e = cudaSuccess, r;
	if((r = set_os_attributes<-1>()) != cudaSuccess) e = r;
	if((r = set_os_attributes<0>()) != cudaSuccess) e = r;
	if((r = set_os_attributes<1>()) != cudaSuccess) e = r;
	if((r = set_os_attributes<2>()) != cudaSuccess) e = r;
	if((r = set_os_attributes<3>()) != cudaSuccess) e = r;
	if((r = set_os_attributes<4>()) != cudaSuccess) e = r;
	if((r = set_os_attributes<5>()) != cudaSuccess) e = r;
	if((r = set_os_attributes<6>()) != cudaSuccess) e = r;
	return e;
}

int onesweep_tile_elements(int valueMode) {
	switch(valueMode) {
		case -1: return OsLayout<-1>::TILE;
		case 0: return OsLayout<0>::TILE;
		case 1: return OsLayout<1>::TILE;
		default: return OsLayout<2>::TILE;
	}
}

size_t onesweep_status_bytes(int n, int valueMode) {
	const int tile = onesweep_tile_elements(valueMode);
	const size_t tiles = ((size_t)n + tile - 1) / tile;
	return tiles * kDigitBins * sizeof(unsigned long long);
}

// Resident CTAs of the onesweep kernel per SM, once per value mode.
template<int VM>
static int os_ctas_per_sm() {
	static int perSM = 0;
	if(!perSM) {
		int v = 0;
		cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v,
			onesweep_kernel<VM, true, OsConfig<VM>::kBallotBits>, OsLayout<VM>::NT,
			OsLayout<VM>::kBytes);
		perSM = v > 0 ? v : 1;
	}
	return perSM;
}

template<int VM>
static cudaError_t launch_os_vm(const OsArgs& a, int numSMs, cudaStream_t stream) {
	using L = OsLayout<VM>;
	constexpr int bb = OsConfig<VM>::kBallotBits;
	const int grid = (int)std::min<long long>(a.numTiles, (long long)numSMs * os_ctas_per_sm<VM>());
	if(a.width == 8 && (a.shift & 7) == 0)
		return launch_dependent(onesweep_kernel<VM, true, bb>, grid, L::NT, L::kBytes,
			stream, a);
	return launch_dependent(onesweep_kernel<VM, false, bb>, grid, L::NT, L::kBytes,
		stream, a);
}

cudaError_t launch_onesweep_pass(const PassBuffers& buf, int valueMode, int n,
	int pass, int exec, const PassPlan& plan, Control* ctrl, void* const status[2],
	bool useBulk, int failTile, volatile unsigned* hostError, int numSMs,
	cudaStream_t stream) {
	if(n <= 0) return cudaSuccess;
	OsArgs a;
	a.buf = buf;
	a.digitStart = ctrl->offsets + plan.binBase[pass];
	a.trivial = ctrl->trivial + pass;
	a.status = static_cast<unsigned long long*>(status[exec & 1]);
	a.statusNext = static_cast<unsigned long long*>(status[(exec + 1) & 1]);
	a.tileCounter = ctrl->tileCounter + exec;
	a.devError = &ctrl->error;
	a.hostError = hostError;
	a.n = n;
	a.numTiles = (int)(((long long)n + onesweep_tile_elements(valueMode) - 1)
		/ onesweep_tile_elements(valueMode));
	a.shift = plan.shift[pass];
	a.width = plan.width[pass];
	a.useBulk = useBulk ? 1 : 0;
	a.failTile = failTile;
	switch(valueMode) {
		case -1: return launch_os_vm<-1>(a, numSMs, stream);
		case 0: return launch_os_vm<0>(a, numSMs, stream);
		case 1: return launch_os_vm<1>(a, numSMs, stream);
		case 2: return launch_os_vm<2>(a, numSMs, stream);
		case 3: return launch_os_vm<3>(a, numSMs, stream);
		case 4: return launch_os_vm<4>(a, numSMs, stream);
		case 5: return launch_os_vm<5>(a, numSMs, stream);
		case 6: return launch_os_vm<6>(a, numSMs, stream);
		default: return cudaErrorInvalidValue;
	}
}

} // namespace mgpusort
