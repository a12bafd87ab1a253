// CPU oracle for the sortArray path. TEST INFRASTRUCTURE ONLY: the tests,
// the smoke check and bench.py's CPU-baseline leg call it as the checker (and
// to time the CPU path); the library never does.
//
// It restates what Modern GPU's sortArray computes, two independent ways:
//
//  * oracle_sort_stable: std::stable_sort of element positions by the bit
//    field (key >> firstBit) & mask(endBit - firstBit). This is the result
//    that every pass of the reference's LSD loop (sort/src/mgpusort/
//    mgpusort.cpp:560-601) composes to, because each pass is a stable
//    partition by its digit. Values move with their keys as 32-bit
//    patterns; valueCount -1 writes each key's source position into the
//    first value array (index mode, sort/src/kernels/sort.cu:306-313,
//    mgpusort.cpp:553).
//
//  * oracle_sort_lsd: the reference CPU radix sort of
//    sort/src/cpusort/cpusort.cpp:122-186 (Sort2Pass: per-block digit count,
//    reduction into global digit counts, exclusive scan, per-block exclusive
//    offsets, per-block scatter), generalised from keys-only 4-bit passes
//    over 32 bits to any pass widths over [firstBit, endBit) with value
//    arrays, and with the per-block phases spread over host threads. It is
//    also the timed CPU baseline.
//
// Both must agree with each other, with the reference's own cpusort.cpp
// built here (oracle/Makefile, `make ref`) on the keys it can sort, and with
// the GPU.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>

namespace {

inline uint32_t field_mask(int bits) {
	return bits >= 32 ? 0xffffffffu : ((1u << bits) - 1u);
}

int num_arrays(int valueCount) { return valueCount == -1 ? 1 : valueCount; }

// Runs f(t) for t in [0, threads) on host threads.
template<typename F> void parallel(int threads, F f) {
	if(threads <= 1) { f(0); return; }
	std::vector<std::thread> pool;
	pool.reserve(threads);
	for(int t = 0; t < threads; ++t) pool.emplace_back(f, t);
	for(auto& th : pool) th.join();
}

} // namespace

extern "C" {

// Stable sort of n keys (and valueCount value arrays, or index mode) by the
// bit field [firstBit, endBit). Outputs go to keysOut / valsOut[i], which
// must not alias the inputs. Returns 0, or -1 for invalid arguments.
int oracle_sort_stable(const uint32_t* keys, const uint32_t* const* vals,
	int valueCount, int n, int firstBit, int endBit, uint32_t* keysOut,
	uint32_t* const* valsOut) {
	if(n < 0 || firstBit < 0 || endBit > 32 || endBit < firstBit ||
		valueCount < -1 || valueCount > 6) return -1;
	const uint32_t mask = field_mask(endBit - firstBit);
	const int shift = firstBit >= 32 ? 0 : firstBit;
	std::vector<uint32_t> order(n);
	std::iota(order.begin(), order.end(), 0u);
	if(endBit > firstBit)
		std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
			return ((keys[a] >> shift) & mask) < ((keys[b] >> shift) & mask);
		});
	for(int i = 0; i < n; ++i) keysOut[i] = keys[order[i]];
	if(valueCount == -1) {
		for(int i = 0; i < n; ++i) valsOut[0][i] = order[i];
	} else {
		for(int v = 0; v < valueCount; ++v)
			for(int i = 0; i < n; ++i) valsOut[v][i] = vals[v][order[i]];
	}
	return 0;
}

// One LSD pass in the blocked form of cpusort.cpp:122-186, over `threads`
// host threads: count per block, reduce + scan, scatter per block.
static void lsd_pass(const uint32_t* keysIn, uint32_t* keysOut,
	const uint32_t* const* valsIn, uint32_t* const* valsOut, int numArrays,
	bool writeIndex, int n, int bit, int width, int blockSize, int threads) {
	const uint32_t buckets = 1u << width;
	const uint32_t mask = buckets - 1;
	const int numBlocks = (n + blockSize - 1) / blockSize;
	std::vector<uint32_t> counts((size_t)numBlocks * buckets, 0);

	// Per-block digit counts (cpusort.cpp:85-95, :133-138).
	parallel(threads, [&](int t) {
		for(int b = t; b < numBlocks; b += threads) {
			uint32_t* c = &counts[(size_t)b * buckets];
			const int end = std::min(n, (b + 1) * blockSize);
			for(int i = b * blockSize; i < end; ++i)
				++c[(keysIn[i] >> bit) & mask];
		}
	});

	// Global counts, their exclusive scan, then per-block exclusive offsets
	// (cpusort.cpp:144-169).
	std::vector<uint32_t> global(buckets, 0), scan(buckets, 0);
	for(int b = 0; b < numBlocks; ++b)
		for(uint32_t d = 0; d < buckets; ++d)
			global[d] += counts[(size_t)b * buckets + d];
	for(uint32_t d = 1; d < buckets; ++d) scan[d] = scan[d - 1] + global[d - 1];
	std::vector<uint32_t> running(scan);
	for(int b = 0; b < numBlocks; ++b)
		for(uint32_t d = 0; d < buckets; ++d) {
			uint32_t c = counts[(size_t)b * buckets + d];
			counts[(size_t)b * buckets + d] = running[d];
			running[d] += c;
		}

	// Per-block scatter in input order (cpusort.cpp:100-119, :176-182).
	parallel(threads, [&](int t) {
		std::vector<uint32_t> offs(buckets);
		for(int b = t; b < numBlocks; b += threads) {
			std::memcpy(offs.data(), &counts[(size_t)b * buckets],
				sizeof(uint32_t) * buckets);
			const int end = std::min(n, (b + 1) * blockSize);
			for(int i = b * blockSize; i < end; ++i) {
				const uint32_t dst = offs[(keysIn[i] >> bit) & mask]++;
				keysOut[dst] = keysIn[i];
				if(writeIndex) valsOut[0][dst] = (uint32_t)i;
				else
					for(int v = 0; v < numArrays; ++v) valsOut[v][dst] = valsIn[v][i];
			}
		}
	});
}

// LSD radix sort over [firstBit, firstBit + sum(widths)) with the given pass
// widths (least significant first), on `threads` host threads. keys and
// vals are sorted in place (scratch is allocated here). Returns 0 or -1.
int oracle_sort_lsd(uint32_t* keys, uint32_t* const* vals, int valueCount,
	int n, int firstBit, const int* widths, int numPasses, int blockSize,
	int threads) {
	if(n < 0 || firstBit < 0 || valueCount < -1 || valueCount > 6 ||
		numPasses < 0 || blockSize <= 0) return -1;
	int total = 0;
	for(int p = 0; p < numPasses; ++p) {
		if(widths[p] < 1 || widths[p] > 16) return -1;
		total += widths[p];
	}
	if(firstBit + total > 32) return -1;
	if(threads < 1) threads = 1;
	const int arrays = num_arrays(valueCount);
	const bool indexMode = valueCount == -1;

	std::vector<uint32_t> keyTmp(n);
	std::vector<std::vector<uint32_t>> valTmp(arrays, std::vector<uint32_t>(n));
	uint32_t* kA = keys;
	uint32_t* kB = keyTmp.data();
	uint32_t* vA[6] = {};
	uint32_t* vB[6] = {};
	for(int v = 0; v < arrays; ++v) { vA[v] = vals[v]; vB[v] = valTmp[v].data(); }

	int bit = firstBit;
	bool first = true;
	for(int p = 0; p < numPasses; ++p) {
		lsd_pass(kA, kB, vA, vB, arrays, indexMode && first, n, bit, widths[p],
			blockSize, threads);
		std::swap(kA, kB);
		for(int v = 0; v < arrays; ++v) std::swap(vA[v], vB[v]);
		bit += widths[p];
		first = false;
	}
	if(indexMode && first)
		for(int i = 0; i < n; ++i) vals[0][i] = (uint32_t)i;
	if(kA != keys) {
		std::memcpy(keys, kA, sizeof(uint32_t) * n);
		for(int v = 0; v < arrays; ++v)
			std::memcpy(vals[v], vA[v], sizeof(uint32_t) * n);
	}
	return 0;
}

// Batched segmented sort: every segment [offsets[i], offsets[i + 1]) sorted
// on its own exactly as oracle_sort_stable sorts one array (index mode:
// positions within the segment). This is what one sortArray call per
// segment computes. Returns 0, or -1 for invalid arguments.
int oracle_sort_segments(const uint32_t* keys, const uint32_t* const* vals,
	int valueCount, const int* offsets, int numSegments, int firstBit,
	int endBit, uint32_t* keysOut, uint32_t* const* valsOut) {
	if(numSegments < 0 || valueCount < -1 || valueCount > 6) return -1;
	const int arrays = num_arrays(valueCount);
	for(int s = 0; s < numSegments; ++s) {
		const int b = offsets[s];
		const int len = offsets[s + 1] - b;
		if(len < 0) return -1;
		const uint32_t* vin[6] = {};
		uint32_t* vout[6] = {};
		for(int v = 0; v < arrays; ++v) {
			if(valueCount > 0) vin[v] = vals[v] + b;
			vout[v] = valsOut[v] + b;
		}
		int rc = oracle_sort_stable(keys + b, vin, valueCount, len, firstBit, endBit,
			keysOut + b, vout);
		if(rc) return rc;
	}
	return 0;
}

// std::sort of keys in place: the keys-only CPU baseline of the harness
// pattern (sort/src/b40c/test/radix_sort/test_sort.cu:241).
void oracle_std_sort_keys(uint32_t* keys, int n) {
	std::sort(keys, keys + n);
}

// Number of passes, and their widths, of the reference's sortArrayEx plan
// (mgpusort.cpp:626-646): ceil(bits / bitPass) passes with `split` passes one
// bit narrower, walked narrow to wide (:574-576).
int oracle_reference_ex_plan(int numBits, int bitPass, int* widths) {
	if(numBits <= 0) return 0;
	if(bitPass <= 0 || bitPass > 6) bitPass = 6;
	if(bitPass > numBits) bitPass = numBits;
	const int passes = (numBits + bitPass - 1) / bitPass;
	const int split = passes * bitPass - numBits;
	int k = 0;
	for(int w = 1; w <= 6; ++w) {
		int count = 0;
		for(int p = 0; p < passes; ++p)
			count += (bitPass - (p < split)) == w;
		for(int j = 0; j < count; ++j) widths[k++] = w;
	}
	return passes;
}

// Burrows-Wheeler block sort of a cyclic block, what bwtSortBlock computes
// (bwt/src/mgpubwt/mgpubwt.cpp:213-371): indices[i] = start of the i-th
// smallest rotation (rotations equal as whole strings in start order),
// transform[i] = block[(indices[i] + count - 1) % count]. segCount /
// avSegSize: the groups of two or more rotations that share their first
// keySize symbols, and their mean size; blocks under 3000 bytes are sorted
// on the host by the reference and report one group of count
// (mgpubwt.cpp:180-205). Returns 0, or -1 for invalid arguments.
int oracle_bwt(const uint8_t* block, int count, int keySize, int* indices,
	uint8_t* transform, int* segCount, float* avSegSize) {
	if(count < 0 || keySize < 1 || keySize > 24) return -1;
	std::vector<uint8_t> sym(2 * (size_t)count + 1);
	if(count) {
		std::memcpy(sym.data(), block, count);
		std::memcpy(sym.data() + count, block, count);
	}
	std::vector<int> order(count);
	std::iota(order.begin(), order.end(), 0);
	std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
		return std::memcmp(sym.data() + a, sym.data() + b, count) < 0;
	});
	int groups = 0;
	long long grouped = 0;
	if(count < 3000) {
		groups = count ? 1 : 0;
		grouped = count;
	} else {
		int start = 0;
		for(int i = 1; i <= count; ++i) {
			const bool head = i == count ||
				std::memcmp(sym.data() + order[i - 1], sym.data() + order[i], keySize) != 0;
			if(!head) continue;
			if(i - start >= 2) {
				++groups;
				grouped += i - start;
			}
			start = i;
		}
	}
	for(int i = 0; i < count; ++i) {
		indices[i] = order[i];
		transform[i] = sym[(size_t)order[i] + count - 1];
	}
	*segCount = groups;
	*avSegSize = count < 3000 ? (float)count
		: (groups ? (float)((double)grouped / groups) : 0.0f);
	return 0;
}

} // extern "C"
