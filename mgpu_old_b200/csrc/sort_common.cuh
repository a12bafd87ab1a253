// Device building blocks shared by the one-array pass kernels of
// sort_kernels.cu (range partition) and onesweep.cu (decoupled lookback):
// programmatic dependent launch, tile staging, digit extraction and the warp
// peer match of the stable ranking. sm_100a only.
#pragma once

#include "sort_kernels.h"
#include "sort_device.cuh"

namespace mgpusort {

// Programmatic dependent launch: the count, scan and sort kernels of the
// passes are launched so that each may be scheduled while its predecessor
// in the stream drains. Each waits (griddepcontrol.wait) for the
// predecessor to complete, with its memory visible, before touching global
// memory. Count and scan then let their successor launch at once; the sort
// kernel releases its successor when it exits. Launched without the
// attribute (or after a non-kernel stream operation) the wait returns at
// once.
__device__ __forceinline__ void wait_for_predecessor() {
	asm volatile("griddepcontrol.wait;" ::: "memory");
}

__device__ __forceinline__ void allow_successor() {
	asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// A launch that returns its own status (cudaGetLastError after a <<<>>>
// launch would also report an earlier, unrelated failure of the thread).
template<typename... Params, typename... Args>
static cudaError_t launch_plain(void (*kernel)(Params...), int grid, int block, size_t smem,
	cudaStream_t stream, Args... args) {
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = dim3(grid);
	cfg.blockDim = dim3(block);
	cfg.dynamicSmemBytes = smem;
	cfg.stream = stream;
	return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// carveout >= 0 also sets this launch's preferred shared-memory carveout
// (percent of the L1/shared capacity).
template<typename Arg>
static cudaError_t launch_dependent(void (*kernel)(Arg), int grid, int block,
	size_t smem, cudaStream_t stream, const Arg& arg, int carveout = -1) {
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = dim3(grid);
	cfg.blockDim = dim3(block);
	cfg.dynamicSmemBytes = smem;
	cfg.stream = stream;
	cudaLaunchAttribute attr[2];
	attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
	attr[0].val.programmaticStreamSerializationAllowed = 1;
	cfg.attrs = attr;
	cfg.numAttrs = 1;
	if(carveout >= 0) {
		attr[1].id = cudaLaunchAttributePreferredSharedMemoryCarveout;
		attr[1].val.sharedMemCarveout = (unsigned)carveout;
		cfg.numAttrs = 2;
	}
	return cudaLaunchKernelEx(&cfg, kernel, arg);
}

// Peers of an 8-bit digit: the lanes of the warp whose digit equals this
// lane's. The low BB bits of the digit are resolved by ballots and a lookup
// table spread over the lanes: from the ballots of bits 0..3, lane l builds
// the entry for low nibble l & 15, the set of lanes whose low nibble equals
// it (nClear[k] is all ones where bit k of lane l is clear, so
// ballot ^ nClear[k] is the set of lanes agreeing with that bit of l), and a
// lane fetches the entry of its own nibble by shuffle. The remaining high
// bits are resolved in one of two ways:
//   BB = 8: four more ballots build a second 16-entry table for the high
//           nibble; peers = low entry & high entry (two shuffles);
//   BB = 5: a fifth ballot widens the table to 32 entries (bit 4 of the
//           lane: blocks are one-dimensional, so threadIdx.x & 16), and
//           match.any on the top three bits gives the rest;
//   BB = 4: match.any on the high nibble.
// All three return the same set; which is fastest depends on the value mode
// and the array size and is a choice of the autotuner.
template<int BB>
__device__ __forceinline__ unsigned match_digit8(unsigned d,
	const unsigned (&nClear)[4]) {
	static_assert(BB == 4 || BB == 5 || BB == 8, "ballot bits: 4, 5 or 8");
	unsigned lo = __ballot_sync(0xffffffffu, d & 1u) ^ nClear[0];
#pragma unroll
	for(int k = 1; k < 4; ++k) lo &= __ballot_sync(0xffffffffu, d & (1u << k)) ^ nClear[k];
	if constexpr(BB == 8) {
		unsigned hi = __ballot_sync(0xffffffffu, d & 16u) ^ nClear[0];
#pragma unroll
		for(int k = 1; k < 4; ++k) hi &= __ballot_sync(0xffffffffu, d & (16u << k)) ^ nClear[k];
		return __shfl_sync(0xffffffffu, lo, d & 15u) & __shfl_sync(0xffffffffu, hi, d >> 4);
	} else if constexpr(BB == 5) {
		const unsigned nClear4 = (threadIdx.x & 16u) ? 0u : 0xffffffffu;
		lo &= __ballot_sync(0xffffffffu, d & 16u) ^ nClear4;
		return __match_any_sync(0xffffffffu, d >> 5) & __shfl_sync(0xffffffffu, lo, d & 31u);
	} else {
		return __match_any_sync(0xffffffffu, d >> 4) & __shfl_sync(0xffffffffu, lo, d & 15u);
	}
}

__device__ __forceinline__ void stage_tile(unsigned* dst, const unsigned* src,
	unsigned bytes, uint64_t* bar) {
	mbar_arrive_expect_tx(bar, bytes);
	bulk_load(dst, src, bytes, bar);
}

// The digit of a key. A whole byte (8-bit digit at a multiple of 8) is one
// byte permute; any other field a shift and a mask.
template<bool BYTE> struct DigitOf {
	int shift;
	unsigned mask;
	unsigned sel;
	__device__ __forceinline__ DigitOf(int s, int width)
		: shift(s), mask((1u << width) - 1), sel(0x4440u | (unsigned)(s >> 3)) { }
	__device__ __forceinline__ unsigned operator()(unsigned k) const {
		if constexpr(BYTE) return __byte_perm(k, 0u, sel);
		else return (k >> shift) & mask;
	}
};

} // namespace mgpusort
