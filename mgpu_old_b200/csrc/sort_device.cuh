// Device-side building blocks shared by the sort kernels: PTX wrappers for
// the mbarrier / bulk-copy (TMA) path, relaxed and streaming global loads,
// and warp scans. sm_100a only.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mgpusort {

// Error bits written to the device error word and to the host-mapped mirror.
constexpr unsigned kErrBarrierTimeout = 2u;
constexpr unsigned kErrInjected = 8u;
constexpr unsigned kErrBadSegments = 16u;

// Bounded waits. A poll of a status word or an mbarrier normally succeeds
// within microseconds. After kSpinFastPolls polls a waiter backs off with
// nanosleep and reads the global timer; once kWaitNs has passed it gives up
// and reports an error instead of hanging.
constexpr unsigned kSpinFastPolls = 256;
constexpr unsigned long long kWaitNs = 500ull * 1000ull * 1000ull;

__device__ __forceinline__ unsigned long long global_ns() {
	unsigned long long t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

// Tracks one bounded wait: call poll() after every unsuccessful attempt;
// it returns false once the wait has run out of time.
struct WaitBudget {
	unsigned polls = 0;
	unsigned long long start = 0;
	__device__ __forceinline__ bool poll() {
		if(++polls <= kSpinFastPolls) return true;
		unsigned long long now = global_ns();
		if(!start) start = now;
		else if(now - start > kWaitNs) return false;
		__nanosleep(128);
		return true;
	}
};

__device__ __forceinline__ unsigned smem_addr(const void* p) {
	return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;"
		:: "r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (bulk copy) accesses to the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar,
	unsigned bytes) {
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
		:: "r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// One bulk (non-tensor, non-multicast) copy global -> shared that completes
// its bytes on *bar. src, dst and bytes must be multiples of 16.
__device__ __forceinline__ void bulk_load(void* dst, const void* src,
	unsigned bytes, uint64_t* bar) {
	asm volatile(
		"cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes"
		" [%0], [%1], %2, [%3];"
		:: "r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
		: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
	unsigned ok;
	asm volatile(
		"{\n\t.reg .pred p;\n\t"
		"mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		"selp.u32 %0, 1, 0, p;\n\t}"
		: "=r"(ok) : "r"(smem_addr(bar)), "r"(parity) : "memory");
	return ok != 0;
}

// Wait for phase `parity` of *bar to complete; false if the cap ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar,
	unsigned parity) {
	WaitBudget budget;
	while(!mbar_try_wait(bar, parity))
		if(!budget.poll()) return false;
	return true;
}

__device__ __forceinline__ unsigned ld_relaxed_u32(const unsigned* p) {
	unsigned v;
	asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];"
		: "=r"(v) : "l"(p) : "memory");
	return v;
}

// Streaming 16-byte load that does not allocate in L1.
__device__ __forceinline__ uint4 ld_stream_u4(const uint4* p) {
	uint4 v;
	asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
		: "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p));
	return v;
}

// 16-byte load cached in L2 only: coherent with stores that other CTAs of
// the same grid made before a grid-wide barrier.
__device__ __forceinline__ uint4 ld_cg_u4(const uint4* p) {
	uint4 v;
	asm volatile("ld.global.cg.v4.u32 {%0,%1,%2,%3}, [%4];"
		: "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p) : "memory");
	return v;
}

// Streaming load of data that no CTA of the running grid writes (NC), or a
// coherent one of data written earlier in the same grid.
template<bool NC>
__device__ __forceinline__ uint4 ld_in_u4(const uint4* p) {
	if constexpr(NC) return ld_stream_u4(p);
	else return ld_cg_u4(p);
}

__device__ __forceinline__ unsigned lanemask_lt() {
	unsigned m;
	asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
	return m;
}

__device__ __forceinline__ unsigned warp_inclusive_scan(unsigned x, int lane) {
#pragma unroll
	for(int d = 1; d < 32; d <<= 1) {
		unsigned y = __shfl_up_sync(0xffffffffu, x, d);
		if(lane >= d) x += y;
	}
	return x;
}

// Record a device error: sticky bit in the device control block and a plain
// store to the host-mapped word, which the host reads without synchronizing.
__device__ __forceinline__ void report_error(unsigned* devError,
	volatile unsigned* hostError, unsigned code) {
	atomicOr(devError, code);
	if(hostError) *hostError = code;
}

} // namespace mgpusort
