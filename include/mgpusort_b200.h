/*
 * mgpusort_b200.h -- entry points of libmgpusort_b200.so that have no
 * counterpart in Modern GPU's inc/mgpusort.h. They sit beside the drop-in
 * API of mgpusort.h and use the same engine handle and status codes.
 */
#ifndef MGPUSORT_B200_EXT_H
#define MGPUSORT_B200_EXT_H

#include "mgpusort.h"

#ifdef __cplusplus
extern "C" {
#endif

/* sortArray on a caller-chosen CUDA stream instead of the legacy default
 * stream. One engine must not run two sorts at the same time: its device
 * scratch is shared, so concurrent streams need one engine each. */
sortStatus_t SORTAPI sortArrayAsync(sortEngine_t engine, sortData_t data,
	CUstream stream);

/* Wait for the engine's last sort to finish. Returns
 * SORT_STATUS_KERNEL_ERROR if a device-side bounded wait of any earlier sort
 * on this engine ran out (its output is then invalid), and clears that
 * error. */
sortStatus_t SORTAPI sortSynchronize(sortEngine_t engine);

/* The pass plan a sort would run, without any device work: bitPass 0 gives
 * sortArray's plan, 1..6 sortArrayEx's. Writes the digit width of each pass,
 * least significant first, into widths (room for 32) and returns the number
 * of passes, 0 for an empty bit range, or -1 for an invalid range. */
int SORTAPI sortPlanPasses(int firstBit, int endBit, int bitPass,
	int* widths);

/* Fault injection for tests of the device-side bounded waits: in the next
 * pass launched by this engine, the CTA that sorts tile `tile` (7680 or 7168
 * elements each) also waits on a barrier that nothing completes, so that
 * bounded wait runs out (about half a second) and the sort reports
 * SORT_STATUS_KERNEL_ERROR through sortSynchronize. -1 turns it off. Nothing
 * faults, traps or hangs; the engine is usable afterwards. */
sortStatus_t SORTAPI sortInjectFault(sortEngine_t engine, int tile);

/* Kernel timing for benchmarks: while enabled, the engine brackets its
 * launches with CUDA events on its stream. sortReadKernelTiming waits for
 * them and returns, since the last read, the summed milliseconds and counts
 * of the counting launches (each pass's count + scan kernels, and the
 * earlyExit histogram kernel) as "upsweep", and of the sort kernel launches
 * (one per pass) as "pass"; then it starts a new count. Any argument may be
 * NULL. */
sortStatus_t SORTAPI sortEnableKernelTiming(sortEngine_t engine, int enable);
sortStatus_t SORTAPI sortReadKernelTiming(sortEngine_t engine,
	double* upsweepMs, int* upsweepLaunches, double* passMs, int* passLaunches);

/* Batched segmented sort: sort each of numSegments independent segments of
 * the array described by `data` stably by its bit field, in one call. No
 * counterpart in the reference, whose callers sort many arrays with one
 * sortArray call each. segmentOffsets is a DEVICE array of numSegments + 1
 * ints: segment i is [segmentOffsets[i], segmentOffsets[i + 1]), with
 * segmentOffsets[0] == 0, non-decreasing, segmentOffsets[numSegments] ==
 * data->numElements (otherwise SORT_STATUS_KERNEL_ERROR is reported, by
 * sortSynchronize, and nothing is sorted). Buffers, value modes, swaps and
 * parity are sortArray's; every segment goes through the same passes, and
 * index mode writes positions within the segment. earlyExit is ignored.
 * Runs on `stream` (0: the legacy default stream); one engine runs one sort
 * at a time. The result equals one sortArray per segment. */
sortStatus_t SORTAPI sortSegmentedArray(sortEngine_t engine, sortData_t data,
	const int* segmentOffsets, int numSegments, CUstream stream);

/* Largest numElements that sortArrayNoAlloc accepts (4 Mi elements). */
#define SORT_NOALLOC_MAX_ELEMENTS 4194304

/* sortArray for callers that cannot allocate device memory. No counterpart
 * in the reference.
 *
 * Who needs it: programs that give all of a GPU's memory to their own
 * allocator or budget up front (so any allocation by a library fails or
 * breaks the budget), and latency-critical loops in which a cudaMalloc or
 * cudaFree would synchronize the device and stall other streams. sortArray's
 * engine allocates its scratch; this entry point takes no engine and calls no
 * cudaMalloc, cudaFree or other allocating routine.
 *
 * Its scratch is one file-scope device array of about 2 MiB (a control block
 * plus the per-pass range counts and offsets), held by every GPU that loads
 * the library until the process exits. The first call on a
 * device, with that device current, looks up the array's device address and
 * clears it (a synchronous cudaMemset); make that first call before any
 * stream capture.
 *
 * Semantics are sortArray's (same buffers, swaps, parity, bit range, value
 * modes, results), on `stream`, except that earlyExit is ignored (every pass
 * runs; the result is the same) and the call returns only after the sort has
 * finished, with SORT_STATUS_KERNEL_ERROR if a device-side wait ran out.
 * numElements above SORT_NOALLOC_MAX_ELEMENTS returns
 * SORT_STATUS_CONFIG_NOT_SUPPORTED without device work.
 *
 * Every call shares the one array: calls whose work overlaps on the GPU (from
 * several host threads, or on several streams) race and corrupt each other's
 * results; issue them one after another. */
sortStatus_t SORTAPI sortArrayNoAlloc(sortData_t data, CUstream stream);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* MGPUSORT_B200_EXT_H */
