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
 * pass launched by this engine, tile `tile` skips publishing its digit counts,
 * so every later tile's lookback wait runs out (about half a second) and the
 * sort reports SORT_STATUS_KERNEL_ERROR through sortSynchronize. -1 turns it
 * off. Nothing faults or traps; the engine is usable afterwards. */
sortStatus_t SORTAPI sortInjectFault(sortEngine_t engine, int tile);

/* Kernel timing for benchmarks: while enabled, every kernel launch of the
 * engine is bracketed by CUDA events on its stream. sortReadKernelTiming
 * waits for them, returns the summed milliseconds and launch counts of the
 * upsweep (histogram) kernel and of the onesweep pass kernel since the last
 * read, and starts a new count. Any argument may be NULL. */
sortStatus_t SORTAPI sortEnableKernelTiming(sortEngine_t engine, int enable);
sortStatus_t SORTAPI sortReadKernelTiming(sortEngine_t engine,
	double* upsweepMs, int* upsweepLaunches, double* passMs, int* passLaunches);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* MGPUSORT_B200_EXT_H */
