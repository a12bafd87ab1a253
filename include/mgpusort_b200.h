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
 * pass launched by this engine, the CTA that sorts tile `tile` (tiles of the
 * value mode's shape in tile_config.h: 5120, 7680 or 6144 elements as
 * shipped) also waits on a barrier that nothing completes, so that
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

/* CUDA graphs of repeated sorts. When a call's launch sequence is the same
 * as an earlier call's (same sizes, bit range, value mode, buffers and
 * parity, same segment-offset pointer and count for sortSegmentedArray), the
 * engine captures the sequence once as a CUDA graph and from then on
 * replays it with one graph launch; buffer contents and segment boundaries
 * may differ between calls. Calls with earlyExit, with kernel timing on or
 * with an injected fault always launch directly. On by default; enable = 0
 * turns it off and frees the cached graphs (at most 8 per engine). */
sortStatus_t SORTAPI sortEnableGraphs(sortEngine_t engine, int enable);

/* Graph replays since the engine was created, and graphs cached now. Either
 * pointer may be NULL. */
sortStatus_t SORTAPI sortGraphStats(sortEngine_t engine, int* replays, int* cached);

/* Key types of sortArrayTyped. */
typedef enum {
	SORT_KEY_UINT32 = 0,
	SORT_KEY_INT32 = 1,
	SORT_KEY_FLOAT32 = 2
} sortKeyType_t;

/* sortArrayAsync for signed or floating-point keys: keys[0] holds int32 or
 * IEEE-754 binary32 bit patterns (keyType, a sortKeyType_t) and the sort
 * orders them numerically, floats in the total order of their sign-magnitude
 * image: -NaN < -inf < ... < -0.0 < +0.0 < ... < +inf < +NaN. The keys are
 * mapped in place to that order-preserving uint32 image before the first
 * pass and back after the last (the transform of the reference's
 * sort/src/kernels/common.cu:159-186), so they come out as the caller's bit
 * patterns; [firstBit, endBit) selects bits of the image. No counterpart in
 * the reference's sort API. An unknown keyType is SORT_STATUS_INVALID_VALUE. */
sortStatus_t SORTAPI sortArrayTyped(sortEngine_t engine, sortData_t data,
	int keyType, CUstream stream);

/* The k-th smallest key by sorting: sortArray on data, then element k of
 * the sorted keys copied to *value (waits for the sort). This is the
 * sort-based selection of the reference's select benchmark
 * (select/src/selecttest/mgpusorttest.cpp:3-32), kept as one call. k outside
 * [0, numElements) or a null value is SORT_STATUS_INVALID_VALUE. */
sortStatus_t SORTAPI sortSelectKey(sortEngine_t engine, sortData_t data, int k,
	unsigned int* value);

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

/* Sort server: requests from host memory are copied in, sorted and copied
 * back by a scheduler thread that keeps a pool of device memory and one
 * engine and stream per slot. Requests are admitted in arrival order while a
 * slot is free and their device footprint (2 x keys + 2 x values) fits the
 * memory budget; small requests (at most coalesceMax elements) of the same
 * kind (values or not, same bit range) are coalesced into one segmented sort.
 * Batches on different slots overlap on the GPU, and requests that arrive
 * while others are in flight join the next batch (continuous batching). Each
 * result equals a sortArray of that request alone. No counterpart in the
 * reference. */
typedef struct sortServer_d* sortServer_t;

typedef struct {
	size_t memoryBudget;   /* device bytes for requests in flight; 0: 64 GiB */
	int slots;             /* batches in flight at once; 0: 4 */
	int coalesceMax;       /* largest request that is coalesced; 0: 1 Mi */
	int maxBatchElements;  /* elements per coalesced batch; 0: 16 Mi */
	int maxBatchRequests;  /* requests per coalesced batch; 0: 4096 */
} sortServerConfig;

/* Start a server on the current device (config may be NULL). */
sortStatus_t SORTAPI sortServerCreate(const sortServerConfig* config,
	sortServer_t* server);

/* Queue a request: sort keys (and values, if non-NULL) by [firstBit,
 * endBit) into keysOut (valuesOut). All four are host buffers that must stay
 * valid until the request is waited for; page-locked memory lets the copies
 * overlap. A request larger than the budget gives
 * SORT_STATUS_CONFIG_NOT_SUPPORTED. */
sortStatus_t SORTAPI sortServerSubmit(sortServer_t server, const unsigned* keys,
	const unsigned* values, int numElements, int firstBit, int endBit,
	unsigned* keysOut, unsigned* valuesOut, unsigned long long* ticket);

/* *done = 1 once the request's results are in its output buffers. */
sortStatus_t SORTAPI sortServerPoll(sortServer_t server, unsigned long long ticket,
	int* done);

/* Block until the request is done; return its status and (if non-NULL) the
 * seconds from submission to completion. The ticket is retired. */
sortStatus_t SORTAPI sortServerWait(sortServer_t server, unsigned long long ticket,
	double* latencySeconds);

/* Finish every queued request, then stop the server and free it. */
sortStatus_t SORTAPI sortServerDestroy(sortServer_t server);

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
 * Every call shares the one array, and calls whose work overlapped on the
 * GPU would race on it. So that none can, a process-wide lock is held from
 * the first launch until the sort has finished on the GPU: calls from several
 * host threads (on any streams) run one after another, and a call waits for
 * the one before it to finish. (Each process has its own copy of the array.)
 * If a launch fails, the call returns SORT_STATUS_LAUNCH_ERROR and leaves the
 * struct's buffers and parity as they were; the buffers' contents are then
 * undefined. */
sortStatus_t SORTAPI sortArrayNoAlloc(sortData_t data, CUstream stream);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* MGPUSORT_B200_EXT_H */
