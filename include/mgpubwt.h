/*
 * mgpubwt.h -- Burrows-Wheeler block sort on the B200 radix sort.
 *
 * The C API of Modern GPU's BWT library (inc/mgpubwt.h), the in-repo caller
 * of sortArray: it sorts the rotations of a block of bytes by their first
 * gpuKeySize symbols with chained multi-array sortArray calls on the GPU
 * (bwt/src/mgpubwt/mgpubwt.cpp:256-291), then finishes the groups of
 * rotations that still tie with a comparison sort on the host
 * (mgpubwt.cpp:318-348). Same functions, status codes and argument
 * meanings; implemented by libmgpusort_b200.so.
 */
#ifndef MGPUBWT_B200_H
#define MGPUBWT_B200_H

#include <cuda.h>

#ifdef _WIN32
#define BWTAPI __stdcall
#else
#define BWTAPI
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes, in the reference's order (inc/mgpubwt.h:21-34). */
typedef enum {
	BWT_STATUS_SUCCESS,
	BWT_STATUS_NOT_INITIALIZED,
	BWT_STATUS_DEVICE_ALLOC_FAILED,
	BWT_STATUS_INVALID_CONTEXT,
	BWT_STATUS_KERNEL_NOT_FOUND,
	BWT_STATUS_KERNEL_ERROR,
	BWT_STATUS_LAUNCH_ERROR,
	BWT_STATUS_INVALID_VALUE,
	BWT_STATUS_DEVICE_ERROR,
	BWT_STATUS_NOT_IMPLEMENTED,
	BWT_STATUS_UNSUPPORTED_DEVICE,
	BWT_STATUS_SORT_ERROR
} bwtStatus_t;

/* Name of a status code, or NULL when out of range (inc/mgpubwt.h:37,
 * bwt/src/mgpubwt/mgpubwt.cpp:20-23). */
const char* BWTAPI bwtStatusString(bwtStatus_t status);

typedef struct bwtEngine_d* bwtEngine_t;

/* Create an engine on the current device (inc/mgpubwt.h:47-48,
 * mgpubwt.cpp:66-105). kernelPath is accepted and ignored: the kernels are
 * in the library. A device other than compute capability 10.0 gives
 * BWT_STATUS_UNSUPPORTED_DEVICE. */
bwtStatus_t BWTAPI bwtCreateEngine(const char* kernelPath, bwtEngine_t* engine);

/* Destroy an engine (inc/mgpubwt.h:50, mgpubwt.cpp:107-110). */
bwtStatus_t BWTAPI bwtDestroyEngine(bwtEngine_t engine);

/* Sort the count cyclic rotations of block (inc/mgpubwt.h:72-74,
 * mgpubwt.cpp:213-371). gpuKeySize (1..24) is the number of leading symbols
 * the GPU radix sort orders; rotations that tie on them are finished on the
 * host. Outputs (each optional):
 *   indices[i]   start of the i-th smallest rotation;
 *   transform[i] the symbol before it, block[(indices[i] + count - 1) % count]
 *                (may alias block);
 *   segCount     number of groups of two or more rotations left tied by the
 *                GPU sort;
 *   avSegSize    their average size (0 when there are none).
 * Blocks shorter than 3000 bytes are sorted on the host only, as in the
 * reference. Rotations that are equal as whole strings are ordered by start
 * position (the reference's quicksort leaves them in an unspecified order;
 * transform is the same either way). */
bwtStatus_t BWTAPI bwtSortBlock(bwtEngine_t engine, const void* block, int count,
	int gpuKeySize, void* transform, int* indices, int* segCount, float* avSegSize);

#ifdef __cplusplus
}
#endif

#endif
