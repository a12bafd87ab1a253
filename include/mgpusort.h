/*
 * mgpusort.h -- C ABI of the B200 radix sort (libmgpusort_b200.so).
 *
 * This header is the drop-in boundary. Every declaration below replaces the
 * declaration of the same name in Modern GPU's sort library, inc/mgpusort.h,
 * with the same argument meaning, the same status codes (same numeric values)
 * and the same sortData_d layout, so that code written against that header
 * compiles and links against this library unchanged. Each entry point cites
 * the reference declaration (file:line) that it replaces and the reference
 * implementation (sort/src/mgpusort/mgpusort.cpp:line) whose behaviour it
 * keeps. Behaviour that differs on purpose is stated at the declaration.
 *
 * Entry points that have no counterpart in the reference live in
 * mgpusort_b200.h.
 */
#ifndef MGPUSORT_B200_MGPUSORT_H
#define MGPUSORT_B200_MGPUSORT_H

#include <cuda.h> /* CUdeviceptr, as in the reference header */

#ifdef __cplusplus
#include <cstddef>
extern "C" {
#else
#include <stddef.h>
#include <stdbool.h>
#endif

#ifndef SORTAPI
#define SORTAPI
#endif

/* Status codes. Same names, order and values as inc/mgpusort.h:21-36. */
typedef enum {
	SORT_STATUS_SUCCESS = 0,
	SORT_STATUS_NOT_INITIALIZED,
	SORT_STATUS_DEVICE_ALLOC_FAILED,
	SORT_STATUS_HOST_ALLOC_FAILED,
	SORT_STATUS_CONFIG_NOT_SUPPORTED,
	SORT_STATUS_CONTEXT_MISMATCH,
	SORT_STATUS_INVALID_CONTEXT,
	SORT_STATUS_KERNEL_NOT_FOUND,
	SORT_STATUS_KERNEL_ERROR,
	SORT_STATUS_LAUNCH_ERROR,
	SORT_STATUS_INVALID_VALUE,
	SORT_STATUS_DEVICE_ERROR,
	SORT_STATUS_INTERNAL_ERROR,
	SORT_STATUS_UNSUPPORTED_DEVICE
} sortStatus_t;

/* Name of a status code, or NULL for a value outside the enum.
 * Replaces inc/mgpusort.h:39 (impl. sort/src/mgpusort/mgpusort.cpp:23-27). */
const char* SORTAPI sortStatusString(sortStatus_t status);

/* Opaque engine handle (inc/mgpusort.h:46-47). */
struct sortEngine_d;
typedef struct sortEngine_d* sortEngine_t;

/* Create an engine on the device of the CUDA context that is current on the
 * calling thread (the runtime's primary context when none is). The engine
 * starts with a reference count of one.
 * kernelPath is accepted and ignored: the sm_100a kernels are linked into the
 * library, there are no .cubin files to load.
 * Returns SORT_STATUS_UNSUPPORTED_DEVICE on anything but compute capability
 * 10.0 (B200), SORT_STATUS_INVALID_CONTEXT when no device can be used.
 * Replaces inc/mgpusort.h:50-51 (impl. mgpusort.cpp:200-250). */
sortStatus_t SORTAPI sortCreateEngine(const char* kernelPath,
	sortEngine_t* engine);

/* Validate a kernel configuration and prepare its launch attributes.
 * numSortThreads must be 128 or 256 and valuesPerThread 4 or 8, as in the
 * reference; useTransList is accepted and ignored (there is one scatter
 * strategy). Replaces inc/mgpusort.h:54-55 (impl. mgpusort.cpp:144-194). */
sortStatus_t SORTAPI sortLoadKernel(sortEngine_t engine, int numSortThreads,
	int valuesPerThread, bool useTransList, int valueCount);

/* Reference counting. sortReleaseEngine frees the engine and its device
 * scratch when the count reaches zero. Not thread-safe, like the reference.
 * Replace inc/mgpusort.h:58-59 (impl. mgpusort.cpp:252-261). */
sortStatus_t SORTAPI sortIncEngine(sortEngine_t engine);
sortStatus_t SORTAPI sortReleaseEngine(sortEngine_t engine);

/*
 * State of one sort job: a key array and up to six value arrays, each a pair
 * of device buffers that the sort ping-pongs between. Layout, member names and
 * anonymous unions are those of inc/mgpusort.h:63-147 so that existing callers
 * compile unchanged; the layout is checked by static_assert in the library.
 *
 * After a successful sort the sorted keys are in keys[0] and the values in
 * values[i][0]; the [1] buffers are scratch. Every executed pass swaps all
 * [0]/[1] pairs and flips parity, so a buffer that was at [0] before the sort
 * is at [parity ^ parity_before] afterwards (inc/mgpusort.h:107-110).
 */
typedef struct {
	/* Capacity, in elements, of every buffer below. */
	int maxElements;
	/* Number of elements to sort; must not exceed maxElements. */
	int numElements;
	/* 0: keys only. 1..6: that many value arrays moved with the keys.
	 * -1: write each key's original position into values1 (index mode). */
	int valueCount;
	/* The sort key is the bit field [firstBit, endBit) of each 32-bit key. */
	int firstBit;
	int endBit;
	/* Accepted for compatibility. This library never writes past
	 * numElements in any buffer, so end keys are always preserved. */
	bool preserveEndKeys;
	/* When true, sortArray reads the digit histograms back to the host once
	 * and skips every pass whose digit is the same for all keys. The result
	 * is identical either way; only the number of executed passes (and so
	 * parity) changes. */
	bool earlyExit;
	/* Flipped once per executed pass. */
	int parity;

	union {
		struct {
			CUdeviceptr keys[2];
			union {
				struct {
					CUdeviceptr values1[2];
					CUdeviceptr values2[2];
					CUdeviceptr values3[2];
					CUdeviceptr values4[2];
					CUdeviceptr values5[2];
					CUdeviceptr values6[2];
				};
				CUdeviceptr values[6][2];
			};
		};
		struct {
			unsigned int* pKeys[2];
			union {
				struct {
					unsigned int* pValues1[2];
					unsigned int* pValues2[2];
					unsigned int* pValues3[2];
					unsigned int* pValues4[2];
					unsigned int* pValues5[2];
					unsigned int* pValues6[2];
				};
				unsigned int* pValues[6][2];
			};
		};
	};
} sortData_d;
typedef sortData_d* sortData_t;

/* Allocate a sortData_d and all of its buffers: capacity maxElements rounded
 * up to a multiple of 2048, firstBit 0, endBit 32.
 * Replaces inc/mgpusort.h:155-156 (impl. mgpusort.cpp:655-682). */
sortStatus_t SORTAPI sortCreateData(sortEngine_t engine, int maxElements,
	int valueCount, sortData_t* data);

/* sortFreeData, then free the struct itself.
 * Replaces inc/mgpusort.h:157 (impl. mgpusort.cpp:684-690). */
sortStatus_t SORTAPI sortDestroyData(sortData_t data);

/* Allocate every buffer that the job needs (keys and |valueCount| value
 * pairs) whose pointer is still 0, with capacity RoundUp(maxElements, 2048).
 * Buffers the caller attached are left alone. Sets parity to 0.
 * Replaces inc/mgpusort.h:164 (impl. mgpusort.cpp:692-719). */
sortStatus_t SORTAPI sortAllocData(sortEngine_t engine, sortData_t data);

/* cudaFree every non-zero buffer pointer, then zero the struct. Callers zero
 * the pointers of buffers they own first (inc/mgpusort.h:97-105).
 * Replaces inc/mgpusort.h:165 (impl. mgpusort.cpp:721-734). */
sortStatus_t SORTAPI sortFreeData(sortData_d* data);

/* Stable radix sort of data->keys[0] (and the value arrays) by the bit field
 * [firstBit, endBit), on the legacy default stream, asynchronous to the host
 * like the reference: a later cudaMemcpy / cuMemcpyDtoH on the default stream
 * orders after it. The pass plan is this library's own (digits of up to
 * 8 bits); it is not the reference's pass table, so parity can end up
 * different from the reference's, while the contents of keys[0] and
 * values[i][0] over [0, numElements) are the same.
 * endBit == firstBit returns SUCCESS without work. numElements > maxElements,
 * a bit range outside [0, 32], a missing buffer or valueCount outside
 * [-1, 6] give SORT_STATUS_INVALID_VALUE. A device-side error (a bounded wait
 * that ran out) is reported as SORT_STATUS_KERNEL_ERROR by the next call on
 * the engine or by sortSynchronize.
 * Replaces inc/mgpusort.h:167 (impl. mgpusort.cpp:607-616, pass loop
 * mgpusort.cpp:541-601). */
sortStatus_t SORTAPI sortArray(sortEngine_t engine, sortData_t data);

/* sortArray with a caller-chosen pass plan: the bit range is split into
 * ceil(bits / bitPass) passes of bitPass or bitPass - 1 bits exactly as the
 * reference does (so parity matches the reference's). numSortThreads must be
 * 128 or 256 and valuesPerThread 8, otherwise SORT_STATUS_INVALID_VALUE;
 * bitPass outside 1..6 means 6. useTransList is accepted and ignored.
 * Replaces inc/mgpusort.h:169-170 (impl. mgpusort.cpp:618-648). */
sortStatus_t SORTAPI sortArrayEx(sortEngine_t engine, sortData_t data,
	int numSortThreads, int valuesPerThread, int bitPass, bool useTransList);

/* Convenience: copy numElements keys (and values, when non-NULL) from host
 * memory to the device, sort the low numBits bits, copy back. Synchronous.
 * The reference copies sizeof(double) * n bytes each way
 * (mgpusort.cpp:751,756,765,770); this copies sizeof(unsigned) * n.
 * Replaces inc/mgpusort.h:183-184 (impl. mgpusort.cpp:740-776). */
sortStatus_t SORTAPI sortHost(sortEngine_t engine, unsigned int* keys,
	unsigned int* values, int numElements, int numBits);

/* Convenience: sort numElements keys (and values, when non-zero) in place in
 * the caller's device buffers by their low numBits bits. Synchronous. The
 * sorted data always ends in the caller's buffers (the reference copies back
 * from the wrong buffer when the pass count is odd, mgpusort.cpp:796-803).
 * The buffers need no padding: nothing past numElements is touched.
 * Replaces inc/mgpusort.h:186-187 (impl. mgpusort.cpp:782-806). */
sortStatus_t SORTAPI sortDevice(sortEngine_t engine, CUdeviceptr keys,
	CUdeviceptr values, int numElements, int numBits);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* MGPUSORT_B200_MGPUSORT_H */
