// Engine functions that other parts of the library use but that are not
// part of its C ABI (the library is built with hidden visibility, so these
// are not exported).
#pragma once

#include "../../include/mgpusort.h"

// Makes the engine's segmented-sort scratch large enough for a batch of up
// to n elements in numSegments segments, now, so that later sortSegmentedArray
// calls within those limits never free or allocate device memory (a free
// waits for all work on the device). Returns SORT_STATUS_DEVICE_ALLOC_FAILED
// if the memory is not available.
sortStatus_t engine_reserve_segmented(sortEngine_t engine, int n, int numSegments);
