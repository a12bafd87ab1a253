// Tile shapes, digit width and warp-ranking method of the sort passes.
//
// These values are the choices of the autotuner (mgpu_old_b200/autotune.py),
// which builds the library once per candidate, times each build on a B200
// over a fixed set of workloads and writes this file with the fastest
// candidate per class. Every value can be overridden at build time with -D.
//
//  * keys: keys only (sort_range_single without values);
//  * single: index mode or one value array (sort_range_single);
//  * multi: two to six value arrays (sort_range_multi);
//  * digits: the widest digit of a pass;
//  * <class>_ballot: digit bits the warp ranking of the class resolves by
//    ballots (match_digit8); single_large_ballot applies to sortArray calls
//    of at least MGPU_SORT_SINGLE_LARGE_ELEMENTS keys, small_ballot to the
//    segmented sort's kernel for segments that fit one tile;
//  * <class>_batch: items per thread whose peers are found before their
//    digit counters are updated (rank_tile).
// Measured by the autotuner (median ms per sort; score = geometric
// mean of time / best time over the class's workloads):
//   keys: chosen 512x14x2
//       512x14x2  score 1.030  keys_u32_1048576 0.059, keys_u32_16777216 0.336, keys_u32_67108864 1.243
//       384x20x2  score 1.036  keys_u32_1048576 0.061, keys_u32_16777216 0.342, keys_u32_67108864 1.202
//       384x24x2  score 1.049  keys_u32_1048576 0.068, keys_u32_16777216 0.328, keys_u32_67108864 1.184
//       256x20x3  score 1.059  keys_u32_1048576 0.068, keys_u32_16777216 0.342, keys_u32_67108864 1.167
//       512x16x2  score 1.077  keys_u32_1048576 0.070, keys_u32_16777216 0.332, keys_u32_67108864 1.229
//   single: chosen 384x20x2
//       384x20x2  score 1.000  index_u32_16777216 0.455, pairs_and24_33554432 0.600, pairs_u32_67108864 1.686
//       512x14x2  score 1.022  index_u32_16777216 0.461, pairs_and24_33554432 0.621, pairs_u32_67108864 1.714
//       256x24x2  score 1.064  index_u32_16777216 0.485, pairs_and24_33554432 0.604, pairs_u32_67108864 1.888
//       384x16x2  score 1.071  index_u32_16777216 0.483, pairs_and24_33554432 0.616, pairs_u32_67108864 1.894
//       768x10x1  score 1.160  index_u32_16777216 0.489, pairs_and24_33554432 0.692, pairs_u32_67108864 2.119
//       256x20x3  score 1.240  index_u32_16777216 0.567, pairs_and24_33554432 0.707, pairs_u32_67108864 2.186
//   multi: chosen 768x8x1
//        768x8x1  score 1.000  multi3_u32_16777216 0.883, multi6_17bit_16777216 1.202
//       512x12x1  score 1.007  multi3_u32_16777216 0.883, multi6_17bit_16777216 1.219
//       384x16x1  score 1.023  multi3_u32_16777216 0.893, multi6_17bit_16777216 1.243
//       576x10x1  score 1.027  multi3_u32_16777216 0.901, multi6_17bit_16777216 1.241
//   digits: chosen 8
//              8  score 1.000  keys_u32_16777216 0.397, pairs_and24_33554432 0.674
//              7  score 1.230  keys_u32_16777216 0.481, pairs_and24_33554432 0.842
//              6  score 1.333  keys_u32_16777216 0.565, pairs_and24_33554432 0.842
//   keys_ballot: chosen 5
//              5  score 1.000  keys_u32_16777216 0.336, keys_u32_67108864 1.243
//              8  score 1.141  keys_u32_16777216 0.381, keys_u32_67108864 1.427
//              4  score 1.150  keys_u32_16777216 0.387, keys_u32_67108864 1.425
//   single_ballot: chosen 5
//              5  score 1.000  index_u32_16777216 0.457, pairs_and24_33554432 0.602, pairs_u32_16777216 0.461, segments_lognormal_10000 3.809
//              4  score 1.060  index_u32_16777216 0.487, pairs_and24_33554432 0.614, pairs_u32_16777216 0.492, segments_lognormal_10000 4.132
//              8  score 1.084  index_u32_16777216 0.494, pairs_and24_33554432 0.664, pairs_u32_16777216 0.494, segments_lognormal_10000 4.120
//   single_large_ballot: chosen 4
//              4  score 1.000  index_u32_67108864 1.669, pairs_u32_100663296 2.460, pairs_u32_67108864 1.679
//              8  score 1.016  index_u32_67108864 1.696, pairs_u32_100663296 2.497, pairs_u32_67108864 1.710
//              5  score 1.045  index_u32_67108864 1.739, pairs_u32_100663296 2.587, pairs_u32_67108864 1.751
//   multi_ballot: chosen 8
//              8  score 1.002  multi3_u32_16777216 0.883, multi6_17bit_16777216 1.212
//              5  score 1.002  multi3_u32_16777216 0.883, multi6_17bit_16777216 1.213
//              4  score 1.008  multi3_u32_16777216 0.879, multi6_17bit_16777216 1.231
//   keys_batch: chosen 5
//              5  score 1.000  keys_u32_16777216 0.336, keys_u32_67108864 1.237
//             20  score 1.002  keys_u32_16777216 0.336, keys_u32_67108864 1.243
//              4  score 1.011  keys_u32_16777216 0.338, keys_u32_67108864 1.255
//              1  score 1.019  keys_u32_16777216 0.342, keys_u32_67108864 1.262
//             10  score 1.020  keys_u32_16777216 0.342, keys_u32_67108864 1.264
//   single_batch: chosen 10
//             10  score 1.000  index_u32_16777216 0.459, pairs_and24_33554432 0.602, pairs_u32_67108864 1.681, segments_lognormal_10000 3.827
//              5  score 1.006  index_u32_16777216 0.461, pairs_and24_33554432 0.605, pairs_u32_67108864 1.700, segments_lognormal_10000 3.832
//              4  score 1.006  index_u32_16777216 0.461, pairs_and24_33554432 0.606, pairs_u32_67108864 1.702, segments_lognormal_10000 3.827
//              1  score 1.024  index_u32_16777216 0.467, pairs_and24_33554432 0.625, pairs_u32_67108864 1.708, segments_lognormal_10000 3.923
//             20  score 1.071  index_u32_16777216 0.490, pairs_and24_33554432 0.666, pairs_u32_67108864 1.859, segments_lognormal_10000 3.852
//   multi_batch: chosen 8
//              8  score 1.000  multi3_u32_16777216 0.883, multi6_17bit_16777216 1.206
//              4  score 1.001  multi3_u32_16777216 0.883, multi6_17bit_16777216 1.208
//              2  score 1.004  multi3_u32_16777216 0.889, multi6_17bit_16777216 1.208
//              1  score 1.008  multi3_u32_16777216 0.893, multi6_17bit_16777216 1.210
//   small_batch: chosen 8
//              8  score 1.000  segments_small_50000 0.993
//             16  score 1.000  segments_small_50000 0.993
//              4  score 1.002  segments_small_50000 0.995
//              2  score 1.014  segments_small_50000 1.008
//              1  score 1.039  segments_small_50000 1.032
//   small_ballot: chosen 5
//              5  score 1.000  segments_small_50000 0.987
//              4  score 1.029  segments_small_50000 1.016
//              8  score 1.079  segments_small_50000 1.065
#pragma once

// 1: the one-array sort passes (keys only, index mode, one value array)
// store their output in aligned 16-byte vectors where a digit run covers
// them (the reordered tile is laid out so that shared and global positions
// agree mod 4); 0: one 4-byte store per element.
#ifndef MGPU_SORT_VECTOR_STORES
#define MGPU_SORT_VECTOR_STORES 0
#endif

#ifndef MGPU_SORT_KEYS_THREADS
#define MGPU_SORT_KEYS_THREADS 512
#endif
#ifndef MGPU_SORT_KEYS_ITEMS
#define MGPU_SORT_KEYS_ITEMS 14
#endif
#ifndef MGPU_SORT_KEYS_MIN_BLOCKS
#define MGPU_SORT_KEYS_MIN_BLOCKS 2
#endif
// The single class was swept again by hand after the autotuner's run above,
// over shapes it had not tried (whole sorts, Gkeys/s, 64 Mi uniform pairs /
// 32 Mi 24-bit skewed pairs / the 10k-segment batch): 384 x 20 (the
// autotuner's choice) 39.8 / 55.8 / 36.9; 256 x 32 41.4 / 57.9 / 36.3;
// 256 x 30 40.1 / 57.5 / 35.8; 256 x 28 37.6 / 57.1 / 36.1; 352 x 22,
// 320 x 24, 416 x 18 and 288 x 26 39.1-39.4 / 51.6-54.8. Fewer, longer warps
// win. The ranking needs a thread per digit, so 256 threads is the floor.
#ifndef MGPU_SORT_SINGLE_THREADS
#define MGPU_SORT_SINGLE_THREADS 256
#endif
// With vector stores the gaps of the reordered tile cost 2 x 3 KB of shared
// memory per CTA: 256 x 28 still fits two CTAs per SM.
#ifndef MGPU_SORT_SINGLE_ITEMS
#if MGPU_SORT_VECTOR_STORES
#define MGPU_SORT_SINGLE_ITEMS 28
#else
#define MGPU_SORT_SINGLE_ITEMS 32
#endif
#endif
#ifndef MGPU_SORT_SINGLE_MIN_BLOCKS
#define MGPU_SORT_SINGLE_MIN_BLOCKS 2
#endif
// The segmented sort's range passes with index mode or one value array: the
// single class's earlier shape, which is faster on their short ranges (10k
// lognormal segments: 36.9 against 36.3 Gkeys/s with 256 x 32).
#ifndef MGPU_SORT_SEG_SINGLE_THREADS
#define MGPU_SORT_SEG_SINGLE_THREADS 384
#endif
#ifndef MGPU_SORT_SEG_SINGLE_ITEMS
#define MGPU_SORT_SEG_SINGLE_ITEMS 20
#endif
#ifndef MGPU_SORT_SEG_SINGLE_MIN_BLOCKS
#define MGPU_SORT_SEG_SINGLE_MIN_BLOCKS 2
#endif
#ifndef MGPU_SORT_SEG_SINGLE_RANK_BATCH
#define MGPU_SORT_SEG_SINGLE_RANK_BATCH 10
#endif
#ifndef MGPU_SORT_MULTI_THREADS
#define MGPU_SORT_MULTI_THREADS 768
#endif
#ifndef MGPU_SORT_MULTI_ITEMS
#define MGPU_SORT_MULTI_ITEMS 8
#endif
#ifndef MGPU_SORT_MULTI_MIN_BLOCKS
#define MGPU_SORT_MULTI_MIN_BLOCKS 1
#endif
// Keys-only passes of sortArray on at least KEYS_LARGE_ELEMENTS keys: their
// own tile shape (the keys class above is tuned on 1 Mi keys). 256 x 20 with
// three CTAs per SM against 512 x 14 x 2, whole sorts of uniform 32-bit
// keys: 4% slower at 16 Mi, 2.2% faster at 32 Mi, 4.0% at 48 Mi, 4.7% at
// 64 Mi, 5.5% at 96 Mi. At 64 Mi keys, 256 x 28 x 3 is 1.8% faster again
// than 256 x 20 x 3 (256 x 32 x 2: 1.2%).
#ifndef MGPU_SORT_KEYS_LARGE_THREADS
#define MGPU_SORT_KEYS_LARGE_THREADS 256
#endif
#ifndef MGPU_SORT_KEYS_LARGE_ITEMS
#define MGPU_SORT_KEYS_LARGE_ITEMS 28
#endif
#ifndef MGPU_SORT_KEYS_LARGE_MIN_BLOCKS
#define MGPU_SORT_KEYS_LARGE_MIN_BLOCKS 3
#endif
#ifndef MGPU_SORT_KEYS_LARGE_ELEMENTS
#define MGPU_SORT_KEYS_LARGE_ELEMENTS 33554432
#endif
// Digit bits the warp ranking resolves by ballots (8, 5 or 4); match.any
// resolves the rest. Keys, single and multi classes as above; "small" is the
// segmented sort's kernel for segments that fit one tile.
#ifndef MGPU_SORT_KEYS_BALLOT_BITS
#define MGPU_SORT_KEYS_BALLOT_BITS 5
#endif
#ifndef MGPU_SORT_SINGLE_BALLOT_BITS
#define MGPU_SORT_SINGLE_BALLOT_BITS 5
#endif
// The single class on sortArray calls of at least LARGE_ELEMENTS keys (the
// scatter then spans a large array; measured crossover between 32M and 48M).
#ifndef MGPU_SORT_SINGLE_LARGE_BALLOT_BITS
#define MGPU_SORT_SINGLE_LARGE_BALLOT_BITS 4
#endif
#ifndef MGPU_SORT_SINGLE_LARGE_ELEMENTS
#define MGPU_SORT_SINGLE_LARGE_ELEMENTS 41943040
#endif
#ifndef MGPU_SORT_MULTI_BALLOT_BITS
#define MGPU_SORT_MULTI_BALLOT_BITS 8
#endif
#ifndef MGPU_SORT_SMALL_BALLOT_BITS
#define MGPU_SORT_SMALL_BALLOT_BITS 5
#endif
// Items of a thread whose peers the warp ranking finds before it updates
// their digit counters (1: one item at a time), per class.
#ifndef MGPU_SORT_KEYS_RANK_BATCH
#define MGPU_SORT_KEYS_RANK_BATCH 5
#endif
// With 256 x 32 tiles: batch 16 41.6 / 57.9, 10 41.4 / 57.9, 8 41.1 / 57.1
// (Gkeys/s, 64 Mi pairs / 32 Mi skewed pairs).
#ifndef MGPU_SORT_SINGLE_RANK_BATCH
#define MGPU_SORT_SINGLE_RANK_BATCH 16
#endif
#ifndef MGPU_SORT_MULTI_RANK_BATCH
#define MGPU_SORT_MULTI_RANK_BATCH 8
#endif
#ifndef MGPU_SORT_SMALL_RANK_BATCH
#define MGPU_SORT_SMALL_RANK_BATCH 8
#endif
// sortArray calls of at most CARVEOUT_MAX_ELEMENTS keys run the count and
// scan kernels with the sort kernel's (largest) shared-memory carveout.
#ifndef MGPU_SORT_CARVEOUT_MAX_ELEMENTS
#define MGPU_SORT_CARVEOUT_MAX_ELEMENTS 1048576
#endif
// Tiles per range of a large segment (a segment gets at most 64 ranges):
// the unit of work of the segmented count and sort kernels.
#ifndef MGPU_SORT_SEG_TILES_PER_RANGE
#define MGPU_SORT_SEG_TILES_PER_RANGE 4
#endif
// 1: the segmented sort's kernels all take the largest carveout.
#ifndef MGPU_SORT_SEG_SHARED_CARVEOUT
#define MGPU_SORT_SEG_SHARED_CARVEOUT 0
#endif
// sortArray on at most this many elements (up to 4096) sorts the whole array
// in one CTA's shared memory through every pass (one launch); 0 turns that off.
#ifndef MGPU_SORT_SMALL_ARRAY_MAX
#define MGPU_SORT_SMALL_ARRAY_MAX 4096
#endif
// Largest CTA of that sort (256, 512 or 1024 threads).
#ifndef MGPU_SORT_SMALL_ARRAY_THREADS
#define MGPU_SORT_SMALL_ARRAY_THREADS 1024
#endif
// sortArray on more than SMALL_ARRAY_MAX and at most COOP_MAX_ELEMENTS keys
// (keys only, index mode or one value array) runs every pass in one
// cooperative launch; 0 turns that off. Off: on B200 it measured slower than
// the three launches per pass at every size from 64 Ki to 16 Mi keys (1 Mi
// keys: 72 us against 59 us).
#ifndef MGPU_SORT_COOP_MAX_ELEMENTS
#define MGPU_SORT_COOP_MAX_ELEMENTS 0
#endif
// Widest digit of sortArray's pass plan (1..8): ceil(bits / width) passes.
#ifndef MGPU_SORT_MAX_DIGIT_BITS
#define MGPU_SORT_MAX_DIGIT_BITS 8
#endif

// Onesweep pass kernels (onesweep.cu): ranking threads (the block has one
// more warp, which does the lookback), keys per thread and CTAs per SM of a
// tile per class (keys only; index mode or one value array; two to six
// value arrays), the warp ranking's ballot bits and batch per class, and
// the staging slots (2: the next tile is copied in while the current one is
// reordered and stored).
#ifndef MGPU_OS_KEYS_THREADS
#define MGPU_OS_KEYS_THREADS 256
#endif
#ifndef MGPU_OS_KEYS_ITEMS
#define MGPU_OS_KEYS_ITEMS 16
#endif
#ifndef MGPU_OS_KEYS_MIN_BLOCKS
#define MGPU_OS_KEYS_MIN_BLOCKS 3
#endif
#ifndef MGPU_OS_KEYS_SLOTS
#define MGPU_OS_KEYS_SLOTS 2
#endif
// 256 x 32 (as the range sort's single class): 34.1 Gkeys/s for 64 Mi pairs
// against 31.0 with 384 x 20 and 32.1 with 256 x 28.
#ifndef MGPU_OS_SINGLE_THREADS
#define MGPU_OS_SINGLE_THREADS 256
#endif
#ifndef MGPU_OS_SINGLE_ITEMS
#define MGPU_OS_SINGLE_ITEMS 32
#endif
#ifndef MGPU_OS_SINGLE_MIN_BLOCKS
#define MGPU_OS_SINGLE_MIN_BLOCKS 2
#endif
#ifndef MGPU_OS_SINGLE_SLOTS
#define MGPU_OS_SINGLE_SLOTS 1
#endif
#ifndef MGPU_OS_MULTI_THREADS
#define MGPU_OS_MULTI_THREADS 256
#endif
#ifndef MGPU_OS_MULTI_ITEMS
#define MGPU_OS_MULTI_ITEMS 12
#endif
#ifndef MGPU_OS_MULTI_MIN_BLOCKS
#define MGPU_OS_MULTI_MIN_BLOCKS 2
#endif
#ifndef MGPU_OS_KEYS_BALLOT_BITS
#define MGPU_OS_KEYS_BALLOT_BITS 5
#endif
#ifndef MGPU_OS_SINGLE_BALLOT_BITS
#define MGPU_OS_SINGLE_BALLOT_BITS 5
#endif
#ifndef MGPU_OS_MULTI_BALLOT_BITS
#define MGPU_OS_MULTI_BALLOT_BITS 5
#endif
#ifndef MGPU_OS_KEYS_RANK_BATCH
#define MGPU_OS_KEYS_RANK_BATCH 8
#endif
#ifndef MGPU_OS_SINGLE_RANK_BATCH
#define MGPU_OS_SINGLE_RANK_BATCH 10
#endif
#ifndef MGPU_OS_MULTI_RANK_BATCH
#define MGPU_OS_MULTI_RANK_BATCH 6
#endif
