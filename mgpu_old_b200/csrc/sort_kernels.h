// Host-visible interface of the sort kernels (sort_kernels.cu): the device
// control block, the pass plan and the launchers the engine calls.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

namespace mgpusort {

// A pass sorts by a digit of at most 8 bits; a 32-bit range needs at most 32
// passes (sortArrayEx with bitPass = 1) and the digit histograms of all
// passes of one plan take at most 4 * 256 bins.
constexpr int kMaxPasses = 32;
constexpr int kMaxBins = 1024;
constexpr int kDigitBins = 256;

// Device control block, one per engine. The upsweep adds every key's digits
// into hist, and its last CTA turns hist into the exclusive offsets, sets
// trivial[p] when pass p has a single non-empty digit, and zeroes hist and
// ticket again. So the block is clean after every complete sort and needs a
// memset only after an error (the error word).
struct Control {
	unsigned hist[kMaxBins];
	unsigned offsets[kMaxBins];
	unsigned trivial[kMaxPasses];
	unsigned ticket;
	unsigned error;
	// Tile counters of the onesweep passes (one per executed pass): each CTA
	// draws its tile from the counter, in launch order. The upsweep zeroes
	// them at the start of every sort.
	unsigned tileCounter[kMaxPasses];
	// Arrivals at the grid-wide barriers of the cooperative sort (zeroed
	// before each launch).
	unsigned coopBarrier;
	unsigned reserved[61];
};

// Digit layout of a sort: pass p sorts by bits [shift[p], shift[p] +
// width[p]) and its histogram lives at hist[binBase[p] .. + 2^width[p]).
struct PassPlan {
	int numPasses;
	int shift[kMaxPasses];
	int width[kMaxPasses];
	int binBase[kMaxPasses];
	int totalBins;
};

// One pass reads keysIn (and valsIn[0..v)) and writes keysOut (valsOut).
struct PassBuffers {
	const unsigned* keysIn;
	unsigned* keysOut;
	const unsigned* valsIn[6];
	unsigned* valsOut[6];
};

// Value modes of a pass: -1 writes each key's source position into
// valsOut[0] (index mode, first pass), 0 moves keys only, 1..6 moves that many
// value arrays with the keys.
constexpr int kValueIndex = -1;

// A pass splits its tiles into at most this many ranges (one CTA each).
constexpr int kMaxRanges = 1024;

// Device scratch of a pass: per-range digit counts and their exclusive
// prefixes over ranges (digit-major, [256][kMaxRanges] each) and the digit
// totals [256]. Reused by every pass; nothing in it needs clearing.
constexpr size_t kPassScratchWords = 2 * (size_t)kDigitBins * kMaxRanges
	+ kDigitBins;

// Elements per tile of the sort kernel for a value mode.
int pass_tile_elements(int valueMode);

// Bytes of the pass scratch (kPassScratchWords words).
size_t pass_scratch_bytes();

// Configure kernel attributes (dynamic shared memory) of every kernel,
// onesweep's included; call once per device.
cudaError_t configure_kernels();
cudaError_t configure_onesweep_kernels();
cudaError_t configure_coop_kernels();

// Cooperative sort (keys only, index mode or one value array): every pass
// of the plan in one launch of co-resident CTAs with grid-wide barriers
// between the count, scan and sort phases. Pass 0 reads buf.*In and writes
// buf.*Out, later passes alternate, so the result lies in buf.*Out after an
// odd number of passes and in buf.*In after an even one. Zeroes
// ctrl->coopBarrier first. Used for sorts of at most coop_max_elements().
int coop_max_elements();
cudaError_t launch_coop_sort(const PassBuffers& buf, int valueMode, int n,
	const PassPlan& plan, Control* ctrl, unsigned* scratch, bool useBulk,
	volatile unsigned* hostError, int numSMs, cudaStream_t stream);

// Digit histograms of every pass of `plan` in one read of the keys, their
// exclusive scans and the per-pass "single digit" flags (earlyExit).
cudaError_t launch_upsweep(const unsigned* keys, int n, const PassPlan& plan,
	Control* ctrl, volatile unsigned* hostError, int numSMs,
	cudaStream_t stream);

// One pass (count, scan and sort kernels) by the digit of plan pass `pass`.
// useBulk: every buffer of the pass is 16-byte aligned, so full tiles are
// staged with bulk copies; otherwise every tile uses plain loads.
// failTile >= 0 makes the CTA that sorts that tile run a bounded wait out
// (fault injection for tests); -1 in normal use.
cudaError_t launch_pass(const PassBuffers& buf, int valueMode, int n,
	int pass, const PassPlan& plan, Control* ctrl, unsigned* scratch,
	bool useBulk, int failTile, volatile unsigned* hostError, int numSMs,
	cudaStream_t stream);

// The two halves of launch_pass: the count and scan kernels, then the sort
// kernel (the engine times them separately).
cudaError_t launch_pass_count(const PassBuffers& buf, int valueMode, int n,
	int pass, const PassPlan& plan, unsigned* scratch, int numSMs,
	cudaStream_t stream);
cudaError_t launch_pass_sort(const PassBuffers& buf, int valueMode, int n,
	int pass, const PassPlan& plan, Control* ctrl, unsigned* scratch,
	bool useBulk, int failTile, volatile unsigned* hostError, int numSMs,
	cudaStream_t stream);

// Segmented sort (sortSegmentedArray). Device scratch for n elements in
// numSegments segments; all three launchers take the same scratch.
size_t seg_scratch_bytes(int n, int numSegments);

// Classify the segments of device `offsets` (numSegments + 1 entries) into
// the work lists in scratch. Bad offsets set an error and empty lists.
cudaError_t launch_seg_plan(const int* offsets, int numSegments, int n,
	int valueMode, void* scratch, Control* ctrl, volatile unsigned* hostError,
	cudaStream_t stream);

// Sort every segment of at most 4096 elements through all passes of `plan`,
// from buf.*In into buf.*Out (which may alias).
cudaError_t launch_seg_small(const PassBuffers& buf, int valueMode,
	const PassPlan& plan, const int* offsets, int numSegments, int n,
	void* scratch, int numSMs, cudaStream_t stream);

// One pass over the larger segments (count, scan and sort kernels).
cudaError_t launch_seg_pass(const PassBuffers& buf, int valueMode, int pass,
	const PassPlan& plan, const int* offsets, int numSegments, int n,
	void* scratch, Control* ctrl, bool useBulk, volatile unsigned* hostError,
	int numSMs, cudaStream_t stream);

cudaError_t launch_iota(unsigned* out, int n, cudaStream_t stream);

// Arrays of at most small_array_max_elements() elements: one CTA sorts the
// whole array through every pass of `plan` in shared memory, from buf.*In
// into buf.*Out (which may alias).
int small_array_max_elements();
cudaError_t launch_small_array(const PassBuffers& buf, int valueMode, const PassPlan& plan,
	int n, cudaStream_t stream);

// Onesweep passes (onesweep.cu): one launch per pass, with the digit offsets
// of every pass from one upsweep and each tile's offsets from a decoupled
// lookback over its predecessors' published digit counts.
//
// Elements per tile of the onesweep pass kernel for a value mode; all modes
// of one sort (index mode, then one value array) share a tile size.
int onesweep_tile_elements(int valueMode);

// Bytes of one lookback buffer for n elements (tiles x 256 64-bit words);
// the engine keeps two, used by alternate executed passes.
size_t onesweep_status_bytes(int n, int valueMode);

// The upsweep of a onesweep sort: every pass's digit histogram and exclusive
// offsets and single-digit flags (as launch_upsweep), and it zeroes the
// tile counters and the first `statusBytes` bytes (a multiple of 4) of
// status0, the first executed pass's lookback buffer.
cudaError_t launch_onesweep_upsweep(const unsigned* keys, int n, const PassPlan& plan,
	Control* ctrl, void* status0, size_t statusBytes, volatile unsigned* hostError,
	int numSMs, cudaStream_t stream);

// One onesweep pass by the digit of plan pass `pass`, the `exec`-th executed
// pass of the sort (0-based): it draws tiles from ctrl->tileCounter[exec],
// looks back in status[exec & 1] and clears status[(exec + 1) & 1] for the
// next executed pass.
cudaError_t launch_onesweep_pass(const PassBuffers& buf, int valueMode, int n,
	int pass, int exec, const PassPlan& plan, Control* ctrl, void* const status[2],
	bool useBulk, int failTile, volatile unsigned* hostError, int numSMs,
	cudaStream_t stream);

// Key types with an order-preserving uint32 image (sortArrayTyped).
constexpr int kKeyUint32 = 0;
constexpr int kKeyInt32 = 1;
constexpr int kKeyFloat32 = 2;

// Maps n keys in place to their uint32 radix image (forward) or back.
cudaError_t launch_key_transform(unsigned* keys, int n, int keyType, bool forward,
	cudaStream_t stream);

} // namespace mgpusort
