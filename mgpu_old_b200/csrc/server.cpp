// Sort server: a request loop that keeps a pool of device memory and several
// engines (one per stream slot), admits sort requests against a device-memory
// budget, coalesces small requests of the same kind (value mode and bit
// range) into one batched segmented sort, and runs batches on different
// streams so that copies and sorts of different batches overlap on the GPU.
// Requests that arrive while others are in flight join the next batch as soon
// as a slot and budget free up (continuous batching). No counterpart in the
// reference, whose callers issue one blocking sortArray per array.

// The library is built with hidden visibility; the C ABI is all it exports.
#pragma GCC visibility push(default)
#include "../../include/mgpusort.h"
#include "../../include/mgpusort_b200.h"
#pragma GCC visibility pop
#include "engine_internal.h"

#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
	unsigned long long ticket = 0;
	const unsigned* keys = nullptr;
	const unsigned* values = nullptr;
	unsigned* keysOut = nullptr;
	unsigned* valuesOut = nullptr;
	int n = 0;
	int firstBit = 0;
	int endBit = 32;
	size_t bytes = 0;               // device bytes while in flight
	Clock::time_point submitted;
	Clock::time_point finished;
	sortStatus_t status = SORT_STATUS_SUCCESS;
	bool done = false;
	int kind() const { return (values ? 1 : 0) | (firstBit << 1) | (endBit << 7); }
};

struct Slot {
	cudaStream_t stream = nullptr;
	sortEngine_t engine = nullptr;
	cudaEvent_t done = nullptr;
	int* hostOffsets = nullptr;     // pinned, maxBatchRequests + 1
	bool busy = false;
	// The batch in flight on this slot.
	std::vector<Request*> reqs;
	size_t bytes = 0;
	sortStatus_t status = SORT_STATUS_SUCCESS;
};

// Device footprint of a request: two buffers for keys, two for values.
size_t request_bytes(int n, bool values) {
	return (size_t)n * sizeof(unsigned) * 2 * (values ? 2 : 1);
}

} // namespace

struct sortServer_d {
	int device = 0;
	sortServerConfig cfg;
	cudaMemPool_t pool = nullptr;
	std::vector<Slot> slots;
	std::mutex mu;
	std::condition_variable wake;   // scheduler: new requests / shutdown
	std::condition_variable doneCv; // waiters
	std::deque<Request*> pending;   // FIFO, not yet in a batch
	std::unordered_map<unsigned long long, std::unique_ptr<Request>> requests;
	unsigned long long nextTicket = 1;
	size_t budgetUsed = 0;
	bool stopping = false;
	std::thread scheduler;
};

namespace {

template<typename T> cudaError_t alloc_async(T** p, size_t bytes, cudaMemPool_t pool,
	cudaStream_t s) {
	return cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), bytes, pool, s);
}

// Copies in, sort, copies out and frees, all ordered on the slot's stream.
sortStatus_t launch_batch(sortServer_d* srv, Slot& slot, std::vector<Request*>& batch) {
	cudaMemPool_t pool = srv->pool;
	cudaStream_t s = slot.stream;
	const bool hasValues = batch[0]->values != nullptr;
	long long total = 0;
	for(Request* r : batch) total += r->n;
	const size_t bytes = (size_t)total * sizeof(unsigned);
	unsigned* k[2] = {};
	unsigned* v[2] = {};
	int* offsets = nullptr;
	bool ok = alloc_async(&k[0], bytes, pool, s) == cudaSuccess &&
		alloc_async(&k[1], bytes, pool, s) == cudaSuccess;
	if(ok && hasValues)
		ok = alloc_async(&v[0], bytes, pool, s) == cudaSuccess &&
			alloc_async(&v[1], bytes, pool, s) == cudaSuccess;
	const bool segmented = batch.size() > 1;
	if(ok && segmented)
		ok = alloc_async(&offsets, sizeof(int) * (batch.size() + 1), pool, s) == cudaSuccess;
	sortStatus_t status = ok ? SORT_STATUS_SUCCESS : SORT_STATUS_DEVICE_ALLOC_FAILED;

	long long at = 0;
	for(size_t i = 0; status == SORT_STATUS_SUCCESS && i < batch.size(); ++i) {
		Request* r = batch[i];
		slot.hostOffsets[i] = (int)at;
		const size_t b = (size_t)r->n * sizeof(unsigned);
		if(cudaMemcpyAsync(k[0] + at, r->keys, b, cudaMemcpyHostToDevice, s) != cudaSuccess ||
			(hasValues && cudaMemcpyAsync(v[0] + at, r->values, b, cudaMemcpyHostToDevice, s)
				!= cudaSuccess))
			status = SORT_STATUS_DEVICE_ERROR;
		at += r->n;
	}
	slot.hostOffsets[batch.size()] = (int)at;

	sortData_d d;
	std::memset(&d, 0, sizeof(d));
	d.maxElements = d.numElements = (int)total;
	d.valueCount = hasValues ? 1 : 0;
	d.firstBit = batch[0]->firstBit;
	d.endBit = batch[0]->endBit;
	d.keys[0] = reinterpret_cast<CUdeviceptr>(k[0]);
	d.keys[1] = reinterpret_cast<CUdeviceptr>(k[1]);
	d.values1[0] = reinterpret_cast<CUdeviceptr>(v[0]);
	d.values1[1] = reinterpret_cast<CUdeviceptr>(v[1]);
	if(status == SORT_STATUS_SUCCESS) {
		if(segmented) {
			if(cudaMemcpyAsync(offsets, slot.hostOffsets, sizeof(int) * (batch.size() + 1),
				cudaMemcpyHostToDevice, s) != cudaSuccess)
				status = SORT_STATUS_DEVICE_ERROR;
			else
				status = sortSegmentedArray(slot.engine, &d, offsets, (int)batch.size(),
					reinterpret_cast<CUstream>(s));
		} else {
			status = sortArrayAsync(slot.engine, &d, reinterpret_cast<CUstream>(s));
		}
	}
	at = 0;
	for(size_t i = 0; status == SORT_STATUS_SUCCESS && i < batch.size(); ++i) {
		Request* r = batch[i];
		const size_t b = (size_t)r->n * sizeof(unsigned);
		const unsigned* rk = reinterpret_cast<const unsigned*>(d.keys[0]) + at;
		const unsigned* rv = reinterpret_cast<const unsigned*>(d.values1[0]) + at;
		if(cudaMemcpyAsync(r->keysOut, rk, b, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
			(hasValues && cudaMemcpyAsync(r->valuesOut, rv, b, cudaMemcpyDeviceToHost, s)
				!= cudaSuccess))
			status = SORT_STATUS_DEVICE_ERROR;
		at += r->n;
	}
	// Stream-ordered frees: the memory returns to the pool after the copies.
	for(int i = 0; i < 2; ++i) {
		if(k[i]) cudaFreeAsync(k[i], s);
		if(v[i]) cudaFreeAsync(v[i], s);
	}
	if(offsets) cudaFreeAsync(offsets, s);
	cudaEventRecord(slot.done, s);
	cudaGetLastError();
	slot.status = status;
	return status;
}

void complete_batch(sortServer_d* srv, Slot& slot) {
	// The engine reports device-side errors of its sorts.
	sortStatus_t st = slot.status;
	if(st == SORT_STATUS_SUCCESS) st = sortSynchronize(slot.engine);
	const auto now = Clock::now();
	std::lock_guard<std::mutex> g(srv->mu);
	for(Request* r : slot.reqs) {
		r->status = st;
		r->finished = now;
		r->done = true;
	}
	srv->budgetUsed -= slot.bytes;
	slot.reqs.clear();
	slot.bytes = 0;
	slot.busy = false;
	srv->doneCv.notify_all();
}

void run_scheduler(sortServer_d* srv) {
	auto& slots = srv->slots;
	auto& pending = srv->pending;
	const sortServerConfig& cfg = srv->cfg;
	cudaSetDevice(srv->device);
	std::unique_lock<std::mutex> lk(srv->mu);
	while(true) {
		// Retire finished batches.
		bool anyBusy = false;
		for(Slot& slot : slots) {
			if(!slot.busy) continue;
			lk.unlock();
			const cudaError_t q = cudaEventQuery(slot.done);
			if(q == cudaSuccess) complete_batch(srv, slot);
			else if(q != cudaErrorNotReady) {
				cudaGetLastError();
				slot.status = SORT_STATUS_DEVICE_ERROR;
				complete_batch(srv, slot);
			}
			lk.lock();
			anyBusy = anyBusy || slot.busy;
		}
		if(srv->stopping && pending.empty() && !anyBusy) break;

		// Admit and launch while a slot is free: the head of the queue goes
		// first; small requests of its kind behind it join its batch while
		// the budget and the batch limits allow.
		bool launched = false;
		for(Slot& slot : slots) {
			if(slot.busy || pending.empty()) continue;
			Request* head = pending.front();
			if(srv->budgetUsed + head->bytes > cfg.memoryBudget && srv->budgetUsed > 0) break;
			std::vector<Request*> batch;
			size_t bytes = 0;
			long long elements = 0;
			if(head->n > cfg.coalesceMax) {
				batch.push_back(head);
				bytes = head->bytes;
				pending.pop_front();
			} else {
				const int kind = head->kind();
				for(auto it = pending.begin(); it != pending.end();) {
					Request* r = *it;
					if(r->kind() != kind || r->n > cfg.coalesceMax) { ++it; continue; }
					if(!batch.empty() &&
						((int)batch.size() >= cfg.maxBatchRequests ||
						 elements + r->n > cfg.maxBatchElements ||
						 srv->budgetUsed + bytes + r->bytes > cfg.memoryBudget)) break;
					batch.push_back(r);
					bytes += r->bytes;
					elements += r->n;
					it = pending.erase(it);
				}
			}
			srv->budgetUsed += bytes;
			slot.busy = true;
			slot.reqs = batch;
			slot.bytes = bytes;
			lk.unlock();
			// Errors of the launch reach the batch's requests when its event
			// (recorded regardless) completes.
			launch_batch(srv, slot, batch);
			lk.lock();
			launched = true;
		}
		if(launched) continue;
		// Nothing to launch: sleep until a submission or a short poll interval
		// (in-flight batches are polled, not waited on).
		srv->wake.wait_for(lk, std::chrono::microseconds(anyBusy ? 20 : 2000));
	}
}

} // namespace

extern "C" {

sortStatus_t SORTAPI sortServerCreate(const sortServerConfig* config,
	sortServer_t* server) {
	if(!server) return SORT_STATUS_INVALID_VALUE;
	*server = nullptr;
	auto s = std::make_unique<sortServer_d>();
	sortServerConfig c = {};
	if(config) c = *config;
	if(!c.memoryBudget) c.memoryBudget = (size_t)64 << 30;
	if(c.slots <= 0) c.slots = 4;
	if(c.coalesceMax <= 0) c.coalesceMax = 1 << 20;
	if(c.maxBatchElements <= 0) c.maxBatchElements = 1 << 24;
	if(c.maxBatchRequests <= 0) c.maxBatchRequests = 4096;
	s->cfg = c;
	if(cudaGetDevice(&s->device) != cudaSuccess) {
		cudaGetLastError();
		return SORT_STATUS_INVALID_CONTEXT;
	}
	// A pool that keeps what it has allocated (up to the budget) instead of
	// handing memory back to the driver after every batch.
	cudaMemPoolProps props = {};
	props.allocType = cudaMemAllocationTypePinned;
	props.location.type = cudaMemLocationTypeDevice;
	props.location.id = s->device;
	if(cudaMemPoolCreate(&s->pool, &props) != cudaSuccess) {
		cudaGetLastError();
		return SORT_STATUS_DEVICE_ALLOC_FAILED;
	}
	unsigned long long keep = c.memoryBudget;
	cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
	s->slots.resize(c.slots);
	for(Slot& slot : s->slots) {
		sortStatus_t st = sortCreateEngine(nullptr, &slot.engine);
		if(st != SORT_STATUS_SUCCESS) {
			sortServerDestroy(s.release());
			return st;
		}
		// Batches come from a memory pool at varying addresses and sizes:
		// their launch sequences seldom repeat, so slots launch directly
		// rather than capture graphs.
		sortEnableGraphs(slot.engine, 0);
		// Scratch for the largest coalesced batch, now: growing it while
		// serving would free device memory, which waits for every slot's work
		// and stalls the scheduler.
		st = engine_reserve_segmented(slot.engine, c.maxBatchElements, c.maxBatchRequests);
		if(st != SORT_STATUS_SUCCESS) {
			sortServerDestroy(s.release());
			return st;
		}
		void* h = nullptr;
		if(cudaStreamCreateWithFlags(&slot.stream, cudaStreamNonBlocking) != cudaSuccess ||
			cudaEventCreateWithFlags(&slot.done, cudaEventDisableTiming) != cudaSuccess ||
			cudaHostAlloc(&h, sizeof(int) * (c.maxBatchRequests + 1), cudaHostAllocDefault)
				!= cudaSuccess) {
			cudaGetLastError();
			sortServerDestroy(s.release());
			return SORT_STATUS_DEVICE_ERROR;
		}
		slot.hostOffsets = static_cast<int*>(h);
	}
	sortServer_d* raw = s.release();
	raw->scheduler = std::thread([raw] { run_scheduler(raw); });
	*server = raw;
	return SORT_STATUS_SUCCESS;
}

sortStatus_t SORTAPI sortServerSubmit(sortServer_t server, const unsigned* keys,
	const unsigned* values, int numElements, int firstBit, int endBit,
	unsigned* keysOut, unsigned* valuesOut, unsigned long long* ticket) {
	if(!server || !keys || !keysOut || !ticket || numElements < 1 ||
		firstBit < 0 || endBit > 32 || endBit <= firstBit || (values && !valuesOut))
		return SORT_STATUS_INVALID_VALUE;
	auto r = std::make_unique<Request>();
	r->keys = keys;
	r->values = values;
	r->keysOut = keysOut;
	r->valuesOut = valuesOut;
	r->n = numElements;
	r->firstBit = firstBit;
	r->endBit = endBit;
	r->bytes = request_bytes(numElements, values != nullptr);
	r->submitted = Clock::now();
	std::lock_guard<std::mutex> g(server->mu);
	if(r->bytes > server->cfg.memoryBudget) return SORT_STATUS_CONFIG_NOT_SUPPORTED;
	r->ticket = server->nextTicket++;
	*ticket = r->ticket;
	server->pending.push_back(r.get());
	server->requests.emplace(r->ticket, std::move(r));
	server->wake.notify_one();
	return SORT_STATUS_SUCCESS;
}

sortStatus_t SORTAPI sortServerPoll(sortServer_t server, unsigned long long ticket,
	int* done) {
	if(!server || !done) return SORT_STATUS_INVALID_VALUE;
	std::lock_guard<std::mutex> g(server->mu);
	auto it = server->requests.find(ticket);
	if(it == server->requests.end()) return SORT_STATUS_INVALID_VALUE;
	*done = it->second->done ? 1 : 0;
	return SORT_STATUS_SUCCESS;
}

sortStatus_t SORTAPI sortServerWait(sortServer_t server, unsigned long long ticket,
	double* latencySeconds) {
	if(!server) return SORT_STATUS_INVALID_VALUE;
	std::unique_lock<std::mutex> lk(server->mu);
	auto it = server->requests.find(ticket);
	if(it == server->requests.end()) return SORT_STATUS_INVALID_VALUE;
	Request* r = it->second.get();
	server->doneCv.wait(lk, [r] { return r->done; });
	const sortStatus_t st = r->status;
	if(latencySeconds)
		*latencySeconds = std::chrono::duration<double>(r->finished - r->submitted).count();
	server->requests.erase(it);
	return st;
}

sortStatus_t SORTAPI sortServerDestroy(sortServer_t server) {
	if(!server) return SORT_STATUS_INVALID_VALUE;
	{
		std::lock_guard<std::mutex> g(server->mu);
		server->stopping = true;
		server->wake.notify_all();
	}
	if(server->scheduler.joinable()) server->scheduler.join();
	for(Slot& slot : server->slots) {
		if(slot.stream) cudaStreamSynchronize(slot.stream);
		if(slot.engine) sortReleaseEngine(slot.engine);
		if(slot.done) cudaEventDestroy(slot.done);
		if(slot.stream) cudaStreamDestroy(slot.stream);
		if(slot.hostOffsets) cudaFreeHost(slot.hostOffsets);
	}
	if(server->pool) cudaMemPoolDestroy(server->pool);
	cudaGetLastError();
	delete server;
	return SORT_STATUS_SUCCESS;
}

} // extern "C"
