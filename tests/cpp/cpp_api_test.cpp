// C++ caller of the drop-in API, written the way the reference's examples
// call it (sort/src/simpletest2/simpletest2.cpp:40-157): a driver-API
// context, MgpuSort / MgpuSortData from mgpusort.hpp, attached buffers, a bit
// range, index mode with earlyExit, then sortArrayEx, sortHost and
// sortDevice. Every result is checked against std::stable_sort. Prints
// "cpp_api_test: OK" and exits 0 on success.
#include "mgpusort.hpp"

#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#define CHECK(x) do { if(!(x)) { std::printf("FAILED %s:%d %s\n", __FILE__, \
	__LINE__, #x); std::exit(1); } } while(0)

static std::vector<unsigned> stable_order(const std::vector<unsigned>& keys,
	int firstBit, int endBit) {
	std::vector<unsigned> order(keys.size());
	std::iota(order.begin(), order.end(), 0u);
	unsigned mask = endBit - firstBit >= 32 ? 0xffffffffu
		: ((1u << (endBit - firstBit)) - 1);
	std::stable_sort(order.begin(), order.end(), [&](unsigned a, unsigned b) {
		return ((keys[a] >> firstBit) & mask) < ((keys[b] >> firstBit) & mask);
	});
	return order;
}

static std::vector<unsigned> download(CUdeviceptr p, size_t n) {
	std::vector<unsigned> h(n);
	CHECK(CUDA_SUCCESS == cuMemcpyDtoH(h.data(), p, 4 * n));
	return h;
}

int main() {
	CHECK(CUDA_SUCCESS == cuInit(0));
	CUdevice dev;
	CHECK(CUDA_SUCCESS == cuDeviceGet(&dev, 0));
	CUcontext ctx;
	CHECK(CUDA_SUCCESS == cuDevicePrimaryCtxRetain(&ctx, dev));
	CHECK(CUDA_SUCCESS == cuCtxSetCurrent(ctx));

	MgpuSort engine("ignored/kernel/path/");
	{
		MgpuSort copy(engine);          // reference-counted copies
		MgpuSort assigned = copy;
		(void)assigned;
	}

	const int n = 100000;
	std::mt19937 gen(5489u);
	std::vector<unsigned> keys(n), idx(n), fl(n);
	for(int i = 0; i < n; ++i) {
		keys[i] = (gen() & ((1u << 18) - 1)) << 7 | (gen() & 0x7f);
		idx[i] = i;
		float f = std::sqrt((float)i);
		std::memcpy(&fl[i], &f, 4);
	}

	// Attached key and two value arrays, bits [7, 25).
	const size_t rounded = (n + 2047) / 2048 * 2048;
	CUdeviceptr dKeys, dV1, dV2;
	CHECK(CUDA_SUCCESS == cuMemAlloc(&dKeys, 4 * rounded));
	CHECK(CUDA_SUCCESS == cuMemAlloc(&dV1, 4 * rounded));
	CHECK(CUDA_SUCCESS == cuMemAlloc(&dV2, 4 * rounded));
	CHECK(CUDA_SUCCESS == cuMemcpyHtoD(dKeys, keys.data(), 4 * n));
	CHECK(CUDA_SUCCESS == cuMemcpyHtoD(dV1, idx.data(), 4 * n));
	CHECK(CUDA_SUCCESS == cuMemcpyHtoD(dV2, fl.data(), 4 * n));
	{
		MgpuSortData data;
		data.AttachKey(dKeys);
		data.AttachVal(0, dV1);
		data.AttachVal(1, dV2);
		CHECK(SORT_STATUS_SUCCESS == data.Alloc(engine, n, 2));
		data.firstBit = 7;
		data.endBit = 25;
		CHECK(SORT_STATUS_SUCCESS == sortArray(engine, &data));
		std::vector<unsigned> k = download(data.keys[0], n);
		std::vector<unsigned> v1 = download(data.values1[0], n);
		std::vector<unsigned> v2 = download(data.values2[0], n);
		std::vector<unsigned> order = stable_order(keys, 7, 25);
		for(int i = 0; i < n; ++i) {
			CHECK(k[i] == keys[order[i]]);
			CHECK(v1[i] == idx[order[i]]);
			CHECK(v2[i] == fl[order[i]]);
		}
		// The attached buffers are at [parity] now.
		CHECK(data.keys[data.parity] == dKeys);
		data.Reset();                   // frees only the library's buffers
	}

	// Index mode over the full range with earlyExit (low 7 and top 7 bits
	// are not all equal here, so passes run; output must be exact).
	CHECK(CUDA_SUCCESS == cuMemcpyHtoD(dKeys, keys.data(), 4 * n));
	{
		MgpuSortData data;
		data.AttachKey(dKeys);
		CHECK(SORT_STATUS_SUCCESS == data.Alloc(engine, n, -1));
		data.firstBit = 0;
		data.endBit = 32;
		data.earlyExit = true;
		CHECK(SORT_STATUS_SUCCESS == sortArray(engine, &data));
		std::vector<unsigned> k = download(data.keys[0], n);
		std::vector<unsigned> v = download(data.values1[0], n);
		std::vector<unsigned> order = stable_order(keys, 0, 32);
		for(int i = 0; i < n; ++i) {
			CHECK(v[i] == order[i]);
			CHECK(k[i] == keys[order[i]]);
		}
	}

	// sortArrayEx with 4-bit passes on a library-created sortData_d.
	{
		sortData_t data = nullptr;
		CHECK(SORT_STATUS_SUCCESS == sortCreateData(engine, n, 1, &data));
		CHECK(CUDA_SUCCESS == cuMemcpyHtoD(data->keys[0], keys.data(), 4 * n));
		CHECK(CUDA_SUCCESS == cuMemcpyHtoD(data->values1[0], idx.data(), 4 * n));
		data->firstBit = 3;
		data->endBit = 29;
		CHECK(SORT_STATUS_SUCCESS == sortArrayEx(engine, data, 128, 8, 4, false));
		CHECK(data->parity == 1);       // 7 passes of 4 (two of 3) bits
		std::vector<unsigned> v = download(data->values1[0], n);
		std::vector<unsigned> order = stable_order(keys, 3, 29);
		for(int i = 0; i < n; ++i) CHECK(v[i] == order[i]);
		CHECK(SORT_STATUS_INVALID_VALUE == sortArrayEx(engine, data, 64, 8, 4, false));
		CHECK(SORT_STATUS_SUCCESS == sortDestroyData(data));
	}

	// sortHost and sortDevice.
	{
		std::vector<unsigned> k(keys), v(idx);
		CHECK(SORT_STATUS_SUCCESS == sortHost(engine, k.data(), v.data(), n, 24));
		std::vector<unsigned> order = stable_order(keys, 0, 24);
		for(int i = 0; i < n; ++i) CHECK(v[i] == order[i] && k[i] == keys[order[i]]);

		CHECK(CUDA_SUCCESS == cuMemcpyHtoD(dKeys, keys.data(), 4 * n));
		CHECK(CUDA_SUCCESS == cuMemcpyHtoD(dV1, idx.data(), 4 * n));
		CHECK(SORT_STATUS_SUCCESS == sortDevice(engine, dKeys, dV1, n, 24));
		std::vector<unsigned> kd = download(dKeys, n), vd = download(dV1, n);
		for(int i = 0; i < n; ++i) CHECK(vd[i] == order[i] && kd[i] == keys[order[i]]);
	}

	try {
		throw MgpuException(SORT_STATUS_INVALID_VALUE);
	} catch(const std::exception& e) {
		CHECK(std::strcmp(e.what(), "SORT_STATUS_INVALID_VALUE") == 0);
	}

	cuMemFree(dKeys);
	cuMemFree(dV1);
	cuMemFree(dV2);
	std::printf("cpp_api_test: OK\n");
	return 0;
}
