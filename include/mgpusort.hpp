/*
 * mgpusort.hpp -- header-only C++ helpers over the C ABI of mgpusort.h.
 *
 * Same classes, members and ownership rules as Modern GPU's
 * inc/mgpusort.hpp:12-114, so C++ callers of that header compile unchanged:
 *   MgpuException  -- a sortStatus_t thrown as an exception (:12-20)
 *   MgpuSortData   -- a sortData_d that owns the buffers the library
 *                     allocated and leaves the ones the caller attached
 *                     (:24-81); attachment is tracked per original slot, so
 *                     Reset() finds attached buffers after parity swaps
 *   MgpuSort       -- an engine handle with reference-counted copies
 *                     (:83-114)
 */
#ifndef MGPUSORT_B200_MGPUSORT_HPP
#define MGPUSORT_B200_MGPUSORT_HPP

#include "mgpusort.h"

#include <cstring>
#include <exception>
#include <utility>

struct MgpuException : std::exception {
	explicit MgpuException(sortStatus_t status) : _status(status) { }

	virtual const char* what() const throw() {
		const char* s = sortStatusString(_status);
		return s ? s : "unknown sortStatus_t";
	}

	sortStatus_t _status;
};

struct MgpuSortData : sortData_d {
	MgpuSortData() { Clear(); }
	~MgpuSortData() { Reset(); }

	// Free the library's buffers, leave the attached ones, zero everything.
	void Reset() {
		for(int i = 0; i < 2; ++i) {
			// A buffer attached at slot i sits at slot i ^ parity now.
			if(_attachedKeys[i]) keys[i ^ parity] = 0;
			for(int j = 0; j < 6; ++j)
				if(_attachedVals[j][i]) values[j][i ^ parity] = 0;
		}
		sortFreeData(this);
		Clear();
	}

	// Allocate every buffer that is not attached (sortAllocData).
	sortStatus_t Alloc(sortEngine_t engine, int maxElements_, int valueCount_) {
		maxElements = maxElements_;
		numElements = maxElements_;
		valueCount = valueCount_;
		return sortAllocData(engine, this);
	}

	void AttachKey(CUdeviceptr p, int i = 0) {
		keys[i] = p;
		_attachedKeys[i ^ parity] = true;
	}
	void AttachKey(unsigned int* p, int i = 0) {
		pKeys[i] = p;
		_attachedKeys[i ^ parity] = true;
	}
	void AttachVal(int j, CUdeviceptr p, int i = 0) {
		values[j][i] = p;
		_attachedVals[j][i ^ parity] = true;
	}
	void AttachVal(int j, unsigned int* p, int i = 0) {
		pValues[j][i] = p;
		_attachedVals[j][i ^ parity] = true;
	}

private:
	MgpuSortData(const MgpuSortData&);
	MgpuSortData& operator=(const MgpuSortData&);

	void Clear() {
		std::memset(static_cast<sortData_d*>(this), 0, sizeof(sortData_d));
		std::memset(_attachedKeys, 0, sizeof(_attachedKeys));
		std::memset(_attachedVals, 0, sizeof(_attachedVals));
	}

	bool _attachedKeys[2];
	bool _attachedVals[6][2];
};

class MgpuSort {
public:
	// Creates an engine; throws MgpuException on failure.
	explicit MgpuSort(const char* kernelPath) {
		sortStatus_t status = sortCreateEngine(kernelPath, &_engine);
		if(SORT_STATUS_SUCCESS != status) throw MgpuException(status);
	}

	// Shares an existing engine (one more reference).
	MgpuSort(sortEngine_t engine) : _engine(engine) {
		if(_engine) sortIncEngine(_engine);
	}

	MgpuSort(const MgpuSort& rhs) : _engine(rhs._engine) {
		if(_engine) sortIncEngine(_engine);
	}

	~MgpuSort() {
		if(_engine) sortReleaseEngine(_engine);
	}

	MgpuSort& operator=(const MgpuSort& rhs) {
		MgpuSort copy(rhs);
		std::swap(_engine, copy._engine);
		return *this;
	}

	operator sortEngine_t() { return _engine; }

private:
	sortEngine_t _engine;
};

#endif /* MGPUSORT_B200_MGPUSORT_HPP */
