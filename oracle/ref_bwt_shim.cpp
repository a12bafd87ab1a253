// Builds the reference's host-side string quicksort of its BWT library,
// bwt/src/mgpubwt/cpusort.cpp (QSortStrings), from its source where it lies
// (the path is given by -DMGPU_REF_BWT_CPUSORT=...), as a shared library with
// a C ABI. TEST INFRASTRUCTURE ONLY: it pins the oracle's block sort of
// rotations to the reference's own comparison sort. Nothing of the
// reference is copied; the file is compiled in place. Its header chain
// needs <cstring> before it and the CUDA include directory on the path.
#include <cassert>
#include <cstring>

#include MGPU_REF_BWT_CPUSORT

extern "C" {

// cpusort.cpp:68-93 -- sorts the rotation starts in [left, right] by the
// count2 symbols at symbols + start.
void ref_bwt_qsort_strings(int* left, int* right, const unsigned char* symbols,
	int count2) {
	QSortStrings(left, right, symbols, count2);
}

}
