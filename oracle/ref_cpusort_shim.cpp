// Builds the reference's own CPU radix sort demo,
// sort/src/cpusort/cpusort.cpp, from its source where it lies (the path is
// given by -DMGPU_REF_CPUSORT=...), as a shared library with a C ABI. TEST
// INFRASTRUCTURE ONLY: it pins the oracle to the reference's CPU code on the
// inputs that code handles (keys only). Nothing of the reference is copied:
// the file is compiled in place, its main() renamed out of the way.
#include <algorithm>
#include <cstdio>
#include <cstddef>

// The reference targets 32-bit builds, where size_t and unsigned are one
// type, so std::min(count - index, blockSize) (cpusort.cpp:136, 180)
// deduces a single type. On LP64 they differ; this overload gives the call
// its 32-bit meaning.
namespace std {
inline size_t min(size_t a, unsigned b) { return a < b ? a : (size_t)b; }
}

#define main mgpu_ref_cpusort_demo_main
#include MGPU_REF_CPUSORT
#undef main

extern "C" {

// cpusort.cpp:68-72 -- eight sequential 4-bit passes over 32-bit keys.
void ref_cpusort_sort1(unsigned* keys, size_t count) { Sort1(keys, count); }

// cpusort.cpp:188-192 -- eight blocked 4-bit passes.
void ref_cpusort_sort2(unsigned* keys, size_t count, unsigned blockSize) {
	Sort2(keys, count, blockSize);
}

// cpusort.cpp:122-186 -- one blocked pass over bits [bit, bit + numBits).
void ref_cpusort_sort2pass(unsigned* keys, unsigned bit, unsigned numBits,
	size_t count, unsigned blockSize) {
	Sort2Pass(keys, bit, numBits, count, blockSize);
}

}
