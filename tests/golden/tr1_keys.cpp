// Prints the keys that the reference's example sort/src/simpletest2/
// simpletest2.cpp:61-71 sorts: a default-seeded std::tr1::mt19937 driving
// std::tr1::uniform_int over [0, 2^18 - 1], each draw shifted left by 7.
// Used only by make_golden.py to build a committed fixture.
#include <cstdio>
#include <cstdlib>
#include <tr1/random>

int main(int argc, char** argv) {
	int n = argc > 1 ? std::atoi(argv[1]) : 128;
	std::tr1::mt19937 gen;
	std::tr1::uniform_int<unsigned> dist(0, (1u << 18) - 1);
	for(int i = 0; i < n; ++i) std::printf("%u\n", dist(gen) << 7);
	return 0;
}
