// Oracle pin (test infrastructure): prints the first N outputs of libstdc++'s
// std::mt19937 for a seed, so the MT19937 restatement can be checked against an
// independent implementation.  Usage: mt_std_check <seed> <count> [skip]
#include <cstdio>
#include <cstdlib>
#include <random>

int main(int argc, char **argv) {
    if (argc < 3) return 2;
    unsigned long seed = std::strtoul(argv[1], nullptr, 10);
    long count = std::strtol(argv[2], nullptr, 10);
    long skip = argc > 3 ? std::strtol(argv[3], nullptr, 10) : 0;
    std::mt19937 g(static_cast<std::mt19937::result_type>(seed));
    if (skip > 0) g.discard(static_cast<unsigned long long>(skip));
    for (long i = 0; i < count; i++) std::printf("%u\n", static_cast<unsigned>(g()));
    return 0;
}
