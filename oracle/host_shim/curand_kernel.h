// TEST INFRASTRUCTURE ONLY: host stand-in for the random-number header.  The host build covers the
// reference's mechanics and diffusion (FM_update, PreLOD, LODsolver), which draw no random
// numbers; its RNG kernels still have to compile, so these declarations exist, and a call aborts.
#pragma once
#include <cstdio>
#include <cstdlib>

struct curandState {
    unsigned s[12];
};
inline void curand_init(unsigned long long, unsigned long long, unsigned long long, curandState*) {
    std::fprintf(stderr, "host build of the reference: random draws are not part of this build\n");
    std::abort();
}
inline float curand_uniform(curandState*) {
    std::fprintf(stderr, "host build of the reference: random draws are not part of this build\n");
    std::abort();
}
