// hashparams.cpp -- the HashOrder hash parameters, drawn the way the reference draws them.
// TEST INFRASTRUCTURE ONLY (the oracle's source of (a_j, b_j), independent of the engine).
//
// btc/operations/reorder.h:495-506: one std::mt19937 seeded with 42, and for each hash
// function j a braced HashInitFunctor{dist(rng), dist(rng)} -- a_j then b_j -- with
// dist = std::uniform_int_distribution<uint32_t>(1, 4294967290).
#include <cstdint>
#include <random>

extern "C" void oracle_hashorder_params(int num_hashes, uint32_t* a, uint32_t* b)
{
    std::mt19937 rng(42);
    std::uniform_int_distribution<uint32_t> dist(1, 4294967290u);
    for (int j = 0; j < num_hashes; ++j) {
        a[j] = dist(rng);
        b[j] = dist(rng);
    }
}
