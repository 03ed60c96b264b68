// ORACLE PIN SHIM — TEST INFRASTRUCTURE ONLY.
// Stand-in for LeMonADE's RandomNumberGenerators, which is not in the reference tree. The
// reference updater calls r250_rand32() twice per sub-step (colour, then sub-step seed,
// src/pscbfm/CRITICAL.cu:509-510); here each call hands out the next word of a draw list that
// the test supplies (oracle/ref_harness.cu), so the reference and the oracle consume the same
// stream.
#pragma once
#include <cstdint>
extern "C" uint32_t bfmref_next_draw(void);
class RandomNumberGenerators
{
public:
    uint32_t r250_rand32() { return bfmref_next_draw(); }
};
