/*
 * oracle/ref_shim/LeMonADE/utility/RandomNumberGenerators.h -- TEST INFRASTRUCTURE.
 *
 * Stand-in for LeMonADE's RandomNumberGenerators (an un-vendored submodule,
 * .gitmodules:1-3).  The reference updater only calls r250_rand32()
 * (UpdaterGPUScBFM_AB_Type.cu:3065-3066).  Like LeMonADE, the generator state
 * is process-global and shared by every instance; it is the published R250
 * restated in oracle/r250.h, seeded through oracle_ref_r250_state().
 */
#pragma once
#include <cstdint>
#include <string>
#include "../../../r250.h"

inline orc::R250State &oracle_ref_r250_state()
{
    static orc::R250State s = [] {
        orc::R250State t;
        orc::r250_seed_u64(t, 0);
        return t;
    }();
    return s;
}

class RandomNumberGenerators {
public:
    uint32_t r250_rand32() { return orc::r250_next(oracle_ref_r250_state()); }
    double r250_drand() { return r250_rand32() * (1.0 / 4294967296.0); }
    void seedAll() { orc::r250_seed_u64(oracle_ref_r250_state(), 0); }
};
