/*
 * UpdaterGPUScBFM_AB_Type.h -- header-only C++ drop-in for the reference's
 * UpdaterGPUScBFM_AB_Type<T> (src/pscbfm/UpdaterGPUScBFM_AB_Type.h:177-518),
 * forwarding every method to the C ABI of libpscbfm_b200.so
 * (pscbfm_b200.h).  The LeMonADE adapter GPUScBFM_AB_Type<Ingredients>
 * (GPUScBFM_AB_Type.h) and the pscbfm simulator compile against it unchanged
 * and link with -lpscbfm_b200.
 *
 * Same method names, dependency order (.h:457-470) and exception types: the
 * reference's std::invalid_argument / std::runtime_error are thrown for the
 * corresponding status codes.  The template parameter (the reference's
 * device coordinate type) does not change the device layout here, which is
 * always 32-bit Z-order codes plus image counters.
 */
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "pscbfm_b200.h"

template <typename T_UCoordinateCuda>
class UpdaterGPUScBFM_AB_Type {
public:
    using T_BoxSize = uint64_t;
    using T_Coordinate = int32_t;
    using T_Id = uint32_t;

    enum class Rng { IntHash = 1, Saru = 2, Philox = 3, Pcg = 4, Xorwow = 5 };

    UpdaterGPUScBFM_AB_Type() { check(bfm_create(&mHandle)); }
    virtual ~UpdaterGPUScBFM_AB_Type() { destruct(); }
    UpdaterGPUScBFM_AB_Type(UpdaterGPUScBFM_AB_Type const &) = delete;
    UpdaterGPUScBFM_AB_Type &operator=(UpdaterGPUScBFM_AB_Type const &) = delete;

    void destruct()
    {
        if (mHandle) bfm_destroy(mHandle);
        mHandle = nullptr;
    }

    void setGpu(int iGpuToUse) { check(bfm_set_gpu(mHandle, iGpuToUse)); }
    void copyBondSet(int dx, int dy, int dz, bool bondForbidden) { check(bfm_copy_bond_set(mHandle, dx, dy, dz, bondForbidden ? 1 : 0)); }
    void setNrOfAllMonomers(T_Id nAllMonomers)
    {
        check(bfm_set_nr_of_all_monomers(mHandle, nAllMonomers));
        mPositions.assign(3 * (size_t)nAllMonomers, 0);
    }
    void setAttribute(T_Id i, int32_t attribute) { check(bfm_set_attribute(mHandle, i, attribute)); }
    void setMonomerCoordinates(T_Id i, T_Coordinate x, T_Coordinate y, T_Coordinate z)
    {
        check(bfm_set_monomer_coordinates(mHandle, i, x, y, z));
        if (3 * (size_t)i + 2 < mPositions.size()) {
            mPositions[3 * (size_t)i] = x;
            mPositions[3 * (size_t)i + 1] = y;
            mPositions[3 * (size_t)i + 2] = z;
        }
    }
    void setConnectivity(T_Id monoidx1, T_Id monoidx2) { check(bfm_set_connectivity(mHandle, monoidx1, monoidx2)); }
    void setLatticeSize(T_BoxSize boxX, T_BoxSize boxY, T_BoxSize boxZ) { check(bfm_set_lattice_size(mHandle, boxX, boxY, boxZ)); }
    void setPeriodicity(bool isPeriodicX, bool isPeriodicY, bool isPeriodicZ)
    {
        check(bfm_set_periodicity(mHandle, isPeriodicX, isPeriodicY, isPeriodicZ));
    }
    void setAge(int64_t rAge) { check(bfm_set_age(mHandle, rAge)); }
    int64_t getAge() const
    {
        int64_t a = 0;
        bfm_get_age(mHandle, &a);
        return a;
    }
    void setRng(Rng x) { check(bfm_set_rng(mHandle, (int)x)); }
    Rng getRng() const
    {
        int r = 1;
        bfm_get_rng(mHandle, &r);
        return (Rng)r;
    }
    void setStepsBetweenSortings(int64_t n)
    {
        check(bfm_set_steps_between_sortings(mHandle, n));
        mSteps = n;
    }
    int64_t getStepsBetweenSortings() const { return mSteps; }

    void initialize() { check(bfm_initialize(mHandle)); }
    bool execute() { return true; }
    void cleanup() { check(bfm_cleanup(mHandle)); }

    /* synchronous like the reference: positions are valid on return */
    void runSimulationOnGPU(uint32_t nrMCS_per_Call)
    {
        check(bfm_run(mHandle, nrMCS_per_Call));
        check(bfm_get_positions(mHandle, mPositions.data(), mPositions.size() / 3));
    }

    int32_t getMonomerPositionInX(T_Id i) { return mPositions.at(3 * (size_t)i); }
    int32_t getMonomerPositionInY(T_Id i) { return mPositions.at(3 * (size_t)i + 1); }
    int32_t getMonomerPositionInZ(T_Id i) { return mPositions.at(3 * (size_t)i + 2); }

private:
    void check(int status) const
    {
        if (status == BFM_OK) return;
        std::string msg = mHandle ? bfm_last_error(mHandle) : "bfm_create failed";
        if (status == BFM_EINVAL) throw std::invalid_argument(msg);
        throw std::runtime_error(msg);
    }

    bfm_handle *mHandle = nullptr;
    std::vector<int32_t> mPositions;
    int64_t mSteps = 5000;
};
