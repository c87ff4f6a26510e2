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

#include <algorithm>
#include <cstdint>
#include <iostream>
#include <ostream>
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

    /* The reference's per-updater log switch (its SelectedLogger mLog,
     * .h:225; the adapter's activateLogging calls mLog.activate(level),
     * GPUScBFM_AB_Type.h:97-106).  Only "Stats" changes anything here: while
     * it is active every runSimulationOnGPU counts the filters as the
     * reference does and prints the analysis to std::cerr after the run, as
     * the reference does (.cu:3348-3387). */
    struct LogLevels {
        std::vector<std::string> active;
        void activate(std::string const &level)
        {
            if (!isActive(level)) active.push_back(level);
        }
        void deactivate(std::string const &level) { active.erase(std::remove(active.begin(), active.end(), level), active.end()); }
        bool isActive(std::string const &level) const { return std::find(active.begin(), active.end(), level) != active.end(); }
    };
    LogLevels mLog;

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
        const bool stats = mLog.isActive("Stats");
        check(bfm_set_filter_stats(mHandle, stats ? 1 : mFilterMode));
        check(bfm_run(mHandle, nrMCS_per_Call));
        check(bfm_get_positions(mHandle, mPositions.data(), mPositions.size() / 3));
        if (stats) printFilterAnalysis(std::cerr);
    }

    /* The reference prints its filter analysis when its "Stats" log level
     * is active (.cu:2917-2936, :3348-3387).  Here: setFilterStats(1) for
     * the reference's numbers (2: the moves made, 0: off), then
     * printFilterAnalysis after a run writes them in the reference's format. */
    void setFilterStats(int mode)
    {
        check(bfm_set_filter_stats(mHandle, mode));
        mFilterMode = mode;
    }
    void printFilterAnalysis(std::ostream &os) const
    {
        static const char *const names[5] = {"Box Boundaries", "Invalid Bonds", "Volume Exclusion",
                                             "! Invalid Bonds && Volume Exclusion",
                                             "! Invalid Bonds && ! Volume Exclusion && Parallel Volume Exclusion"};
        uint32_t k = 0;
        check(bfm_get_nspecies(mHandle, &k));
        std::vector<double> st(25 * (size_t)k);
        check(bfm_get_filter_stats(mHandle, st.data(), st.size()));
        os << "Filter analysis. Format:\n" << "Filter Reason: min | mean +- stddev | max\n";
        for (uint32_t g = 0; g < k; ++g) {
            size_t n = 0;
            check(bfm_get_species_order(mHandle, g, nullptr, 0, &n));
            const double pct = 100. / (double)n;
            os << "\n=== Group " << char('A' + g) << " (" << n << ") ===\n";
            for (int f = 0; f < 5; ++f) {
                const double *v = &st[((size_t)g * 5 + f) * 5];
                os << names[f] << ": " << v[0] << "(" << pct * v[0] << "%) | " << v[1] << "(" << pct * v[1]
                   << "%) +- " << v[2] << " | " << v[3] << "(" << pct * v[3] << "%)\n";
            }
            const double *v1 = &st[((size_t)g * 5 + 1) * 5], *v3 = &st[((size_t)g * 5 + 3) * 5];
            const double left = (double)n - (v1[1] * v1[4] + v3[1] * v3[4]) / v3[4];
            os << "Remaining after 1st kernel: " << left << "(" << pct * left << "%)\n";
        }
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
    int mFilterMode = 0;
};
