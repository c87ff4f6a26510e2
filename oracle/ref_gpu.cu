/*
 * oracle/ref_gpu.cu -- TEST INFRASTRUCTURE.
 *
 * A C-ABI wrapper around the reference's own, unmodified GPU updater
 * (src/pscbfm/UpdaterGPUScBFM_AB_Type.{h,cu}), compiled from the reference's
 * sources for sm_100a by oracle/Makefile into oracle/_ref/libref_pscbfm.so.
 * It drives the updater the way the LeMonADE adapter does
 * (GPUScBFM_AB_Type.h:121-184 set-up, :192-242 execute, :244-251 cleanup) so
 * that GPU tests can compare the product and the CPU oracle with the
 * reference's own kernels on the same inputs.
 */
#include <cstdint>
#include <cstring>
#include <exception>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "UpdaterGPUScBFM_AB_Type.h"

namespace {

struct RefBase {
    virtual ~RefBase() {}
    virtual void run(uint32_t nmcs) = 0;
    virtual void get(int32_t *pos3, uint32_t n) = 0;
    virtual int64_t age() = 0;
};

template <typename T>
struct Ref : RefBase {
    UpdaterGPUScBFM_AB_Type<T> u;
    void run(uint32_t nmcs) override { u.runSimulationOnGPU(nmcs); }
    void get(int32_t *pos3, uint32_t n) override
    {
        for (uint32_t i = 0; i < n; ++i) {
            pos3[3 * i] = u.getMonomerPositionInX(i);
            pos3[3 * i + 1] = u.getMonomerPositionInY(i);
            pos3[3 * i + 2] = u.getMonomerPositionInZ(i);
        }
    }
    int64_t age() override { return u.getAge(); }
};

/* periodicity (bit a: axis a periodic) of the next ref_create */
int g_periodic = 7;

template <typename T>
RefBase *make(int gpu, uint32_t Lx, uint32_t Ly, uint32_t Lz, uint32_t n, const int32_t *pos3,
              const uint32_t *nnbr, const uint32_t *nbr8, const uint8_t *allowed512, int rng, int64_t age,
              int64_t sortEvery)
{
    /* The adapter calls setGpu() first (GPUScBFM_AB_Type.h:131).  On this GPU
     * it throws: setGpu prints the device table, and getCudaCodeName
     * (cudacommon.hpp:1032-1043) returns 0 into a std::string for every
     * compute capability above 7.  The device is therefore selected with
     * cudaSetDevice; initialize() queries it itself (.cu:2535-2536). */
    if (cudaSetDevice(gpu) != cudaSuccess) throw std::runtime_error("cudaSetDevice failed");
    auto *r = new Ref<T>();
    auto &u = r->u;
    u.setRng((typename UpdaterGPUScBFM_AB_Type<T>::Rng)rng);
    u.setAge(age);
    u.setStepsBetweenSortings(sortEvery);
    u.setPeriodicity((g_periodic & 1) != 0, (g_periodic & 2) != 0, (g_periodic & 4) != 0);
    u.setLatticeSize(Lx, Ly, Lz);
    u.setNrOfAllMonomers(n);
    for (uint32_t i = 0; i < n; ++i) u.setMonomerCoordinates(i, pos3[3 * i], pos3[3 * i + 1], pos3[3 * i + 2]);
    for (uint32_t i = 0; i < n; ++i) u.setAttribute(i, 1);
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t j = 0; j < nnbr[i]; ++j) u.setConnectivity(i, nbr8[(size_t)i * 8 + j]);
    /* allowed512 is indexed by (dx&7)|(dy&7)<<3|(dz&7)<<6, the loop mirrors
     * GPUScBFM_AB_Type.h:168-175 */
    for (int dx = -4; dx < 4; ++dx)
        for (int dy = -4; dy < 4; ++dy)
            for (int dz = -4; dz < 4; ++dz)
                u.copyBondSet(dx, dy, dz, !allowed512[(dx & 7) | ((dy & 7) << 3) | ((dz & 7) << 6)]);
    u.initialize();
    return r;
}

thread_local std::string g_err;

} // namespace

extern "C" {

const char *ref_last_error() { return g_err.c_str(); }

/* setPeriodicity of the next ref_create (bit a: axis a periodic; default 7) */
void ref_set_periodicity(int mask) { g_periodic = mask; }

/* ctype: 0 = int32_t (the adapter's default instantiation), 1 = uint8_t,
 * 2 = uint16_t (GPUScBFM_AB_Type.h:253-285) */
void *ref_create(int gpu, int ctype, uint32_t Lx, uint32_t Ly, uint32_t Lz, uint32_t n, const int32_t *pos3,
                 const uint32_t *nnbr, const uint32_t *nbr8, const uint8_t *allowed512, int rng, int64_t age,
                 int64_t sortEvery)
{
    try {
        if (ctype == 1) return make<uint8_t>(gpu, Lx, Ly, Lz, n, pos3, nnbr, nbr8, allowed512, rng, age, sortEvery);
        if (ctype == 2) return make<uint16_t>(gpu, Lx, Ly, Lz, n, pos3, nnbr, nbr8, allowed512, rng, age, sortEvery);
        return make<int32_t>(gpu, Lx, Ly, Lz, n, pos3, nnbr, nbr8, allowed512, rng, age, sortEvery);
    } catch (std::exception const &e) {
        g_err = e.what();
        return nullptr;
    }
}

int ref_run(void *h, uint32_t nmcs)
{
    try {
        ((RefBase *)h)->run(nmcs);
        return 0;
    } catch (std::exception const &e) {
        g_err = e.what();
        return 1;
    }
}

/* runSimulationOnGPU with the reference's "Stats" log level active for its
 * updater (the constructor switches it off, .cu:1416-1423): the filter
 * analysis it prints to std::cerr (.cu:3348-3387) is returned as text, at
 * most cap - 1 bytes and NUL-terminated.  Returns the length of the full
 * text, or -1 when the run failed. */
long ref_run_stats(void *h, uint32_t nmcs, char *text, size_t cap)
{
    auto &logger = SelectiveLogger::getInstance();
    logger.activate("UpdaterGPUScBFM_AB_Type.cu", "Stats");
    std::ostringstream out;
    std::streambuf *saved = std::cerr.rdbuf(out.rdbuf());
    const int rc = ref_run(h, nmcs);
    std::cerr.rdbuf(saved);
    logger.deactivate("UpdaterGPUScBFM_AB_Type.cu", "Stats");
    const std::string s = out.str();
    if (text && cap) {
        const size_t m = s.size() < cap - 1 ? s.size() : cap - 1;
        std::memcpy(text, s.data(), m);
        text[m] = 0;
    }
    return rc == 0 ? (long)s.size() : -1;
}

void ref_get(void *h, int32_t *pos3, uint32_t n) { ((RefBase *)h)->get(pos3, n); }
int64_t ref_age(void *h) { return ((RefBase *)h)->age(); }
void ref_destroy(void *h) { delete (RefBase *)h; }

void ref_r250_set(const uint32_t *state251)
{
    auto &s = oracle_ref_r250_state();
    std::memcpy(s.buf, state251, sizeof(s.buf));
    s.idx = state251[250];
}
void ref_r250_get(uint32_t *state251)
{
    auto &s = oracle_ref_r250_state();
    std::memcpy(state251, s.buf, sizeof(s.buf));
    state251[250] = s.idx;
}

} /* extern "C" */
