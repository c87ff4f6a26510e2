/*
 * pscbfm_main.cpp -- command-line simulator, the counterpart of the
 * reference's src/pscbfm/mainCUDASimulatorGPUScBFM_AB_Type.cpp (same options,
 * :25-54 and :79-120).  It reads the last conformation of a .bfm file, runs
 * the colored BFM sweep on the GPU through the drop-in
 * UpdaterGPUScBFM_AB_Type class (include/UpdaterGPUScBFM_AB_Type.h), and
 * appends a conformation to the output file after every save interval, as
 * the reference's TaskManager loop with AnalyzerWriteBfmFile does (:157-176).
 *
 *   pscbfm -i in.bfm -e x.seeds -o out.bfm -m MCS -s SAVE -g GPU -r RNG
 *   pscbfm --dry-run -i in.bfm -o out.bfm     (read and rewrite, no GPU)
 */
#include <getopt.h>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <random>
#include <string>

#include "UpdaterGPUScBFM_AB_Type.h"
#include "bfm_io.hpp"

static void printHelp()
{
    std::cout << "usage: pscbfm [options]\n"
              << "\n"
              << "Colored bond-fluctuation-model sweep on the GPU (B200)\n"
              << "\n"
              << "    -e, --seeds <file path>\n"
              << "        seed file for reproducible runs: at least 250 unsigned 32-bit values\n"
              << "    -i, --initial-state <file path>\n"
              << "        (required) BFM file; its last conformation is simulated\n"
              << "    -m, --max-mcs <integer>\n"
              << "        (required) total Monte-Carlo steps to simulate\n"
              << "    -r, --rng <integer>\n"
              << "        random number generator: 1: IntHash, 2: Saru\n"
              << "    -s, --save-interval <integer>\n"
              << "        append the conformation to the output file every <integer> steps\n"
              << "    -o, --output <file path>\n"
              << "        output file (default outfile.bfm)\n"
              << "    -g, --gpu <integer>\n"
              << "        GPU to use\n"
              << "    -d, --dry-run\n"
              << "        read the input and write it to the output file without simulating\n"
              << "    -v, --version\n";
}

int main(int argc, char **argv)
{
    using hrclock = std::chrono::high_resolution_clock;
    const auto tProgram0 = hrclock::now();
    std::string infile, outfile = "outfile.bfm", seedFileName;
    uint32_t maxMcs = 0, saveInterval = 0;
    int gpu = 0, rngToUse = -1;
    bool dryRun = false;
    if (argc <= 1) {
        printHelp();
        return 0;
    }
    static struct option opts[] = {{"seeds", required_argument, 0, 'e'},       {"gpu", required_argument, 0, 'g'},
                                   {"help", no_argument, 0, 'h'},              {"initial-state", required_argument, 0, 'i'},
                                   {"max-mcs", required_argument, 0, 'm'},     {"output", required_argument, 0, 'o'},
                                   {"rng", required_argument, 0, 'r'},         {"save-interval", required_argument, 0, 's'},
                                   {"version", no_argument, 0, 'v'},           {"dry-run", no_argument, 0, 'd'},
                                   {0, 0, 0, 0}};
    for (;;) {
        int idx = 0;
        const int c = getopt_long(argc, argv, "e:g:hi:m:o:r:s:vd", opts, &idx);
        if (c == -1) break;
        switch (c) {
        case 'e': seedFileName = optarg; break;
        case 'g': gpu = std::atoi(optarg); break;
        case 'h': printHelp(); return 0;
        case 'i': infile = optarg; break;
        case 'm': maxMcs = (uint32_t)std::atol(optarg); break;
        case 'o': outfile = optarg; break;
        case 'r': rngToUse = std::atoi(optarg); break;
        case 's': saveInterval = (uint32_t)std::atol(optarg); break;
        case 'd': dryRun = true; break;
        case 'v': std::cout << "pscbfm (pscbfm_b200)\n"; return 0;
        default: std::cerr << "Unknown option\n"; return 1;
        }
    }
    try {
        if (infile.empty()) throw std::invalid_argument("-i/--initial-state is required");
        bfmio::Conformation conf = bfmio::read_bfm(infile);
        const auto ids = conf.bondIds.empty() ? bfmio::standard_bond_ids() : conf.bondIds;
        if (dryRun) {
            bfmio::write_header(outfile, conf, ids);
            bfmio::append_frame(outfile, conf, ids);
            return 0;
        }
        if (maxMcs == 0) throw std::invalid_argument("-m/--max-mcs is required");
        if (saveInterval == 0) saveInterval = maxMcs;

        /* seed the colour/seed generator (:122-127) and draw the values the
         * reference's main draws once before it starts (:132-134) */
        if (!seedFileName.empty()) {
            const auto w = bfmio::read_seeds(seedFileName);
            bfm_r250_seed_words(w.data(), w.size());
        } else {
            std::random_device rd;
            bfm_r250_seed(((uint64_t)rd() << 32) | rd());
        }
        (void)bfm_r250_rand32();
        (void)bfm_r250_rand32();

        UpdaterGPUScBFM_AB_Type<int32_t> u;
        u.setGpu(gpu);
        if (rngToUse != -1) u.setRng((UpdaterGPUScBFM_AB_Type<int32_t>::Rng)rngToUse);
        u.setAge(conf.age);
        u.setPeriodicity(conf.periodic[0], conf.periodic[1], conf.periodic[2]);
        u.setLatticeSize(conf.box[0], conf.box[1], conf.box[2]);
        u.setNrOfAllMonomers(conf.n);
        for (uint32_t i = 0; i < conf.n; ++i) u.setMonomerCoordinates(i, conf.xyz[3 * i], conf.xyz[3 * i + 1], conf.xyz[3 * i + 2]);
        for (uint32_t i = 0; i < conf.n; ++i) u.setAttribute(i, conf.attr[i]);
        for (uint32_t i = 0; i < conf.n; ++i)
            for (uint32_t k : conf.nbr[i]) u.setConnectivity(i, k);
        std::map<std::array<int, 3>, int> allowed;
        for (auto &kv : ids) allowed[kv.second] = 1;
        for (int dx = -4; dx < 4; ++dx)
            for (int dy = -4; dy < 4; ++dy)
                for (int dz = -4; dz < 4; ++dz) u.copyBondSet(dx, dy, dz, !allowed.count({dx, dy, dz}));
        u.initialize();

        bfmio::write_header(outfile, conf, ids);
        bfmio::append_frame(outfile, conf, ids);
        const auto t0 = hrclock::now();
        const uint32_t rounds = maxMcs / saveInterval;
        for (uint32_t r = 0; r < rounds; ++r) {
            u.setAge(conf.age);
            u.runSimulationOnGPU(saveInterval);
            for (uint32_t i = 0; i < conf.n; ++i) {
                conf.xyz[3 * i] = u.getMonomerPositionInX(i);
                conf.xyz[3 * i + 1] = u.getMonomerPositionInY(i);
                conf.xyz[3 * i + 2] = u.getMonomerPositionInZ(i);
            }
            conf.age += saveInterval;
            bfmio::append_frame(outfile, conf, ids);
        }
        const double dt = std::chrono::duration<double>(hrclock::now() - t0).count();
        std::cerr << "tTaskLoop = " << dt << "s\n";
        std::cerr << "mcs " << conf.age << " with " << (double)rounds * saveInterval * conf.n / dt << " [attempted moves/s]\n";
    } catch (std::exception const &e) {
        std::cerr << "[pscbfm] Caught exception: " << e.what() << std::endl;
        return 1;
    }
    std::cerr << "tProgram = " << std::chrono::duration<double>(hrclock::now() - tProgram0).count() << "s\n";
    return 0;
}
