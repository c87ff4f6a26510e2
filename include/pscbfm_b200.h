/*
 * pscbfm_b200.h -- C ABI of the B200-native colored bond-fluctuation-model
 * (BFM) sweep.
 *
 * One handle is one simulated system, with the life cycle of the reference's
 * UpdaterGPUScBFM_AB_Type<T> (src/pscbfm/UpdaterGPUScBFM_AB_Type.h:177-518):
 * setters -> bfm_initialize -> bfm_run (any number of times) -> read back ->
 * bfm_cleanup / bfm_destroy.  Each entry point below names the reference
 * method it replaces.  All functions return a status code (BFM_OK on
 * success); bfm_last_error() gives the message of the last failure on that
 * handle.  Plain pointers and sizes only: the library owns every device
 * buffer, the caller owns the host buffers it passes in.
 *
 * Threading: one host thread per handle; handles are independent (each has
 * its own stream and keeps its box constants in kernel arguments, unlike the
 * reference's global __constant__ tables, .cu:84-133).
 */
#ifndef PSCBFM_B200_H
#define PSCBFM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
enum {
    BFM_OK = 0,
    BFM_EINVAL = 1,      /* invalid argument: the reference throws std::invalid_argument */
    BFM_ERUNTIME = 2,    /* invalid state / bond set / box: the reference throws std::runtime_error */
    BFM_ECUDA = 3,       /* a CUDA call failed (the reference exit()s, cudacommon.hpp:36-51) */
    BFM_ETIMEOUT = 4,    /* a bounded device-side wait gave up */
    BFM_ENOTINIT = 5,    /* call needs bfm_initialize first */
    BFM_EUNSUPPORTED = 6, /* feature not provided by this build */
    BFM_ETOOLARGE = 7     /* size beyond the fixed maximum of bfm_substep_noalloc */
};

/* random number generators, numbering of the reference's enum class Rng
 * (UpdaterGPUScBFM_AB_Type.h:413-420) */
enum { BFM_RNG_INTHASH = 1, BFM_RNG_SARU = 2, BFM_RNG_PHILOX = 3, BFM_RNG_PCG = 4, BFM_RNG_XORWOW = 5 };

typedef struct bfm_handle bfm_handle;

/* constructor / destructor: UpdaterGPUScBFM_AB_Type() / ~UpdaterGPUScBFM_AB_Type()
 * (UpdaterGPUScBFM_AB_Type.h:453-454) */
int bfm_create(bfm_handle **out);
int bfm_destroy(bfm_handle *h);
const char *bfm_last_error(const bfm_handle *h);

/* setGpu (UpdaterGPUScBFM_AB_Type.h:490) */
int bfm_set_gpu(bfm_handle *h, int gpu);
/* copyBondSet (.h:491), dx, dy, dz in [-4, 3]; forbidden != 0 marks a forbidden bond */
int bfm_copy_bond_set(bfm_handle *h, int dx, int dy, int dz, int forbidden);
/* setNrOfAllMonomers (.h:492); may be called once per set-up */
int bfm_set_nr_of_all_monomers(bfm_handle *h, uint32_t n);
/* setAttribute (.h:493); stored, not used for the colouring */
int bfm_set_attribute(bfm_handle *h, uint32_t i, int32_t attribute);
/* setMonomerCoordinates (.h:494) */
int bfm_set_monomer_coordinates(bfm_handle *h, uint32_t i, int32_t x, int32_t y, int32_t z);
/* setConnectivity (.h:495): directed, the caller adds both directions; at most 8 per monomer */
int bfm_set_connectivity(bfm_handle *h, uint32_t i, uint32_t j);
/* setLatticeSize (.h:496): powers of two, 8 <= L <= 1024 per axis */
int bfm_set_lattice_size(bfm_handle *h, uint64_t bx, uint64_t by, uint64_t bz);
/* setPeriodicity (.h:505).  Along a non-periodic axis the box has walls: a
 * cube corner takes the coordinates 0 .. L-2 and a move that would leave
 * them is refused (the check of .cu:988-996 for unsigned coordinates, with
 * each axis' own size); initialize refuses a monomer outside the walls. */
int bfm_set_periodicity(bfm_handle *h, int px, int py, int pz);
/* setAge / getAge (.h:506-507) */
int bfm_set_age(bfm_handle *h, int64_t age);
int bfm_get_age(const bfm_handle *h, int64_t *age);
/* setRng / getRng (.h:508-509); IntHash (default, as .cu:1407), Saru, Philox */
int bfm_set_rng(bfm_handle *h, int rng);
int bfm_get_rng(const bfm_handle *h, int *rng);
/* setStepsBetweenSortings (.h:513), default 5000 (.cu:1379) */
int bfm_set_steps_between_sortings(bfm_handle *h, int64_t steps);

/* bulk variants of setMonomerCoordinates / setConnectivity for large systems:
 * xyz holds 3*n int32; deg holds n counts, nbr8 holds 8 ids per monomer */
int bfm_set_all_coordinates(bfm_handle *h, const int32_t *xyz, size_t n);
int bfm_set_all_connectivity(bfm_handle *h, const uint8_t *deg, const uint32_t *nbr8, size_t n);

/* initialize (.h:485, .cu:2393-2537): colouring, species slabs, lattices, first spatial sort */
int bfm_initialize(bfm_handle *h);
/* runSimulationOnGPU (.h:498, .cu:2902-3400): nmcs Monte-Carlo steps;
 * synchronous, positions can be read back on return */
int bfm_run(bfm_handle *h, uint32_t nmcs);
/* getMonomerPositionInX/Y/Z (.h:501-503) */
int bfm_get_monomer_position(bfm_handle *h, uint32_t i, int32_t *x, int32_t *y, int32_t *z);
/* all positions (unfolded, as doCopyBack .cu:3402-3484 returns them), 3*n
 * int32; a page-locked buffer (cudaHostAlloc'd or registered) is filled by
 * one device-to-host copy, any other through the engine's staging buffer */
int bfm_get_positions(bfm_handle *h, int32_t *xyz, size_t n);

/* ---- chain analysis on the device (the reference's AnalyzerMsd,
 * src/AnalyzerMsd.tpp, for systems of linear chains) ----
 * Chains, their end monomers and middle monomer are found once by the
 * reference analyzer's rule (AnalyzerMsd.tpp:193-280); BFM_EINVAL when the
 * bond graph is not a set of linear chains. */
int bfm_analyzer_init(bfm_handle *h, uint32_t *n_chains);
/* Observables of the current state, computed on the device:
 * out[0] chains, out[1] <R_e^2>, out[2] <R_g^2>, out[3..7] g1..g5 against the
 * time origin (first, middle, last monomer, chain centre of mass -- each
 * minus the box centre-of-mass drift when there is more than one chain --
 * and middle monomer minus chain centre of mass; AnalyzerMsd.tpp:392-421;
 * zero before an origin is set), out[8..10] the box centre of mass, and
 * with n_out >= 12 out[11] the end-to-end vector autocorrelation against the
 * origin, sum_c R_c(t).R_c(0) / sum_c |R_c(0)|^2 (0 before an origin).
 * set_origin != 0 makes the current state the time origin afterwards. */
int bfm_analyze(bfm_handle *h, int set_origin, double *out, size_t n_out);
/* original monomer ids of every chain's first end, middle and last end */
int bfm_analyzer_chain_ids(bfm_handle *h, uint32_t *first, uint32_t *middle, uint32_t *last, uint32_t n_chains);
/* per-chain R_e^2, R_g^2 and centre of mass (x, y, z per chain) of the last bfm_analyze */
int bfm_analyze_per_chain(bfm_handle *h, double *re2, double *rg2, double *com, uint32_t n_chains);

/* The reference's "Stats" filter analysis (runSimulationOnGPU with the
 * "Stats" log active: .cu:2917-2936, :3141-3152, :3186-3197, :3316-3330,
 * printed at :3348-3387).  While on, bfm_run runs the per-substep kernels
 * (same trajectory) and counts, per colour substep,
 *   [0] moves out of the box (non-periodic axes; the reference never fills it),
 *   [1] invalid bonds, [2] occupied leading faces, [3] occupied leading
 *   faces with valid bonds (kernelCountFilteredCheck, .cu:1033-1097),
 *   [4] parallel refusals (kernelCountFilteredPerform, .cu:1192-1216).
 * mode 1 reproduces the reference's printed numbers: filters 0-3 for
 * IntHash directions whatever the RNG (.cu:1030-1032); filter 4 after the
 * move (an accepted monomer is tested from its new corner), and with
 * checkFront's byte fetch on the reference's bit-packed target lattice
 * (UpdaterGPUScBFM_AB_Type.h:30, .cu:420-428, :1213): a face site s counts
 * when any target bit of sites 8s .. 8s+7 is set and s < Lx*Ly*Lz/8.
 * mode 2 counts the moves made: this RNG's directions, filter 4 = the
 * candidates refused.  Mode 0 (default) is off.
 * bfm_get_filter_stats: for the last run, per species s and filter f,
 * out[(s * 5 + f) * 5 + 0..4] = min, mean, standard deviation (the
 * reference's n/(n-1) form, .cu:3363-3366, NaN for one substep), max over
 * the substeps of that species, and the number of those substeps (the
 * reference's ns); n_out >= 25 * species; zeros where the species did not run. */
int bfm_set_filter_stats(bfm_handle *h, int mode);
int bfm_get_filter_stats(const bfm_handle *h, double *out, size_t n_out);

/* ---- batched ensembles: many independent systems in one persistent launch.
 * No counterpart class in the reference; each system follows exactly the
 * trajectory of a single updater (this library's bfm_* handle, and so the
 * reference's runSimulationOnGPU, .cu:2902-3400) started from the same
 * positions, bonds, bond set, RNG, age, sorting interval and R250 state:
 * the colour and seed of every substep come from the system's own R250
 * stream, drawn on the device.  Box edges may be any multiple of 8 in
 * 8 .. 1024 (the reference needs powers of two); boxes are periodic; at
 * most 16 colours per system. */
typedef struct bfm_batch bfm_batch;
int bfm_batch_create(int gpu, bfm_batch **out);
int bfm_batch_destroy(bfm_batch *b);
const char *bfm_batch_last_error(const bfm_batch *b);
/* Adds one system (before bfm_batch_initialize).  pos3: n x (x, y, z)
 * unfolded corners; deg: bonds per monomer; nbr8: 8 partner ids per monomer;
 * allowed512: 1 for an allowed bond, index (dx&7)|(dy&7)<<3|(dz&7)<<6
 * (108 allowed, as initializeBondTable requires, .cu:1516-1559); rng as
 * BFM_RNG_*; r250_state251: 250 R250 words and the index (as
 * bfm_r250_get_state gives), or NULL to seed it from r250_seed as
 * bfm_r250_seed does.  *sys receives the system's index. */
int bfm_batch_add_system(bfm_batch *b, uint32_t Lx, uint32_t Ly, uint32_t Lz, uint32_t n, const int32_t *pos3, const uint8_t *deg,
                         const uint32_t *nbr8, const uint8_t *allowed512, int rng, int64_t age, int64_t sort_every,
                         const uint32_t *r250_state251, uint64_t r250_seed, uint32_t *sys);
/* colours, slabs, lattices and device state of every system (initialize,
 * .cu:2393-2537, per system) */
int bfm_batch_initialize(bfm_batch *b);
/* systems whose lattice exceeds 64^3 (padded) are shared by a cluster of
 * `size` CTAs: 2, 4 (default; 1 also selects it) or 8; 0 runs every system
 * on one CTA.  Every size gives the same trajectories. */
int bfm_batch_set_clusters(bfm_batch *b, int size);
/* autotuner: the next bfm_batch_run times, on trial launches (each an
 * eighth of the longest pending work, 2 .. 50 MCS; part of the run, same
 * trajectories), first the cluster sizes 4, 2, 8 and off, then 1 and 4
 * monomers per thread in flight against the default 2, then the cluster
 * kernel also for systems of 48^3..64^3 sites (whose lattices otherwise sit
 * in one CTA's shared memory); at every stage the default stays unless a
 * candidate is more than 3% faster per attempted move.  Trials that affect
 * no system of the batch are skipped. */
int bfm_batch_set_autotune(bfm_batch *b, int on);
/* fix the tile shape by hand: monomers in flight per thread (1, 2, 4) and
 * whether systems above 32^3 sites also go to the cluster kernel */
int bfm_batch_set_shape(bfm_batch *b, int in_flight, int clusters_from_48);
/* the shape in use and the autotuner's seven trials (ns per attempted move,
 * 0 = skipped; order as in bfm_batch_set_autotune); any pointer may be NULL */
int bfm_batch_get_tuning(const bfm_batch *b, int *cluster_size, int *in_flight, uint32_t *cluster_above_words, int *tuned,
                         double *trial_ns_per_move7);
/* the cluster size in use, whether the autotuner has chosen it, and its four
 * trial times (ns per attempted move, sizes 4, 2, 8, off; any pointer may be NULL) */
int bfm_batch_get_clusters(const bfm_batch *b, int *size, int *tuned, double *trial_ns_per_move4);
/* system s advances by mcs[s] Monte-Carlo steps (0 leaves it as it is); nsys
 * must equal the number of systems */
int bfm_batch_run(bfm_batch *b, const uint32_t *mcs, size_t nsys);
/* unfolded positions of system sys, original monomer order (doCopyBack, .cu:3402-3484) */
int bfm_batch_get_positions(bfm_batch *b, uint32_t sys, int32_t *pos3, size_t n);
/* positions of every system at once: systems in the order added, each in
 * its original monomer order (n_total >= all monomers; 3 ints each) */
int bfm_batch_get_all_positions(bfm_batch *b, int32_t *pos3, size_t n_total);
/* unfolded positions of m selected monomers (3 ints each, in the order
 * asked): ids[k] = (system index << 32) | original monomer id.  For
 * observables of many systems between runs (molecule ends for R_e^2 and
 * the end-to-end autocorrelation) without reading whole ensembles back.
 * No counterpart in the reference (one system per updater there). */
int bfm_batch_gather_positions(bfm_batch *b, const uint64_t *ids, size_t m, int32_t *pos3);
/* age, R250 state (251 words) and counters (attempts, candidates, accepts) of system sys; any pointer may be NULL */
int bfm_batch_get_state(bfm_batch *b, uint32_t sys, int64_t *age, uint32_t *r250_state251, uint64_t *counters3);
/* occupation bits of system sys (Z-order of the box padded to powers of two); *needed receives the word count */
int bfm_batch_get_lattice(bfm_batch *b, uint32_t sys, uint32_t *words, size_t nwords, size_t *needed);
/* systems, monomers, largest colour count; time, launches and attempted moves of the last bfm_batch_run */
int bfm_batch_info(const bfm_batch *b, uint32_t *nsys, uint64_t *monomers, uint32_t *nspecies_max, double *last_ms,
                   uint64_t *last_launches, uint64_t *last_attempts);

/* ---- the learned schedule's network (no counterpart in the reference):
 * in -> 128 -> 128 -> out with ReLU, trained and evaluated on the GPU by the
 * library's own kernel on the tcgen05 tensor cores (bf16 operands in shared
 * memory, fp32 accumulators in tensor memory; fp32 master parameters and
 * Adam moments; forward, backward and Adam of many steps in one cooperative
 * launch).  Parameters are one fp32 vector [W1 (hidden x in), b1,
 * W2 (hidden x hidden), b2, W3 (out x hidden), b3], row-major (out x in);
 * He-uniform start from seed.  Widths: in and out 1..16, hidden 128.
 * x: batch x in, y and targets: batch x out, row-major host arrays;
 * out_weight (NULL = all 1) weights the squared error of each output;
 * loss = sum_o w_o (y - t)^2 averaged over the batch. */
typedef struct bfm_mlp bfm_mlp;
int bfm_mlp_create(int gpu, uint32_t n_in, uint32_t n_hidden, uint32_t n_out, uint64_t seed, bfm_mlp **out);
int bfm_mlp_destroy(bfm_mlp *m);
const char *bfm_mlp_last_error(const bfm_mlp *m);
int bfm_mlp_num_params(const bfm_mlp *m, size_t *n);
/* setting the parameters also resets the Adam moments */
int bfm_mlp_set_params(bfm_mlp *m, const float *params, size_t n);
int bfm_mlp_get_params(bfm_mlp *m, float *params, size_t n);
int bfm_mlp_forward(bfm_mlp *m, const float *x, uint32_t batch, float *y);
/* loss and its gradient with respect to every parameter (no update) */
int bfm_mlp_gradients(bfm_mlp *m, const float *x, const float *y_target, const float *out_weight, uint32_t batch, float *grad,
                      size_t n, float *loss);
/* one Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the batch; *loss is the loss before the step */
int bfm_mlp_train_step(bfm_mlp *m, const float *x, const float *y_target, const float *out_weight, uint32_t batch, float lr,
                       float *loss);
/* n_steps Adam steps in one launch over a data set of n_rows rows: step s
 * takes the step_rows[s] rows listed next in row_index (indices < n_rows);
 * losses[s] (may be NULL) is the loss of step s before its update.  The
 * same as n_steps calls of bfm_mlp_train_step on those rows, bit for bit. */
int bfm_mlp_train_steps(bfm_mlp *m, const float *x, const float *y_target, const float *out_weight, uint32_t n_rows,
                        const uint32_t *row_index, const uint32_t *step_rows, uint32_t n_steps, float lr, float *losses);
/* device time of the latest forward / gradients / training launch, in ms */
int bfm_mlp_last_ms(const bfm_mlp *m, double *ms);

/* cleanup (.h:487, .cu:3486-3502): frees the set-up; setters may be used again */
int bfm_cleanup(bfm_handle *h);

/* diagnostics used by the parity tests */
/* the occupation bit lattice, Z-order, 32-bit words (bit i of word w = site 32*w+i) */
int bfm_get_lattice(bfm_handle *h, uint32_t *words, size_t nwords);
int bfm_get_lattice_words(const bfm_handle *h, size_t *nwords);
int bfm_get_nspecies(const bfm_handle *h, uint32_t *nspecies);
/* colour of every monomer (after initialize) */
int bfm_get_colors(const bfm_handle *h, uint32_t *colors, size_t n);
/* original ids of species sp in slot order (the RNG subsequence order); *count receives the size */
int bfm_get_species_order(bfm_handle *h, uint32_t sp, uint32_t *ids, size_t cap, size_t *count);
/* [attempted moves, candidates after the check kernel, accepted moves] since initialize */
int bfm_get_counters(bfm_handle *h, uint64_t out3[3]);
/* device time of the kernels of the last bfm_run, milliseconds (CUDA events on the handle's stream) */
int bfm_get_last_run_ms(const bfm_handle *h, double *ms);
/* kernel launches issued by the last bfm_run */
int bfm_get_last_run_launches(const bfm_handle *h, uint64_t *launches);
/* runs nmcs Monte-Carlo steps like bfm_run (same trajectory) with CUDA
 * events on the handle's stream around every sweep-kernel launch (CUDA
 * graphs replaced by direct launches): summed device time in ms, number of
 * launches and attempted moves covered */
int bfm_time_kernels(bfm_handle *h, uint32_t nmcs, double *ms, uint64_t *launches, uint64_t *attempts);
/* launch path: 0 = one persistent cooperative kernel per schedule chunk
 * (default); 1 = one check + one perform kernel per colour substep, captured
 * in CUDA graphs; 2 = the same kernels launched one by one */
int bfm_set_launch_mode(bfm_handle *h, int mode);
/* shape of the persistent kernel chosen at initialize: mode 0 = bonds tested
 * from the partners' positions, 1 = from stored bond codes, 2 = stored codes
 * with the CTA's slab segments staged in shared memory by bulk copies, 6..8 =
 * stored codes with the independent work of each substep done inside the
 * grid-barrier waits, 9, 10 the same on one cluster of 8 or 16 CTAs
 * (negative: -launch path of the per-substep kernels);
 * CTAs, threads per CTA and dynamic shared memory per CTA */
int bfm_get_launch_info(const bfm_handle *h, int *mode, int *grid, int *threads, size_t *smem_bytes);
/* force a shape of the persistent kernel (tests, tuning): -1 automatic
 * (default), 0 gather, 1 stored codes, 2 staged; 3..5 the same with the
 * candidate lists in global instead of shared memory (1 and 4 test the
 * bonds of every item first and the leading face only of the items that
 * pass); 6..8 windowed with
 * 1, 2, 4 items per thread in flight (one CTA per SM, grid barriers; 8
 * tests the bonds of every item first and the leading face only of the
 * items that pass, the automatic shape from 2048 items of a colour per SM
 * on, 7 below);
 * 9, 10 windowed with 2 in flight on one thread-block cluster of 8 or 16
 * CTAs (hardware cluster barriers; small systems).
 * BFM_ERUNTIME when the shape does not fit this system. */
int bfm_set_sweep_shape(bfm_handle *h, int shape);
/* launch-shape autotuner (no counterpart in the reference, whose launch
 * configuration is fixed, UpdaterGPUScBFM_AB_Type.cu:2952-2981): with `on`,
 * the first schedule chunk of the next run is split into equal pieces: one
 * untimed piece of the automatic shape (warm caches), then two rounds of
 * trial launches of the automatic shape, the windowed shapes 6..10, the
 * stored and staged shapes 1, 2 and the windowed shape with one more round
 * of items per thread (smaller CTAs), each timed with events, each shape
 * keeping the faster of its two; the trials are part of the run (every
 * shape gives the same trajectory) and the fastest per attempted move is
 * kept unless the automatic shape is within 3% of it.  Shapes that do not
 * fit the system are skipped. */
int bfm_set_sweep_autotune(bfm_handle *h, int on);
/* the autotuner's trials (up to cap): shape, extra rounds, threads per CTA
 * and ns per attempted move; *tuned = 1 once it has chosen */
int bfm_get_sweep_tuning(const bfm_handle *h, int *tuned, uint32_t *count, int *shapes, int *extra_rounds, int *threads,
                         double *ns_per_move, uint32_t cap);
/* bound of every grid-barrier wait in the persistent kernel (default 2000 ms);
 * a wait that runs out ends the launch and bfm_run returns BFM_ETIMEOUT */
int bfm_set_barrier_timeout_ms(bfm_handle *h, uint32_t ms);
/* Failure-detection check of the bounded grid barrier: `rounds` barriers of
 * a cooperative kernel with one CTA per SM that expects extra_arrivals more
 * CTAs than exist.  extra_arrivals = 0 returns BFM_OK; > 0 makes every wait
 * run into timeout_ms and returns BFM_ETIMEOUT, with the context intact. */
int bfm_barrier_selftest(int gpu, uint32_t timeout_ms, uint32_t extra_arrivals, uint32_t rounds, double *elapsed_ms);
/* the same with a choice of barrier (counting = 1: monotone counter with
 * release reductions, the one the sweep uses; 0: generation barrier) and of
 * CTAs per SM; also measures the cost of one barrier (elapsed / rounds) */
int bfm_barrier_selftest_variant(int gpu, uint32_t timeout_ms, uint32_t extra_arrivals, uint32_t rounds, int counting,
                                 uint32_t ctas_per_sm, double *elapsed_ms);

/* The species colouring initialize() uses (the reference's graphColoring,
 * graphColoring.tpp:103-439, with uniform rebalancing as called at
 * UpdaterGPUScBFM_AB_Type.cu:1566-1570); host only.  deg[n], nbr8[8n];
 * colors[n] receives the colours, *ncolors their number. */
int bfm_color_graph(uint32_t n, const uint8_t *deg, const uint32_t *nbr8, int uniform, uint32_t *colors,
                    uint32_t *ncolors);
/* The same colours as bfm_color_graph, with the reference's depth-first
 * walk (graphColoring.tpp:176-351) replaced on every tree component (linear
 * chains, stars, combs) by a parity union-find on GPU `gpu`: on a tree the
 * walk gives every node the parity of its distance to the lowest id of its
 * component.  Components with a cycle (crosslinks) are walked on the host
 * -- the walk colours each component from its own nodes, so the result is
 * the walk's over the whole graph -- and the uniform rebalancing pass runs
 * on the host.  *on_device: 1 every component on the device, 2 the tree
 * components on the device and the others on the host, 0 all on the host. */
int bfm_color_graph_device(int gpu, uint32_t n, const uint8_t *deg, const uint32_t *nbr8, int uniform, uint32_t *colors,
                           uint32_t *ncolors, int *on_device);
/* colouring at initialize: 0 the host walk (default), 1 the device path of
 * bfm_color_graph_device (same colours); bfm_get_coloring reports the mode
 * and, as bfm_color_graph_device's *on_device, how the last initialize
 * coloured */
int bfm_set_coloring(bfm_handle *h, int mode);
int bfm_get_coloring(const bfm_handle *h, int *mode, int *on_device);

/* One colour substep (check + perform) on device arrays the caller owns,
 * without allocating any device memory.  No counterpart in the reference:
 * it is for callers that cannot call cudaMalloc while they step a system --
 * e.g. a host simulation that hands the library slices of one device pool
 * it manages itself, or runs under a fixed device-memory budget, where the
 * allocation calls (which may also synchronize the device) are not allowed.
 * The library's own scratch for this call (target bit lattice and
 * check/perform flags) is a fixed 512 KiB static device array, held by every
 * GPU that loads the library until the process exits.
 *   pos       device, npad Z-order codes (bit 3k: x_k, 3k+1: y_k, 3k+2: z_k)
 *   img       device int32[3][npad] image counters, or NULL
 *   nbr, deg  device neighbour slot ids (row j at nbr + j*npad) and counts
 *   lattice   device occupation bits, Z-order, 32-bit words, max(L)^3/32 words
 *   allowed512 host table, index (dx&7)|(dy&7)<<3|(dz&7)<<6, 108 entries set
 *   slot_offset, count: the colour's slab; local index = RNG subsequence
 *   seed, iteration: as drawn per substep by runSimulationOnGPU
 *   rng       BFM_RNG_INTHASH or BFM_RNG_SARU only; Philox (whose offset is
 *             the full 64-bit age) is refused with BFM_EINVAL
 *   stream    cudaStream_t to enqueue on (asynchronous; NULL = legacy stream)
 * Every axis is periodic (there are no walls in this call).
 * Limits: max(L)^3 <= 128^3 sites and count <= 262144, else BFM_ETOOLARGE.
 * A bond table without exactly 108 allowed entries is BFM_EINVAL.  If a CUDA
 * error from the caller's earlier work is pending, nothing runs and the call
 * returns BFM_ECUDA, leaving that error for the caller to read.
 * The first call on a device looks up the scratch array's address (one
 * cudaGetSymbolAddress, no allocation) and loads the call's kernels; make
 * that first call before any stream capture.  After it, no call loads or
 * allocates anything.  All calls share the one scratch array, so calls that
 * overlap on the GPU (concurrent streams, several host threads) race. */
int bfm_substep_noalloc(uint32_t *pos, int32_t *img, const uint32_t *nbr, const uint8_t *deg, uint32_t npad,
                        uint32_t *lattice, uint32_t box_x, uint32_t box_y, uint32_t box_z, const uint8_t *allowed512,
                        uint32_t slot_offset, uint32_t count, uint32_t seed, uint32_t iteration, int rng, void *stream);

/* Diagnostic: for k < n, out_pairs[2k] = the library's Philox4x32-10 word at
 * (seed, subsequence, offset + k) and out_pairs[2k+1] = curand() after
 * curand_init(seed, subsequence, offset + k) on the GPU, the generator the
 * reference's Philox option uses (rngs/lemonade_philox.h:48-56). */
int bfm_debug_philox_vs_curand(int gpu, uint64_t seed, uint64_t subsequence, uint64_t offset, uint32_t n,
                               uint32_t *out_pairs);

/* Process-global R250 colour/seed generator, the counterpart of LeMonADE's
 * RandomNumberGenerators whose r250_rand32() the reference calls
 * (UpdaterGPUScBFM_AB_Type.cu:3065-3066).  State = 250 words + index. */
int bfm_r250_seed(uint64_t seed);
int bfm_r250_seed_words(const uint32_t *words, size_t n); /* n >= 250 */
int bfm_r250_get_state(uint32_t state251[251]);
int bfm_r250_set_state(const uint32_t state251[251]);
uint32_t bfm_r250_rand32(void);

#ifdef __cplusplus
}
#endif

#endif /* PSCBFM_B200_H */
