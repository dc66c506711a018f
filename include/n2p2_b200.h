/*
 * n2p2_b200 — C-ABI of the B200 implementation of n2p2's 2G-HDNNP
 * prediction path (neighbor list, symmetry functions + derivatives, atomic
 * neural networks, energy, forces).
 *
 * Every entry point returns an int status (0 = success, negative = error) and
 * never throws; n2p2b_last_error() returns the message of the last failure
 * on a context.  The n2p2 C++ API reports the same conditions with
 * std::runtime_error / std::range_error / std::out_of_range; the C++ and
 * Python shims re-raise them.
 *
 * Units: positions, box and results are in the potential's PHYSICAL units
 * (those of input.data).  If input.nn normalizes (mean_energy, conv_energy,
 * conv_length) the conversion happens inside, exactly as
 * Prediction::readStructureFromFile / Prediction::predict do it.
 * Intermediate arrays (G, dE/dG, dG/dr, neighbor displacements) are returned
 * in the normalized units the reference holds them in during evaluateNNP.
 *
 * Threading: a context is used by one host thread at a time (as nnp::Mode).
 * All device work of a context runs in order on one CUDA stream.
 */
#ifndef N2P2_B200_H
#define N2P2_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct n2p2b_context n2p2b_context;

/* Status codes. */
#define N2P2B_OK                 0
#define N2P2B_ERR_ARGUMENT      -1  /* invalid argument                      */
#define N2P2B_ERR_SETUP         -2  /* input.nn / scaling / weights problem  */
#define N2P2B_ERR_CUDA          -3  /* CUDA runtime error                    */
#define N2P2B_ERR_CAPACITY      -4  /* capacity exceeded and not recoverable */
#define N2P2B_ERR_STATE         -5  /* call out of order (no setup/structure)*/
#define N2P2B_ERR_INTERNAL      -6  /* broken invariant (reported, not hit)  */
#define N2P2B_ERR_EXTRAPOLATION -7  /* extrapolation warning with "stop on
                                       warning" set (the reference's
                                       std::out_of_range); results are
                                       computed all the same               */

/* Where an array argument lives. */
#define N2P2B_HOST               0
#define N2P2B_DEVICE             1

/* n2p2b_set_structure flags. */
#define N2P2B_REMAP              1  /* wrap periodic positions into the cell
                                       (Structure::remap, as readFromLines) */

/* ---- context ---------------------------------------------------------- */

/* Creates a context on CUDA device `device`.  Replaces constructing
 * nnp::Mode / nnp::Prediction (libnnp/Mode.h:86, Prediction.h:27).
 * device = -1 creates a host-only context: setup and potential queries work,
 * evaluation calls return N2P2B_ERR_STATE. */
int         n2p2b_create(int device, n2p2b_context** ctx);
void        n2p2b_destroy(n2p2b_context* ctx);
const char* n2p2b_last_error(const n2p2b_context* ctx);
/* Runs the context's device work on `stream` (a cudaStream_t, NULL = own). */
int         n2p2b_set_stream(n2p2b_context* ctx, void* stream);

/* Arithmetic of the evaluation.  No counterpart in the reference (it always
 * computes in double).  N2P2B_PRECISION_FP64 (default) is the plain form.
 * The two mixed forms compute symmetry functions and dG/dr in FP32 and the
 * atomic NNs on the tensor cores with BF16 operands and FP32 accumulation;
 * neighbor displacements, the energy sum and the force accumulation stay
 * FP64.  N2P2B_PRECISION_MIXED splits each NN operand into BF16 high and low
 * parts (three tensor-core products per step, about 16 significant bits);
 * N2P2B_PRECISION_BF16 splits the operands of the forward sweep and of
 * dE/dG as MIXED does and keeps the back-propagated derivatives of the
 * hidden layers above the first in single BF16 (8 significant bits) against
 * split weights (two products per step): roundings there perturb each
 * atom's forces independently, while rounded weights or activations of the
 * forward sweep bias every atom's energy alike.
 * Getters return the FP32 intermediates widened to double.  Returns
 * N2P2B_ERR_SETUP if the potential's networks do not fit the tensor-core
 * kernel (more than one output, a layer wider than 256). */
#define N2P2B_PRECISION_FP64     0
#define N2P2B_PRECISION_MIXED    1
#define N2P2B_PRECISION_BF16     2
int         n2p2b_set_precision(n2p2b_context* ctx, int mode);
int         n2p2b_get_precision(const n2p2b_context* ctx);

/* ---- setup (nnp::Mode / nnp::Prediction) ------------------------------ */

/* Mode::loadSettingsFile (libnnp/Mode.cpp:161-210). */
int n2p2b_load_settings_file(n2p2b_context* ctx, const char* path);
/* Mode::setupGeneric (libnnp/Mode.cpp:212-236): normalization, elements,
 * cutoff, symmetry functions, dG/dr slot tables, SF groups, NN topology.
 * Includes Mode::setupSymmetryFunctionGroups (libnnp/Mode.cpp:842-892). */
int n2p2b_setup_generic(n2p2b_context* ctx);
/* Mode::setupSymmetryFunctionScaling (libnnp/Mode.cpp:712-840); path NULL
 * = Mode::setupSymmetryFunctionScalingNone. */
int n2p2b_setup_symmetry_function_scaling(n2p2b_context* ctx,
                                          const char* path);
/* Mode::setupNeuralNetworkWeights (libnnp/Mode.cpp:1451-1478); format is a
 * printf pattern taking the atomic number, e.g. "dir/weights.%03zu.data". */
int n2p2b_setup_neural_network_weights(n2p2b_context* ctx,
                                       const char* format);
/* Prediction::setup (libnnp/Prediction.cpp:34-46) on a potential directory
 * holding input.nn, scaling.data and weights.%03zu.data. */
int n2p2b_setup(n2p2b_context* ctx, const char* directory);

/* ---- potential queries ------------------------------------------------ */

int    n2p2b_num_elements(const n2p2b_context* ctx);
/* Element symbol of element index e (element order = n2p2's ElementMap). */
int    n2p2b_element_symbol(const n2p2b_context* ctx, int e, char* buf,
                            size_t len);
int    n2p2b_element_index(const n2p2b_context* ctx, const char* symbol);
/* Element::numSymmetryFunctions. */
int    n2p2b_num_symmetry_functions(const n2p2b_context* ctx, int e);
/* Element::getSymmetryFunctionNumTable()[ne] (libnnp/Element.cpp:289-311). */
int    n2p2b_num_slots(const n2p2b_context* ctx, int e, int ne);
/* Mode::getMaxCutoffRadius (normalized units, libnnp/Mode.h:693). */
double n2p2b_max_cutoff_radius(const n2p2b_context* ctx);
/* Element::getAtomicEnergyOffset and atomic number of element e. */
double n2p2b_atomic_energy_offset(const n2p2b_context* ctx, int e);
int    n2p2b_atomic_number(const n2p2b_context* ctx, int e);
/* mean_energy, conv_energy, conv_length of input.nn (1 / 0 when the
 * potential does not normalize); returns 1 if it normalizes. */
int    n2p2b_unit_conversion(const n2p2b_context* ctx, double* mean_energy,
                             double* conv_energy, double* conv_length);
/* Parameters of symmetry function s (sorted index = NN input index) of
 * element e, as Element::getSymmetryFunction(s) holds them (normalized
 * units): out[0..9] = type, e1, e2 (-1 for radial), eta, rs, rc, zeta,
 * lambda, scaling factor, input.nn line number (0-based).  Compact types
 * 20-22 give rl in place of eta, the subtype's rank in string order
 * (e = 0, p1 = 1, p1a = 2, ..., p4a = 8) in place of rs, and the left and
 * right angle (degrees) in place of zeta and lambda. */
int    n2p2b_symmetry_function_params(const n2p2b_context* ctx, int e, int s,
                                      double* out);
/* Element::setupSymmetryFunctionGroups: number of groups of element e and
 * the SF indices of group g's members in member order (returns the member
 * count; writes at most cap indices). */
int    n2p2b_num_groups(const n2p2b_context* ctx, int e);
int    n2p2b_group_members(const n2p2b_context* ctx, int e, int g,
                           int32_t* idx, int cap);

/* ---- structure (nnp::Structure) --------------------------------------- */

/* Sets the atoms to evaluate: Structure::readFromLines's data
 * (libnnp/Structure.cpp:142-271) without text parsing.  box: 9 doubles,
 * box[3k+c] = component c of lattice vector k, or NULL for a non-periodic
 * structure.  positions: num_atoms x 3 (physical units), host or device.
 * elements: num_atoms element indices (host).  flags: N2P2B_REMAP. */
int n2p2b_set_structure(n2p2b_context* ctx, int64_t num_atoms,
                        const double* box, const double* positions,
                        int positions_location, const int32_t* elements,
                        int flags);
/* New coordinates for the current atoms (next frame / MD step). */
int n2p2b_set_positions(n2p2b_context* ctx, const double* positions,
                        int positions_location);

/* ---- evaluation steps (nnp::Mode) ------------------------------------- */

/* Structure::calculateNeighborList(getMaxCutoffRadius(), false)
 * (libnnp/Structure.cpp:287-399). */
int n2p2b_calculate_neighbor_list(n2p2b_context* ctx);
/* Mode::calculateSymmetryFunctionGroups (libnnp/Mode.cpp:1561-1640). */
int n2p2b_calculate_symmetry_function_groups(n2p2b_context* ctx,
                                             int derivatives);
/* Mode::calculateAtomicNeuralNetworks (libnnp/Mode.cpp:1642-1751). */
int n2p2b_calculate_atomic_neural_networks(n2p2b_context* ctx,
                                           int derivatives);
/* Mode::calculateEnergy (libnnp/Mode.cpp:1803-1828). */
int n2p2b_calculate_energy(n2p2b_context* ctx);
/* Mode::calculateForces (libnnp/Mode.cpp:1849-1912). */
int n2p2b_calculate_forces(n2p2b_context* ctx);
/* Mode::evaluateNNP (libnnp/Mode.cpp:1967-2016) followed by the physical
 * unit conversion and energy offsets of Prediction::predict
 * (libnnp/Prediction.cpp:65-76). */
int n2p2b_evaluate(n2p2b_context* ctx, int use_forces);
/* Enqueues the whole evaluation on the context's stream without any host
 * synchronization (capacities must already fit, e.g. after one
 * n2p2b_evaluate on a structure of the same size).  Check the outcome with
 * n2p2b_finish. */
int n2p2b_evaluate_async(n2p2b_context* ctx, int use_forces);
/* Waits for the context's stream and reports capacity / invariant flags. */
int n2p2b_finish(n2p2b_context* ctx);

/* ---- neighbor list supplied by an MD engine (InterfaceLammps) ---------- */

/* InterfaceLammps::setLocalAtoms + allocateNeighborlists + addNeighbor +
 * finalizeNeighborList (libnnpif/LAMMPS/InterfaceLammps.cpp:267-304,
 * 400-457) in one call: num_atoms local atoms with their element indices;
 * atom i has neighbor_counts[i] entries (concatenated over atoms) with the
 * neighbor's position in the engine's force array (local atoms first, then
 * ghost atoms; num_targets in all), its element index and
 * dr = r_i - r_neighbor in the potential's physical units (the engine
 * converts by cflength first).  The library builds no neighbor list of its
 * own; the next evaluation (InterfaceLammps::process, libnnpif/LAMMPS/
 * InterfaceLammps.cpp:463-487) uses this one, and n2p2b_get_energy returns
 * the local atoms' energy. */
int n2p2b_set_neighbor_list(n2p2b_context* ctx, int64_t num_atoms,
                            const int32_t* elements,
                            const int64_t* neighbor_counts,
                            const int64_t* neighbor_index,
                            const int32_t* neighbor_elements,
                            const double* dr, int64_t num_targets);
/* InterfaceLammps::getForces (libnnpif/LAMMPS/InterfaceLammps.cpp:533-581):
 * forces on all num_targets local and ghost atoms (num_targets x 3,
 * overwritten; the engine adds them to its own force array), physical
 * units: each local atom's self term plus every pair term pointing at the
 * target, summed in a fixed order. */
int n2p2b_get_target_forces(n2p2b_context* ctx, double* forces);

/* ---- batches of independent structures -------------------------------- */

/* No direct counterpart in the reference, which evaluates one Structure at
 * a time (nnp-predict's loop over input.data).  Sets num_structures
 * independent structures in one call: atom_counts[s] atoms each, positions
 * (sum of counts x 3) and elements concatenated in structure order, boxes
 * (9 doubles per structure, rows = lattice vectors) or NULL for open
 * structures.  Every structure gets exactly the neighbor list, energy and
 * forces it gets alone; one evaluation runs all of them.  Per-atom getters
 * address the concatenated atoms; n2p2b_get_energy returns the sum. */
int n2p2b_set_structures(n2p2b_context* ctx, int64_t num_structures,
                         const int64_t* atom_counts, const double* boxes,
                         const double* positions, int positions_location,
                         const int32_t* elements, int flags);
/* Structure::energy of every structure of the batch (after predict's unit
 * conversion and offsets); one value for a single structure. */
int n2p2b_get_structure_energies(n2p2b_context* ctx, double* energies);

/* Captures one whole evaluation (neighbor list to forces, every kernel of
 * it) into a CUDA graph on the context's stream; n2p2b_launch_graph replays
 * it with one launch after new positions (n2p2b_set_positions) and
 * n2p2b_finish checks it.  Changing the structure, precision, student or
 * statistics settings, or growing a buffer, invalidates the capture. */
int n2p2b_capture_graph(n2p2b_context* ctx, int use_forces);
int n2p2b_launch_graph(n2p2b_context* ctx);

/* Autotuner: times every launch configuration (symmetry-function kernel
 * variant and work ordering, neighbor-list warps per block for batches) on
 * the current structure(s), keeps the fastest for their size bucket
 * (log2 atoms per structure, per precision) and applies it to later
 * structures of that bucket.  `report` receives the choice. */
int n2p2b_autotune(n2p2b_context* ctx, int use_forces, int repetitions,
                   char* report, size_t report_len);

/* ---- extrapolation warnings (Element::updateSymmetryFunctionStatistics) */

/* Mode::setupSymmetryFunctionStatistics (libnnp/Mode.cpp:1103-1137): after
 * every symmetry-function calculation, count the symmetry functions whose
 * unscaled value lies outside scaling.data's [Gmin, Gmax] by more than
 * 1000 DBL_EPSILON (libnnp/Element.cpp:462-541).  write_ew prints the
 * reference's "### NNP EXTRAPOLATION WARNING ###" lines to stderr;
 * stop_on_ew makes the evaluation return N2P2B_ERR_EXTRAPOLATION.
 * collect_statistics (the SF statistics of the training tools) is not
 * supported and must be 0. */
int n2p2b_setup_symmetry_function_statistics(n2p2b_context* ctx,
                                             int collect_statistics,
                                             int collect_ew, int write_ew,
                                             int stop_on_ew);
/* Mode::getNumExtrapolationWarnings / resetExtrapolationWarnings
 * (libnnp/Mode.h:478-486): warnings counted since the last reset. */
int64_t n2p2b_get_num_extrapolation_warnings(const n2p2b_context* ctx);
int     n2p2b_reset_extrapolation_warnings(n2p2b_context* ctx);
/* Warnings per atom of the last evaluation (num_atoms ints). */
int     n2p2b_get_extrapolation_counts(n2p2b_context* ctx, int32_t* counts);
/* The warnings of the last evaluation, one record each, in the order the
 * reference records them (atom by atom, each atom's symmetry functions in
 * order; Element::updateSymmetryFunctionStatistics, libnnp/Element.cpp:
 * 462-541, with the fields of SymFncStatistics::addExtrapolationWarning,
 * libnnp/SymFncStatistics.cpp:91-110).  At most `capacity` records into
 * `out`; *count receives their number (also when it is larger). */
typedef struct n2p2b_extrapolation_warning
{
    int64_t atom;      /* atom index in the structure (0-based) */
    int32_t element;   /* element index */
    int32_t sf;        /* symmetry function, element-local index (0-based) */
    int32_t type;      /* symmetry-function type */
    int32_t reserved;
    double  value;     /* unscaled value */
    double  gmin;      /* scaling.data minimum */
    double  gmax;      /* scaling.data maximum */
} n2p2b_extrapolation_warning;
int n2p2b_get_extrapolation_warnings(n2p2b_context* ctx, int64_t capacity,
                                     n2p2b_extrapolation_warning* out,
                                     int64_t* count);

/* ---- distilled student network --------------------------------------- */

/* No counterpart in the reference.  A student is a smaller atomic network
 * (its own potential directory: input.nn with exactly this potential's
 * symmetry functions, the same scaling.data, weights.%03zu.data, and
 * training_range.data once trained) that runs in FP32 on the FP32 symmetry
 * functions of a mixed precision.  Gated, every atom that has a symmetry
 * function outside the student's training range (the test of
 * Element::updateSymmetryFunctionStatistics with that range) is re-evaluated
 * by this potential's own network on the tensor cores. */
#define N2P2B_STUDENT_OFF        0  /* the potential's network only        */
#define N2P2B_STUDENT_GATED      1  /* student, teacher outside its range  */
#define N2P2B_STUDENT_ONLY       2  /* student for every atom              */
int n2p2b_setup_student(n2p2b_context* ctx, const char* directory);
int n2p2b_set_student_mode(n2p2b_context* ctx, int mode);
/* Atoms the teacher re-evaluated in the last gated evaluation. */
int n2p2b_get_student_gated_count(n2p2b_context* ctx, int64_t* count);
/* One Adam step (hand-written kernels) on a batch of the current structure:
 * loss = w_energy / B sum (E_i - E_i^label)^2
 *      + w_force / (3B) sum |F_i - F_i^label|^2 over the batch atoms.
 * Symmetry functions with derivatives must be current
 * (n2p2b_calculate_symmetry_function_groups).  energy_labels (num_atoms,
 * the units of n2p2b_get_atomic_energies), force_labels (num_atoms x 3, the
 * units of n2p2b_get_forces) and batch
 * (batch_size atom indices) are device arrays.  loss (host, 2 doubles: the
 * energy and force terms, or NULL) synchronizes.  Training needs one hidden
 * tanh layer and a linear output. */
int n2p2b_student_train_step(n2p2b_context* ctx, const double* energy_labels,
                             const double* force_labels, const int32_t* batch,
                             int batch_size, double w_energy, double w_force,
                             double learning_rate, double* loss);
int n2p2b_student_reset_optimizer(n2p2b_context* ctx);
/* The student's FP32 parameter blob as doubles (per element and layer: W
 * out x in, W^T, b; `size` receives its length).  which = 0: the weights
 * (get and/or set; W and W^T must be set consistently); which = 1: the
 * gradient summed in the last training step (get only; the W^T and
 * unused positions are 0). */
int n2p2b_student_weights(n2p2b_context* ctx, double* get, const double* set,
                          int64_t* size, int which);
/* reset = 1 empties the training range; reset = 0 widens it to cover the
 * current structure's symmetry functions. */
int n2p2b_student_update_range(n2p2b_context* ctx, int reset);
/* Writes weights.%03zu.data and training_range.data into `directory`. */
int n2p2b_student_write(n2p2b_context* ctx, const char* directory);

/* ---- results ---------------------------------------------------------- */

/* Structure::energy after Prediction::predict (physical units, offsets). */
int n2p2b_get_energy(n2p2b_context* ctx, double* energy);
/* Atom::f after Prediction::predict: num_atoms x 3, physical units. */
int n2p2b_get_forces(n2p2b_context* ctx, double* forces, int location);
/* Atom::energy after Prediction::predict (physical units, no offsets). */
int n2p2b_get_atomic_energies(n2p2b_context* ctx, double* energies);
/* Atom::numNeighbors per atom. */
int n2p2b_get_neighbor_counts(n2p2b_context* ctx, int64_t* counts);
/* Atom::neighbors (index, dr, d) concatenated per atom, in the reference's
 * list order (j ascending, then image). */
int n2p2b_get_neighbor_list(n2p2b_context* ctx, int64_t* index, double* dr,
                            double* d);
/* Atom::G / Atom::dEdG as [atom][stride]. */
int n2p2b_get_symmetry_functions(n2p2b_context* ctx, double* G, int stride);
int n2p2b_get_dEdG(n2p2b_context* ctx, double* dEdG, int stride);
/* Atom::dGdr ([atom][sf_stride][3]) and Neighbor::dGdr ([entry][slot_stride]
 * [3], entries in n2p2b_get_neighbor_list order). */
int n2p2b_get_dGdr(n2p2b_context* ctx, double* self, int sf_stride,
                   double* neighbor, int slot_stride);

/* ---- diagnostics (no counterpart in the reference) -------------------- */

/* Records CUDA events around each stage of every following evaluation on
 * the context's stream (device time; no host synchronization added). */
int n2p2b_set_profiling(n2p2b_context* ctx, int enable);
/* Summed device milliseconds per stage since the last reset: ms[0..4] =
 * neighbor list, symmetry functions, atomic NNs, energy, forces; *runs =
 * number of profiled evaluations.  Synchronizes the context's stream. */
int n2p2b_get_stage_times(n2p2b_context* ctx, double* ms, int64_t* runs,
                          int reset);
/* Number of kernel launches this library has issued in this process. */
uint64_t n2p2b_kernel_launch_count(void);
/* Diagnostics (no reference counterpart): evaluates on the current device
 * the FP64 exponential the symmetry-function kernels use for arguments
 * x <= 0 (y[i], i < n) and CUDA's exp (y[n + i]); x host, n values; y host,
 * 2 n values. */
int n2p2b_check_exp(const double* x, double* y, int64_t n);

/* ---- neighbor list without memory allocation -------------------------- */

/* No counterpart in the reference (n2p2 always builds neighbor lists into
 * std::vectors it allocates).  For callers that cannot allocate device
 * memory while they run -- an MD engine that reserves all GPU memory up
 * front, or code that must not trigger the device-wide synchronization of
 * cudaMalloc/cudaFree -- this computes the neighbor list of
 * Structure::calculateNeighborList (every (j, image) with
 * |r_i - r_j + image|^2 <= cutoff^2, bit-exact, in j-ascending, image
 * order) into buffers the caller owns, and allocates nothing.
 *
 * Its only other memory is one static device array of about 1.3 MB, held by
 * every GPU that loads this library until the process exits.  That array
 * sets the limits: at most N2P2B_NOALLOC_MAX_ATOMS atoms and
 * N2P2B_NOALLOC_MAX_NEIGHBORS neighbors per atom; larger inputs are
 * rejected with N2P2B_ERR_CAPACITY and a message in `err`.  All calls share
 * the array and it keeps the last call's contents (each call clears what
 * must start at zero), so calls whose GPU work overlaps (other streams or
 * host threads) race: serialize them.  The first call for a device looks up
 * the array's device address (cudaGetSymbolAddress) and should come before
 * any stream capture.  With CUDA's lazy module loading (the default) that
 * first call also loads the library's device code and the array onto the
 * device, which needs device memory: make one warm-up call before the host
 * reserves its GPU memory, or run with CUDA_MODULE_LOADING=EAGER.
 *
 * device:    CUDA device to run on (the caller's current device is kept).
 * stream:    cudaStream_t for the work (NULL = default stream); the call
 *            returns after that stream has finished it.
 * box:       host, 9 doubles (rows = lattice vectors) or NULL (non-periodic).
 * positions: device, num_atoms x 3, used as given (no remap, no units).
 * counts:    device, num_atoms          neighbors per atom (output)
 * offsets:   device, num_atoms + 1      exclusive prefix of counts (output)
 * index, dr, d: device, capacity, 3 x capacity, capacity: neighbor index,
 *            displacement r_i - r_j + image and distance (output).
 * total:     host, number of entries (also when capacity was too small;
 *            lists of more than 2^31 - 1 entries do not fit the int32
 *            offsets and are rejected with N2P2B_ERR_CAPACITY).
 * err:       optional host buffer for a message. */
#define N2P2B_NOALLOC_MAX_ATOMS      65536
#define N2P2B_NOALLOC_MAX_NEIGHBORS  1024
int n2p2b_neighbor_list_noalloc(int device, void* stream, int64_t num_atoms,
                                const double* box, const double* positions,
                                double cutoff, int32_t* counts,
                                int32_t* offsets, int32_t* index, double* dr,
                                double* d, int64_t capacity, int64_t* total,
                                char* err, size_t err_len);

/* ---- one call per frame ----------------------------------------------- */

/* Prediction::readStructureFromFile + Prediction::predict on in-memory
 * host arrays: sets the structure (with remap), evaluates, copies energy and
 * forces (num_atoms x 3) back to the host. */
int n2p2b_predict(n2p2b_context* ctx, int64_t num_atoms, const double* box,
                  const double* positions, const int32_t* elements,
                  double* energy, double* forces);

#ifdef __cplusplus
}
#endif

#endif /* N2P2_B200_H */
