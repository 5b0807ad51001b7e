/*
 * rascal_b200.h -- C ABI of the B200 descriptor/GAP library.
 *
 * One shared library (librascal_b200/_lib/librascal_b200.so) holds the
 * sm_100a CUDA kernels and the C++ host code that drives them. The entry
 * points below are the drop-in boundary for librascal's SOAP + sparse-GAP
 * hot path: each one names the reference interface it replaces (paths are
 * relative to the librascal source tree). Arguments are plain pointers and
 * sizes; every array argument is a HOST pointer unless its name ends in
 * `_dev`.
 *
 * Every function returns an rgpu_status (0 = success). On failure the message
 * of the matching reference exception is available from
 * rgpu_last_error() (thread-local), and rgpu_error_kind() tells which C++
 * exception type the reference throws for it (see rgpu_error_kind_t), so a
 * binding can re-raise the same Python exception class.
 *
 * Threading: a handle is used by one host thread at a time; each structure
 * set owns one CUDA stream. This matches the reference, which is serial and
 * releases the GIL around compute
 * (bindings/bind_py_representation_calculator.cc:57-62).
 */
#ifndef RASCAL_B200_H_
#define RASCAL_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int rgpu_status;
enum {
  RGPU_OK = 0,
  RGPU_ERR_INVALID_ARGUMENT = 1, /* bad hypers / sizes: std::logic_error, runtime_error */
  RGPU_ERR_STRUCTURE = 2,        /* atom outside cell, zero cell, type range: runtime_error */
  RGPU_ERR_CAPACITY = 3,         /* device buffer too small (retried internally) */
  RGPU_ERR_TIMEOUT = 4,          /* a bounded device-side wait gave up */
  RGPU_ERR_CUDA = 5,             /* CUDA runtime error */
  RGPU_ERR_OVERFLOW = 6,         /* 1F1 overflow: std::overflow_error */
  RGPU_ERR_NOT_COMPUTED = 7      /* features requested before compute */
};

/* Which reference exception a status maps to. */
typedef enum {
  RGPU_EXC_NONE = 0,
  RGPU_EXC_RUNTIME_ERROR = 1,
  RGPU_EXC_LOGIC_ERROR = 2,
  RGPU_EXC_OVERFLOW_ERROR = 3
} rgpu_error_kind_t;

const char * rgpu_last_error(void);
int rgpu_error_kind(void);
int rgpu_version(void);

/* Opaque handles. */
typedef struct rgpu_calculator rgpu_calculator;
typedef struct rgpu_structures rgpu_structures;
typedef struct rgpu_gap_model rgpu_gap_model;

/* Arithmetic of a compute call. */
enum {
  RGPU_PRECISION_FP64 = 0, /* plain path: FP64 everywhere, reference data flow */
  RGPU_PRECISION_FP32 = 1  /* fast path: FP32 features, BF16x3 tensor-core GEMMs, adjoint forces */
};

/* ---------------------------------------------------------------------- */
/* Calculators.
 * Replaces CalculatorSphericalInvariants(hypers) / CalculatorSphericalExpansion
 * (hypers) constructed from JSON:
 *   bindings/bind_py_representation_calculator.cc:43-47 (py::init from dict)
 *   src/rascal/representations/calculator_spherical_invariants.hh:171-176,257-292
 *   src/rascal/representations/calculator_spherical_expansion.hh:1596-1742
 * `kind` is "sphericalinvariants" or "sphericalexpansion"; `hypers_json` is the
 * hypers dict the reference's Python wrapper builds
 * (bindings/rascal/representations/spherical_invariants.py:209-294). The GTO
 * radial spline is built here in FP64 on the host and uploaded. */
rgpu_status rgpu_calculator_create(const char * kind, const char * hypers_json,
                                   rgpu_calculator ** out);
rgpu_status rgpu_calculator_destroy(rgpu_calculator * calc);
/* Name used by the reference to register results: prefix + hypers dump
 * (src/rascal/representations/calculator_base.hh:105-112). */
rgpu_status rgpu_calculator_name(const rgpu_calculator * calc, char * buf,
                                 size_t buflen);
/* Shape of the radial spline (grid points, values per point). */
rgpu_status rgpu_calculator_spline_shape(const rgpu_calculator * calc,
                                         int32_t * grid_size, int32_t * width);
/* Copy out the FP64 spline (grid, values y, y''h^2/6), each grid_size x width,
 * for parity checks of the host spline builder
 * (src/rascal/math/interpolator.hh:976-1287). */
rgpu_status rgpu_calculator_spline_table(const rgpu_calculator * calc,
                                         double * grid, double * y,
                                         double * y2h);

/* ---------------------------------------------------------------------- */
/* Structure sets.
 * Replaces ManagerCollection(adaptors) + add_structures(AtomicStructureList)
 * (src/rascal/structure_managers/structure_manager_collection.hh:178-184,
 *  bindings/bind_py_structure_manager.cc:472-560). Structures are flat arrays:
 *   atom_offsets  int64  [n_structures + 1]
 *   positions     double [n_atoms * 3]
 *   numbers       int32  [n_atoms]   atomic numbers in [0, 130)
 *   cells         double [n_structures * 9], row-major, ROWS are lattice
 *                 vectors (ASE convention; the reference transposes,
 *                 src/rascal/structure_managers/atomic_structure.hh:413-449)
 *   pbc           int32  [n_structures * 3]
 *   center_mask   uint8  [n_atoms] or NULL (all atoms are centres)
 * Input validation follows StructureManagerCenters::build
 * (structure_manager_centers.cc:39-94): positions must be inside the cell
 * (scaled coordinates in [-1e-10, 1+1e-10]), the cell must not be zero and
 * types must be in [0, 130). */
rgpu_status rgpu_structures_create(rgpu_structures ** out);
rgpu_status rgpu_structures_destroy(rgpu_structures * s);
rgpu_status rgpu_structures_set(rgpu_structures * s, int32_t n_structures,
                                const int64_t * atom_offsets,
                                const double * positions,
                                const int32_t * numbers, const double * cells,
                                const int32_t * pbc,
                                const uint8_t * center_mask);
/* Replace positions only (same atoms, same cells): an MD-style update. */
rgpu_status rgpu_structures_update_positions(rgpu_structures * s,
                                             const double * positions);
/* Mark the neighbour list and the features out of date without touching the
 * inputs already on the device, so that the next call recomputes them (the
 * reference's per-manager update flags, updateable_base.hh:91). */
rgpu_status rgpu_structures_invalidate(rgpu_structures * s);
/* The CUDA stream (cudaStream_t) this structure set's work runs on. */
rgpu_status rgpu_structures_stream(const rgpu_structures * s, void ** stream);

/* ---------------------------------------------------------------------- */
/* Neighbour list.
 * Replaces the adaptor stack centers -> neighbourlist(cutoff) ->
 * centercontribution -> strict(cutoff)
 * (bindings/rascal/representations/spherical_invariants.py:285-290;
 *  src/rascal/structure_managers/adaptor_neighbour_list.hh:903-1118,
 *  adaptor_center_contribution.hh:333-406, adaptor_strict.hh:373-455).
 * Pairs are grouped by centre, self pair first, then the linked-cell stencil
 * order of the reference. */
rgpu_status rgpu_neighbour_list_build(rgpu_structures * s, double cutoff);
rgpu_status rgpu_neighbour_list_size(const rgpu_structures * s,
                                     int64_t * n_centers, int64_t * n_pairs);
/* Export. centers: center_atom [n_centers] (global atom index),
 * pair_offsets [n_centers + 1]; pairs: j_atom [n_pairs] (global index of the
 * real atom), shift [n_pairs * 3] (periodic image), distance [n_pairs],
 * direction [n_pairs * 3]. Any pointer may be NULL.
 * Replaces ManagerCollection.get_distances / get_direction_vectors /
 * get_gradients_info (bindings/bind_py_structure_manager.cc:708-905). */
rgpu_status rgpu_neighbour_list_get(const rgpu_structures * s,
                                    int32_t * center_atom,
                                    int64_t * pair_offsets, int32_t * j_atom,
                                    int32_t * shift, double * distance,
                                    double * direction);

/* ---------------------------------------------------------------------- */
/* Representations.
 * Replaces calculator.compute(managers)
 * (bind_py_representation_calculator.cc:57-62 ->
 *  calculator_spherical_invariants.hh:674-931 /
 *  calculator_spherical_expansion.hh:2139-2411). Builds the neighbour list
 * with the calculator's cutoff when needed. `gradients` follows the
 * compute_gradients hyper unless forced to 1 here. */
rgpu_status rgpu_compute(rgpu_calculator * calc, rgpu_structures * s,
                         int precision, int gradients);
/* Dense features (rows = centres, columns = sorted keys x inner block):
 * get_features (bindings/bind_py_structure_manager.cc:573-614;
 * property_block_sparse.hh:911-931). The species list of the dense layout is
 * returned by rgpu_get_species; rgpu_get_feature_keys gives the keys present
 * in the batch (keys[k*2+0..1]; expansion keys use only keys[k*2]).
 * `out` is n_centers x (n_keys * inner) FP64. */
rgpu_status rgpu_get_species(const rgpu_structures * s, int32_t * n_species,
                             int32_t * species /* >= 130 entries */);
rgpu_status rgpu_get_feature_keys(const rgpu_calculator * calc,
                                  const rgpu_structures * s, int32_t * n_keys,
                                  int32_t * keys /* >= 2 * n_keys */);
rgpu_status rgpu_get_features(const rgpu_calculator * calc,
                              const rgpu_structures * s, int32_t n_keys,
                              const int32_t * keys, double * out);
/* Dense gradients, 3 rows (x, y, z) per pair including self pairs:
 * get_features_gradient (bind_py_structure_manager.cc:621-668;
 * property_block_sparse.hh:961-987). `out` is 3*n_pairs x (n_keys * inner).
 * Needs a compute with gradients at RGPU_PRECISION_FP64. For a spherical
 * expansion the rows are the reference's grad C blocks
 * (calculator_spherical_expansion.hh:2327-2366): a self pair carries every
 * centre key, a neighbour pair only the key of its neighbour's species. */
rgpu_status rgpu_get_features_gradient(const rgpu_calculator * calc,
                                       const rgpu_structures * s,
                                       int32_t n_keys, const int32_t * keys,
                                       double * out);

/* ---------------------------------------------------------------------- */
/* Sparse GAP model.
 * Replaces KRR(weights, Kernel(GAP, zeta), SparsePoints) prediction:
 *   models/krr.py:92-166, models/sparse_kernels.hh:104-131,
 *   models/sparse_kernel_predict.hh:70-266, models/sparse_points.hh:179-338.
 * Sparse points are given dense: T [n_sparse x D] FP64 in the power-spectrum
 * layout of `species` (sorted, n_species entries; D = n_species*(n_species+1)/2
 * * n^2 * (l+1)), one row per sparse environment, with its central species in
 * sparse_species [n_sparse]; weights [n_sparse] (NULL: zero weights, for a
 * model used only for its kernel matrices); self_contributions [n_species]
 * (energy baseline per species, models/krr.py:68-90). */
rgpu_status rgpu_gap_model_create(rgpu_calculator * calc, int32_t n_species,
                                  const int32_t * species, int32_t n_sparse,
                                  const int32_t * sparse_species,
                                  const double * T, const double * weights,
                                  int32_t zeta,
                                  const double * self_contributions,
                                  rgpu_gap_model ** out);
rgpu_status rgpu_gap_model_destroy(rgpu_gap_model * m);
/* Energies (n_structures, baseline included) and forces (n_atoms x 3, FP64,
 * = -dE/dr). RGPU_PRECISION_FP64 runs the reference's own algorithm on the
 * GPU (materialised dX/dr contracted with the scaled sparse points);
 * RGPU_PRECISION_FP32 runs the adjoint path (dE/dC contracted with dC/dr
 * recomputed per pair). Either output may be NULL. */
rgpu_status rgpu_gap_predict(rgpu_gap_model * m, rgpu_structures * s,
                             int precision, double * energies,
                             double * forces);
/* rgpu_gap_predict plus the negative stress of every structure,
 * neg_stress[n_structures][6] in the Voigt order xx, yy, zz, yz, xz, xy: the
 * sum over pairs of r_ji (x) dE_i/dr_j divided by the cell volume. Replaces
 * compute_sparse_kernel_neg_stress (models/sparse_kernel_predict.hh:291-377)
 * behind KRR.predict_stress, which returns -neg_stress
 * (bindings/rascal/models/krr.py:168-210). neg_stress must not be NULL;
 * energies and forces may be. */
rgpu_status rgpu_gap_predict_stress(rgpu_gap_model * m, rgpu_structures * s,
                                    int precision, double * energies,
                                    double * forces, double * neg_stress);

/* The adjoint path split for automatic differentiation (a
 * torch.autograd.Function): the reference computes energies and forces in
 * separate calls, KRR.predict and KRR.predict_forces
 * (bindings/rascal/models/krr.py:92-166); here the forward keeps on the
 * device what the force pass needs, and the backward applies an upstream
 * gradient per structure. Both run the FP32 path; DEVICE pointers, ordered on
 * the structure set's stream (rgpu_structures_stream), which is synchronised
 * before the calls return.
 * Forward: positions_dev [n_atoms x 3] FP64 (NULL: keep the current
 * positions; otherwise they replace them, inside the cells as for
 * rgpu_structures_set) -> energies_dev [n_structures] FP64, baseline
 * included. */
rgpu_status rgpu_gap_forward_dev(rgpu_gap_model * m, rgpu_structures * s,
                                 const double * positions_dev,
                                 double * energies_dev);
/* Backward of the last rgpu_gap_forward_dev of the same model on the same
 * structures (RGPU_ERR_NOT_COMPUTED if another call on the structures came
 * in between): grad_dev [n_atoms x 3] FP64 = sum_A energies_grad_dev[A]
 * dE_A/dr. */
rgpu_status rgpu_gap_backward_dev(rgpu_gap_model * m, rgpu_structures * s,
                                  const double * energies_grad_dev,
                                  double * grad_dev);

/* One step of a molecular-dynamics loop on the structures of the last
 * rgpu_structures_set (same atoms, types and cells; positions wrapped into
 * the cells): new positions [n_atoms x 3] in; energies, forces and, when
 * neg_stress is not NULL, the negative stress out, as rgpu_gap_predict_stress
 * gives them on the FP32 path. The first call runs the ordinary path, then
 * records the step, neighbour list included, as a CUDA graph with the list
 * built to capacities 25 % above that step's counts; later calls copy the
 * positions into pinned memory and replay the graph, with one
 * synchronisation per step. A step whose neighbour list outgrows the
 * capacities, or whose input is invalid, is recomputed by the ordinary path
 * (which reports input errors with the reference's messages) and the graph
 * is recorded again. Another call that reallocates a device buffer of this
 * handle, of the model or of its calculator makes the next step record
 * anew. Replaces, for the FP32 path, the
 * per-step predict calls of GenericMDCalculator.calculate
 * (bindings/rascal/models/genericmd.py:84-130). */
rgpu_status rgpu_md_step(rgpu_gap_model * m, rgpu_structures * s, const double * positions,
                         double * energies, double * forces, double * neg_stress);
/* Whether the structures handle holds a recorded MD step (1) or will run
 * the ordinary path next (0); info (may be NULL) receives the
 * neighbour-list capacities of the recording (sites, boxes, pairs), the
 * number of replays since it was recorded, and why the last recording was
 * not replayed (0 none, 1 one of its device buffers was reallocated by
 * another call on this handle or model, 3 another model,
 * layout or stress setting, 100 + status code when the replayed step set
 * one, e.g. 204 for outgrown capacities) and the number of kernels one
 * replay launches. No counterpart in the reference. */
rgpu_status rgpu_md_step_info(const rgpu_structures * s, int32_t * recorded, int64_t * info /* [6] */);

/* Sparse kernel matrices for training a GAP model, FP64 (the reference's
 * arithmetic). Columns follow the order of the model's sparse points;
 * weights and self contributions are not used.
 * K_NM energy rows: SparseKernel::compute with a GAP kernel
 * (models/sparse_kernels.hh:104-131 for target_atom = 0: out[n_structures]
 * [n_sparse], the sum over each structure's centres of (X_i . T_m)^zeta for
 * the sparse points of the centre's species; :165-191 for target_atom = 1:
 * out[n_centers][n_sparse]), behind Kernel.__call__(managers, sparse_points)
 * (bindings/rascal/models/kernels.py:122-164). */
rgpu_status rgpu_sparse_kernel(rgpu_gap_model * m, rgpu_structures * s,
                               int32_t target_atom, double * out);
/* K_NM gradient rows: SparseKernel::compute_derivative
 * (models/sparse_kernels.hh:258-499, 577-619) behind
 * Kernel.__call__(managers, sparse_points, grad=(True, False),
 * compute_neg_stress) (bindings/rascal/models/kernels.py:150-156).
 * out[3 * n_centers (+ 6 * n_structures if neg_stress)][n_sparse]: row
 * 3a + c is d/dr_a[c] of the structure's summed kernel; the stress rows
 * (Voigt xx, yy, zz, yz, xz, xy, divided by the cell volume) follow. As in
 * the reference, a structure none of whose centre species has sparse points
 * ends the computation: its rows and those of all later structures are 0.
 * Centre masks are rejected, as with gradients in the reference. */
rgpu_status rgpu_sparse_kernel_derivative(rgpu_gap_model * m, rgpu_structures * s,
                                          int32_t neg_stress, double * out);
/* K_MM: SparseKernel::compute(sparse_points) (models/sparse_kernels.hh:
 * 141-156, models/sparse_points.hh:144-170): out[n_sparse][n_sparse] =
 * (T_a . T_b)^zeta for points of one species, 0 across species. */
rgpu_status rgpu_sparse_kernel_mm(rgpu_gap_model * m, double * out);

/* ---------------------------------------------------------------------- */
/* Timing support: synchronise the structure set's stream; number of kernels
 * this library launched since the counter was last reset. */
rgpu_status rgpu_synchronize(rgpu_structures * s);
int64_t rgpu_kernel_launches(int reset);
/* Device time (ms) of the stages of the last rgpu_gap_predict call, from
 * CUDA events on the structure set's stream: 0 = whole call, 1 = neighbour
 * list, 2 = expansion, 3 = power spectrum, 4 = forward GEMMs, 5 = backward
 * GEMMs, 6 = power-spectrum backward (plain path: the materialised gradient
 * chunks and their contraction), 7 = pair adjoint. After
 * rgpu_sparse_kernel_derivative: 0 = its device time after the features and
 * before the copy to the host, 4 = the zeta k^(zeta-1) GEMMs, 6 = the
 * gradient chunks (materialised dX/dr and the gathered GEMMs). */
rgpu_status rgpu_stage_times(const rgpu_structures * s, double * ms_out,
                             int32_t n_stages);
/* Launch shapes of the FP32 path per feature shape (n_species, max_radial,
 * max_angular), as chosen by the project's autotuner
 * (librascal_b200/tune.py, which times candidates with CUDA events and
 * commits its table; the Python package installs the table when it loads
 * the library). values[8] = neighbour pairs per chunk of the expansion (8,
 * 16 or 32), centres per block of the expansion (1..8), threads per block of
 * the pair adjoint (32..128, multiple of 32), its grid cap in blocks per SM
 * (1..256), threads per block of the power-spectrum forward (64..256) and
 * backward (64..320), both multiples of 32, the grouped GEMM pipeline
 * (0: 4 stages of K blocks of 32, 1: 3 of 32, 2: 2 of 64), and the
 * power-spectrum forward (0: FP32 pipe, 1: tcgen05 Gram products). n_values
 * = 0 removes the shape's entry (back to the defaults 16, 4, 128, 64, 256,
 * 320, 0, 0); values out of range are rejected. Process-wide; no counterpart in
 * the reference (its kernels are serial C++ loops). */
rgpu_status rgpu_set_tile_config(int32_t n_species, int32_t max_radial, int32_t max_angular,
                                 const int32_t * values, int32_t n_values);
rgpu_status rgpu_get_tile_config(int32_t n_species, int32_t max_radial, int32_t max_angular,
                                 int32_t * values /* [8] */);

/* FP32 predictions as recorded CUDA graphs. With graphs on (the default),
 * rgpu_gap_predict and rgpu_gap_predict_stress at RGPU_PRECISION_FP32 record
 * the whole call (neighbour list, features, GEMMs, backward, adjoint, output
 * copies) as a CUDA graph per size bucket: the model, whether outputs and
 * the stress are asked for, the numbers of structures and atoms, the species
 * layout and the centres per species, and the addresses of the device
 * buffers involved. The first call of a bucket runs the ordinary path
 * (which sizes buffers through a few host synchronisations) and records the
 * bucket with the neighbour list built to capacities 12.5 % above its
 * counts; later calls of the bucket replay the graph with one
 * synchronisation. A replay whose list outgrows the capacities, or whose
 * input is invalid, is redone by the ordinary path (which reports input
 * errors with the reference's messages) and the bucket is recorded again.
 * A handle keeps at most four buckets (least recently used dropped). A
 * replayed call records no stage times (rgpu_stage_times keeps those of the
 * last ordinary call). The reference has no counterpart: it prepares each
 * manager on the host (structure_manager_collection.hh:178-184). */
rgpu_status rgpu_structures_use_graphs(rgpu_structures * s, int enable);
/* info[0] = recorded buckets held, info[1] = replays, info[2] = recordings,
 * info[3] = kernels launched by the last replayed graph. */
rgpu_status rgpu_structures_graph_info(const rgpu_structures * s, int64_t * info /* [4] */);
/* Measured FMA throughput of the current device's CUDA cores in TFLOP/s,
 * FP32 (RGPU_PRECISION_FP32) or FP64 (RGPU_PRECISION_FP64) pipe: every SM
 * filled with independent FMA chains, best of five launches timed with CUDA
 * events (2 flops per FMA). The denominator of the FP32- and FP64-pipe
 * roofline fractions. No counterpart in the reference. */
rgpu_status rgpu_measure_fma_peak(int precision, double * tflops);

/* ---------------------------------------------------------------------- */
/* Unit-test hook for the tensor-core GEMM (no reference counterpart; the
 * reference computes these contractions as per-centre GEMVs,
 * models/sparse_kernels.hh:104-131 and sparse_kernel_predict.hh:130-172).
 * DEVICE pointers, row-major FP32: A [M x K], B [N x K]. mode 0: C = A B^T
 * [M x N]; mode 1: the GAP forward epilogue with alpha [N] and zeta,
 * C = alpha zeta (A B^T)^(zeta-1) [M x N] (read back from its BF16 split) and
 * e [M] = sum_n alpha_n (A B^T)^zeta. `stream` is a cudaStream_t or NULL. */
rgpu_status rgpu_debug_gemm_bf16x3(int mode, int64_t M, int64_t N, int64_t K,
                                   const float * A_dev, const float * B_dev,
                                   const float * alpha_dev, int32_t zeta,
                                   float * C_dev, float * e_dev,
                                   void * stream);

/* Test hook for the bounded waits of the tensor-core GEMMs (no reference
 * counterpart): the number of polls after which the MMA warp's wait for
 * staged operands gives up (0: at once; negative: the default, about 4 M
 * polls). A wait that gives up makes the GEMM wind down (copies and MMAs
 * already started are waited for, TMEM is freed) and the call return
 * RGPU_ERR_TIMEOUT; the status is cleared for the next call. Process-wide;
 * restore the default after use. */
rgpu_status rgpu_debug_set_gemm_wait_limit(int64_t polls);

/* Test hook for the packed column layout of the FP32 path (no reference
 * counterpart; host arithmetic only, no device needed). For S species,
 * max_radial n and max_angular l: *D and *Dg receive the reference's row
 * length and the packed row length; when `ref` is given (D values in the
 * reference's dense order) `packed` receives its packed form (Dg values,
 * same-species pairs (n1 n2) and (n2 n1) folded into one column) and
 * `unpacked` that packed row mapped back to the reference's order through
 * FP32, as the FP32 feature export does. */
rgpu_status rgpu_debug_packed_layout(int32_t S, int32_t max_radial, int32_t max_angular, int64_t * D, int64_t * Dg,
                                     const double * ref, double * packed, double * unpacked);

/* ---------------------------------------------------------------------- */
/* GAP energies without device allocation. No counterpart in the reference:
 * it is the per-row energy of the mode-1 GEMM above,
 * e_dev[r] = sum_n alpha_dev[n] (A_r . B_n)^zeta, for callers that must not
 * allocate or free device memory during a call (cudaMalloc and cudaFree
 * synchronise the whole device, stalling every other stream of a process
 * that shares the GPU, such as an MD integrator's own kernels).
 * DEVICE pointers, row-major FP32: A [M x K], B [N x K], alpha [N], e [M].
 * All scratch lives in one static 16 MiB device array, which every GPU that
 * loads the library holds until the process exits; sizes needing more
 * (about 4 M Kp + 4 N Kp + 4 M ceil(N/256) bytes, Kp = K rounded up to 64)
 * return RGPU_ERR_CAPACITY before any pointer is touched.
 * The first call on each device does the setup (the address lookup of the
 * static arrays, kept for the life of the process; a cudaDeviceReset after
 * it is not supported). The work is ordered on `stream` (a cudaStream_t or NULL), and the call synchronises
 * that stream before it returns, to read the GEMM's status word. Calls that
 * overlap in time share the scratch and race, so callers serialise them. */
rgpu_status rgpu_gap_energies_noalloc(int64_t M, int64_t N, int64_t K,
                                      const float * A_dev, const float * B_dev,
                                      const float * alpha_dev, int32_t zeta,
                                      float * e_dev, void * stream);

#ifdef __cplusplus
}
#endif

#endif /* RASCAL_B200_H_ */
