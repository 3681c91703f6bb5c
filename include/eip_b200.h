/*
 * libmolecular_integral.so -- B200 (sm_100a) McMurchie-Davidson integrals.
 *
 * Drop-in C ABI.  The first four entry points are exactly the symbols the
 * reference front end binds with ctypes.cdll.LoadLibrary("libmolecular_integral.so")
 * (electron_integral_playground/molecular_integral/*.py:7) and have the same
 * signatures, argument meaning, accumulate-into-output semantics, supported
 * classes and error behaviour (return 0 on success; print a message and
 * return 1 for an unsupported angular class).  Additionally they return 2 on
 * a CUDA failure (no device, allocation or launch error); eip_last_error()
 * then describes it.  All pointers are host pointers to C-contiguous arrays;
 * positions in Bohr; (n,4) rows are [x, y, z, exponent].
 *
 * Layouts of the outputs (the caller zero-fills; the library adds):
 *   three_center       J3c[n_aux][n_ao][n_ao]
 *   two_center         J2c[n_aux][n_aux]
 *   nuclear_attraction V[n_ao][n_ao][n_charge]   (not scaled by -Z)
 *   overlap            S[n_ao][n_ao]
 */
#ifndef EIP_B200_H
#define EIP_B200_H

#include <stdbool.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces the reference three_center
 * (electron_integral_playground/c_library/molecular_integral/three_center.cpp:321-340).
 * One (l_i, l_j | l_k) class: i_L <= j_L <= 6, k_L <= 9. */
int three_center(const int i_L, const int j_L, const int k_L,
                 const double* pair_P_p, const double* pair_A_a, const double* pair_B_b,
                 const double* pair_coefficient, const int* pair_i_ao_start, const int* pair_j_ao_start,
                 const int n_pair_ij, const double* aux_A_a, const double* aux_coefficient,
                 const int* aux_i_aux_start, const int n_aux_primitive_k, double* J3c_matrix,
                 const int n_ao, const int n_aux, const bool spherical, const double omega);

/* Replaces the reference two_center
 * (electron_integral_playground/c_library/molecular_integral/two_center.cpp:239-252).
 * i_L <= j_L <= 9; for i_L == j_L, primitive pairs with i_aux_start > j_aux_start
 * are skipped and the other triangle is filled by mirroring, as in the reference. */
int two_center(const int i_L, const int j_L,
               const double* aux_A_a, const double* aux_i_coefficient, const int* aux_i_aux_start,
               const int n_aux_primitive_i, const double* aux_B_b, const double* aux_j_coefficient,
               const int* aux_j_aux_start, const int n_aux_primitive_j, double* J2c_matrix,
               const int n_aux, const bool spherical, const double omega);

/* Replaces the reference nuclear_attraction
 * (electron_integral_playground/c_library/molecular_integral/nuclear_attraction.cpp:199-213).
 * charge_position: (n_charge, 3) rows.  i_L <= j_L <= 6. */
int nuclear_attraction(const int i_L, const int j_L,
                       const double* pair_P_p, const double* pair_A_a, const double* pair_B_b,
                       const double* pair_coefficient, const int* pair_i_ao_start,
                       const int* pair_j_ao_start, const int n_pair, const double* charge_position,
                       const int n_charge, double* V_tensor, const int n_ao, const bool spherical,
                       const double omega);

/* Replaces the reference overlap
 * (electron_integral_playground/c_library/molecular_integral/overlap.cpp:149-159).  i_L <= j_L <= 6. */
int overlap(const int i_L, const int j_L, const double* pair_A_a, const double* pair_B_b,
            const double* pair_coefficient, const int* pair_i_ao_start, const int* pair_j_ao_start,
            const int n_pair, double* S_matrix, const int n_ao, const bool spherical);

/* ---- extensions (no counterpart in the reference) ------------------------ */

/* Select the device (or -1: the current one) and create the library's stream
 * and device tables.  Optional: every entry point initialises lazily.  The
 * reference-ABI entry points run on this device (the first one initialised)
 * whatever device the calling thread has current, and restore the caller's
 * device; a batch runs on the device it was built on.  Each device that is
 * used gets its own constant tables and launch set-up. */
int eip_init(int device);

/* Description of the last CUDA failure of the calling thread ("" if none). */
const char* eip_last_error(void);

/* Number of kernels this process has launched through the library. */
unsigned long long eip_kernel_launch_count(void);

/* Device time (CUDA events on the library's stream) of the kernels of the
 * last reference-ABI call, in milliseconds. */
float eip_last_kernel_ms(void);

/* Tuning variant (0..5) of the fast (mu nu|P) kernel of class (i_L, j_L | k_L),
 * i_L <= j_L <= 2 or (i_L, j_L) = (0, 3), (0, 4), k_L <= 4: accumulator budget and register cap (see
 * k3c_fast.cuh).  Affects launches made after the call (a batch's graph keeps
 * the variants it was captured with).  set returns 1 for an invalid
 * class/variant; get returns -1 for a class without fast kernels. */
int eip_tune_set(int i_L, int j_L, int k_L, int variant);
int eip_tune_get(int i_L, int j_L, int k_L);
/* The same for the FP32 kernels of the mixed-precision path: variants 0, 2, 3, 4. */
int eip_tune_set_fp32(int i_L, int j_L, int k_L, int variant);
int eip_tune_get_fp32(int i_L, int j_L, int k_L);

/* Device Boys function: F[i*(L+1)+m] = F_m(T[i]), m = 0..L <= 21 (host buffers). */
int eip_boys(int L, const double* T, int n, double* F);

/* (mu nu|P) of one class like three_center(), for callers that cannot let the
 * library allocate device memory (a framework's memory pool or a program that
 * reserves device memory up front owns it; an allocation could stall or fail
 * mid-run or synchronise the device).  No counterpart in the reference.
 * Every pointer is a DEVICE pointer; J3c_matrix[n_aux][n_ao][n_ao] is
 * accumulated (+=) asynchronously on `stream` (a cudaStream_t, 0 = default).
 * Nothing is allocated: working memory is one fixed 16 MiB device array per
 * GPU (eip_noalloc_scratch_bytes()), held from module load until exit.  Limit:
 * a call needing more of it, or more than 65535 auxiliary primitives, returns
 * 4 and launches nothing; eip_three_center_noalloc_check() tells beforehand,
 * on the host, without any CUDA call.  All calls share the array: calls whose
 * kernels overlap on the GPU race, so order them (one stream).  The first call
 * on each device (with it current) looks up the array's address and uploads
 * the constant tables, once per device under a lock; make it before any stream
 * capture.  Returns 0, 1 (unsupported class), 2 (CUDA failure) or 4 (too
 * large); for 2 and 4, eip_last_error() describes the failure. */
int eip_three_center_noalloc(const int i_L, const int j_L, const int k_L,
                             const double* pair_P_p, const double* pair_A_a, const double* pair_B_b,
                             const double* pair_coefficient, const int* pair_i_ao_start,
                             const int* pair_j_ao_start, const int n_pair_ij, const double* aux_A_a,
                             const double* aux_coefficient, const int* aux_i_aux_start,
                             const int n_aux_primitive_k, double* J3c_matrix, const int n_ao, const int n_aux,
                             const bool spherical, const double omega, void* stream);
/* Host-side admission test of eip_three_center_noalloc for one class and size:
 * 0 = fits (*bytes_needed = its working memory, 0 for an empty call),
 * 1 = unsupported class, 4 = too large (*bytes_needed = what it would need). */
int eip_three_center_noalloc_check(const int i_L, const int j_L, const int k_L, const int n_pair_ij,
                                   const int n_aux_primitive_k, const bool spherical, size_t* bytes_needed);
/* Size of the fixed working array of eip_three_center_noalloc, in bytes. */
size_t eip_noalloc_scratch_bytes(void);

/* ---- screened pair tables built on the device (no counterpart in the C ABI:
 * replaces the reference front end's Python form_pair_data,
 * electron_integral_playground/pair_utility.py:6-188) ----------------------
 * Shells in basis order: angular momentum, atom, first AO, primitive count;
 * their primitives' exponents and (normalised) coefficients concatenated;
 * geometry (n_atom, 3) in Bohr.  Keeps the primitive pairs whose bound is
 * >= threshold (the reference front end uses 1e-14), stably sorted by
 * descending bound per (l_i, l_j) class, with the reference's bound
 * construction.  Results are held by the returned object: eip_pairs_count
 * gives a class's row count (0 if absent), eip_pairs_copy copies its rows
 * into host arrays (P_p, A_a, B_b: 4 doubles a row). */
typedef struct eip_pairs eip_pairs;
eip_pairs* eip_pairs_build(int n_shell, const int* shell_l, const int* shell_atom, const int* shell_ao,
                           const int* shell_nprim, const double* prim_exp, const double* prim_coef, int n_atom,
                           const double* geometry, double threshold);
const char* eip_pairs_error(eip_pairs* pairs);
int eip_pairs_count(eip_pairs* pairs, int i_L, int j_L);
int eip_pairs_copy(eip_pairs* pairs, int i_L, int j_L, double* P_p, double* A_a, double* B_b, double* coefficient,
                   int* i_ao_start, int* j_ao_start, int* i_atom, int* j_atom, double* upper_bound);
void eip_pairs_destroy(eip_pairs* pairs);

/* FMA-throughput microbenchmark on the current device (fp64 != 0: double,
 * else float), best of 5 runs, in TFLOP/s: the denominators of the rooflines. */
int eip_measure_fma_peak(int fp64, double* tflops);

/* ---- batched (mu nu|P) over many molecules (no counterpart in the reference) --
 *
 * Usage: create -> add_pairs / add_aux per molecule and class (host arrays in
 * the reference ABI's formats; may be called repeatedly) -> build (groups the
 * primitives, uploads device-resident tables) -> alloc_output or bind_output
 * -> run (one CUDA-graph launch: every class kernel of every molecule) -> sync.
 * Output: one packed block per (molecule, class) at eip_batch_block()'s
 * offset, layout [pair shell][I][J][K][aux shell] with spherical components
 * I, J, K (Cartesian when spherical is false); pair shells are ordered by
 * (i_ao_start, j_ao_start), auxiliary shells by aux start.  Each element is
 * written once; nothing is accumulated.  Returns: 0 ok, 1 unsupported class,
 * 2 failure (eip_batch_error). */
typedef struct eip_batch eip_batch;

eip_batch* eip_batch_create(int n_molecules, bool spherical, double omega);
int eip_batch_add_pairs(eip_batch* batch, int molecule, int i_L, int j_L, const double* pair_P_p,
                        const double* pair_A_a, const double* pair_B_b, const double* pair_coefficient,
                        const int* pair_i_ao_start, const int* pair_j_ao_start, int n_pair);
int eip_batch_add_aux(eip_batch* batch, int molecule, int k_L, const double* aux_A_a,
                      const double* aux_coefficient, const int* aux_i_aux_start, int n_primitive);
/* Unit point charges at position[3 c .. 3 c + 2] (the charge_position argument
 * of nuclear_attraction): adds the ket class k_L = EIP_POINT_CHARGES, whose
 * blocks hold V[mu nu C] (not scaled by -Z), one "auxiliary shell" per charge
 * with one component, always computed in FP64.  Charges of repeated calls for
 * one molecule are numbered on in call order. */
#define EIP_POINT_CHARGES (-1)
int eip_batch_add_charges(eip_batch* batch, int molecule, const double* position, int n_charge);
/* Precision of the batch (before build): mode 0 = FP64 everywhere (default);
 * mode 1 = mixed: a shell pair of a fast class is computed with FP32 R
 * tetrahedron, ket, bra and accumulation (FP64 Boys, R^m_000, E recurrences
 * and prefactors) when Q_pair * max Q_aux * (transform gains) < fp32_threshold,
 * where Q are Schwarz-type upper bounds built like the reference front end's
 * pair bound; every other shell pair stays FP64. */
int eip_batch_set_precision(eip_batch* batch, int mode, double fp32_threshold);
/* Number of streams (1..8, default 1) the class kernels of a run are forked
 * over; set before the first run. */
int eip_batch_set_streams(eip_batch* batch, int n_streams);
int eip_batch_build(eip_batch* batch);
/* Contracted triplets of a class computed in FP64 and in FP32 (after build). */
int eip_batch_precision_split(eip_batch* batch, int i_L, int j_L, int k_L, long long* triplets_fp64,
                              long long* triplets_fp32);
long long eip_batch_output_elems(eip_batch* batch);
int eip_batch_block(eip_batch* batch, int molecule, int i_L, int j_L, int k_L, long long* offset,
                    int* n_pair_shells, int* n_aux_shells);
int eip_batch_alloc_output(eip_batch* batch);
int eip_batch_bind_output(eip_batch* batch, double* device_output);
double* eip_batch_output_device(eip_batch* batch);
/* checksum != 0: also accumulate, per molecule, the sum of its written values. */
int eip_batch_run(eip_batch* batch, int checksum);
/* Launch the kernels of one (i_L, j_L | k_L) class alone, on the batch stream,
 * outside the graph (per-kernel timing); returns 1 if the class is absent. */
int eip_batch_run_class(eip_batch* batch, int i_L, int j_L, int k_L);
/* Auxiliary-window runs: compute only the auxiliary shells whose first
 * function lies in [fn_lo[m], fn_hi[m]) for molecule m (NULL arrays: all),
 * reusing the batch's resident tables (a molecule whose whole output does not
 * fit device memory is computed window by window without rebuilding them).
 * window_plan sets the window and returns its packed output size in doubles
 * (-1 on error); point-charge classes are included only with with_charges.
 * The window's layout is the batch layout with each molecule's auxiliary
 * shells restricted to the window, blocks at eip_batch_window_block()'s
 * offsets.  run_window launches it (direct launches, not the graph) on the
 * batch stream into device_output.  Runs of one batch execute in order; the
 * window maps cycle through 4 slots, so a window_plan waits (on the host) only
 * while the run planned 4 windows earlier has not started. */
long long eip_batch_window_plan(eip_batch* batch, const int* fn_lo, const int* fn_hi, int with_charges);
int eip_batch_window_block(eip_batch* batch, int molecule, int i_L, int j_L, int k_L, long long* offset,
                           int* n_pair_shells, int* n_aux_shells);
int eip_batch_run_window(eip_batch* batch, double* device_output, int checksum);
int eip_batch_sync(eip_batch* batch);
/* 0 if every class kernel of the last run passed its self-checks, 3 if one
 * recorded an inconsistency (eip_batch_error names it). */
int eip_batch_status(eip_batch* batch);
/* Re-copy every input table from the batch's pinned host copy to the device. */
int eip_batch_upload(eip_batch* batch);
long long eip_batch_table_bytes(eip_batch* batch);
/* Device memory the built batch holds besides its output: input tables, E
 * tables, window maps and work lists (bytes; -1 before build).  A server
 * that keeps many batches alive budgets with it. */
long long eip_batch_device_bytes(eip_batch* batch);
/* How the class (i_L, j_L | k_L) runs: 0 on a fast kernel, n >= 1 on the
 * general kernel with every block split into n items over shares of its
 * primitive units, -1 if the batch has no such class (or is not built). */
int eip_batch_class_splits(eip_batch* batch, int i_L, int j_L, int k_L);
unsigned long long eip_batch_launches_per_run(eip_batch* batch);
int eip_batch_checksums(eip_batch* batch, double* host_checksums);
int eip_batch_copy_output(eip_batch* batch, long long offset, long long count, double* host);
void* eip_batch_stream(eip_batch* batch);
/* Density-fitted Coulomb contractions over the batch's packed (mu nu|P)
 * output, on the batch stream (no counterpart in the reference, whose
 * consumers read its dense tensor):
 *   gamma_P   = sum_{mu nu} (mu nu|P) D_{mu nu}
 *   J_{mu nu} = sum_P (mu nu|P) c_P
 * for every molecule at once.  df_plan (after build, with the molecules'
 * n_ao and n_aux) lists the blocks; then, after a run into the bound output,
 * df_gamma / df_coulomb take DEVICE arrays: D and J hold the molecules'
 * n_ao x n_ao row-major matrices one after the other, gamma and c their
 * n_aux vectors.  gamma and J are overwritten.  Point-charge classes are not
 * part of the contraction. */
int eip_batch_df_plan(eip_batch* batch, const int* n_ao, const int* n_aux);
int eip_batch_df_gamma(eip_batch* batch, const double* D, double* gamma);
int eip_batch_df_coulomb(eip_batch* batch, const double* c, double* J);
const char* eip_batch_error(eip_batch* batch);
void eip_batch_destroy(eip_batch* batch);

#ifdef __cplusplus
}
#endif

#endif /* EIP_B200_H */
