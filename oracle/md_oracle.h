/*
 * CPU oracle for the McMurchie-Davidson integral path -- TEST INFRASTRUCTURE.
 *
 * A plain-C restatement of the reference's four integral drivers, used only
 * by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, to
 * verify results against.  Never linked into the product library.
 *
 * Entry points take exactly the arguments of the reference C ABI
 * (electron_integral_playground/c_library/molecular_integral/*.cpp) and have
 * the same accumulate-into-output semantics; output offsets use 64-bit
 * arithmetic.  Return 0 on success, 1 on an unsupported class.
 *
 * Pinning: checked against the reference's PySCF golden vectors
 * (tests/golden/) and against the reference library itself built from its
 * sources (oracle/_ref/), see tests/test_oracle.py.
 */
#ifndef MD_ORACLE_H
#define MD_ORACLE_H

#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

int oracle_three_center(int i_L, int j_L, int k_L,
                        const double* pair_P_p, const double* pair_A_a, const double* pair_B_b,
                        const double* pair_coefficient, const int* pair_i_ao_start, const int* pair_j_ao_start,
                        int n_pair_ij, const double* aux_A_a, const double* aux_coefficient,
                        const int* aux_i_aux_start, int n_aux_primitive_k, double* J3c_matrix,
                        int n_ao, int n_aux, bool spherical, double omega);

int oracle_two_center(int i_L, int j_L,
                      const double* aux_A_a, const double* aux_i_coefficient, const int* aux_i_aux_start,
                      int n_aux_primitive_i, const double* aux_B_b, const double* aux_j_coefficient,
                      const int* aux_j_aux_start, int n_aux_primitive_j, double* J2c_matrix,
                      int n_aux, bool spherical, double omega);

int oracle_nuclear_attraction(int i_L, int j_L,
                              const double* pair_P_p, const double* pair_A_a, const double* pair_B_b,
                              const double* pair_coefficient, const int* pair_i_ao_start,
                              const int* pair_j_ao_start, int n_pair, const double* charge_position,
                              int n_charge, double* V_tensor, int n_ao, bool spherical, double omega);

int oracle_overlap(int i_L, int j_L, const double* pair_A_a, const double* pair_B_b,
                   const double* pair_coefficient, const int* pair_i_ao_start, const int* pair_j_ao_start,
                   int n_pair, double* S_matrix, int n_ao, bool spherical);

/* F_m(x) for m = 0..L into y[0..L] (long-double series; reference for the device Boys). */
void oracle_boys(int L, double x, double* y);
void oracle_boys_many(int L, int n, const double* x, double* y);

/* Real-solid-harmonic coefficients P_l[m][c] (row-major, (2l+1) x (l+1)(l+2)/2). */
void oracle_spherical_matrix(int l, double* out);

#ifdef __cplusplus
}
#endif

#endif
