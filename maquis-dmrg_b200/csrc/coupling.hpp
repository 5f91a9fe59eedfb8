// SU(2) recoupling coefficients for the SU2U1 schedule builder.
//
// The reference evaluates Wigner 9j symbols through a vendored GSL routine
// (dmrg/framework/dmrg/block_matrix/symmetry/gsl_coupling.h:30-47) and combines
// them into four "reduced matrix element" couplings per (A, K, A') triple
// (gsl_coupling.h:72-92, cached per (J, I, I') at :145-207).  This file
// evaluates the same quantities from the textbook formulas:
//   * Wigner 6j by the Racah single-sum formula,
//   * Wigner 9j as the sum over x of (-1)^(2x) (2x+1) times three 6j symbols,
// all arguments given as twice the angular momentum (integers).
#pragma once

#include <cmath>
#include <vector>

namespace dmrgb200 {

double wigner6j(int two_j1, int two_j2, int two_j3, int two_j4, int two_j5, int two_j6);
double wigner9j(int two_j1, int two_j2, int two_j3, int two_j4, int two_j5, int two_j6,
                int two_j7, int two_j8, int two_j9);

// sqrt((g+1)(h+1)(c+1)(f+1)) * 9j(a b c; d e f; g h i)  (gsl_coupling.h:38-47)
double mod_coupling(int a, int b, int c, int d, int e, int f, int g, int h, int i);

// Four couplings for the operator-entry spin cases (row spin == 2, column
// spin == 2) as selected by casenr in op_iterate (op_iterate.hpp:56-63); the
// prefactor and case split follow gsl_coupling.h:72-92.
void set_coupling(int a, int b, int c, int d, int e, int f, int g, int h, int i, double init,
                  double couplings[4]);

// Hermitian-conjugate correction of a reduced SU2 boundary block
// (dmrg/framework/dmrg/mp_tensors/boundary.h:43-62); lspin/rspin are 2S.
double conjugate_correction_su2(int lspin, int rspin);

}  // namespace dmrgb200
