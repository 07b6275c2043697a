// Oracle harness (test infrastructure only): the reference's src/enfwi/
// Matrix.cpp, compiled in place, exposes clipPosition and the element-wise
// matrix helpers of the EnKF analysis through a C ABI for the tests.  The
// rest of the analysis needs MPI and LAPACK and is restated in
// oracle/enkf_oracle.py instead.
#include <cstring>
#include <mpi.h>
#include "Matrix.h"

// Single-rank stand-ins for the two MPI calls Matrix.cpp makes.
int MPI_Reduce(const void *in, void *out, int count, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  std::memcpy(out, in, (size_t)count * (t == MPI_DOUBLE ? 8 : 4));
  return 0;
}
int MPI_Gather(const void *in, int n, MPI_Datatype t, void *out, int, MPI_Datatype, int, MPI_Comm) {
  std::memcpy(out, in, (size_t)n * (t == MPI_DOUBLE ? 8 : 4));
  return 0;
}

extern "C" {

// clipPosition (Matrix.cpp:170-185) of the n singular values s.
int ref_clip_position(const double *s, int n) {
  Matrix m(1, n);
  std::memcpy(m.getData(), s, sizeof(double) * n);
  return clipPosition(m);
}

// A_plus_B / A_minus_B (Matrix.cpp:130-168) on n doubles.
void ref_a_plus_b(const double *a, const double *b, double *c, int n) {
  Matrix A(1, n), B(1, n), Cm(1, n);
  std::memcpy(A.getData(), a, sizeof(double) * n);
  std::memcpy(B.getData(), b, sizeof(double) * n);
  A_plus_B(A, B, Cm);
  std::memcpy(c, Cm.getData(), sizeof(double) * n);
}

}  // extern "C"
