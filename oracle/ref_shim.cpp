// Single-process C ABI around the reference's own tricubic interpolation
// kernels (TEST INFRASTRUCTURE: only tests/ load the library built from this
// file and the reference's src/interp3.cpp by oracle/build_ref.py).
//
// The library is compiled from the reference's source where it lies; this
// file adds only what a single process without MPI needs:
// * definitions of the MPI functions src/interp3.cpp references (in its
//   distributed drivers, which are not called here); each returns an error;
// * the periodic ghost layer of width g that accfft_get_ghost_xyz
//   (src/ghost.cpp:555-613) builds, for one process owning the whole grid;
// * the rescale of the query points to ghost coordinates, done by the
//   reference's own rescale_xyz (src/interp3.cpp:24-60), and the call of its
//   kernel optimized_interp3_ghost_xyz_p (src/interp3.cpp:2492-2719), the one
//   Interp3_Plan::interpolate runs (src/Interp3_Plan.cpp:720-749) in both
//   precisions when the reference is built with GCC: its header undefines
//   FAST_INTERPV, the switch to the AVX kernels, for any compiler but Intel's
//   (include/interp3.hpp:37-39).
#include <mpi.h>

#include <cstring>
#include <vector>

#if defined(PETSC_USE_REAL_SINGLE)
typedef float Real;
#else
typedef double Real;
#endif

// the reference's kernels and rescale (defined in src/interp3.cpp)
void rescale_xyz(const int g_size, int* N_reg, int* N_reg_g, int* istart, int* isize, int* isize_g,
                 const int N_pts, Real* Q_);
void optimized_interp3_ghost_xyz_p(Real* reg_grid_vals, int data_dof, int* N_reg, int* N_reg_g, int* isize_g,
                                   int* istart, const int N_pts, const int g_size, Real* query_points_in,
                                   Real* query_values, bool query_values_already_scaled);

// MPI functions of the reference's distributed drivers: never reached here
int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { return 1; }
int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { return 1; }
int MPI_Wait(MPI_Request*, MPI_Status*) { return 1; }
int MPI_Type_vector(int, int, int, MPI_Datatype, MPI_Datatype*) { return 1; }
int MPI_Type_commit(MPI_Datatype*) { return 1; }
int MPI_Type_free(MPI_Datatype*) { return 1; }
int MPI_Comm_size(MPI_Comm, int* s) { if (s) *s = 1; return 0; }
int MPI_Comm_rank(MPI_Comm, int* r) { if (r) *r = 0; return 0; }
int MPI_Alltoall(const void*, int, MPI_Datatype, void*, int, MPI_Datatype, MPI_Comm) { return 1; }

extern "C" {

// Precision of this build: 8 (double) or 4 (float).
int ref_real_bytes(void) { return (int)sizeof(Real); }

// Tricubic interpolation of the periodic field f (n[0] x n[1] x n[2], x3
// fastest) at npts query points Q (3 per point, coordinates normalised to
// [0, 1) as the reference's trajectory stores them, already wrapped into
// (-h, 1) as Interp3_Plan::fast_scatter leaves them).  npts must be a
// multiple of 16: rescale_xyz writes padding entries up to the next multiple
// of 16.  Returns 0, or -1 for an invalid argument.
int ref_interp3(const Real* f, const int* n, int npts, const Real* Q, Real* out) {
  const int g = 3;  // ghost width = interpolation order (src/SemiLagrangian.cpp:553-554)
  if (!f || !n || !Q || !out || npts <= 0 || (npts % 16) != 0) return -1;
  int N[3] = {n[0], n[1], n[2]};
  int Ng[3] = {n[0] + 2 * g, n[1] + 2 * g, n[2] + 2 * g};
  int istart[3] = {0, 0, 0};
  int isize[3] = {n[0], n[1], n[2]};
  for (int k = 0; k < 3; ++k)
    if (N[k] < g) return -1;
  std::vector<Real> ghost((size_t)Ng[0] * Ng[1] * Ng[2]);
  for (int a = 0; a < Ng[0]; ++a) {
    const int i1 = (a - g + N[0]) % N[0];
    for (int b = 0; b < Ng[1]; ++b) {
      const int i2 = (b - g + N[1]) % N[1];
      const Real* row = f + ((size_t)i1 * N[1] + i2) * N[2];
      Real* o = ghost.data() + ((size_t)a * Ng[1] + b) * Ng[2];
      for (int c = 0; c < Ng[2]; ++c) o[c] = row[(c - g + N[2]) % N[2]];
    }
  }
  std::vector<Real> q(Q, Q + (size_t)3 * npts);
  rescale_xyz(g, N, Ng, istart, isize, Ng, npts, q.data());
  optimized_interp3_ghost_xyz_p(ghost.data(), 1, N, Ng, Ng, istart, npts, g, q.data(), out, true);
  return 0;
}

}  // extern "C"
