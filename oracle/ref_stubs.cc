// Test infrastructure: link-time stand-ins for the Fortran BLAS/LAPACK routines
// the reference Kernel declares (Kernel/Math/SmallMatrix_impl.h). The DEM time
// step never calls them; if anything does, the process aborts loudly instead of
// computing a wrong answer.
#include <cstdio>
#include <cstdlib>

extern "C" {
void dgemm_() { std::fprintf(stderr, "oracle: dgemm_ stub called\n"); std::abort(); }
void dgemv_() { std::fprintf(stderr, "oracle: dgemv_ stub called\n"); std::abort(); }
void dgesv_() { std::fprintf(stderr, "oracle: dgesv_ stub called\n"); std::abort(); }
}
