// Oracle test infrastructure: wrapper translation unit for the reference's
// Poisson/PoissonSolver.cpp, compiled unmodified.
//
// Poisson/FFTW_dirichlet.h:51 reads "static constexpr tol = 0.1;" (no type).
// g++ 13 rejects that declaration outright, even with -fpermissive, and
// PoissonSolver.cpp:14 includes the header unconditionally.  This unit
// includes the header first while the keyword constexpr expands to
// "constexpr auto", which gives tol the type double and the written value 0.1
// (the stated intent of FFTW_dirichlet.h:44-47, a 0.1 blend of the spectral
// and finite-difference denominators).  The header's #pragma once then makes
// PoissonSolver.cpp's own include a no-op.  No other token is affected: the
// header's only constexpr is that line, and every header it includes is
// already included before the macro is defined.
#include "Poisson/PoissonSolver.h"
#include <fftw3.h>
#define constexpr constexpr auto
#include "Poisson/FFTW_dirichlet.h"
#undef constexpr
#include "Poisson/PoissonSolver.cpp"
