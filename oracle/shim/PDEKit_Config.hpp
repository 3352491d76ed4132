// Build configuration consumed by the reference sources when they are compiled as the
// test oracle (oracle/_ref). Selects the plain "netlib" LAPACKE front end, which this
// directory provides as lapacke.h + lapacke_gepp.cpp (no external LAPACK is linked).
#ifndef PDEKIT_CONFIG_HPP
#define PDEKIT_CONFIG_HPP
#define PDEKIT_BLAS_LAPACK_PROVIDER_IS_NETLIB 1
#endif
