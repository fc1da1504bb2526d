/* Minimal stand-in for the CMake-generated configure.hpp of the reference
 * (src/configure.hpp.in): single rank, no MPI, no tracer, no BLAS.  Used
 * only by the oracle/_ref build of the reference's own GLLBasis and GMTK
 * sources (test infrastructure). */
#ifndef GEOFLOW_CONFIG_HPP_IN_
#define GEOFLOW_CONFIG_HPP_IN_
#define GEOFLOW_INSURE_LOOP
#define GEOFLOW_INSURE_USE
#endif
