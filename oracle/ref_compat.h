/*
 * Force-included (g++ -include) into every PAWAN source compiled for the parity
 * oracle.  TEST INFRASTRUCTURE ONLY.
 *
 * PAWAN's __interaction::getVi (src/interaction/interaction.cpp:464-465) calls
 * KERNEL(rho, sigma, q, F, Z) with five arguments, while the Gaussian kernel it
 * includes (src/interaction/gaussian.h:47-60) only defines the six-argument
 * form (…, Z, n).  As shipped that translation unit does not compile.  The
 * declaration below supplies the five-argument overload; its definition
 * (oracle/ref_harness.cpp) forwards to the six-argument kernel and drops n,
 * which getVi never reads.  No PAWAN source file is edited.
 */
#ifndef PAWAN_ORACLE_REF_COMPAT_H_
#define PAWAN_ORACLE_REF_COMPAT_H_
void KERNEL(const double &rho, const double &sigma, double &q, double &F, double &Z);
#endif
