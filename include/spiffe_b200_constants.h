/* spiffe_b200_constants.h
 *
 * Physical constants used by every arithmetic path of spiffe_b200 (the CUDA
 * kernels, the host runtime and the CPU checkers).  One definition keeps the
 * FP64 GPU path, the CPU restatement and the compiled reference build in exact
 * agreement: each value is a decimal literal that round-trips to one IEEE
 * double.
 *
 * Values: c and e, m_e and k_B are the exact / CODATA-2018 SI values;
 * mu_0 = 4*pi*1e-7 H/m and eps_0 = 1/(mu_0 c^2), the classical pair, each
 * rounded once to double.  The reference takes these from the SDDS `mdb.h`
 * header (used at integrate.c:94, :291-292, advance_particles.c:285, :610-619,
 * cathode.c:200, :311, poisson_correction.c:161); that header is not part of
 * the reference source tree, so these literals pin the values for every build.
 */
#ifndef SPIFFE_B200_CONSTANTS_H
#define SPIFFE_B200_CONSTANTS_H

#define SPIFFE_PI 3.141592653589793238462643
#define SPIFFE_PIx2 6.28318530717958647692528
#define SPIFFE_C_MKS 2.99792458e8
#define SPIFFE_E_MKS 1.602176634e-19
#define SPIFFE_ME_MKS 9.1093837015e-31
#define SPIFFE_KB_MKS 1.380649e-23
#define SPIFFE_MU_O 1.2566370614359173e-06
#define SPIFFE_EPSILON_O 8.85418781762039e-12
#define SPIFFE_ME_MEV 0.51099895000 /* electron rest energy in MeV (secondaryEmission.c:104-105, :198) */

#endif
