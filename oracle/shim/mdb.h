/* oracle/shim/mdb.h -- TEST INFRASTRUCTURE (checker only, never shipped).
 *
 * Project-written stand-in for the SDDS toolkit's `mdb.h`, which the reference
 * spiffe sources include (spiffe.h:6) but which is not part of the reference
 * tree.  It declares only what the reference hot-path translation units use:
 * constants, allocation, the RNG, table interpolation, the complete elliptic
 * integrals, moment helpers and a few string utilities.  Implementations live
 * in oracle/shim/shim.c.  The RNG is the project's counter-based generator, the
 * same one the CUDA path uses, so emission draws agree by construction.
 */
#ifndef SPIFFE_SHIM_MDB_H
#define SPIFFE_SHIM_MDB_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <float.h>
#include <inttypes.h>
#include <limits.h>
#include <stdint.h>

#include "../../include/spiffe_b200_constants.h"

#define PI SPIFFE_PI
#define PIx2 SPIFFE_PIx2
#define c_mks SPIFFE_C_MKS
#define e_mks SPIFFE_E_MKS
#define me_mks SPIFFE_ME_MKS
#define k_boltzmann_mks SPIFFE_KB_MKS
#define mu_o SPIFFE_MU_O
#define epsilon_o SPIFFE_EPSILON_O
/* electron rest energy in MeV (CODATA 2018); only the secondary-emission
 * setup uses it */
#define me_mev 0.51099895000

#define sqr(x) ((x) * (x))
#ifndef MIN
#define MIN(a, b) ((a) < (b) ? (a) : (b))
#endif
#ifndef MAX
#define MAX(a, b) ((a) > (b) ? (a) : (b))
#endif
#define SIGN(x) ((x) > 0 ? 1 : ((x) < 0 ? -1 : 0))
/* linear interpolation of y between (x0,y0) and (x1,y1) */
#define INTERPOLATE(y1, y0, x1, x0, x) (((y1) - (y0)) / ((x1) - (x0)) * ((x) - (x0)) + (y0))

#define EXACT_MATCH 1
#define UNIQUE_MATCH 2

void bomb(char *error, char *usage);
void *tmalloc(uint64_t size);
void *trealloc(void *ptr, uint64_t size);
void *array_1d(uint64_t size_of_elem, int64_t lower, int64_t upper);
void **zarray_2d(uint64_t size, uint64_t n1, uint64_t n2);
int free_zarray_2d(void **array, uint64_t n1, uint64_t n2);

double random_1(long iseed);
double random_2(long iseed);
double gauss_rn_lim(double mean, double sigma, double limit_in_sigmas, double (*urandom)(long iseed));
int32_t startHaltonSequence(int32_t *radix, double value);
double nextHaltonSequencePoint(long ID);

double interp(double *f, double *x, long n, double xo, long warnings, long order, long *returnCode);
double K_cei(double k);
double E_cei(double k);
double ipow(double x, long p);
long binaryArraySearch(void *array, size_t elementSize, long elements, void *key,
                       int (*compare)(const void *c1, const void *c2), long bracket);
long computeMoments(double *mean, double *rms, double *standDev, double *meanAbsoluteDev, double *x, long n);
int find_min_max(double *min, double *max, double *list, int64_t n);
void SavitzkyGolaySmooth(double *data, long rows, long order, long nLeft, long nRight, long derivativeOrder);

long match_string(char *string, char **option, long n_options, long mode);
char *str_tolower(char *s);
char *str_in(char *s, char *t);
char *replace_string(char *target, char *source, char *orig, char *newStr);
char *cp_str(char **s, char *t);
FILE *fopen_e(char *file, char *open_mode, long mode);

#endif
