/* Test infrastructure for the oracle build of the reference (not product code).
 *
 * Force-included ahead of every reference source.  It takes the include guard
 * of the reference's param.h so that header's body is skipped, and restates
 * its constants with one change: offlvl = -1, which sends every dense level
 * to the reference's own CPU (MKL-path) branch (SnuMat_factorize.cu:221, 247,
 * 258; solver.cu:43), so the oracle build makes no cuBLAS/cuSOLVER call.
 */
#ifndef SNUSOLVER_PARAM
#define SNUSOLVER_PARAM
const double eps = 1e-15;
const int offlvl = -1;
#define MEASURE_TIME
const int LEVEL = 9;
const int NP = 1 << LEVEL;
#endif
