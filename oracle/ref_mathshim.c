/*
 * ref_mathshim.c — test infrastructure, not product code.
 *
 * Linked into the "exact" build of the reference (oracle/_ref/trinity_ref_exact)
 * so that the reference's std::log / std::exp / std::pow calls resolve to the
 * project's own functions (trinity_b200/csrc/trn_libm.h) instead of glibc's.
 * With that, and FMA contraction off, the 1-thread reference, the C oracle and
 * the CUDA kernels all evaluate the same FP64 expressions to the same bits.
 * The timed baseline build (oracle/_ref/trinity_ref) does NOT link this file.
 */
#include "../trinity_b200/csrc/trn_libm.h"

double log(double x) { return trn_log(x); }
double exp(double x) { return trn_exp(x); }
double pow(double x, double y) { return trn_pow(x, y); }
