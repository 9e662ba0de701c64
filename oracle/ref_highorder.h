/*
 * Force-included (g++ -include, after ref_compat.h) into every PAWAN source of
 * the high-order oracle build, oracle/_ref/libpawanref_ho.so.  TEST
 * INFRASTRUCTURE ONLY.
 *
 * PAWAN selects its regularisation kernel at compile time with
 * `#define HIGHORDER 0` / `#define GAUSSIAN 1` inside
 * src/interaction/interaction_utils.h:13-20, which then includes either
 * highorder.h or gaussian.h.  Those are plain #defines in a header, so they
 * cannot be overridden from the command line.  Instead this header includes
 * PAWAN's highorder.h first and defines gaussian.h's include guard, so that
 * interaction_utils.h's `#include "src/interaction/gaussian.h"` expands to
 * nothing and every KERNEL / ZETASIG / QSIG / ENST call in PAWAN's unmodified
 * sources binds to the high-order functions.  No PAWAN source file is edited.
 */
#ifndef PAWAN_ORACLE_REF_HIGHORDER_H_
#define PAWAN_ORACLE_REF_HIGHORDER_H_
#include "src/interaction/highorder.h"
#define GAUSSIAN_H_
#endif
