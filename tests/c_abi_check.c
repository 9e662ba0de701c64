/* A plain C99 caller of the C ABI (include/pawan_gpu.h), as a PAWAN or other
 * non-C++ host would bind it.  It only calls entry points that need no GPU:
 * the configuration defaults, the compiled shapes, the version string, the
 * host-only combination of diagnostic fields, and a pgpu_create that is
 * refused for its configuration before any device is touched. */
#include <stdio.h>
#include <string.h>

#include "pawan_gpu.h"

int main(void) {
  pgpu_config cfg;
  pgpu_ctx *ctx = NULL;
  pgpu_surrogate_config sc;
  int block[16], tpt[16];
  double fields[PGPU_DIAG_FIELDS], out[15], vbi[3], zc = -1.0;
  int k, nshapes;

  pgpu_config_default(&cfg);
  if (cfg.precision != PGPU_FP32C || cfg.kernel != PGPU_KERNEL_GAUSSIAN || cfg.use_graphs != 1) return 1;
  nshapes = pgpu_kernel_shapes(block, tpt, 16);
  if (nshapes < 4) return 2;
  for (k = 0; k < nshapes; ++k)
    if (block[k] <= 0 || tpt[k] <= 0) return 3;

  cfg.precision = 7; /* neither PGPU_FP32C nor PGPU_FP64 */
  if (pgpu_create(&ctx, &cfg) != PGPU_EINVAL || ctx != NULL) return 4;
  if (strstr(pgpu_last_error(NULL), "unknown precision 7") == NULL) return 5;

  pgpu_surrogate_config_default(&sc);
  if (sc.order != 2 || sc.tolerance != 1e-4) return 6;

  /* one wake with no particles: every diagnostic is zero */
  memset(fields, 0, sizeof(fields));
  if (pgpu_diagnose_combine(fields, 1, 0.0, out, vbi, &zc) != PGPU_OK) return 7;
  for (k = 0; k < 15; ++k)
    if (out[k] != 0.0) return 8;

  printf("%s\n", pgpu_version());
  return 0;
}
