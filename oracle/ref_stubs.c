/*
 * ref_stubs.c -- link-time stand-in for the one CUDA driver call of the
 * reference MEX source (cuMemGetInfo, cuda/source/BiotSavartMex.cu:679), so
 * the reference's host path can be loaded and run on machines without the
 * driver library. It is reached only on the reference's GPU branch, which the
 * oracle never takes; it reports "not supported".
 */
#include <stddef.h>
int cuMemGetInfo_v2(size_t *free_b, size_t *total_b) {
  if (free_b) *free_b = 0;
  if (total_b) *total_b = 0;
  return 801; /* CUDA_ERROR_NOT_SUPPORTED */
}
