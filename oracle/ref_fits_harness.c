/* Checker of the GPU cube ingest and the FITS readers: the reference's own FITS
 * readers (readFitsSpectroImage utilsFits.c:25-368, readFitsLambdaToArray
 * :749-833, readFitsStrayLightFile :881-1199), built unmodified against the
 * CFITSIO read shim (ref_shim/fits_shim.c).  Test infrastructure only. */
#include <stdlib.h>
#include <string.h>

#include "utilsFits.h"

/* Read a cube the way pmilos reads it for its parallel path (forParallel = 1):
 * out receives [pixel][stokes][lambda] float32, pixel = col * rows + row. */
int pmref_fits_read(const char *path, int nlambda, float *out, long long out_cap, int *rows, int *cols) {
  FitsImage *im = readFitsSpectroImage(path, 1, nlambda);
  if (!im) return -1;
  const long long n = (long long)im->numPixels * im->nLambdas * im->numStokes;
  if (n > out_cap) return -2;
  memcpy(out, im->spectroImagen, (size_t)n * sizeof(float));
  *rows = im->rows;
  *cols = im->cols;
  return 0;
}

/* readFitsStrayLightFile on a file: out receives [4][nlambda] (2-D file) or
 * [pixel][stokes][lambda] (4-D file); nx, ny are 0 for a 2-D file. */
int pmref_fits_straylight(const char *path, float *out, long long out_cap, int *nl, int *ns, int *nx, int *ny) {
  static ConfigControl cfg;
  memset(&cfg, 0, sizeof cfg);
  strncpy(cfg.StrayLightFile, path, sizeof cfg.StrayLightFile - 1);
  *nx = *ny = 0;
  float *sl = readFitsStrayLightFile(&cfg, nl, ns, nx, ny);
  if (!sl) return -1;
  const long long n = (long long)(*nl) * (*ns) * ((*nx && *ny) ? (long long)(*nx) * (*ny) : 1);
  if (n > out_cap) return -2;
  memcpy(out, sl, (size_t)n * sizeof(float));
  free(sl);
  return 0;
}

/* readFitsLambdaToArray on a 2-D wavelength file (the 4-D branch of that
 * function reads into a null pointer and is never called here). */
int pmref_fits_lambda(const char *path, double *out, int out_cap, int *index_line, int *nl) {
  double *v = readFitsLambdaToArray(path, index_line, nl);
  if (!v) return -1;
  if (*nl > out_cap) return -2;
  memcpy(out, v, (size_t)(*nl) * sizeof(double));
  free(v);
  return 0;
}
