/* Checker of the GPU cube ingest: the reference's own FITS spectro-cube reader
 * (readFitsSpectroImage, utilsFits.c:25-368), built unmodified against the
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
