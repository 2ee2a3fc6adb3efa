/* Read-side stand-in for the CFITSIO calls of the reference's FITS readers
 * (utilsFits.c), so that readFitsSpectroImage runs unmodified here as the
 * checker of the GPU cube ingest.  Test infrastructure only.
 *
 * Supported: a primary image HDU; header cards in 2880-byte blocks up to END;
 * string values of keys (TSTRING); BITPIX/NAXIS/NAXISn; reading the whole image
 * as TFLOAT from big-endian float32 (BITPIX = -32) data.  Every writer and any
 * other data type sets an error status (the checker never writes FITS). */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fitsio.h"

struct pm_shim_fitsfile {
  char (*cards)[81];
  int ncards;
  long data_off;
  FILE* f;
  int bitpix, naxis;
  long naxes[8];
};

static int key_matches(const char* card, const char* key) {
  size_t n = strlen(key);
  if (n > 8 || strncmp(card, key, n) != 0) return 0;
  for (size_t i = n; i < 8; ++i)
    if (card[i] != ' ') return 0;
  return 1;
}

static const char* card_value(const char* card) { return (card[8] == '=' && card[9] == ' ') ? card + 10 : NULL; }

static long card_long(const char* card) {
  const char* v = card_value(card);
  return v ? strtol(v, NULL, 10) : 0;
}

/* the quoted string value, trailing blanks removed */
static int card_string(const char* card, char* out) {
  const char* v = card_value(card);
  if (!v) return -1;
  while (*v == ' ') ++v;
  if (*v != '\'') return -1;
  ++v;
  int n = 0;
  while (*v && n < 68) {
    if (*v == '\'') {
      if (v[1] == '\'') {
        out[n++] = '\'';
        v += 2;
        continue;
      }
      break;
    }
    out[n++] = *v++;
  }
  while (n > 0 && out[n - 1] == ' ') --n;
  out[n] = 0;
  return 0;
}

int fits_open_file(fitsfile** fptr, const char* name, int mode, int* status) {
  if (*status) return *status;
  (void)mode;
  FILE* f = fopen(name, "rb");
  if (!f) return *status = FILE_NOT_OPENED;
  fitsfile* p = calloc(1, sizeof *p);
  int cap = 0, end = 0;
  char block[2880];
  while (!end && fread(block, 1, sizeof block, f) == sizeof block) {
    for (int i = 0; i < 36 && !end; ++i) {
      const char* c = block + 80 * i;
      if (p->ncards == cap) {
        cap = cap ? 2 * cap : 64;
        p->cards = realloc(p->cards, (size_t)cap * sizeof *p->cards);
      }
      memcpy(p->cards[p->ncards], c, 80);
      p->cards[p->ncards][80] = 0;
      if (key_matches(c, "END")) end = 1;
      else ++p->ncards;
    }
  }
  if (!end) {
    fclose(f);
    free(p->cards);
    free(p);
    return *status = NO_END;
  }
  p->data_off = ftell(f);
  p->f = f;
  for (int i = 0; i < p->ncards; ++i) {
    const char* c = p->cards[i];
    if (key_matches(c, "BITPIX")) p->bitpix = (int)card_long(c);
    else if (key_matches(c, "NAXIS")) p->naxis = (int)card_long(c);
    else if (strncmp(c, "NAXIS", 5) == 0 && c[5] >= '1' && c[5] <= '8' && c[6] == ' ')
      p->naxes[c[5] - '1'] = card_long(c);
  }
  *fptr = p;
  return 0;
}

int fits_close_file(fitsfile* fptr, int* status) {
  if (fptr) {
    if (fptr->f) fclose(fptr->f);
    free(fptr->cards);
    free(fptr);
  }
  return *status;
}

int fits_get_hdu_type(fitsfile* fptr, int* hdutype, int* status) {
  (void)fptr;
  if (*status) return *status;
  *hdutype = IMAGE_HDU;
  return 0;
}

int fits_read_key(fitsfile* fptr, int datatype, const char* keyname, void* value, char* comment, int* status) {
  if (*status) return *status;
  if (comment) comment[0] = 0;
  for (int i = 0; i < fptr->ncards; ++i) {
    if (!key_matches(fptr->cards[i], keyname)) continue;
    if (datatype == TSTRING) {
      if (card_string(fptr->cards[i], (char*)value)) return *status = VALUE_UNDEFINED;
      return 0;
    }
    if (datatype == TINT) {
      *(int*)value = (int)card_long(fptr->cards[i]);
      return 0;
    }
    if (datatype == TLONG) {
      *(long*)value = card_long(fptr->cards[i]);
      return 0;
    }
    if (datatype == TDOUBLE) {
      const char* v = card_value(fptr->cards[i]);
      *(double*)value = v ? strtod(v, NULL) : 0.0;
      return 0;
    }
    return *status = BAD_DATATYPE;
  }
  return *status = KEY_NO_EXIST;
}

int fits_get_img_param(fitsfile* fptr, int maxdim, int* bitpix, int* naxis, long* naxes, int* status) {
  if (*status) return *status;
  *bitpix = fptr->bitpix;
  *naxis = fptr->naxis;
  for (int i = 0; i < maxdim && i < fptr->naxis; ++i) naxes[i] = fptr->naxes[i];
  return 0;
}

int fits_get_hdrspace(fitsfile* fptr, int* nkeys, int* morekeys, int* status) {
  if (*status) return *status;
  *nkeys = fptr->ncards;
  if (morekeys) *morekeys = 0;
  return 0;
}

int fits_read_record(fitsfile* fptr, int nrec, char* card, int* status) {
  if (*status) return *status;
  if (nrec < 1 || nrec > fptr->ncards) return *status = KEY_OUT_BOUNDS;
  memcpy(card, fptr->cards[nrec - 1], 81);
  return 0;
}

int fits_read_keyn(fitsfile* fptr, int nkey, char* keyname, char* value, char* comment, int* status) {
  if (*status) return *status;
  if (nkey < 1 || nkey > fptr->ncards) return *status = KEY_OUT_BOUNDS;
  const char* c = fptr->cards[nkey - 1];
  int n = 0;
  while (n < 8 && c[n] != ' ') {
    keyname[n] = c[n];
    ++n;
  }
  keyname[n] = 0;
  if (value) {
    const char* v = card_value(c);
    if (v) {
      strncpy(value, v, 70);
      value[70] = 0;
    } else {
      value[0] = 0;
    }
  }
  if (comment) comment[0] = 0;
  return 0;
}

static float be_float(const unsigned char* b) {
  uint32_t u = ((uint32_t)b[0] << 24) | ((uint32_t)b[1] << 16) | ((uint32_t)b[2] << 8) | (uint32_t)b[3];
  float x;
  memcpy(&x, &u, 4);
  return x;
}

static double be_double(const unsigned char* b) {
  uint64_t u = 0;
  for (int i = 0; i < 8; ++i) u = (u << 8) | (uint64_t)b[i];
  double x;
  memcpy(&x, &u, 8);
  return x;
}

int fits_read_pix(fitsfile* fptr, int datatype, long* fpixel, long nelements, void* nulval, void* array, int* anynul,
                  int* status) {
  (void)nulval;
  if (*status) return *status;
  /* float32 or float64 pixels, converted to the requested float or double as
   * CFITSIO converts them */
  if ((datatype != TFLOAT && datatype != TDOUBLE) || (fptr->bitpix != FLOAT_IMG && fptr->bitpix != DOUBLE_IMG))
    return *status = BAD_DATATYPE;
  const int width = fptr->bitpix == FLOAT_IMG ? 4 : 8;
  long first = 0, stride = 1;
  for (int i = 0; i < fptr->naxis; ++i) {
    first += (fpixel[i] - 1) * stride;
    stride *= fptr->naxes[i];
  }
  if (first + nelements > stride) return *status = BAD_PIX_NUM;
  unsigned char* raw = malloc((size_t)nelements * width);
  if (fseek(fptr->f, fptr->data_off + width * first, SEEK_SET) ||
      fread(raw, width, (size_t)nelements, fptr->f) != (size_t)nelements) {
    free(raw);
    return *status = READ_ERROR;
  }
  for (long i = 0; i < nelements; ++i) {
    const double v = width == 4 ? (double)be_float(raw + 4 * i) : be_double(raw + 8 * i);
    if (datatype == TFLOAT) ((float*)array)[i] = (float)v;
    else ((double*)array)[i] = v;
  }
  free(raw);
  if (anynul) *anynul = 0;
  return 0;
}

void fits_report_error(FILE* stream, int status) { fprintf(stream, "fits shim: status %d\n", status); }

/* writers and subset readers: never used by the checker */
#define PM_SHIM_UNSUPPORTED(name, ...) \
  int name(__VA_ARGS__, int* status) { return *status = SHIM_UNSUPPORTED; }
PM_SHIM_UNSUPPORTED(fits_create_file, fitsfile** f, const char* n)
PM_SHIM_UNSUPPORTED(fits_create_img, fitsfile* f, int b, int n, long* a)
PM_SHIM_UNSUPPORTED(fits_write_img, fitsfile* f, int t, long long fe, long long ne, void* a)
PM_SHIM_UNSUPPORTED(fits_write_subset, fitsfile* f, int t, long* fp, long* lp, void* a)
PM_SHIM_UNSUPPORTED(fits_update_key, fitsfile* f, int t, const char* k, void* v, const char* c)
PM_SHIM_UNSUPPORTED(fits_update_card, fitsfile* f, const char* k, const char* c)
PM_SHIM_UNSUPPORTED(fits_read_subset, fitsfile* f, int t, long* fp, long* lp, long* inc, void* nv, void* a, int* an)
PM_SHIM_UNSUPPORTED(fits_read_img, fitsfile* f, int t, long long fe, long long ne, void* nv, void* a, int* an)
