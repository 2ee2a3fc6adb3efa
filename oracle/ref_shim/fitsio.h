/* Minimal stand-in for CFITSIO's fitsio.h so that the P-MILOS sources compile
 * without CFITSIO: the hot-path sources include it through defines.h only for
 * the FLEN_CARD constant used in struct FITS_IMAGE; utilsFits.c's readers call
 * the read-side functions declared below (fits_shim.c).  Test infrastructure
 * only. */
#ifndef PM_SHIM_FITSIO_H
#define PM_SHIM_FITSIO_H
#define FLEN_CARD 81
#define FLEN_KEYWORD 75
#define FLEN_VALUE 71
#define FLEN_COMMENT 73
#define FLEN_ERRMSG 81
#define FLEN_STATUS 31
#define FLOAT_IMG (-32)
#define DOUBLE_IMG (-64)
#define READONLY 0
#define READWRITE 1
#define TFLOAT 42
#define TDOUBLE 82
#define TSTRING 16
typedef struct pm_shim_fitsfile fitsfile;

/* The read side used by utilsFits.c's readers, implemented in fits_shim.c. */
#include <stdio.h>
#define IMAGE_HDU 0
#define TINT 31
#define TLONG 41
#define FILE_NOT_OPENED 104
#define READ_ERROR 108
#define KEY_NO_EXIST 202
#define KEY_OUT_BOUNDS 203
#define VALUE_UNDEFINED 204
#define NO_END 210
#define BAD_PIX_NUM 321
#define BAD_DATATYPE 410
#define SHIM_UNSUPPORTED 999
int fits_open_file(fitsfile **fptr, const char *name, int mode, int *status);
int fits_close_file(fitsfile *fptr, int *status);
int fits_get_hdu_type(fitsfile *fptr, int *hdutype, int *status);
int fits_read_key(fitsfile *fptr, int datatype, const char *keyname, void *value, char *comment, int *status);
int fits_get_img_param(fitsfile *fptr, int maxdim, int *bitpix, int *naxis, long *naxes, int *status);
int fits_get_hdrspace(fitsfile *fptr, int *nkeys, int *morekeys, int *status);
int fits_read_record(fitsfile *fptr, int nrec, char *card, int *status);
int fits_read_keyn(fitsfile *fptr, int nkey, char *keyname, char *value, char *comment, int *status);
int fits_read_pix(fitsfile *fptr, int datatype, long *fpixel, long nelements, void *nulval, void *array,
                  int *anynul, int *status);
void fits_report_error(FILE *stream, int status);
/* never used by the checker: they set SHIM_UNSUPPORTED */
int fits_create_file(fitsfile **fptr, const char *name, int *status);
int fits_create_img(fitsfile *fptr, int bitpix, int naxis, long *naxes, int *status);
int fits_write_img(fitsfile *fptr, int datatype, long long firstelem, long long nelem, void *array, int *status);
int fits_write_subset(fitsfile *fptr, int datatype, long *fpixel, long *lpixel, void *array, int *status);
int fits_update_key(fitsfile *fptr, int datatype, const char *keyname, void *value, const char *comment,
                    int *status);
int fits_update_card(fitsfile *fptr, const char *keyname, const char *card, int *status);
int fits_read_subset(fitsfile *fptr, int datatype, long *fpixel, long *lpixel, long *inc, void *nulval, void *array,
                     int *anynul, int *status);
int fits_read_img(fitsfile *fptr, int datatype, long long firstelem, long long nelem, void *nulval, void *array,
                  int *anynul, int *status);
#endif
