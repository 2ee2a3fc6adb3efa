/* Minimal stand-in for CFITSIO's fitsio.h so that the P-MILOS hot-path sources
 * (which include it through defines.h only for the FLEN_CARD constant used in
 * struct FITS_IMAGE) compile without CFITSIO.  Test infrastructure only: the
 * oracle harness never reads or writes FITS through this header. */
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
#endif
