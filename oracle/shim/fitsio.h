/* TEST INFRASTRUCTURE ONLY — the cfitsio calls of common/tomo_struct/
 * intersample.cpp (open, NAXIS keys, read image, close), so that file compiles
 * unchanged into oracle/_ref. cfitsio is not in the image: the "files" are
 * arrays registered in memory by oracle/ref_dense_shim.cpp under their base
 * names (idx.fits, abs2fi.fits, otftel.fits). */
#ifndef MOAO_ORACLE_SHIM_FITSIO_H
#define MOAO_ORACLE_SHIM_FITSIO_H

#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct moao_shim_fitsfile fitsfile;
#define READONLY 0
#define TLONG 41
#define TDOUBLE 82

int fits_open_file(fitsfile** fptr, const char* name, int mode, int* status);
int fits_read_keys_lng(fitsfile* fptr, const char* keyroot, int nstart, int nmax, long* value,
                       int* nfound, int* status);
int fits_read_img(fitsfile* fptr, int datatype, long firstelem, long nelem, void* nulval,
                  void* array, int* anynul, int* status);
int fits_close_file(fitsfile* fptr, int* status);
void fits_report_error(FILE* stream, int status);

#ifdef __cplusplus
}
#endif

#endif
