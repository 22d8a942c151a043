/* Minimal stand-in for libtiff's tiffio.h (declarations only; every function
 * is defined as an aborting stub in ref_io_stubs.c). */
#ifndef SETSM_ORACLE_STUB_TIFFIO_H
#define SETSM_ORACLE_STUB_TIFFIO_H
#include <stdarg.h>
#include <stddef.h>
#include "tiff.h"
typedef struct tiff TIFF;
typedef void *tdata_t;
typedef long tsize_t;
typedef long tmsize_t;
typedef uint32 ttile_t;
typedef uint32 tstrip_t;
typedef uint64 toff_t;
typedef struct {
    uint32 field_tag; short field_readcount; short field_writecount;
    TIFFDataType field_type; unsigned short field_bit; unsigned char field_oktochange;
    unsigned char field_passcount; char *field_name;
} TIFFFieldInfo;
typedef void (*TIFFErrorHandler)(const char *, const char *, va_list);
#ifdef __cplusplus
extern "C" {
#endif
TIFF *TIFFOpen(const char *, const char *);
void TIFFClose(TIFF *);
int TIFFGetField(TIFF *, uint32, ...);
int TIFFSetField(TIFF *, uint32, ...);
tmsize_t TIFFScanlineSize(TIFF *);
tmsize_t TIFFTileSize(TIFF *);
int TIFFReadScanline(TIFF *, void *, uint32, uint16);
int TIFFWriteScanline(TIFF *, void *, uint32, uint16);
tmsize_t TIFFReadTile(TIFF *, void *, uint32, uint32, uint32, uint16);
TIFFErrorHandler TIFFSetWarningHandler(TIFFErrorHandler);
int TIFFMergeFieldInfo(TIFF *, const TIFFFieldInfo[], uint32);
void TIFFError(const char *, const char *, ...);
void *_TIFFmalloc(tmsize_t);
void _TIFFfree(void *);
#ifdef __cplusplus
}
#endif
#endif
