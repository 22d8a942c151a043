/* Stand-in for libgeotiff's xtiffio.h (declarations only). */
#ifndef SETSM_ORACLE_STUB_XTIFFIO_H
#define SETSM_ORACLE_STUB_XTIFFIO_H
#include "tiffio.h"
#ifdef __cplusplus
extern "C" {
#endif
TIFF *XTIFFOpen(const char *, const char *);
void XTIFFClose(TIFF *);
#ifdef __cplusplus
}
#endif
#endif
