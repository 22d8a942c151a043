/*
 * ref_io_stubs.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * The reference build links libtiff / libgeotiff and its own setsmgeo.cpp for
 * file I/O.  None of those are installed here and none is on the
 * VerticalLineLocus path, so the oracle build of the reference defines each
 * unresolved I/O symbol as a stub that aborts if it is ever reached.
 */
#include <cstdio>
#include <cstdlib>
#include "tiffio.h"
#include "xtiffio.h"
#include "geotiffio.h"
#include "setsmgeo.hpp"

[[noreturn]] static void io_unreachable(const char *what) {
    fprintf(stderr, "oracle reference build: %s is not available (file I/O is stubbed)\n", what);
    abort();
}

extern "C" {
TIFF *TIFFOpen(const char *, const char *) { io_unreachable("TIFFOpen"); }
void TIFFClose(TIFF *) { io_unreachable("TIFFClose"); }
int TIFFGetField(TIFF *, uint32, ...) { io_unreachable("TIFFGetField"); }
int TIFFSetField(TIFF *, uint32, ...) { io_unreachable("TIFFSetField"); }
tmsize_t TIFFScanlineSize(TIFF *) { io_unreachable("TIFFScanlineSize"); }
tmsize_t TIFFTileSize(TIFF *) { io_unreachable("TIFFTileSize"); }
int TIFFReadScanline(TIFF *, void *, uint32, uint16) { io_unreachable("TIFFReadScanline"); }
int TIFFWriteScanline(TIFF *, void *, uint32, uint16) { io_unreachable("TIFFWriteScanline"); }
tmsize_t TIFFReadTile(TIFF *, void *, uint32, uint32, uint32, uint16) { io_unreachable("TIFFReadTile"); }
TIFFErrorHandler TIFFSetWarningHandler(TIFFErrorHandler) { return nullptr; }
int TIFFMergeFieldInfo(TIFF *, const TIFFFieldInfo[], uint32) { io_unreachable("TIFFMergeFieldInfo"); }
void TIFFError(const char *, const char *, ...) { io_unreachable("TIFFError"); }
void *_TIFFmalloc(tmsize_t) { io_unreachable("_TIFFmalloc"); }
void _TIFFfree(void *) { io_unreachable("_TIFFfree"); }
TIFF *XTIFFOpen(const char *, const char *) { io_unreachable("XTIFFOpen"); }
void XTIFFClose(TIFF *) { io_unreachable("XTIFFClose"); }
GTIF *GTIFNew(void *) { io_unreachable("GTIFNew"); }
void GTIFFree(GTIF *) { io_unreachable("GTIFFree"); }
int GTIFKeyGet(GTIF *, geokey_t, void *, int, int) { io_unreachable("GTIFKeyGet"); }
int GTIFKeyInfo(GTIF *, geokey_t, int *, tagtype_t *) { io_unreachable("GTIFKeyInfo"); }
int GTIFKeySet(GTIF *, geokey_t, tagtype_t, int, ...) { io_unreachable("GTIFKeySet"); }
int GTIFWriteKeys(GTIF *) { io_unreachable("GTIFWriteKeys"); }
}

int WriteGeotiff(char *, void *, size_t, size_t, double, double, double, int, int, int, int) { io_unreachable("WriteGeotiff"); }
int WriteGeotiff_round(char *, void *, size_t, size_t, double, double, double, int, int, int, int) { io_unreachable("WriteGeotiff_round"); }
uint8 ReadGeotiff_bits(char *) { io_unreachable("ReadGeotiff_bits"); }
CSize ReadGeotiff_info(const char *, double *, double *, double *) { io_unreachable("ReadGeotiff_info"); }
CSize ReadGeotiff_info_dxy(char *, double *, double *, double *, double *) { io_unreachable("ReadGeotiff_info_dxy"); }
