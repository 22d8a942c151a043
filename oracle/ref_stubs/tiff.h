/* Minimal stand-in for libtiff's tiff.h: only the integer typedefs the
 * SETSM headers rely on.  The reference is compiled here purely as a test
 * oracle; no TIFF file is ever opened. */
#ifndef SETSM_ORACLE_STUB_TIFF_H
#define SETSM_ORACLE_STUB_TIFF_H
#include <stdint.h>
typedef int8_t int8;
typedef uint8_t uint8;
typedef int16_t int16;
typedef uint16_t uint16;
typedef int32_t int32;
typedef uint32_t uint32;
typedef int64_t int64;
typedef uint64_t uint64;
#define TIFFTAG_IMAGEWIDTH 256
#define TIFFTAG_IMAGELENGTH 257
#define TIFFTAG_BITSPERSAMPLE 258
#define TIFFTAG_COMPRESSION 259
#define TIFFTAG_PHOTOMETRIC 262
#define TIFFTAG_SAMPLESPERPIXEL 277
#define TIFFTAG_ROWSPERSTRIP 278
#define TIFFTAG_PLANARCONFIG 284
#define TIFFTAG_PREDICTOR 317
#define TIFFTAG_TILEWIDTH 322
#define TIFFTAG_TILELENGTH 323
#define TIFFTAG_SAMPLEFORMAT 339
#define TIFFTAG_GEOPIXELSCALE 33550
#define TIFFTAG_GEOTIEPOINTS 33922
#define COMPRESSION_NONE 1
#define COMPRESSION_LZW 5
#define PHOTOMETRIC_MINISBLACK 1
#define PLANARCONFIG_CONTIG 1
#define SAMPLEFORMAT_UINT 1
#define SAMPLEFORMAT_INT 2
#define SAMPLEFORMAT_IEEEFP 3
typedef enum { TIFF_NOTYPE = 0, TIFF_BYTE = 1, TIFF_ASCII = 2, TIFF_SHORT = 3,
               TIFF_LONG = 4, TIFF_RATIONAL = 5, TIFF_DOUBLE = 12 } TIFFDataType;
#endif
