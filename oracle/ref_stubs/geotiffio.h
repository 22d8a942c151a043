/* Stand-in for libgeotiff's geotiffio.h (declarations only). */
#ifndef SETSM_ORACLE_STUB_GEOTIFFIO_H
#define SETSM_ORACLE_STUB_GEOTIFFIO_H
#include "tiffio.h"
typedef struct gtiff GTIF;
typedef unsigned short geocode_t;
typedef int geokey_t;
/* GeoKey / code values named by the reference's GeoTIFF reader (never
 * executed in the oracle build; values follow the GeoTIFF specification). */
enum { GTCitationGeoKey = 1026, ProjCoordTransGeoKey = 3075,
       ProjNatOriginLatGeoKey = 3081 };
enum { CT_PolarStereographic = 15 };
typedef enum { TYPE_BYTE = 1, TYPE_SHORT = 2, TYPE_LONG = 3, TYPE_RATIONAL = 4,
               TYPE_ASCII = 5, TYPE_DOUBLE = 12 } tagtype_t;
#ifdef __cplusplus
extern "C" {
#endif
GTIF *GTIFNew(void *);
void GTIFFree(GTIF *);
int GTIFKeyGet(GTIF *, geokey_t, void *, int, int);
int GTIFKeyInfo(GTIF *, geokey_t, int *, tagtype_t *);
int GTIFKeySet(GTIF *, geokey_t, tagtype_t, int, ...);
int GTIFWriteKeys(GTIF *);
#ifdef __cplusplus
}
#endif
#endif
