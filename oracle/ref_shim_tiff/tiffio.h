/*
 * TEST INFRASTRUCTURE ONLY.  Declaration stub standing in for libtiff's
 * header (absent from this image) so that LibAPR's tiled converter
 * (APRConverterBatch.hpp, gated on HAVE_LIBTIFF) compiles.  The TIFF reader
 * and writer are never called: the oracle feeds tiles from memory, and the
 * symbols are left unresolved at link time.
 */
#ifndef ORACLE_TIFFIO_STUB_H
#define ORACLE_TIFFIO_STUB_H
#include <stdint.h>
#include <sys/types.h>

typedef struct tiff TIFF;
typedef uint16_t uint16;
typedef uint32_t uint32;
typedef int64_t tmsize_t;
typedef tmsize_t tsize_t;
typedef uint32_t tstrip_t;
typedef void *tdata_t;
typedef uint64_t toff_t;
typedef uint32_t ttag_t;

#define TIFFTAG_IMAGEWIDTH 256
#define TIFFTAG_IMAGELENGTH 257
#define TIFFTAG_BITSPERSAMPLE 258
#define TIFFTAG_PHOTOMETRIC 262
#define TIFFTAG_ORIENTATION 274
#define TIFFTAG_SAMPLESPERPIXEL 277
#define TIFFTAG_ROWSPERSTRIP 278
#define TIFFTAG_PLANARCONFIG 284
#define TIFFTAG_SAMPLEFORMAT 339
#define SAMPLEFORMAT_UINT 1
#define SAMPLEFORMAT_INT 2
#define SAMPLEFORMAT_IEEEFP 3
#define PHOTOMETRIC_MINISBLACK 1
#define PLANARCONFIG_CONTIG 1
#define ORIENTATION_TOPLEFT 1

#ifdef __cplusplus
extern "C" {
#endif
TIFF *TIFFOpen(const char *, const char *);
void TIFFClose(TIFF *);
int TIFFGetField(TIFF *, uint32_t, ...);
int TIFFSetField(TIFF *, uint32_t, ...);
uint32_t TIFFNumberOfStrips(TIFF *);
tmsize_t TIFFStripSize(TIFF *);
tmsize_t TIFFScanlineSize(TIFF *);
tmsize_t TIFFReadEncodedStrip(TIFF *, uint32_t, void *, tmsize_t);
tmsize_t TIFFWriteEncodedStrip(TIFF *, uint32_t, void *, tmsize_t);
int TIFFSetDirectory(TIFF *, uint16_t);
uint16_t TIFFNumberOfDirectories(TIFF *);
int TIFFWriteDirectory(TIFF *);
uint32_t TIFFDefaultStripSize(TIFF *, uint32_t);
#ifdef __cplusplus
}
#endif
#endif
