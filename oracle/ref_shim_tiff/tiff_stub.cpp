/*
 * TEST INFRASTRUCTURE ONLY.  Definitions for the libtiff entry points named
 * by the reference's TIFF helpers, so that the reference build loads with
 * immediate binding.  They are never reached: the oracle passes tiles from
 * memory and never asks the reference to read or write a file.
 */
#include "tiffio.h"

extern "C" {
TIFF *TIFFOpen(const char *, const char *) { return nullptr; }
void TIFFClose(TIFF *) {}
int TIFFGetField(TIFF *, uint32_t, ...) { return 0; }
int TIFFSetField(TIFF *, uint32_t, ...) { return 0; }
uint32_t TIFFNumberOfStrips(TIFF *) { return 0; }
tmsize_t TIFFStripSize(TIFF *) { return 0; }
tmsize_t TIFFScanlineSize(TIFF *) { return 0; }
tmsize_t TIFFReadEncodedStrip(TIFF *, uint32_t, void *, tmsize_t) { return -1; }
tmsize_t TIFFWriteEncodedStrip(TIFF *, uint32_t, void *, tmsize_t) { return -1; }
int TIFFSetDirectory(TIFF *, uint16_t) { return 0; }
uint16_t TIFFNumberOfDirectories(TIFF *) { return 0; }
int TIFFWriteDirectory(TIFF *) { return 0; }
uint32_t TIFFDefaultStripSize(TIFF *, uint32_t r) { return r; }
}
