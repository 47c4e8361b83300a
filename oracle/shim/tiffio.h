/*
 * Declarations that let the reference's include/tiff.h compile in the checker
 * build (TEST INFRASTRUCTURE ONLY).  libtiff is absent here and the checker
 * never reads or writes TIFF files: every function fails (TIFFOpen returns
 * null), so a call through this stub cannot succeed silently.
 */
#ifndef ORACLE_SHIM_TIFFIO_H
#define ORACLE_SHIM_TIFFIO_H

#include <cstdint>
#include <cstdlib>

typedef struct oracle_tiff_s TIFF;
typedef int64_t tsize_t;
typedef uint16_t tdir_t;

enum {
    TIFFTAG_IMAGEWIDTH = 256, TIFFTAG_IMAGELENGTH = 257, TIFFTAG_BITSPERSAMPLE = 258,
    TIFFTAG_COMPRESSION = 259, TIFFTAG_PHOTOMETRIC = 262, TIFFTAG_IMAGEDESCRIPTION = 270,
    TIFFTAG_ORIENTATION = 274, TIFFTAG_SAMPLESPERPIXEL = 277, TIFFTAG_ROWSPERSTRIP = 278,
    TIFFTAG_PLANARCONFIG = 284, TIFFTAG_SAMPLEFORMAT = 339
};
enum { COMPRESSION_NONE = 1, COMPRESSION_LZW = 5 };
enum { PHOTOMETRIC_MINISBLACK = 1, PHOTOMETRIC_RGB = 2 };
enum { ORIENTATION_TOPLEFT = 1 };
enum { PLANARCONFIG_CONTIG = 1 };
enum { SAMPLEFORMAT_UINT = 1, SAMPLEFORMAT_IEEEFP = 3 };

inline TIFF *TIFFOpen(const char *, const char *) { return nullptr; }
inline void TIFFClose(TIFF *) {}
inline int TIFFReadDirectory(TIFF *) { return 0; }
inline int TIFFSetDirectory(TIFF *, tdir_t) { return 0; }
inline int TIFFWriteDirectory(TIFF *) { return 0; }
inline int TIFFGetField(TIFF *, uint32_t, ...) { return 0; }
inline int TIFFSetField(TIFF *, uint32_t, ...) { return 0; }
inline tsize_t TIFFScanlineSize(TIFF *) { return -1; }
inline int TIFFReadScanline(TIFF *, void *, uint32_t, uint16_t = 0) { return -1; }
inline int TIFFWriteScanline(TIFF *, void *, uint32_t, uint16_t = 0) { return -1; }
inline void *_TIFFmalloc(tsize_t n) { return std::malloc((size_t)n); }
inline void _TIFFfree(void *p) { std::free(p); }

#endif
