/* Minimal stand-in for the libtiff header, written for this project: the
 * types, tags and entry points the reference's file/tiff.cpp names, implemented
 * as failing no-ops by oracle/ref_codegen/stubs.cpp (the kernel dump uses .bin
 * files only). TEST INFRASTRUCTURE ONLY. */
#ifndef MAP_STUB_TIFFIO_H
#define MAP_STUB_TIFFIO_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef struct tiff TIFF;
typedef int64_t tsize_t;
typedef uint32_t uint32;
typedef uint16_t uint16;
typedef uint8_t uint8;
typedef int16_t int16;
typedef int32_t int32;
typedef int8_t int8;
typedef enum { TIFF_NOTYPE = 0, TIFF_BYTE = 1, TIFF_DOUBLE = 12 } TIFFDataType;
typedef struct {
  uint32_t field_tag;
  short field_readcount;
  short field_writecount;
  TIFFDataType field_type;
  unsigned short field_bit;
  unsigned char field_oktochange;
  unsigned char field_passcount;
  char *field_name;
} TIFFFieldInfo;
typedef void (*TIFFExtendProc)(TIFF *);
#define FIELD_CUSTOM 65
#define SAMPLEFORMAT_UINT 1
#define SAMPLEFORMAT_INT 2
#define SAMPLEFORMAT_IEEEFP 3
#define PHOTOMETRIC_MINISBLACK 1
#define COMPRESSION_NONE 1
#define ORIENTATION_TOPLEFT 1
#define PLANARCONFIG_CONTIG 1
#define TIFFTAG_IMAGEWIDTH 256
#define TIFFTAG_IMAGELENGTH 257
#define TIFFTAG_BITSPERSAMPLE 258
#define TIFFTAG_COMPRESSION 259
#define TIFFTAG_PHOTOMETRIC 262
#define TIFFTAG_STRIPOFFSETS 273
#define TIFFTAG_ORIENTATION 274
#define TIFFTAG_SAMPLESPERPIXEL 277
#define TIFFTAG_ROWSPERSTRIP 278
#define TIFFTAG_STRIPBYTECOUNTS 279
#define TIFFTAG_PLANARCONFIG 284
#define TIFFTAG_TILEWIDTH 322
#define TIFFTAG_TILELENGTH 323
#define TIFFTAG_SAMPLEFORMAT 339
TIFF *TIFFOpen(const char *, const char *);
void TIFFClose(TIFF *);
int TIFFGetField(TIFF *, uint32_t, ...);
int TIFFSetField(TIFF *, uint32_t, ...);
int TIFFMergeFieldInfo(TIFF *, const TIFFFieldInfo *, uint32_t);
TIFFExtendProc TIFFSetTagExtender(TIFFExtendProc);
tsize_t TIFFReadTile(TIFF *, void *, uint32_t, uint32_t, uint32_t, uint16_t);
tsize_t TIFFWriteTile(TIFF *, void *, uint32_t, uint32_t, uint32_t, uint16_t);
#ifdef __cplusplus
}
#endif
#endif
