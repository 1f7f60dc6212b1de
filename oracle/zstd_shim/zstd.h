/* Minimal declarations of the libzstd 1.5 public API that the reference's
 * single-header SFA library calls.  The image ships the runtime
 * (libzstd.so.1) but not the development header; these prototypes match the
 * documented zstd API so the reference CPU stepper can be compiled and linked
 * against the runtime with -l:libzstd.so.1.  Test infrastructure only. */
#ifndef SCP_ORACLE_ZSTD_SHIM_H
#define SCP_ORACLE_ZSTD_SHIM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
#define ZSTD_CONTENTSIZE_UNKNOWN (0ULL - 1)
#define ZSTD_CONTENTSIZE_ERROR   (0ULL - 2)
size_t ZSTD_compress(void *dst, size_t dstCapacity, const void *src, size_t srcSize,
                     int compressionLevel);
size_t ZSTD_decompress(void *dst, size_t dstCapacity, const void *src, size_t compressedSize);
size_t ZSTD_compressBound(size_t srcSize);
unsigned ZSTD_isError(size_t code);
const char *ZSTD_getErrorName(size_t code);
unsigned long long ZSTD_getFrameContentSize(const void *src, size_t srcSize);
#ifdef __cplusplus
}
#endif
#endif
