/* Minimal declarations of the libzstd 1.5 public API that the reference's
 * single-header SFA library (sfa/format/sfa.h) calls.  The image ships the
 * zstd runtime (libzstd.so.1) but not its development header; these
 * prototypes follow the documented zstd API so the host driver, which
 * compiles sfa.h, links against the runtime with -l:libzstd.so.1. */
#ifndef SCP_HOST_ZSTD_SHIM_H
#define SCP_HOST_ZSTD_SHIM_H
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
