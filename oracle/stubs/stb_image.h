/* Stand-in for the third-party stb_image header, which the reference fetches at configure time
 * (CMakeLists.txt FetchContent, pinned commit 2c980bb59875b0d32144a71867fbdebb2f77cd20) and which
 * is absent here. Image decoding is not on the path-tracing hot path; every call reports failure,
 * so a scene that needs an image file fails loudly instead of rendering without it. Test
 * infrastructure of the oracle build only. */
#ifndef OWE_ORACLE_STB_IMAGE_STUB_H
#define OWE_ORACLE_STB_IMAGE_STUB_H
#include <stddef.h>
static inline int stbi_is_hdr(const char* path) { (void)path; return 0; }
static inline int stbi_info(const char* path, int* x, int* y, int* comp) {
    (void)path; (void)x; (void)y; (void)comp; return 0;
}
static inline float* stbi_loadf(const char* path, int* x, int* y, int* comp, int req) {
    (void)path; (void)x; (void)y; (void)comp; (void)req; return NULL;
}
static inline unsigned char* stbi_load(const char* path, int* x, int* y, int* comp, int req) {
    (void)path; (void)x; (void)y; (void)comp; (void)req; return NULL;
}
static inline const char* stbi_failure_reason(void) { return "image decoding is not part of the oracle build"; }
static inline void stbi_image_free(void* p) { (void)p; }
#endif
